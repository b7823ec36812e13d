"""bench.py's reference arm on the CPU: it runs the compiled reference on the field both arms
share, without mapping the engine's library."""
import pytest


def test_reference_arm_runs_without_the_engine():
    """bench.py --impl reference times the compiled reference on the shared host-made field and
    never maps the engine's library; its metric string is the one the engine arm prints."""
    import json
    import subprocess
    import sys
    from pathlib import Path

    from oracle import ref as oref
    root = Path(__file__).resolve().parents[1]
    if not oref.available("su3_fund_ap"):
        pytest.skip("oracle/_ref not built")
    out = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference", "--dims", "8", "8", "8", "8",
                          "--steps", "2", "--warmup", "1"], capture_output=True, text=True, timeout=600, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["engine_loaded"] is False
    assert line["steps"] == 2 and line["warmup"] == 1
    import bench
    assert line["metric"] == bench.METRIC
    assert line["iterations"] > 0 and line["value"] > 0


def test_hmc_program_chain_on_the_cpu_build(tmp_path):
    """The configuration chain of bench.py --hmc (pure-gauge start, saved configuration,
    fermion trajectories counted from the start file's number, hmc.cpp:148) run with YaHMC's
    CPU build of the same program on 8^4, and its log parsed as the leg parses it."""
    import subprocess
    from pathlib import Path

    import bench
    exe = Path(bench.ROOT) / "oracle" / "_ref" / "hmc_su3_fund_ap"
    if not exe.exists():
        pytest.skip("oracle/_ref/hmc_su3_fund_ap not built")
    dims = dict(T=8, X=8, Y=8, Z=8, dir=str(tmp_path))

    def run(name, text):
        (tmp_path / f"{name}.cfg").write_text(text)
        r = subprocess.run([str(exe), "-i", f"{name}.cfg", "-o", f"{name}.log"], cwd=tmp_path, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, r.stderr[-1000:]
        return bench._hmc_log(str(tmp_path / f"{name}.log"))

    therm = run("therm", bench.HMC_CFG.format(seed=5, prefix="therm", start="random", last=3, freq=3, **dims)
                + bench.GAUGE_ONLY)
    assert len(therm["seconds"]) == 3 and (tmp_path / "therm_8x8x8x8_nc3_n0003").exists()
    nf2 = run("nf2", bench.HMC_CFG.format(seed=6, prefix="nf2", start="therm_8x8x8x8_nc3_n0003", last=4, freq=4,
                                          **dims) + bench.NF2.format(mass=-0.5))
    assert len(nf2["seconds"]) == 1 and len(nf2["dH"]) == 1 and len(nf2["accepted"]) == 1
    assert nf2["mvm"][0] > 0 and len(nf2["plaquette"]) == 1
    assert (tmp_path / "nf2_8x8x8x8_nc3_n0004").exists()
