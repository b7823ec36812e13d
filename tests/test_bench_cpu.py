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
