"""Build YaHMC on top of the B200 engine: the reference's own sources with the shim.

Compiles every .cpp file of YaHMC's library/, library/monomials/, checks/ and observables/
directories, where they lie in the YaHMC tree and unmodified, EXCEPT the eight files that
integration/yahmc_gpu_shim.cpp replaces (REPLACED below), plus the shim itself, with g++
-O3 -fopenmp and YaHMC's compile-time switches (programs/Makefile:1-45: NC, REPR_*,
CLOVER_TERM, UPDATE_EO, BC_*; no MPI), and links them against the engine
(yahmc_b200/_lib/libyahmc_b200.so).  The result is YaHMC's `hmc` program
(programs/hmc.cpp, unchanged) running its fermion path on the GPU:

    integration/_build/hmc_<config>    e.g.  hmc_su3_fund_ap -i hmc.cfg -o hmc.log [--run-checks]

GSL, YaHMC's only external library (random numbers alone), is absent on this machine, so
the headers in integration/gsl_compat stand in for it; a YaHMC installation links -lgsl.
Outputs go to integration/_build/ (git-ignored; carried to GPU boxes with the tree).

Usage:  python integration/build.py [--src DIR] [config ...]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "_build"
ENGINE_DIR = ROOT / "yahmc_b200" / "_lib"
DEFAULT_SRC = Path(os.environ.get("YAHMC_REFERENCE_SRC", ROOT.parent / "reference"))

# YaHMC library files whose functions the shim provides
REPLACED = ("dirac.cpp", "linalg.cpp", "cg.cpp", "bicgstab.cpp", "minres.cpp", "inverter.cpp", "forces.cpp",
            "clover.cpp")

# name -> (NC, REPR, BC, clover, even-odd): YaHMC's compile-time physics switches
CONFIGS = {
    "su3_fund_ap":      (3, "FUNDAMENTAL",   "ANTIPERIODIC", True,  True),
    "su3_fund_per":     (3, "FUNDAMENTAL",   "PERIODIC",     True,  True),
    "su3_fund_open":    (3, "FUNDAMENTAL",   "OPEN",         True,  True),
    "su3_fund_ap_nocl": (3, "FUNDAMENTAL",   "ANTIPERIODIC", False, True),
    "su2_adj_ap":       (2, "ADJOINT",       "ANTIPERIODIC", True,  True),
}


def flags(name: str, src: Path) -> list[str]:
    nc, repr_, bc, clover, eo = CONFIGS[name]
    f = ["-O3", "-fPIC", "-fopenmp", "-std=c++11", "-w", f"-I{HERE / 'gsl_compat'}", f"-I{src / 'include'}",
         f"-I{ROOT / 'include'}", f"-DNC={nc}", f"-DREPR_{repr_}", f"-DBC_{bc}"]
    if clover:
        f.append("-DCLOVER_TERM")
    if eo:
        f.append("-DUPDATE_EO")
    return f


def sources(src: Path) -> list[Path]:
    """YaHMC's sources minus the replaced files (the Makefile's SOURCES, programs/Makefile:40)."""
    files = [p for p in sorted((src / "library").glob("*.cpp")) if p.name not in REPLACED]
    files += sorted((src / "library" / "monomials").glob("*.cpp"))
    files += sorted((src / "checks").glob("*.cpp"))
    files += sorted((src / "observables").glob("*.cpp"))
    return files


def _compile(args):
    cpp, obj, fl = args
    obj.parent.mkdir(parents=True, exist_ok=True)
    if obj.exists() and obj.stat().st_mtime >= cpp.stat().st_mtime:
        return None
    r = subprocess.run(["g++", *fl, "-c", str(cpp), "-o", str(obj)], capture_output=True, text=True)
    return f"{cpp}: {r.stderr[-2000:]}" if r.returncode else None


def objects(name: str, src: Path = DEFAULT_SRC, extra: tuple = (), jobs: int = 0) -> list[Path]:
    """Object files of YaHMC's kept sources, the shim, and any `extra` sources (compiled with
    the same switches) for one configuration."""
    if not (src / "library" / "update.cpp").exists():
        raise FileNotFoundError(f"YaHMC sources not found under {src}")
    fl = flags(name, src)
    objdir = OUT / f"obj_{name}"
    todo = []
    for cpp in sources(src):
        todo.append((cpp, objdir / (str(cpp.relative_to(src)).replace("/", "__") + ".o"), fl))
    for cpp in (HERE / "yahmc_gpu_shim.cpp", *map(Path, extra)):
        todo.append((cpp, objdir / f"{cpp.parent.name}__{cpp.name}.o", fl))
    # the shim's object also depends on the engine header
    shim_obj = objdir / "integration__yahmc_gpu_shim.cpp.o"
    hdr = ROOT / "include" / "yahmc_gpu.h"
    if shim_obj.exists() and shim_obj.stat().st_mtime < hdr.stat().st_mtime:
        shim_obj.unlink()
    with cf.ThreadPoolExecutor(jobs or os.cpu_count() or 4) as ex:
        errs = [e for e in ex.map(_compile, todo) if e]
    if errs:
        raise RuntimeError("build failed:\n" + "\n".join(errs))
    return [o for _, o, _ in todo]


def link_flags() -> list[str]:
    engine = ENGINE_DIR / "libyahmc_b200.so"
    if not engine.exists():
        raise FileNotFoundError(f"{engine} missing: run `python -m yahmc_b200.build` first")
    return [f"-L{ENGINE_DIR}", "-lyahmc_b200", f"-Wl,-rpath,{ENGINE_DIR}", "-fopenmp", "-lm"]


def build_program(name: str, src: Path = DEFAULT_SRC, program: str = "hmc") -> Path:
    """YaHMC's programs/<program>.cpp, unchanged, linked with the shim and the engine."""
    main = src / "programs" / f"{program}.cpp"
    objs = objects(name, src, extra=(main,))
    exe = OUT / f"{program}_{name}"
    newest = max(o.stat().st_mtime for o in objs + [ENGINE_DIR / "libyahmc_b200.so"])
    if not exe.exists() or exe.stat().st_mtime < newest:
        r = subprocess.run(["g++", "-o", str(exe), *map(str, objs), *link_flags()], capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"link of {exe} failed:\n{r.stderr[-3000:]}")
    return exe


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("names", nargs="*")
    ap.add_argument("--src", type=Path, default=DEFAULT_SRC)
    a = ap.parse_args(argv)
    for name in a.names or ["su3_fund_ap"]:
        print(build_program(name, a.src))


if __name__ == "__main__":
    sys.exit(main())
