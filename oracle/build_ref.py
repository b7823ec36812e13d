"""Build recipe for oracle/_ref: the UNMODIFIED reference, compiled from its sources.

Test infrastructure.  For each physics configuration below, every .cpp file of
the reference's library/, library/monomials/ and checks/ directories is
compiled (with observables/propagator.cpp, mesons.cpp, wilsonflow.cpp and
fermionflow.cpp), where it
lies in the reference tree, with g++ -O3 -fopenmp and the
compile-time switches of the reference's programs/Makefile:1-45 (NC, REPR_*,
CLOVER_TERM, UPDATE_EO, BC_*; no MPI), then linked with oracle/ref_harness.cpp
into ``oracle/_ref/libyahmc_ref_<name>.so``.  GSL (the reference's only
external library, used for random numbers alone) is absent here, so the
project-written headers in integration/gsl_compat stand in for it.

Only outputs land in oracle/_ref/ (git-ignored, but carried to GPU boxes with
the rest of the tree).  Nothing here is part of the product.

Usage:  python oracle/build_ref.py [--src DIR] [--jobs N] [name ...]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
DEFAULT_SRC = Path(os.environ.get("YAHMC_REFERENCE_SRC", HERE.parent.parent / "reference"))

# name -> (NC, REPR, BC, clover, even-odd)
CONFIGS = {
    "su3_fund_ap":       (3, "FUNDAMENTAL",   "ANTIPERIODIC", True,  True),
    "su3_fund_per":      (3, "FUNDAMENTAL",   "PERIODIC",     True,  True),
    "su3_fund_open":     (3, "FUNDAMENTAL",   "OPEN",         True,  True),
    "su3_fund_sf":       (3, "FUNDAMENTAL",   "SF",           True,  True),
    "su3_fund_ap_nocl":  (3, "FUNDAMENTAL",   "ANTIPERIODIC", False, True),
    "su3_fund_ap_full":  (3, "FUNDAMENTAL",   "ANTIPERIODIC", True,  False),
    "su2_fund_ap":       (2, "FUNDAMENTAL",   "ANTIPERIODIC", True,  True),
    "su2_adj_ap":        (2, "ADJOINT",       "ANTIPERIODIC", True,  True),
    "su3_sym_ap":        (3, "SYMMETRIC",     "ANTIPERIODIC", True,  True),
    "su3_asym_ap":       (3, "ANTISYMMETRIC", "ANTIPERIODIC", True,  True),
    "su3_adj_ap":        (3, "ADJOINT",       "ANTIPERIODIC", True,  True),
    "su4_fund_ap":       (4, "FUNDAMENTAL",   "ANTIPERIODIC", True,  True),
    "su4_asym_ap":       (4, "ANTISYMMETRIC", "ANTIPERIODIC", True,  True),
}


def lib_path(name: str) -> Path:
    return OUT / f"libyahmc_ref_{name}.so"


def _flags(name: str, src: Path) -> list[str]:
    nc, repr_, bc, clover, eo = CONFIGS[name]
    f = ["-O3", "-fPIC", "-fopenmp", "-std=c++11", "-w",
         f"-I{HERE.parent / 'integration' / 'gsl_compat'}", f"-I{src / 'include'}",
         f"-DNC={nc}", f"-DREPR_{repr_}", f"-DBC_{bc}"]
    if clover:
        f.append("-DCLOVER_TERM")
    if eo:
        f.append("-DUPDATE_EO")
    return f


def _sources(src: Path) -> list[Path]:
    files = sorted((src / "library").glob("*.cpp"))
    files += sorted((src / "library" / "monomials").glob("*.cpp"))
    files += sorted((src / "checks").glob("*.cpp"))
    files += [src / "observables" / n for n in ("propagator.cpp", "mesons.cpp", "wilsonflow.cpp", "fermionflow.cpp")]
    return files


def _compile(args):
    cpp, obj, flags = args
    obj.parent.mkdir(parents=True, exist_ok=True)
    if obj.exists() and obj.stat().st_mtime >= cpp.stat().st_mtime:
        return None
    r = subprocess.run(["g++", *flags, "-c", str(cpp), "-o", str(obj)],
                       capture_output=True, text=True)
    if r.returncode != 0:
        return f"{cpp}: {r.stderr[-2000:]}"
    return None


def build(names=None, src: Path = DEFAULT_SRC, jobs: int = 0, force: bool = False) -> list[Path]:
    """Compile the requested configurations; returns the library paths built or found."""
    names = list(names or CONFIGS)
    if not (src / "library" / "dirac.cpp").exists():
        raise FileNotFoundError(f"reference sources not found under {src}")
    jobs = jobs or os.cpu_count() or 4
    harness = HERE / "ref_harness.cpp"
    built = []
    for name in names:
        lib = lib_path(name)
        newest = max(p.stat().st_mtime for p in [harness, *_sources(src)])
        if lib.exists() and lib.stat().st_mtime >= newest and not force:
            built.append(lib)
            continue
        flags = _flags(name, src)
        objdir = OUT / f"obj_{name}"
        jobs_list = []
        for cpp in _sources(src):
            rel = cpp.relative_to(src)
            obj = objdir / (str(rel).replace("/", "__") + ".o")
            jobs_list.append((cpp, obj, flags))
        jobs_list.append((harness, objdir / "ref_harness.o", flags))
        with cf.ThreadPoolExecutor(jobs) as ex:
            errs = [e for e in ex.map(_compile, jobs_list) if e]
        if errs:
            raise RuntimeError("reference build failed:\n" + "\n".join(errs))
        objs = [str(o) for _, o, _ in jobs_list]
        r = subprocess.run(["g++", "-shared", "-fopenmp", "-o", str(lib), *objs, "-lm"],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link of {lib} failed:\n{r.stderr[-3000:]}")
        built.append(lib)
    return built


def build_program(name: str = "su3_fund_ap", src: Path = DEFAULT_SRC, program: str = "hmc") -> Path:
    """The reference's own programs/<program>.cpp linked with the CPU build of its sources:
    ``oracle/_ref/<program>_<name>`` (what programs/Makefile builds, with the GSL stand-in)."""
    build([name], src)
    flags = _flags(name, src)
    objdir = OUT / f"obj_{name}"
    main = src / "programs" / f"{program}.cpp"
    extra = [src / "observables" / n for n in ("polyakov.cpp", "sf_mpcac.cpp", "md_forces.cpp")]
    jobs = [(cpp, objdir / (str(cpp.relative_to(src)).replace("/", "__") + ".o"), flags) for cpp in [main, *extra]]
    errs = [e for e in map(_compile, jobs) if e]
    if errs:
        raise RuntimeError("reference build failed:\n" + "\n".join(errs))
    objs = [objdir / (str(c.relative_to(src)).replace("/", "__") + ".o") for c in _sources(src)] + [o for _, o, _ in jobs]
    exe = OUT / f"{program}_{name}"
    if not exe.exists() or exe.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        r = subprocess.run(["g++", "-o", str(exe), *map(str, objs), "-fopenmp", "-lm"], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link of {exe} failed:\n{r.stderr[-3000:]}")
    return exe


def shim_lib_path(name: str) -> Path:
    return OUT / f"libyahmc_shim_{name}.so"


def build_shim(names=("su3_fund_ap",), src: Path = DEFAULT_SRC) -> list[Path]:
    """The same harness over YaHMC built on the engine (integration/build.py: YaHMC's sources
    minus the files integration/yahmc_gpu_shim.cpp replaces, plus the shim), linked against
    libyahmc_b200.so: ``oracle/_ref/libyahmc_shim_<name>.so``.  The parity tests drive it
    exactly like the CPU build."""
    sys.path.insert(0, str(HERE.parent))
    from integration import build as ib
    built = []
    for name in names:
        objs = ib.objects(name, src, extra=(HERE / "ref_harness.cpp",))
        lib = shim_lib_path(name)
        engine = ib.ENGINE_DIR / "libyahmc_b200.so"
        newest = max(o.stat().st_mtime for o in objs + [engine])
        if not lib.exists() or lib.stat().st_mtime < newest:
            OUT.mkdir(parents=True, exist_ok=True)
            r = subprocess.run(["g++", "-shared", "-o", str(lib), *map(str, objs), *ib.link_flags()],
                               capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"link of {lib} failed:\n{r.stderr[-3000:]}")
        built.append(lib)
    return built


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("names", nargs="*")
    ap.add_argument("--src", type=Path, default=DEFAULT_SRC)
    ap.add_argument("--jobs", type=int, default=0)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--shim", action="store_true", help="build the harness over YaHMC on the engine instead")
    ap.add_argument("--program", action="store_true", help="build the reference's own hmc program (CPU)")
    a = ap.parse_args(argv)
    if a.program:
        for n in a.names or ("su3_fund_ap",):
            print(build_program(n, a.src))
        return
    if a.shim:
        for p in build_shim(a.names or ("su3_fund_ap",), a.src):
            print(p)
        return
    for p in build(a.names or None, a.src, a.jobs, a.force):
        print(p)


if __name__ == "__main__":
    sys.exit(main())
