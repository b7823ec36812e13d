"""Build the engine's shared library in-tree: yahmc_b200/_lib/libyahmc_b200.so.

Every CUDA translation unit under yahmc_b200/csrc is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with -lineinfo, in parallel, and
linked with the static CUDA runtime.  Object files are cached by modification time.

Usage:  python -m yahmc_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import re
import shutil
import subprocess
import sys
import time
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "_lib"
OBJ = OUT / "obj"
LIB = OUT / "libyahmc_b200.so"
ROOT = PKG.parent

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              f"-I{ROOT / 'include'}"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def sources():
    return sorted(CSRC.glob("*.cu"))


def headers():
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "yahmc_gpu.h"]


def deps(src: Path, seen=None) -> set:
    """The file and every quoted #include it reaches (resolved relative to the includer)."""
    seen = set() if seen is None else seen
    if src in seen or not src.exists():
        return seen
    seen.add(src)
    for line in src.read_text().splitlines():
        m = re.match(r'\s*#\s*include\s+"([^"]+)"', line)
        if m:
            deps((src.parent / m.group(1)).resolve(), seen)
    return seen


def _compile(args):
    src, obj, flags, verbose = args
    t0 = time.time()
    cmd = [nvcc(), *ARCH, *flags, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return f"{src.name}:\n{r.stderr[-6000:]}"
    if verbose:
        print(f"{src.name}: {time.time() - t0:.0f} s", file=sys.stderr)
        if r.stderr:
            print(r.stderr, file=sys.stderr)
    return None


def build(force: bool = False, verbose: bool = False, extra_flags=None, out: Path | None = None) -> Path:
    out_dir = Path(out) if out else OUT
    obj_dir = out_dir / "obj"
    lib = out_dir / LIB.name
    obj_dir.mkdir(parents=True, exist_ok=True)
    flags = NVCC_FLAGS + list(extra_flags or [])
    jobs = []
    # largest translation units first so that the parallel build ends sooner
    weight = {"yg_inst_d15_op": 0, "yg_inst_d10_op": 1, "yg_inst_d15_aux": 2, "yg_inst_d10_aux": 3,
              "yg_inst_d8_op": 4, "yg_inst_d8_aux": 5}
    srcs = sorted(sources(), key=lambda s: (weight.get(s.stem, 99), s.name))
    for src in srcs:
        obj = obj_dir / (src.stem + ".o")
        newest = max(p.stat().st_mtime for p in deps(src.resolve()))
        stale = force or not obj.exists() or obj.stat().st_mtime < newest
        if stale:
            jobs.append((src, obj, flags, verbose))
    if jobs:
        with cf.ThreadPoolExecutor(max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
            errs = [e for e in ex.map(_compile, jobs) if e]
        if errs:
            raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [obj_dir / (s.stem + ".o") for s in sources()]
    if jobs or not lib.exists() or lib.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        tmp = lib.with_suffix(".so.tmp")
        cmd = [nvcc(), *ARCH, "-shared", "-cudart=static", "-o", str(tmp), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr[-4000:])
        os.replace(tmp, lib)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose))


if __name__ == "__main__":
    main()
