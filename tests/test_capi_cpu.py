"""CPU-side checks of the C ABI: the library loads and exports every entry point that
include/yahmc_gpu.h declares (no compute calls: there may be no GPU here)."""
import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"\b(yg_[A-Za-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "yg_Dphi" in syms and "yg_cg_inverter" in syms and "yg_wilson_fermion_force" in syms
    assert len(syms) > 60


def test_library_exports_every_declared_symbol():
    from yahmc_b200 import LIB_PATH
    if not LIB_PATH.exists():
        pytest.fail(f"{LIB_PATH} missing: run `python -m yahmc_b200.build`")
    lib = ctypes.CDLL(str(LIB_PATH))
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_binding_covers_the_abi():
    """Every C entry point has a ctypes signature in the Python mirror."""
    import yahmc_b200
    missing = [s for s in declared_symbols() if s not in yahmc_b200._SIGNATURES and s not in ("yg_last_error", "yg_launch_count")]
    assert not missing, missing


def test_lattice_creation_fails_loudly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from yahmc_b200 import Lattice, YGError
    with pytest.raises(YGError):
        Lattice((4, 4, 4, 4))


def test_noalloc_rejects_misaligned_pointers_before_any_cuda_call():
    """yg_field_sqnorm_noalloc checks its pointers on the host first: a misaligned view is
    an argument error even on a machine without a GPU (nothing is dereferenced)."""
    from yahmc_b200 import LIB_PATH
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.yg_field_sqnorm_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p]
    lib.yg_last_error.restype = ctypes.c_char_p
    assert lib.yg_field_sqnorm_noalloc(0x10008, 4, 0x20000, None) == 1
    assert b"16-byte" in lib.yg_last_error()
    assert lib.yg_field_sqnorm_noalloc(0x10000, 4, 0x20004, None) == 1
    assert b"8-byte" in lib.yg_last_error()
    assert lib.yg_field_sqnorm_noalloc(0x10000, 16_777_217, 0x20000, None) == 1
