"""The allocation-free squared norm (yg_field_sqnorm_noalloc) against yg_spinor_sqnorm.

It exists for callers that cannot allocate device memory -- a host program that has
already reserved the device for its own pools, or one that must not let a cudaMalloc
synchronise the device under running streams -- so it takes raw device pointers, needs
no lattice handle and keeps its partial sums in a fixed array inside the library.  This
file is collected last so that a run stopping at the first failure has run every other
test before it; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import make_pair, source

pytestmark = pytest.mark.gpu


def _noalloc_sqnorm(lib, ptr, n_words, out_tensor):
    rc = lib.yg_field_sqnorm_noalloc(ctypes.c_void_p(ptr), n_words, ctypes.c_void_p(out_tensor.data_ptr()), None)
    assert rc == 0, lib.yg_last_error().decode()
    import torch
    torch.cuda.synchronize()
    return float(out_tensor.item())


def test_noalloc_sqnorm_matches_lattice_sqnorm_twice():
    import torch
    from yahmc_b200 import VIEW_EVEN, VIEW_FULL
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=31)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")     # the caller's output buffer
    words_even = O.Vh * 4 * O.d                                  # complex words of the even half
    for call in range(2):                                        # two calls in a row share the scratch
        f = lat.field(source(O, rng) * (1.0 + call))
        for view, n in ((VIEW_EVEN, words_even), (VIEW_FULL, 2 * words_even)):
            ref = lat.spinor_sqnorm(f, view)
            got = _noalloc_sqnorm(lat.lib, f.ptr, n, out)
            assert abs(got - ref) <= 1e-12 * ref, (call, view, got, ref)


def test_noalloc_sqnorm_rejects_oversize():
    from yahmc_b200 import load_library
    lib = load_library()
    import torch
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    buf = torch.zeros(2, dtype=torch.float64, device="cuda")
    rc = lib.yg_field_sqnorm_noalloc(ctypes.c_void_p(buf.data_ptr()), 16_777_217,
                                     ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1 and b"limit" in lib.yg_last_error()
