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


def test_noalloc_sqnorm_ragged_sizes_against_host():
    """Word counts that leave a partial last block (the i < n tail) and a lattice whose
    half volume is not a multiple of the block's 2048 words, against numpy on the
    downloaded field rearranged into the device's word order."""
    import torch
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for name, dims, seed in (("su3_fund_ap", (8, 8, 8, 8), 5), ("su2_adj_ap", (4, 6, 4, 8), 6)):
        lat, O, rng = make_pair(name, dims, seed=seed)
        f = lat.field(source(O, rng))
        host = lat.download(f)                                   # (V, d, 4): colour, spin
        # device word (blk*4d + spin*d + colour)*Vh + h for site id = blk*Vh + h
        words = host.reshape(2, O.Vh, O.d, 4).transpose(0, 3, 2, 1).reshape(-1)
        for n in (words.size, words.size // 2 - 1, 2049, 1):
            got = _noalloc_sqnorm(lat.lib, f.ptr, n, out)
            ref = float((np.abs(words[:n]) ** 2).sum())
            assert abs(got - ref) <= 1e-12 * ref, (name, n, got, ref)


def test_noalloc_sqnorm_largest_size():
    """Exactly 16,777,216 complex words (256 MiB): all 8192 blocks of scratch in use."""
    import torch
    from yahmc_b200 import load_library
    lib = load_library()
    n = 16_777_216
    g = torch.Generator(device="cuda").manual_seed(11)
    buf = torch.randn(2 * n, dtype=torch.float64, device="cuda", generator=g)
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(2):
        got = _noalloc_sqnorm(lib, buf.data_ptr(), n, out)
        ref = float((buf.cpu().numpy() ** 2).sum())
        assert abs(got - ref) <= 1e-12 * ref, (got, ref)
    del buf


def test_noalloc_sqnorm_rejects_misaligned_pointers():
    """A view starting an odd number of doubles into a buffer is refused before any launch."""
    import torch
    from yahmc_b200 import load_library
    lib = load_library()
    out = torch.zeros(2, dtype=torch.float64, device="cuda")
    buf = torch.zeros(64, dtype=torch.float64, device="cuda")
    rc = lib.yg_field_sqnorm_noalloc(ctypes.c_void_p(buf.data_ptr() + 8), 4, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1 and b"16-byte" in lib.yg_last_error()
    rc = lib.yg_field_sqnorm_noalloc(ctypes.c_void_p(buf.data_ptr()), 4, ctypes.c_void_p(out.data_ptr() + 4), None)
    assert rc == 1 and b"8-byte" in lib.yg_last_error()
    one = torch.zeros(1, dtype=torch.float64, device="cuda")
    got = _noalloc_sqnorm(lib, buf.data_ptr(), 4, one)          # the aligned call still works
    assert got == 0.0


def test_noalloc_sqnorm_rejects_oversize():
    from yahmc_b200 import load_library
    lib = load_library()
    import torch
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    buf = torch.zeros(2, dtype=torch.float64, device="cuda")
    rc = lib.yg_field_sqnorm_noalloc(ctypes.c_void_p(buf.data_ptr()), 16_777_217,
                                     ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 1 and b"limit" in lib.yg_last_error()
