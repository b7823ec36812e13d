"""Mixed-precision CG with the compressed d = 3 inner operator (FP32/FP16 spinors, 18- or
12-real links, packed clover blocks).

The inner iterations only approximate Hphi_sq, so the solution is checked the way the
reference's own inverter checks are (checks/inverters.cpp:7-191): the TRUE FP64 residual
|b - A x|^2 / |b|^2 recomputed with the engine's FP64 operator must be below prec.  A wrong
inner operator (a sign on the reconstructed row, a transposed clover block) makes the
inner solver diverge from the FP64 one and the solve stall into its FP64 fallback, so the
tests also require fallback == 0 and an iteration count near the FP64 CG count.
"""
import pytest

from tests.helpers import make_pair, source

pytestmark = pytest.mark.gpu


def _true_residual(lat, op, mass, x, b):
    v, xc = lat.field(), lat.field()
    lat.spinor_copy(xc, x)
    getattr(lat, op)(mass, v, xc)
    lat.spinor_sub_assign(v, b)
    return lat.spinor_sqnorm(v) / lat.spinor_sqnorm(b)


CASES = [("su3_fund_ap", 32, 12, 0, 0), ("su3_fund_ap", 32, 18, 0, 0), ("su3_fund_ap", 16, 12, 0, 0),
         ("su3_fund_ap", 16, 18, 0, 0), ("su3_fund_open", 16, 12, 0, 0), ("su3_fund_sf", 32, 12, 0, 0),
         ("su3_fund_per", 16, 12, 0, 0), ("su3_fund_ap_nocl", 16, 12, 0, 0), ("su2_adj_ap", 32, 18, 0, 0),
         ("su2_adj_ap", 16, 18, 0, 0),
         ("su3_fund_ap", 0, 18, 0, 0), ("su2_adj_ap", 0, 18, 0, 0),          # 0: the generic FP32 inner operator
         # int16 fixed-point links / clover blocks (storage 15)
         ("su3_fund_ap", 32, 12, 15, 32), ("su3_fund_ap", 32, 12, 15, 15), ("su3_fund_open", 32, 12, 15, 15),
         ("su3_fund_sf", 32, 18, 15, 15), ("su3_fund_ap_nocl", 32, 12, 15, 15), ("su2_adj_ap", 32, 18, 15, 15),
         ("su3_fund_ap", 16, 12, 15, 15), ("su3_fund_ap", 16, 12, 32, 32),
         # 8-real FP32 links (periodic / antiperiodic lattices)
         ("su3_fund_ap", 32, 8, 0, 0), ("su3_fund_ap", 16, 8, 32, 32), ("su3_fund_per", 16, 8, 32, 32),
         ("su3_fund_ap_nocl", 32, 8, 0, 0)]


@pytest.mark.parametrize("name,inner,reals,lfmt,cfmt", CASES)
def test_compressed_inner_cg(name, inner, reals, lfmt, cfmt):
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=31)
    b0 = source(O, rng)
    mass = -0.4
    x64, b = lat.field(), lat.field(b0)
    it64 = lat.cg_inverter("Hphi_sq", mass, 1e-24, x64, b)
    for prec in (1e-24, 1e-28):
        x = lat.field()
        st = lat.cg_mixed("Hphi_sq", mass, prec, x, b, inner_precision=inner, link_reals=reals, delta=0.1,
                          link_storage=lfmt, clover_storage=cfmt)
        assert st["status"] == 0, st
        assert st["fallback"] == 0, st
        assert st["true_residual"] < prec
        assert _true_residual(lat, "Hphi_sq", mass, x, b) < prec
        if prec == 1e-24:
            assert st["iterations"] <= 1.5 * it64 + 10, (st, it64)


def test_storage_format_errors():
    from yahmc_b200 import YGError
    lat, O, rng = make_pair("su3_fund_ap", (4, 4, 4, 4), seed=37)
    b, x = lat.field(source(O, rng)), lat.field()
    for lfmt, cfmt in [(16, 32), (32, 16), (15, 16), (7, 7)]:          # combinations not built
        with pytest.raises(YGError):
            lat.cg_mixed("Hphi_sq", -0.4, 1e-20, x, b, inner_precision=32, link_reals=12, link_storage=lfmt,
                         clover_storage=cfmt)
    with pytest.raises(YGError):                                       # 8-real links are FP32 only
        lat.cg_mixed("Hphi_sq", -0.4, 1e-20, x, b, inner_precision=16, link_reals=8, link_storage=16,
                     clover_storage=16)
    lat2, O2, rng2 = make_pair("su3_fund_open", (4, 4, 4, 4), seed=38)
    with pytest.raises(YGError):                                       # not for open / SF boundaries
        lat2.cg_mixed("Hphi_sq", -0.4, 1e-20, lat2.field(), lat2.field(source(O2, rng2)), inner_precision=32,
                      link_reals=8)


@pytest.mark.parametrize("delta", [0.01, 0.3, 1e-4])
def test_compressed_inner_delta(delta):
    """delta = 1e-4 lies below what FP16 storage can resolve: the iterated residual levels
    off, the stagnation guard forces reliable updates and the solve still ends (possibly
    through the FP64 fallback) with the true residual below prec."""
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=32)
    b = lat.field(source(O, rng))
    x = lat.field()
    st = lat.cg_mixed("Hphi_sq", -0.4, 1e-26, x, b, inner_precision=16, link_reals=12, delta=delta)
    assert st["status"] == 0, st
    if delta >= 0.01:
        assert st["fallback"] == 0, st
    assert _true_residual(lat, "Hphi_sq", -0.4, x, b) < 1e-26


def test_compressed_inner_nonzero_guess():
    """x on entry is the initial guess, as for cg_inverter (cg.cpp:44-53)."""
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=33)
    b = lat.field(source(O, rng))
    x = lat.field()
    lat.cg_inverter("Hphi_sq", -0.4, 1e-10, x, b)
    st = lat.cg_mixed("Hphi_sq", -0.4, 1e-26, x, b, inner_precision=16, link_reals=12)
    assert st["status"] == 0 and st["fallback"] == 0, st
    assert _true_residual(lat, "Hphi_sq", -0.4, x, b) < 1e-26


def test_compressed_inner_gauge_change():
    """A new gauge field invalidates the compressed copy (rebuilt on the next solve)."""
    from yahmc_b200 import fields
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=34)
    b = lat.field(source(O, rng))
    x = lat.field()
    st = lat.cg_mixed("Hphi_sq", -0.4, 1e-24, x, b, inner_precision=16, link_reals=12)
    assert st["status"] == 0
    U = fields.haar_su(3, O.V * 4, rng).reshape(O.V, 4, 3, 3)
    lat.set_links(U)
    x = lat.field()
    st = lat.cg_mixed("Hphi_sq", -0.4, 1e-24, x, b, inner_precision=16, link_reals=12)
    assert st["status"] == 0 and st["fallback"] == 0, st
    assert _true_residual(lat, "Hphi_sq", -0.4, x, b) < 1e-24


def test_compressed_inner_argument_errors():
    from yahmc_b200 import YGError
    lat, O, rng = make_pair("su2_adj_ap", (4, 4, 4, 4), seed=35)
    b, x = lat.field(source(O, rng)), lat.field()
    with pytest.raises(YGError):
        lat.cg_mixed("Hphi_sq", -0.4, 1e-20, x, b, inner_precision=16, link_reals=12)   # 12 reals: SU(3) only
    with pytest.raises(YGError):
        lat.cg_mixed("Hphi_sq", -0.4, 1e-20, x, b, inner_precision=8, link_reals=18)
    lat4, O4, rng4 = make_pair("su2_fund_ap", (4, 4, 4, 4), seed=36)
    b4, x4 = lat4.field(source(O4, rng4)), lat4.field()
    with pytest.raises(YGError):
        lat4.cg_mixed("Hphi_sq", -0.4, 1e-20, x4, b4, inner_precision=32, link_reals=18)   # d = 2


def test_precision_ladder():
    """A delta far below FP16's resolution stalls the FP16 inner solve; with escalation the
    solve restarts the inner CG with FP32 storage from its best iterate (fallback bit 1)
    and still meets the true residual."""
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=38)
    b = lat.field(source(O, rng))
    x = lat.field()
    st = lat.cg_mixed("Hphi_sq", -0.4, 1e-26, x, b, inner_precision=16, link_reals=12, delta=1e-5, escalate=True)
    assert st["status"] == 0, st
    assert st["fallback"] & 2, st
    assert _true_residual(lat, "Hphi_sq", -0.4, x, b) < 1e-26
    # the library default (FP16 spinors, FP32 matrices, escalation on)
    x = lat.field()
    st = lat.cg_mixed("Hphi_sq", -0.4, 1e-26, x, b)
    assert st["status"] == 0 and st["fallback"] == 0, st
    assert _true_residual(lat, "Hphi_sq", -0.4, x, b) < 1e-26


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su2_adj_ap"])
def test_link_format_autotuner(name):
    """yg_tune_inner_links times the FP32 link formats allowed on the lattice and keeps the
    fastest; the default mixed solve then uses it and meets the true FP64 residual"""
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=39)
    reals, ms = lat.tune_inner_links(-0.4)
    allowed = {"su3_fund_ap": {18, 12, 8}, "su3_fund_open": {18, 12}, "su2_adj_ap": {18}}[name]
    assert {r for r, t in ms.items() if t > 0} == allowed
    assert reals in allowed and ms[reals] == min(t for t in ms.values() if t > 0)
    b, x = lat.field(source(O, rng)), lat.field()
    st = lat.cg_mixed("Hphi_sq", -0.4, 1e-24, x, b)
    assert st["status"] == 0 and st["true_residual"] < 1e-24
    assert _true_residual(lat, "Hphi_sq", -0.4, x, b) < 1e-24
