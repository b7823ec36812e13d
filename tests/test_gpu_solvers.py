"""Parity of the CUDA linear algebra and inverters with the oracle.

Solvers run the reference's recurrences in FP64, so iteration counts agree (to +-2 for
rounding of the stopping test) and solutions agree to the accuracy the stopping criterion
implies; every solution is also checked on its TRUE residual |b - A x|^2 / |b|^2 < prec,
recomputed with the engine's operator (checks/inverters.cpp:7-191).
"""
import numpy as np
import pytest

from tests.helpers import make_pair, rel, source

pytestmark = pytest.mark.gpu


def test_linalg_views():
    from yahmc_b200 import VIEW_DEFAULT, VIEW_EVEN, VIEW_ODD, VIEW_FULL
    lat, O, rng = make_pair("su3_fund_ap", (4, 4, 4, 6), seed=10)
    a0, b0 = source(O, rng), source(O, rng)
    a, b = lat.field(a0), lat.field(b0)
    for view, (lo, hi) in [(VIEW_DEFAULT, (0, O.Vh)), (VIEW_EVEN, (0, O.Vh)), (VIEW_ODD, (O.Vh, O.V)),
                           (VIEW_FULL, (0, O.V))]:
        sl = slice(lo, hi)
        n2 = np.sum(np.abs(a0[sl]) ** 2)
        assert abs(lat.spinor_sqnorm(a, view) - n2) < 1e-12 * n2
        p = np.sum(a0[sl] * np.conj(b0[sl]))           # spinor_product = sum a conj(b), spinor.cpp:553-571
        assert abs(lat.spinor_product(a, b, view) - p) < 1e-12 * abs(p) + 1e-12
        assert abs(lat.spinor_product_re(a, b, view) - p.real) < 1e-12 * abs(p) + 1e-12
    c = 0.3 - 0.7j
    ops = [
        ("spinor_add_assign", (b,), lambda x: x + b0),
        ("spinor_sub_assign", (b,), lambda x: x - b0),
        ("spinor_mulr", (1.7, b), lambda x: 1.7 * b0),
        ("spinor_mulc", (c, b), lambda x: c * b0),
        ("spinor_mulr_assign", (-2.5,), lambda x: -2.5 * x),
        ("spinor_mulc_assign", (c,), lambda x: c * x),
        ("spinor_mulr_add_assign", (0.4, b), lambda x: x + 0.4 * b0),
        ("spinor_mulc_add_assign", (c, b), lambda x: x + c * b0),
        ("spinor_mulr_sub_assign", (0.4, b), lambda x: x - 0.4 * b0),
        ("spinor_mulc_sub_assign", (c, b), lambda x: x - c * b0),
    ]
    for fn, args, f in ops:
        for view, (lo, hi) in [(VIEW_EVEN, (0, O.Vh)), (VIEW_ODD, (O.Vh, O.V)), (VIEW_FULL, (0, O.V))]:
            x0 = source(O, rng)
            x = lat.field(x0)
            getattr(lat, fn)(x, *args, view)
            expect = x0.copy()
            expect[lo:hi] = f(x0)[lo:hi]
            assert rel(lat.download(x), expect) < 1e-15, (fn, view)
    g = lat.field(a0)
    lat.spinor_g5(g, VIEW_ODD)
    e = a0.copy()
    e[O.Vh:, :, 2:] *= -1
    assert rel(lat.download(g), e) == 0
    lat.spinor_zero(g)
    assert np.abs(lat.download(g)).max() == 0
    lat.spinor_copy(g, a)
    assert rel(lat.download(g), a0) == 0


def _true_residual(lat, op, mass, x, b, shift=0.0):
    v, xc = lat.field(), lat.field()
    lat.spinor_copy(xc, x)
    getattr(lat, op)(mass, v, xc)
    if shift:
        lat.spinor_mulr_add_assign(v, shift, x)
    lat.spinor_sub_assign(v, b)
    return lat.spinor_sqnorm(v) / lat.spinor_sqnorm(b)


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su3_fund_ap_nocl", "su3_fund_ap_full", "su2_adj_ap"])
def test_inverters(name):
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=11)
    b0 = source(O, rng)
    lo, hi = O.default_range()
    m, prec = -0.2, 1e-28                 # checks/inverters.cpp:7-8
    for fn, op in [("cg_inverter", "Hphi_sq"), ("bicgstab_inverter", "Dphi"), ("minres_inverter", "Hphi"),
                   ("auto_inverter", "Hphi_sq"), ("auto_inverter", "Hphi")]:
        x, b = lat.field(), lat.field(b0)
        it = getattr(lat, fn)(op, m, prec, x, b)
        x2 = O.new_field()
        ofn = {"cg_inverter": "cg", "bicgstab_inverter": "bicgstab", "minres_inverter": "minres",
               "auto_inverter": "auto_inverter"}[fn]
        it2 = getattr(O, ofn)(op, m, prec, x2, b0.copy())
        assert abs(it - it2) <= 2, (fn, op, it, it2)
        assert rel(lat.download(x)[lo:hi], x2[lo:hi]) < 1e-10, (fn, op)
        assert rel(lat.download(b), b0) < 1e-15            # source restored by the gamma5 sandwiches
        assert _true_residual(lat, op, m, x, b) < 1e-26, (fn, op)


def test_cg_mshift_and_rational():
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=12)
    b0 = source(O, rng)
    lo, hi = O.default_range()
    shifts = [0.50, 0.10, 0.05, 1.05]          # checks/inverters.cpp:143-146
    xs = [lat.field() for _ in shifts]
    b = lat.field(b0)
    it = lat.cg_mshift("Hphi_sq", -0.2, 1e-28, shifts, xs, b)
    it2, xs2 = O.cg_mshift("Hphi_sq", -0.2, 1e-28, shifts, b0.copy())
    assert abs(it - it2) <= 1
    for s, x, x2 in zip(shifts, xs, xs2):
        assert rel(lat.download(x)[lo:hi], x2[lo:hi]) < 1e-10
        assert _true_residual(lat, "Hphi_sq", -0.2, x, b, shift=s) < 1e-26
    # rational_calc = a0 b + sum r_i (A + p_i)^-1 b (rational.cpp:134-166)
    a0, poles, res = 0.37, [0.05, 0.4, 2.0], [0.11, 0.23, 0.9]
    x = lat.field()
    lat.rational_calc("Hphi_sq", -0.2, 1e-28, a0, poles, res, x, b)
    _, xs3 = O.cg_mshift("Hphi_sq", -0.2, 1e-28, poles, b0.copy())
    expect = a0 * b0 + sum(r * y for r, y in zip(res, xs3))
    assert rel(lat.download(x)[lo:hi], expect[lo:hi]) < 1e-10


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su2_adj_ap", "su3_fund_ap_nocl"])
def test_mixed_precision_cg(name):
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=13)
    b0 = source(O, rng)
    for prec in (1e-24, 1e-28):
        x, b = lat.field(), lat.field(b0)
        st = lat.cg_mixed("Hphi_sq", -0.4, prec, x, b)
        assert st["status"] == 0, st
        assert st["true_residual"] < prec
        assert _true_residual(lat, "Hphi_sq", -0.4, x, b) < prec
        assert st["reliable_updates"] >= 1


def test_maxiter_status():
    lat, O, rng = make_pair("su3_fund_ap", (4, 4, 4, 4), seed=14)
    x, b = lat.field(), lat.field(source(O, rng))
    it = lat.cg_inverter("Hphi_sq", -0.2, 1e-28, x, b, maxiter=3)
    assert it == 3 and lat.last_status == 4
