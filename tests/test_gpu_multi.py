"""Several cg_inverter solves advanced together (yg_cg_inverter_multi).

Each system must reproduce the single-system CG (the reference's recurrence, cg.cpp:132-202):
the same iteration count (the batched reductions add in another order, so +-1 near the
stopping threshold) and the same solution to the accuracy the stopping rule implies, its
true residual below prec, and, for one system, the oracle's solution."""
import numpy as np
import pytest

from tests.helpers import make_pair, rel, source

pytestmark = pytest.mark.gpu


def _true_residual(lat, op, mass, x, b):
    v, xc = lat.field(), lat.field()
    lat.spinor_copy(xc, x)
    getattr(lat, op)(mass, v, xc)
    lat.spinor_sub_assign(v, b)
    return lat.spinor_sqnorm(v) / lat.spinor_sqnorm(b)


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su3_fund_sf", "su3_fund_ap_nocl", "su2_adj_ap"])
def test_multi_matches_single(name):
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=51)
    nb, mass, prec = 5, -0.4, 1e-24
    srcs = [source(O, rng) for _ in range(nb)]
    guess = 0.01 * source(O, rng)
    bs = [lat.field(s) for s in srcs]
    xs = [lat.field() for _ in range(nb)]
    lat.upload(xs[2], guess)                          # one non-zero initial guess
    its = lat.cg_inverter_multi("Hphi_sq", mass, prec, xs, bs)
    assert lat.last_status == 0
    lo, hi = 0, O.Vh
    for i in range(nb):
        x1 = lat.field()
        if i == 2:
            lat.upload(x1, guess)
        it1 = lat.cg_inverter("Hphi_sq", mass, prec, x1, bs[i])
        assert abs(its[i] - it1) <= 1, (i, its, it1)
        assert rel(lat.download(xs[i])[lo:hi], lat.download(x1)[lo:hi]) < 1e-9
        assert _true_residual(lat, "Hphi_sq", mass, xs[i], bs[i]) < 10 * prec
    # the oracle's CG on system 0
    x_o = np.zeros_like(srcs[0])
    it_o = O.cg("Hphi_sq", mass, prec, x_o, srcs[0].copy())
    assert abs(its[0] - it_o) <= 1
    assert rel(lat.download(xs[0])[lo:hi], x_o[lo:hi]) < 1e-9


def test_multi_twelve_sources_and_maxiter():
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=52)
    srcs = [source(O, rng) for _ in range(12)]
    bs = [lat.field(s) for s in srcs]
    xs = [lat.field() for _ in range(12)]
    its = lat.cg_inverter_multi("Hphi_sq", -0.4, 1e-22, xs, bs)
    for i in (0, 7, 11):
        assert _true_residual(lat, "Hphi_sq", -0.4, xs[i], bs[i]) < 1e-21
    assert min(its) > 0
    # a capped run stops every system after maxiter steps, like cg_inverter (status MAXITER)
    ys = [lat.field() for _ in range(3)]
    its = lat.cg_inverter_multi("Hphi", -0.4, 1e-30, ys, bs[:3], maxiter=6)
    assert lat.last_status == 4 and its == [6, 6, 6]
    for i in range(3):
        y1 = lat.field()
        lat.cg_inverter("Hphi", -0.4, 1e-30, y1, bs[i], maxiter=6)
        # CG on the indefinite Hphi amplifies the different summation order of the batched
        # reductions; six steps stay within 1e-9
        assert rel(lat.download(ys[i])[:O.Vh], lat.download(y1)[:O.Vh]) < 1e-9


def test_multi_argument_errors():
    from yahmc_b200 import YGError
    lat, O, rng = make_pair("su3_fund_ap", (4, 4, 4, 4), seed=53)
    b = lat.field(source(O, rng))
    with pytest.raises(YGError):
        lat.cg_inverter_multi("Hphi_sq", -0.4, 1e-20, [lat.field() for _ in range(17)], [b] * 17)
    with pytest.raises(YGError):
        lat.cg_inverter_multi("Dphi", -0.4, 1e-20, [lat.field()], [b])
    lat2, O2, rng2 = make_pair("su2_fund_ap", (4, 4, 4, 4), seed=54)
    b2 = lat2.field(source(O2, rng2))
    with pytest.raises(YGError):
        lat2.cg_inverter_multi("Hphi_sq", -0.4, 1e-20, [lat2.field()], [b2])


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su3_fund_ap_nocl", "su2_adj_ap"])
def test_mixed_multi_true_residuals(name):
    """The batched mixed CG: every system meets its true FP64 residual, without fallback,
    in about the single-system FP64 iteration count."""
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=55)
    nb, mass = 6, -0.4
    srcs = [source(O, rng) for _ in range(nb)]
    bs = [lat.field(s) for s in srcs]
    xs = [lat.field() for _ in range(nb)]
    lat.upload(xs[1], 0.01 * source(O, rng))
    x64 = lat.field()
    it64 = lat.cg_inverter("Hphi_sq", mass, 1e-24, x64, bs[0])
    for prec in (1e-24, 1e-28):
        for x in xs:
            lat.spinor_zero(x)
        sts = lat.cg_mixed_multi("Hphi_sq", mass, prec, xs, bs, delta=0.1)
        assert lat.last_status == 0
        for i in range(nb):
            assert sts[i]["fallback"] == 0, sts[i]
            assert sts[i]["true_residual"] < prec
            assert _true_residual(lat, "Hphi_sq", mass, xs[i], bs[i]) < prec
        if prec == 1e-24:
            assert sts[0]["iterations"] <= 1.5 * it64 + 10, (sts[0], it64)


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_ap_nocl", "su2_adj_ap"])
def test_mixed_multi_masses(name):
    """A mass per system (yg_cg_mixed_multi_masses), as the HMC (m + dm) and Hasenbusch (m)
    monomials' solves of one force evaluation: every system meets its true FP64 residual with
    its own mass, and matches a single-mass solve of the same system."""
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=56)
    masses = [-0.4, -0.2, -0.4, -0.3, -0.2]
    prec = 1e-24
    bs = [lat.field(source(O, rng)) for _ in masses]
    xs = [lat.field() for _ in masses]
    sts = lat.cg_mixed_multi("Hphi_sq", 0.0, prec, xs, bs, delta=0.1, masses=masses)
    assert lat.last_status == 0
    for i, m in enumerate(masses):
        assert sts[i]["fallback"] == 0, sts[i]
        assert sts[i]["true_residual"] < prec
        assert _true_residual(lat, "Hphi_sq", m, xs[i], bs[i]) < prec
    lo, hi = O.default_range()
    for i in (1, 3):
        x1 = lat.field()
        st = lat.cg_mixed_multi("Hphi_sq", masses[i], prec, [x1], [bs[i]], delta=0.1)
        assert st[0]["true_residual"] < prec
        a, c = lat.download(xs[i])[lo:hi], lat.download(x1)[lo:hi]
        assert np.abs(a - c).max() <= 1e-7 * np.abs(c).max()      # both at |r|^2 < 1e-24 |b|^2
    with pytest.raises(Exception):
        lat.cg_mixed_multi("Hphi_sq", 0.0, prec, xs, bs, masses=[-0.1, -0.2, -0.3, -0.4, -0.5])


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su3_fund_ap_nocl", "su2_adj_ap"])
def test_bicgstab_multi_matches_single(name):
    """Batched bicgstab_inverter on Dphi (yg_bicgstab_inverter_multi): each system reproduces
    the single-system BiCGstab (bicgstab.cpp:9-97) to the accuracy its stopping rule implies,
    with about its iteration count (the batched reductions add in another order), and system
    0 matches the oracle."""
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=56)
    nb, mass, prec = 5, -0.4, 1e-24
    srcs = [source(O, rng) for _ in range(nb)]
    guess = 0.01 * source(O, rng)
    bs = [lat.field(s) for s in srcs]
    xs = [lat.field() for _ in range(nb)]
    lat.upload(xs[3], guess)
    its = lat.bicgstab_inverter_multi("Dphi", mass, prec, xs, bs)
    assert lat.last_status == 0
    lo, hi = O.default_range()
    for i in range(nb):
        x1 = lat.field()
        if i == 3:
            lat.upload(x1, guess)
        it1 = lat.bicgstab_inverter("Dphi", mass, prec, x1, bs[i])
        assert abs(its[i] - it1) <= 4, (i, its, it1)
        assert rel(lat.download(xs[i])[lo:hi], lat.download(x1)[lo:hi]) < 1e-8
        assert _true_residual(lat, "Dphi", mass, xs[i], bs[i]) < 10 * prec
    x_o = np.zeros_like(srcs[0])
    it_o = O.bicgstab("Dphi", mass, prec, x_o, srcs[0].copy())
    assert abs(its[0] - it_o) <= 4
    assert rel(lat.download(xs[0])[lo:hi], x_o[lo:hi]) < 1e-8
    with pytest.raises(Exception):
        lat.bicgstab_inverter_multi("Hphi_sq", mass, prec, xs[:1], bs[:1])
