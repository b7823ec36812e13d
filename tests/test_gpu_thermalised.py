"""The solvers on a thermalised field instead of Haar-random links.

Haar-random links make the Wilson-clover operator well conditioned, so a solver that
converges on them proves little about the fields HMC produces.  Here the links are a
beta = 5.6 heatbath field (8^4, tiled to 16^4: a periodic field with the local action density
of the heatbath), m = -0.75 (about 1000 CG iterations, the regime of the benchmark), and
every solution is checked by the FP64 oracle: its own Hphi_sq (dirac.cpp:738-781) applied to
the GPU's x gives the true residual |b - A x|^2 / |b|^2, which must meet prec."""
import numpy as np
import pytest

from tests.helpers import CONFIGS

pytestmark = pytest.mark.gpu

DIMS, BASE = (16, 16, 16, 16), (8, 8, 8, 8)
MASS, PREC = -0.75, 1e-24


@pytest.fixture(scope="module")
def setup():
    from oracle import yahmc_oracle as yo
    from yahmc_b200 import Lattice, fields, heatbath, thermalize
    U8, hist = heatbath.thermalised_field(BASE, 5.6, 30, 11)
    U = thermalize.tile(U8, BASE, DIMS)
    nc, rep, bc, clover, eo = CONFIGS["su3_fund_ap"]
    lat = Lattice(DIMS, nc=nc, repr=rep, bc=bc, clover=clover, eo=eo, csw=1.0)
    lat.set_links(U)
    O = yo.Oracle(yo.Params(DIMS, nc, rep, bc, clover, eo, 1.0, 1.0))
    O.set_links(U)
    rng = np.random.default_rng(12)
    srcs = [fields.gaussian_spinor(O.V, O.d, rng) for _ in range(4)]
    return lat, O, srcs, float(hist[-1])


def _oracle_residual(O, x, b):
    """|b - Hphi_sq x|^2 / |b|^2 on the even sites, in numpy FP64"""
    lo, hi = O.default_range()
    xs = x.copy()
    xs[hi:] = 0.0
    ax = O.new_field()
    O.Hphi_sq(MASS, ax, xs)
    r = b[lo:hi] - ax[lo:hi]
    return float(np.sum(np.abs(r) ** 2) / np.sum(np.abs(b[lo:hi]) ** 2))


def test_field_is_thermalised(setup):
    _, _, _, plaq = setup
    assert 0.50 < plaq < 0.56           # beta = 5.6 Wilson action: plaquette about 0.53


def test_fp64_and_mixed_cg_on_thermalised_field(setup):
    lat, O, srcs, _ = setup
    b = lat.field(srcs[0])
    x64 = lat.field()
    it64 = lat.cg_inverter("Hphi_sq", MASS, PREC, x64, b)
    assert it64 > 300                    # a hard system, unlike the Haar-random test fields
    xm = lat.field()
    st = lat.cg_mixed("Hphi_sq", MASS, PREC, xm, b)
    assert st["status"] == 0 and st["fallback"] == 0, st
    assert st["iterations"] <= 1.2 * it64 + 20, (st, it64)
    bh = lat.download(b)
    res64 = _oracle_residual(O, lat.download(x64), bh)
    resm = _oracle_residual(O, lat.download(xm), bh)
    assert resm < PREC, resm
    assert res64 < 10 * PREC, res64      # the FP64 CG stops on its recursive residual
    lo, hi = O.default_range()
    a, c = lat.download(xm)[lo:hi], lat.download(x64)[lo:hi]
    assert np.abs(a - c).max() <= 1e-6 * np.abs(c).max()


def test_multi_rhs_mixed_cg_on_thermalised_field(setup):
    lat, O, srcs, _ = setup
    bs = [lat.field(s) for s in srcs]
    xs = [lat.field() for _ in srcs]
    sts = lat.cg_mixed_multi("Hphi_sq", MASS, PREC, xs, bs, delta=0.1)
    assert lat.last_status == 0
    for st, x, b in zip(sts, xs, bs):
        assert st["fallback"] == 0, st
        assert _oracle_residual(O, lat.download(x), lat.download(b)) < PREC


def test_hasenbusch_pair_on_thermalised_field(setup):
    """The HMC (m + 0.2) and Hasenbusch (m) solves of one force evaluation in one call."""
    lat, O, srcs, _ = setup
    masses = [MASS + 0.2, MASS]
    bs = [lat.field(s) for s in srcs[:2]]
    xs = [lat.field() for _ in masses]
    sts = lat.cg_mixed_multi("Hphi_sq", MASS, PREC, xs, bs, delta=0.1, masses=masses)
    assert lat.last_status == 0
    lo, hi = O.default_range()
    for st, m, x, b in zip(sts, masses, xs, bs):
        assert st["fallback"] == 0 and st["true_residual"] < PREC, st
        xh = lat.download(x)
        xh[hi:] = 0.0
        ax = O.new_field()
        O.Hphi_sq(m, ax, xh)
        bh = lat.download(b)
        r = bh[lo:hi] - ax[lo:hi]
        assert np.sum(np.abs(r) ** 2) / np.sum(np.abs(bh[lo:hi]) ** 2) < PREC
