"""Parity of the molecular-dynamics kernels (fundamental links, FP64) with the oracle:
weighted Wilson loops and gauge action (wilsonloop.cpp:56-133, monomials/gauge.cpp:21-40),
Wilson and Symanzik gauge forces (forces.cpp:262-309, staples.cpp:7-107), update_links
with the momentum and link boundary conditions (update.cpp:228-247, bcs.cpp:166-262),
reunitarize (update.cpp:269-279), the momentum part of hamiltonian() (update.cpp:201-220),
and gauge_field_backup/restore (gaugefield.cpp:32-42).  The momentum refresh draws from a
different generator than the reference's, so it is checked on its distribution."""
import numpy as np
import pytest

from tests.helpers import make_pair, rel
from yahmc_b200 import fields

pytestmark = pytest.mark.gpu

MD_CASES = ["su3_fund_ap", "su3_fund_per", "su3_fund_open", "su3_fund_sf", "su2_fund_ap", "su4_fund_ap"]


def _with_momenta(name, seed):
    lat, O, rng = make_pair(name, (8, 8, 8, 8), seed=seed)
    nc = O.nc
    mom = rng.normal(0.0, 2 ** -0.5, (O.V, 4, nc * nc - 1))
    lat.set_momenta(mom)
    O.mom[:] = mom
    return lat, O, rng


@pytest.mark.parametrize("name", MD_CASES)
def test_wilson_loops_and_action(name):
    lat, O, rng = _with_momenta(name, 41)
    for h, w in [(1, 1), (1, 2), (2, 1), (2, 2)]:
        assert abs(lat.avr_wilson(h, w) - O.avr_wilson(h, w)) < 1e-13
    assert abs(lat.plaquette() - O.plaquette()) < 1e-13
    for c0 in (1.0, 5.0 / 3.0):
        a = lat.gauge_action(5.6, c0)
        assert abs(a - O.gauge_action(5.6, c0)) < 1e-12 * abs(a)


@pytest.mark.parametrize("name", MD_CASES)
def test_gauge_forces(name):
    lat, O, rng = _with_momenta(name, 42)
    lat.wilson_gauge_force(0.1, 5.6)
    O.wilson_gauge_force(0.1, 5.6)
    assert rel(lat.momenta(), O.mom, 1.0) < 1e-13
    c0 = 5.0 / 3.0
    lat.improved_gauge_force(0.07, 5.6, c0, (1 - c0) / 8)
    O.improved_gauge_force(0.07, 5.6, c0, (1 - c0) / 8)
    assert rel(lat.momenta(), O.mom, 1.0) < 1e-13


@pytest.mark.parametrize("name", MD_CASES)
def test_update_links_and_momenta_action(name):
    lat, O, rng = _with_momenta(name, 43)
    h = lat.momenta_action()
    assert abs(h - O.hamiltonian_momenta()) < 1e-13 * abs(h)
    assert rel(lat.momenta(), O.mom, 1.0) < 1e-15          # boundary conditions applied in place
    lat.update_links(0.13)
    O.update_links(0.13)
    assert rel(lat.get_links(), O.fund, 1.0) < 1e-13
    lat.represent_gauge_field()
    O.represent_gauge_field()
    assert rel(lat.repr_links(), O.links, 1.0) < 1e-13
    b = fields.gaussian_spinor(O.V, O.d, rng)
    O.bcs_on_spinor(b)
    x, y = lat.field(b), lat.field()
    lat.Dphi(-0.3, y, x)
    d = np.zeros_like(b)
    O.Dphi(-0.3, d, b.copy())
    assert rel(lat.download(y)[:O.Vh], d[:O.Vh], 1.0) < 1e-12


@pytest.mark.parametrize("name", ["su3_fund_ap", "su2_fund_ap", "su4_fund_ap"])
def test_reunitarize(name):
    lat, O, rng = make_pair(name, (4, 4, 4, 8), seed=44)
    Up = O.fund + 1e-3 * (rng.normal(size=O.fund.shape) + 1j * rng.normal(size=O.fund.shape))
    lat.set_links(Up)
    O.fund = Up.copy()
    lat.reunitarize()
    O.reunitarize_links()
    U = lat.get_links()
    assert rel(U, O.fund, 1.0) < 1e-12
    eye = np.eye(O.nc)
    assert np.abs(U @ np.conj(np.swapaxes(U, -1, -2)) - eye).max() < 1e-14
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-13


def test_backup_restore():
    lat, O, rng = _with_momenta("su3_fund_ap", 45)
    U0 = lat.get_links()
    lat.gauge_backup()
    lat.update_links(0.2)
    assert np.abs(lat.get_links() - U0).max() > 1e-3
    lat.gauge_restore()
    assert np.array_equal(lat.get_links(), U0)


def test_momenta_gaussian_distribution():
    """Every algebra component ~ N(0, 1/2) (rand_gaussian, random.h:15), independent over
    links and components; the same seed reproduces the field."""
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=46)
    lat.momenta_gaussian(1234)
    m = lat.momenta()
    n = m.size                                    # 131072 samples
    assert abs(m.mean()) < 5 * np.sqrt(0.5 / n)
    assert abs(m.var() - 0.5) < 5 * 0.5 * np.sqrt(2.0 / n)
    assert abs(np.mean(m ** 4) / m.var() ** 2 - 3.0) < 0.1          # Gaussian kurtosis
    assert abs(np.corrcoef(m.reshape(-1)[:-1], m.reshape(-1)[1:])[0, 1]) < 0.02
    lat.momenta_gaussian(1234)
    assert np.array_equal(lat.momenta(), m)
    lat.momenta_gaussian(1235)
    assert not np.array_equal(lat.momenta(), m)
    # kinetic term of N(0,1/2) momenta: (TF/2) sum P^2 with TF = 2, mean = n/2
    assert abs(lat.momenta_action() - 0.5 * n) < 5 * np.sqrt(0.5 * n)


@pytest.mark.parametrize("name,c0", [("su3_fund_per", 1.0), ("su3_fund_ap", 5.0 / 3.0), ("su3_fund_open", 1.0)])
def test_leapfrog_reversibility(name, c0):
    """Pure-gauge leapfrog with the engine's force and link update: dH is small, and
    integrating back with negated momenta returns the links and H to |dH| <= 1e-8."""
    lat, O, rng = make_pair(name, (8, 8, 8, 8), seed=47)
    beta, n, dt = 5.6, 10, 0.02
    c1 = (1 - c0) / 8

    def force(h):
        if c0 == 1.0:
            lat.wilson_gauge_force(h, beta)
        else:
            lat.improved_gauge_force(h, beta, c0, c1)

    def H():
        return lat.momenta_action() + lat.gauge_action(beta, c0)

    def trajectory():
        force(dt / 2)
        for k in range(n):
            lat.update_links(dt)
            force(dt if k < n - 1 else dt / 2)

    lat.momenta_gaussian(99)
    lat.update_links(0.0)            # a start field that satisfies the link boundary conditions
    U0 = lat.get_links()
    h0 = H()
    trajectory()
    h1 = H()
    assert abs(h1 - h0) < 1e-3 * abs(h0)
    lat.set_momenta(-lat.momenta())
    trajectory()
    assert abs(H() - h0) <= 1e-8 * abs(h0)
    assert np.abs(lat.get_links() - U0).max() < 1e-11
