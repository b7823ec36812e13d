"""Chronological initial guess (mre.cpp:15-117, lu of solver.cpp:4-95) on the device against
the oracle, and its effect: the guess from past solutions of nearby systems shortens CG."""
import numpy as np
import pytest

from tests.helpers import make_pair, rel, source

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su2_adj_ap", "su3_fund_ap_nocl",
                                  "su3_fund_ap_full"])
def test_mre_guess_matches_oracle(name):
    dims = (8, 8, 8, 8) if name.startswith("su3") else (4, 6, 4, 8)
    lat, O, rng = make_pair(name, dims, seed=61)
    m = lat.mre(4, "Hphi_sq", -0.3)
    O.mre_init(4, "Hphi_sq", -0.3)
    for _ in range(6):                      # more stores than the history holds
        s = source(O, rng)
        m.store(lat.field(s))
        O.mre_store(s)
    src = source(O, rng)
    d = lat.field()
    m.guess(d, lat.field(src))
    d_o = O.new_field()
    O.mre_guess(d_o, src.copy())
    lo, hi = O.default_range()
    assert rel(lat.download(d)[lo:hi], d_o[lo:hi]) < 1e-11


def test_mre_disabled_and_reset():
    lat, O, rng = make_pair("su3_fund_ap", (4, 4, 4, 4), seed=62)
    m0 = lat.mre(0, "Hphi_sq", -0.3)             # max = 0: the guess leaves dst alone
    d0 = source(O, rng)
    d = lat.field(d0)
    m0.guess(d, lat.field(source(O, rng)))
    assert np.array_equal(lat.download(d), d0)
    m = lat.mre(3, "Hphi_sq", -0.3)
    m.store(lat.field(source(O, rng)))
    m.reset()                                     # nothing stored: the guess is zero
    m.guess(d, lat.field(source(O, rng)))
    assert not np.any(lat.download(d))


def test_mre_shortens_cg():
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=63)
    mass, prec = -0.4, 1e-22
    b0, v = source(O, rng), source(O, rng)
    m = lat.mre(5, "Hphi_sq", mass)
    its_cold, its_mre = [], []
    # a source drifting linearly: from the third solve on, the solution lies in the span of
    # the stored ones and the extrapolated guess is already close to it
    for k in range(6):
        bk = b0 + 0.05 * k * v
        b = lat.field(bk)
        x = lat.field()
        its_cold.append(lat.cg_inverter("Hphi_sq", mass, prec, x, b))
        y = lat.field()
        m.guess(y, b)
        its_mre.append(lat.cg_inverter("Hphi_sq", mass, prec, y, b))
        m.store(y)
        assert rel(lat.download(y)[:O.Vh], lat.download(x)[:O.Vh]) < 1e-8
    assert sum(its_mre[2:]) < 0.5 * sum(its_cold[2:]), (its_cold, its_mre)
