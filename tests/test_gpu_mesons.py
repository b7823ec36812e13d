"""Sources, propagators and meson contractions through the C ABI against the oracle.

The oracle's create_point_source / create_semwall_source and calc_propagator are pinned at
full precision to the reference's propagator.cpp, and its meson_measure to the correlators
the reference prints (observables/mesons.cpp), including the semwall noise order and the
channel mislabel of the print list."""
import numpy as np
import pytest

from oracle import yahmc_oracle as yo
from tests.helpers import make_pair, rel, source
from yahmc_b200 import fields
from yahmc_b200.spectrum import POINT, SEMWALL, Mesons

pytestmark = pytest.mark.gpu


def _dims(name):
    return (8, 8, 8, 8) if name.startswith("su3_fund") else (8, 4, 4, 4)


def _z2(rng, d, vol3):
    return np.where(rng.random(2 * d * vol3) < 0.5, 2 ** -0.5, -2 ** -0.5)


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_ap_full", "su2_adj_ap", "su2_asym_ap", "su4_adj_ap"])
def test_sources(name):
    lat, O, rng = make_pair(name, _dims(name), seed=71)
    f = lat.field()
    for n in sorted({0, O.d + 1, 4 * O.d - 1}):
        for tau in (0, 3):
            lat.create_point_source(n, tau, f)
            assert np.array_equal(lat.download(f), O.create_point_source(n, tau))
    z2 = _z2(rng, O.d, O.V // O.dims[0])
    fo = O.new_field()
    for n in range(4):
        lat.create_semwall_source(n, 5, f, z2 if n == 0 else None)
        O.create_semwall_source(n, 5, fo, z2 if n == 0 else None)
        assert np.array_equal(lat.download(f), fo), n


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su3_fund_sf", "su3_fund_ap_nocl",
                                  "su3_fund_ap_full", "su2_adj_ap"])
def test_calc_propagator(name):
    lat, O, rng = make_pair(name, _dims(name), seed=72)
    src = source(O, rng)
    x0 = 0.01 * source(O, rng)
    s_dev, x_dev = lat.field(src), lat.field(x0)
    it = lat.calc_propagator(-0.3, 1e-24, x_dev, s_dev)
    assert lat.last_status == 0 and it > 0
    xo, so = x0.copy(), src.copy()
    it_o = O.calc_propagator(-0.3, 1e-24, xo, so)
    assert abs(it - it_o) <= 2, (it, it_o)
    assert rel(lat.download(x_dev), xo) < 1e-9
    assert rel(lat.download(s_dev), so) < 1e-15          # the source's side effects


@pytest.mark.parametrize("name,method", [("su3_fund_ap", POINT), ("su3_fund_ap", SEMWALL), ("su3_fund_ap_full", POINT),
                                         ("su2_asym_ap", POINT), ("su2_adj_ap", SEMWALL), ("su3_adj_ap", POINT),
                                         ("su4_sym_ap", POINT), ("su4_adj_ap", POINT), ("su4_adj_ap", SEMWALL)])
def test_contraction(name, method):
    """all sixteen channels of contract_all_correlators on arbitrary fields"""
    lat, O, rng = make_pair(name, _dims(name), seed=73)
    n = 4 * O.d if method == POINT else 4
    props = [fields.gaussian_spinor(O.V, O.d, rng) for _ in range(n)]
    dev = [lat.field(p) for p in props]
    for tau in (0, 5):
        got = lat.meson_contract(method, tau, dev)
        want = O.meson_contract(method, tau, props)
        assert np.abs(got - want).max() < 1e-12 * np.abs(want).max(), tau
    acc = lat.meson_contract(method, 2, dev)
    lat.meson_contract(method, 2, dev, acc)                # accumulates
    assert np.abs(acc - 2 * O.meson_contract(method, 2, props)).max() < 1e-12 * np.abs(acc).max()


@pytest.mark.parametrize("name,method,hits", [("su3_fund_ap", POINT, 1), ("su3_fund_ap", SEMWALL, 2),
                                              ("su3_fund_open", SEMWALL, 1), ("su3_fund_ap_nocl", POINT, 1)])
def test_meson_measure(name, method, hits):
    """meson_measure end to end (sources, propagators, contractions, print normalisation)"""
    lat, O, rng = make_pair(name, _dims(name), seed=74)
    M = Mesons(lat, -0.3, 1e-24, hits, method, rng=np.random.default_rng(5))
    got = M.measure()
    noises = None
    if method == SEMWALL:
        r2 = np.random.default_rng(5)
        noises = []
        for _ in range(hits):
            if O.p.bc not in ("open", "sf"):
                r2.random()
            noises.append(_z2(r2, O.d, O.V // O.dims[0]))
    if O.p.bc in ("open", "sf"):
        assert M.taus == [1] * hits
    raw = O.meson_measure(-0.3, 1e-24, method, M.taus, noises)
    want = yo.meson_print_values(raw, method, hits, O.V // O.dims[0])
    for lab in want:
        assert np.abs(got[lab] - want[lab]).max() < 1e-9 * np.abs(want[lab]).max(), lab
    assert len(M.lines()) == 16 and M.lines()[12].startswith("g0g5g1: ")


@pytest.mark.parametrize("solver", ["bicgstab", "cg_mixed", "cg"])
def test_batched_propagators(solver):
    """the twelve point-source propagators of a slice through the batched solvers agree with
    the one-at-a-time BiCGstab solves, and so do the correlators"""
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=75)
    A = Mesons(lat, -0.3, 1e-24, 1, POINT)
    A.measure(taus=[3])
    B = Mesons(lat, -0.3, 1e-24, 1, POINT, batched=True, solver=solver)
    B.measure(taus=[3])
    assert lat.last_status == 0
    for n in (0, 5, 11):
        assert rel(lat.download(B.prop[n]), lat.download(A.prop[n])) < 1e-9
    for lab, v in A.values().items():
        assert np.abs(B.values()[lab] - v).max() < 1e-9 * np.abs(v).max(), lab


def test_errors():
    from yahmc_b200 import YGError
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=76)
    f = lat.field()
    with pytest.raises(YGError):
        lat.create_point_source(12, 0, f)
    with pytest.raises(YGError):
        lat.create_point_source(0, 8, f)
    with pytest.raises(YGError):
        lat._check(lat.lib.yg_create_semwall_source(lat.h, 0, 1, None, f.ptr))
    with pytest.raises(YGError):
        lat.meson_contract(POINT, 0, [f] * 4)
    with pytest.raises(YGError):
        lat.meson_contract(7, 0, [f] * 4)
    full, _, _ = make_pair("su3_fund_ap_full", (8, 8, 8, 8), seed=77)
    with pytest.raises(YGError):
        full.calc_propagator_multi(-0.3, 1e-20, [full.field()], [full.field()])
