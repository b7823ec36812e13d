"""Wilson and fermion flow through the C ABI (yg_wf_*) against the oracle.

The oracle's restatement of observables/wilsonflow.cpp and observables/fermionflow.cpp is
pinned to the reference's own functions to rounding (test_oracle_pinning.py); here the
engine's flowed links, energy densities, topological charge and flowed fields are checked
against it on every boundary condition, several groups and representations, and the full
(unpreconditioned) lattice."""
import numpy as np
import pytest

from oracle import yahmc_oracle as yo
from tests.helpers import make_pair, rel
from yahmc_b200 import fields

pytestmark = pytest.mark.gpu

NAMES = ["su3_fund_ap", "su3_fund_per", "su3_fund_open", "su3_fund_sf", "su2_adj_ap", "su2_fund_ap", "su4_fund_ap",
         "su4_adj_ap", "su3_fund_ap_full"]


def _smooth_pair(name, seed):
    dims = (8, 8, 8, 8) if name.startswith("su3") else (8, 4, 4, 6)
    lat, O, rng = make_pair(name, dims, seed=seed)
    nc = O.nc
    U = yo.exp_algebra(nc, rng.normal(0, 0.5, (O.V, 4, nc * nc - 1)), 1.0)
    O.fund = U
    O.bcs_on_gauge()
    lat.set_links(O.fund)
    O.set_links(O.fund.copy())
    return lat, O, rng


def _obs_close(got, O):
    want = np.array([O.wf_e_plaq(), O.wf_e_sym(), O.wf_charge()])
    assert np.all(np.abs(np.array(got) - want) < 1e-12 * np.maximum(np.abs(want), 1.0)), (got, want)


@pytest.mark.parametrize("name", NAMES)
def test_wilson_flow(name):
    lat, O, rng = _smooth_pair(name, 81)
    _obs_close(lat.wf_observables(), O)
    lat.wf_init()
    O.wf_init()
    for _ in range(3):
        lat.wf_iterate(0.02)
        O.wf_iterate(0.02)
    assert rel(lat.get_links(), O.fund) < 1e-13
    _obs_close(lat.wf_observables(), O)
    # the two halves of a stage on their own
    lat.wf_zeta(0.01)
    O.wf_zeta(0.01)
    lat.wf_update(0.5)
    O.wf_update(0.5)
    assert rel(lat.get_links(), O.fund) < 1e-13


def test_flow_smooths_and_keeps_charge_small():
    """the flow lowers the action density of a rough field monotonically"""
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=82)
    lat.wf_init()
    e = [lat.wf_observables()[0]]
    for _ in range(10):
        lat.wf_iterate(0.01)
        e.append(lat.wf_observables()[0])
    assert all(b < a for a, b in zip(e, e[1:])), e


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su3_fund_sf", "su2_adj_ap", "su3_fund_ap_full",
                                  "su4_adj_ap"])
def test_fermion_flow(name):
    lat, O, rng = _smooth_pair(name, 83)
    phis = [fields.gaussian_spinor(O.V, O.d, rng) for _ in range(3)]
    dev = [lat.field(p) for p in phis]
    lat.wf_fermion_init(3)
    O.wf_fermion_init(phis)
    for _ in range(2):
        lat.wf_fermion_iterate(0.02, dev)
        O.wf_fermion_iterate(0.02)
    for f, p in zip(dev, phis):
        assert rel(lat.download(f), p) < 1e-13
    assert rel(lat.get_links(), O.fund) < 1e-13
    # the represented field of the flowed links gives the oracle's Dirac operator
    lat.represent_gauge_field()
    O.represent_gauge_field()
    src = fields.gaussian_spinor(O.V, O.d, rng)
    O.bcs_on_spinor(src)
    d_dev, d_o = lat.field(), O.new_field()
    lat.Dphi(-0.4, d_dev, lat.field(src))
    O.Dphi(-0.4, d_o, src.copy())
    assert rel(lat.download(d_dev), d_o) < 1e-12


def test_errors():
    from yahmc_b200 import YGError
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=84)
    with pytest.raises(YGError):
        lat.wf_fermion_init(0)
    with pytest.raises(YGError):
        lat.wf_fermion_iterate(0.01, [lat.field() for _ in range(33)])
