"""Parity of the CUDA fermion forces (and gauge support) with the oracle, FP64, rel 1e-13."""
import pytest

from tests.helpers import CONFIGS, make_pair, rel, source

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _dims(name):
    nc, rep, *_ = CONFIGS[name]
    return (8, 8, 8, 8) if (nc == 3 and rep == "fundamental") else (4, 6, 4, 8)


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_sf", "su3_fund_ap_nocl", "su3_fund_ap_full",
                                  "su2_adj_ap", "su3_sym_ap", "su4_asym_ap", "su2_fund_ap",
                                  "su3_adj_ap", "su4_sym_ap", "su4_adj_ap", "su2_asym_ap"])
def test_fermion_forces(name):
    lat, O, rng = make_pair(name, _dims(name), seed=20)
    lat.zero_momenta()
    O.mom[:] = 0
    lat.begin_fermion_force()
    O.begin_fermion_force()
    a0, b0 = source(O, rng), source(O, rng)
    a, b = lat.field(a0), lat.field(b0)
    a2, b2 = a0.copy(), b0.copy()
    lat.wilson_fermion_force(0.1, -0.75, 1.3, a, b)
    O.wilson_fermion_force(0.1, -0.75, 1.3, a2, b2)
    assert rel(lat.momenta(), O.mom, floor=1.0) < TOL
    # the odd halves of both arguments are replaced in place (forces.cpp:182-188)
    assert rel(lat.download(a), a2) < TOL and rel(lat.download(b), b2) < TOL
    lat.wilson_fermion_force_q(0.07, -0.75, 0.9, b)
    O.wilson_fermion_force_q(0.07, -0.75, 0.9, b2)
    assert rel(lat.momenta(), O.mom, floor=1.0) < TOL
    if O.p.clover:
        assert rel(lat.clover_force(), O.cl_force, floor=1.0) < TOL
        if O.p.eo:
            lat.clover_logdet_force(-0.75, 2.0)
            O.clover_logdet_force(-0.75, 2.0)
            assert rel(lat.clover_force(), O.cl_force, floor=1.0) < TOL
        lat.end_fermion_force(0.1)
        O.end_fermion_force(0.1)
        assert rel(lat.momenta(), O.mom, floor=1.0) < TOL


@pytest.mark.parametrize("name", ["su3_fund_ap", "su2_fund_ap", "su4_fund_ap"])
def test_gauge_force_and_plaquette(name):
    lat, O, rng = make_pair(name, (4, 6, 4, 8), seed=21)
    lat.zero_momenta()
    O.mom[:] = 0
    lat.wilson_gauge_force(0.1, 5.6)
    O.wilson_gauge_force(0.1, 5.6)
    assert rel(lat.momenta(), O.mom, floor=1.0) < TOL
    assert abs(lat.plaquette() - O.plaquette()) < 1e-14


@pytest.mark.parametrize("name", ["su3_fund_ap", "su2_adj_ap", "su3_fund_ap_nocl", "su3_fund_open", "su3_fund_ap_full"])
def test_rhmc_pole_force_batched(name):
    """The pole loop of MonomialRHMC::update (rhmc.cpp:100-103) as one batched force: momenta,
    clover force and the in-place odd halves agree with the poles applied one by one, on the
    engine and in the oracle."""
    lat, O, rng = make_pair(name, _dims(name), seed=22)
    residues = [0.31, 1.7, 0.05, 2.9, 0.8]
    srcs = [source(O, rng) for _ in residues]
    dt, mass = 0.06, -0.7
    lat.zero_momenta()
    O.mom[:] = 0
    lat.begin_fermion_force()
    O.begin_fermion_force()
    fs = [lat.field(s) for s in srcs]
    lat.wilson_fermion_force_q_multi(dt, mass, residues, fs)
    hs = [s.copy() for s in srcs]
    for r, h in zip(residues, hs):
        O.wilson_fermion_force_q(dt, mass, r, h)
    assert rel(lat.momenta(), O.mom, floor=1.0) < 1e-12
    for f, h in zip(fs, hs):
        assert rel(lat.download(f), h) < TOL
    if O.p.clover:
        assert rel(lat.clover_force(), O.cl_force, floor=1.0) < 1e-12
    # the same through the single-pole entry point, pole by pole
    mom_b = lat.momenta()
    lat.zero_momenta()
    lat.begin_fermion_force()
    for r, s in zip(residues, srcs):
        lat.wilson_fermion_force_q(dt, mass, r, lat.field(s))
    assert rel(lat.momenta(), mom_b, floor=1.0) < 1e-12
