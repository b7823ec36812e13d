"""Parity of the CUDA Dirac operator, clover term and representation map with the oracle.

FP64 throughout: the tolerance is relative 1e-13 (the reference's own checks use 1e-14
on self-consistency; agreement with the CPU code is asked to 1e-13).  Small lattices
(ragged 4x6x4x8 shapes) keep the oracle fast; 8^4 covers the SU(3) fundamental configs.
"""
import numpy as np
import pytest

from tests.helpers import CONFIGS, make_pair, rel, source

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _dims(name):
    nc, rep, *_ = CONFIGS[name]
    return (8, 8, 8, 8) if (nc == 3 and rep == "fundamental") else (4, 6, 4, 8)


@pytest.mark.parametrize("name", list(CONFIGS))
def test_links_clover_ldl(name):
    lat, O, rng = make_pair(name, _dims(name), seed=1)
    assert rel(lat.repr_links(), O.links) < TOL
    assert np.array_equal(lat.get_links(), O.fund)
    if O.p.clover:
        assert rel(lat.clover_term(), O.cl_term, floor=1.0) < TOL
        for m in (-0.75, 0.3):
            lo = O.compute_ldl(4 + m)
            lg = lat.ldl(m)
            assert rel(lg[O.Vh:], lo[O.Vh:]) < TOL
            assert abs(lat.clover_logdet(m) - O.clover_logdet(m)) < 1e-12 * abs(O.clover_logdet(m))


@pytest.mark.parametrize("name", list(CONFIGS))
def test_operators(name):
    lat, O, rng = make_pair(name, _dims(name), seed=2)
    src = source(O, rng)
    fns = [("Dphi", -0.75), ("Hphi", -0.3), ("Hphi_sq", -0.75)]
    if O.p.eo:
        fns += [("Dphi_oe", None), ("Dphi_eo", None)]
        if O.p.clover:
            fns += [("Dphi_ee", -0.75), ("Dphi_oo", 0.2), ("Dphi_oo_inv", -0.75)]
    for fn, mass in fns:
        s_dev = lat.field(src)
        d_dev = lat.field()
        s2 = src.copy()
        d2 = O.new_field()
        margs = [mass] if mass is not None else []
        getattr(lat, fn)(*margs, d_dev, s_dev)
        getattr(O, fn)(*margs, d2, s2)
        assert rel(lat.download(d_dev), d2) < TOL, fn
        # the in-place side effect on the source (dirac.cpp:743) is part of the contract
        assert rel(lat.download(s_dev), s2) < TOL, fn


def test_unprojected_source_boundary_semantics():
    """Open boundaries with a source that violates them: the reference zeroes boundary slices
    of both the output and the source of every hop (bcs.cpp:139-146)."""
    from yahmc_b200 import fields
    lat, O, rng = make_pair("su3_fund_open", (4, 4, 4, 6), seed=3)
    src = fields.gaussian_spinor(O.V, O.d, rng)        # boundary slices not zero
    for fn in ("Dphi_oe", "Dphi"):
        s_dev, d_dev = lat.field(src), lat.field(fields.gaussian_spinor(O.V, O.d, rng))
        d2 = lat.download(d_dev)
        s2 = src.copy()
        args = [-0.6] if fn == "Dphi" else []
        getattr(lat, fn)(*args, d_dev, s_dev)
        getattr(O, fn)(*args, d2, s2)
        assert rel(lat.download(d_dev), d2) < TOL
        assert rel(lat.download(s_dev), s2) < TOL


def test_mvm_counter():
    lat, O, rng = make_pair("su3_fund_ap", (4, 4, 4, 4), seed=4)
    s, d = lat.field(source(O, rng)), lat.field()
    lat.mvm_reset()
    lat.Hphi_sq(-0.5, d, s)            # 4 hops, counted /2 with even-odd (dirac.cpp:11-18)
    assert lat.mvm_get() == 2
    lat.Dphi_oe(d, s)
    lat.Dphi_eo(d, s)
    assert lat.mvm_get() == 3


def test_hermiticity_and_clover_inverse():
    """checks/dirac.cpp:7-90 on the device: <u,Hv> = <Hu,v> and D_oo^-1 D_oo u = u."""
    from yahmc_b200 import VIEW_ODD
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=5)
    u, v = lat.field(source(O, rng)), lat.field(source(O, rng))
    Mu, Mv = lat.field(), lat.field()
    lat.Hphi(-0.5, Mu, u)
    lat.Hphi(-0.5, Mv, v)
    norm = np.sqrt(lat.spinor_sqnorm(u) * lat.spinor_sqnorm(v))
    r = abs(lat.spinor_product(u, Mv) - lat.spinor_product(Mu, v)) / norm
    assert r < 1e-14
    a, b = lat.field(source(O, rng)), lat.field()
    n0 = lat.spinor_sqnorm(a, VIEW_ODD)
    lat.Dphi_oo(-0.5, b, a)
    lat.Dphi_oo_inv(-0.5, b, b)
    lat.spinor_sub_assign(a, b, VIEW_ODD)
    assert np.sqrt(lat.spinor_sqnorm(a, VIEW_ODD) / n0) < 1e-14


def test_gauge_covariance():
    """checks/dirac.cpp:92-189: D[U^g] (g psi) = g D[U] psi for a random gauge transformation."""
    from yahmc_b200 import fields
    from oracle import yahmc_oracle as yo
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=6)
    src = source(O, rng)
    s, d1 = lat.field(src), lat.field()
    lat.Dphi(-0.5, d1, s)
    r1 = lat.download(d1)
    g = fields.haar_su(3, O.V, rng)
    Ug = np.einsum("vab,vmbc->vmac", g, O.fund)
    for mu in range(4):
        Ug[:, mu] = Ug[:, mu] @ yo.dagger(g[O.fw[:, mu]])
    lat.set_links(Ug)
    s2, d2 = lat.field(yo.col_apply(g, src)), lat.field()
    lat.Dphi(-0.5, d2, s2)
    lo, hi = O.default_range()
    expect = yo.col_apply(g, r1)
    assert rel(lat.download(d2)[lo:hi], expect[lo:hi]) < 1e-13
