"""Pin the numpy oracle (oracle/yahmc_oracle.py) to the unmodified reference.

The reference is compiled from its own sources into oracle/_ref by
oracle/build_ref.py; these tests feed both the same seeded 8^4 fields (8^4 is
the smallest lattice the reference accepts, geometry.cpp:1140-1144) and
require agreement to rounding.  Skipped when oracle/_ref has not been built
(for example on a machine without the reference sources); the committed golden
vectors in tests/golden/ pin the oracle there instead.
"""
import numpy as np
import pytest

from oracle import ref, yahmc_oracle as yo
from yahmc_b200 import fields

DIMS = (8, 8, 8, 8)
TOL = 1e-13


def _setup(name, seed):
    if not ref.available(name):
        pytest.skip("oracle/_ref not built")
    nc, rep, bc, clover, eo = ref.CONFIGS[name]
    R = ref.get(name, DIMS)
    O = yo.Oracle(yo.Params(DIMS, nc, rep, bc, clover, eo, 1.0, 1.0))
    rng = np.random.default_rng(seed)
    U = fields.haar_su(nc, O.V * 4, rng).reshape(O.V, 4, nc, nc)
    R.set_links(fields.complex_to_raw(U))
    O.set_links(U)
    src = fields.gaussian_spinor(O.V, O.d, rng)
    O.bcs_on_spinor(src)
    return R, O, rng, src


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("name", list(ref.CONFIGS))
def test_geometry_links_clover(name):
    R, O, rng, src = _setup(name, 1)
    c, f, b = R.geometry()
    assert np.array_equal(c, O.coord) and np.array_equal(f, O.fw) and np.array_equal(b, O.bk)
    V, d = O.V, O.d
    assert _rel(yo.mat_from_raw(R.repr_links(), d).reshape(V, 4, d, d), O.links) < TOL
    gf, gr = R.generators()
    assert _rel(yo.mat_from_raw(gf, O.nc), O.itfund) < TOL
    assert _rel(yo.mat_from_raw(gr, d), O.itrepr) < TOL
    if O.p.clover:
        assert _rel(yo.mat_from_raw(R.clover_term(), d).reshape(V, 4, d, d), O.cl_term) < TOL
        for m in (-0.75, 0.1):
            lr = R.ldl(m).reshape(V, 2, d * (2 * d + 1), 2)
            lr = lr[..., 0] + 1j * lr[..., 1]
            lo = O.compute_ldl(4 + m)
            assert _rel(lr[V // 2:], lo[V // 2:]) < TOL
            assert abs(R.call("clover_logdet", m) - O.clover_logdet(m)) < 1e-12 * abs(O.clover_logdet(m))


@pytest.mark.parametrize("name", list(ref.CONFIGS))
def test_dirac_operators(name):
    R, O, rng, src = _setup(name, 2)
    d = O.d
    fns = [("Dphi", -0.75), ("Hphi", -0.3), ("Hphi_sq", -0.75)]
    if O.p.eo:
        fns += [("Dphi_oe", None), ("Dphi_eo", None)]
        if O.p.clover:
            fns += [("Dphi_ee", -0.75), ("Dphi_oo", 0.2), ("Dphi_oo_inv", -0.75)]
    for fn, mass in fns:
        s1 = yo.spinor_to_raw(src)
        d1 = R.spinor()
        args = ([mass] if mass is not None else []) + [d1, s1]
        R.call(fn, *args)
        s2 = src.copy()
        d2 = O.new_field()
        getattr(O, fn)(*(([mass] if mass is not None else []) + [d2, s2]))
        assert _rel(yo.spinor_from_raw(d1, d), d2) < TOL, fn
        # aliasing semantics: Dphi writes scratch into the odd half of its source
        assert _rel(yo.spinor_from_raw(s1, d), s2) < TOL, fn


@pytest.mark.parametrize("name", ["su3_fund_ap", "su2_adj_ap", "su3_fund_open", "su3_fund_ap_nocl", "su3_fund_ap_full"])
def test_inverters(name):
    R, O, rng, src = _setup(name, 3)
    d = O.d
    lo, hi = O.default_range()
    m = -0.2
    cases = [("cg", 2, "Hphi_sq"), ("bicgstab", 0, "Dphi"), ("minres", 1, "Hphi"), ("auto_inverter", 2, "Hphi_sq")]
    for fn, op, opn in cases:
        x1 = R.spinor()
        b1 = yo.spinor_to_raw(src)
        it1 = R.call(fn, op, m, 1e-24, x1, b1)
        x2 = O.new_field()
        it2 = getattr(O, fn)(opn, m, 1e-24, x2, src.copy())
        assert abs(it1 - it2) <= 2, (fn, it1, it2)
        assert _rel(yo.spinor_from_raw(x1, d)[lo:hi], x2[lo:hi]) < 1e-11, fn
    sh = np.array([0.5, 0.1, 0.05, 1.05])     # the shifts of checks/inverters.cpp:143-146
    xs1 = np.zeros(4 * O.V * 8 * d)
    it1 = R.call("cg_mshift", 2, m, 1e-24, 4, sh, xs1, yo.spinor_to_raw(src))
    it2, xs2 = O.cg_mshift("Hphi_sq", m, 1e-24, list(sh), src.copy())
    assert abs(it1 - it2) <= 1
    xs1 = yo.spinor_from_raw(xs1, d).reshape(4, O.V, d, 4)
    for i in range(4):
        assert _rel(xs1[i][lo:hi], xs2[i][lo:hi]) < 1e-11


@pytest.mark.parametrize("name", ["su3_fund_ap", "su2_adj_ap", "su3_sym_ap", "su3_fund_sf", "su3_fund_ap_nocl"])
def test_forces(name):
    R, O, rng, src = _setup(name, 4)
    V, d = O.V, O.d
    R.zero_momenta()
    O.mom[:] = 0
    R.call("begin_fermion_force")
    O.begin_fermion_force()
    a = fields.gaussian_spinor(V, d, rng)
    b = fields.gaussian_spinor(V, d, rng)
    O.bcs_on_spinor(a)
    O.bcs_on_spinor(b)
    a1, b1 = yo.spinor_to_raw(a), yo.spinor_to_raw(b)
    a2, b2 = a.copy(), b.copy()
    R.call("wilson_fermion_force", 0.1, -0.75, 1.3, a1, b1)
    O.wilson_fermion_force(0.1, -0.75, 1.3, a2, b2)
    assert _rel(R.momenta().reshape(V, 4, -1), O.mom) < TOL
    assert _rel(yo.spinor_from_raw(a1, d), a2) < TOL and _rel(yo.spinor_from_raw(b1, d), b2) < TOL
    R.call("wilson_fermion_force_q", 0.07, -0.75, 0.9, b1)
    O.wilson_fermion_force_q(0.07, -0.75, 0.9, b2)
    if O.p.clover:
        assert _rel(yo.mat_from_raw(R.clover_force(), d).reshape(V, 6, d, d), O.cl_force) < TOL
        R.call("clover_logdet_force", -0.75, 2.0)
        O.clover_logdet_force(-0.75, 2.0)
        assert _rel(yo.mat_from_raw(R.clover_force(), d).reshape(V, 6, d, d), O.cl_force) < TOL
        R.call("end_fermion_force", 0.1)
        O.end_fermion_force(0.1)
    assert _rel(R.momenta().reshape(V, 4, -1), O.mom) < TOL


@pytest.mark.parametrize("name", ["su3_fund_ap", "su2_fund_ap", "su4_fund_ap"])
def test_gauge_support(name):
    R, O, rng, src = _setup(name, 5)
    R.zero_momenta()
    O.mom[:] = 0
    R.call("wilson_gauge_force", 0.1, 5.6)
    O.wilson_gauge_force(0.1, 5.6)
    assert _rel(R.momenta().reshape(O.V, 4, -1), O.mom) < TOL
    assert abs(R.call("avr_wilson", 1, 1) - O.plaquette()) < 1e-14


def test_reference_self_checks_pass():
    """The reference's own --run-checks (checks/check.cpp:4-26) pass on the compiled oracle."""
    if not ref.available("su3_fund_ap"):
        pytest.skip("oracle/_ref not built")
    R = ref.get("su3_fund_ap", DIMS, seed=99)
    R.set_random_links()
    assert R.call("check_group") == 0
    assert R.call("check_dirac") == 0
    assert R.call("check_inverters") == 0


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_per", "su3_fund_open", "su3_fund_sf", "su2_fund_ap",
                                  "su4_fund_ap"])
def test_md_support(name):
    """Weighted Wilson loops, the Symanzik force, the momentum part of hamiltonian(),
    update_links (exp, momentum and link boundary conditions) and reunitarize."""
    R, O, rng, src = _setup(name, 6)
    V, nc = O.V, O.nc
    mom = rng.normal(0.0, 2 ** -0.5, (V, 4, nc * nc - 1))
    R.lib.yref_set_momenta(ref._ptr(np.ascontiguousarray(mom.reshape(-1))))
    O.mom[:] = mom
    for h, w in [(1, 1), (1, 2), (2, 1)]:
        assert abs(R.call("avr_wilson", h, w) - O.avr_wilson(h, w)) < 1e-14
    c0 = 5.0 / 3.0
    R.call("improved_gauge_force", 0.1, 5.6, c0, (1 - c0) / 8)
    O.improved_gauge_force(0.1, 5.6, c0, (1 - c0) / 8)
    assert _rel(R.momenta().reshape(V, 4, -1), O.mom) < TOL
    h_ref = R.call("hamiltonian")
    assert abs(h_ref - O.hamiltonian_momenta()) < 1e-13 * abs(h_ref)
    assert _rel(R.momenta().reshape(V, 4, -1), O.mom) < TOL
    R.call("update_links", 0.13)
    O.update_links(0.13)
    assert _rel(yo.mat_from_raw(R.get_links(), nc).reshape(V, 4, nc, nc), O.fund) < 1e-13
    R.call("represent_gauge_field")
    O.represent_gauge_field()
    assert _rel(yo.mat_from_raw(R.repr_links(), O.d).reshape(V, 4, O.d, O.d), O.links) < 1e-13
    Up = O.fund + 1e-3 * (rng.normal(size=O.fund.shape) + 1j * rng.normal(size=O.fund.shape))
    R.set_links(fields.complex_to_raw(Up))
    O.fund = Up.copy()
    R.call("reunitarize")
    O.reunitarize_links()
    assert _rel(yo.mat_from_raw(R.get_links(), nc).reshape(V, 4, nc, nc), O.fund) < 1e-12


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su2_adj_ap", "su3_fund_ap_nocl"])
def test_mre_guess(name):
    """mre_store / mre_guess (mre.cpp:15-117) with lu (solver.cpp:4-95): 6 stored solutions in
    a 4-deep history, then the extrapolated guess for a new source."""
    R, O, rng, src = _setup(name, 8)
    R.call("mre_init", 4, 2, -0.3)
    O.mre_init(4, "Hphi_sq", -0.3)
    for _ in range(6):
        s = fields.gaussian_spinor(O.V, O.d, rng)
        O.bcs_on_spinor(s)
        R.call("mre_store", yo.spinor_to_raw(s))
        O.mre_store(s)
    d_r = np.zeros(O.V * 8 * O.d)
    R.call("mre_guess", d_r, yo.spinor_to_raw(src))
    d_o = O.new_field()
    O.mre_guess(d_o, src.copy())
    lo, hi = O.default_range()
    assert _rel(yo.spinor_from_raw(d_r, O.d)[lo:hi], d_o[lo:hi]) < 1e-12


@pytest.mark.parametrize("name", ["su3_fund_ap", "su2_adj_ap", "su3_fund_open"])
def test_gauge_files(name, tmp_path):
    """gauge_field_save/load (gaugefield.cpp:44-161) and the HiRep pair (hirep.cpp:56-212):
    the oracle reads the reference's files bit-exactly, and the reference loads the
    oracle's files into the same links (boundary conditions applied)."""
    R, O, rng, src = _setup(name, 9)
    nc = O.nc
    U = yo.mat_from_raw(R.get_links(), nc).reshape(O.V, 4, nc, nc)
    p = tmp_path / "a.cfg"
    R.call("gauge_save", str(p).encode())
    c = yo.cfg_read(p)
    assert c["ident"] == yo.CFG_IDENT and c["version"] == yo.CFG_VERSION
    assert c["dims"] == DIMS and c["nc"] == nc and c["repr"] == yo.REPR_NAMES.index(O.p.rep)
    assert np.array_equal(c["U"], U)
    assert abs(c["plaquette"] - R.call("avr_wilson", 1, 1)) < 1e-15
    h = tmp_path / "a.hirep"
    R.call("gauge_save_hirep", str(h).encode())
    hr = yo.hirep_read(h)
    assert hr["dims"] == DIMS and hr["nc"] == nc and np.array_equal(hr["U"], U)
    W = fields.haar_su(nc, O.V * 4, rng).reshape(O.V, 4, nc, nc)
    O.fund = W.copy()
    O.bcs_on_gauge()
    q = tmp_path / "b.cfg"
    yo.cfg_write(q, W, DIMS, nc, yo.REPR_NAMES.index(O.p.rep), 0.5, 7, 3)
    R.call("gauge_load", str(q).encode())
    assert np.array_equal(yo.mat_from_raw(R.get_links(), nc).reshape(O.V, 4, nc, nc), O.fund)
    R.set_links(fields.complex_to_raw(U))
    q = tmp_path / "run1_n42"
    yo.hirep_write(q, W, DIMS, nc, 0.25)
    R.call("gauge_load_hirep", str(q).encode())
    assert np.array_equal(yo.mat_from_raw(R.get_links(), nc).reshape(O.V, 4, nc, nc), O.fund)


@pytest.mark.parametrize("name,method", [("su3_fund_ap", yo.POINT), ("su3_fund_ap", yo.SEMWALL),
                                         ("su3_fund_open", yo.POINT), ("su3_fund_ap_nocl", yo.POINT),
                                         ("su2_adj_ap", yo.SEMWALL), ("su3_fund_ap_full", yo.SEMWALL)])
def test_mesons(name, method):
    """meson_init + meson_measure (mesons.cpp:150-298, with create_*_source and
    calc_propagator of propagator.cpp): the oracle's correlators against the ones the
    reference prints (%1.6e, so to half a unit in the 7th digit).  The source time slices
    are read from its log; the semwall noise is the reference's own stream, replayed with
    rand_store / rand_load."""
    R, O, rng, src = _setup(name, 10)
    hits = 1 if method == yo.POINT else 2
    state = np.zeros(512)
    sz = R.call("rand_store", state)
    taus, printed = ref.mesons(R, -0.3, 1e-24, hits, method)
    assert len(taus) == hits and len(printed) == 16
    noises = None
    if method == yo.SEMWALL:
        R.call("rand_load", state, sz)
        vol3, noises, replay = O.V // DIMS[0], [], []
        for _ in range(hits):
            if O.p.bc in ("open", "sf"):
                replay.append(1)                     # random_timeslice, propagator.cpp:10-19
            else:
                u = np.zeros(1)
                R.call("rand_uniform", 1, u)
                replay.append(int(u[0] * DIMS[0]))
            u = np.zeros(2 * O.d * vol3)
            R.call("rand_uniform", len(u), u)
            noises.append(np.where(u < 0.5, 2 ** -0.5, -2 ** -0.5))
        assert replay == taus
    raw = O.meson_measure(-0.3, 1e-24, method, taus, noises)
    mine = yo.meson_print_values(raw, method, hits, O.V // DIMS[0])
    for lab, v in printed.items():
        scale = np.abs(v).max()
        assert np.all(np.abs(mine[lab] - v) <= 5.01e-7 * np.abs(v) + 1e-12 * scale), lab


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_ap_nocl", "su3_fund_ap_full", "su2_adj_ap"])
def test_sources_and_propagator(name):
    """create_point_source, create_semwall_source (noise order = the reference's draw order)
    and calc_propagator at full precision."""
    R, O, rng, src = _setup(name, 11)
    d = O.d
    for n in (0, d + 1, 4 * d - 1):
        r = np.zeros(O.V * 8 * d)
        R.call("point_source", n, 3, r)
        assert np.array_equal(yo.spinor_from_raw(r, d), O.create_point_source(n, 3))
    state = np.zeros(512)
    sz = R.call("rand_store", state)
    f = np.zeros(O.V * 8 * d)
    R.call("semwall_source", 0, 5, f)
    R.call("rand_load", state, sz)
    u = np.zeros(2 * d * (O.V // DIMS[0]))
    R.call("rand_uniform", len(u), u)
    fo = O.new_field()
    O.create_semwall_source(0, 5, fo, np.where(u < 0.5, 2 ** -0.5, -2 ** -0.5))
    assert np.array_equal(yo.spinor_from_raw(f, d), fo)
    for n in (1, 2, 3):
        R.call("semwall_source", n, 5, f)
        O.create_semwall_source(n, 5, fo)
        assert np.array_equal(yo.spinor_from_raw(f, d), fo)
    x0 = 0.01 * fields.gaussian_spinor(O.V, d, rng)
    dr, sr = yo.spinor_to_raw(x0).copy(), yo.spinor_to_raw(src).copy()
    R.call("calc_propagator", -0.3, 1e-24, dr, sr)
    do, so = x0.copy(), src.copy()
    O.calc_propagator(-0.3, 1e-24, do, so)
    assert _rel(yo.spinor_from_raw(dr, d), do) < 1e-12
    assert np.array_equal(yo.spinor_from_raw(sr, d), so)


@pytest.mark.parametrize("name", ["su3_fund_ap", "su3_fund_open", "su3_fund_sf", "su2_adj_ap", "su3_fund_ap_full",
                                  "su4_fund_ap"])
def test_wilson_flow(name):
    """wf_iterate, wf_e_plaq, wf_e_sym, wf_charge (wilsonflow.cpp) and wf_fermion_iterate
    (fermionflow.cpp) on a smooth field: links, observables and flowed fields to rounding."""
    R, O, rng, src = _setup(name, 12)
    nc = O.nc
    U = yo.exp_algebra(nc, rng.normal(0, 0.5, (O.V, 4, nc * nc - 1)), 1.0)
    O.fund = U
    O.bcs_on_gauge()
    U = O.fund.copy()
    R.set_links(fields.complex_to_raw(U))
    O.set_links(U)

    def check_obs():
        r = np.zeros(3)
        R.call("wf_observables", r)
        o = np.array([O.wf_e_plaq(), O.wf_e_sym(), O.wf_charge()])
        assert np.all(np.abs(r - o) < 1e-12 * np.maximum(np.abs(o), 1.0)), (r, o)

    check_obs()
    R.call("wf_init")
    O.wf_init()
    for _ in range(2):
        R.call("wf_iterate", 0.02)
        O.wf_iterate(0.02)
    assert _rel(yo.mat_from_raw(R.get_links(), nc).reshape(O.V, 4, nc, nc), O.fund) < 1e-13
    check_obs()
    phis = [fields.gaussian_spinor(O.V, O.d, rng) for _ in range(2)]
    raws = [yo.spinor_to_raw(p).copy() for p in phis]
    ptrs = np.array([r.ctypes.data for r in raws], dtype=np.uint64)
    R.lib.yref_wf_fermion_init(ptrs.ctypes.data_as(ref.ctypes.c_void_p), 2)
    O.wf_fermion_init(phis)
    for _ in range(2):
        R.call("wf_fermion_iterate", 0.02)
        O.wf_fermion_iterate(0.02)
    for r, p in zip(raws, phis):
        assert _rel(yo.spinor_from_raw(r, O.d), p) < 1e-13
    assert _rel(yo.mat_from_raw(R.get_links(), nc).reshape(O.V, 4, nc, nc), O.fund) < 1e-13
