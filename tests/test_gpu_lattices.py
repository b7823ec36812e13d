"""Independent CG solves on several lattices at once (yg_cg_inverter_lattices).

Hphi_sq solves on even-odd lattices of one representation dimension (2, 3, 4 or 6), all with
or all without a clover term and without open/SF boundaries, run as one persistent kernel:
each lattice's whole cg_inverter loop (cg.cpp:132-202) runs on a group of blocks with
bounded barriers.  Its reductions add the same terms in another order than the engine's
single-lattice BLAS, so solutions agree with one-at-a-time calls to rounding (relative 1e-10)
and iteration counts within one.  Any other mix runs each lattice's single-lattice solve in
its own host thread and must match one-at-a-time calls bit for bit."""
import numpy as np
import pytest

from tests.helpers import make_pair, source

pytestmark = pytest.mark.gpu


def _setup(case, mass=-0.4, prec=1e-22):
    solves, refs = [], []
    for k, (name, dims) in enumerate(case):
        lat, O, rng = make_pair(name, dims, seed=90 + k)
        b = lat.field(source(O, rng))
        x1 = lat.field()
        it1 = lat.cg_inverter("Hphi_sq", mass, prec, x1, b)
        refs.append((lat.download(x1), it1))
        solves.append((lat, mass, prec, lat.field(), b, 0))
    return solves, refs


def _even(lat, f):
    return lat.download(f)[:lat.V // 2]


PERSISTENT = [
    [("su3_fund_ap", (8, 8, 8, 8)), ("su3_fund_ap", (12, 12, 12, 12)), ("su3_fund_ap", (16, 16, 16, 16))],
    [("su2_adj_ap", (4, 6, 4, 8)), ("su3_fund_ap", (8, 8, 8, 8)), ("su3_fund_per", (6, 4, 4, 4))],
    [("su3_fund_ap_nocl", (12, 8, 8, 8)), ("su3_fund_ap_nocl", (4, 4, 4, 4))],
    [("su2_fund_ap", (8, 8, 8, 8)), ("su2_fund_ap", (4, 4, 4, 6))],
    [("su4_fund_ap", (8, 4, 4, 4)), ("su4_fund_ap", (4, 4, 4, 4))],
    [("su3_sym_ap", (4, 4, 4, 4)), ("su4_asym_ap", (6, 4, 4, 4))],
]


@pytest.mark.parametrize("case", PERSISTENT)
def test_persistent_batch_matches_one_at_a_time(case):
    from yahmc_b200 import cg_inverter_lattices
    solves, refs = _setup(case)
    for _ in range(2):                                   # twice: scratch fields and buffers reused
        for s in solves:
            s[0].spinor_zero(s[3])
        its, rc, path = cg_inverter_lattices(solves, with_path=True)
        assert rc == 0 and path == 1
        for (lat, _, _, x, _, _), (xr, itr), it in zip(solves, refs, its):
            assert abs(it - itr) <= 1, (it, itr)
            got, ref = _even(lat, x), xr[:lat.V // 2]
            assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


def test_persistent_batch_maxiter_and_converged_start():
    """A lattice that stops at maxiter reports YG_MAXITER and exactly maxiter iterations; a
    lattice whose initial guess already meets prec reports 0 iterations (cg.cpp:151-153), as
    cg_inverter does; the others are unaffected."""
    from yahmc_b200 import cg_inverter_lattices
    case = [("su3_fund_ap", (8, 8, 8, 8)), ("su3_fund_ap", (12, 8, 8, 8)), ("su3_fund_ap", (4, 4, 4, 4))]
    solves, refs = _setup(case)
    lat0, m, p, x0, b0, _ = solves[0]
    solves[0] = (lat0, m, p, x0, b0, 7)                  # stops after 7 iterations
    lat2, _, _, x2, b2, _ = solves[2]
    lat2.upload(x2, refs[2][0])                          # starts at a solution to 1e-22 ...
    solves[2] = (lat2, m, 1e-16, x2, b2, 0)              # ... of a system asked for 1e-16
    lat0.spinor_zero(x0)
    solves[1][0].spinor_zero(solves[1][3])
    its, rc, path = cg_inverter_lattices(solves, with_path=True)
    assert path == 1 and rc == 4
    assert its[0] == 7
    assert abs(its[1] - refs[1][1]) <= 1
    assert its[2] == lat2.cg_inverter("Hphi_sq", m, 1e-16, lat2.field(refs[2][0]), b2) == 0
    x7 = lat0.field()
    assert lat0.cg_inverter("Hphi_sq", m, p, x7, b0, maxiter=7) == 7
    a, c = _even(lat0, x0), _even(lat0, x7)
    assert np.abs(a - c).max() <= 1e-10 * np.abs(c).max()


def test_persistent_batch_wait_limit_returns_timeout():
    """A barrier wait limit of a few cycles runs out at the first barrier: the kernel returns
    (no trap, no hang), the call reports YG_TIMEOUT, and the next call on the same lattices
    solves them normally."""
    from yahmc_b200 import cg_inverter_lattices
    case = [("su3_fund_ap", (8, 8, 8, 8)), ("su3_fund_ap", (16, 16, 16, 16))]
    solves, refs = _setup(case)
    its, rc, path = cg_inverter_lattices(solves, wait_cycles=8, with_path=True)
    assert path == 1 and rc == 7
    for s in solves:
        s[0].spinor_zero(s[3])
    its, rc = cg_inverter_lattices(solves)
    assert rc == 0
    for (lat, _, _, x, _, _), (xr, itr), it in zip(solves, refs, its):
        assert abs(it - itr) <= 1
        got, ref = _even(lat, x), xr[:lat.V // 2]
        assert np.abs(got - ref).max() <= 1e-10 * np.abs(ref).max()


@pytest.mark.parametrize("case", [
    [("su3_fund_open", (8, 8, 8, 8)), ("su2_adj_ap", (4, 6, 4, 8)), ("su3_fund_ap_full", (8, 8, 8, 8)),
     ("su3_fund_ap_nocl", (12, 8, 8, 8))],
    [("su3_adj_ap", (4, 4, 4, 4)), ("su3_adj_ap", (6, 4, 4, 4))],          # d = 8: host threads
])
def test_threads_equal_sequential(case):
    from yahmc_b200 import cg_inverter_lattices
    solves, refs = _setup(case)
    for _ in range(2):
        for s in solves:
            s[0].spinor_zero(s[3])
        its, rc, path = cg_inverter_lattices(solves, with_path=True)
        assert rc == 0 and path == 0
        for (lat, _, _, x, _, _), (xr, itr), it in zip(solves, refs, its):
            assert it == itr
            assert np.array_equal(lat.download(x), xr)


def test_errors():
    from yahmc_b200 import YGError, cg_inverter_lattices
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=99)
    b = lat.field(source(O, rng))
    with pytest.raises(YGError):
        cg_inverter_lattices([(lat, -0.4, 1e-20, lat.field(), b), (lat, -0.4, 1e-20, lat.field(), b)])
