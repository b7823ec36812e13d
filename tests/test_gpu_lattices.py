"""Independent CG solves on several lattices at once (yg_cg_inverter_lattices): each lattice's
solve runs in its own host thread on the lattice's own stream.  Every solve is the
single-lattice cg_inverter with deterministic reductions, so the solutions and iteration
counts must equal those of one-at-a-time calls bit for bit, whatever the sizes and
configurations mixed in one call."""
import numpy as np
import pytest

from tests.helpers import make_pair, source

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", [
    [("su3_fund_ap", (8, 8, 8, 8)), ("su3_fund_ap", (12, 12, 12, 12)), ("su3_fund_ap", (16, 16, 16, 16))],
    [("su3_fund_open", (8, 8, 8, 8)), ("su2_adj_ap", (4, 6, 4, 8)), ("su3_fund_ap_full", (8, 8, 8, 8)),
     ("su3_fund_ap_nocl", (12, 8, 8, 8))],
])
def test_concurrent_equals_sequential(case):
    from yahmc_b200 import cg_inverter_lattices
    solves, refs = [], []
    for k, (name, dims) in enumerate(case):
        lat, O, rng = make_pair(name, dims, seed=90 + k)
        b = lat.field(source(O, rng))
        x1 = lat.field()
        it1 = lat.cg_inverter("Hphi_sq", -0.4, 1e-22, x1, b)
        refs.append((lat.download(x1), it1))
        solves.append((lat, -0.4, 1e-22, lat.field(), b))
    for _ in range(2):                                   # twice: scratch fields reused
        for s in solves:
            s[0].spinor_zero(s[3])
        its, rc = cg_inverter_lattices(solves)
        assert rc == 0
        for (lat, _, _, x, _), (xr, itr), it in zip(solves, refs, its):
            assert it == itr
            assert np.array_equal(lat.download(x), xr)


def test_errors():
    from yahmc_b200 import YGError, cg_inverter_lattices
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=99)
    b = lat.field(source(O, rng))
    with pytest.raises(YGError):
        cg_inverter_lattices([(lat, -0.4, 1e-20, lat.field(), b), (lat, -0.4, 1e-20, lat.field(), b)])
