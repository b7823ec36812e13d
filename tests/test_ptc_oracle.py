"""The FP64 restatement of the learned preconditioner (oracle/ptc_oracle.py) on the CPU:
its gradients agree with finite differences of its loss, its layer and adjoint are adjoint
to each other, the network is exactly gauge-equivariant, and flexible GCR solves the Schur
system with any preconditioner."""
import numpy as np
import pytest

from oracle import ptc_oracle as po
from oracle import yahmc_oracle as yo
from yahmc_b200 import fields


def _setup(dims=(4, 4, 4, 4), seed=3, name="su3_fund_ap"):
    from tests.helpers import CONFIGS
    nc, rep, bc, clover, eo = CONFIGS[name]
    O = yo.Oracle(yo.Params(tuple(dims), nc, rep, bc, clover, eo, 1.0, 1.0))
    rng = np.random.default_rng(seed)
    O.set_links(fields.haar_su(nc, O.V * 4, rng).reshape(O.V, 4, nc, nc))
    return O, rng


def _rand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)


def test_layer_adjoint():
    O, rng = _setup()
    W = _rand(rng, (9, 3, 2, 4, 4))
    f = _rand(rng, (O.V, 2, O.d, 4))
    g = _rand(rng, (O.V, 3, O.d, 4))
    lhs = np.vdot(g, po.layer(O, W, f))
    rhs = np.vdot(po.layer_adjoint(O, W, g), f)
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_gradients_match_finite_differences():
    O, rng = _setup()
    net = po.Net.init((1, 2, 2, 1), rng)
    pairs = []
    for _ in range(2):
        e = _rand(rng, (O.Vh, O.d, 4))
        pairs.append((po.dhat(O, -0.5, e), e))
    L, grads = po.loss_and_grads(O, net, pairs)
    eps = 1e-6
    for l, idx in ((0, (3, 1, 0, 2, 1)), (1, (0, 1, 1, 0, 3)), (2, (7, 0, 1, 3, 3))):
        for unit in (1.0, 1j):
            Wp = [w.copy() for w in net.W]
            Wm = [w.copy() for w in net.W]
            Wp[l][idx] += eps * unit
            Wm[l][idx] -= eps * unit
            fd = (po.loss_and_grads(O, po.Net(Wp), pairs)[0] - po.loss_and_grads(O, po.Net(Wm), pairs)[0]) / (2 * eps)
            g = grads[l][idx]
            an = 2 * (g.real if unit == 1.0 else g.imag)
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (l, idx, unit, fd, an)


@pytest.mark.parametrize("name", ["su3_fund_ap", "su2_adj_ap"])
def test_network_is_gauge_equivariant(name):
    """N[U^Omega](Omega psi) = Omega N[U](psi) with U_mu(x) -> Omega(x) U_mu(x) Omega(x+mu)^dag,
    psi(x) -> Omega(x) psi(x) (checks/dirac.cpp:92-189 transforms the fields the same way)."""
    O, rng = _setup(name=name)
    net = po.Net.init((1, 3, 3, 1), rng)
    f = _rand(rng, (O.V, 1, O.d, 4))
    y = net.forward(O, f)
    om = fields.haar_su(O.nc, O.V, rng)
    om_r = yo.represent(om.reshape(O.V, 1, O.nc, O.nc), O.nc, O.p.rep)[:, 0]
    U = O.fund.copy()
    Ut = np.einsum("xab,xmbc,xmdc->xmad", om, U, np.conj(om[O.fw]))
    O.set_links(Ut)
    yt = net.forward(O, np.einsum("xab,xcbs->xcas", om_r, f))
    assert np.abs(yt - np.einsum("xab,xcbs->xcas", om_r, y)).max() <= 1e-12 * np.abs(y).max()


def test_fgcr_solves_with_a_preconditioner():
    O, rng = _setup(seed=4)
    mass, prec = -0.5, 1e-20
    b = _rand(rng, (O.Vh, O.d, 4))
    net = po.Net.near_identity((1, 2, 1), rng)
    for pre in (lambda r: r, lambda r: po.apply_even(O, net, r)):
        x, it = po.fgcr(O, mass, prec, b, pre)
        r = b - po.dhat(O, mass, x)
        assert np.vdot(r, r).real < 10 * prec * np.vdot(b, b).real
        assert it > 0
