"""The learned preconditioner on the GPU (yg_ptc_*, yg_fgcr, yg_solve_learned) against its FP64
restatement (oracle/ptc_oracle.py), whose gradients are checked against finite differences on
the CPU (tests/test_ptc_oracle.py).

Tolerances: the tensor-core products take BF16 operands (8 significant bits) and accumulate in
FP32, so a layer agrees with the FP64 layer to about 1e-2 of the output's largest entry."""
import numpy as np
import pytest

from oracle import ptc_oracle as po
from tests.helpers import make_pair, source

pytestmark = pytest.mark.gpu

TOL = 2e-2


def _planes(x):
    """oracle field (V, C, d, 4) complex -> activation site blocks: channel ch of site id is 24
    floats at (ch*V + id)*24, float (spin*3 + colour)*2 + re/im"""
    t = np.transpose(x, (1, 0, 3, 2))          # (C, V, 4, d)
    p = np.empty(t.shape + (2,), dtype=np.float32)
    p[..., 0] = t.real
    p[..., 1] = t.imag
    return p.reshape(-1)


def _from_planes(p, V, C, d=3):
    p = p.reshape(C, V, 4, d, 2)
    z = p[..., 0] + 1j * p[..., 1]
    return np.transpose(z, (1, 0, 3, 2))       # (V, C, d, 4)


def _rand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) / np.sqrt(2)


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("channels", [(1, 16, 16, 1), (1, 8, 8, 1)])
@pytest.mark.parametrize("name,dims", [("su3_fund_ap", (4, 4, 4, 4)), ("su3_fund_ap", (4, 6, 4, 8)),
                                       ("su2_adj_ap", (4, 4, 4, 4))])
def test_layers_and_adjoints_match_oracle(channels, name, dims):
    import torch
    from yahmc_b200 import Ptc
    lat, O, rng = make_pair(name, dims, seed=81)
    net = Ptc(lat, channels)
    Ws = [_rand(rng, s) / np.sqrt(9 * s[2] * 4) for s in net.shapes()]
    net.set_weights(Ws)
    for l, W in enumerate(Ws):
        ci, co = W.shape[2], W.shape[1]
        for adjoint in (0, 1):
            cin, cout = (co, ci) if adjoint else (ci, co)
            x = _rand(rng, (O.V, cin, O.d, 4))
            xin = torch.tensor(_planes(x), device="cuda")
            xout = torch.full((cout * 24 * O.V,), float("nan"), dtype=torch.float32, device="cuda")
            net.layer(l, adjoint, xin.data_ptr(), xout.data_ptr())
            got = _from_planes(xout.cpu().numpy(), O.V, cout, O.d)
            ref = po.layer_adjoint(O, W, x) if adjoint else po.layer(O, W, x)
            assert np.isfinite(got).all()
            assert _rel(got, ref) < TOL, (l, adjoint, _rel(got, ref))


def _even_pairs(lat, O, rng, n, mass):
    pairs, host = [], []
    for _ in range(n):
        e = source(O, rng)
        e[O.Vh:] = 0
        r = np.zeros_like(e)
        r[:O.Vh] = po.dhat(O, mass, e[:O.Vh])
        pairs.append((lat.field(r), lat.field(e)))
        host.append((r[:O.Vh], e[:O.Vh]))
    return pairs, host


def test_gradients_match_oracle_and_finite_differences():
    from yahmc_b200 import Ptc
    lat, O, rng = make_pair("su3_fund_ap", (4, 4, 4, 4), seed=82)
    mass = -0.5
    net = Ptc(lat, (1, 8, 8, 1))
    Ws = [_rand(rng, s) / np.sqrt(9 * s[2] * 4) for s in net.shapes()]
    for W in Ws:
        W[0, 0, 0] += np.eye(4)
    net.set_weights(Ws)
    pairs, host = _even_pairs(lat, O, rng, 2, mass)
    loss, grads = net.gradient(pairs)
    onet = po.Net(Ws)
    oloss, ograds = po.loss_and_grads(O, onet, host)
    assert abs(loss - oloss) <= TOL * abs(oloss), (loss, oloss)
    for l in range(3):
        assert _rel(grads[l], ograds[l]) < 5 * TOL, (l, _rel(grads[l], ograds[l]))
    # finite differences of the FP64 loss at two weights of each layer
    eps = 1e-5
    for l, idx in ((0, (1, 3, 0, 2, 2)), (1, (0, 0, 0, 1, 1)), (2, (5, 0, 4, 0, 3))):
        Wp = [w.copy() for w in Ws]
        Wm = [w.copy() for w in Ws]
        Wp[l][idx] += eps
        Wm[l][idx] -= eps
        fd = (po.loss_and_grads(O, po.Net(Wp), host)[0] - po.loss_and_grads(O, po.Net(Wm), host)[0]) / (2 * eps)
        scale = np.abs(ograds[l]).max()
        assert abs(2 * grads[l][idx].real - fd) <= 0.1 * scale + 1e-9, (l, idx, 2 * grads[l][idx].real, fd)


def test_network_is_gauge_equivariant_on_the_gpu():
    from yahmc_b200 import Ptc, fields
    from oracle import yahmc_oracle as yo
    lat, O, rng = make_pair("su3_fund_ap", (4, 4, 4, 4), seed=83)
    net = Ptc(lat, (1, 8, 8, 1))
    net.set_weights([_rand(rng, s) / np.sqrt(9 * s[2] * 4) for s in net.shapes()])
    r = source(O, rng)
    r[O.Vh:] = 0
    y = lat.field()
    net.apply(y, lat.field(r))
    y0 = lat.download(y)[:O.Vh]
    om = fields.haar_su(3, O.V, rng)
    Ut = np.einsum("xab,xmbc,xmdc->xmad", om, O.fund, np.conj(om[O.fw]))
    lat.set_links(Ut)
    rt = np.einsum("xab,xbs->xas", om, r)
    yt = lat.field()
    net.apply(yt, lat.field(rt))
    y1 = lat.download(yt)[:O.Vh]
    assert _rel(y1, np.einsum("xab,xbs->xas", om[:O.Vh], y0)) < TOL


def test_fgcr_meets_true_residual_and_falls_back_with_a_useless_network():
    from yahmc_b200 import Ptc
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=84)
    mass, prec = -0.4, 1e-22
    b = lat.field(source(O, rng))
    x0 = lat.field()
    st0 = lat.fgcr(mass, prec, x0, b, net=None)
    assert st0["status"] == 0 and st0["fallback"] == 0 and st0["true_residual"] < prec
    zero = Ptc(lat, (1, 8, 8, 1))                       # all weights zero: z = 0, no progress
    x1 = lat.field()
    st1 = lat.fgcr(mass, prec, x1, b, net=zero)
    assert st1["status"] == 0 and st1["fallback"] == 1 and st1["true_residual"] < prec
    lo, hi = O.default_range()
    a, c = lat.download(x0)[lo:hi], lat.download(x1)[lo:hi]
    assert _rel(c, a) < 1e-8


def test_trained_network_cuts_fgcr_iterations():
    """Ablation: the network, started from the first-order hopping expansion of the Schur
    inverse and trained on CG errors of this lattice's own solves, needs fewer flexible-GCR
    iterations than GCR without it (both stop on the same true residual)."""
    from yahmc_b200 import Ptc, heatbath, learned
    lat, O, rng = make_pair("su3_fund_ap", (8, 8, 8, 8), seed=85)
    U, _ = heatbath.thermalised_field((8, 8, 8, 8), 5.6, 30, 2)
    lat.set_links(U)
    mass, prec = -0.7, 1e-20
    b = lat.field(source(O, rng))
    plain = lat.fgcr(mass, prec, lat.field(), b, net=None)
    net = Ptc(lat, (1, 8, 8, 1))
    net.set_weights(learned.hopping_start(net.shapes(), mass, rng))
    start = lat.fgcr(mass, prec, lat.field(), b, net=net)
    pairs = learned.training_pairs(lat, mass, 3, rng, stops=(10, 25, 50, 100), random_pairs=2)
    hist = learned.train(net, pairs, steps=100, lr=1e-4, batch=4, rng=rng)
    assert np.mean(hist[-10:]) < np.mean(hist[:10])
    trained = lat.fgcr(mass, prec, lat.field(), b, net=net)
    for st in (plain, start, trained):
        assert st["status"] == 0 and st["fallback"] == 0 and st["true_residual"] < prec
    assert trained["iterations"] < plain["iterations"], (trained, start, plain)
