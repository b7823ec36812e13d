"""Training of the learned preconditioner (the gauge-covariant PTC network of yg_ptc_*).

The network N should approximate the inverse of the even-odd Schur operator D-hat (Dphi) on
the vectors a Krylov solver struggles with.  Training pairs (r, e) with D-hat e = r come from
solves the engine runs itself: for a source b, the CG iterates x_k of Hphi_sq x = b (CG from a
zero guess is deterministic, so x_k is the solve stopped after k iterations) give the errors
e_k = x - x_k, dominated by the low modes of D-hat^dag D-hat as k grows, and r_k = D-hat e_k.
The loss  sum_k |N(r_k) - e_k|^2 / |e_k|^2  and its gradient come from the engine's forward and
backward kernels (yg_ptc_gradient, BF16 tensor-core products with FP32 accumulation); the
weights (about 10^4 complex numbers) are updated on the host with Adam (Kingma and Ba, 2015)
on their real and imaginary parts.

The network starts as the identity (channel 0 passes the input through every layer) plus small
noise, so the untrained network is the unpreconditioned method.
"""
from __future__ import annotations

import numpy as np

from . import fields


# the reference's chiral gamma matrices (spinor.cpp:191-264), acting on the spin index
_I = 1j
GAMMA = np.array([
    [[0, 0, -1, 0], [0, 0, 0, -1], [-1, 0, 0, 0], [0, -1, 0, 0]],
    [[0, 0, 0, -_I], [0, 0, -_I, 0], [0, _I, 0, 0], [_I, 0, 0, 0]],
    [[0, 0, 0, -1], [0, 0, 1, 0], [0, 1, 0, 0], [-1, 0, 0, 0]],
    [[0, 0, -_I, 0], [0, 0, 0, _I], [_I, 0, 0, 0], [0, -_I, 0, 0]],
], dtype=complex)


def hopping_start(shapes, mass, rng, noise=0.0):
    """Weights of the first-order hopping expansion of the Schur inverse, an exact network of
    three layers: with the Wilson hop H = -1/2 sum_mu [(1 - g_mu) U_mu(x) T+ + (1 + g_mu) U_mu(x-mu)^dag T-]
    (dirac.cpp:258-697) and D-hat = A_ee - H A_oo^-1 H ~ (4+m) (1 - H^2 / (4+m)^2),
        D-hat^-1 ~ (1 / (4+m)) (1 + H_eo H_oe / (4+m)^2):
    layer 1 puts H psi in channel 0 and psi in channel 1, layer 2 applies H to channel 0 and
    passes channel 1, the last layer adds them with the weights above.  Other weights start at
    `noise` times Gaussian numbers."""
    if len(shapes) != 3:
        raise ValueError("the hopping start is a three-layer network")
    k = 4.0 + mass
    Ws = []
    for shp in shapes:
        W = noise * (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)) / np.sqrt(2 * 9 * 4 * shp[2])
        Ws.append(W)
    one = np.eye(4, dtype=complex)
    for l in (0, 1):
        for mu in range(4):
            Ws[l][1 + mu, 0, 0] = -0.5 * (one - GAMMA[mu])
            Ws[l][5 + mu, 0, 0] = -0.5 * (one + GAMMA[mu])
    Ws[0][0, 1, 0] = one
    Ws[1][0, 1, 1] = one
    Ws[2][0, 0, 1] = one / k
    Ws[2][0, 0, 0] = one / k ** 3
    return Ws


def near_identity(shapes, rng, noise=0.02):
    Ws = []
    for shp in shapes:
        W = noise * (rng.standard_normal(shp) + 1j * rng.standard_normal(shp)) / np.sqrt(2 * np.prod(shp[2:4]) * 9)
        W[0, 0, 0] += np.eye(4)
        Ws.append(W)
    return Ws


def training_pairs(lat, mass, nsrc, rng, stops=(10, 25, 50, 100, 200), prec=1e-20, random_pairs=1):
    """(r, e) field pairs on the even sites: CG errors at the given iteration counts for nsrc
    Gaussian sources, plus `random_pairs` Gaussian e per source."""
    pairs = []
    for _ in range(nsrc):
        b = lat.field(fields.gaussian_spinor(lat.V, lat.d, rng))
        xs = lat.field()
        lat.cg_inverter("Hphi_sq", mass, prec, xs, b)
        for k in stops:
            xk = lat.field()
            lat.cg_inverter("Hphi_sq", mass, prec, xk, b, maxiter=k)
            e = lat.field()
            lat.spinor_copy(e, xs)
            lat.spinor_sub_assign(e, xk)
            pairs.append(_pair(lat, mass, e))
        for _ in range(random_pairs):
            pairs.append(_pair(lat, mass, lat.field(fields.gaussian_spinor(lat.V, lat.d, rng))))
    return pairs


def _pair(lat, mass, e):
    """(D-hat e, e) with e restricted to the even sites."""
    from . import VIEW_ODD
    lat.spinor_mulr_assign(e, 0.0, view=VIEW_ODD)
    src = lat.field()
    lat.spinor_copy(src, e)
    r = lat.field()
    lat.Dphi(mass, r, src)
    return r, e


class Adam:
    def __init__(self, Ws, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps
        self.m = [np.zeros_like(W) for W in Ws]
        self.v = [np.zeros(W.shape) for W in Ws]
        self.t = 0

    def step(self, Ws, grads):
        self.t += 1
        out = []
        for W, g, m, v in zip(Ws, grads, self.m, self.v):
            gr = 2.0 * g                                # d loss / d Re + i d loss / d Im
            m *= self.b1
            m += (1 - self.b1) * gr
            v *= self.b2
            v += (1 - self.b2) * (gr.real ** 2 + gr.imag ** 2)
            mh = m / (1 - self.b1 ** self.t)
            vh = v / (1 - self.b2 ** self.t)
            out.append(W - self.lr * mh / (np.sqrt(vh) + self.eps))
        return out


class ResidualLoss:
    """L(v) = |D-hat N(v) - v|^2 / |v|^2: the network as a right preconditioner, D-hat N close to
    the identity.  Its gradient with respect to conj(N(v)) is D-hat^dag (D-hat N(v) - v) / |v|^2
    with D-hat^dag = gamma5 D-hat gamma5 (Hphi = gamma5 D-hat is Hermitian)."""

    def __init__(self, lat, mass):
        self.lat, self.mass = lat, mass
        self.y, self.s, self.w, self.t = lat.field(), lat.field(), lat.field(), lat.field()

    def __call__(self, net, v):
        lat, m = self.lat, self.mass
        net.apply(self.y, v)
        lat.spinor_copy(self.s, self.y)
        lat.Dphi(m, self.w, self.s)
        lat.spinor_sub_assign(self.w, v)                 # d = D N v - v
        nv = lat.spinor_sqnorm(v)
        loss = lat.spinor_sqnorm(self.w) / nv
        lat.spinor_g5(self.w)
        lat.Dphi(m, self.t, self.w)
        lat.spinor_g5(self.t)
        lat.spinor_mulr_assign(self.t, 1.0 / nv)        # gout = D^dag d / |v|^2
        return loss, net.backward(v, self.t)


def train_residual(net, lat, mass, vectors, steps=200, lr=5e-3, batch=4, rng=None, log=None):
    """Adam on the right-preconditioner loss over mini-batches of source vectors."""
    rng = rng or np.random.default_rng(0)
    lossf = ResidualLoss(lat, mass)
    Ws = net.get_weights()
    opt = Adam(Ws, lr=lr)
    hist = []
    for s in range(steps):
        idx = rng.choice(len(vectors), size=min(batch, len(vectors)), replace=False)
        tot, gsum = 0.0, None
        for i in idx:
            l, g = lossf(net, vectors[i])
            tot += l
            gsum = g if gsum is None else [a + b for a, b in zip(gsum, g)]
        Ws = opt.step(Ws, gsum)
        net.set_weights(Ws)
        hist.append(tot / len(idx))
        if log is not None and (s % max(1, steps // 10) == 0 or s == steps - 1):
            log(f"step {s}: loss {hist[-1]:.4f}")
    return hist


def train(net, pairs, steps=100, lr=2e-3, batch=4, rng=None, log=None):
    """Adam on the network's weights over mini-batches of the pairs; returns the loss history
    (mean per pair)."""
    rng = rng or np.random.default_rng(0)
    Ws = net.get_weights()
    opt = Adam(Ws, lr=lr)
    hist = []
    for s in range(steps):
        idx = rng.choice(len(pairs), size=min(batch, len(pairs)), replace=False)
        loss, grads = net.gradient([pairs[i] for i in idx])
        Ws = opt.step(Ws, grads)
        net.set_weights(Ws)
        hist.append(loss / len(idx))
        if log is not None and (s % max(1, steps // 10) == 0 or s == steps - 1):
            log(f"step {s}: loss {hist[-1]:.4f}")
    return hist
