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
