"""FP64 restatement of the learned preconditioner (test infrastructure).

The preconditioner has no counterpart in the reference; this file restates, in plain
numpy and double precision, what the engine's CUDA kernels compute, so that the tests can
check them:

* the gauge-covariant parallel-transport convolution ("PTC") layer
      out[x, o] = sum_p sum_i W[p, o, i] (T_p in_i)(x),
  with nine paths p (0 the site itself, 1..4 a hop forward along mu = p - 1, 5..8 a hop
  backward along mu = p - 5), T_p the parallel transport through the represented links the
  Dirac operator uses (antiperiodic sign included)
      (T_{mu+} f)(x) = U_mu(x) f(x + mu),   (T_{mu-} f)(x) = U_mu(x - mu)^dag f(x - mu),
  and W[p, o, i] a complex 4x4 matrix on the spin index (o output channel, i input channel);
  the colour index only ever meets the links, so the layer commutes with gauge
  transformations exactly;
* its adjoint (the gradient with respect to the layer input): the same layer with the
  weights conjugate-transposed in (spin, channel) and every path reversed, since
  T_{mu+}^dag = T_{mu-};
* the weight gradient  dW[p, o, i][s, s'] = sum_{x, c} g[x, o, c, s] conj((T_p in_i)[x, c, s'])
  (the derivative of a real loss with respect to conj(W));
* the network: layers with channels 1 -> C -> ... -> 1, no nonlinearity (the target, the
  inverse of the even-odd operator, is linear); on the even-odd system an even-site vector
  is embedded in the whole lattice with zero odd sites and the output's even sites are kept
  (the even-even block of D^-1 is the inverse of the Schur operator);
* the loss  L = sum_k |N(r_k) - e_k|^2 / |e_k|^2  over pairs with D-hat e_k = r_k;
* flexible GCR (right preconditioned, restarted) on the Schur operator Dphi with the
  reference's squared relative residual as the stopping rule.

Field layout: (V, C, d, 4) complex, sites in the reference's order (the oracle's).
"""
from __future__ import annotations

import numpy as np

NPATH = 9


def opposite(p: int) -> int:
    return 0 if p == 0 else (p + 4 if p <= 4 else p - 4)


def transport(O, f: np.ndarray, p: int) -> np.ndarray:
    """T_p f for a field f (V, C, d, 4) with the oracle's represented links O.links (V, 4, d, d)."""
    if p == 0:
        return f
    if p <= 4:
        mu = p - 1
        return np.einsum("xab,xcbs->xcas", O.links[:, mu], f[O.fw[:, mu]])
    mu = p - 5
    b = O.bk[:, mu]
    return np.einsum("xba,xcbs->xcas", np.conj(O.links[b, mu]), f[b])


def layer(O, W: np.ndarray, f: np.ndarray) -> np.ndarray:
    """W (9, Co, Ci, 4, 4) complex; f (V, Ci, d, 4) -> (V, Co, d, 4)."""
    out = np.zeros((f.shape[0], W.shape[1], f.shape[2], 4), dtype=complex)
    for p in range(NPATH):
        out += np.einsum("oist,xict->xocs", W[p], transport(O, f, p))
    return out


def adjoint_weights(W: np.ndarray) -> np.ndarray:
    """Weights of the adjoint layer: W'[p', i, o] = W[p, o, i]^dag with p' = opposite(p)."""
    Wa = np.zeros((NPATH, W.shape[2], W.shape[1], 4, 4), dtype=complex)
    for p in range(NPATH):
        Wa[opposite(p)] = np.conj(np.transpose(W[p], (1, 0, 3, 2)))
    return Wa


def layer_adjoint(O, W: np.ndarray, g: np.ndarray) -> np.ndarray:
    return layer(O, adjoint_weights(W), g)


def weight_grad(O, g: np.ndarray, f: np.ndarray) -> np.ndarray:
    """dL/dconj(W) for out = layer(W, f) and g = dL/dconj(out)."""
    G = np.zeros((NPATH, g.shape[1], f.shape[1], 4, 4), dtype=complex)
    for p in range(NPATH):
        G[p] = np.einsum("xocs,xict->oist", g, np.conj(transport(O, f, p)))
    return G


class Net:
    """Linear PTC network: a list of weight arrays, channels 1 -> C -> ... -> 1."""

    def __init__(self, Ws):
        self.W = [np.array(w, dtype=complex) for w in Ws]

    @staticmethod
    def init(channels, rng, scale=None):
        Ws = []
        for ci, co in zip(channels[:-1], channels[1:]):
            s = scale if scale is not None else 1.0 / np.sqrt(NPATH * ci * 4)
            Ws.append(s * (rng.standard_normal((NPATH, co, ci, 4, 4)) + 1j * rng.standard_normal((NPATH, co, ci, 4, 4)))
                      / np.sqrt(2))
        return Net(Ws)

    @staticmethod
    def near_identity(channels, rng, noise=0.05):
        """Channel 0 passes the input through each layer (W[0][0, 0] = 1 on spin), plus noise."""
        net = Net.init(channels, rng, scale=noise)
        for W in net.W:
            W[0, 0, 0] += np.eye(4)
        return net

    def forward(self, O, f: np.ndarray, keep=False):
        acts = [f]
        for W in self.W:
            acts.append(layer(O, W, acts[-1]))
        return (acts[-1], acts) if keep else acts[-1]

    def backward(self, O, acts, g: np.ndarray):
        """Weight gradients for dL/dconj(output) = g."""
        grads = [None] * len(self.W)
        for l in range(len(self.W) - 1, -1, -1):
            grads[l] = weight_grad(O, g, acts[l])
            if l > 0:
                g = layer_adjoint(O, self.W[l], g)
        return grads


def embed_even(O, r_even: np.ndarray) -> np.ndarray:
    """An even-site spinor (Vh, d, 4) as a one-channel whole-lattice field (V, 1, d, 4)."""
    f = np.zeros((O.V, 1, O.d, 4), dtype=complex)
    f[:O.Vh, 0] = r_even
    return f


def apply_even(O, net: Net, r_even: np.ndarray) -> np.ndarray:
    return net.forward(O, embed_even(O, r_even))[:O.Vh, 0]


def loss_and_grads(O, net: Net, pairs):
    """L = sum_k |N(r_k) - e_k|^2 / |e_k|^2 over (r_k, e_k) even-site pairs, and dL/dconj(W)."""
    L = 0.0
    grads = [np.zeros_like(w) for w in net.W]
    for r, e in pairs:
        y, acts = net.forward(O, embed_even(O, r), keep=True)
        d = y[:O.Vh, 0] - e
        n = float(np.vdot(e, e).real)
        L += float(np.vdot(d, d).real) / n
        g = np.zeros_like(y)
        g[:O.Vh, 0] = d / n
        for acc, gw in zip(grads, net.backward(O, acts, g)):
            acc += gw
    return L, grads


def dhat(O, mass: float, v_even: np.ndarray) -> np.ndarray:
    """The even-odd Schur operator Dphi (dirac.cpp:738-751) on an even-site vector."""
    src = O.new_field()
    src[:O.Vh] = v_even
    dst = O.new_field()
    O.Dphi(mass, dst, src)
    return dst[:O.Vh].copy()


def fgcr(O, mass: float, prec: float, b_even: np.ndarray, precond, restart: int = 16, maxiter: int = 2000):
    """Right-preconditioned flexible GCR for Dphi x = b on the even sites, from x = 0: z = M r,
    w = D z orthogonalised against the previous w (the same combination applied to z), then
    x += a z, r -= a w with a = <w, r> / <w, w>.  Stops on |r|^2 < prec |b|^2 (recursive
    residual, checked against the true one at the end).  Returns (x, iterations)."""
    x = np.zeros_like(b_even)
    r = b_even.copy()
    target = prec * float(np.vdot(b_even, b_even).real)
    it = 0
    Z, Wv = [], []
    while it < maxiter:
        if float(np.vdot(r, r).real) < target:
            break
        z = precond(r)
        w = dhat(O, mass, z)
        for zj, wj in zip(Z, Wv):
            beta = np.vdot(wj, w) / np.vdot(wj, wj)
            w = w - beta * wj
            z = z - beta * zj
        a = np.vdot(w, r) / np.vdot(w, w)
        x = x + a * z
        r = r - a * w
        Z.append(z)
        Wv.append(w)
        if len(Z) >= restart:
            Z, Wv = [], []
            r = b_even - dhat(O, mass, x)
        it += 1
    return x, it
