"""Quenched SU(3) gauge fields on the host: Cabibbo-Marinari heatbath (numpy, no device code).

Used to make synthetic benchmark inputs that every process can regenerate bit for bit on
the same machine without the engine: a thermalised Wilson-action field at a given beta,
built on a small periodic lattice and tiled onto the benchmark lattice.

One sweep updates every link once: for each direction mu and site parity p (links of one
direction and one parity never appear in each other's staples), the staple sum A of the
Wilson action S = -(beta/N) sum Re tr(U A) is formed, and the link is multiplied from the
left by an SU(2) element in each of the three SU(2) subgroups of SU(3) in turn (Cabibbo and
Marinari, Phys. Lett. B 119 (1982) 387).  The SU(2) element is drawn from its exact
conditional distribution by the Kennedy-Pendleton algorithm (Phys. Lett. B 156 (1985) 393):
for the subgroup block w of U A, projected onto k v with v in SU(2), x = r v is sampled with
density sqrt(1 - x0^2) exp(2 beta k x0 / N), and r = x v^dagger.  Each heatbath sweep is
followed by `n_or` overrelaxation sweeps (r = (v^dagger)^2, which leaves the action
unchanged; Brown and Woch, Phys. Rev. Lett. 58 (1987) 2394).

The equilibrium distribution is the same as that of pure-gauge HMC at the same beta (the
reference's update() with a gauge monomial only); the sample path is not.
"""
from __future__ import annotations

import numpy as np

NC = 3
SUBGROUPS = ((0, 1), (0, 2), (1, 2))


def _mm(a, b):
    return np.matmul(a, b)


def _dag(a):
    return np.conj(np.swapaxes(a, -1, -2))


class Heatbath:
    """Wilson-action SU(3) heatbath on a periodic T x X x Y x Z lattice (all extents even)."""

    def __init__(self, dims, beta, seed, n_or=2):
        self.dims = tuple(int(d) for d in dims)
        if any(d % 2 for d in self.dims):
            raise ValueError("extents must be even")
        self.beta = float(beta)
        self.n_or = int(n_or)
        self.rng = np.random.default_rng(seed)
        T, X, Y, Z = self.dims
        self.V = T * X * Y * Z
        t, x, y, z = np.meshgrid(np.arange(T), np.arange(X), np.arange(Y), np.arange(Z), indexing="ij")
        coords = (t.ravel(), x.ravel(), y.ravel(), z.ravel())
        self.lex = lambda c: ((c[0] % T * X + c[1] % X) * Y + c[2] % Y) * Z + c[3] % Z
        self.parity = (coords[0] + coords[1] + coords[2] + coords[3]) % 2
        unit = np.zeros(4, dtype=int)
        self.fw = np.empty((4, self.V), dtype=np.int64)
        self.bk = np.empty((4, self.V), dtype=np.int64)
        for mu in range(4):
            e = unit.copy()
            e[mu] = 1
            self.fw[mu] = self.lex([c + e[i] for i, c in enumerate(coords)])
            self.bk[mu] = self.lex([c - e[i] for i, c in enumerate(coords)])
        self.sites = [np.nonzero(self.parity == p)[0] for p in (0, 1)]
        # cold start: unit links, shape (V, 4, 3, 3), lexicographic site order
        self.U = np.broadcast_to(np.eye(NC, dtype=complex), (self.V, 4, NC, NC)).copy()

    # ---- staples
    def staple_sum(self, mu, s):
        """A(x) for the links U_mu(x), x in the index array s: the sum over nu != mu of the
        forward and backward staples, so that Re tr(U_mu(x) A(x)) is the link's part of the
        plaquette sum."""
        U = self.U
        A = np.zeros((len(s), NC, NC), dtype=complex)
        xmu = self.fw[mu][s]
        for nu in range(4):
            if nu == mu:
                continue
            xnu = self.fw[nu][s]
            xmnu = self.bk[nu][s]
            xmunu = self.bk[nu][xmu]
            # U_nu(x+mu) U_mu(x+nu)^dag U_nu(x)^dag
            A += _mm(_mm(U[xmu, nu], _dag(U[xnu, mu])), _dag(U[s, nu]))
            # U_nu(x+mu-nu)^dag U_mu(x-nu)^dag U_nu(x-nu)
            A += _mm(_mm(_dag(U[xmunu, nu]), _dag(U[xmnu, mu])), U[xmnu, nu])
        return A

    # ---- SU(2) subgroup pieces
    @staticmethod
    def _project(W, i, j):
        """Quaternion part of the (i, j) block of W: alpha, beta with w~ = [[a, b], [-b*, a*]]."""
        a = 0.5 * (W[:, i, i] + np.conj(W[:, j, j]))
        b = 0.5 * (W[:, i, j] - np.conj(W[:, j, i]))
        return a, b

    def _kp_x0(self, a):
        """x0 with density sqrt(1 - x0^2) exp(a x0) (Kennedy-Pendleton), vectorised with
        per-element retries."""
        n = a.shape[0]
        x0 = np.empty(n)
        todo = np.arange(n)
        rng = self.rng
        while todo.size:
            r1 = 1.0 - rng.random(todo.size)
            r2 = rng.random(todo.size)
            r3 = 1.0 - rng.random(todo.size)
            r4 = rng.random(todo.size)
            lam2 = -(np.log(r1) + np.cos(2 * np.pi * r2) ** 2 * np.log(r3)) / (2.0 * a[todo])
            ok = r4 * r4 <= 1.0 - lam2
            x0[todo[ok]] = 1.0 - 2.0 * lam2[ok]
            todo = todo[~ok]
        return x0

    def _sphere(self, n):
        c = 2.0 * self.rng.random(n) - 1.0
        phi = 2.0 * np.pi * self.rng.random(n)
        s = np.sqrt(1.0 - c * c)
        return s * np.cos(phi), s * np.sin(phi), c

    def _apply_left(self, s, mu, i, j, ra, rb):
        """U_mu(x) <- R U_mu(x), R the SU(3) embedding of [[ra, rb], [-rb*, ra*]] at (i, j)."""
        U = self.U[s, mu]
        ri = ra[:, None] * U[:, i, :] + rb[:, None] * U[:, j, :]
        rj = -np.conj(rb)[:, None] * U[:, i, :] + np.conj(ra)[:, None] * U[:, j, :]
        U[:, i, :] = ri
        U[:, j, :] = rj
        self.U[s, mu] = U

    def _update(self, mu, p, overrelax):
        s = self.sites[p]
        A = self.staple_sum(mu, s)
        for i, j in SUBGROUPS:
            W = _mm(self.U[s, mu], A)
            a, b = self._project(W, i, j)
            k = np.sqrt(np.abs(a) ** 2 + np.abs(b) ** 2)
            k = np.maximum(k, 1e-300)
            va, vb = a / k, b / k                      # v = [[va, vb], [-vb*, va*]]
            # v^dagger = [[va*, -vb], [vb*, va]]
            if overrelax:
                # r = (v^dagger)^2
                ra = np.conj(va) * np.conj(va) - vb * np.conj(vb)
                rb = -np.conj(va) * vb - vb * va
            else:
                x0 = self._kp_x0(2.0 * self.beta * k / NC)
                n1, n2, n3 = self._sphere(len(s))
                rad = np.sqrt(np.maximum(1.0 - x0 * x0, 0.0))
                xa = x0 + 1j * rad * n3                # x = x0 + i x.sigma = [[xa, xb], [-xb*, xa*]]
                xb = rad * (n2 + 1j * n1)
                # r = x v^dagger
                ra = xa * np.conj(va) + xb * np.conj(vb)
                rb = -xa * vb + xb * va
            self._apply_left(s, mu, i, j, ra, rb)

    def reunitarize(self):
        """Gram-Schmidt on the rows, third row = conj(row0 x row1): keeps rounding from
        accumulating over many sweeps."""
        U = self.U
        r0 = U[..., 0, :]
        r0 = r0 / np.linalg.norm(r0, axis=-1, keepdims=True)
        r1 = U[..., 1, :]
        r1 = r1 - np.sum(np.conj(r0) * r1, axis=-1, keepdims=True) * r0
        r1 = r1 / np.linalg.norm(r1, axis=-1, keepdims=True)
        r2 = np.conj(np.cross(r0, r1))
        self.U = np.stack([r0, r1, r2], axis=-2)

    def sweep(self):
        for mu in range(4):
            for p in (0, 1):
                self._update(mu, p, overrelax=False)
        for _ in range(self.n_or):
            for mu in range(4):
                for p in (0, 1):
                    self._update(mu, p, overrelax=True)
        self.reunitarize()

    def plaquette(self):
        """Average of Re tr(U_p)/N over all plaquettes (avr_wilson(1, 1))."""
        U = self.U
        tot = 0.0
        for mu in range(4):
            for nu in range(mu + 1, 4):
                P = _mm(_mm(U[:, mu], U[self.fw[mu], nu]), _mm(_dag(U[self.fw[nu], mu]), _dag(U[:, nu])))
                tot += np.trace(P, axis1=-2, axis2=-1).real.sum()
        return tot / (6 * self.V * NC)

    def links_eo(self):
        """The links in the reference's even-odd site order id = (parity V + lex)/2, shape
        (V, 4, 3, 3)."""
        lex = np.arange(self.V)
        ids = (self.parity * self.V + lex) // 2
        out = np.empty_like(self.U)
        out[ids] = self.U
        return out


def thermalised_field(dims, beta, sweeps, seed, n_or=2):
    """(links in even-odd site order, plaquette history) after `sweeps` heatbath sweeps from
    a cold start."""
    hb = Heatbath(dims, beta, seed, n_or=n_or)
    hist = []
    for _ in range(sweeps):
        hb.sweep()
        hist.append(hb.plaquette())
    return hb.links_eo(), hist
