"""CPU oracle: a numpy restatement of YaHMC's fermion hot path.

TEST INFRASTRUCTURE.  Only tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of bench.py may import this module, and only as the
checker: the product (yahmc_b200) never imports, links or calls it.

Pinning.  tests/test_oracle_pinning.py checks every function here against the
unmodified reference compiled from its own sources (oracle/_ref, built by
oracle/build_ref.py) on seeded 8^4 inputs, and tests/test_oracle_golden.py
checks it against the committed golden vectors in tests/golden/ that
tests/golden/make_golden.py generated from that same compiled reference.
The reference ships no golden vectors or fixtures of its own; its runtime
self-checks (checks/*.cpp) are restated as tests too.

Every function cites the reference file:line it restates (paths within the
reference project).  Floating-point results agree with the reference to
rounding (the summation order differs), i.e. to ~1e-15 relative.

Data layouts (the reference's own, as complex numpy arrays):
  spinor field   (V, d, 4)        Spinor{re[d][4], im[d][4]}   include/spinor.h:7-9
  links          (V, 4, d, d)     gfield_repr[4*id+mu]        include/gaugefield.h:9-10
  fund links     (V, 4, N, N)     gfield_fund[4*id+mu]        include/gaugefield.h:6-7
  clover term    (V, 4, d, d)     cl_term[4*id+mu]            include/clover.h:12-13
  clover force   (V, 6, d, d)     cl_force[6*id+mu]           include/clover.h:15-16
  LDL factors    (V, 2, P)        cl_ldl[id].upper/lower       include/clover.h:24-33, P = d(2d+1)
  momenta        (V, 4, NG) real  afield_momenta[4*id+mu]     include/gaugefield.h:12-13
Site index: even-odd order (geometry.cpp:756-878, single rank): lex =
((t*X+x)*Y+y)*Z+z, parity p = (t+x+y+z)%2, id = (p*V+lex)//2 with even-odd
preconditioning and id = lex without it.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

SQRT2 = math.sqrt(2.0)
TF = 2.0                     # include/repr.h:4-6
EVEN, ODD, BOTH = 1, 2, 3    # include/global.h:11-13
BC_NAMES = ("periodic", "antiperiodic", "open", "sf")
REPR_NAMES = ("fundamental", "adjoint", "symmetric", "antisymmetric")   # REPR_ID order, repr.h:9-39


def repr_dim(nc: int, rep: str) -> int:
    """REPR_DIM, include/repr.h:9-39."""
    return {"fundamental": nc, "adjoint": nc * nc - 1,
            "symmetric": nc * (nc + 1) // 2, "antisymmetric": nc * (nc - 1) // 2}[rep]


# ---------------------------------------------------------------- raw layouts
def spinor_from_raw(raw: np.ndarray, d: int) -> np.ndarray:
    r = np.asarray(raw, dtype=np.float64).reshape(-1, 2, d, 4)
    return r[:, 0] + 1j * r[:, 1]


def spinor_to_raw(s: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(np.stack([s.real, s.imag], axis=1)).reshape(-1)


def mat_from_raw(raw: np.ndarray, n: int) -> np.ndarray:
    r = np.asarray(raw, dtype=np.float64).reshape(-1, 2, n, n)
    return r[:, 0] + 1j * r[:, 1]


def mat_to_raw(m: np.ndarray) -> np.ndarray:
    m = np.asarray(m).reshape(-1, m.shape[-2], m.shape[-1])
    return np.ascontiguousarray(np.stack([m.real, m.imag], axis=1)).reshape(-1)


# ---------------------------------------------------------------- gamma matrices
def _spin_matrices():
    """Chiral basis of spinor.cpp:191-264 as 4x4 matrices acting on the spin index."""
    i = 1j
    g = np.zeros((4, 4, 4), dtype=complex)
    g[0] = [[0, 0, -1, 0], [0, 0, 0, -1], [-1, 0, 0, 0], [0, -1, 0, 0]]           # gamma0 :191-205
    g[1] = [[0, 0, 0, -i], [0, 0, -i, 0], [0, i, 0, 0], [i, 0, 0, 0]]               # gamma1 :207-221
    g[2] = [[0, 0, 0, -1], [0, 0, 1, 0], [0, 1, 0, 0], [-1, 0, 0, 0]]               # gamma2 :223-237
    g[3] = [[0, 0, -i, 0], [0, 0, 0, i], [i, 0, 0, 0], [0, -i, 0, 0]]               # gamma3 :239-253
    g5 = np.diag([1, 1, -1, -1]).astype(complex)                                  # gamma5 :255-264
    return g, g5


GAMMA, GAMMA5 = _spin_matrices()
ONE4 = np.eye(4, dtype=complex)


def _g5_sigma_matrices():
    """Spinor::g5_sigma(mu,nu) for mu<nu, spinor.cpp:266-438."""
    i = 1j
    s = {}
    s[(0, 1)] = -i * np.array([[0, 1, 0, 0], [1, 0, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]])   # :270-282
    s[(0, 2)] = np.array([[0, -1, 0, 0], [1, 0, 0, 0], [0, 0, 0, -1], [0, 0, 1, 0]])       # :298-310
    s[(1, 2)] = np.diag([i, -i, -i, i])                                                     # :354-366
    s[(0, 3)] = np.diag([-i, i, -i, i])                                                     # :326-338
    s[(1, 3)] = np.array([[0, -1, 0, 0], [1, 0, 0, 0], [0, 0, 0, 1], [0, 0, -1, 0]])       # :382-394
    s[(2, 3)] = np.array([[0, i, 0, 0], [i, 0, 0, 0], [0, 0, 0, -i], [0, 0, -i, 0]])       # :410-422
    return {k: np.asarray(v, dtype=complex) for k, v in s.items()}


G5_SIGMA = _g5_sigma_matrices()
# clover-force slot order of clover_fermion_force, forces.cpp:130-170
CLOVER_PAIRS = [(0, 1), (0, 2), (1, 2), (0, 3), (1, 3), (2, 3)]


def spin_apply(m: np.ndarray, s: np.ndarray) -> np.ndarray:
    """(m psi)_s = sum_t m[s,t] psi_t for psi of shape (..., d, 4)."""
    return np.einsum("st,...it->...is", m, s)


def col_apply(u: np.ndarray, s: np.ndarray) -> np.ndarray:
    """suNf * Spinor, spinor.cpp:20-79: colour matrix on the colour index."""
    return np.einsum("...ij,...js->...is", u, s)


def dagger(u: np.ndarray) -> np.ndarray:
    return np.conj(np.swapaxes(u, -1, -2))


# ---------------------------------------------------------------- group / representation
def su_generator(nc: int, alg: np.ndarray) -> np.ndarray:
    """suNg(suNa&): anti-Hermitian matrix from algebra coordinates, suNg.cpp:15-58.

    alg has shape (..., NG); returns (..., N, N) complex."""
    alg = np.asarray(alg, dtype=float)
    out = np.zeros(alg.shape[:-1] + (nc, nc), dtype=complex)
    n = 0
    for i in range(nc):
        for j in range(nc):
            if i > j:
                out[..., i, j] += 1j * alg[..., n]
                out[..., j, i] += 1j * alg[..., n]
                n += 1
            elif i < j:
                out[..., i, j] += alg[..., n]
                out[..., j, i] -= alg[..., n]
                n += 1
            elif i > 0:
                v = math.sqrt(2.0 / (i * (i + 1)))
                for k in range(i):
                    out[..., k, k] += 1j * v * alg[..., n]
                out[..., i, i] -= 1j * i * v * alg[..., n]
                n += 1
    return out


def repr_basis(nc: int, rep: str) -> np.ndarray:
    """basis[] of repr_init, repr.cpp:25-59."""
    d = repr_dim(nc, rep)
    b = np.zeros((d, nc, nc), dtype=complex)
    if rep == "symmetric":
        n = 0
        for i in range(nc):
            for j in range(i + 1):
                if i == j:
                    b[n, i, i] = 1
                else:
                    b[n, i, j] = b[n, j, i] = 1 / SQRT2
                n += 1
    elif rep == "antisymmetric":
        n = 0
        for i in range(nc):
            for j in range(i):
                b[n, j, i] = 1 / SQRT2
                b[n, i, j] = -1 / SQRT2
                n += 1
    elif rep == "adjoint":
        ng = nc * nc - 1
        for n in range(ng):
            e = np.zeros(ng)
            e[n] = 1
            b[n] = (-1j / SQRT2) * su_generator(nc, e)
    return b


def generators(nc: int, rep: str):
    """iTfund / iTrepr, repr.cpp:61-104.  Returns (NG,N,N), (NG,d,d)."""
    ng = nc * nc - 1
    tf = su_generator(nc, np.eye(ng))
    if rep == "fundamental":
        return tf, tf.copy()
    b = repr_basis(nc, rep)
    bt = np.swapaxes(b, -1, -2)
    tr = np.zeros((ng, b.shape[0], b.shape[0]), dtype=complex)
    for k in range(ng):
        t = tf[k]
        for i in range(b.shape[0]):
            for j in range(b.shape[0]):
                if rep == "adjoint":
                    m = b[j] @ b[i] @ t + b[i] @ b[j] @ dagger(t)
                elif rep == "symmetric":
                    m = b[j] @ b[i] @ t + b[i] @ b[j] @ t.T
                else:
                    m = b[j] @ bt[i] @ t + bt[i] @ b[j] @ t.T
                tr[k, i, j] = np.trace(m)
    return tf, tr


def represent(u: np.ndarray, nc: int, rep: str) -> np.ndarray:
    """represent_links fund -> fermion representation, repr.cpp:107-263.

    Fundamental: copy.  Symmetric / antisymmetric: the 2x2 minors with the
    sqrt(2) factors of repr.cpp:114-160.  Adjoint: R_nm = tr(b_n U b_m U^dag)
    in the Hermitian orthonormal basis b of repr.cpp:52-59, which is what the
    explicit real formulas of repr.cpp:162-259 evaluate (imaginary part 0)."""
    u = np.asarray(u)
    if rep == "fundamental":
        return u.copy()
    d = repr_dim(nc, rep)
    out = np.zeros(u.shape[:-2] + (d, d), dtype=complex)
    if rep == "antisymmetric":
        pairs = [(i, j) for i in range(1, nc) for j in range(i)]
        for n, (i, j) in enumerate(pairs):
            for m, (k, l) in enumerate(pairs):
                out[..., n, m] = u[..., i, k] * u[..., j, l] - u[..., i, l] * u[..., j, k]
    elif rep == "symmetric":
        pairs = [(i, j) for i in range(nc) for j in range(i + 1)]
        for n, (i, j) in enumerate(pairs):
            for m, (k, l) in enumerate(pairs):
                if i == j and k == l:
                    out[..., n, m] = u[..., i, k] * u[..., j, l]
                elif i == j or k == l:
                    out[..., n, m] = SQRT2 * u[..., i, k] * u[..., j, l]
                else:
                    out[..., n, m] = u[..., i, k] * u[..., j, l] + u[..., i, l] * u[..., j, k]
    else:
        b = repr_basis(nc, rep)
        ud = dagger(u)
        for n in range(d):
            lhs = np.einsum("ab,...bc->...ac", b[n], u)
            for m in range(d):
                rhs = np.einsum("ab,...bc->...ac", b[m], ud)
                out[..., n, m] = np.einsum("...ab,...ba->...", lhs, rhs).real
    return out


def exp_algebra(nc: int, alg: np.ndarray, coeff: float = 1.0) -> np.ndarray:
    """exp(suNa, coeff): Taylor series then reunitarize, suNa.cpp:113-134.  Each matrix adds
    terms (coeff/k) X^k / ... until the last added term has squared norm <= 1e-24, exactly
    as the reference's loop does per matrix (the batch keeps a mask of unfinished ones)."""
    x = su_generator(nc, alg)
    xk = np.broadcast_to(np.eye(nc, dtype=complex), x.shape).copy()
    ret = xk.copy()
    active = np.ones(x.shape[:-2], dtype=bool)
    k = 1
    while np.any(active):
        xk = (coeff / k) * (xk @ x)
        ret[active] += xk[active]
        err = np.sum(np.abs(xk) ** 2, axis=(-1, -2))
        active &= err > 1e-24
        k += 1
    return reunitarize(ret)


def reunitarize(u: np.ndarray) -> np.ndarray:
    """suNg::reunitarize, suNg.cpp:171-359: Gram-Schmidt on the rows; SU(2)/SU(3) build the
    last row from the others, larger N fix det=1 by a phase on the last row."""
    u = np.array(u, dtype=complex, copy=True)
    nc = u.shape[-1]
    if nc == 2:
        r0 = u[..., 0, :] / np.linalg.norm(u[..., 0, :], axis=-1, keepdims=True)
        u[..., 0, :] = r0
        u[..., 1, 0] = -np.conj(r0[..., 1])
        u[..., 1, 1] = np.conj(r0[..., 0])
        return u
    if nc == 3:
        r0 = u[..., 0, :] / np.linalg.norm(u[..., 0, :], axis=-1, keepdims=True)
        r1 = u[..., 1, :]
        c = np.sum(np.conj(r0) * r1, axis=-1, keepdims=True)
        r1 = r1 - c * r0
        r1 = r1 / np.linalg.norm(r1, axis=-1, keepdims=True)
        u[..., 0, :] = r0
        u[..., 1, :] = r1
        u[..., 2, :] = np.conj(np.cross(r0, r1))
        return u
    for i in range(nc):
        u[..., i, :] /= np.linalg.norm(u[..., i, :], axis=-1, keepdims=True)
        for j in range(i + 1, nc):
            c = np.sum(np.conj(u[..., i, :]) * u[..., j, :], axis=-1, keepdims=True)
            u[..., j, :] -= c * u[..., i, :]
    det = np.linalg.det(u)
    ph = np.exp(-1j * np.angle(det))
    u[..., nc - 1, :] *= ph[..., None]
    return u


def algebra_project(m: np.ndarray, gens: np.ndarray, coeff) -> np.ndarray:
    """algebra_project(suNf&/suNg&, coeff): av[a] = coeff/(-TF) * Re tr(iT[a] m), suNa.cpp:91-111."""
    c = np.asarray(coeff, dtype=float) / (-TF)
    tr = np.einsum("aik,...ki->...a", gens, m).real
    return c[..., None] * tr if np.ndim(c) else c * tr


# ---------------------------------------------------------------- lattice + operator
@dataclass
class Params:
    dims: tuple
    nc: int = 3
    rep: str = "fundamental"
    bc: str = "antiperiodic"
    clover: bool = True
    eo: bool = True
    csw: float = 1.0
    cf: float = 1.0


class Oracle:
    """Global state of one reference configuration: geometry (geometry.cpp), links
    (gaugefield.cpp, repr.cpp), boundary conditions (bcs.cpp) and clover term (clover.cpp)."""

    def __init__(self, p: Params):
        self.p = p
        T, X, Y, Z = p.dims
        self.dims = p.dims
        self.V = T * X * Y * Z
        self.Vh = self.V // 2
        self.nc = p.nc
        self.d = repr_dim(p.nc, p.rep)
        self.ng = p.nc * p.nc - 1
        self.itfund, self.itrepr = generators(p.nc, p.rep)
        self._geometry()
        self._bcs_init()
        self.fund = None
        self.links = None
        self.cl_term = None
        self.cl_force = np.zeros((self.V, 6, self.d, self.d), dtype=complex)
        self.mom = np.zeros((self.V, 4, self.ng))
        self._ldl_sigma = None
        self._ldl = None
        self.mvm = 0

    # ---- geometry.cpp:756-878 (no MPI: border 0) and 1161-1187
    def index(self, t, x, y, z):
        T, X, Y, Z = self.dims
        lex = ((t * X + x) * Y + y) * Z + z
        if not self.p.eo:
            return lex
        par = (t + x + y + z) % 2
        return (par * self.V + lex) // 2

    def _geometry(self):
        T, X, Y, Z = self.dims
        t, x, y, z = np.meshgrid(np.arange(T), np.arange(X), np.arange(Y), np.arange(Z), indexing="ij")
        c = np.stack([t.ravel(), x.ravel(), y.ravel(), z.ravel()], axis=1)
        ids = self.index(*c.T)
        self.coord = np.zeros((self.V, 4), dtype=np.int64)
        self.coord[ids] = c
        L = np.array(self.dims)
        self.fw = np.zeros((self.V, 4), dtype=np.int64)
        self.bk = np.zeros((self.V, 4), dtype=np.int64)
        for mu in range(4):
            e = np.zeros(4, dtype=np.int64)
            e[mu] = 1
            f = (self.coord + e) % L
            b = (self.coord - e + L) % L
            self.fw[:, mu] = self.index(*f.T)
            self.bk[:, mu] = self.index(*b.T)
        self.t = self.coord[:, 0]

    def part_range(self, part):
        """spinor_select_even/odd/full, linalg.cpp:272-291.  The ranges are the two halves of
        the site index in either layout (without even-odd ordering they are simply the
        first and second half of the lexicographic order, as odd_sites_for in geometry.h:18-19)."""
        return {EVEN: (0, self.Vh), ODD: (self.Vh, self.V), BOTH: (0, self.V)}[part]

    def default_range(self):
        """spinor_type_default, linalg.cpp:321-328."""
        return self.part_range(EVEN) if self.p.eo else self.part_range(BOTH)

    # ---- bcs.cpp
    def _bcs_init(self):
        T = self.dims[0]
        bc = self.p.bc
        self.Ta = self.Tb = None
        self.spinor_zero_t = []
        if bc == "open":
            self.spinor_zero_t = [0, T - 1]               # listB, bcs.cpp:44-66, 139-146
            self.Ta, self.Tb = 1, T - 2                    # bcs.cpp:68-70
            self.clover_zero_t = [0, T - 1]                # clover.cpp:106-108
        elif bc == "sf":
            self.spinor_zero_t = [0, T - 2, T - 1]        # listA/B/C, bcs.cpp:148-163
            self.Ta, self.Tb = 1, T - 3                    # bcs.cpp:131-133
            self.clover_zero_t = [0, T - 1, T - 2]         # clover.cpp:102-104
        else:
            self.clover_zero_t = []
        self.boundary_term = bc in ("open", "sf")          # bcs.h:7-9, 25-28

    def bcs_on_spinor(self, s):
        """apply_bcs_on_spinor_field, bcs.cpp:139-164 (all sites of the boundary slices)."""
        for tt in self.spinor_zero_t:
            s[self.t == tt] = 0

    def cf_shift(self):
        """Dirac boundary term cf-1 at t in {Ta,Tb}, dirac.cpp:52-59, clover.cpp:32-37."""
        out = np.zeros(self.V)
        if self.boundary_term:
            out[(self.t == self.Ta) | (self.t == self.Tb)] = self.p.cf - 1.0
        return out

    # ---- gauge field: represent_gauge_field, repr.cpp:265-280
    def set_links(self, fund: np.ndarray):
        self.fund = np.array(fund, dtype=complex).reshape(self.V, 4, self.nc, self.nc)
        self.links = represent(self.fund, self.nc, self.p.rep)
        if self.p.clover:
            self.compute_clover_term()
        if self.p.bc == "antiperiodic":                    # bcs.cpp:18-27, 264-272
            self.links[self.t == 0, 0] *= -1

    # ---- clover.cpp
    def clover_leaves(self, mu, nu):
        """clover_repr(id,mu,nu), wilsonloop.cpp:5-31: four plaquette leaves, each
        represented separately, summed."""
        U = self.fund
        x = np.arange(self.V)
        a = self.fw[x, mu]
        b = self.fw[x, nu]
        g0 = U[x, mu] @ U[a, nu] @ dagger(U[x, nu] @ U[b, mu])
        a = self.bk[x, mu]
        b = self.fw[a, nu]
        g1 = U[x, nu] @ dagger(U[a, nu] @ U[b, mu]) @ U[a, mu]
        a = self.bk[x, mu]
        b = self.bk[x, nu]
        c = self.bk[a, nu]
        g2 = dagger(U[c, nu] @ U[a, mu]) @ U[c, mu] @ U[b, nu]
        a = self.bk[x, nu]
        b = self.fw[a, mu]
        g3 = dagger(U[a, nu]) @ U[a, mu] @ U[b, nu] @ dagger(U[x, mu])
        r = [represent(g, self.nc, self.p.rep) for g in (g0, g1, g2, g3)]
        return r[0] + r[1] + r[2] + r[3]

    def compute_clover_term(self):
        """compute_clover_term / _compute_clover_term, clover.cpp:120-168, 330-347."""
        csw = -self.p.csw / 16.0
        t = [self.clover_leaves(m, n) for (m, n) in [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]]
        re = [q.real for q in t]
        im = [q.imag for q in t]
        T = lambda a: np.swapaxes(a, -1, -2)
        a_re = im[2] + T(im[2])
        a_im = T(re[2]) - re[2]
        b_re = im[3] + T(im[3])
        b_im = re[3] - T(re[3])
        c_re = im[0] + T(im[0]) - re[1] + T(re[1])
        c_im = T(re[0]) - re[0] - im[1] - T(im[1])
        d_re = re[4] - T(re[4]) + im[5] + T(im[5])
        d_im = im[4] + T(im[4]) - re[5] + T(re[5])
        cl = np.zeros((self.V, 4, self.d, self.d), dtype=complex)
        cl[:, 0] = csw * (a_re - b_re) + 1j * csw * (a_im + b_im)
        cl[:, 1] = csw * (c_re - d_re) + 1j * csw * (c_im - d_im)
        cl[:, 2] = -csw * (a_re + b_re) + 1j * csw * (b_im - a_im)
        cl[:, 3] = -csw * (c_re + d_re) - 1j * csw * (c_im + d_im)
        for tt in self.clover_zero_t:                      # _bcs_clover_term, clover.cpp:93-118
            cl[self.t == tt] = 0
        self.cl_term = cl
        self._ldl_sigma = None                             # cl_sigma = 0xF00F, clover.cpp:337

    def ldl_blocks(self, sigma):
        """Hermitian 2d x 2d blocks of _compute_ldl_decomp (lower triangles used),
        clover.cpp:40-75.  Returns A, B of shape (V, 2d, 2d)."""
        d = self.d
        cl = self.cl_term
        n = 2 * d
        A = np.zeros((self.V, n, n), dtype=complex)
        B = np.zeros((self.V, n, n), dtype=complex)
        A[:, d:, :d] = np.conj(np.swapaxes(cl[:, 1], -1, -2))
        B[:, d:, :d] = np.conj(np.swapaxes(cl[:, 3], -1, -2))
        tri = np.tril(np.ones((d, d), dtype=bool))
        A[:, :d, :d] = np.where(tri, cl[:, 0], 0)
        A[:, d:, d:] = np.where(tri, -cl[:, 0], 0)
        B[:, :d, :d] = np.where(tri, cl[:, 2], 0)
        B[:, d:, d:] = np.where(tri, -cl[:, 2], 0)
        diag = sigma + self.cf_shift()
        idx = np.arange(n)
        A[:, idx, idx] += diag[:, None]
        B[:, idx, idx] += diag[:, None]
        return A, B

    @staticmethod
    def ldl_factor(A):
        """ldl(N, A): in-place LDL^dag on the lower triangle, solver.cpp:97-117 (vectorised over sites)."""
        A = A.copy()
        n = A.shape[-1]
        for i in range(n):
            for k in range(i):
                A[:, i, i] = A[:, i, i].real - (np.abs(A[:, i, k]) ** 2) * A[:, k, k].real
            for j in range(i + 1, n):
                for k in range(i):
                    A[:, j, i] -= A[:, j, k] * np.conj(A[:, i, k]) * A[:, k, k].real
                A[:, j, i] /= A[:, i, i].real
        return A

    def compute_ldl(self, sigma):
        """compute_ldl_decomp(sigma), clover.cpp:307-328: odd sites only, cached on sigma.
        Returns packed (V, 2, P) with [:,0] upper and [:,1] lower blocks."""
        if self._ldl_sigma == sigma:
            return self._ldl
        A, B = self.ldl_blocks(sigma)
        lo, hi = self.part_range(ODD)
        n = 2 * self.d
        P = self.d * (2 * self.d + 1)
        out = np.zeros((self.V, 2, P), dtype=complex)
        fa = self.ldl_factor(A[lo:hi])
        fb = self.ldl_factor(B[lo:hi])
        k = 0
        for i in range(n):
            for j in range(i + 1):
                out[lo:hi, 0, k] = fa[:, i, j]
                out[lo:hi, 1, k] = fb[:, i, j]
                k += 1
        self._ldl_sigma = sigma
        self._ldl = out
        return out

    @staticmethod
    def ldl_unpack(packed, n):
        L = np.zeros(packed.shape[:-1] + (n, n), dtype=complex)
        k = 0
        for i in range(n):
            for j in range(i + 1):
                L[..., i, j] = packed[..., k]
                k += 1
        return L

    def clover_logdet(self, mass):
        """clover_logdet, clover.cpp:281-305: sum over odd sites of log prod D_nn (both blocks)."""
        if not self.p.clover:
            return 0.0
        ldl = self.compute_ldl(4.0 + mass)
        lo, hi = self.part_range(ODD)
        n = 2 * self.d
        L = self.ldl_unpack(ldl[lo:hi], n)
        dg = np.real(np.diagonal(L, axis1=-2, axis2=-1))
        return float(np.sum(np.log(np.prod(dg, axis=(-1, -2)))))

    # ---- dirac.cpp
    def clover_apply(self, mass, src, lo, hi):
        """clover_kernel body, dirac.cpp:60-96: (4+m+cf) psi + the two 2d x 2d blocks."""
        s = src[lo:hi]
        cl = self.cl_term[lo:hi]
        out = (4.0 + mass + self.cf_shift()[lo:hi])[:, None, None] * s
        c = lambda k, v: np.einsum("vij,vj->vi", cl[:, k], v)
        ch = lambda k, v: np.einsum("vji,vj->vi", np.conj(cl[:, k]), v)
        out[:, :, 0] += c(0, s[:, :, 0]) + c(1, s[:, :, 1])
        out[:, :, 1] += ch(1, s[:, :, 0]) - c(0, s[:, :, 1])
        out[:, :, 2] += c(2, s[:, :, 2]) + c(3, s[:, :, 3])
        out[:, :, 3] += ch(3, s[:, :, 2]) - c(2, s[:, :, 3])
        return out

    def clover_inv_apply(self, mass, src, lo, hi):
        """clover_inv_kernel body, dirac.cpp:135-212: forward substitution, divide by D,
        back substitution with conj(L), per 2d block."""
        d = self.d
        n = 2 * d
        ldl = self.compute_ldl(4.0 + mass)
        out = np.zeros_like(src[lo:hi])
        for blk, (s0, s1) in enumerate([(0, 1), (2, 3)]):
            L = self.ldl_unpack(ldl[lo:hi, blk], n)
            x = np.concatenate([src[lo:hi, :, s0], src[lo:hi, :, s1]], axis=1)
            for i in range(1, n):
                x[:, i] -= np.sum(L[:, i, :i] * x[:, :i], axis=1)
            for i in range(n - 1, -1, -1):
                x[:, i] /= L[:, i, i].real
                if i + 1 < n:
                    x[:, i] -= np.sum(np.conj(L[:, i + 1:, i]) * x[:, i + 1:], axis=1)
            out[:, :, s0] = x[:, :d]
            out[:, :, s1] = x[:, d:]
        return out

    def hop(self, src, lo, hi, sign):
        """dirac_kernel body, dirac.cpp:258-697:
        -sign/2 * sum_mu [(1-g_mu) U(x,mu) psi(x+mu) + (1+g_mu) U(x-mu,mu)^dag psi(x-mu)]."""
        x = np.arange(lo, hi)
        acc = np.zeros((hi - lo, self.d, 4), dtype=complex)
        for mu in range(4):
            f = self.fw[x, mu]
            b = self.bk[x, mu]
            up = col_apply(self.links[x, mu], src[f])
            dn = col_apply(dagger(self.links[b, mu]), src[b])
            acc += spin_apply(ONE4 - GAMMA[mu], up) + spin_apply(ONE4 + GAMMA[mu], dn)
        return (-0.5 * sign) * acc

    def dirac_kernel(self, dst, src, part, sign, assign=False):
        """dirac_kernel, dirac.cpp:227-704, including apply_bcs_on_spinor_field(dst)."""
        self.mvm += 1
        lo, hi = self.part_range(part)
        r = self.hop(src, lo, hi, sign)
        if assign:
            dst[lo:hi] += r
        else:
            dst[lo:hi] = r
        self.bcs_on_spinor(dst)

    def clover_kernel(self, mass, dst, src, part, assign=False):
        lo, hi = self.part_range(part)
        r = self.clover_apply(mass, src, lo, hi)
        if assign:
            dst[lo:hi] += r
        else:
            dst[lo:hi] = r

    def clover_inv_kernel(self, mass, dst, src, part, assign=False):
        lo, hi = self.part_range(part)
        r = self.clover_inv_apply(mass, src, lo, hi)
        if assign:
            dst[lo:hi] += r
        else:
            dst[lo:hi] = r

    def new_field(self):
        return np.zeros((self.V, self.d, 4), dtype=complex)

    def Dphi_oe(self, dst, src):
        """dirac.cpp:706-710"""
        self.dirac_kernel(dst, src, ODD, 1)

    def Dphi_eo(self, dst, src):
        """dirac.cpp:712-716"""
        self.dirac_kernel(dst, src, EVEN, 1)

    def Dphi_ee(self, mass, dst, src):
        """dirac.cpp:718-722"""
        self.clover_kernel(mass, dst, src, EVEN)

    def Dphi_oo(self, mass, dst, src):
        """dirac.cpp:724-728"""
        self.clover_kernel(mass, dst, src, ODD)

    def Dphi_oo_inv(self, mass, dst, src):
        """dirac.cpp:730-734"""
        self.clover_inv_kernel(mass, dst, src, ODD)

    def Dphi(self, mass, dst, src):
        """EO Schur operator, dirac.cpp:738-765.  Like the reference, writes scratch into
        the odd half of src (and zeroes src's boundary slices for open/SF)."""
        if self.p.clover and self.p.eo:
            tmp = self.new_field()
            self.dirac_kernel(src, src, ODD, -1)
            self.clover_inv_kernel(mass, tmp, src, ODD)
            self.dirac_kernel(dst, tmp, EVEN, 1)
            self.clover_kernel(mass, dst, src, EVEN, True)
        elif self.p.clover:
            self.dirac_kernel(dst, src, BOTH, 1)
            self.clover_kernel(mass, dst, src, BOTH, True)
        elif self.p.eo:
            self.dirac_kernel(src, src, ODD, -1)
            self.dirac_kernel(dst, src, EVEN, 1)
            lo, hi = self.default_range()
            dst[lo:hi] += (4.0 + mass) * (4.0 + mass) * src[lo:hi]
        else:
            self.dirac_kernel(dst, src, BOTH, 1)
            dst[:] += (4.0 + mass) * src

    def Hphi(self, mass, dst, src):
        """dirac.cpp:769-773"""
        self.Dphi(mass, dst, src)
        self.spinor_g5(dst)

    def Hphi_sq(self, mass, dst, src):
        """dirac.cpp:775-781"""
        tmp = self.new_field()
        self.Hphi(mass, tmp, src)
        self.Hphi(mass, dst, tmp)

    def op(self, name):
        return {"Dphi": self.Dphi, "Hphi": self.Hphi, "Hphi_sq": self.Hphi_sq}[name]

    # ---- linalg.cpp (default view unless a range is given)
    def _r(self, view):
        return self.default_range() if view is None else self.part_range(view)

    def spinor_g5(self, s, view=None):
        lo, hi = self._r(view)
        s[lo:hi] = spin_apply(GAMMA5, s[lo:hi])

    def sqnorm(self, s, view=None):
        lo, hi = self._r(view)
        return float(np.sum(np.abs(s[lo:hi]) ** 2))

    def product(self, a, b, view=None):
        """spinor_product: sum a * conj(b), spinor.cpp:553-571."""
        lo, hi = self._r(view)
        return complex(np.sum(a[lo:hi] * np.conj(b[lo:hi])))

    def product_re(self, a, b, view=None):
        lo, hi = self._r(view)
        return float(np.sum((a[lo:hi] * np.conj(b[lo:hi])).real))

    # ---- inverters
    def cg(self, op, mass, prec, x, b, maxiter=100000):
        """cg_inverter, cg.cpp:132-202.  Returns iterations (0 if the initial guess passes)."""
        A = self.op(op)
        lo, hi = self.default_range()
        V = slice(lo, hi)
        p = self.new_field()
        qqp = self.new_field()
        p[:] = x
        A(mass, qqp, p)
        r = b.copy()
        r[V] -= qqp[V]
        p[:] = r
        norm = self.sqnorm(b)
        btmp = self.sqnorm(r)
        it = -1 if btmp < norm * prec else 0
        while True:
            it += 1
            if it == 0 or it > maxiter:
                break
            A(mass, qqp, p)
            atmp = self.sqnorm(r)
            btmp = self.product_re(p, qqp)
            alpha = atmp / btmp
            x[V] += alpha * p[V]
            r[V] -= alpha * qqp[V]
            btmp = self.sqnorm(r)
            beta = btmp / atmp
            if btmp < norm * prec:
                break
            p[V] *= beta
            p[V] += r[V]
        return it

    # ---- mre.cpp:15-117 (chronological initial guess) with lu of solver.cpp:4-95
    def mre_init(self, max_, op, mass):
        self.mre = {"max": min(max_, 15), "op": op, "mass": mass, "num": 0,
                    "s": [self.new_field() for _ in range(min(max_, 15))]}

    def mre_store(self, sol):
        m = self.mre
        if m["max"] == 0:
            return
        tmp = m["s"].pop()
        m["s"].insert(0, tmp)
        tmp[:] = sol                       # spinor_copy: the whole field
        m["num"] += 1

    def mre_guess(self, dst, src):
        """dst = sum_k x_k s_k; the stored solutions are orthonormalised in place with the
        reference's coefficient <s_i, s_j> = sum s_i conj(s_j) (mre.cpp:14-33)."""
        m = self.mre
        if m["max"] == 0:
            return
        lo, hi = self.default_range()
        V = slice(lo, hi)
        k = min(m["num"], m["max"])
        dst[:] = 0
        s = m["s"]
        for i in range(k):
            s[i][V] *= 1.0 / np.sqrt(np.sum(np.abs(s[i][V]) ** 2))
            for j in range(i + 1, k):
                rij = np.sum(s[i][V] * np.conj(s[j][V]))
                s[j][V] -= rij * s[i][V]
        A = np.zeros((k, k), dtype=complex)
        b = np.zeros(k, dtype=complex)
        A_op = self.op(m["op"])
        out = self.new_field()
        for i in range(k):
            A_op(m["mass"], out, s[i])
            for j in range(k):
                A[j, i] = np.sum(out[V] * np.conj(s[j][V]))
            b[i] = np.sum(src[V] * np.conj(s[i][V]))
        if k == 0:
            return
        x = np.linalg.solve(A, b)
        for i in range(k):
            dst[V] += x[i] * s[i][V]

    def cg_mshift(self, op, mass, prec, shifts, b, maxiter=100000):
        """cg_mshift, cg.cpp:11-130.  Returns (iterations, [x_n])."""
        A = self.op(op)
        lo, hi = self.default_range()
        V = slice(lo, hi)
        num = len(shifts)
        r = b.copy()
        p = b.copy()
        qqp = self.new_field()
        xs = [self.new_field() for _ in range(num)]
        ks = [b.copy() for _ in range(num)]
        c1 = [1.0] * num
        c2 = [1.0] * num
        c3 = [0.0] * num
        flag = [False] * num
        beta, alpha = 1.0, 0.0
        norm = self.sqnorm(b)
        it = 0
        while True:
            it += 1
            A(mass, qqp, p)
            atmp = self.sqnorm(r)
            btmp = self.product_re(p, qqp)
            beta_old = beta
            beta = -(atmp / btmp)
            for n in range(num):
                if flag[n]:
                    continue
                c3[n] = c2[n] * c1[n] * beta_old
                c3[n] /= (beta * alpha * (c1[n] - c2[n])) + (c1[n] * beta_old * (1 - shifts[n] * beta))
                bt = beta * (c3[n] / c2[n])
                xs[n][V] -= bt * ks[n][V]
            r[V] += beta * qqp[V]
            btmp = self.sqnorm(r)
            alpha = btmp / atmp
            notconv = 0
            for n in range(num):
                if flag[n]:
                    continue
                at = alpha * (c3[n] * c3[n]) / (c2[n] * c2[n])
                ks[n][V] *= at
                ks[n][V] += c3[n] * r[V]
                if btmp * c3[n] * c3[n] < norm * prec:
                    flag[n] = True
                else:
                    notconv += 1
                c1[n] = c2[n]
                c2[n] = c3[n]
            if notconv == 0 or it >= maxiter:
                break
            p[V] *= alpha
            p[V] += r[V]
        return it, xs

    def bicgstab(self, op, mass, prec, x, b, maxiter=100000):
        """bicgstab_inverter, bicgstab.cpp:9-97.  Returns 2*iterations."""
        A = self.op(op)
        lo, hi = self.default_range()
        V = slice(lo, hi)
        p = self.new_field()
        v = self.new_field()
        t = self.new_field()
        A(mass, p, x)
        r = b.copy()
        r[V] -= p[V]
        r0 = r.copy()
        p[:] = r
        norm = self.sqnorm(b)
        rho0 = self.product(r, r0)
        it = -1 if rho0.real < norm * prec else 0
        while True:
            it += 1
            if it == 0 or it > maxiter:
                break
            A(mass, v, p)
            alpha = rho0 / self.product(v, r0)
            r[V] -= alpha * v[V]
            A(mass, t, r)
            omega = self.product(r, t) / self.sqnorm(t)
            x[V] += alpha * p[V]
            x[V] += omega * r[V]
            r[V] -= omega * t[V]
            rho1 = self.product(r, r0)
            beta = (rho1 / rho0) * (alpha / omega)
            p[V] *= beta
            p[V] += r[V]
            p[V] -= (beta * omega) * v[V]
            if self.sqnorm(r) < norm * prec:
                break
            rho0 = rho1
        return 2 * it

    def minres(self, op, mass, prec, x, b, maxiter=100000):
        """minres_inverter, minres.cpp:12-117."""
        A = self.op(op)
        lo, hi = self.default_range()
        V = slice(lo, hi)
        tmp = self.new_field()
        A(mass, tmp, x)
        v1 = b.copy()
        v1[V] -= tmp[V]
        v0 = self.new_field()
        w0 = self.new_field()
        w1 = self.new_field()
        g0 = g1 = 1.0
        s0 = s1 = 0.0
        norm = self.sqnorm(b)
        residue = self.sqnorm(v1)
        beta0 = math.sqrt(residue)
        eta = beta0
        it = -1 if residue < norm * prec else 0
        while True:
            it += 1
            if it == 0 or it > maxiter:
                break
            v1[V] *= 1.0 / beta0
            A(mass, tmp, v1)
            alpha = self.product_re(v1, tmp)
            tmp[V] -= alpha * v1[V]
            tmp[V] -= beta0 * v0[V]
            v0, v1, tmp = v1, tmp, v0
            beta1 = math.sqrt(self.sqnorm(v1))
            delta = g1 * alpha - g0 * s1 * beta0
            rho1 = math.sqrt(delta * delta + beta1 * beta1)
            rho2 = s1 * alpha + g0 * g1 * beta0
            rho3 = s0 * beta0
            g0 = g1
            g1 = delta / rho1
            s0 = s1
            s1 = beta1 / rho1
            tmp[V] = (1.0 / rho1) * v0[V]
            tmp[V] -= (rho3 / rho1) * w0[V]
            tmp[V] -= (rho2 / rho1) * w1[V]
            w0, w1, tmp = w1, tmp, w0
            x[V] += (g1 * eta) * w1[V]
            eta = -s1 * eta
            beta0 = beta1
            residue = eta * eta
            if residue < norm * prec:
                break
        return it

    def auto_inverter(self, op, mass, prec, x, b):
        """auto_inverter, inverter.cpp:9-55: BiCGstab on Dphi with gamma5 sandwiches."""
        if op == "Hphi_sq":
            tmp = self.new_field()
            self.spinor_g5(b)
            it = self.bicgstab("Dphi", mass, prec, tmp, b)
            self.spinor_g5(tmp)
            it += self.bicgstab("Dphi", mass, prec, x, tmp)
            self.spinor_g5(b)
            return it
        if op == "Hphi":
            self.spinor_g5(b)
            it = self.bicgstab("Dphi", mass, prec, x, b)
            self.spinor_g5(b)
            return it
        return self.bicgstab("Dphi", mass, prec, x, b)

    # ---- observables/propagator.cpp
    def create_point_source(self, n, tau):
        """create_point_source, propagator.cpp:58-73: a unit source in spin n // d, colour
        n % d at (tau, 0, 0, 0)."""
        f = self.new_field()
        f[self.index(tau, 0, 0, 0), n % self.d, n // self.d] = 1.0
        return f

    def timeslice_sites(self, tau):
        """the site ids of time slice tau in increasing order (the sites_for order in which
        create_semwall_source draws its noise)"""
        return np.sort(np.nonzero(self.t == tau)[0])

    def create_semwall_source(self, n, tau, f, z2=None):
        """create_semwall_source, propagator.cpp:22-56.  n = 0: Z2 noise on spin 0 of slice
        tau, z2[k, i] = (re, im) of colour i at the k-th slice site (rand_z2() values in the
        reference's draw order); n > 0: spin n-1 moves to spin n."""
        if n == 0:
            f[:] = 0
            z = np.asarray(z2, dtype=np.float64).reshape(-1, self.d, 2)
            f[self.timeslice_sites(tau), :, 0] = z[..., 0] + 1j * z[..., 1]
        else:
            f[:, :, n] = f[:, :, n - 1]
            f[:, :, n - 1] = 0

    def calc_propagator(self, mass, prec, dst, src):
        """calc_propagator, propagator.cpp:75-166: with even-odd preconditioning the even
        system D x_e = b_e - D_eo D_oo^-1 b_o (clover) or (4+m) b_e - D_eo b_o (Wilson) is
        solved by auto_inverter (BiCGstab on Dphi, dst as the initial guess) and the odd
        sites follow from x_o = D_oo^-1 (b_o - D_oe x_e); without it, D x = b directly."""
        if not self.p.eo:
            return self.auto_inverter("Dphi", mass, prec, dst, src)
        lo, hi = self.part_range(EVEN)
        olo, ohi = self.part_range(ODD)
        tmp, eo = self.new_field(), self.new_field()
        if self.p.clover:
            self.Dphi_oo_inv(mass, tmp, src)
            self.Dphi_eo(tmp, tmp)
            eo[lo:hi] = -1.0 * tmp[lo:hi]
            eo[lo:hi] += src[lo:hi]
            it = self.auto_inverter("Dphi", mass, prec, dst, eo)
            self.Dphi_oe(tmp, dst)
            dst[olo:ohi] = 1.0 * src[olo:ohi]
            dst[olo:ohi] -= tmp[olo:ohi]
            self.Dphi_oo_inv(mass, dst, dst)
        else:
            m4 = 4.0 + mass
            self.Dphi_eo(tmp, src)
            eo[lo:hi] = m4 * src[lo:hi]
            eo[lo:hi] -= tmp[lo:hi]
            it = self.auto_inverter("Dphi", mass, prec, dst, eo)
            self.Dphi_oe(tmp, dst)
            dst[olo:ohi] = (1.0 / m4) * src[olo:ohi]
            dst[olo:ohi] -= (1.0 / m4) * tmp[olo:ohi]
        return it

    # ---- observables/mesons.cpp
    def meson_measure(self, mass, prec, method, taus, noises=None, props=None):
        """the hit loop of meson_measure, mesons.cpp:215-259, with the source time slices
        (random_timeslice) and, for SEMWALL, each hit's z2 noise given.  The propagators
        persist across hits as the solver's initial guesses, as the reference's static
        prop[] do.  Returns the raw correlators (MESON_CHANNELS x T)."""
        ninv = 4 if method == SEMWALL else 4 * self.d
        if props is None:
            props = [self.new_field() for _ in range(ninv)]
        raw = np.zeros((len(MESON_CHANNELS), self.dims[0]))
        source = self.new_field()
        for h, tau in enumerate(taus):
            for n in range(ninv):
                if method == SEMWALL:
                    self.create_semwall_source(n, tau, source, noises[h] if n == 0 else None)
                else:
                    source = self.create_point_source(n, tau)
                self.calc_propagator(mass, prec, props[n], source)
            raw += self.meson_contract(method, tau, props)
        return raw

    def meson_contract(self, method, tau, props):
        """contract_all_correlators, mesons.cpp:55-128: raw[ch, (t - tau) mod T] summed over
        the sites of each slice, channels in MESON_CHANNELS order.  props: 4 (SEMWALL,
        prop[A] for source spin A) or 4d (POINT, prop[c*d + x] for source spin c, colour x)
        fields.  Per site, Re sum_{a,c} v1[a] v2[c] sum_{x,y} P[c,x](col1[a], y) conj(P[col2[c],x](a, y))."""
        ns = 1 if method == SEMWALL else self.d
        P = np.stack(props).reshape(4, ns, self.V, self.d, 4)
        T = self.dims[0]
        trel = (self.t - tau + T) % T
        out = np.zeros((len(MESON_CHANNELS), T))
        for k, (g1, g2) in enumerate(MESON_PAIRS):
            c1, v1 = MESON_GAMMA[g1]
            c2, v2 = MESON_GAMMA[g2]
            site = np.zeros(self.V, dtype=complex)
            for a in range(4):
                for c in range(4):
                    site += v1[a] * v2[c] * np.einsum("xvy,xvy->v", P[c, :, :, :, c1[a]], np.conj(P[c2[c], :, :, :, a]))
            out[k] = np.bincount(trel, weights=site.real, minlength=T)
        return out

    # ---- forces.cpp
    @staticmethod
    def fmat_create(a_lhs, a_rhs, b_lhs, b_rhs):
        """fmat = a_lhs # a_rhs + b_lhs # b_rhs (outer product over spin), forces.cpp:13-30."""
        return np.einsum("vik,vjk->vij", a_lhs, np.conj(a_rhs)) + \
            np.einsum("vik,vjk->vij", b_lhs, np.conj(b_rhs))

    def clover_fermion_force(self, residue, lhs, rhs):
        """forces.cpp:122-172 (all local sites)."""
        for slot, (m, n) in enumerate(CLOVER_PAIRS):
            S = G5_SIGMA[(m, n)]
            tl = spin_apply(S, lhs)
            tr = spin_apply(S, rhs)
            self.cl_force[:, slot] += residue * self.fmat_create(tl, rhs, tr, lhs)

    def wilson_fermion_force(self, dt, mass, residue, lhs, rhs):
        """forces.cpp:175-227: (EO) odd halves replaced in place by D_oo^-1 D_oe X_e, then the
        clover force and the hopping force P(x,mu) += coeff Proj[U(x,mu) fmat]."""
        coeff = dt * residue
        if self.p.eo:
            self.Dphi_oe(rhs, rhs)
            self.Dphi_oe(lhs, lhs)
            if self.p.clover:
                self.Dphi_oo_inv(mass, rhs, rhs)
                self.Dphi_oo_inv(mass, lhs, lhs)
            coeff = -coeff
        if self.p.clover:
            self.clover_fermion_force(residue, lhs, rhs)
        x = np.arange(self.V)
        for mu in range(4):
            f = self.fw[x, mu]
            M = GAMMA5 @ (ONE4 - GAMMA[mu])                # g5_one_minus_gamma, spinor.cpp:440-500
            tl = spin_apply(M, lhs[f])
            tr = spin_apply(M, rhs[f])
            fm = self.fmat_create(tl, rhs, tr, lhs)
            fm = self.links[:, mu] @ fm
            self.mom[:, mu] += algebra_project(fm, self.itrepr, coeff)

    def wilson_fermion_force_q(self, dt, mass, residue, rhs):
        """forces.cpp:230-236"""
        tmp = self.new_field()
        self.Hphi(mass, tmp, rhs)
        self.wilson_fermion_force(dt, mass, residue, tmp, rhs)

    def begin_fermion_force(self):
        """forces.cpp:239-251"""
        self.cl_force[:] = 0

    def compute_clover_force(self, mass, coeff):
        """compute_clover_force / _compute_clover_force, clover.cpp:170-279: columns of
        coeff * D_oo^-1 from the LDL factors, combined into X_mu,nu on odd sites."""
        if not self.p.clover:
            return
        d = self.d
        n = 2 * d
        ldl = self.compute_ldl(4.0 + mass)
        lo, hi = self.part_range(ODD)
        inv = []
        for blk in range(2):
            L = self.ldl_unpack(ldl[lo:hi, blk], n)
            M = np.zeros((hi - lo, n, n), dtype=complex)
            for c in range(n):
                M[:, c, c] = coeff
                for i in range(c, n):
                    for k in range(i):
                        M[:, i, c] -= L[:, i, k] * M[:, k, c]
                for i in range(n - 1, c - 1, -1):
                    M[:, i, c] /= L[:, i, i].real
                    for k in range(i + 1, n):
                        M[:, i, c] -= np.conj(L[:, k, i]) * M[:, k, c]
            inv.append(M)
        A, B = inv
        F = np.zeros((hi - lo, 6, d, d), dtype=complex)
        for i in range(d):
            for j in range(d):
                a21 = A[:, i + d, j]
                a12 = np.conj(A[:, j + d, i])
                a43 = B[:, i + d, j]
                a34 = np.conj(B[:, j + d, i])
                if i < j:
                    a11 = np.conj(A[:, j, i])
                    a22 = np.conj(A[:, j + d, i + d])
                    a33 = np.conj(B[:, j, i])
                    a44 = np.conj(B[:, j + d, i + d])
                else:
                    a11 = A[:, i, j]
                    a22 = A[:, i + d, j + d]
                    a33 = B[:, i, j]
                    a44 = B[:, i + d, j + d]
                R = lambda z: z.real
                I = lambda z: z.imag
                F[:, 0, i, j] = (I(a12) + I(a21) - I(a34) - I(a43)) + 1j * (-R(a12) - R(a21) + R(a34) + R(a43))
                F[:, 1, i, j] = (R(a12) - R(a21) + R(a43) - R(a34)) + 1j * (I(a12) - I(a21) + I(a43) - I(a34))
                F[:, 2, i, j] = (I(a22) - I(a11) + I(a44) - I(a33)) + 1j * (R(a11) - R(a22) + R(a33) - R(a44))
                F[:, 3, i, j] = (I(a11) - I(a22) + I(a44) - I(a33)) + 1j * (R(a22) - R(a11) + R(a33) - R(a44))
                F[:, 4, i, j] = (R(a12) - R(a21) + R(a34) - R(a43)) + 1j * (I(a12) - I(a21) + I(a34) - I(a43))
                F[:, 5, i, j] = (-I(a12) - I(a21) - I(a34) - I(a43)) + 1j * (R(a12) + R(a21) + R(a34) + R(a43))
        self.cl_force[lo:hi] += F

    def clover_logdet_force(self, mass, residue):
        """forces.cpp:109-119"""
        self.compute_clover_force(mass, residue)

    def clover_force_core(self, dt):
        """forces.cpp:33-106: 6-link assembly of the clover force into the momenta."""
        coeff = self.p.csw * dt / 8.0
        U = self.links
        x = np.arange(self.V)
        Zf = self.cl_force
        for mu in range(4):
            for nu in range(4):
                if mu == nu:
                    continue
                o1 = self.fw[x, mu]
                o2 = self.fw[x, nu]
                o3 = self.bk[x, nu]
                o4 = self.fw[o3, mu]
                o5 = self.fw[o2, mu]
                if mu < nu:
                    num, sign = nu * (nu - 1) // 2 + mu, 1.0
                else:
                    num, sign = mu * (mu - 1) // 2 + nu, -1.0
                Z0, Z1, Z2, Z3, Z4, Z5 = (Zf[o, num] for o in (x, o1, o3, o4, o5, o2))
                W0 = dagger(U[o3, mu])
                W1 = U[o3, nu]
                W2 = U[o1, nu]
                W3 = dagger(U[o2, mu])
                W4 = dagger(U[x, nu])
                W5 = dagger(U[o4, nu])
                W6 = W0 @ W1
                W7 = W2 @ W3
                W8 = W7 @ W4 - W5 @ W6
                fm = W8 @ Z0 + Z1 @ W8
                fm = fm - W5 @ (W0 @ Z2 @ W1 + Z3 @ W6)
                fm = fm + (W2 @ Z4 @ W3 + W7 @ Z5) @ W4
                fm = U[x, mu] @ fm
                self.mom[:, mu] += algebra_project(fm, self.itrepr, sign * coeff)

    def end_fermion_force(self, dt):
        """forces.cpp:254-259"""
        if self.p.clover:
            self.clover_force_core(dt)

    # ---- gauge support (bcs.cpp, staples.cpp, wilsonloop.cpp, forces.cpp:262-309, update.cpp)
    def plaq_weights(self):
        """plaq_weight(id,mu,nu) as a (V, 4, 4) array, bcs.cpp:29-133: 1 everywhere except
        0.5 on the spatial planes of t = 0 and t = T-1 (open) or t = 0 and t = T-2 (sf)."""
        w = np.ones((self.V, 4, 4))
        T = self.dims[0]
        slices = {"open": [0, T - 1], "sf": [0, T - 2]}.get(self.p.bc, [])
        for tt in slices:
            for mu in (1, 2, 3):
                for nu in (1, 2, 3):
                    if mu != nu:
                        w[self.t == tt, mu, nu] = 0.5
        return w

    def rect_weights(self):
        """rect_weight(id,mu,nu), bcs.cpp:29-133: the plaquette weights (open: same array),
        or for sf 0 on the planes (1,2),(1,3),(2,3) of t = 0 and T-2 and 1.5 on (0,1),(0,2),
        (0,3) of t = 0 and T-3."""
        if self.p.bc != "sf":
            return self.plaq_weights()
        w = np.ones((self.V, 4, 4))
        T = self.dims[0]
        for tt in (0, T - 2):
            for (mu, nu) in ((1, 2), (1, 3), (2, 3)):
                w[self.t == tt, mu, nu] = 0.0
        for tt in (0, T - 3):
            for nu in (1, 2, 3):
                w[self.t == tt, 0, nu] = 1.5
        return w

    def volume(self):
        """the global `volume` of the gauge action: V, (T-1) V3 for open, (T-2) V3 for sf
        (bcs.cpp:32, 76)."""
        v3 = self.V // self.dims[0]
        return {"open": (self.dims[0] - 1) * v3, "sf": (self.dims[0] - 2) * v3}.get(self.p.bc, self.V)

    def staples_wilson(self, mu):
        """staples_wilson, staples.cpp:83-107."""
        U, pw = self.fund, self.plaq_weights()
        x = np.arange(self.V)
        st = np.zeros((self.V, self.nc, self.nc), dtype=complex)
        for nu in range(4):
            if nu == mu:
                continue
            o1 = self.fw[x, mu]
            o2 = self.fw[x, nu]
            st += pw[x, mu, nu][:, None, None] * (U[o1, nu] @ dagger(U[x, nu] @ U[o2, mu]))
            o1 = self.bk[x, nu]
            o2 = self.fw[o1, mu]
            st += pw[o1, nu, mu][:, None, None] * (dagger(U[o1, mu] @ U[o2, nu]) @ U[o1, nu])
        return st

    def staples_symanzik(self, mu):
        """staples_symanzik, staples.cpp:7-81: the six 2x1 rectangles through link (x,mu)
        for each nu != mu."""
        U, rw = self.fund, self.rect_weights()
        fw, bk = self.fw, self.bk
        x = np.arange(self.V)
        st = np.zeros((self.V, self.nc, self.nc), dtype=complex)

        def w(site, a, b):
            return rw[site, a, b][:, None, None]

        for nu in range(4):
            if nu == mu:
                continue
            o1 = fw[x, mu]; o2 = fw[o1, nu]; o3 = fw[x, nu]; o4 = fw[o3, nu]
            st += w(x, mu, nu) * (U[o1, nu] @ U[o2, nu] @ dagger(U[x, nu] @ U[o3, nu] @ U[o4, mu]))
            o1 = bk[x, nu]; o2 = bk[o1, nu]; o3 = fw[o2, mu]; o4 = fw[o3, nu]
            st += w(o2, mu, nu) * (dagger(U[o2, mu] @ U[o3, nu] @ U[o4, nu]) @ U[o2, nu] @ U[o1, nu])
            o1 = bk[x, nu]; o2 = fw[o1, mu]; o3 = fw[o2, mu]; o4 = fw[x, mu]
            st += w(o1, nu, mu) * (U[o4, mu] @ dagger(U[o1, mu] @ U[o2, mu] @ U[o3, nu]) @ U[o1, nu])
            o1 = fw[x, mu]; o2 = fw[o1, mu]; o3 = fw[x, nu]; o4 = fw[o3, mu]
            st += w(x, nu, mu) * (U[o1, mu] @ U[o2, nu] @ dagger(U[x, nu] @ U[o3, mu] @ U[o4, mu]))
            o1 = bk[x, mu]; o2 = bk[o1, nu]; o3 = fw[o2, mu]; o4 = fw[o3, mu]
            st += w(o2, nu, mu) * (dagger(U[o2, mu] @ U[o3, mu] @ U[o4, nu]) @ U[o2, nu] @ U[o1, mu])
            o1 = bk[x, mu]; o2 = fw[o1, nu]; o3 = fw[o2, mu]; o4 = fw[x, mu]
            st += w(o1, nu, mu) * (U[o4, nu] @ dagger(U[o1, nu] @ U[o2, mu] @ U[o3, mu]) @ U[o1, mu])
        return st

    def wilson_gauge_force(self, dt, beta):
        """forces.cpp:262-283"""
        coeff = dt * (beta / self.nc)
        for mu in range(4):
            f = self.fund[:, mu] @ self.staples_wilson(mu)
            self.mom[:, mu] -= algebra_project(f, self.itfund, coeff)

    def improved_gauge_force(self, dt, beta, c0, c1):
        """forces.cpp:285-309"""
        coeff = dt * (beta / self.nc)
        for mu in range(4):
            f = c0 * (self.fund[:, mu] @ self.staples_wilson(mu)) + c1 * (self.fund[:, mu] @ self.staples_symanzik(mu))
            self.mom[:, mu] -= algebra_project(f, self.itfund, coeff)

    def wilson_loop(self, mu, nu, height, width):
        """wilson_loop(id,mu,nu,height,width) for every site, wilsonloop.cpp:56-114."""
        U, fw = self.fund, self.fw
        x = np.arange(self.V)
        one = U[x, mu].copy()
        two = U[x, nu].copy()
        pos = x
        for _ in range(1, height):
            pos = fw[pos, mu]
            one = one @ U[pos, mu]
        pos = fw[pos, mu]
        one = one @ U[pos, nu]
        for _ in range(1, width):
            pos = fw[pos, nu]
            one = one @ U[pos, nu]
        pos = x
        for _ in range(1, width):
            pos = fw[pos, nu]
            two = two @ U[pos, nu]
        pos = fw[pos, nu]
        two = two @ U[pos, mu]
        for _ in range(1, height):
            pos = fw[pos, mu]
            two = two @ U[pos, mu]
        tr = np.einsum("vij,vji->v", one, dagger(two)).real
        if (height, width) == (1, 1):
            tr = tr * self.plaq_weights()[x, mu, nu]
        elif (height, width) == (1, 2):
            tr = tr * self.rect_weights()[x, mu, nu]
        elif (height, width) == (2, 1):
            tr = tr * self.rect_weights()[x, nu, mu]
        return tr

    def avr_wilson(self, height, width):
        """wilsonloop.cpp:116-133"""
        s = 0.0
        for (mu, nu) in [(1, 0), (2, 0), (2, 1), (3, 0), (3, 1), (3, 2)]:
            s += self.wilson_loop(mu, nu, height, width).sum()
        return s / (self.nc * 6 * self.volume())

    def plaquette(self):
        """avr_wilson(1,1)"""
        return self.avr_wilson(1, 1)

    def gauge_action(self, beta, c0):
        """MonomialGauge::action, monomials/gauge.cpp:21-40 (c1 = (1-c0)/8)."""
        c1 = (1.0 - c0) / 8.0
        if abs(c1) > 1e-8:
            v = c0 * self.avr_wilson(1, 1) + c1 * (self.avr_wilson(2, 1) + self.avr_wilson(1, 2))
        else:
            v = self.avr_wilson(1, 1)
        return -beta * v * 6 * self.volume()

    def bcs_on_momenta(self):
        """apply_bcs_on_momentum_field, bcs.cpp:166-199"""
        T = self.dims[0]
        if self.p.bc == "open":
            self.mom[self.t == T - 1, 0] = 0
        elif self.p.bc == "sf":
            self.mom[self.t == 0, 1:] = 0
            self.mom[self.t == T - 2] = 0
            self.mom[self.t == T - 1] = 0

    def sf_boundary_links(self):
        """C1, C2 of apply_bcs_on_gauge_field (bcs.cpp:211-245): diag exp(i v_k / L)."""
        nc = self.nc
        if nc == 2:
            v1, v2, L = [-math.pi, math.pi], [-3 * math.pi, 3 * math.pi], 4 * self.dims[1]
        elif nc == 3:
            v1, v2, L = [-math.pi, 0, math.pi], [-5 * math.pi, 2 * math.pi, 3 * math.pi], 6 * self.dims[1]
        else:
            raise ValueError("sf boundary fields exist for SU(2) and SU(3)")
        c1 = np.diag(np.exp(1j * np.array(v1) / L))
        c2 = np.diag(np.exp(1j * np.array(v2) / L))
        return c1, c2

    def bcs_on_gauge(self):
        """apply_bcs_on_gauge_field, bcs.cpp:201-262"""
        T = self.dims[0]
        if self.p.bc == "open":
            self.fund[self.t == T - 1, 0] = 0
        elif self.p.bc == "sf":
            c1, c2 = self.sf_boundary_links()
            self.fund[self.t == 0, 1:] = c1
            self.fund[self.t == T - 2, 0] = 0
            self.fund[self.t == T - 2, 1:] = c2
            self.fund[self.t == T - 1] = 0

    # ---- observables/wilsonflow.cpp
    def wf_init(self):
        """wilsonflow.cpp:149-157"""
        self.mom[:] = 0

    def wf_zeta(self, alpha):
        """wilsonflow.cpp:8-23: P -= algebra_project(U staple, alpha)"""
        for mu in range(4):
            f = self.fund[:, mu] @ self.staples_wilson(mu)
            self.mom[:, mu] -= algebra_project(f, self.itfund, alpha)

    def wf_update(self, val):
        """wilsonflow.cpp:25-41: U <- exp(P) U, P <- val P, then the link boundary values"""
        self.fund = exp_algebra(self.nc, self.mom, 1.0) @ self.fund
        self.mom *= val
        self.bcs_on_gauge()

    def wf_iterate(self, eps):
        """wilsonflow.cpp:43-53"""
        self.wf_zeta(eps / 4.0)
        self.wf_update(-17.0 / 9.0)
        self.wf_zeta(8.0 * eps / 9.0)
        self.wf_update(-1.0)
        self.wf_zeta(3.0 * eps / 4.0)
        self.wf_update(0.0)

    def clover_fund(self, mu, nu):
        """clover_fund(id,mu,nu), wilsonloop.cpp:33-54: the four leaves, unrepresented"""
        U, x = self.fund, np.arange(self.V)
        a, b = self.fw[x, mu], self.fw[x, nu]
        r = U[x, mu] @ U[a, nu] @ dagger(U[x, nu] @ U[b, mu])
        a = self.bk[x, mu]
        b = self.fw[a, nu]
        r = r + U[x, nu] @ dagger(U[a, nu] @ U[b, mu]) @ U[a, mu]
        a, b = self.bk[x, mu], self.bk[x, nu]
        c = self.bk[a, nu]
        r = r + dagger(U[c, nu] @ U[a, mu]) @ U[c, mu] @ U[b, nu]
        a = self.bk[x, nu]
        b = self.fw[a, mu]
        return r + dagger(U[a, nu]) @ U[a, mu] @ U[b, nu] @ dagger(U[x, mu])

    def wf_e_plaq(self):
        """wilsonflow.cpp:55-74: 2/V sum_x sum_{mu>nu} (N - weighted Re tr P)"""
        s = 0.0
        for mu in range(1, 4):
            for nu in range(mu):
                s += np.sum(self.nc - self.wilson_loop(mu, nu, 1, 1))
        return 2 * s / self.V

    def wf_e_sym(self):
        """wilsonflow.cpp:76-101"""
        norm = math.sqrt(2.0 * TF)
        s = 0.0
        for mu in range(1, 4):
            for nu in range(mu):
                s += np.sum(algebra_project(self.clover_fund(mu, nu), self.itfund, norm) ** 2)
        return 2 * s / (16 * 4 * self.V)

    def wf_charge(self):
        """wilsonflow.cpp:103-147"""
        norm = math.sqrt(2.0 * TF)
        tc = 0.0
        for (m1, n1), (m2, n2) in (((0, 3), (1, 2)), ((0, 2), (3, 1)), ((0, 1), (2, 3))):
            a1 = algebra_project(self.clover_fund(m1, n1), self.itfund, norm)
            a2 = algebra_project(self.clover_fund(m2, n2), self.itfund, norm)
            tc += np.sum(a1 * a2)
        return 2 * tc / (16 * 16 * math.pi * math.pi)

    # ---- observables/fermionflow.cpp
    def wf_laplacian(self, src):
        """fermionflow.cpp:11-26: -8 s(x) + sum_mu U(x,mu) s(x+mu) + U(x-mu,mu)^dag s(x-mu),
        represented links (with the antiperiodic sign), every site"""
        x = np.arange(self.V)
        out = -8.0 * src
        for mu in range(4):
            fw, bk = self.fw[x, mu], self.bk[x, mu]
            out = out + np.einsum("vij,vjs->vis", self.links[x, mu], src[fw])
            out = out + np.einsum("vji,vjs->vis", np.conj(self.links[bk, mu]), src[bk])
        return out

    def wf_fermion_init(self, phis):
        """fermionflow.cpp:76-92: phis are flowed in place"""
        self.wf_phi0 = phis
        self.wf_phi1 = [self.new_field() for _ in phis]
        self.wf_phi2 = [self.new_field() for _ in phis]
        self.wf_init()

    def wf_fermion_iterate(self, eps):
        """fermionflow.cpp:28-74; spinor_copy copies whole fields (linalg.cpp:71-76), the
        other vector updates cover the default view, as the reference's spinor_* calls do"""
        lo, hi = self.default_range()
        p0, p1, p2 = self.wf_phi0, self.wf_phi1, self.wf_phi2
        self.represent_gauge_field()
        for i in range(len(p0)):
            d = self.wf_laplacian(p0[i])
            p1[i][:] = p0[i]
            p1[i][lo:hi] += (eps / 4.0) * d[lo:hi]
        self.wf_zeta(eps / 4.0)
        self.wf_update(-17.0 / 9.0)
        self.represent_gauge_field()
        for i in range(len(p0)):
            d = self.wf_laplacian(p1[i])
            p2[i][lo:hi] = (-8.0 / 9.0) * p1[i][lo:hi]
            p2[i][lo:hi] += (17.0 / 9.0) * p0[i][lo:hi]
            p2[i][lo:hi] += (8.0 * eps / 9.0) * d[lo:hi]
        self.wf_zeta(8.0 * eps / 9.0)
        self.wf_update(-1.0)
        self.represent_gauge_field()
        for i in range(len(p0)):
            d = self.wf_laplacian(p2[i])
            p0[i][:] = p1[i]
            p0[i][lo:hi] += (3.0 * eps / 4.0) * d[lo:hi]
        self.wf_zeta(3.0 * eps / 4.0)
        self.wf_update(0.0)

    def update_links(self, eps):
        """update.cpp:228-247: U <- exp(eps P) U with the boundary conditions.  As there, the
        represented field is rebuilt only by represent_gauge_field()."""
        self.bcs_on_momenta()
        self.fund = exp_algebra(self.nc, self.mom, eps) @ self.fund
        self.bcs_on_gauge()

    def represent_gauge_field(self):
        """repr.cpp:265-280 (with the clover term and the antiperiodic sign)"""
        self.set_links(self.fund)

    def reunitarize_links(self):
        """update.cpp:269-279 (the represented field is rebuilt by the caller, as there)."""
        self.fund = reunitarize(self.fund)

    def hamiltonian_momenta(self):
        """the momentum part of hamiltonian(), update.cpp:201-226: (TF/2) sum |P|^2 after the
        momentum boundary conditions."""
        self.bcs_on_momenta()
        return TF / 2.0 * float(np.sum(self.mom ** 2))


# ---------------------------------------------------------------- gauge configuration files
# gaugefield.cpp:44-179 (CFG, native byte order) and hirep.cpp:56-212 (HiRep, big-endian).
# U is (V, 4, N, N) complex in the even-odd site order; files run over t, x, y, z.
# ---- meson channels, observables/mesons.cpp:12-27 and include/spectrum.h:7-13.  Each
# g5*Gamma is a signed spin permutation: row a has its one entry val[a] in column col[a].
SEMWALL, POINT = 0x01, 0x02
_I1 = 1j
MESON_GAMMA = {
    "ID": ((0, 1, 2, 3), (1, 1, -1, -1)),
    "G1": ((3, 2, 1, 0), (-_I1, -_I1, -_I1, -_I1)),
    "G2": ((3, 2, 1, 0), (-1, 1, -1, 1)),
    "G3": ((2, 3, 0, 1), (-_I1, _I1, -_I1, _I1)),
    "G5": ((0, 1, 2, 3), (1, 1, 1, 1)),
    "G5G1": ((3, 2, 1, 0), (-_I1, -_I1, _I1, _I1)),
    "G5G2": ((3, 2, 1, 0), (-1, 1, 1, -1)),
    "G5G3": ((2, 3, 0, 1), (-_I1, _I1, _I1, -_I1)),
    "G0G1": ((1, 0, 3, 2), (-_I1, -_I1, -_I1, -_I1)),
    "G0G2": ((1, 0, 3, 2), (-1, 1, -1, 1)),
    "G0G3": ((0, 1, 2, 3), (-_I1, _I1, -_I1, _I1)),
    "G0G5": ((2, 3, 0, 1), (1, 1, 1, 1)),
    "G0G5G1": ((1, 0, 3, 2), (_I1, _I1, -_I1, -_I1)),
    "G0G5G2": ((1, 0, 3, 2), (1, -1, -1, 1)),
    "G0G5G3": ((0, 1, 2, 3), (_I1, -_I1, -_I1, _I1)),
}
MESON_CHANNELS = ("id", "g1", "g2", "g3", "g5", "g5g1", "g5g2", "g5g3", "g0g1", "g0g2", "g0g3", "g0g5",
                  "g0g5g1", "g0g5g2", "g0g5g3", "g5_g0g5")
MESON_PAIRS = tuple((c.upper(), c.upper()) for c in MESON_CHANNELS[:15]) + (("G0G5", "G5"),)
# meson_measure's print list, mesons.cpp:280-295: (label, printed channel, sign).  As in the
# reference, "g0g5g1" prints the g0g5g2 correlator and "g0g5g2" the g0g5g3 one.
MESON_PRINT = (("id", "id", -1.0), ("g1", "g1", -1.0), ("g2", "g2", -1.0), ("g3", "g3", -1.0), ("g5", "g5", 1.0),
               ("g5g1", "g5g1", -1.0), ("g5g2", "g5g2", -1.0), ("g5g3", "g5g3", -1.0), ("g0g1", "g0g1", -1.0),
               ("g0g2", "g0g2", -1.0), ("g0g3", "g0g3", -1.0), ("g0g5", "g0g5", 1.0), ("g0g5g1", "g0g5g2", 1.0),
               ("g0g5g2", "g0g5g3", 1.0), ("g0g5g3", "g0g5g3", 1.0), ("g5_g0g5", "g5_g0g5", 1.0))


def meson_print_values(raw, method, hits, vol3):
    """{label: values} as meson_measure prints them (print_correlator, mesons.cpp:131-148):
    sign / (norm * hits) with norm = vol3 for SEMWALL and 1 for POINT."""
    norm = vol3 if method == SEMWALL else 1
    idx = {c: k for k, c in enumerate(MESON_CHANNELS)}
    return {lab: sign / (norm * hits) * np.asarray(raw[idx[ch]]) for lab, ch, sign in MESON_PRINT}


CFG_IDENT, CFG_VERSION = 0x47464359, 0x20          # include/gaugefield.h:20-21
_CFG_HEADER = np.dtype([("ident", "<i4"), ("version", "<i4"), ("dim_t", "<i4"), ("dim_x", "<i4"),
                        ("dim_y", "<i4"), ("dim_z", "<i4"), ("nc", "<i4"), ("repr", "<i4"),
                        ("num_cnfg", "<i4"), ("num_accept", "<i4"), ("plaquette", "<f8"),
                        ("reserved", "V208")])      # header_t, packed, 256 bytes


def _file_order(dims, eo=True):
    """site ids of the lexicographic t, x, y, z loop (ipt, geometry.cpp:756-878): the
    even-odd order with even-odd preconditioning, the loop index itself without"""
    T, X, Y, Z = dims
    V = T * X * Y * Z
    lex = np.arange(V)
    if not eo:
        return lex
    t, r = np.divmod(lex, X * Y * Z)
    x, r = np.divmod(r, Y * Z)
    y, z = np.divmod(r, Z)
    return (((t + x + y + z) & 1) * V + lex) // 2


def _links_to_file(U, dims, dtype, eo=True):
    """(V,4,N,N) complex -> the per-site (re, im) interleaved doubles of suNg::write"""
    nc = U.shape[-1]
    u = U[_file_order(dims, eo)].reshape(-1, 4, nc * nc)
    out = np.empty(u.shape + (2,), dtype=dtype)
    out[..., 0] = u.real
    out[..., 1] = u.imag
    return out.reshape(-1)


def _links_from_file(raw, dims, nc, eo=True):
    V = int(np.prod(dims))
    r = np.asarray(raw, dtype=np.float64).reshape(V, 4, nc * nc, 2)
    u = (r[..., 0] + 1j * r[..., 1]).reshape(V, 4, nc, nc)
    U = np.empty_like(u)
    U[_file_order(dims, eo)] = u
    return U


def cfg_write(path, U, dims, nc, repr_id, plaquette, num_cnfg=0, num_accept=0, eo=True):
    h = np.zeros(1, dtype=_CFG_HEADER)
    h["ident"], h["version"] = CFG_IDENT, CFG_VERSION
    h["dim_t"], h["dim_x"], h["dim_y"], h["dim_z"] = dims
    h["nc"], h["repr"], h["num_cnfg"], h["num_accept"], h["plaquette"] = nc, repr_id, num_cnfg, num_accept, plaquette
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(_links_to_file(U, dims, "<f8", eo).tobytes())


def cfg_read(path, eo=True):
    with open(path, "rb") as f:
        h = np.frombuffer(f.read(_CFG_HEADER.itemsize), dtype=_CFG_HEADER)[0]
        dims = (int(h["dim_t"]), int(h["dim_x"]), int(h["dim_y"]), int(h["dim_z"]))
        nc = int(h["nc"])
        raw = np.frombuffer(f.read(), dtype="<f8")
    return {"ident": int(h["ident"]), "version": int(h["version"]), "dims": dims, "nc": nc, "repr": int(h["repr"]),
            "num_cnfg": int(h["num_cnfg"]), "num_accept": int(h["num_accept"]), "plaquette": float(h["plaquette"]),
            "U": _links_from_file(raw, dims, nc, eo)}


def hirep_write(path, U, dims, nc, plaquette, eo=True):
    with open(path, "wb") as f:
        f.write(np.array([nc, *dims], dtype=">i4").tobytes())
        f.write(np.array([plaquette], dtype=">f8").tobytes())
        f.write(_links_to_file(U, dims, ">f8", eo).tobytes())


def hirep_read(path, eo=True):
    with open(path, "rb") as f:
        info = np.frombuffer(f.read(20), dtype=">i4")
        plaq = float(np.frombuffer(f.read(8), dtype=">f8")[0])
        raw = np.frombuffer(f.read(), dtype=">f8").astype(np.float64)
    nc, dims = int(info[0]), tuple(int(v) for v in info[1:5])
    return {"nc": nc, "dims": dims, "plaquette": plaq, "U": _links_from_file(raw, dims, nc, eo)}
