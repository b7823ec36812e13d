"""Host-side field generators and layout helpers (numpy).

These produce gauge fields and sources in the reference's own host layouts,
the layouts the C-ABI upload entry points accept:

* fundamental links: ``4*V`` suNg records ``{re[N*N], im[N*N]}`` in site order
  ``4*id+mu`` (include/gaugefield.h:6-7, include/suN.h:31-33);
* spinor fields: ``V`` Spinor records ``{re[d][4], im[d][4]}`` (include/spinor.h:7-9).

Site ``id`` follows the reference's even-odd order (geometry.cpp:756-878):
``lex = ((t*X+x)*Y+y)*Z+z``, ``id = (parity*V + lex)//2``.
"""
from __future__ import annotations

import numpy as np


def complex_to_raw(m: np.ndarray) -> np.ndarray:
    """(..., a, b) complex -> flat doubles with re block then im block per record."""
    m = np.asarray(m)
    rec = m.reshape((-1,) + m.shape[-2:])
    return np.ascontiguousarray(np.stack([rec.real, rec.imag], axis=1)).reshape(-1)


def raw_to_complex(raw: np.ndarray, a: int, b: int) -> np.ndarray:
    r = np.asarray(raw, dtype=np.float64).reshape(-1, 2, a, b)
    return r[:, 0] + 1j * r[:, 1]


def haar_su(nc: int, n: int, rng: np.random.Generator) -> np.ndarray:
    """n Haar-distributed SU(N) matrices: QR of a complex Gaussian matrix with the
    phases of R's diagonal moved into Q (Mezzadri, Notices AMS 54 (2007) 592), then
    the determinant phase divided out."""
    z = (rng.standard_normal((n, nc, nc)) + 1j * rng.standard_normal((n, nc, nc))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    ph = np.diagonal(r, axis1=-2, axis2=-1)
    ph = ph / np.abs(ph)
    q = q * ph[:, None, :]
    det = np.linalg.det(q)
    q = q * (det ** (-1.0 / nc))[:, None, None]
    return q


def su_algebra_matrix(nc: int, alg: np.ndarray) -> np.ndarray:
    """Anti-Hermitian traceless matrix from algebra coordinates, in the generator
    basis of suNg(suNa&) (library/suNg.cpp:15-58)."""
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
                v = np.sqrt(2.0 / (i * (i + 1)))
                for k in range(i):
                    out[..., k, k] += 1j * v * alg[..., n]
                out[..., i, i] -= 1j * i * v * alg[..., n]
                n += 1
    return out


def random_start_su(nc: int, n: int, rng: np.random.Generator, width: float = 1.0) -> np.ndarray:
    """exp(X) with X from algebra coordinates drawn N(0, width^2/2): the distribution of the
    reference's random start (suNg::random, library/suNg.cpp:375-380, random.h:13-15) for
    width=1.  The exponential is taken exactly through the eigen-decomposition of the
    Hermitian matrix -iX."""
    alg = rng.standard_normal((n, nc * nc - 1)) * (width / np.sqrt(2.0))
    x = su_algebra_matrix(nc, alg)
    w, v = np.linalg.eigh(-1j * x)
    u = np.einsum("nij,nj,nkj->nik", v, np.exp(1j * w), np.conj(v))
    return u


def gaussian_spinor(V: int, d: int, rng: np.random.Generator) -> np.ndarray:
    """Complex Gaussian source, standard deviation 1/sqrt(2) per real component (unit
    variance per complex component), as Spinor::randomize (library/spinor.cpp:538-551)."""
    return (rng.standard_normal((V, d, 4)) + 1j * rng.standard_normal((V, d, 4))) / np.sqrt(2.0)


def eo_index(dims, t, x, y, z, eo=True):
    T, X, Y, Z = dims
    V = T * X * Y * Z
    lex = ((t * X + x) * Y + y) * Z + z
    if not eo:
        return lex
    return ((t + x + y + z) % 2 * V + lex) // 2
