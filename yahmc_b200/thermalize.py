"""Gauge-field generation on the GPU: pure-gauge HMC trajectories through the engine's
molecular-dynamics entry points, and periodic tiling of a field onto a larger lattice.

The trajectory follows the reference's update() (update.cpp:280-339): back up the links,
refresh the momenta, H = (TF/2) sum P^2 + S_gauge, integrate, accept with probability
min(1, exp(-dH)), reunitarize on acceptance, restore on rejection.  The integrator is the
second-order minimal-norm scheme of integrator.cpp:41-62 (or the leap-frog of :21-38) on a
single gauge level.  Only the
momentum generator differs from the reference (Philox instead of ranlux), so the chain is
the same Markov process, not the same sample path.
"""
from __future__ import annotations

import math

import numpy as np


def leapfrog(lat, beta, c0, length, steps):
    """o2lf_multilevel with one gauge level (integrator.cpp:21-38)."""
    dt = length / steps
    c1 = (1.0 - c0) / 8.0

    def force(h):
        if abs(c1) > 1e-8:
            lat.improved_gauge_force(h, beta, c0, c1)
        else:
            lat.wilson_gauge_force(h, beta)

    for n in range(steps):
        force(dt / 2 if n == 0 else dt)
        lat.update_links(dt)
    force(dt / 2)


def minimal_norm(lat, beta, c0, length, steps):
    """o2mn_multilevel with one gauge level (integrator.cpp:41-62): the second-order
    minimal-norm (Omelyan) scheme, lambda = 0.1931833275037836."""
    a = 0.1931833275037836
    dt = length / steps
    c1 = (1.0 - c0) / 8.0

    def force(h):
        if abs(c1) > 1e-8:
            lat.improved_gauge_force(h, beta, c0, c1)
        else:
            lat.wilson_gauge_force(h, beta)

    for n in range(steps):
        force(a * dt if n == 0 else 2 * a * dt)
        lat.update_links(dt / 2)
        force((1 - 2 * a) * dt)
        lat.update_links(dt / 2)
    force(a * dt)


INTEGRATORS = {"o2lf": leapfrog, "o2mn": minimal_norm}


def hmc_trajectory(lat, beta, c0, length, steps, seed, rng, integrator="o2mn", metropolis=True):
    """One pure-gauge HMC trajectory; returns (accepted, dH).  metropolis=False accepts
    unconditionally (a molecular-dynamics warm-up trajectory, for starts far from
    equilibrium)."""
    lat.gauge_backup()
    lat.momenta_gaussian(seed)
    h0 = lat.momenta_action() + lat.gauge_action(beta, c0)
    INTEGRATORS[integrator](lat, beta, c0, length, steps)
    h1 = lat.momenta_action() + lat.gauge_action(beta, c0)
    dh = h1 - h0
    p = 1.0 if dh < 0 else math.exp(-dh)
    accepted = bool(rng.uniform() < p) or not metropolis
    if accepted:
        lat.reunitarize()
    else:
        lat.gauge_restore()
    return accepted, dh


def thermalize(lat, beta, n_traj, steps=100, length=1.0, c0=1.0, seed=1, integrator="o2mn", n_warm=0, log=None):
    """n_traj pure-gauge HMC trajectories from the field currently on the lattice, the first
    n_warm of them without the accept/reject step.  The represented links (and clover
    term) are rebuilt at the end.  Returns the list of (accepted, dH, plaquette)."""
    rng = np.random.default_rng(seed)
    hist = []
    for k in range(n_traj):
        acc, dh = hmc_trajectory(lat, beta, c0, length, steps, (seed << 20) + k, rng, integrator, k >= n_warm)
        plaq = lat.plaquette()
        hist.append((acc, dh, plaq))
        if log:
            log(f"trajectory {k}: accepted={acc} dH={dh:.4e} plaquette={plaq:.6f}")
    lat.represent_gauge_field()
    return hist


def site_coords(dims):
    """(V, 4) coordinates (t, x, y, z) of the engine's even-odd site order: site id holds
    lexicographic index lex with parity p = (t+x+y+z) mod 2 at id = (p V + lex) // 2
    (geometry.cpp ordering with UPDATE_EO)."""
    T, X, Y, Z = dims
    V = T * X * Y * Z
    lex = np.arange(V)
    t, r = np.divmod(lex, X * Y * Z)
    x, r = np.divmod(r, Y * Z)
    y, z = np.divmod(r, Z)
    p = (t + x + y + z) & 1
    ids = (p * V + lex) // 2
    out = np.empty((V, 4), dtype=np.int64)
    out[ids] = np.stack([t, x, y, z], axis=1)
    return out


def site_index(dims, c):
    """even-odd site id of coordinates c (..., 4)"""
    T, X, Y, Z = dims
    V = T * X * Y * Z
    c = np.asarray(c)
    lex = ((c[..., 0] * X + c[..., 1]) * Y + c[..., 2]) * Z + c[..., 3]
    p = c.sum(axis=-1) & 1
    return (p * V + lex) // 2


def tile(U_small, small_dims, big_dims):
    """Periodic tiling: U_big(t,x,y,z) = U_small(t mod T', x mod X', ...).  Each big
    extent must be a multiple of the small one; the result is again a periodic field with
    the same local action density.  U arrays are (V, 4, N, N) in even-odd site order."""
    for b, s in zip(big_dims, small_dims):
        if b % s:
            raise ValueError("tile: big extents must be multiples of the small ones")
    cb = site_coords(big_dims)
    src = site_index(small_dims, cb % np.asarray(small_dims))
    return np.ascontiguousarray(U_small[src])
