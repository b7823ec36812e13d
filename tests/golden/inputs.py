"""Seeded inputs and the compact summary used by the golden vectors (tests/golden/*.npz).

Inputs are regenerated from fixed seeds with numpy's PCG64 generator; the links are Haar
SU(N) matrices (QR of a complex Gaussian matrix), the sources complex Gaussians with the
boundary conditions applied, as spinor_random does (linalg.cpp:42-53).
"""
from __future__ import annotations

import numpy as np

from oracle import yahmc_oracle as yo
from yahmc_b200 import fields

DIMS = (8, 8, 8, 8)          # the smallest lattice the reference accepts (geometry.cpp:1140-1144)
# configs of oracle/build_ref.py that have golden vectors
CASES = ["su3_fund_ap", "su3_fund_open", "su2_adj_ap", "su3_sym_ap", "su3_fund_ap_nocl"]
SEEDS = {"su3_fund_ap": 101, "su3_fund_open": 102, "su2_adj_ap": 103, "su3_sym_ap": 104, "su3_fund_ap_nocl": 105}
N_SAMPLE = 24


def config(name):
    from oracle.ref import CONFIGS
    return CONFIGS[name]


def oracle_for(name):
    nc, rep, bc, clover, eo = config(name)
    return yo.Oracle(yo.Params(DIMS, nc, rep, bc, clover, eo, 1.0, 1.0))


def inputs(name):
    nc, rep, bc, clover, eo = config(name)
    O = oracle_for(name)
    rng = np.random.default_rng(SEEDS[name])
    U = fields.haar_su(nc, O.V * 4, rng).reshape(O.V, 4, nc, nc)
    src = fields.gaussian_spinor(O.V, O.d, rng)
    O.bcs_on_spinor(src)
    src2 = fields.gaussian_spinor(O.V, O.d, rng)
    O.bcs_on_spinor(src2)
    probe = np.random.default_rng(SEEDS[name] + 1000)
    return U, src, src2, probe


def sample_sites(n_sites):
    return np.random.default_rng(7).choice(n_sites, size=min(N_SAMPLE, n_sites), replace=False)


def summarize(v, probe_rng=None):
    """Sampled rows + squared norm + inner product with a fixed probe of the same shape."""
    v = np.asarray(v)
    if v.ndim == 0:
        return {"scalar": v}
    sites = sample_sites(v.shape[0])
    rng = np.random.default_rng(v.size)
    probe = rng.standard_normal(v.shape) + (1j * rng.standard_normal(v.shape) if np.iscomplexobj(v) else 0)
    return {"sample": v[sites], "sqnorm": np.array(np.sum(np.abs(v) ** 2)),
            "probe": np.array(np.sum(np.conj(probe) * v))}


def compare(summary, v, tol):
    """Max relative deviation of v's summary from a stored summary."""
    if "scalar" in summary:
        s = float(summary["scalar"])
        return abs(float(v) - s) / max(abs(s), 1.0)
    got = summarize(v)
    scale = max(np.abs(summary["sample"]).max(), 1e-300)
    e1 = np.abs(got["sample"] - summary["sample"]).max() / scale
    e2 = abs(got["sqnorm"] - summary["sqnorm"]) / max(abs(summary["sqnorm"]), 1e-300)
    e3 = abs(got["probe"] - summary["probe"]) / max(np.sqrt(abs(summary["sqnorm"]) * v.size), 1e-300)
    return float(max(e1, e2, e3))


def load(path):
    z = np.load(path)
    out = {}
    for key in z.files:
        k, part = key.split("|")
        out.setdefault(k, {})[part] = z[key]
    return out
