"""Generate the golden vectors in tests/golden/ from the compiled reference (oracle/_ref).

The reference ships no golden vectors, so these are made here: seeded inputs (regenerated
bit-for-bit from the seeds by tests/golden/inputs.py) are fed to the UNMODIFIED reference
compiled from its sources, and its outputs are stored compactly -- every field at a fixed
sample of sites plus its full squared norm and its inner product with a seeded probe
field -- so that machines without the reference sources can still pin the oracle and the
CUDA engine.

Usage:  python tests/golden/make_golden.py      (needs oracle/_ref; run oracle/build_ref.py)
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref as oref                      # noqa: E402
from oracle import yahmc_oracle as yo               # noqa: E402
from tests.golden.inputs import CASES, DIMS, inputs, summarize  # noqa: E402


def make(name):
    nc, rep, bc, clover, eo = oref.CONFIGS[name]
    R = oref.get(name, DIMS)
    U, src, src2, probe = inputs(name)
    V = U.shape[0]
    d = yo.repr_dim(nc, rep)
    R.set_links(yo.mat_to_raw(U))
    out = {}
    out["repr_links"] = yo.mat_from_raw(R.repr_links(), d).reshape(V, 4, d, d)
    if clover:
        out["clover_term"] = yo.mat_from_raw(R.clover_term(), d).reshape(V, 4, d, d)
        out["logdet"] = np.array(R.call("clover_logdet", -0.75))
    ops = [("Dphi", -0.75), ("Hphi", -0.3), ("Hphi_sq", -0.75)]
    if eo:
        ops += [("Dphi_oe", None), ("Dphi_eo", None)]
        if clover:
            ops += [("Dphi_ee", -0.75), ("Dphi_oo", 0.2), ("Dphi_oo_inv", -0.75)]
    for fn, mass in ops:
        s = yo.spinor_to_raw(src)
        dd = R.spinor()
        R.call(fn, *([mass] if mass is not None else []), dd, s)
        out[fn] = yo.spinor_from_raw(dd, d)
        out[fn + ":src"] = yo.spinor_from_raw(s, d)
    for fn, op, opn in [("cg", 2, "Hphi_sq"), ("bicgstab", 0, "Dphi"), ("minres", 1, "Hphi")]:
        x = R.spinor()
        it = R.call(fn, op, -0.2, 1e-24, x, yo.spinor_to_raw(src))
        out[f"{fn}:x"] = yo.spinor_from_raw(x, d)
        out[f"{fn}:iters"] = np.array(it)
    xs = np.zeros(2 * V * 8 * d)
    it = R.call("cg_mshift", 2, -0.2, 1e-24, 2, np.array([0.1, 0.5]), xs, yo.spinor_to_raw(src))
    xs = yo.spinor_from_raw(xs, d).reshape(2, V, d, 4)
    out["mshift:x0"], out["mshift:x1"], out["mshift:iters"] = xs[0], xs[1], np.array(it)
    R.zero_momenta()
    R.call("begin_fermion_force")
    R.call("wilson_fermion_force", 0.1, -0.75, 1.3, yo.spinor_to_raw(src), yo.spinor_to_raw(src2))
    out["mom_wff"] = R.momenta().reshape(V, 4, -1)
    if clover:
        out["cl_force"] = yo.mat_from_raw(R.clover_force(), d).reshape(V, 6, d, d)
        if eo:
            R.call("clover_logdet_force", -0.75, 2.0)
        R.call("end_fermion_force", 0.1)
        out["mom_end"] = R.momenta().reshape(V, 4, -1)
    return {k: summarize(v) for k, v in out.items()}


def main():
    if not oref.available("su3_fund_ap"):
        raise SystemExit("oracle/_ref not built: python oracle/build_ref.py")
    for name in CASES:
        g = make(name)
        flat = {}
        for k, parts in g.items():
            for pk, pv in parts.items():
                flat[f"{k}|{pk}"] = pv
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **flat)
        print(path, os.path.getsize(path))


if __name__ == "__main__":
    main()
