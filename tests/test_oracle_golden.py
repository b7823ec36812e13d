"""Pin the numpy oracle to the golden vectors made from the compiled reference.

tests/golden/*.npz hold the reference's outputs (tests/golden/make_golden.py) on seeded
8^4 inputs; this test needs no reference sources.  Tolerance: 1e-12 relative for the
FP64 operator, clover and force outputs, 1e-9 for solver solutions (prec 1e-24), and the
iteration counts to +-2.
"""
import os

import numpy as np
import pytest

from tests.golden.inputs import CASES, compare, config, inputs, load, oracle_for

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def oracle_outputs(name):
    nc, rep, bc, clover, eo = config(name)
    O = oracle_for(name)
    U, src, src2, _ = inputs(name)
    O.set_links(U)
    out = {"repr_links": O.links}
    if clover:
        out["clover_term"] = O.cl_term
        out["logdet"] = np.array(O.clover_logdet(-0.75))
    ops = [("Dphi", -0.75), ("Hphi", -0.3), ("Hphi_sq", -0.75)]
    if eo:
        ops += [("Dphi_oe", None), ("Dphi_eo", None)]
        if clover:
            ops += [("Dphi_ee", -0.75), ("Dphi_oo", 0.2), ("Dphi_oo_inv", -0.75)]
    for fn, mass in ops:
        s, d = src.copy(), O.new_field()
        getattr(O, fn)(*([mass] if mass is not None else []), d, s)
        out[fn], out[fn + ":src"] = d, s
    for fn, opn in [("cg", "Hphi_sq"), ("bicgstab", "Dphi"), ("minres", "Hphi")]:
        x = O.new_field()
        out[f"{fn}:iters"] = np.array(getattr(O, fn)(opn, -0.2, 1e-24, x, src.copy()))
        out[f"{fn}:x"] = x
    it, xs = O.cg_mshift("Hphi_sq", -0.2, 1e-24, [0.1, 0.5], src.copy())
    out["mshift:x0"], out["mshift:x1"], out["mshift:iters"] = xs[0], xs[1], np.array(it)
    O.mom[:] = 0
    O.begin_fermion_force()
    O.wilson_fermion_force(0.1, -0.75, 1.3, src.copy(), src2.copy())
    out["mom_wff"] = O.mom.copy()
    if clover:
        out["cl_force"] = O.cl_force.copy()
        if eo:
            O.clover_logdet_force(-0.75, 2.0)
        O.end_fermion_force(0.1)
        out["mom_end"] = O.mom.copy()
    return out


def check(gold, got):
    for key, summary in gold.items():
        assert key in got, key
        if key.endswith(":iters"):
            assert abs(int(got[key]) - int(summary["scalar"])) <= 2, key
            continue
        tol = 1e-9 if (":x" in key) else 1e-12
        err = compare(summary, got[key], tol)
        assert err < tol, (key, err)


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_golden(name):
    path = os.path.join(HERE, f"{name}.npz")
    assert os.path.exists(path), f"missing golden file {path}"
    check(load(path), oracle_outputs(name))
