"""Writes yahmc_b200/data/rational_order12.json: the order-12 rational approximation of
x^(-1/2) from the reference's own table (include/approx.h), rescaled to the spectral bound 8,
with its partial-fraction residues, computed by the reference's rational.cpp functions
(rescale, residue) through the compiled reference (oracle/_ref, yref_rational_order).

This is the pole set of the RHMC force and action (monomials/rhmc.cpp:46-57 ask rational_find
for x^(-1/2)) at a fixed order of 12, as the batched-solve benchmark uses it; the reference's
own rational_find would pick a higher order for a spectral range as wide as [1e-4, 8], so the
approximation is valid on the narrower interval stored with it.

Usage:  python oracle/make_rational_fixture.py
"""
import ctypes
import json
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))

from oracle import ref as oref   # noqa: E402


def main():
    R = oref.get("su2_adj_ap", (8, 8, 8, 8))
    out = np.zeros(5 + 2 * 48)
    R.lib.yref_rational_order.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
    rc = R.lib.yref_rational_order(-1, 2, 12, 8.0, out.ctypes.data_as(ctypes.c_void_p))
    if rc != 0:
        raise SystemExit("no order-12 entry for x^(1/2) in the table")
    n = int(out[0])
    # rescale() multiplies the poles by k = 8 / (table maximum) and divides the stored interval by
    # k; the interval on which the rescaled approximation holds is the table's times k
    k = np.sqrt(8.0 / out[4])
    data = {"power": "-1/2", "order": n, "a0": out[1], "table_precision": out[2],
            "valid_interval": [out[3] * k * k, out[4] * k * k],
            "poles": out[5:5 + n].tolist(), "residues": out[5 + n:5 + 2 * n].tolist(),
            "source": "reference include/approx.h through rational.cpp rescale()/residue(), "
                      "oracle/make_rational_fixture.py"}
    dst = HERE.parent / "yahmc_b200" / "data" / "rational_order12.json"
    dst.parent.mkdir(exist_ok=True)
    dst.write_text(json.dumps(data, indent=1) + "\n")
    print(dst)


if __name__ == "__main__":
    main()
