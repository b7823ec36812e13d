"""Shared test helpers: seeded inputs and paired (GPU engine, CPU oracle) set-ups."""
import numpy as np

from oracle import yahmc_oracle as yo
from yahmc_b200 import fields

# name -> (nc, repr, bc, clover, eo); covers every representation, boundary condition and
# the clover / no-clover, even-odd / full variants of the reference's compile-time switches
CONFIGS = {
    "su3_fund_ap": (3, "fundamental", "antiperiodic", True, True),
    "su3_fund_per": (3, "fundamental", "periodic", True, True),
    "su3_fund_open": (3, "fundamental", "open", True, True),
    "su3_fund_sf": (3, "fundamental", "sf", True, True),
    "su3_fund_ap_nocl": (3, "fundamental", "antiperiodic", False, True),
    "su3_fund_ap_full": (3, "fundamental", "antiperiodic", True, False),
    "su3_fund_ap_full_nocl": (3, "fundamental", "antiperiodic", False, False),
    "su2_fund_ap": (2, "fundamental", "antiperiodic", True, True),
    "su2_adj_ap": (2, "adjoint", "antiperiodic", True, True),
    "su2_sym_ap": (2, "symmetric", "antiperiodic", True, True),
    "su2_asym_ap": (2, "antisymmetric", "antiperiodic", True, True),
    "su3_sym_ap": (3, "symmetric", "antiperiodic", True, True),
    "su3_asym_ap": (3, "antisymmetric", "antiperiodic", True, True),
    "su3_adj_ap": (3, "adjoint", "antiperiodic", True, True),
    "su4_fund_ap": (4, "fundamental", "antiperiodic", True, True),
    "su4_asym_ap": (4, "antisymmetric", "antiperiodic", True, True),
    "su4_sym_ap": (4, "symmetric", "periodic", True, True),
    "su4_adj_ap": (4, "adjoint", "antiperiodic", True, True),
}


def rel(a, b, floor=1e-300):
    """max |a-b| / max |b|; `floor` bounds the denominator from below for fields that are
    zero up to rounding (e.g. the clover term of a one-dimensional representation)."""
    return float(np.abs(a - b).max() / max(np.abs(b).max(), floor))


def make_pair(name, dims, seed=0, csw=1.0, cf=1.0):
    """A GPU lattice and the oracle for the same configuration, with the same seeded
    Haar-random links.  Returns (lat, oracle, rng)."""
    from yahmc_b200 import Lattice
    nc, rep, bc, clover, eo = CONFIGS[name]
    lat = Lattice(dims, nc=nc, repr=rep, bc=bc, clover=clover, eo=eo, csw=csw, cf=cf)
    O = yo.Oracle(yo.Params(tuple(dims), nc, rep, bc, clover, eo, csw, cf))
    rng = np.random.default_rng(seed)
    U = fields.haar_su(nc, O.V * 4, rng).reshape(O.V, 4, nc, nc)
    lat.set_links(U)
    O.set_links(U)
    return lat, O, rng


def source(O, rng):
    s = fields.gaussian_spinor(O.V, O.d, rng)
    O.bcs_on_spinor(s)          # spinor_random applies the boundary conditions (linalg.cpp:42-53)
    return s
