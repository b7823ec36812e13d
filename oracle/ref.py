"""ctypes access to the compiled reference in oracle/_ref (test infrastructure).

Each ``libyahmc_ref_<config>.so`` holds the reference's global state (geometry,
links, clover term) for one compile-time configuration.  The reference can set
its geometry up only once per process, so every (config, lattice size) pair is
served by its own private copy of the library file, loaded under a distinct
path (dlopen then gives it separate globals).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg use
this; the product never does.
"""
from __future__ import annotations

import ctypes
import os
import shutil
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"

_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.c_void_p

# reference configuration name -> (nc, repr, bc, clover, eo); mirrors oracle/build_ref.py
CONFIGS = {
    "su3_fund_ap":      (3, "fundamental",   "antiperiodic", True,  True),
    "su3_fund_per":     (3, "fundamental",   "periodic",     True,  True),
    "su3_fund_open":    (3, "fundamental",   "open",         True,  True),
    "su3_fund_sf":      (3, "fundamental",   "sf",           True,  True),
    "su3_fund_ap_nocl": (3, "fundamental",   "antiperiodic", False, True),
    "su3_fund_ap_full": (3, "fundamental",   "antiperiodic", True,  False),
    "su2_fund_ap":      (2, "fundamental",   "antiperiodic", True,  True),
    "su2_adj_ap":       (2, "adjoint",       "antiperiodic", True,  True),
    "su3_sym_ap":       (3, "symmetric",     "antiperiodic", True,  True),
    "su3_asym_ap":      (3, "antisymmetric", "antiperiodic", True,  True),
    "su3_adj_ap":       (3, "adjoint",       "antiperiodic", True,  True),
    "su4_fund_ap":      (4, "fundamental",   "antiperiodic", True,  True),
    "su4_asym_ap":      (4, "antisymmetric", "antiperiodic", True,  True),
}

_cache: dict = {}


def available(name: str = "su3_fund_ap") -> bool:
    return (REF_DIR / f"libyahmc_ref_{name}.so").exists()


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_P)


class RefLattice:
    """One initialised instance of the reference for (config, dims)."""

    def __init__(self, name: str, dims, csw=1.0, cf=1.0, threads=0, seed=1234, log_level=-1, kind="ref"):
        """kind "ref": the reference compiled for the CPU; kind "shim": the same sources with
        the eight files integration/yahmc_gpu_shim.cpp replaces taken out, running on the
        engine (needs a GPU)."""
        src = REF_DIR / f"libyahmc_{kind}_{name}.so"
        if not src.exists():
            raise FileNotFoundError(f"{src} missing: run oracle/build_ref.py" + (" --shim" if kind == "shim" else ""))
        self.kind = kind
        tmpdir = Path(tempfile.mkdtemp(prefix="yref_"))
        dst = tmpdir / f"libyahmc_ref_{name}_{'x'.join(map(str, dims))}.so"
        shutil.copy(src, dst)
        self.lib = lib = ctypes.CDLL(str(dst), mode=ctypes.RTLD_LOCAL)
        os.unlink(dst)
        self.name = name
        self.dims = tuple(dims)
        threads = threads or os.cpu_count() or 1
        lib.yref_init.argtypes = [_I, _I, _I, _I, _D, _D, _I, _I, _I]
        rc = lib.yref_init(*self.dims, csw, cf, threads, seed, log_level)
        if rc != 0:
            raise RuntimeError(f"yref_init failed: {rc}")
        info = (ctypes.c_int * 10)()
        lib.yref_info(info)
        self.nc, self.d, self.ng, self.repr_id, clover, eo, bc = list(info)[:7]
        self.clover = bool(clover)
        self.eo = bool(eo)
        self.bc = ("periodic", "antiperiodic", "open", "sf")[bc]
        self.spinor_doubles = 8 * self.d
        lib.yref_volume.restype = ctypes.c_long
        self.V = int(lib.yref_volume())
        self.csw = csw
        self.cf = cf
        for fn in ("yref_spinor_sqnorm", "yref_spinor_product_re", "yref_clover_logdet",
                   "yref_timestamp", "yref_avr_wilson", "yref_hamiltonian", "yref_hmc_hamiltonian"):
            getattr(lib, fn).restype = _D
        for fn, args in {
            "yref_Dphi_ee": [_D, _P, _P], "yref_Dphi_oo": [_D, _P, _P], "yref_Dphi_oo_inv": [_D, _P, _P],
            "yref_Dphi": [_D, _P, _P], "yref_Hphi": [_D, _P, _P], "yref_Hphi_sq": [_D, _P, _P],
            "yref_get_ldl": [_D, _P], "yref_clover_logdet": [_D],
            "yref_spinor_sqnorm": [_P, _I], "yref_spinor_product_re": [_P, _P, _I],
            "yref_spinor_product": [_P, _P, _I, _P], "yref_spinor_axpy": [_I, _P, _D, _D, _P, _I],
            "yref_cg": [_I, _D, _D, _P, _P], "yref_bicgstab": [_I, _D, _D, _P, _P],
            "yref_minres": [_I, _D, _D, _P, _P], "yref_auto_inverter": [_I, _D, _D, _P, _P],
            "yref_cg_mshift": [_I, _D, _D, _I, _P, _P, _P],
            "yref_rational": [_I, _I, _D, _D, _D, _I, _D, _D, _P, _P, _P],
            "yref_end_fermion_force": [_D],
            "yref_wilson_fermion_force": [_D, _D, _D, _P, _P],
            "yref_wilson_fermion_force_q": [_D, _D, _D, _P],
            "yref_clover_fermion_force": [_D, _P, _P],
            "yref_clover_logdet_force": [_D, _D],
            "yref_wilson_gauge_force": [_D, _D],
            "yref_improved_gauge_force": [_D, _D, _D, _D],
            "yref_avr_wilson": [_I, _I],
            "yref_update_links": [_D], "yref_reunitarize": [], "yref_represent_gauge_field": [],
            "yref_hamiltonian": [],
            "yref_gauge_save": [ctypes.c_char_p], "yref_gauge_load": [ctypes.c_char_p],
            "yref_point_source": [_I, _I, _P], "yref_semwall_source": [_I, _I, _P],
            "yref_calc_propagator": [_D, _D, _P, _P], "yref_rand_store": [_P], "yref_rand_load": [_P, _I], "yref_rand_uniform": [_I, _P],
            "yref_mesons": [_D, _D, _I, _I, ctypes.c_char_p],
            "yref_wf_init": [], "yref_wf_zeta": [_D], "yref_wf_update": [_D], "yref_wf_iterate": [_D],
            "yref_wf_observables": [_P], "yref_wf_fermion_init": [_P, _I], "yref_wf_fermion_iterate": [_D],
            "yref_gauge_save_hirep": [ctypes.c_char_p], "yref_gauge_load_hirep": [ctypes.c_char_p],
            "yref_mre_init": [_I, _I, _D], "yref_mre_store": [_P], "yref_mre_guess": [_P, _P], "yref_mre_reset": [],
            "yref_represent": [_P, _P, _I],
            "yref_hmc_init": [ctypes.c_char_p], "yref_hmc_reset": [], "yref_hmc_hamiltonian": [],
            "yref_hmc_integrate": [_D, _I, _P, _P], "yref_hmc_update": [_D], "yref_hmc_counters": [_P],
            "yref_gauge_backup": [], "yref_gauge_restore": [], "yref_set_momenta": [_P],
            "yref_check_group": [], "yref_check_dirac": [], "yref_check_inverters": [],
        }.items():
            getattr(lib, fn).argtypes = args

    # ---- fields in the reference's raw double layouts
    def spinor(self):
        return np.zeros(self.V * self.spinor_doubles)

    def set_links(self, fund_raw: np.ndarray):
        self.lib.yref_set_links(_ptr(np.ascontiguousarray(fund_raw, dtype=np.float64)))

    def get_links(self):
        out = np.zeros(self.V * 4 * 2 * self.nc * self.nc)
        self.lib.yref_get_links(_ptr(out))
        return out

    def set_random_links(self):
        self.lib.yref_set_random_links()

    def repr_links(self):
        out = np.zeros(self.V * 4 * 2 * self.d * self.d)
        self.lib.yref_get_repr_links(_ptr(out))
        return out

    def clover_term(self):
        out = np.zeros(self.V * 4 * 2 * self.d * self.d)
        self.lib.yref_get_clover_term(_ptr(out))
        return out

    def ldl(self, mass):
        out = np.zeros(self.V * 2 * self.d * (2 * self.d + 1) * 2)
        self.lib.yref_get_ldl(mass, _ptr(out))
        return out

    def clover_force(self):
        out = np.zeros(self.V * 6 * 2 * self.d * self.d)
        self.lib.yref_get_clover_force(_ptr(out))
        return out

    def generators(self):
        f = np.zeros(self.ng * 2 * self.nc * self.nc)
        r = np.zeros(self.ng * 2 * self.d * self.d)
        self.lib.yref_get_generators(_ptr(f), _ptr(r))
        return f, r

    def represent(self, fund_raw: np.ndarray, count: int):
        out = np.zeros(count * 2 * self.d * self.d)
        self.lib.yref_represent(_ptr(out), _ptr(np.ascontiguousarray(fund_raw)), count)
        return out

    def geometry(self):
        c = np.zeros(self.V * 4, dtype=np.int32)
        f = np.zeros(self.V * 4, dtype=np.int32)
        b = np.zeros(self.V * 4, dtype=np.int32)
        self.lib.yref_geometry(c.ctypes.data_as(_P), f.ctypes.data_as(_P), b.ctypes.data_as(_P))
        return c.reshape(-1, 4), f.reshape(-1, 4), b.reshape(-1, 4)

    def momenta(self):
        out = np.zeros(self.V * 4 * self.ng)
        self.lib.yref_get_momenta(_ptr(out))
        return out

    def zero_momenta(self):
        self.lib.yref_zero_momenta()

    def set_momenta(self, raw: np.ndarray):
        self.lib.yref_set_momenta(_ptr(np.ascontiguousarray(raw, dtype=np.float64)))

    # ---- HMC through the reference's own update.cpp / integrator.cpp / monomials
    def hmc_init(self, cfg_text: str):
        rc = self.lib.yref_hmc_init(cfg_text.encode())
        if rc != 0:
            raise RuntimeError(f"yref_hmc_init: {rc}")

    def hmc_integrate(self, length, levels):
        """levels: [(type, steps)] from the outermost level inward; type o2lf/o2mn/o4mn."""
        code = {"o2lf": 0, "o2mn": 1, "o4mn": 2}
        types = np.array([code[t] for t, _ in levels], dtype=np.int32)
        steps = np.array([n for _, n in levels], dtype=np.int32)
        self.lib.yref_hmc_integrate(length, len(levels), types.ctypes.data_as(_P), steps.ctypes.data_as(_P))

    def hmc_counters(self):
        out = np.zeros(2, dtype=np.int32)
        self.lib.yref_hmc_counters(out.ctypes.data_as(_P))
        return int(out[0]), int(out[1])

    # ---- operators / linalg / inverters
    def call(self, fn: str, *args):
        conv = [(_ptr(a) if isinstance(a, np.ndarray) else a) for a in args]
        return getattr(self.lib, "yref_" + fn)(*conv)


def _parse_mesons(text):
    taus, vals = [], {}
    for line in text.splitlines():
        if not line.startswith("[MESONS]"):
            continue
        body = line.split("]", 2)[2]
        if "timeslice" in body:
            taus.append(int(body.split()[-1]))
        elif ": " in body:
            lab, rest = body.split(": ", 1)
            try:
                vals[lab] = np.array([float(v) for v in rest.split()])
            except ValueError:
                pass
    return taus, vals


def mesons(R: "RefLattice", mass, prec, hits, method):
    """The reference's meson_init + meson_measure (observables/mesons.cpp:150-298) on R's
    current links.  Returns (source time slices, {label: printed values}) read from its log."""
    import os
    import tempfile
    if getattr(R, "_meson_log", None) is None:
        fd, R._meson_log = tempfile.mkstemp(prefix="yahmc_ref_mesons_")
        os.close(fd)
    off = os.path.getsize(R._meson_log)
    R.call("mesons", mass, prec, hits, method, R._meson_log.encode())
    with open(R._meson_log) as f:
        f.seek(off)
        return _parse_mesons(f.read())


def shim_available(name: str = "su3_fund_ap") -> bool:
    return (REF_DIR / f"libyahmc_shim_{name}.so").exists()


def get(name: str, dims=(8, 8, 8, 8), **kw) -> RefLattice:
    key = (name, tuple(dims), tuple(sorted(kw.items())))
    if key not in _cache:
        _cache[key] = RefLattice(name, dims, **kw)
    return _cache[key]
