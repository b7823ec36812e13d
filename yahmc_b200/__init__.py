"""yahmc_b200 -- B200 (sm_100a) engine for YaHMC's fermion hot path.

Python mirror of the reference's C++ call surface (dirac.h, inverter.h, linalg.h,
clover.h, forces.h) over the C ABI of include/yahmc_gpu.h, which is implemented by
the in-tree library yahmc_b200/_lib/libyahmc_b200.so (build it with
``python -m yahmc_b200.build``).  There is no CPU fallback: importing works
anywhere, but creating a Lattice needs the library and a CUDA device and raises
otherwise.

Host arrays use the reference's own layouts as complex numpy arrays:
  spinor field  (V, d, 4)       Spinor{re[d][4], im[d][4]}
  fund links    (V, 4, N, N)    gfield_fund[4*id+mu]
  repr links    (V, 4, d, d)    gfield_repr[4*id+mu]
  momenta       (V, 4, NG)      afield_momenta[4*id+mu]
with sites in the reference's order (even-odd: id = (parity*V + lex)//2).
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

from .fields import complex_to_raw, raw_to_complex

__all__ = ["Lattice", "Field", "YGError", "load_library", "LIB_PATH", "cg_inverter_lattices", "Ptc",
           "VIEW_DEFAULT", "VIEW_EVEN", "VIEW_ODD", "VIEW_FULL", "OP_DPHI", "OP_HPHI", "OP_HPHI_SQ"]

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libyahmc_b200.so"

VIEW_DEFAULT, VIEW_EVEN, VIEW_ODD, VIEW_FULL = 0, 1, 2, 3
OP_DPHI, OP_HPHI, OP_HPHI_SQ = 0, 1, 2
_OPS = {"Dphi": OP_DPHI, "Hphi": OP_HPHI, "Hphi_sq": OP_HPHI_SQ}
_BC = {"periodic": 0, "antiperiodic": 1, "open": 2, "sf": 3}
_REPR = {"fundamental": 0, "adjoint": 1, "symmetric": 2, "antisymmetric": 3}
STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_OOM", 4: "MAXITER", 5: "STALL", 6: "NONFINITE", 7: "TIMEOUT"}


class YGError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class _Params(ctypes.Structure):
    _fields_ = [("dims", ctypes.c_int * 4), ("nc", ctypes.c_int), ("repr", ctypes.c_int), ("bc", ctypes.c_int),
                ("clover", ctypes.c_int), ("eo", ctypes.c_int), ("csw", ctypes.c_double), ("cf", ctypes.c_double)]


class _Info(ctypes.Structure):
    _fields_ = [("volume", ctypes.c_long), ("half_volume", ctypes.c_long), ("repr_dim", ctypes.c_int),
                ("nc", ctypes.c_int), ("ng", ctypes.c_int), ("field_doubles", ctypes.c_long),
                ("link_doubles", ctypes.c_long), ("fund_doubles", ctypes.c_long), ("mom_doubles", ctypes.c_long)]


class InvPar(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int), ("mass", ctypes.c_double), ("prec", ctypes.c_double), ("log", ctypes.c_int),
                ("maxiter", ctypes.c_int)]


class MixedOpts(ctypes.Structure):
    _fields_ = [("inner_precision", ctypes.c_int), ("link_reals", ctypes.c_int), ("delta", ctypes.c_double),
                ("link_storage", ctypes.c_int), ("clover_storage", ctypes.c_int), ("escalate", ctypes.c_int)]


class SolveStats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("reliable_updates", ctypes.c_int), ("fallback", ctypes.c_int),
                ("true_residual", ctypes.c_double), ("seconds", ctypes.c_double)]


_lib = None
_D = ctypes.c_double
_I = ctypes.c_int
_P = ctypes.c_void_p

_SIGNATURES = {
    "yg_lattice_create": [ctypes.POINTER(_Params), ctypes.POINTER(_P)], "yg_set_device": [_I],
    "yg_lattice_destroy": [_P], "yg_lattice_query": [_P, ctypes.POINTER(_Info)],
    "yg_set_stream": [_P, _P], "yg_synchronize": [_P],
    "yg_gauge_upload_fund": [_P, _P], "yg_host_register": [_P, ctypes.c_size_t], "yg_host_unregister": [_P],
    "yg_field_alloc": [_P, ctypes.POINTER(_P)], "yg_field_free": [_P, _P],
    "yg_field_upload": [_P, _P, _P], "yg_field_download": [_P, _P, _P],
    "yg_gauge_upload": [_P, _P], "yg_gauge_download": [_P, _P], "yg_repr_links_download": [_P, _P],
    "yg_clover_term_download": [_P, _P], "yg_ldl_download": [_P, _D, _P],
    "yg_Dphi_oe": [_P, _P, _P], "yg_Dphi_eo": [_P, _P, _P], "yg_Dphi_ee": [_P, _D, _P, _P],
    "yg_Dphi_oo": [_P, _D, _P, _P], "yg_Dphi_oo_inv": [_P, _D, _P, _P], "yg_Dphi": [_P, _D, _P, _P],
    "yg_Hphi": [_P, _D, _P, _P], "yg_Hphi_sq": [_P, _D, _P, _P], "yg_mvm_get": [_P], "yg_mvm_reset": [_P],
    "yg_clover_logdet": [_P, _D, _P],
    "yg_spinor_zero": [_P, _P], "yg_spinor_copy": [_P, _P, _P], "yg_spinor_g5": [_P, _P, _I],
    "yg_spinor_sqnorm": [_P, _P, _I, _P], "yg_spinor_product": [_P, _P, _P, _I, _P],
    "yg_spinor_product_re": [_P, _P, _P, _I, _P],
    "yg_spinor_add_assign": [_P, _P, _P, _I], "yg_spinor_sub_assign": [_P, _P, _P, _I],
    "yg_spinor_mulr": [_P, _P, _D, _P, _I], "yg_spinor_mulc": [_P, _P, _D, _D, _P, _I],
    "yg_spinor_mulr_assign": [_P, _P, _D, _I], "yg_spinor_mulc_assign": [_P, _P, _D, _D, _I],
    "yg_spinor_mulr_add_assign": [_P, _P, _D, _P, _I], "yg_spinor_mulc_add_assign": [_P, _P, _D, _D, _P, _I],
    "yg_spinor_mulr_sub_assign": [_P, _P, _D, _P, _I], "yg_spinor_mulc_sub_assign": [_P, _P, _D, _D, _P, _I],
    "yg_cg_inverter": [_P, ctypes.POINTER(InvPar), _P, _P, ctypes.POINTER(_I)],
    "yg_bicgstab_inverter": [_P, ctypes.POINTER(InvPar), _P, _P, ctypes.POINTER(_I)],
    "yg_minres_inverter": [_P, ctypes.POINTER(InvPar), _P, _P, ctypes.POINTER(_I)],
    "yg_auto_inverter": [_P, ctypes.POINTER(InvPar), _P, _P, ctypes.POINTER(_I)],
    "yg_cg_mshift": [_P, ctypes.POINTER(InvPar), _I, _P, _P, _P, ctypes.POINTER(_I)],
    "yg_rational_calc": [_P, ctypes.POINTER(InvPar), _D, _I, _P, _P, _P, _P, ctypes.POINTER(_I)],
    "yg_cg_mixed": [_P, ctypes.POINTER(InvPar), _P, _P, ctypes.POINTER(SolveStats)],
    "yg_cg_mixed_opts": [_P, ctypes.POINTER(InvPar), ctypes.POINTER(MixedOpts), _P, _P, ctypes.POINTER(SolveStats)],
    "yg_cg_inverter_multi": [_P, _P, _I, _P, _P, _P], "yg_bicgstab_inverter_multi": [_P, _P, _I, _P, _P, _P],
    "yg_cg_mixed_multi": [_P, _P, _I, _P, _P, _D, _P],
    "yg_cg_mixed_multi_masses": [_P, _P, _I, _P, _P, _P, _D, _P],
    "yg_inner_hop_profile": [_P, _D, _I, _P, _P],
    "yg_mre_init": [_P, _I, _I, _D, _P], "yg_mre_store": [_P, _P], "yg_mre_guess": [_P, _P, _P],
    "yg_mre_reset": [_P], "yg_mre_free": [_P],
    "yg_create_point_source": [_P, _I, _I, _P], "yg_create_semwall_source": [_P, _I, _I, _P, _P],
    "yg_calc_propagator": [_P, _D, _D, _P, _P, _P], "yg_calc_propagator_multi": [_P, _D, _D, _I, _P, _P, _I, _P],
    "yg_meson_contract": [_P, _I, _I, _P, _I, _P],
    "yg_tune_inner_links": [_P, _D, _P, _P], "yg_cg_inverter_lattices": [_I, _P, _P, _P, _P, _P],
    "yg_cg_inverter_lattices_ex": [_I, _P, _P, _P, _P, _P, ctypes.c_longlong, _P],
    "yg_wf_init": [_P], "yg_wf_zeta": [_P, _D], "yg_wf_update": [_P, _D], "yg_wf_iterate": [_P, _D],
    "yg_wf_observables": [_P, _P, _P, _P], "yg_wf_fermion_init": [_P, _I], "yg_wf_fermion_iterate": [_P, _D, _P, _I],
    "yg_gauge_save_cfg": [_P, ctypes.c_char_p, _I, _I], "yg_gauge_load_cfg": [_P, ctypes.c_char_p, _P, _P, _P],
    "yg_gauge_save_hirep": [_P, ctypes.c_char_p], "yg_gauge_load_hirep": [_P, ctypes.c_char_p, _P, _P],
    "yg_momenta_upload": [_P, _P], "yg_momenta_download": [_P, _P], "yg_momenta_zero": [_P],
    "yg_clover_force_download": [_P, _P], "yg_begin_fermion_force": [_P], "yg_end_fermion_force": [_P, _D],
    "yg_wilson_fermion_force": [_P, _D, _D, _D, _P, _P], "yg_wilson_fermion_force_q": [_P, _D, _D, _D, _P],
    "yg_clover_fermion_force": [_P, _D, _P, _P], "yg_clover_logdet_force": [_P, _D, _D],
    "yg_wilson_gauge_force": [_P, _D, _D], "yg_avr_plaquette": [_P, _P],
    "yg_improved_gauge_force": [_P, _D, _D, _D, _D], "yg_avr_wilson": [_P, _I, _I, _P],
    "yg_gauge_action": [_P, _D, _D, _P], "yg_update_links": [_P, _D], "yg_represent_gauge_field": [_P],
    "yg_reunitarize": [_P], "yg_momenta_gaussian": [_P, ctypes.c_ulonglong], "yg_momenta_action": [_P, _P],
    "yg_gauge_backup": [_P], "yg_gauge_restore": [_P],
    "yg_field_sqnorm_noalloc": [_P, ctypes.c_long, _P, _P],
    "yg_wilson_fermion_force_q_multi": [_P, _D, _D, _I, _P, _P],
    "yg_ptc_create": [_P, _I, _P, _P], "yg_ptc_destroy": [_P], "yg_ptc_set_weights": [_P, _I, _P],
    "yg_ptc_get_weights": [_P, _I, _P], "yg_ptc_layer": [_P, _I, _I, _P, _P], "yg_ptc_apply": [_P, _P, _P],
    "yg_ptc_gradient": [_P, _I, _P, _P, _P, _P], "yg_ptc_backward": [_P, _P, _P, _P],
    "yg_fgcr": [_P, _P, ctypes.POINTER(InvPar), _I, _P, _P, ctypes.POINTER(SolveStats)],
    "yg_solve_learned": [_P, _P, ctypes.POINTER(InvPar), _I, _P, _P, ctypes.POINTER(SolveStats)],
}


def load_library(path: Path | str | None = None):
    """Load the engine library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path or os.environ.get("YAHMC_B200_LIB", LIB_PATH))
    if not p.exists():
        raise RuntimeError(f"{p} not found: build the CUDA library with `python -m yahmc_b200.build`")
    lib = ctypes.CDLL(str(p))
    lib.yg_last_error.restype = ctypes.c_char_p
    lib.yg_launch_count.restype = ctypes.c_long
    lib.yg_launch_count.argtypes = []
    for name, args in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = None if name in ("yg_lattice_destroy", "yg_mvm_reset") else ctypes.c_int
    _lib = lib
    return lib


class Mre:
    """Chronological initial guess (mre.h): store past solutions, extrapolate a guess."""

    def __init__(self, lat, max_, op, mass):
        self.lat, self.lib = lat, lat.lib
        h = ctypes.c_void_p()
        lat._check(self.lib.yg_mre_init(lat.h, int(max_), _OPS[op] if isinstance(op, str) else int(op), mass,
                                        ctypes.byref(h)))
        self.h = h

    def store(self, f): self.lat._check(self.lib.yg_mre_store(self.h, f.ptr))

    def guess(self, dst, src): self.lat._check(self.lib.yg_mre_guess(self.h, dst.ptr, src.ptr))

    def reset(self): self.lat._check(self.lib.yg_mre_reset(self.h))

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.yg_mre_free(self.h)
            self.h = None


class Ptc:
    """The learned preconditioner (yg_ptc_*): a linear gauge-covariant parallel-transport
    network with channels 1 -> C -> ... -> 1 on a lattice.  Weights per layer are complex
    arrays of shape (9, Co, Ci, 4, 4): path, output channel, input channel, spin, spin."""

    def __init__(self, lat, channels):
        self.lat, self.lib = lat, lat.lib
        self.channels = tuple(int(c) for c in channels)
        ch = (ctypes.c_int * len(self.channels))(*self.channels)
        h = ctypes.c_void_p()
        lat._check(self.lib.yg_ptc_create(lat.h, len(self.channels) - 1, ch, ctypes.byref(h)))
        self.h = h

    def shapes(self):
        return [(9, co, ci, 4, 4) for ci, co in zip(self.channels[:-1], self.channels[1:])]

    def set_weights(self, Ws):
        for l, W in enumerate(Ws):
            W = np.ascontiguousarray(np.asarray(W, dtype=complex).reshape(self.shapes()[l]))
            raw = np.ascontiguousarray(W.view(np.float64))
            self.lat._check(self.lib.yg_ptc_set_weights(self.h, l, _ptr(raw)))

    def get_weights(self):
        out = []
        for l, shp in enumerate(self.shapes()):
            raw = np.empty(int(np.prod(shp)) * 2)
            self.lat._check(self.lib.yg_ptc_get_weights(self.h, l, _ptr(raw)))
            out.append(raw.view(complex).reshape(shp).copy())
        return out

    def layer(self, l, adjoint, dev_in: int, dev_out: int):
        """One layer on device activations (site blocks; raw device pointers)."""
        self.lat._check(self.lib.yg_ptc_layer(self.h, int(l), int(adjoint), ctypes.c_void_p(dev_in),
                                              ctypes.c_void_p(dev_out)))

    def apply(self, dst, src):
        self.lat._check(self.lib.yg_ptc_apply(self.h, dst.ptr, src.ptr))

    def gradient(self, pairs):
        """(loss, per-layer complex gradients d loss / d conj(W)) over (r, e) field pairs."""
        n = len(pairs)
        pr = (ctypes.c_void_p * n)(*[r.ptr for r, _ in pairs])
        pe = (ctypes.c_void_p * n)(*[e.ptr for _, e in pairs])
        sizes = [int(np.prod(s)) for s in self.shapes()]
        raw = np.zeros(2 * sum(sizes))
        loss = ctypes.c_double()
        self.lat._check(self.lib.yg_ptc_gradient(self.h, n, pr, pe, ctypes.byref(loss), _ptr(raw)))
        grads, off = [], 0
        for shp, sz in zip(self.shapes(), sizes):
            grads.append(raw[2 * off:2 * (off + sz)].view(complex).reshape(shp).copy())
            off += sz
        return loss.value, grads

    def backward(self, src, gout):
        """Per-layer gradients d loss / d conj(W) given gout = d loss / d conj(N(src))."""
        sizes = [int(np.prod(s)) for s in self.shapes()]
        raw = np.zeros(2 * sum(sizes))
        self.lat._check(self.lib.yg_ptc_backward(self.h, src.ptr, gout.ptr, _ptr(raw)))
        grads, off = [], 0
        for shp, sz in zip(self.shapes(), sizes):
            grads.append(raw[2 * off:2 * (off + sz)].view(complex).reshape(shp).copy())
            off += sz
        return grads

    def __del__(self):
        if getattr(self, "h", None):
            try:
                self.lib.yg_ptc_destroy(self.h)
            except Exception:
                pass
            self.h = None


def set_device(device: int) -> None:
    """CUDA device of the lattices this thread creates next (one process per GPU)."""
    lib = load_library()
    if lib.yg_set_device(int(device)) != 0:
        raise YGError(1, lib.yg_last_error().decode())


def cg_inverter_lattices(solves, op="Hphi_sq", wait_cycles=0, with_path=False):
    """Independent cg_inverter solves on several lattices at once (yg_cg_inverter_lattices_ex):
    `solves` is a list of (lattice, mass, prec, x, b) or (lattice, mass, prec, x, b, maxiter);
    returns (iteration counts, status), plus 1 / 0 for the persistent kernel / the host
    threads when with_path.  wait_cycles bounds each barrier wait of the persistent kernel
    (0: the default); a wait that runs out gives status 7 (YG_TIMEOUT)."""
    lib = load_library()
    n = len(solves)
    lats = (ctypes.c_void_p * n)(*[s[0].h for s in solves])
    pars = (InvPar * n)(*[Lattice._par(op, s[1], s[2], 0, s[5] if len(s) > 5 else 0) for s in solves])
    xs = (ctypes.c_void_p * n)(*[s[3].ptr for s in solves])
    bs = (ctypes.c_void_p * n)(*[s[4].ptr for s in solves])
    its = (ctypes.c_int * n)()
    path = ctypes.c_int(-1)
    rc = lib.yg_cg_inverter_lattices_ex(n, lats, pars, xs, bs, its, int(wait_cycles), ctypes.byref(path))
    if rc not in (0, 4, 7):
        raise YGError(rc, lib.yg_last_error().decode())
    return (list(its), rc, path.value) if with_path else (list(its), rc)


def launch_count() -> int:
    """Kernels launched by the engine library since it was loaded."""
    return int(load_library().yg_launch_count())


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(_P)


class Field:
    """A device spinor field (SpinorField with its storage on the GPU)."""

    def __init__(self, lat: "Lattice"):
        self.lat = lat
        p = _P()
        lat._check(lat.lib.yg_field_alloc(lat.h, ctypes.byref(p)))
        self.ptr = p.value

    def free(self):
        if self.ptr and self.lat.h:
            self.lat.lib.yg_field_free(self.lat.h, self.ptr)
        self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Lattice:
    """One lattice with its device gauge field, clover term and momenta.  Method names and
    argument order follow the reference (dirac.h, inverter.h, linalg.h, forces.h)."""

    def __init__(self, dims, nc=3, repr="fundamental", bc="antiperiodic", clover=True, eo=True,
                 csw=1.0, cf=1.0, lib=None):
        self.lib = lib or load_library()
        p = _Params()
        for i in range(4):
            p.dims[i] = int(dims[i])
        p.nc, p.repr, p.bc = int(nc), _REPR[repr], _BC[bc]
        p.clover, p.eo, p.csw, p.cf = int(bool(clover)), int(bool(eo)), float(csw), float(cf)
        h = _P()
        self.h = None
        self._check(self.lib.yg_lattice_create(ctypes.byref(p), ctypes.byref(h)))
        self.h = h.value
        info = _Info()
        self._check(self.lib.yg_lattice_query(self.h, ctypes.byref(info)))
        self.dims = tuple(int(x) for x in dims)
        self.V, self.Vh, self.d, self.nc, self.ng = info.volume, info.half_volume, info.repr_dim, info.nc, info.ng
        self.field_doubles = info.field_doubles
        self.eo, self.clover, self.bc, self.repr = bool(eo), bool(clover), bc, repr
        self.last_status = 0

    # ---- plumbing
    def _check(self, rc):
        if rc != 0:
            raise YGError(rc, self.lib.yg_last_error().decode())
        return rc

    def close(self):
        if self.h:
            self.lib.yg_lattice_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def synchronize(self):
        self._check(self.lib.yg_synchronize(self.h))

    def set_stream(self, stream_ptr: int):
        self._check(self.lib.yg_set_stream(self.h, stream_ptr))

    # ---- fields
    def field(self, host=None) -> Field:
        f = Field(self)
        if host is not None:
            self.upload(f, host)
        return f

    def upload(self, f: Field, host):
        host = np.asarray(host)
        raw = host if (host.dtype == np.float64 and host.ndim == 1) else complex_to_raw(host)
        raw = np.ascontiguousarray(raw, dtype=np.float64)
        assert raw.size == self.field_doubles
        self._check(self.lib.yg_field_upload(self.h, f.ptr, _ptr(raw)))

    def download(self, f: Field, raw=False, out=None):
        """Field to host; `out` (a contiguous float64 buffer, e.g. pinned) receives the raw
        reference-layout doubles when given."""
        if out is None:
            out = np.empty(self.field_doubles)
        self._check(self.lib.yg_field_download(self.h, _ptr(out), f.ptr))
        return out if raw else raw_to_complex(out, self.d, 4)

    # ---- gauge field (represent_gauge_field, repr.cpp:265-280)
    def set_links(self, fund):
        fund = np.asarray(fund)
        raw = np.ascontiguousarray(complex_to_raw(fund) if np.iscomplexobj(fund) else fund, dtype=np.float64)
        self._check(self.lib.yg_gauge_upload(self.h, _ptr(raw)))

    def get_links(self):
        out = np.empty(self.V * 4 * 2 * self.nc * self.nc)
        self._check(self.lib.yg_gauge_download(self.h, _ptr(out)))
        return raw_to_complex(out, self.nc, self.nc).reshape(self.V, 4, self.nc, self.nc)

    def repr_links(self):
        out = np.empty(self.V * 4 * 2 * self.d * self.d)
        self._check(self.lib.yg_repr_links_download(self.h, _ptr(out)))
        return raw_to_complex(out, self.d, self.d).reshape(self.V, 4, self.d, self.d)

    def clover_term(self):
        out = np.empty(self.V * 4 * 2 * self.d * self.d)
        self._check(self.lib.yg_clover_term_download(self.h, _ptr(out)))
        return raw_to_complex(out, self.d, self.d).reshape(self.V, 4, self.d, self.d)

    def ldl(self, mass):
        P = self.d * (2 * self.d + 1)
        out = np.empty(self.V * 2 * P * 2)
        self._check(self.lib.yg_ldl_download(self.h, mass, _ptr(out)))
        r = out.reshape(self.V, 2, P, 2)
        return r[..., 0] + 1j * r[..., 1]

    # ---- dirac.h
    def Dphi_oe(self, dst, src): self._check(self.lib.yg_Dphi_oe(self.h, dst.ptr, src.ptr))
    def Dphi_eo(self, dst, src): self._check(self.lib.yg_Dphi_eo(self.h, dst.ptr, src.ptr))
    def Dphi_ee(self, m, dst, src): self._check(self.lib.yg_Dphi_ee(self.h, m, dst.ptr, src.ptr))
    def Dphi_oo(self, m, dst, src): self._check(self.lib.yg_Dphi_oo(self.h, m, dst.ptr, src.ptr))
    def Dphi_oo_inv(self, m, dst, src): self._check(self.lib.yg_Dphi_oo_inv(self.h, m, dst.ptr, src.ptr))
    def Dphi(self, m, dst, src): self._check(self.lib.yg_Dphi(self.h, m, dst.ptr, src.ptr))
    def Hphi(self, m, dst, src): self._check(self.lib.yg_Hphi(self.h, m, dst.ptr, src.ptr))
    def Hphi_sq(self, m, dst, src): self._check(self.lib.yg_Hphi_sq(self.h, m, dst.ptr, src.ptr))
    def mvm_get(self): return self.lib.yg_mvm_get(self.h)
    def mvm_reset(self): self.lib.yg_mvm_reset(self.h)

    def clover_logdet(self, mass):
        out = ctypes.c_double()
        self._check(self.lib.yg_clover_logdet(self.h, mass, ctypes.byref(out)))
        return out.value

    # ---- linalg.h
    def spinor_zero(self, f): self._check(self.lib.yg_spinor_zero(self.h, f.ptr))
    def spinor_copy(self, dst, src): self._check(self.lib.yg_spinor_copy(self.h, dst.ptr, src.ptr))
    def spinor_g5(self, f, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_g5(self.h, f.ptr, view))

    def spinor_sqnorm(self, f, view=VIEW_DEFAULT):
        out = ctypes.c_double()
        self._check(self.lib.yg_spinor_sqnorm(self.h, f.ptr, view, ctypes.byref(out)))
        return out.value

    def spinor_product(self, a, b, view=VIEW_DEFAULT):
        out = (ctypes.c_double * 2)()
        self._check(self.lib.yg_spinor_product(self.h, a.ptr, b.ptr, view, out))
        return complex(out[0], out[1])

    def spinor_product_re(self, a, b, view=VIEW_DEFAULT):
        out = ctypes.c_double()
        self._check(self.lib.yg_spinor_product_re(self.h, a.ptr, b.ptr, view, ctypes.byref(out)))
        return out.value

    def spinor_add_assign(self, a, b, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_add_assign(self.h, a.ptr, b.ptr, view))
    def spinor_sub_assign(self, a, b, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_sub_assign(self.h, a.ptr, b.ptr, view))
    def spinor_mulr(self, a, v, b, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_mulr(self.h, a.ptr, v, b.ptr, view))
    def spinor_mulc(self, a, c, b, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_mulc(self.h, a.ptr, c.real, c.imag, b.ptr, view))
    def spinor_mulr_assign(self, a, v, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_mulr_assign(self.h, a.ptr, v, view))
    def spinor_mulc_assign(self, a, c, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_mulc_assign(self.h, a.ptr, c.real, c.imag, view))
    def spinor_mulr_add_assign(self, a, v, b, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_mulr_add_assign(self.h, a.ptr, v, b.ptr, view))
    def spinor_mulc_add_assign(self, a, c, b, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_mulc_add_assign(self.h, a.ptr, c.real, c.imag, b.ptr, view))
    def spinor_mulr_sub_assign(self, a, v, b, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_mulr_sub_assign(self.h, a.ptr, v, b.ptr, view))
    def spinor_mulc_sub_assign(self, a, c, b, view=VIEW_DEFAULT): self._check(self.lib.yg_spinor_mulc_sub_assign(self.h, a.ptr, c.real, c.imag, b.ptr, view))

    # ---- inverter.h
    @staticmethod
    def _par(op, mass, prec, log=0, maxiter=0):
        return InvPar(_OPS[op] if isinstance(op, str) else int(op), float(mass), float(prec), int(log), int(maxiter))

    def _solve(self, fn, op, mass, prec, x, b, log, maxiter, allow=(0, 4)):
        it = ctypes.c_int()
        par = self._par(op, mass, prec, log, maxiter)
        rc = fn(self.h, ctypes.byref(par), x.ptr, b.ptr, ctypes.byref(it))
        if rc not in allow:
            self._check(rc)
        self.last_status = rc
        return it.value

    def cg_inverter(self, op, mass, prec, x, b, log=0, maxiter=0):
        return self._solve(self.lib.yg_cg_inverter, op, mass, prec, x, b, log, maxiter)

    def bicgstab_inverter(self, op, mass, prec, x, b, log=0, maxiter=0):
        return self._solve(self.lib.yg_bicgstab_inverter, op, mass, prec, x, b, log, maxiter)

    def minres_inverter(self, op, mass, prec, x, b, log=0, maxiter=0):
        return self._solve(self.lib.yg_minres_inverter, op, mass, prec, x, b, log, maxiter)

    def auto_inverter(self, op, mass, prec, x, b, log=0, maxiter=0):
        return self._solve(self.lib.yg_auto_inverter, op, mass, prec, x, b, log, maxiter)

    def cg_mshift(self, op, mass, prec, shifts, xs, b, log=0, maxiter=0):
        it = ctypes.c_int()
        par = self._par(op, mass, prec, log, maxiter)
        sh = np.ascontiguousarray(shifts, dtype=np.float64)
        ptrs = (_P * len(xs))(*[x.ptr for x in xs])
        rc = self.lib.yg_cg_mshift(self.h, ctypes.byref(par), len(xs), _ptr(sh), ptrs, b.ptr, ctypes.byref(it))
        if rc not in (0, 4):
            self._check(rc)
        self.last_status = rc
        return it.value

    def rational_calc(self, op, mass, prec, a0, poles, residues, x, b, log=0):
        it = ctypes.c_int()
        par = self._par(op, mass, prec, log, 0)
        po = np.ascontiguousarray(poles, dtype=np.float64)
        re = np.ascontiguousarray(residues, dtype=np.float64)
        self._check(self.lib.yg_rational_calc(self.h, ctypes.byref(par), a0, len(po), _ptr(po), _ptr(re),
                                              x.ptr, b.ptr, ctypes.byref(it)))
        return it.value

    def cg_inverter_multi(self, op, mass, prec, xs, bs, log=0, maxiter=0):
        """len(xs) cg_inverter solves sharing every operator application; returns the
        iteration count of each system"""
        n = len(xs)
        if n != len(bs):
            raise ValueError("xs and bs differ in length")
        par = self._par(op, mass, prec, log, maxiter)
        px = (ctypes.c_void_p * n)(*[x.ptr for x in xs])
        pb = (ctypes.c_void_p * n)(*[b.ptr for b in bs])
        its = (ctypes.c_int * n)()
        rc = self.lib.yg_cg_inverter_multi(self.h, ctypes.byref(par), n, px, pb, its)
        self.last_status = rc
        if rc not in (0, 4):
            self._check(rc)
        return list(its)

    def bicgstab_inverter_multi(self, op, mass, prec, xs, bs, log=0, maxiter=0):
        """len(xs) bicgstab_inverter solves on Dphi sharing every operator application;
        returns the iteration count of each system (2 per iteration, as the reference)"""
        n = len(xs)
        if n != len(bs):
            raise ValueError("xs and bs differ in length")
        par = self._par(op, mass, prec, log, maxiter)
        px = (ctypes.c_void_p * n)(*[x.ptr for x in xs])
        pb = (ctypes.c_void_p * n)(*[b.ptr for b in bs])
        its = (ctypes.c_int * n)()
        rc = self.lib.yg_bicgstab_inverter_multi(self.h, ctypes.byref(par), n, px, pb, its)
        self.last_status = rc
        if rc not in (0, 4):
            self._check(rc)
        return list(its)

    def tune_inner_links(self, mass):
        """times the FP32 link formats of the compressed inner operator on this lattice and
        keeps the fastest for cg_mixed's default; returns (link_reals, {reals: ms per hop})"""
        r = ctypes.c_int()
        ms = np.zeros(3)
        self._check(self.lib.yg_tune_inner_links(self.h, mass, ctypes.byref(r), _ptr(ms)))
        return r.value, {18: ms[0], 12: ms[1], 8: ms[2]}

    # ---- sources, propagators, meson contractions (observables/propagator.cpp, mesons.cpp)
    def create_point_source(self, n, tau, src):
        self._check(self.lib.yg_create_point_source(self.h, int(n), int(tau), src.ptr))

    def create_semwall_source(self, n, tau, src, z2=None):
        """z2: for n = 0, the 2*d*vol3 rand_z2 values (slice sites by increasing index, per site
        re, im of each colour)"""
        zp = None
        if n == 0:
            z2 = np.ascontiguousarray(z2, dtype=np.float64)
            vol3 = self.V // self.dims[0]
            if z2.size != 2 * self.d * vol3:
                raise ValueError(f"z2 needs {2 * self.d * vol3} values")
            zp = _ptr(z2)
        self._check(self.lib.yg_create_semwall_source(self.h, int(n), int(tau), zp, src.ptr))

    def calc_propagator(self, mass, prec, dst, src):
        """calc_propagator; dst holds the initial guess.  Returns the solver's iterations."""
        it = ctypes.c_int()
        rc = self.lib.yg_calc_propagator(self.h, mass, prec, dst.ptr, src.ptr, ctypes.byref(it))
        self.last_status = rc
        if rc not in (0, 4):
            self._check(rc)
        return it.value

    def calc_propagator_multi(self, mass, prec, dsts, srcs, solver="bicgstab"):
        """len(dsts) <= 16 propagators with shared operator applications: solver "bicgstab"
        (batched BiCGstab on the even-site system, dsts hold the initial guesses), "cg_mixed"
        or "cg" (batched CG on Hphi_sq); returns the iteration counts"""
        code = {"bicgstab": 0, "cg_mixed": 1, "cg": 2}[solver]
        n = len(dsts)
        if n != len(srcs):
            raise ValueError("dsts and srcs differ in length")
        pd = (ctypes.c_void_p * n)(*[x.ptr for x in dsts])
        ps = (ctypes.c_void_p * n)(*[b.ptr for b in srcs])
        its = (ctypes.c_int * n)()
        rc = self.lib.yg_calc_propagator_multi(self.h, mass, prec, n, pd, ps, code, its)
        self.last_status = rc
        if rc not in (0, 4):
            self._check(rc)
        return list(its)

    def meson_contract(self, method, tau, props, corr=None):
        """adds the sixteen slice-summed channels of one source slice to corr (16 x T)"""
        T = self.dims[0]
        if corr is None:
            corr = np.zeros((16, T))
        if corr.shape != (16, T) or corr.dtype != np.float64 or not corr.flags.c_contiguous:
            raise ValueError("corr must be a C-contiguous float64 (16, T) array")
        pp = (ctypes.c_void_p * len(props))(*[f.ptr for f in props])
        self._check(self.lib.yg_meson_contract(self.h, int(method), int(tau), pp, len(props), _ptr(corr)))
        return corr

    # ---- Wilson and fermion flow (observables/wilsonflow.cpp, fermionflow.cpp)
    def wf_init(self):
        self._check(self.lib.yg_wf_init(self.h))

    def wf_zeta(self, alpha):
        self._check(self.lib.yg_wf_zeta(self.h, alpha))

    def wf_update(self, val):
        self._check(self.lib.yg_wf_update(self.h, val))

    def wf_iterate(self, eps):
        self._check(self.lib.yg_wf_iterate(self.h, eps))

    def wf_observables(self):
        """(E_plaq, E_sym, topological charge) as wf_e_plaq, wf_e_sym, wf_charge"""
        e, s, q = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.yg_wf_observables(self.h, ctypes.byref(e), ctypes.byref(s), ctypes.byref(q)))
        return e.value, s.value, q.value

    def wf_fermion_init(self, n):
        self._check(self.lib.yg_wf_fermion_init(self.h, int(n)))

    def wf_fermion_iterate(self, eps, phis):
        pp = (ctypes.c_void_p * len(phis))(*[f.ptr for f in phis])
        self._check(self.lib.yg_wf_fermion_iterate(self.h, eps, pp, len(phis)))

    # ---- gauge configuration files (gaugefield.cpp:44-179, hirep.cpp:56-212)
    def gauge_field_save(self, path, num_cnfg=0, num_accept=0):
        self._check(self.lib.yg_gauge_save_cfg(self.h, str(path).encode(), int(num_cnfg), int(num_accept)))

    def gauge_field_load(self, path):
        """returns (num_cnfg, num_accept, |stored - loaded plaquette|)"""
        nc_, na, pd = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.yg_gauge_load_cfg(self.h, str(path).encode(), ctypes.byref(nc_), ctypes.byref(na),
                                               ctypes.byref(pd)))
        return nc_.value, na.value, pd.value

    def gauge_field_save_hirep(self, path):
        self._check(self.lib.yg_gauge_save_hirep(self.h, str(path).encode()))

    def gauge_field_load_hirep(self, path):
        """returns (num_cnfg, |stored - loaded plaquette|)"""
        nc_, pd = ctypes.c_int(), ctypes.c_double()
        self._check(self.lib.yg_gauge_load_hirep(self.h, str(path).encode(), ctypes.byref(nc_), ctypes.byref(pd)))
        return nc_.value, pd.value

    def mre(self, max_, op, mass):
        """mre_init (mre.cpp:85-111): a history of up to max_ past solutions of `op`"""
        return Mre(self, max_, op, mass)

    def inner_hop_profile(self, mass, reps=50):
        """(ms per launch, compulsory bytes per launch) of the mixed solver's dominant kernel"""
        ms, by = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.yg_inner_hop_profile(self.h, mass, int(reps), ctypes.byref(ms), ctypes.byref(by)))
        return ms.value, by.value

    def cg_mixed_multi(self, op, mass, prec, xs, bs, delta=0.1, log=0, maxiter=0, masses=None):
        """len(xs) mixed-precision solves advanced together; one stats dict per system.
        masses (a mass per system, at most 4 distinct) replaces mass."""
        n = len(xs)
        if n != len(bs):
            raise ValueError("xs and bs differ in length")
        par = self._par(op, mass, prec, log, maxiter)
        px = (ctypes.c_void_p * n)(*[x.ptr for x in xs])
        pb = (ctypes.c_void_p * n)(*[b.ptr for b in bs])
        sts = (SolveStats * n)()
        if masses is None:
            rc = self.lib.yg_cg_mixed_multi(self.h, ctypes.byref(par), n, px, pb, float(delta), sts)
        else:
            if len(masses) != n:
                raise ValueError("one mass per system")
            pm = (ctypes.c_double * n)(*[float(m) for m in masses])
            rc = self.lib.yg_cg_mixed_multi_masses(self.h, ctypes.byref(par), n, pm, px, pb, float(delta), sts)
        self.last_status = rc
        if rc not in (0, 4, 5):
            self._check(rc)
        return [{"status": rc, "iterations": st.iterations, "reliable_updates": st.reliable_updates,
                 "fallback": st.fallback, "true_residual": st.true_residual, "seconds": st.seconds} for st in sts]

    def cg_mixed(self, op, mass, prec, x, b, log=0, maxiter=0, inner_precision=None, link_reals=18, delta=0.1,
                 link_storage=0, clover_storage=0, escalate=False):
        """Mixed-precision CG (true FP64 stopping criterion).  inner_precision None: the
        library's choice (yg_cg_mixed); 0: the generic FP32 inner operator; 32 or 16: the
        compressed d = 3 inner operator with link_reals 18, 12 or 8 (8: FP32 links,
        periodic or antiperiodic lattices) and reliable-update threshold delta; link_storage / clover_storage 0 (as the spinors), 32, 16 or 15
        (int16 fixed point)."""
        st = SolveStats()
        par = self._par(op, mass, prec, log, maxiter)
        if inner_precision is None:
            rc = self.lib.yg_cg_mixed(self.h, ctypes.byref(par), x.ptr, b.ptr, ctypes.byref(st))
        else:
            o = MixedOpts(int(inner_precision), int(link_reals), float(delta), int(link_storage), int(clover_storage),
                          int(bool(escalate)))
            rc = self.lib.yg_cg_mixed_opts(self.h, ctypes.byref(par), ctypes.byref(o), x.ptr, b.ptr, ctypes.byref(st))
        if rc not in (0, 4, 5):
            self._check(rc)
        return {"status": rc, "iterations": st.iterations, "reliable_updates": st.reliable_updates,
                "fallback": st.fallback, "true_residual": st.true_residual, "seconds": st.seconds}

    def fgcr(self, mass, prec, x, b, net=None, restart=16, log=0, maxiter=0):
        """Flexible GCR on Dphi with the network `net` (a Ptc, or None) as right preconditioner."""
        st = SolveStats()
        par = self._par("Dphi", mass, prec, log, maxiter)
        rc = self.lib.yg_fgcr(self.h, net.h if net is not None else None, ctypes.byref(par), int(restart), x.ptr,
                              b.ptr, ctypes.byref(st))
        if rc not in (0, 4, 5):
            self._check(rc)
        return {"status": rc, "iterations": st.iterations, "fallback": st.fallback,
                "true_residual": st.true_residual, "seconds": st.seconds}

    def solve_learned(self, mass, prec, x, b, net=None, restart=16, maxiter=0):
        """Hphi_sq x = b as two preconditioned Dphi solves (yg_solve_learned)."""
        st = SolveStats()
        par = self._par("Hphi_sq", mass, prec, 0, maxiter)
        rc = self.lib.yg_solve_learned(self.h, net.h if net is not None else None, ctypes.byref(par), int(restart),
                                       x.ptr, b.ptr, ctypes.byref(st))
        if rc not in (0, 4, 5):
            self._check(rc)
        return {"status": rc, "iterations": st.iterations, "fallback": st.fallback,
                "true_residual": st.true_residual, "seconds": st.seconds}

    # ---- forces.h
    def momenta(self):
        out = np.empty(self.V * 4 * self.ng)
        self._check(self.lib.yg_momenta_download(self.h, _ptr(out)))
        return out.reshape(self.V, 4, self.ng)

    def set_momenta(self, mom):
        raw = np.ascontiguousarray(mom, dtype=np.float64).reshape(-1)
        self._check(self.lib.yg_momenta_upload(self.h, _ptr(raw)))

    def zero_momenta(self): self._check(self.lib.yg_momenta_zero(self.h))

    def clover_force(self):
        out = np.empty(self.V * 6 * 2 * self.d * self.d)
        self._check(self.lib.yg_clover_force_download(self.h, _ptr(out)))
        return raw_to_complex(out, self.d, self.d).reshape(self.V, 6, self.d, self.d)

    def begin_fermion_force(self): self._check(self.lib.yg_begin_fermion_force(self.h))
    def end_fermion_force(self, dt): self._check(self.lib.yg_end_fermion_force(self.h, dt))

    def wilson_fermion_force(self, dt, mass, residue, lhs, rhs):
        self._check(self.lib.yg_wilson_fermion_force(self.h, dt, mass, residue, lhs.ptr, rhs.ptr))

    def wilson_fermion_force_q(self, dt, mass, residue, rhs):
        self._check(self.lib.yg_wilson_fermion_force_q(self.h, dt, mass, residue, rhs.ptr))

    def wilson_fermion_force_q_multi(self, dt, mass, residues, rhs):
        """The pole loop of MonomialRHMC::update as one batched force (yg_wilson_fermion_force_q_multi)."""
        n = len(rhs)
        res = np.ascontiguousarray(residues, dtype=np.float64)
        pr = (ctypes.c_void_p * n)(*[f.ptr for f in rhs])
        self._check(self.lib.yg_wilson_fermion_force_q_multi(self.h, dt, mass, n, _ptr(res), pr))

    def clover_fermion_force(self, residue, lhs, rhs):
        self._check(self.lib.yg_clover_fermion_force(self.h, residue, lhs.ptr, rhs.ptr))

    def clover_logdet_force(self, mass, residue):
        self._check(self.lib.yg_clover_logdet_force(self.h, mass, residue))

    def wilson_gauge_force(self, dt, beta):
        self._check(self.lib.yg_wilson_gauge_force(self.h, dt, beta))

    def plaquette(self):
        out = ctypes.c_double()
        self._check(self.lib.yg_avr_plaquette(self.h, ctypes.byref(out)))
        return out.value

    # ---- molecular dynamics (update.cpp, forces.cpp:262-309, wilsonloop.cpp)
    def improved_gauge_force(self, dt, beta, c0, c1):
        self._check(self.lib.yg_improved_gauge_force(self.h, dt, beta, c0, c1))

    def avr_wilson(self, height, width):
        out = ctypes.c_double()
        self._check(self.lib.yg_avr_wilson(self.h, int(height), int(width), ctypes.byref(out)))
        return out.value

    def gauge_action(self, beta, c0=1.0):
        """MonomialGauge::action with c1 = (1 - c0)/8"""
        out = ctypes.c_double()
        self._check(self.lib.yg_gauge_action(self.h, beta, c0, ctypes.byref(out)))
        return out.value

    def update_links(self, eps):
        """U <- exp(eps P) U on the fundamental links; call represent_gauge_field() before
        the Dirac operator sees them, as in the reference"""
        self._check(self.lib.yg_update_links(self.h, eps))

    def represent_gauge_field(self): self._check(self.lib.yg_represent_gauge_field(self.h))

    def reunitarize(self): self._check(self.lib.yg_reunitarize(self.h))

    def momenta_gaussian(self, seed):
        self._check(self.lib.yg_momenta_gaussian(self.h, int(seed) & 0xFFFFFFFFFFFFFFFF))

    def momenta_action(self):
        """(TF/2) sum P^2 after the momentum boundary conditions (applied in place)"""
        out = ctypes.c_double()
        self._check(self.lib.yg_momenta_action(self.h, ctypes.byref(out)))
        return out.value

    def gauge_backup(self): self._check(self.lib.yg_gauge_backup(self.h))

    def gauge_restore(self): self._check(self.lib.yg_gauge_restore(self.h))
