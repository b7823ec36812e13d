"""Benchmark: CG time-to-solution on the even-odd Wilson-clover operator, one B200.

Workload (defaults): 32^4 SU(3) fundamental, even-odd preconditioned Wilson-clover,
m = -0.75, csw = 1.0, periodic space / antiperiodic time.  One step = one solve of
Hphi_sq x = b (the D^dag D system of cg_inverter, cg.cpp:132-202) to a TRUE FP64
relative residual of 1e-12 (prec = 1e-24 in the reference's squared convention), with
the mixed-precision solver (FP32 arithmetic on FP16 spinors with per-site norms, FP32
12-real links and clover blocks; FP64 reliable updates and stopping test).

Reported beside it: the same solve with the plain FP64 CG (the reference's algorithm on
the GPU), the FP64 Dslash (Dphi_oe) bandwidth against the measured HBM peak, the same
metric end to end through the public API with the source uploaded from pinned host
memory and the solution downloaded every step, and the reference's own CPU code
(oracle/_ref, built from the reference sources) timed on this host's cores.

Synthetic inputs: a thermalised beta = 5.6 field made on the host without the engine, so
that both arms read the same field: a Wilson-action heatbath (100 sweeps from a cold start)
on 8^4, tiled to 32^4 (a periodic field with the same local action density); the source is
a complex Gaussian, unit variance per component.  Every input (links 604 MB, clover 604 MB,
fields 201 MB each) is larger than the 126 MB L2, so no flush is needed between steps.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                       [--dims T X Y Z] [--no-cpu-baseline]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

from yahmc_b200 import replicas

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

MASS, CSW, PREC = -0.75, 1.0, 1e-24
CPU_SAMPLE_PREC = 1e-8      # squared relative residual of the bounded CPU-baseline sample
REF_SAMPLE_PREC = 1e-3      # squared relative residual of each step of the reference arm
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dims", type=int, nargs=4, default=[32, 32, 32, 32])
    ap.add_argument("--seed", type=int, default=20241203)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dslash-iters", type=int, default=50)
    ap.add_argument("--inner", default="f16spinor-l12", choices=list(INNER),
                    help="inner operator of the mixed solver: generic FP32, or the compressed d = 3 "
                         "operator with FP32/FP16 spinors and 18/12-real links")
    ap.add_argument("--delta", type=float, default=0.1, help="reliable-update threshold")
    ap.add_argument("--variants", action="store_true", help="also time every inner operator once")
    ap.add_argument("--field-cache", default=None,
                    help="npz file holding the generated field: loaded when present, written otherwise "
                         "(lets a profiled run skip the field generation)")
    ap.add_argument("--nrhs", type=int, default=12, help="systems of the batched-CG measurement (<= 1: skip)")
    ap.add_argument("--batched-only", action="store_true",
                    help="time only the batched CG of --nrhs systems (for profiling; not the bench line)")
    ap.add_argument("--solve-only", action="store_true",
                    help="time only the mixed solve and print its time (for profiling; not the bench line)")
    ap.add_argument("--mesons", action="store_true",
                    help="time the 12 point-source propagators of one slice (one at a time and batched) and the "
                         "16-channel contraction on 48x24x24x24 (not the bench line)")
    ap.add_argument("--lattices", action="store_true",
                    help="time FP64 CG solves on 8^4, 12^4 and 16^4 lattices one after another and "
                         "concurrently (yg_cg_inverter_lattices; not the bench line)")
    ap.add_argument("--mshift", action="store_true",
                    help="time a 12-shift cg_mshift on SU(2) adjoint 48x24x24x24 against the 12 shifted "
                         "systems solved one at a time (not the bench line)")
    ap.add_argument("--hmc", action="store_true",
                    help="configuration 2: Nf=2 HMC + Hasenbusch trajectories on 16^3x32 through YaHMC's own hmc "
                         "program built on the engine, FP64 and mixed-precision solvers (not the bench line)")
    ap.add_argument("--hmc-trajectories", type=int, default=4)
    ap.add_argument("--hmc-fermion-therm", type=int, default=0,
                    help="Nf=2 trajectories between the pure-gauge start and the measured ones")
    ap.add_argument("--hmc-mass", type=float, default=-0.75,
                    help="bare mass m of the HMC (m + 0.2) and Hasenbusch (m) monomials")
    ap.add_argument("--rhmc", action="store_true",
                    help="configuration 4(i): order-12 rational approximation via one multishift solve and the "
                         "batched pole force, SU(2) adjoint 48x24^3 (not the bench line)")
    ap.add_argument("--learned", action="store_true",
                    help="configuration 5: learned preconditioner trained on 48x24^3, deployed on 64x32^3 "
                         "(not the bench line)")
    ap.add_argument("--train-steps", type=int, default=100)
    ap.add_argument("--train-dims", type=int, nargs=4, default=[48, 24, 24, 24],
                    help="lattice of the learned preconditioner's training (T X Y Z)")
    ap.add_argument("--deploy-dims", type=int, nargs=4, default=[64, 32, 32, 32],
                    help="lattice the trained preconditioner is deployed on (T X Y Z)")
    ap.add_argument("--contract-only", action="store_true",
                    help="with --mesons: only the contraction, on random propagators (for profiling)")
    return ap.parse_args()


# inner operator of the mixed-precision solver: None = generic FP32 (every representation),
# (spinor bits, link reals) = the compressed d = 3 operator
INNER = {"generic-f32": (0, 18, 0, 0), "f32-l18": (32, 18, 0, 0), "f32-l12": (32, 12, 0, 0),
         "f16-l18": (16, 18, 0, 0), "f16-l12": (16, 12, 0, 0),
         "f32-i16links-l12": (32, 12, 15, 32), "f32-i16-l12": (32, 12, 15, 15), "f16-i16-l12": (16, 12, 15, 15),
         "f16spinor-l12": (16, 12, 32, 32), "f16spinor-l8": (16, 8, 32, 32), "f32-l8": (32, 8, 32, 32)}


DTYPE = {"generic-f32": "f32 inner / f64 reliable updates and residual",
         "f32-l18": "f32 inner / f64 reliable updates and residual",
         "f32-l12": "f32 inner (12-real links) / f64 reliable updates and residual",
         "f16-l18": "f32 inner arithmetic on f16 storage / f64 reliable updates and residual",
         "f16-l12": "f32 inner arithmetic on f16 storage (12-real links) / f64 reliable updates and residual",
         "f32-i16links-l12": "f32 inner (int16 12-real links) / f64 reliable updates and residual",
         "f32-i16-l12": "f32 inner (int16 12-real links and clover) / f64 reliable updates and residual",
         "f16-i16-l12": "f32 inner arithmetic on f16 spinors, int16 links and clover / f64 reliable updates and residual",
         "f16spinor-l12": "f32 inner arithmetic on f16 spinors, f32 12-real links and clover / f64 reliable updates and residual",
         "f16spinor-l8": "f32 inner arithmetic on f16 spinors, f32 8-real links, f32 clover / f64 reliable updates and residual",
         "f32-l8": "f32 inner (8-real links) / f64 reliable updates and residual"}


# DRAM bytes (read + write) of one launch of the inner operator's step 1 as ncu counted them
# (dram__bytes_read.sum + dram__bytes_write.sum), with the output sites of that launch; the
# bench line scales them to its own lattice by the number of output sites
INNER_NCU = {"f16spinor-l12": (191.3e6 + 9.8e6, 262144,
                               "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_shop<16,32,32,6,1,0> launch "
                               "at 32x32x32x16 (262,144 output sites), scaled by output sites to this lattice")}


def inner_traffic(inner, sites):
    if inner not in INNER_NCU:
        return None
    nbytes, nsites, _ = INNER_NCU[inner]
    return nbytes / nsites * sites


def solve_mixed(lat, x, b, inner, delta):
    spec = INNER[inner]
    return lat.cg_mixed("Hphi_sq", MASS, PREC, x, b, inner_precision=spec[0], link_reals=spec[1], delta=delta,
                        link_storage=spec[2], clover_storage=spec[3])


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


THERM = {"beta": 5.6, "c0": 1.0, "trajectories": 150, "warmup_md": 10, "steps": 100, "length": 1.0,
         "integrator": "o2mn", "start": "cold"}

# the benchmark field: Wilson-action heatbath at beta 5.6 on a small periodic lattice, tiled
FIELD = {"beta": 5.6, "base": 8, "sweeps": 100, "overrelax": 2, "start": "cold"}

METRIC = "CG time-to-solution (true rel. residual 1e-12)"


def thermalised_links(dims, seed, trajectories=None):
    """A thermalised SU(3) field made on the GPU (used by --mesons): pure-gauge HMC (Wilson
    action, beta 5.6) on the lattice with the spatial extents halved, from a cold start, then
    tiled 1x2x2x2.  Returns (U, plaquette, acceptance)."""
    import yahmc_b200 as yg
    from yahmc_b200 import thermalize as th
    small = (dims[0],) + tuple(d // 2 if d % 4 == 0 else d for d in dims[1:])
    lat = yg.Lattice(small, nc=3, repr="fundamental", bc="periodic", clover=False, eo=True)
    lat.set_links(np.broadcast_to(np.eye(3, dtype=complex), (lat.V, 4, 3, 3)).copy())
    n_traj = THERM["trajectories"] if trajectories is None else trajectories
    hist = th.thermalize(lat, THERM["beta"], n_traj, steps=THERM["steps"], length=THERM["length"], c0=THERM["c0"],
                         seed=seed, integrator=THERM["integrator"], n_warm=min(THERM["warmup_md"], n_traj))
    acc = float(np.mean([h[0] for h in hist[THERM["warmup_md"]:]])) if n_traj > THERM["warmup_md"] else 1.0
    U = th.tile(lat.get_links(), small, tuple(dims))
    plaq = float(hist[-1][2])
    del lat
    return U, plaq, acc


def bench_field(dims, seed, cache=None):
    """The benchmark's gauge field, made on the host without the engine so that the reference
    arm and this arm use the same field: Cabibbo-Marinari heatbath (2 overrelaxation sweeps per
    heatbath sweep) at beta 5.6 on a periodic 8^4 lattice from a cold start, 100 sweeps, then
    tiled onto `dims` (again a periodic field with the same local action density).  The
    result is cached in the temporary directory (and in `cache` when given), keyed by its
    parameters, so the second arm on the same machine reads what the first one made.
    Returns (U in even-odd site order, plaquette of the 8^4 field)."""
    from yahmc_b200 import heatbath, thermalize
    base = tuple(min(FIELD["base"], d) for d in dims)
    key = f"{'x'.join(map(str, base))}_{'x'.join(map(str, dims))}_{FIELD['beta']}_{FIELD['sweeps']}_" \
          f"{FIELD['overrelax']}_{seed}"
    paths = [p for p in (cache, os.path.join(tempfile.gettempdir(), f"yahmc_bench_field_{key}.npz")) if p]
    for p in paths:
        if os.path.exists(p):
            try:
                z = np.load(p)
                if str(z["key"]) == key:
                    return z["U"], float(z["plaquette"])
            except Exception:
                pass
    U8, hist = heatbath.thermalised_field(base, FIELD["beta"], FIELD["sweeps"], seed, n_or=FIELD["overrelax"])
    U = thermalize.tile(U8, base, tuple(dims)) if base != tuple(dims) else U8
    plaq = float(hist[-1])
    for p in paths:
        try:
            tmp = p + f".{os.getpid()}.tmp.npz"
            np.savez(tmp, U=U, plaquette=plaq, key=key)
            os.replace(tmp, p)
        except OSError:
            pass
    return U, plaq


def make_inputs(dims, seed, rank=0, cache=None):
    """(links, source, description): the shared field and this rank's Gaussian source."""
    from yahmc_b200 import fields
    U, plaq = bench_field(dims, seed, cache)
    T, X, Y, Z = dims
    V = T * X * Y * Z
    rng = np.random.default_rng(replicas.rank_seed(seed, rank))
    b = fields.gaussian_spinor(V, 3, rng)
    return U, b, {"plaquette": plaq}


def links_desc(info, dims):
    base = tuple(min(FIELD["base"], d) for d in dims)
    return (f"thermalised on the host: Wilson-action heatbath (Cabibbo-Marinari, Kennedy-Pendleton, "
            f"{FIELD['overrelax']} overrelaxation sweeps each) at beta {FIELD['beta']}, {FIELD['sweeps']} sweeps "
            f"from a cold start on {'x'.join(map(str, base))}, tiled to {'x'.join(map(str, dims))}; "
            f"plaquette {info['plaquette']:.6f}")


def workload_name(dims):
    return f"{'x'.join(map(str, dims))} SU(3) fund even-odd Wilson-clover CG on Hphi_sq to true rel. residual 1e-12"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, gpu_index=0):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ reference (CPU) arm
def engine_loaded():
    """Whether this process has mapped the engine's shared library (the reference arm must not)."""
    try:
        with open("/proc/self/maps") as f:
            return "libyahmc_b200.so" in f.read()
    except OSError:
        return None


class ReferenceCG:
    """The reference's own cg_inverter (cg.cpp:132-202, compiled unmodified into oracle/_ref) on
    Hphi_sq with the benchmark's links and source, on this host's cores."""

    def __init__(self, dims, U, b, threads):
        from oracle import ref as oref
        from oracle import yahmc_oracle as yo
        from yahmc_b200 import fields
        self.R = oref.get("su3_fund_ap", tuple(dims), csw=CSW, cf=1.0, threads=threads)
        self.R.lib.yref_set_threads(threads)
        self.R.set_links(fields.complex_to_raw(U))
        self.braw = yo.spinor_to_raw(b)
        self.threads = threads

    def solve(self, prec):
        """One solve from a zero guess to squared precision prec: (ms, iterations)."""
        x = self.R.spinor()
        bb = self.braw.copy()
        t0 = time.perf_counter()
        it = self.R.call("cg", 2, MASS, prec, x, bb)
        return (time.perf_counter() - t0) * 1e3, int(it)


def run_reference(a, rank, world):
    """--impl reference: the reference's CPU CG on the same field and source.  One full solve to
    prec 1e-24 gives the iteration count of the workload and its time; each warm-up and timed
    step is then a bounded sample (the same solve stopped at squared residual 1e-3, about a tenth
    of the iterations) whose time per iteration, times the full iteration count, is the step's
    time-to-solution.  Runs on rank 0 only, with every host core; the engine is not loaded."""
    if rank != 0:
        return
    from oracle import ref as oref
    if not oref.available("su3_fund_ap"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (no reference sources on this host)"}))
        return
    threads = os.cpu_count() or 1
    U, b, info = make_inputs(a.dims, a.seed, 0, a.field_cache)
    ref = ReferenceCG(a.dims, U, b, threads)
    full_ms, n_full = ref.solve(PREC)
    times, sample_its = [], []
    for i in range(a.warmup + a.steps):
        ms, it = ref.solve(REF_SAMPLE_PREC)
        if i >= a.warmup:
            times.append(ms / max(it, 1) * n_full)
            sample_its.append(it)
    value = float(np.median(times))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "ms",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(a.dims), "mass": MASS, "csw": CSW, "prec_squared": PREC,
                   "links": links_desc(info, a.dims), "parallelism": "host cores"},
        "iterations": n_full, "full_solve_ms": full_ms, "threads": threads,
        "cpu_baseline": {"value": value, "unit": "ms", "cores": threads, "kind": "reference",
                         "sample": f"per step: the reference's cg_inverter stopped at squared residual "
                                   f"{REF_SAMPLE_PREC:g} ({sample_its[-1] if sample_its else 0} iterations) on "
                                   f"{threads} OpenMP threads, time per iteration x the {n_full} iterations of the "
                                   f"full solve to 1e-24 (that full solve, run once first: {full_ms / 1e3:.1f} s)"},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "engine_loaded": engine_loaded(),
    }
    print(json.dumps(line))


# ------------------------------------------------------------------ our arm
def run_mesons(a):
    """The point-source meson workload on one GPU: the 12 propagators of one source slice on a
    thermalised 48x24^3 SU(3) field (m = -0.6, prec 1e-20), solved one at a time with
    calc_propagator (BiCGstab, the reference's path) and through the batched solvers (BiCGstab
    on D; CG on Hphi_sq, mixed and FP64), then the sixteen-channel contraction timed with CUDA
    events."""
    import torch
    import yahmc_b200 as yg
    from yahmc_b200 import fields
    from yahmc_b200.spectrum import POINT, Mesons
    torch.cuda.set_device(0)
    yg.set_device(0)
    dims = (48, 24, 24, 24)
    mass, prec, tau = -0.6, 1e-20, 5
    out = {"workload": "12 point-source propagators of one slice + 16-channel contraction, 48x24x24x24 SU(3) "
                       "fund even-odd Wilson-clover", "mass": mass, "prec_squared": prec}
    lat = yg.Lattice(dims, nc=3, repr="fundamental", bc="antiperiodic", clover=True, eo=True, csw=CSW)
    if a.contract_only:
        rng = np.random.default_rng(a.seed)
        lat.set_links(fields.haar_su(3, lat.V * 4, rng).reshape(lat.V, 4, 3, 3))
        props = [lat.field(fields.gaussian_spinor(lat.V, 3, rng)) for _ in range(12)]
    else:
        if a.field_cache and os.path.exists(a.field_cache):
            z = np.load(a.field_cache)
            U, plaq = z["U"], float(z["plaquette"])
        else:
            U, plaq, _ = thermalised_links(dims, a.seed, trajectories=40)
            if a.field_cache:
                np.savez(a.field_cache, U=U, plaquette=plaq, acceptance=0.0)
        lat.set_links(U)
        out["links"] = f"thermalised: 40 pure-gauge HMC trajectories at beta 5.6, plaquette {plaq:.5f}"

        def run(**kw):
            M = Mesons(lat, mass, prec, 1, POINT, **kw)
            M.measure(taus=[tau])                              # warm-up: tuning, allocations
            for f in M.prop:
                lat.spinor_zero(f)                             # timed solves start from zero
            M.iterations = 0
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            M.measure(taus=[tau])
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1), M

        t1, A = run()
        t2, B = run(batched=True, solver="bicgstab")
        t3, C = run(batched=True, solver="cg_mixed")
        t4, D = run(batched=True, solver="cg")
        va = A.values()
        out["one_at_a_time_bicgstab"] = {"ms": t1, "iterations": A.iterations}
        out["batched_bicgstab"] = {"ms": t2, "iterations": B.iterations}
        out["batched_mixed_cg"] = {"ms": t3, "iterations": C.iterations}
        out["batched_fp64_cg"] = {"ms": t4, "iterations": D.iterations}
        out["max_rel_diff_of_correlators"] = max(
            float(np.abs(M.values()[k] - va[k]).max() / np.abs(va[k]).max()) for M in (B, C, D) for k in va)
        props = A.prop
    corr = np.zeros((16, dims[0]))
    for _ in range(3):
        lat.meson_contract(POINT, tau, props, corr)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        lat.meson_contract(POINT, tau, props, corr)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    nbytes = 12 * lat.field_doubles * 8
    pk, kind = hbm_peak()
    gbs = nbytes / (ms * 1e-3) / 1e9
    out["contraction"] = {"ms_per_call_incl_readback": ms, "algorithmic_bytes": nbytes, "GB_s": gbs,
                          "peak_GB_s": pk, "peak_kind": kind, "frac": gbs / pk}
    print(json.dumps(out))


def run_mshift(a):
    """The RHMC-shaped multishift solve: SU(2) adjoint (d = 3, real links stored complex)
    48x24x24x24 even-odd Wilson-clover on a Haar-random field, m = -0.2, Hphi_sq + s_k for 12
    shifts log-spaced on [1e-4, 8] (the pole range of an RHMC approximation), prec 1e-20; one
    cg_mshift call against the 12 systems solved one at a time (one shift per call), CUDA events."""
    import torch
    import yahmc_b200 as yg
    from yahmc_b200 import fields
    torch.cuda.set_device(0)
    yg.set_device(0)
    dims = (48, 24, 24, 24)
    lat = yg.Lattice(dims, nc=2, repr="adjoint", bc="antiperiodic", clover=True, eo=True, csw=CSW)
    rng = np.random.default_rng(a.seed)
    lat.set_links(fields.haar_su(2, lat.V * 4, rng).reshape(lat.V, 4, 2, 2))
    b = lat.field(fields.gaussian_spinor(lat.V, 3, rng))
    shifts = np.geomspace(1e-4, 8.0, 12)
    xs = [lat.field() for _ in shifts]
    mass, prec = -0.2, 1e-20

    def ev_time(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    def together():
        return lat.cg_mshift("Hphi_sq", mass, prec, shifts, xs, b)

    def apart():
        return [lat.cg_mshift("Hphi_sq", mass, prec, shifts[k:k + 1], xs[k:k + 1], b) for k in range(len(shifts))]

    def true_residuals():
        out = []
        bn = lat.spinor_sqnorm(b)
        for s_, x in zip(shifts, xs):
            xc, r = lat.field(), lat.field()
            lat.spinor_copy(xc, x)
            lat.Hphi_sq(mass, r, xc)
            lat.spinor_mulr_add_assign(r, float(s_), x)
            lat.spinor_sub_assign(r, b)
            out.append(lat.spinor_sqnorm(r) / bn)
        return out

    t1, it1 = ev_time(together)
    res1 = true_residuals()
    x_together = [lat.download(x) for x in xs]
    t2, it2 = ev_time(apart)
    res2 = true_residuals()
    diff = max(float(np.abs(lat.download(x) - xt).max() / np.abs(xt).max()) for x, xt in zip(xs, x_together))
    valid = max(res1 + res2) < 10 * prec
    print(json.dumps({"workload": "12-shift CG on Hphi_sq + s, SU(2) adjoint 48x24x24x24 even-odd Wilson-clover, "
                                  "Haar-random links", "shifts": list(shifts), "mass": mass, "prec_squared": prec,
                      "cg_mshift_ms": t1, "cg_mshift_iterations": it1, "one_shift_at_a_time_ms": t2,
                      "one_shift_iterations": it2, "speedup": t2 / t1,
                      "true_residuals_together": res1, "true_residuals_apart": res2,
                      "max_rel_diff_of_solutions": diff,
                      "valid": bool(valid), "validity": "every true residual below 10 x prec (the multishift "
                                                        "stops on recursive residuals)"}))


HMC_CFG = """[lattice]
dim_t = {T}
dim_x = {X}
dim_y = {Y}
dim_z = {Z}
[parallel]
threads = 0
np_t = 1
np_x = 1
np_y = 1
np_z = 1
[log]
level = 30
[rand]
seed = {seed}
[cnfg]
dir = {dir}
prefix = {prefix}
start = {start}
last = {last}
freq = {freq}
[clover]
csw = 1.0
cf = 1.0
[traj]
length = 1.0
[observables]
plaq_freq = 1
poly_freq = 0
mes_freq = 0
"""

GAUGE_ONLY = """[integrator]
level = 0
type = o2mn
steps = 10
[monomial]
level = 0
type = gauge
beta = 5.6
c0 = 1.0
"""

NF2 = """[integrator]
level = 0
type = o2mn
steps = 1
[integrator]
level = 1
type = o2mn
steps = 10
[monomial]
level = 0
type = gauge
beta = 5.6
c0 = 1.0
[monomial]
level = 1
type = hmc
mass = {mass}
dm = 0.2
prec = 1e-24
mre_past = 5
[monomial]
level = 1
type = hasenbusch
mass = {mass}
dm = 0.2
prec = 1e-24
"""


def _hmc_log(path):
    import re
    text = open(path).read()
    traj = [(float(t), int(m)) for t, m in re.findall(r"Trajectory finished in ([0-9.]+) seconds \(MVM = (\d+)\)", text)]
    dh = [float(x) for x in re.findall(r"dH = ([-+0-9.e]+)", text)]
    acc = re.findall(r"Configuration (accepted|rejected)", text)
    plaq = [float(x) for x in re.findall(r"Plaquette: ([-+0-9.e]+)", text)]
    return {"seconds": [t for t, _ in traj], "mvm": [m for _, m in traj], "dH": dh, "accepted": [x == "accepted" for x in acc],
            "plaquette": plaq}


def run_hmc(a):
    """Configuration 2 through YaHMC's own hmc program (programs/hmc.cpp and every library file
    but the eight the shim replaces, unchanged) built on the engine: SU(3) fundamental 16^3x32,
    Wilson gauge action beta 5.6, clover csw 1, an HMC monomial (m = -0.75, dm = 0.2) and a
    Hasenbusch monomial (m = -0.75, dm = 0.2) on level 1 with 10 o2mn steps, the gauge monomial
    on level 0 with 1 step, trajectory length 1, prec 1e-24 (relative residual 1e-12).  The
    start is 20 pure-gauge trajectories from the reference's random start (seed given), then
    --hmc-fermion-therm trajectories of the full action.  Then --hmc-trajectories trajectories
    with the reference's FP64 solvers and the same number with the mixed-precision CG for the
    Hphi_sq solves (YAHMC_GPU_SOLVER=mixed), both from that start with the same seed; the
    program's own log gives trajectory times, MVM counts, dH, <exp(-dH)> and acceptance.  The
    CPU build of the same program (oracle/_ref) runs one trajectory from the same start for
    comparison."""
    exe = os.path.join(ROOT, "integration", "_build", "hmc_su3_fund_ap")
    cpu_exe = os.path.join(ROOT, "oracle", "_ref", "hmc_su3_fund_ap")
    if not os.path.exists(exe):
        print(json.dumps({"hmc": "unavailable", "why": "integration/_build/hmc_su3_fund_ap not built"}))
        return
    T, X, Y, Z = 32, 16, 16, 16
    work = tempfile.mkdtemp(prefix="yahmc_hmc_")
    dims = dict(T=T, X=X, Y=Y, Z=Z, dir=work)

    def run(exe_path, cfg_text, name, env=None):
        cfg = os.path.join(work, f"{name}.cfg")
        with open(cfg, "w") as f:
            f.write(cfg_text)
        log = os.path.join(work, f"{name}.log")
        t0 = time.perf_counter()
        r = subprocess.run([exe_path, "-i", cfg, "-o", log], cwd=work, capture_output=True, text=True,
                           env={**os.environ, **(env or {})})
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            raise RuntimeError(f"{name}: rc {r.returncode}: {r.stderr[-1000:]}")
        out = _hmc_log(log)
        out["wall_s"] = wall
        with open(log) as f:
            out["log_tail"] = f.read()[-1500:]
        return out

    seed = a.seed % 100000
    therm = run(exe, HMC_CFG.format(seed=seed, prefix="therm", start="random", last=20, freq=20, **dims) + GAUGE_ONLY,
                "therm")
    # then --hmc-fermion-therm trajectories with the fermions (the mixed solver), so that the
    # measured trajectories start near equilibrium of the full action
    nt = a.hmc_fermion_therm
    start = f"therm_{T}x{X}x{Y}x{Z}_nc3_n0020"
    ftherm = None
    if nt > 0:
        # the program saves when the configuration number is a multiple of freq: only the last one
        ftherm = run(exe, HMC_CFG.format(seed=seed + 2, prefix="ftherm", start=start, last=20 + nt, freq=20 + nt,
                                         **dims) + NF2.format(mass=a.hmc_mass), "ftherm", {"YAHMC_GPU_SOLVER": "mixed"})
        if len(ftherm["seconds"]) != nt:
            raise RuntimeError(f"ftherm: {len(ftherm['seconds'])} trajectories in the log, expected {nt}; log "
                               f"ends:\n{ftherm['log_tail']}")
        start = f"ftherm_{T}x{X}x{Y}x{Z}_nc3_n{20 + nt:04d}"
    n0 = 20 + nt
    n = a.hmc_trajectories
    res = {"workload": "Nf=2 HMC + Hasenbusch trajectory, 16^3x32 SU(3) fund clover even-odd, YaHMC's hmc program "
                       f"on the engine, m = {a.hmc_mass}", "start": f"20 pure-gauge trajectories from the random start (plaquette "
                       f"{therm['plaquette'][-1]:.6f}), then {nt} Nf=2 trajectories"
                       + (f" (plaquette {ftherm['plaquette'][-1]:.6f}, dH of the last {ftherm['dH'][-1]:.4f})"
                          if ftherm else ""),
           "thermalisation_s": therm["wall_s"] + (ftherm["wall_s"] if ftherm else 0.0)}
    for solver, env in (("fp64", None), ("mixed", {"YAHMC_GPU_SOLVER": "mixed"})):
        # the program counts configurations from the start file's number (hmc.cpp:148): last is absolute
        r = run(exe, HMC_CFG.format(seed=seed + 1, prefix="nf2", start=start, last=n0 + n, freq=0, **dims)
                + NF2.format(mass=a.hmc_mass), f"nf2_{solver}", env)
        if len(r["seconds"]) != n:
            raise RuntimeError(f"nf2_{solver}: {len(r['seconds'])} trajectories in the log, expected {n}; log ends:\n"
                               f"{r['log_tail']}")
        dh = np.array(r["dH"])
        emdh = np.exp(-dh)
        res[solver] = {"trajectory_s": r["seconds"], "mean_trajectory_s": float(np.mean(r["seconds"])),
                       "mvm": r["mvm"], "dH": r["dH"], "exp_minus_dH_mean": float(np.mean(emdh)),
                       "exp_minus_dH_stderr": float(np.std(emdh, ddof=1) / np.sqrt(len(emdh))) if len(emdh) > 1
                       else None, "acceptance": float(np.mean(r["accepted"])), "plaquette": r["plaquette"]}
    if os.path.exists(cpu_exe) and not a.no_cpu_baseline:
        r = run(cpu_exe, HMC_CFG.format(seed=seed + 1, prefix="cpu", start=start, last=n0 + 1, freq=0, **dims)
                + NF2.format(mass=a.hmc_mass), "cpu")
        if len(r["seconds"]) != 1:
            raise RuntimeError("cpu: no trajectory in the log")
        res["cpu_reference"] = {"trajectory_s": r["seconds"], "mvm": r["mvm"], "dH": r["dH"],
                                "threads": os.cpu_count(), "plaquette": r["plaquette"]}
        res["speedup_fp64_vs_cpu"] = r["seconds"][0] / res["fp64"]["trajectory_s"][0]
        res["dH_first_trajectory_gpu_minus_cpu"] = res["fp64"]["dH"][0] - r["dH"][0]
    print(json.dumps(res))


def run_rhmc(a):
    """Configuration 4(i): the RHMC force and action pieces for Nf = 1 in the SU(2) adjoint
    representation on 24^3x48 (even-odd clover, m = -0.2): the order-12 rational approximation
    of x^(-1/2) from the reference's table, rescaled to the spectral bound 8
    (yahmc_b200/data/rational_order12.json).  Timed with CUDA events: rational_calc (one 12-shift
    cg_mshift, rational.cpp:134-166) against the 12 shifted systems solved one at a time, and
    the pole loop of MonomialRHMC::update (rhmc.cpp:100-103) as one batched force against 12
    separate wilson_fermion_force_q calls.  The field: 40 pure-gauge HMC trajectories of SU(2)
    at beta 2.2 on 24^3x48 (the engine's molecular-dynamics kernels)."""
    import torch
    import yahmc_b200 as yg
    from yahmc_b200 import fields
    from yahmc_b200 import thermalize as th
    torch.cuda.set_device(0)
    yg.set_device(0)
    with open(os.path.join(ROOT, "yahmc_b200", "data", "rational_order12.json")) as f:
        ra = json.load(f)
    dims = (48, 24, 24, 24)
    mass, prec = -0.2, 1e-20
    lat = yg.Lattice(dims, nc=2, repr="adjoint", bc="antiperiodic", clover=True, eo=True, csw=CSW)
    gl = yg.Lattice(dims, nc=2, repr="fundamental", bc="periodic", clover=False, eo=True)
    gl.set_links(np.broadcast_to(np.eye(2, dtype=complex), (gl.V, 4, 2, 2)).copy())
    hist = th.thermalize(gl, 2.2, 40, steps=40, length=1.0, c0=1.0, seed=a.seed, integrator="o2mn", n_warm=10)
    lat.set_links(gl.get_links())
    plaq = float(hist[-1][2])
    del gl
    rng = np.random.default_rng(a.seed)
    b = lat.field(fields.gaussian_spinor(lat.V, lat.d, rng))
    poles, res = ra["poles"], ra["residues"]
    n = len(poles)

    def ev(fn, k=1):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = [fn() for _ in range(k)]
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, out[-1]

    x = lat.field()
    calc = lambda: lat.rational_calc("Hphi_sq", mass, prec, ra["a0"], poles, res, x, b)
    calc()
    ms_calc, it_calc = ev(calc, 2)
    xs = [lat.field() for _ in range(n)]

    def one_by_one():
        its = 0
        for p_, xi in zip(poles, xs):
            its += lat.cg_mshift("Hphi_sq", mass, prec, [p_], [xi], b)
        return its

    one_by_one()
    ms_sep, it_sep = ev(one_by_one, 1)
    # the same combination from the separate solves: a0 b + sum r_i x_i
    xc = lat.field()
    lat.spinor_mulr(xc, ra["a0"], b)
    for r_, xi in zip(res, xs):
        lat.spinor_mulr_add_assign(xc, r_, xi)
    lat.spinor_sub_assign(xc, x)
    diff = (lat.spinor_sqnorm(xc) / lat.spinor_sqnorm(x)) ** 0.5
    # the force of all poles: batched against one pole at a time, from the same solutions
    ms_xs = lat.cg_mshift("Hphi_sq", mass, prec, poles, xs, b)
    srcs = [lat.download(xi) for xi in xs]
    fields_b = [lat.field(s_) for s_ in srcs]
    lat.zero_momenta()
    lat.begin_fermion_force()

    # the force writes the odd half of each field from its even half and reads only the even
    # half otherwise, so repeated calls on the same fields give the same force
    def batched():
        lat.wilson_fermion_force_q_multi(0.1, mass, res, fields_b)

    def separate():
        for r_, f_ in zip(res, fields_b):
            lat.wilson_fermion_force_q(0.1, mass, r_, f_)

    batched()
    lat.zero_momenta()
    ms_fb, _ = ev(batched, 3)
    mom_b = lat.momenta()
    lat.zero_momenta()
    lat.begin_fermion_force()
    separate()
    lat.zero_momenta()
    ms_fs, _ = ev(separate, 3)
    mom_s = lat.momenta()
    print(json.dumps({
        "workload": "RHMC Nf=1 pieces, SU(2) adjoint 48x24x24x24 even-odd clover, m = -0.2, order-12 x^(-1/2) "
                    "rational approximation from the reference's table (valid on "
                    f"[{ra['valid_interval'][0]:.3g}, {ra['valid_interval'][1]:.3g}])",
        "links": f"40 pure-gauge HMC trajectories at beta 2.2, plaquette {plaq:.5f}",
        "rational_calc": {"one_mshift_ms": ms_calc, "iterations": it_calc, "shifts_one_at_a_time_ms": ms_sep,
                          "iterations_one_at_a_time": it_sep, "speedup": ms_sep / ms_calc,
                          "rel_diff_of_results": diff, "prec_squared": prec},
        "pole_force": {"batched_ms": ms_fb, "one_at_a_time_ms": ms_fs, "speedup": ms_fs / ms_fb,
                       "max_rel_diff_momenta": float(np.abs(mom_b - mom_s).max() / np.abs(mom_s).max()),
                       "poles": n, "mshift_iterations": ms_xs}}))


def run_learned(a):
    """Configuration 5: the learned preconditioner.  Trained on a 24^3x48 SU(3) field (beta 5.6
    heatbath field tiled from 8^4, m = -0.78): the network starts from the first-order hopping
    expansion of the Schur inverse and is trained on CG errors of that lattice's own solves;
    deployed on 32^3x64 (another heatbath field, same beta and mass).  Hphi_sq x = b to true
    relative residual 1e-12 three ways: the plain even-odd CG (FP64), the learned solve (two
    flexible-GCR Dphi solves with the network as right preconditioner, the FP64 CG finishing
    if needed), and the same without the network (plain GCR) for the ablation."""
    import torch
    import yahmc_b200 as yg
    from yahmc_b200 import Ptc, fields, learned
    torch.cuda.set_device(0)
    yg.set_device(0)
    mass, prec, C = -0.78, PREC, 8
    tdims, ddims = tuple(a.train_dims), tuple(a.deploy_dims)
    out = {"workload": f"learned preconditioner: train {'x'.join(map(str, tdims))}, deploy "
                       f"{'x'.join(map(str, ddims))}, SU(3) fund even-odd Wilson-clover, m = -0.78, Hphi_sq to "
                       "true rel. residual 1e-12", "channels": [1, C, C, 1]}
    U, plaq = bench_field(tdims, a.seed + 5)
    lt = yg.Lattice(tdims, nc=3, repr="fundamental", bc="antiperiodic", clover=True, eo=True, csw=CSW)
    lt.set_links(U)
    del U
    rng = np.random.default_rng(a.seed)
    net = Ptc(lt, (1, C, C, 1))
    net.set_weights(learned.hopping_start(net.shapes(), mass, rng))
    t0 = time.perf_counter()
    pairs = learned.training_pairs(lt, mass, 2, rng, stops=(25, 50, 100, 200), prec=1e-16, random_pairs=2)
    t1 = time.perf_counter()
    hist = learned.train(net, pairs, steps=a.train_steps, lr=1e-4, batch=4, rng=rng)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    out["training"] = {"pairs": len(pairs), "pair_generation_s": t1 - t0, "steps": a.train_steps, "train_s": t2 - t1,
                       "loss_first10": float(np.mean(hist[:10])), "loss_last10": float(np.mean(hist[-10:])),
                       "train_links_plaquette": plaq}
    Ws = net.get_weights()
    del net, pairs, lt
    U, plaq2 = bench_field(ddims, a.seed + 6)
    ld = yg.Lattice(ddims, nc=3, repr="fundamental", bc="antiperiodic", clover=True, eo=True, csw=CSW)
    ld.set_links(U)
    del U
    dnet = Ptc(ld, (1, C, C, 1))
    dnet.set_weights(Ws)
    b = ld.field(fields.gaussian_spinor(ld.V, 3, rng))

    def ev(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), r

    def true_res(x):
        xc, r = ld.field(), ld.field()
        ld.spinor_copy(xc, x)
        ld.Hphi_sq(mass, r, xc)
        ld.spinor_sub_assign(r, b)
        return ld.spinor_sqnorm(r) / ld.spinor_sqnorm(b)

    x = ld.field()
    ms, it = ev(lambda: ld.cg_inverter("Hphi_sq", mass, prec, x, b))
    out["plain_eo_cg_fp64"] = {"ms": ms, "iterations": it, "true_residual": true_res(x)}
    x = ld.field()
    ms, st = ev(lambda: ld.solve_learned(mass, prec, x, b, net=dnet))
    out["learned_fgcr"] = {"ms": ms, "gcr_iterations": st["iterations"], "fallback": st["fallback"],
                           "true_residual": true_res(x)}
    x = ld.field()
    ms, st = ev(lambda: ld.solve_learned(mass, prec, x, b, net=None))
    out["plain_gcr_no_network"] = {"ms": ms, "gcr_iterations": st["iterations"], "fallback": st["fallback"],
                                   "true_residual": true_res(x)}
    x = ld.field()
    ms, st = ev(lambda: ld.cg_mixed("Hphi_sq", mass, prec, x, b))
    out["mixed_cg"] = {"ms": ms, "iterations": st["iterations"], "true_residual": true_res(x)}
    out["deploy_links_plaquette"] = plaq2
    y = ld.field()
    ms, _ = ev(lambda: [dnet.apply(y, b) for _ in range(10)])
    out["network_apply_ms"] = ms / 10
    print(json.dumps(out))


def run_lattices(a):
    """FP64 CG (Hphi_sq, m = -0.6, prec 1e-20) on SU(3) fundamental 8^4, 12^4 and 16^4 lattices
    with thermalised-like fields from the engine's own HMC (20 trajectories each): the three
    solves one after another, then through one yg_cg_inverter_lattices call."""
    import torch
    import yahmc_b200 as yg
    from yahmc_b200 import fields
    torch.cuda.set_device(0)
    yg.set_device(0)
    solves = []
    for k, L in enumerate((8, 12, 16)):
        dims = (L, L, L, L)
        U, plaq, _ = thermalised_links(dims, a.seed + k, trajectories=20)
        lat = yg.Lattice(dims, nc=3, repr="fundamental", bc="antiperiodic", clover=True, eo=True, csw=CSW)
        lat.set_links(U)
        b = lat.field(fields.gaussian_spinor(lat.V, 3, np.random.default_rng(a.seed + 100 + k)))
        solves.append((lat, -0.6, 1e-20, lat.field(), b))

    def sequential():
        its = []
        for lat, m, pr, x, b in solves:
            lat.spinor_zero(x)
            its.append(lat.cg_inverter("Hphi_sq", m, pr, x, b))
        return its

    path = []

    def concurrent():
        for lat, m, pr, x, b in solves:
            lat.spinor_zero(x)
        its, rc, p = yg.cg_inverter_lattices(solves, with_path=True)
        if rc != 0:
            raise RuntimeError(f"cg_inverter_lattices status {rc}")
        path.append(p)
        return its

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            its = fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) * 1e3 / a.steps, its

    t_seq, it_seq = timed(sequential)
    t_con, it_con = timed(concurrent)
    print(json.dumps({"workload": "FP64 CG on Hphi_sq, SU(3) fund even-odd Wilson-clover 8^4 + 12^4 + 16^4",
                      "sequential_ms": t_seq, "concurrent_ms": t_con, "speedup": t_seq / t_con,
                      "iterations": it_seq, "iterations_concurrent": it_con,
                      "concurrent_path": "one persistent kernel" if path and path[-1] == 1 else "host threads",
                      "timing": "host wall clock around the solves, synchronised, mean of --steps"}))


def run_ours(a, rank, world, dist):
    import torch
    import yahmc_b200 as yg
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
    dev = torch.cuda.current_device()
    yg.set_device(dev)
    U, b, info = make_inputs(a.dims, a.seed, rank, a.field_cache)
    lat = yg.Lattice(a.dims, nc=3, repr="fundamental", bc="antiperiodic", clover=True, eo=True, csw=CSW)
    lat.set_links(U)
    V, d = lat.V, lat.d
    field_bytes = lat.field_doubles * 8
    bf = lat.field(b)
    x = lat.field()

    def barrier():
        replicas.barrier(dist, torch.cuda.synchronize)

    def timed(fn, k):
        """k calls of fn bracketed by a barrier + synchronize on both sides, CUDA events on the
        default stream (the engine's stream); returns per-call ms, max over ranks."""
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = [fn() for _ in range(k)]
        e1.record()
        torch.cuda.synchronize()
        barrier()
        ms = replicas.max_over_ranks(e0.elapsed_time(e1) / k, dist, "cuda")
        return ms, out

    def mixed():
        lat.spinor_zero(x)
        return solve_mixed(lat, x, bf, a.inner, a.delta)

    def fp64():
        lat.spinor_zero(x)
        return lat.cg_inverter("Hphi_sq", MASS, PREC, x, bf)

    if a.batched_only:
        rng_b = np.random.default_rng(a.seed + 17)
        from yahmc_b200 import fields as yf
        bsrc = [lat.field(yf.gaussian_spinor(V, 3, rng_b)) for _ in range(a.nrhs)]
        bx = [lat.field() for _ in range(a.nrhs)]

        def multi_only():
            for f in bx:
                lat.spinor_zero(f)
            return lat.cg_mixed_multi("Hphi_sq", MASS, PREC, bx, bsrc, delta=0.1)

        for _ in range(max(1, a.warmup)):
            multi_only()
        ms_b, sts_b = timed(multi_only, a.steps)
        if rank == 0:
            print(json.dumps({"batched_mixed_ms": ms_b, "nrhs": a.nrhs,
                              "iterations": [st["iterations"] for st in sts_b[-1]],
                              "worst_true_residual": max(st["true_residual"] for st in sts_b[-1])}))
        return

    # warm-up (W >= 3 solves), then the timed mixed-precision solves with clocks sampled
    for _ in range(max(3, a.warmup)):
        mixed()
    clk = Clocks(dev)
    n0 = yg.launch_count()
    ms_mixed, stats = timed(mixed, a.steps)
    launches = (yg.launch_count() - n0) // a.steps
    clocks = clk.stop()
    st = stats[-1]
    if a.solve_only:
        if rank == 0:
            print(json.dumps({"solve_ms": ms_mixed, "inner": a.inner, "delta": a.delta, "launches": int(launches),
                              "solver": st}))
        return
    # independent check of the stopping criterion on the true residual
    xc, r = lat.field(), lat.field()
    lat.spinor_copy(xc, x)
    lat.Hphi_sq(MASS, r, xc)
    lat.spinor_sub_assign(r, bf)
    true_res = lat.spinor_sqnorm(r) / lat.spinor_sqnorm(bf)

    # plain FP64 CG (the reference's algorithm on the GPU)
    fp64()
    ms_fp64, its = timed(fp64, max(1, min(a.steps, 3)))
    it_fp64 = its[-1]

    # FP64 Dslash (Dphi_oe): one hop over V/2 output sites
    src, dst = lat.field(b), lat.field()
    for _ in range(5):
        lat.Dphi_oe(dst, src)
    ms_hop, _ = timed(lambda: lat.Dphi_oe(dst, src), a.dslash_iters)
    link_reals = 2 * d * d
    bytes_per_site = (2 * 8 * d + 8 * link_reals) * 8          # 1 spinor in + 1 out + 8 links, FP64
    hop_bytes = bytes_per_site * (V // 2)
    hop_gbs = hop_bytes / (ms_hop * 1e-3) / 1e9
    peak, peak_kind = hbm_peak()
    # the dominant kernel of the timed solve: step 1 of the mixed solver's inner operator
    # (FP16 spinors with per-site norms, FP32 12-real links, FP32 packed clover blocks)
    ms_inner, inner_bytes = lat.inner_hop_profile(MASS, reps=a.dslash_iters)
    inner_gbs = inner_bytes / (ms_inner * 1e-3) / 1e9

    # end to end through the public API: pinned host source in, solution out, every step
    hb = torch.empty(lat.field_doubles, dtype=torch.float64, pin_memory=True).numpy()
    hx = torch.empty(lat.field_doubles, dtype=torch.float64, pin_memory=True).numpy()
    from yahmc_b200.fields import complex_to_raw
    hb[:] = complex_to_raw(b)

    def e2e():
        lat.upload(bf, hb)
        lat.spinor_zero(x)
        s = solve_mixed(lat, x, bf, a.inner, a.delta)
        lat.download(x, raw=True, out=hx)
        return s

    e2e()
    ms_e2e, _ = timed(e2e, a.steps)

    # several right-hand sides at once: 12 sources (the point-source count of a meson
    # measurement) through the batched FP64 CG, per-system results identical to cg_inverter
    batched = None
    if a.nrhs > 1:
        rng_b = np.random.default_rng(a.seed + 17)
        from yahmc_b200 import fields as yf
        bsrc = [lat.field(yf.gaussian_spinor(V, 3, rng_b)) for _ in range(a.nrhs)]
        bx = [lat.field() for _ in range(a.nrhs)]

        def multi():
            for f in bx:
                lat.spinor_zero(f)
            return lat.cg_inverter_multi("Hphi_sq", MASS, PREC, bx, bsrc)

        def multi_mixed():
            for f in bx:
                lat.spinor_zero(f)
            return lat.cg_mixed_multi("Hphi_sq", MASS, PREC, bx, bsrc, delta=0.1)

        multi()
        ms_multi, its_multi = timed(multi, 1)
        multi_mixed()
        ms_mm, sts_mm = timed(multi_mixed, 2)
        worst = max(st["true_residual"] for st in sts_mm[-1])

        # the Hasenbusch pair: the Hphi_sq solves of the HMC monomial (m + dm) and of the
        # Hasenbusch monomial (m) of one force evaluation, separately and in one call
        pair = (MASS + 0.2, MASS)

        def pair_separate():
            out = []
            for k, m in enumerate(pair):
                lat.spinor_zero(bx[k])
                out.append(lat.cg_mixed_multi("Hphi_sq", m, PREC, [bx[k]], [bsrc[k]], delta=0.1)[0])
            return out

        def pair_joint():
            for k in range(2):
                lat.spinor_zero(bx[k])
            return lat.cg_mixed_multi("Hphi_sq", MASS, PREC, bx[:2], bsrc[:2], delta=0.1, masses=list(pair))

        pair_separate()
        ms_ps, sts_ps = timed(pair_separate, 2)
        pair_joint()
        ms_pj, sts_pj = timed(pair_joint, 2)
        batched = {"nrhs": a.nrhs,
                   "fp64": {"solver": "FP64 CG, all systems per operator launch", "ms_total": ms_multi,
                            "ms_per_rhs": ms_multi / a.nrhs, "iterations": its_multi[-1],
                            "speedup_per_rhs_vs_fp64_cg": ms_fp64 / (ms_multi / a.nrhs)},
                   "mixed": {"solver": "inner CG on FP16 spinors with per-site norms, FP32 12-real links and "
                                       "packed clover, FP64 reliable updates; all systems per operator launch, "
                                       "systems per thread chosen by the tuner; true residual per system",
                             "ms_total": ms_mm, "ms_per_rhs": ms_mm / a.nrhs,
                             "iterations": [st["iterations"] for st in sts_mm[-1]],
                             "reliable_updates": sts_mm[-1][0]["reliable_updates"],
                             "fallbacks": sum(st["fallback"] for st in sts_mm[-1]), "worst_true_residual": worst,
                             "speedup_per_rhs_vs_fp64_cg": ms_fp64 / (ms_mm / a.nrhs)},
                   "hasenbusch_pair": {"masses": list(pair), "separate_ms": ms_ps, "one_call_ms": ms_pj,
                                       "speedup": ms_ps / ms_pj,
                                       "iterations": [st["iterations"] for st in sts_pj[-1]],
                                       "true_residuals": [st["true_residual"] for st in sts_pj[-1]],
                                       "fallbacks": sum(st["fallback"] for st in sts_pj[-1] + sts_ps[-1])}}
        del bsrc, bx

    variants = None
    if a.variants:
        variants = {}
        for name in INNER:
            def one(name=name):
                lat.spinor_zero(x)
                return solve_mixed(lat, x, bf, name, a.delta)
            one()
            vms, vst = timed(one, 2)
            variants[name] = {"ms": vms, "iterations": vst[-1]["iterations"],
                              "reliable_updates": vst[-1]["reliable_updates"], "fallback": vst[-1]["fallback"],
                              "true_residual": vst[-1]["true_residual"]}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            from oracle import ref as oref
            if oref.available("su3_fund_ap"):
                threads = os.cpu_count() or 1
                cms, cit = ReferenceCG(a.dims, U, b, threads).solve(CPU_SAMPLE_PREC)
                cpu = {"value": cms / cit * it_fp64, "unit": "ms", "cores": threads, "kind": "reference",
                       "sample": f"reference cg_inverter on the same system stopped at prec {CPU_SAMPLE_PREC:g} "
                                 f"({cit} iterations, {cms / 1e3:.1f} s on {threads} OpenMP threads), scaled to the "
                                 f"{it_fp64} iterations of the full solve (the FP64 CG on the GPU runs the "
                                 f"reference's iteration)"}
            else:
                cpu = {"value": None, "unit": "ms", "cores": 0, "kind": "reference",
                       "sample": "oracle/_ref not built on this host"}
        except Exception as e:     # the baseline is reported, never required
            cpu = {"value": None, "unit": "ms", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    if rank != 0:
        return
    value = replicas.job_time_per_solve(ms_mixed, world)
    line = {
        "metric": METRIC,
        "value": value, "unit": "ms", "n_gpus": world, "steps": a.steps, "warmup": max(3, a.warmup),
        "ms_per_step": ms_mixed, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "mixed precision: " + DTYPE[a.inner], "data": "synthetic",
        "config": {"workload": workload_name(a.dims), "mass": MASS, "csw": CSW, "prec_squared": PREC,
                   "links": links_desc(info, a.dims),
                   "l2": "inputs larger than L2 (links 604 MB, clover 604 MB), no flush",
                   "parallelism": f"replicas x{world}"},
        "solver": {"inner": a.inner, "delta": a.delta, "iterations": st["iterations"],
                   "reliable_updates": st["reliable_updates"], "fallback": st["fallback"], "true_residual": true_res},
        "fp64_cg": {"ms": ms_fp64, "iterations": it_fp64, "speedup_mixed_vs_fp64": ms_fp64 / ms_mixed},
        "dslash_fp64": {"ms": ms_hop, "GB_s": hop_gbs, "bytes_per_site": bytes_per_site, "sites": V // 2},
        "roofline": {"bound": "hbm",
                     "kernel": "inner operator step 1 (k_shop<16,32,32,6,1,0>, or k_shop_shaped in the block shape "
                               "the tuner chose for this lattice: FP16 spinors + norms, FP32 12-real links, FP32 "
                               "packed clover; 2 of the 5 launches of an inner iteration)",
                     "achieved": inner_gbs, "peak": peak, "unit": "GB/s", "frac": inner_gbs / peak,
                     "peak_kind": peak_kind, "traffic": inner_traffic(a.inner, V // 2),
                     "traffic_source": INNER_NCU.get(a.inner, (0, 0, "no ncu capture of this inner format"))[2],
                     "ms_per_launch": ms_inner,
                     "bytes_per_launch": inner_bytes,
                     "bytes_per_site": inner_bytes / (V // 2)},
        "e2e": {"value": replicas.job_time_per_solve(ms_e2e, world), "unit": "ms", "h2d_bytes_per_step": field_bytes,
                "d2h_bytes_per_step": field_bytes},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    if variants is not None:
        line["inner_variants"] = variants
    if batched is not None:
        line["batched"] = batched
    print(json.dumps(line))


def main():
    a = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        import datetime
        backend = "nccl" if a.impl == "ours" else "gloo"
        if a.impl == "ours":
            import torch
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        dist_mod.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
        dist = dist_mod
    try:
        if a.mesons:
            run_mesons(a)
        elif a.lattices:
            run_lattices(a)
        elif a.hmc:
            run_hmc(a)
        elif a.rhmc:
            run_rhmc(a)
        elif a.learned:
            run_learned(a)
        elif a.mshift:
            run_mshift(a)
        elif a.impl == "reference":
            run_reference(a, rank, world)
        else:
            run_ours(a, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
