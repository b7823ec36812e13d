/*
 * yahmc_gpu.h -- C ABI of the B200 (sm_100a) fermion engine for YaHMC.
 *
 * The engine replaces YaHMC's fermion hot path: the even-odd preconditioned
 * Wilson-clover Dirac operator, the clover term and its site-local inverse, the
 * inverters, the spinor-field linear algebra and the fermion forces.  Every
 * entry point below names the reference function it replaces (file:line in
 * the YaHMC tree).  A C++ shim with YaHMC's own signatures (dirac.h,
 * inverter.h, linalg.h, clover.h, forces.h) sits on top of this ABI
 * (integration/yahmc_gpu_shim.cpp).
 *
 * Conventions
 *  - Plain C types only.  Every function returns an int status (yg_status);
 *    yg_last_error() gives the message of the last failure on this thread.
 *  - A lattice handle owns the device copies of the global state the reference
 *    keeps in globals: represented links (gfield_repr), fundamental links
 *    (gfield_fund), clover term (cl_term), LDL factors (cl_ldl), clover force
 *    (cl_force) and momenta (afield_momenta).
 *  - Spinor fields are device buffers of yg_info.field_doubles doubles
 *    allocated by yg_field_alloc.  Their device layout is private (site-major
 *    structure of arrays); yg_field_upload / yg_field_download convert from /
 *    to the reference's host layout: V records Spinor{re[d][4], im[d][4]}
 *    (include/spinor.h:7-9) in the reference's site order.
 *  - view arguments select the site range like spinor_select_* / spinor_type_*
 *    (linalg.cpp:272-329): YG_VIEW_DEFAULT (even sites with even-odd
 *    preconditioning, all sites without), YG_VIEW_EVEN, YG_VIEW_ODD, YG_VIEW_FULL.
 *  - Precisions are squared relative residuals, as in the reference
 *    (README.md:154, cg.cpp:189).
 *  - All work is issued on the lattice's stream (default: the legacy default
 *    stream); functions returning host scalars synchronise it.
 */
#ifndef YAHMC_GPU_H
#define YAHMC_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  YG_OK = 0,
  YG_ERR_ARG = 1,          /* invalid argument or unsupported configuration */
  YG_ERR_CUDA = 2,         /* CUDA runtime error */
  YG_ERR_OOM = 3,          /* device allocation failed (memory.cpp:11-18 analogue) */
  YG_MAXITER = 4,          /* solver reached maxiter before the stopping criterion */
  YG_STALL = 5,            /* solver stopped making progress */
  YG_NONFINITE = 6,        /* NaN/Inf met in a reduction */
  YG_TIMEOUT = 7           /* a bounded device-side wait gave up */
} yg_status;

enum { YG_BC_PERIODIC = 0, YG_BC_ANTIPERIODIC = 1, YG_BC_OPEN = 2, YG_BC_SF = 3 };
enum { YG_REPR_FUNDAMENTAL = 0, YG_REPR_ADJOINT = 1, YG_REPR_SYMMETRIC = 2, YG_REPR_ANTISYMMETRIC = 3 };
enum { YG_VIEW_DEFAULT = 0, YG_VIEW_EVEN = 1, YG_VIEW_ODD = 2, YG_VIEW_FULL = 3 };
enum { YG_OP_DPHI = 0, YG_OP_HPHI = 1, YG_OP_HPHI_SQ = 2 };

typedef struct yg_lattice yg_lattice;

/* Compile-time physics switches of the reference (programs/Makefile:6-45)
 * become run-time parameters: NC, REPR_*, BC_*, CLOVER_TERM, UPDATE_EO. */
typedef struct {
  int dims[4];   /* T, X, Y, Z: even, >= 2 (the reference itself needs >= 8, geometry.cpp:1140) */
  int nc;        /* N of SU(N): 2, 3 or 4 */
  int repr;      /* YG_REPR_*, the REPR_ID of include/repr.h:9-39 */
  int bc;        /* YG_BC_* (include/bcs.h:1-31) */
  int clover;    /* CLOVER_TERM */
  int eo;        /* UPDATE_EO */
  double csw;    /* clover coefficient (clover_init, clover.cpp:349-361) */
  double cf;     /* Dirac boundary coefficient for open / SF (bcs_init, bcs.cpp:68, 131) */
} yg_params;

typedef struct {
  long volume;         /* V (outer.vol4 on one rank) */
  long half_volume;    /* V/2 */
  int repr_dim;        /* d = REPR_DIM */
  int nc;
  int ng;              /* NC*NC-1 */
  long field_doubles;  /* doubles per spinor field = 8*d*V */
  long link_doubles;   /* doubles of the represented links = 4*V*2*d*d */
  long fund_doubles;   /* doubles of the fundamental links = 4*V*2*N*N */
  long mom_doubles;    /* doubles of the momenta = 4*V*NG */
} yg_info;

typedef struct {
  int op;              /* YG_OP_*: the mvm of inv_par (inverter.h:6-16) */
  double mass;         /* inv_par.mass */
  double prec;         /* inv_par.prec: squared relative residual */
  int log;             /* inv_par.log: print one line per solve to stderr */
  int maxiter;         /* 0 = unlimited, as the reference */
} yg_inv_par;

typedef struct {
  int iterations;      /* inner (operator-level) iterations */
  int reliable_updates;
  int fallback;        /* 1 if the solver fell back to plain FP64 CG */
  double true_residual;/* |b - A x|^2 / |b|^2 recomputed in FP64 at exit */
  double seconds;
} yg_solve_stats;

/* ---- lifecycle --------------------------------------------------------- */
/* replaces geometry_init + repr_init + bcs_init + clover_init + gauge_field_init
 * (programs/hmc.cpp:94-117; geometry.cpp:1032-1191, repr.cpp:17-105,
 * bcs.cpp:11-137, clover.cpp:349-361, gaugefield.cpp:15-30) */
int yg_lattice_create(const yg_params *p, yg_lattice **out);
/* No reference counterpart (the reference is CPU/MPI): selects the CUDA device on which the
 * calling thread's next yg_lattice_create places its state (one process per GPU: call it
 * with the local rank first).  Each lattice keeps the device it was created on. */
int yg_set_device(int device);
void yg_lattice_destroy(yg_lattice *lat);
int yg_lattice_query(const yg_lattice *lat, yg_info *out);
int yg_set_stream(yg_lattice *lat, void *cuda_stream);
int yg_synchronize(yg_lattice *lat);
const char *yg_last_error(void);
/* No reference counterpart: page-lock (and release) a host array that is copied to and from
 * the device often, e.g. the host application's gfield_fund and afield_momenta, so that those
 * copies run at full PCIe speed.  bytes > 0. */
int yg_host_register(void *host, size_t bytes);
int yg_host_unregister(void *host);
/* No reference counterpart: number of kernels this library has launched since it was
 * loaded (all lattices); benchmarks difference it around a timed region. */
long yg_launch_count(void);

/* ---- spinor fields (SpinorField, spinorfield.h:6-39; spinor_allocate linalg.cpp:10-27) */
int yg_field_alloc(yg_lattice *lat, double **dev_field);
int yg_field_free(yg_lattice *lat, double *dev_field);
int yg_field_upload(yg_lattice *lat, double *dev_field, const double *host_spinors);
int yg_field_download(yg_lattice *lat, double *host_spinors, const double *dev_field);

/* ---- gauge field ------------------------------------------------------- */
/* gfield_fund upload + represent_gauge_field (repr.cpp:265-280): represent links
 * (repr.cpp:107-263), rebuild the clover term (clover.cpp:330-347) and apply the
 * antiperiodic sign (bcs.cpp:264-272).  host: 4*V suNg records, index 4*id+mu. */
int yg_gauge_upload(yg_lattice *lat, const double *host_fund_links);
/* gfield_fund upload alone, without represent_gauge_field: the state the reference is in
 * after update_links (update.cpp:228-247) changed the links on the host and before the
 * next represent_gauge_field; the gauge forces read these links, the fermion operators
 * keep the represented field and clover term of the last yg_gauge_upload. */
int yg_gauge_upload_fund(yg_lattice *lat, const double *host_fund_links);
int yg_gauge_download(yg_lattice *lat, double *host_fund_links);
/* gfield_repr (4*V suNf records), cl_term (4*V suNf), cl_ldl for sigma=4+mass (V ldl_t) */
int yg_repr_links_download(yg_lattice *lat, double *host);
int yg_clover_term_download(yg_lattice *lat, double *host);
int yg_ldl_download(yg_lattice *lat, double mass, double *host);

/* ---- Dirac operator (dirac.h:6-16, dirac.cpp:706-781) ------------------ */
int yg_Dphi_oe(yg_lattice *lat, double *dst, double *src);
int yg_Dphi_eo(yg_lattice *lat, double *dst, double *src);
int yg_Dphi_ee(yg_lattice *lat, double mass, double *dst, double *src);
int yg_Dphi_oo(yg_lattice *lat, double mass, double *dst, double *src);
int yg_Dphi_oo_inv(yg_lattice *lat, double mass, double *dst, double *src);
/* Dphi writes scratch into the odd half of src, like the reference (dirac.cpp:743). */
int yg_Dphi(yg_lattice *lat, double mass, double *dst, double *src);
int yg_Hphi(yg_lattice *lat, double mass, double *dst, double *src);
int yg_Hphi_sq(yg_lattice *lat, double mass, double *dst, double *src);
int yg_mvm_get(yg_lattice *lat);                       /* dirac.cpp:11-18 */
void yg_mvm_reset(yg_lattice *lat);                    /* dirac.cpp:20-23 */

/* ---- clover (clover.h:39-44) ------------------------------------------- */
int yg_clover_logdet(yg_lattice *lat, double mass, double *out);   /* clover.cpp:281-305 */

/* ---- spinor linear algebra (linalg.h:7-34, linalg.cpp:29-270) ---------- */
int yg_spinor_zero(yg_lattice *lat, double *f);
int yg_spinor_copy(yg_lattice *lat, double *dst, const double *src);
int yg_spinor_g5(yg_lattice *lat, double *f, int view);
int yg_spinor_sqnorm(yg_lattice *lat, const double *f, int view, double *out);
int yg_spinor_product(yg_lattice *lat, const double *a, const double *b, int view, double *out_re_im);
int yg_spinor_product_re(yg_lattice *lat, const double *a, const double *b, int view, double *out);
int yg_spinor_add_assign(yg_lattice *lat, double *lhs, const double *rhs, int view);
int yg_spinor_sub_assign(yg_lattice *lat, double *lhs, const double *rhs, int view);
int yg_spinor_mulr(yg_lattice *lat, double *lhs, double v, const double *rhs, int view);
int yg_spinor_mulc(yg_lattice *lat, double *lhs, double re, double im, const double *rhs, int view);
int yg_spinor_mulr_assign(yg_lattice *lat, double *lhs, double v, int view);
int yg_spinor_mulc_assign(yg_lattice *lat, double *lhs, double re, double im, int view);
int yg_spinor_mulr_add_assign(yg_lattice *lat, double *lhs, double v, const double *rhs, int view);
int yg_spinor_mulc_add_assign(yg_lattice *lat, double *lhs, double re, double im, const double *rhs, int view);
int yg_spinor_mulr_sub_assign(yg_lattice *lat, double *lhs, double v, const double *rhs, int view);
int yg_spinor_mulc_sub_assign(yg_lattice *lat, double *lhs, double re, double im, const double *rhs, int view);

/* ---- inverters (inverter.h:18-22); iterations returned through *iters --- */
int yg_cg_inverter(yg_lattice *lat, const yg_inv_par *par, double *x, double *b, int *iters);        /* cg.cpp:132-202 */
int yg_bicgstab_inverter(yg_lattice *lat, const yg_inv_par *par, double *x, double *b, int *iters);  /* bicgstab.cpp:9-97 */
int yg_minres_inverter(yg_lattice *lat, const yg_inv_par *par, double *x, double *b, int *iters);    /* minres.cpp:12-117 */
int yg_auto_inverter(yg_lattice *lat, const yg_inv_par *par, double *x, double *b, int *iters);      /* inverter.cpp:9-55 */
/* cg.cpp:11-130; xs: num device fields; x_n solves (A + shifts[n]) x_n = b from a zero guess */
int yg_cg_mshift(yg_lattice *lat, const yg_inv_par *par, int num, const double *shifts,
                 double *const *xs, double *b, int *iters);
/* rational.cpp:134-166: x = a0*b + sum_i residues[i] * (A + poles[i])^-1 b */
int yg_rational_calc(yg_lattice *lat, const yg_inv_par *par, double a0, int order, const double *poles,
                     const double *residues, double *x, double *b, int *iters);
/* No reference counterpart: CG on the same operator with FP32 inner iterations and FP64
 * reliable updates; stops on the TRUE FP64 squared residual |b-Ax|^2 < prec*|b|^2.  Uses
 * the compressed inner operator for d = 3 (FP16 spinors with per-site norms, FP32 links in
 * the format yg_tune_inner_links measures fastest on the lattice at the first call, FP32
 * clover blocks, delta 0.1, the CG update fused into the operator, launch shapes tuned at
 * the first call; if that stalls, the inner solve restarts with FP32 spinors from its best
 * iterate) and the generic FP32 operator otherwise.  stats->fallback: bit 0 the FP64 CG
 * finished the solve, bit 1 the inner storage was raised to FP32.  Returns YG_STALL when even
 * the FP64 CG cannot bring the true residual below prec (x then holds the FP64 CG's solution,
 * which met prec on its recursive residual). */
int yg_cg_mixed(yg_lattice *lat, const yg_inv_par *par, double *x, double *b, yg_solve_stats *stats);

/* No reference counterpart: nrhs cg_inverter solves (cg.cpp:132-202) of the same operator
 * (Hphi or Hphi_sq) advanced together.  Every system follows the reference's recurrence,
 * initial guess (xs[i] on entry), stopping rule |r_i|^2 < prec |b_i|^2 and iteration count
 * (iters[i]); the operator is applied to all systems in one launch per step, so the links
 * and the clover term are read once for all of them.  1 <= nrhs <= 16, d = 3, even-odd.
 * Sources must vanish on the open/SF boundary slices, as spinor_random's do. */
int yg_cg_inverter_multi(yg_lattice *lat, const yg_inv_par *par, int nrhs, double *const *xs, double *const *bs,
                         int *iters);
/* No reference counterpart: n <= 64 independent cg_inverter solves, one per lattice (lattices of
 * any sizes and configurations, each at most once), run concurrently.  Hphi_sq solves on
 * even-odd lattices of one representation dimension d (2, 3, 4 or 6), all with or all without
 * a clover term and without open/SF boundaries, run as ONE persistent cooperative kernel: a
 * group of blocks per lattice, sized by its volume, runs the lattice's whole CG loop on the
 * device with bounded barriers.  Other mixes run a host thread and the lattice's own stream
 * per solve.  Results and iteration counts are those of separate yg_cg_inverter calls (to
 * rounding); returns the worst status.  Every lattice must have been created on the calling
 * thread's current device (YG_ERR_ARG otherwise). */
int yg_cg_inverter_lattices(int n, yg_lattice *const *lats, const yg_inv_par *pars, double *const *xs,
                            double *const *bs, int *iters);
/* As yg_cg_inverter_lattices, with the persistent kernel's barrier wait limit in GPU clock
 * cycles (<= 0: the default, about 10 s): a wait that runs out ends the launch and the call
 * returns YG_TIMEOUT (the fields then hold a partial solve; the context stays usable).
 * *persistent (may be NULL) is set to 1 when the persistent kernel ran, 0 for the threads. */
int yg_cg_inverter_lattices_ex(int n, yg_lattice *const *lats, const yg_inv_par *pars, double *const *xs,
                               double *const *bs, int *iters, long long wait_cycles, int *persistent);
/* No reference counterpart: nrhs <= 16 bicgstab_inverter solves on Dphi (bicgstab.cpp:9-97,
 * each system with its own scalars, stopping test and iteration count) sharing every operator
 * application; even-odd lattices with d = 3 */
int yg_bicgstab_inverter_multi(yg_lattice *lat, const yg_inv_par *par, int nrhs, double *const *xs,
                               double *const *bs, int *iters);

/* No reference counterpart: nrhs solves of Hphi_sq with low-precision inner iterations (the
 * compressed operator: FP16 spinors with per-site norms, FP32 links and clover blocks, one
 * launch per Schur step for all systems, the CG update fused into the last step) and FP64
 * reliable updates, advanced together; every system stops on its own TRUE FP64 residual
 * |b_i - A x_i|^2 < prec |b_i|^2 (a system that stalls continues with the FP64 CG).
 * stats[i] per system.  1 <= nrhs <= 16, d = 3, even-odd; xs[i] on entry is the initial guess. */
int yg_cg_mixed_multi(yg_lattice *lat, const yg_inv_par *par, int nrhs, double *const *xs, double *const *bs,
                      double delta, yg_solve_stats *stats);
/* As yg_cg_mixed_multi with a mass per system (masses[i] replaces par->mass; at most 4
 * distinct values): the solves of several monomials at once, e.g. the Hphi_sq solves of the
 * HMC monomial (mass m + dm) and of the Hasenbusch monomial (mass m) of one force evaluation
 * (hmc.cpp:68-94, hasenbusch.cpp:67-96) in the same operator launches. */
int yg_cg_mixed_multi_masses(yg_lattice *lat, const yg_inv_par *par, int nrhs, const double *masses,
                             double *const *xs, double *const *bs, double delta, yg_solve_stats *stats);

/* No reference counterpart (measurement support): mean time per launch of `reps` launches of
 * step 1 of yg_cg_mixed's inner operator (its dominant kernel), timed with CUDA events on the
 * lattice's stream, and the compulsory bytes one launch moves. */
int yg_inner_hop_profile(yg_lattice *lat, double mass, int reps, double *ms_per_launch, double *bytes_per_launch);

/* No reference counterpart: options of the mixed-precision solver.
 *   inner_precision  32 (FP32 storage) or 16 (FP16 storage with per-site norms), FP32
 *                    arithmetic; 0 selects the generic FP32 operator of yg_cg_mixed (any d)
 *   link_reals       18, or 12 (two rows, third rebuilt; SU(3) fundamental only), or 8 (SU(3)
 *                    fundamental, FP32 link storage, periodic or antiperiodic boundaries: one row
 *                    and the smaller of two first-column entries in full, two phases; rebuilt
 *                    from unitarity and det = 1)
 *   delta            reliable update when |r| falls below delta * |r| at the last update
 *   link_storage,    storage of the inner operator's links and clover blocks; the combinations
 *   clover_storage   built are all-FP32, FP32 spinors with int16 links (FP32 or int16 clover),
 *                    and FP16 spinors with FP32, FP16 or int16 matrices
 * The compressed inner operator exists for d = 3 representations with even-odd
 * preconditioning; the stopping test is the true FP64 residual, as for yg_cg_mixed. */
typedef struct {
  int inner_precision;
  int link_reals;
  double delta;
  int link_storage;     /* 0: as inner_precision; 32 FP32, 16 FP16, 15 int16 fixed point (entries / 32767) */
  int clover_storage;   /* 0: as inner_precision; 32, 16, or 15 (int16 with a per-site scale) */
  int escalate;         /* 1: a stalled FP16 inner solve restarts with FP32 storage (as yg_cg_mixed) */
} yg_mixed_opts;
int yg_cg_mixed_opts(yg_lattice *lat, const yg_inv_par *par, const yg_mixed_opts *opts, double *x, double *b,
                     yg_solve_stats *stats);

/* No reference counterpart (autotuning): times the step-1 hop of the compressed inner operator
 * for each FP32 link format allowed on this lattice (18 reals; 12 for SU(3) fundamental; 8 as
 * well on periodic / antiperiodic lattices) and keeps the fastest for yg_cg_mixed, which runs
 * this itself at its first call on a lattice.  ms_per_hop (may be NULL): 3 doubles, the mean
 * hop time of the 18-, 12- and 8-real formats, 0 where not a candidate. */
int yg_tune_inner_links(yg_lattice *lat, double mass, int *link_reals, double *ms_per_hop);

/* ---- propagators and mesons (observables/propagator.cpp, observables/mesons.cpp) ---- */
enum { YG_MESON_SEMWALL = 0x01, YG_MESON_POINT = 0x02 };   /* include/spectrum.h:7-8 */
/* create_point_source (propagator.cpp:58-73): src = unit vector of spin n / d, colour n % d
 * at (tau, 0, 0, 0) */
int yg_create_point_source(yg_lattice *lat, int n, int tau, double *src);
/* create_semwall_source (propagator.cpp:22-56).  For n = 0, z2 holds the 2*d*vol3 rand_z2()
 * values in the reference's draw order: the sites of slice tau by increasing site index, per
 * site re, im of colour 0..d-1 (a shim that draws them with the reference's generator
 * reproduces its sources exactly); z2 is ignored for n > 0 (spin n-1 moves to spin n). */
int yg_create_semwall_source(yg_lattice *lat, int n, int tau, const double *z2, double *src);
/* calc_propagator (propagator.cpp:75-166): dst holds the initial guess */
int yg_calc_propagator(yg_lattice *lat, double mass, double prec, double *dst, double *src, int *iters);
/* No reference counterpart: n <= 16 propagators of one source slice (d = 3) with every operator
 * application shared.  solver 0: batched BiCGstab on the even-site system (the reference's
 * recurrence per system, dst[i] the initial guess); 1: batched mixed-precision CG on Hphi_sq;
 * 2: batched FP64 CG on Hphi_sq (both from zero).  Same stopping rule as calc_propagator. */
int yg_calc_propagator_multi(yg_lattice *lat, double mass, double prec, int n, double *const *dst,
                             double *const *src, int solver, int *iters);
/* contract_all_correlators (mesons.cpp:105-128): corr[16*T] += the slice sums of the sixteen
 * channels (order id g1 g2 g3 g5 g5g1 g5g2 g5g3 g0g1 g0g2 g0g3 g0g5 g0g5g1 g0g5g2 g0g5g3
 * g5_g0g5) at t - tau; props: 4 (SEMWALL) or 4*d (POINT, index spin*d + colour) fields */
int yg_meson_contract(yg_lattice *lat, int method, int tau, const double *const *props, int nprops, double *corr);

/* ---- Wilson and fermion flow (observables/wilsonflow.cpp, observables/fermionflow.cpp) ---- */
/* wf_init (wilsonflow.cpp:149-157): zero the flow's momentum field (the MD momenta) */
int yg_wf_init(yg_lattice *lat);
/* wf_zeta (wilsonflow.cpp:8-23) and wf_update (wilsonflow.cpp:25-41), the two halves of a stage */
int yg_wf_zeta(yg_lattice *lat, double alpha);
int yg_wf_update(yg_lattice *lat, double val);
/* wf_iterate (wilsonflow.cpp:43-53): one third-order Runge-Kutta step of the Wilson flow.
 * Like the reference it changes the fundamental links only: call yg_represent_gauge_field
 * before applying a Dirac operator to the flowed field. */
int yg_wf_iterate(yg_lattice *lat, double eps);
/* wf_e_plaq, wf_e_sym, wf_charge (wilsonflow.cpp:55-147) from one pass; any pointer may be NULL */
int yg_wf_observables(yg_lattice *lat, double *e_plaq, double *e_sym, double *charge);
/* wf_fermion_init (fermionflow.cpp:76-92) for n <= 32 fields, and wf_fermion_iterate
 * (fermionflow.cpp:28-74): one step of the gauge flow with the n fields phi[i] flowed in place
 * (pass the same fields, in the same order, at every step) */
int yg_wf_fermion_init(yg_lattice *lat, int n);
int yg_wf_fermion_iterate(yg_lattice *lat, double eps, double *const *phi, int n);

/* ---- gauge configuration files (gaugefield.cpp:44-179, hirep.cpp:56-212) ---- */
/* CFG: 256-byte header (ident, version, dims, nc, repr, num_cnfg, num_accept, plaquette),
 * HiRep: big-endian (N, T, X, Y, Z, plaquette); both then every site's four links in
 * t, x, y, z order.  Loading checks the header against the lattice (an error where the
 * reference stops), applies the gauge boundary conditions, represents the field, and
 * returns |stored plaquette - plaquette of the loaded field|. */
int yg_gauge_save_cfg(yg_lattice *lat, const char *path, int num_cnfg, int num_accept);
int yg_gauge_load_cfg(yg_lattice *lat, const char *path, int *num_cnfg, int *num_accept, double *plaquette_diff);
int yg_gauge_save_hirep(yg_lattice *lat, const char *path);
int yg_gauge_load_hirep(yg_lattice *lat, const char *path, int *num_cnfg, double *plaquette_diff);

/* ---- learned preconditioner (no reference counterpart) ------------------
 * A gauge-covariant parallel-transport convolution network: each layer maps Ci channels of
 * spinor fields on the whole lattice to Co channels,
 *     out[x, o] = sum_p sum_i W[p, o, i] (T_p in_i)(x),
 * over nine paths p (0 the site, 1..4 a hop forward along mu = p-1 through U_mu(x), 5..8 a hop
 * backward through U_mu(x-mu)^dag, the represented links the Dirac operator uses), W[p, o, i]
 * a complex 4x4 spin matrix.  Colour meets only the links, so the network commutes with gauge
 * transformations exactly.  Channels 1 -> C -> ... -> C -> 1 with C = 8 or 16, d = 3; layers
 * are linear.  The per-site channel mixing runs as BF16 products with FP32 accumulation on the
 * tensor cores (forward, adjoint and weight gradient).
 * Weights: 9*Co*Ci*4*4 complex numbers as (re, im) doubles, index ((p*Co + o)*Ci + i)*16 + s*4 + s'.
 * Activations (yg_ptc_layer): float site blocks, channel ch of site id (the reference's site
 * order) is 24 floats at (ch*V + id)*24, float (spin*3 + colour)*2 + re/im. */
typedef struct yg_ptc yg_ptc;
int yg_ptc_create(yg_lattice *lat, int nlayers, const int *channels, yg_ptc **out);
int yg_ptc_destroy(yg_ptc *net);
int yg_ptc_set_weights(yg_ptc *net, int layer, const double *w);
int yg_ptc_get_weights(yg_ptc *net, int layer, double *w);
/* one layer on device activations; adjoint = 1: the input-gradient layer (Co -> Ci) */
int yg_ptc_layer(yg_ptc *net, int layer, int adjoint, const float *dev_in, float *dev_out);
/* dst (even sites) = the network applied to the even-site field src embedded with zero odd
 * sites (the even-even block of D^-1 is the inverse of the Schur operator Dphi) */
int yg_ptc_apply(yg_ptc *net, double *dst, const double *src);
/* training: loss = sum_k |N(r_k) - e_k|^2 / |e_k|^2 over even-site pairs with Dphi e_k = r_k,
 * and its gradient d loss / d conj(W), all layers' weights concatenated in the layout above */
int yg_ptc_gradient(yg_ptc *net, int npairs, double *const *r, double *const *e, double *loss, double *grads);
/* weight gradients d loss / d conj(W) for any loss whose derivative with respect to conj(N(src))
 * (on the even sites) is the field gout: forward on src, backward from gout */
int yg_ptc_backward(yg_ptc *net, const double *src, const double *gout, double *grads);
/* flexible GCR on Dphi with the network as right preconditioner (net may be NULL: plain GCR),
 * restarted every `restart` directions; the true FP64 residual |b - Dphi x|^2 < prec |b|^2 ends
 * the solve; no progress over four restart cycles hands over to the plain even-odd CG on the
 * normal equations (stats->fallback = 1) */
int yg_fgcr(yg_lattice *lat, yg_ptc *net, const yg_inv_par *par, int restart, double *x, double *b,
            yg_solve_stats *stats);
/* Hphi_sq x = b as two such Dphi solves (gamma5 D gamma5 D, as auto_inverter, inverter.cpp:27-34);
 * the true Hphi_sq residual decides, and the FP64 CG finishes if it is not met (fallback bit 1) */
int yg_solve_learned(yg_lattice *lat, yg_ptc *net, const yg_inv_par *par, int restart, double *x, double *b,
                     yg_solve_stats *stats);

/* ---- chronological initial guess (mre.h) -------------------------------- */
/* The past solutions live on the device.  op is YG_OP_DPHI / HPHI / HPHI_SQ (mre_par.mvm),
 * max <= 15 (MRE_MAX); max = 0 disables the extrapolation (yg_mre_guess leaves dst alone). */
typedef struct yg_mre yg_mre;
int yg_mre_init(yg_lattice *lat, int max, int op, double mass, yg_mre **out);   /* mre.cpp:85-111 */
int yg_mre_store(yg_mre *m, const double *solution);                          /* mre.cpp:35-51 */
int yg_mre_guess(yg_mre *m, double *dst, const double *src);                  /* mre.cpp:53-83 */
int yg_mre_reset(yg_mre *m);                                                   /* mre.cpp:113-116 */
int yg_mre_free(yg_mre *m);

/* ---- forces (forces.h:6-15) -------------------------------------------- */
int yg_momenta_upload(yg_lattice *lat, const double *host);     /* afield_momenta, 4*V suNa */
int yg_momenta_download(yg_lattice *lat, double *host);
int yg_momenta_zero(yg_lattice *lat);
int yg_clover_force_download(yg_lattice *lat, double *host);    /* cl_force, 6*V suNf */
int yg_begin_fermion_force(yg_lattice *lat);                                                        /* forces.cpp:239-251 */
int yg_end_fermion_force(yg_lattice *lat, double dt);                                               /* forces.cpp:254-259 */
int yg_wilson_fermion_force(yg_lattice *lat, double dt, double mass, double residue, double *lhs, double *rhs); /* forces.cpp:175-227 */
int yg_wilson_fermion_force_q(yg_lattice *lat, double dt, double mass, double residue, double *rhs);            /* forces.cpp:230-236 */
int yg_clover_fermion_force(yg_lattice *lat, double residue, double *lhs, double *rhs);             /* forces.cpp:122-172 */
/* The pole loop of MonomialRHMC::update (monomials/rhmc.cpp:100-103): wilson_fermion_force_q(dt, mass,
 * residues[k], rhs[k]) for k < n <= 32, as one batched force (the links are read, and cl_force and the
 * momenta written, once for all poles); the odd halves of rhs[k] are replaced as by the reference */
int yg_wilson_fermion_force_q_multi(yg_lattice *lat, double dt, double mass, int n, const double *residues,
                                    double *const *rhs);
int yg_clover_logdet_force(yg_lattice *lat, double mass, double residue);                           /* forces.cpp:109-119 */
int yg_wilson_gauge_force(yg_lattice *lat, double dt, double beta);                                 /* forces.cpp:262-283 */
int yg_avr_plaquette(yg_lattice *lat, double *out);                                                 /* wilsonloop.cpp:116-133 (1x1) */

/* ---- molecular dynamics on the fundamental links (update.cpp, forces.cpp, wilsonloop.cpp) ----
 * Momenta stay on the device between these calls (yg_momenta_upload/download move them). */
int yg_improved_gauge_force(yg_lattice *lat, double dt, double beta, double c0, double c1);        /* forces.cpp:285-309 */
int yg_avr_wilson(yg_lattice *lat, int height, int width, double *out);                            /* wilsonloop.cpp:116-133 */
int yg_gauge_action(yg_lattice *lat, double beta, double c0, double *out);                         /* monomials/gauge.cpp:21-40 */
/* update.cpp:228-247: U <- exp(eps P) U with the momentum and link boundary conditions; like
 * the reference it changes the fundamental links only, the represented field (and the clover
 * term) follow at yg_represent_gauge_field */
int yg_update_links(yg_lattice *lat, double eps);
int yg_represent_gauge_field(yg_lattice *lat);                                                     /* repr.cpp:265-280 */
int yg_reunitarize(yg_lattice *lat);                                                               /* update.cpp:269-279 */
/* reset_variables, momentum part (update.cpp:254-267): Gaussian algebra components with the
 * reference's standard deviation 1/sqrt(2) (random.h:15), drawn from a Philox4x32-10 stream
 * keyed by seed (the reference's ranlux stream is not reproduced) */
int yg_momenta_gaussian(yg_lattice *lat, unsigned long long seed);
int yg_momenta_action(yg_lattice *lat, double *out);                /* hamiltonian(), momentum part: update.cpp:201-220 */
int yg_gauge_backup(yg_lattice *lat);                                                              /* gaugefield.cpp:32-36 */
int yg_gauge_restore(yg_lattice *lat);                                                             /* gaugefield.cpp:38-42 */

/* ---- allocation-free reduction ------------------------------------------ */
/* No counterpart in the reference.  For callers that cannot allocate device memory (no
 * lattice handle needed): sum of |a_i|^2 over n_words complex FP64 words at dev_words,
 * written to the device double *dev_out on the given stream (NULL = legacy default).
 * Uses a fixed 128 KiB scratch array inside the library instead of cudaMalloc, so
 * n_words <= 16,777,216 (larger sizes return YG_ERR_ARG).  dev_words must be 16-byte
 * aligned (the words are read as pairs of doubles) and dev_out 8-byte aligned; other
 * pointers return YG_ERR_ARG before anything is launched.  The first call on a device
 * looks up that array's device address (cached per process, safe from several host
 * threads) and should come before any stream capture; calls that overlap on the GPU
 * share the array and race. */
int yg_field_sqnorm_noalloc(const double *dev_words, long n_words, double *dev_out, void *stream);

#ifdef __cplusplus
}
#endif

#endif
