// Private state of a yg_lattice handle and the engine functions shared by the host
// translation units.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <atomic>
#include <string>
#include <vector>
#include <stdexcept>
#include "yg_core.cuh"
#include "../../include/yahmc_gpu.h"

namespace yg {

// Error carrying a yg_status; the C ABI layer converts it to a return code.
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

void check_cuda(cudaError_t e, const char *what);
#define YG_CUDA(x) ::yg::check_cuda((x), #x)

// Kernels launched by this library since load (all lattices).  Every launch site is followed
// by YG_LAUNCHED(), which checks the launch and counts it (atomically: the concurrent
// per-lattice solves launch from several host threads).
extern std::atomic<long> g_launch_count;
#define YG_LAUNCHED()                                              \
  do {                                                             \
    ::yg::check_cuda(cudaGetLastError(), "kernel launch");         \
    ++::yg::g_launch_count;                                        \
  } while (0)

// Device buffer owned by a lattice.
struct DevBuf {
  void *p = nullptr;
  size_t bytes = 0;
  void alloc(size_t n);
  void release();
  template <typename T> T *as() const { return reinterpret_cast<T *>(p); }
};

// Device tables describing the representation.
struct ReprTables {
  double2 *basis;    // d x N x N basis matrices b_n (repr.cpp:25-59)
  double2 *itrepr;   // NG x d x d generators of the fermion representation (repr.cpp:73-104)
  double2 *itfund;   // NG x N x N generators of the fundamental representation
};

constexpr int kStep2Shapes = 3;   // register variants of the inner operator's step-2 kernels

struct Lattice {
  yg_params p{};
  Geom g{};
  int d = 0, nc = 0, ng = 0;
  long V = 0, Vh = 0;
  cudaStream_t stream = 0;
  int mvm = 0;
  int device = 0;          // the CUDA device the lattice was created on

  DevBuf fund;      // fundamental links, 4 x N x N per site        (gfield_fund)
  DevBuf fund_backup;  // gauge_field_backup copy of fund
  DevBuf links;     // represented links with the AP sign, 4 x d x d (gfield_repr)
  DevBuf clover;    // clover term, 4 x d x d per site                (cl_term)
  DevBuf ldl;       // LDL factors, 2 x d(2d+1) per site of block 1   (cl_ldl)
  double ldl_sigma = 0;
  bool ldl_valid = false;
  DevBuf cpk64;     // packed Hermitian FP64 inverse of the odd-site blocks, d <= 6 (rebuilt with ldl)
  DevBuf cl_force;  // 6 x d x d per site                            (cl_force)
  DevBuf mom;       // 4 x NG per site                               (afield_momenta)
  DevBuf tables;    // basis / generators
  ReprTables rt{};

  // reduction scratch: per-block partial sums + result
  DevBuf red_partial;
  DevBuf red_result;
  double *host_result = nullptr;   // pinned
  int red_blocks = 0;

  // scratch spinor fields (the reference's static SpinorFields, e.g. dirac.cpp:741)
  std::vector<double *> scratch;
  double *scratch_field(int i);

  // single-precision mirrors for the mixed-precision solver
  DevBuf links_f;   // represented links in float2
  DevBuf clover_f;  // clover term in float2
  DevBuf cinv_f;    // explicit inverse of the odd-site clover blocks, float2
  double cinv_f_sigma = 0;
  bool links_f_valid = false;
  bool cinv_f_valid = false;

  // compressed inner operator of the mixed solver for d = 3 (yg_sloppy.cu)
  DevBuf sl_links;  // 12 or 18 reals per link, FP32 or FP16
  DevBuf sl_clover; // packed Hermitian blocks: M_e on even sites, M_o^-1 on odd sites
  int sl_prec = 0, sl_reals = 0, sl_lfmt = 0, sl_cfmt = 0;
  DevBuf sl_cnorm;     // per-site scales of int16 clover records
  double sl_mass = 0;
  bool sl_valid = false;
  int sl_tuned_reals = 0;  // link format of the default mixed solve (tune_inner_links), 0 = not yet
  int sl_shape = 0;        // block shape of the inner step-1 hop (tune_shape), 0 = the default
  int sl_shape_reals = 0;  // link reals sl_shape was tuned for, 0 = not yet
  DevBuf sl_part;      // per-block partial sums of the device-scalar reductions
  int sl_grid_vec = 0; // blocks of the inner vector kernels
  // resident-grid sizes of the two step-2 kernels of an inner iteration (the hop forming
  // <p, A p>, and the last Schur step with the fused CG update) for each register variant,
  // the variants in use (tuned), and where the |r|^2 partials start in sl_part
  int sl_gnrm[kStep2Shapes] = {0, 0, 0}, sl_gcg[kStep2Shapes] = {0, 0, 0};
  int sl_shape_n = 0, sl_shape_c = 0;
  int sl_part_off = 0;
  DevBuf sl_scal;      // device scalars of the inner CG (rr, alpha, beta, ...) + completion counter
  double *sl_hist = nullptr;          // mapped pinned host ring of inner |r|^2 (written by the GPU)
  cudaEvent_t sl_ev[2] = {nullptr, nullptr};

  // multi-right-hand-side mixed CG (yg_mrhs.cu): per-system working storage, device
  // scalars, reduction partials and the mapped host ring of per-system |r|^2
  DevBuf mr_work;
  int mr_cap = 0;
  DevBuf mr_scal, mr_part;
  DevBuf mr_clov;      // packed FP32 clover blocks of the further masses of a multi-mass call
  double *mr_hist = nullptr;
  int mr_tile[17] = {};   // measured inner-operator variant (tile, threads per site) + 1, + 8 for 18-real
                          // links, per system count

  long field_doubles() const { return 8L * d * V; }
  size_t field_bytes() const { return sizeof(double) * field_doubles(); }

  // site range of a view (spinor_select_* / spinor_type_*, linalg.cpp:272-329)
  void view_range(int view, long &lo, long &n) const;

  ~Lattice();
};

// ---- yg_lattice.cu
Lattice *lattice_create(const yg_params &p);
void represent_and_clover(Lattice &L);
void ensure_ldl(Lattice &L, double sigma);
constexpr int kPackedInverseMaxD = 6;   // largest d whose FP64 Schur step uses the packed inverse
void gauge_upload(Lattice &L, const double *host);
void gauge_upload_fund(Lattice &L, const double *host);
void gauge_download(Lattice &L, double *host);
void repr_download(Lattice &L, double *host);
void clover_download(Lattice &L, double *host);
void clover_force_download(Lattice &L, double *host);
void ldl_download(Lattice &L, double mass, double *host);
void field_upload(Lattice &L, double *dev, const double *host);
void field_download(Lattice &L, double *host, const double *dev);
void momenta_upload(Lattice &L, const double *host);
void momenta_download(Lattice &L, double *host);

// ---- yg_dirac.cu: hop (dirac_kernel, dirac.cpp:227-704); part 1 even, 2 odd, 3 both
void bc_zero_field(Lattice &L, double *f);
void hop(Lattice &L, double *dst, const double *src, int part, double sign, bool assign);
void clover_apply(Lattice &L, double mass, double *dst, const double *src, int part, bool assign);
void clover_inv_apply(Lattice &L, double mass, double *dst, const double *src, int part, bool assign);
//   step 1: tmp_o = A_oo^-1 ( 1/2 H_oe src_e ), optionally also writing 1/2 H_oe src_e to clob_o
//   step 2: dst_e = A_ee src_e - 1/2 H_eo tmp_o  [then gamma5]
void schur_step1(Lattice &L, double mass, double *tmp, const double *src, double *clob);
void schur_step2(Lattice &L, double mass, double *dst, const double *tmp, const double *src, bool g5);
void dphi(Lattice &L, double mass, double *dst, double *src);
void hphi(Lattice &L, double mass, double *dst, double *src);
void hphi_sq(Lattice &L, double mass, double *dst, double *src);
void apply_op(Lattice &L, int op, double mass, double *dst, double *src);
void hphi_float(Lattice &L, double mass, float2 *dst, float2 *src, float2 *tmp);

// ---- yg_blas.cu: BLAS-1 (linalg.cpp) over [lo, lo+n) sites
double blas_sqnorm(Lattice &L, const double *a, long lo, long n);
double2 blas_product(Lattice &L, const double *a, const double *b, long lo, long n);
double blas_product_re(Lattice &L, const double *a, const double *b, long lo, long n);
// lhs = alpha*lhs + beta*rhs (complex coefficients; rhs may be null)
void blas_axpby(Lattice &L, double *lhs, double2 alpha, double2 beta, const double *rhs, long lo, long n);
void blas_g5(Lattice &L, double *f, long lo, long n);
void blas_copy(Lattice &L, double *dst, const double *src);
void blas_zero(Lattice &L, double *f, long lo, long n);
// fused CG update: x += a p ; r -= a q ; return |r|^2
double blas_cg_update(Lattice &L, double *x, double *r, const double *p, const double *q, double a, long lo, long n);
double sum_device(Lattice &L, const double *v, long n);
// sum the first `grid` double2 partials in L.red_partial (deterministic), to the host
double2 reduce_partials(Lattice &L, int grid);
constexpr int kMaxShifts = 50;          // MAX of cg.cpp:5
// cg_mshift passes over all active shifts at once: r += beta q, x_n -= bt_n k_n (returns
// |r|^2); and k_n = at_n k_n + c3_n r, p = alpha p + r (p may be null)
double blas_mshift_xr(Lattice &L, double *r, const double *q, double beta, int num, double *const *x,
                      double *const *k, const double *bt, long lo, long n);
void blas_mshift_kp(Lattice &L, double *p, const double *r, double alpha, int num, double *const *k,
                    const double *at, const double *c3, long lo, long n);
// FP32 helpers of the mixed-precision solver (counts in complex words)
void f_from_d(Lattice &L, float *dst, const double *src, long cnt);
void d_add_f(Lattice &L, double *dst, const float *src, long cnt);
double f_sqnorm(Lattice &L, const float *a, long cnt);
double f_product_re(Lattice &L, const float *a, const float *b, long cnt);
double f_cg_update(Lattice &L, float *x, float *r, const float *p, const float *q, float a, long cnt);
void f_xpay(Lattice &L, float *p, float b, const float *r, long cnt);

// ---- yg_solvers.cu
int cg(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters);
// cg on several lattices at once, one host thread and the lattice's own stream each (yg_solvers.cu)
int cg_lattices(int n, Lattice *const *L, const yg_inv_par *par, double *const *xs, double *const *bs, int *iters,
                long long wait_cycles = 0, int *persistent = nullptr);
bool batch_eligible(int n, Lattice *const *L, const yg_inv_par *par);
int cg_lattices_persistent(int n, Lattice *const *L, const yg_inv_par *par, double *const *xs, double *const *bs,
                           int *iters, long long wait_cycles);
int cg_mshift(Lattice &L, const yg_inv_par &par, int num, const double *shift, double *const *xs, double *b, int *iters);
int bicgstab(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters);
int minres(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters);
int auto_inverter(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters);
int rational_calc(Lattice &L, const yg_inv_par &par, double a0, int order, const double *poles,
                  const double *residues, double *x, double *b, int *iters);
int cg_mixed(Lattice &L, const yg_inv_par &par, double *x, double *b, yg_solve_stats *st);
int cg_mixed_sloppy(Lattice &L, const yg_inv_par &par, int prec, int reals, int lfmt, int cfmt, double delta,
                    double *x, double *b, yg_solve_stats *st, bool escalate = false);

// ---- yg_forces.cu
void clover_fermion_force(Lattice &L, double residue, double *lhs, double *rhs);
void wilson_fermion_force(Lattice &L, double dt, double mass, double residue, double *lhs, double *rhs);
void wilson_fermion_force_q(Lattice &L, double dt, double mass, double residue, double *rhs);
void wilson_fermion_force_q_multi(Lattice &L, double dt, double mass, int n, const double *residue, double *const *rhs);
void begin_fermion_force(Lattice &L);
void end_fermion_force(Lattice &L, double dt);
void clover_logdet_force(Lattice &L, double mass, double residue);
void wilson_gauge_force(Lattice &L, double dt, double beta);
double clover_logdet(Lattice &L, double mass);
double avr_plaquette(Lattice &L);

// molecular-dynamics support on the fundamental links (yg_gauge.cu)
void improved_gauge_force(Lattice &L, double dt, double beta, double c0, double c1);
double avr_wilson(Lattice &L, int height, int width);
double gauge_action(Lattice &L, double beta, double c0);
void update_links(Lattice &L, double eps);
void reunitarize(Lattice &L);
void momenta_gaussian(Lattice &L, unsigned long long seed);
double momenta_action(Lattice &L);
void gauge_backup(Lattice &L);
void gauge_restore(Lattice &L);
void apply_gauge_bcs(Lattice &L);
void gauge_upload_with_bcs(Lattice &L, const double *host);
// gauge configuration files (yg_gaugeio.cu)
void gauge_save_cfg(Lattice &L, const char *path, int num_cnfg, int num_accept);
void gauge_load_cfg(Lattice &L, const char *path, int *num_cnfg, int *num_accept, double *plaq_diff);
void gauge_save_hirep(Lattice &L, const char *path);
void gauge_load_hirep(Lattice &L, const char *path, int *num_cnfg, double *plaq_diff);

// Wilson and fermion flow (yg_gauge.cu); scratch slots of the flow
constexpr int kFlowDensities = 190, kFlowDphi = 191, kFlowPhi1 = 200, kFlowMaxFields = 32,
              kFlowPhi2 = kFlowPhi1 + kFlowMaxFields;
void wf_init(Lattice &L);
void wf_zeta(Lattice &L, double alpha);
void wf_update(Lattice &L, double val);
void wf_iterate(Lattice &L, double eps);
void wf_observables(Lattice &L, double *e_plaq, double *e_sym, double *charge);
void wf_laplacian(Lattice &L, double *dst, const double *src);
void wf_fermion_init(Lattice &L, int n);
void wf_fermion_iterate(Lattice &L, double eps, double *const *phi0, int n);

// sources, propagators and meson contractions (yg_mesons.cu)
void create_point_source(Lattice &L, int n, int tau, double *src);
void create_semwall_source(Lattice &L, int n, int tau, const double *z2, double *src);
int calc_propagator(Lattice &L, double mass, double prec, double *dst, double *src, int *iters);
int calc_propagator_multi(Lattice &L, double mass, double prec, int n, double *const *dst, double *const *src,
                          int solver, int *iters);
void meson_contract(Lattice &L, int method, int tau, const double *const *props, int nprops, double *corr);

// several cg_inverter solves sharing every operator application (yg_multi.cu)
int cg_multi(Lattice &L, const yg_inv_par &par, int nrhs, double *const *xs, double *const *bs, int *iters);
// several bicgstab_inverter solves on Dphi sharing every operator application (yg_multi.cu)
int bicgstab_multi(Lattice &L, const yg_inv_par &par, int nrhs, double *const *xs, double *const *bs, int *iters);
// the same systems with FP32 inner iterations and FP64 reliable updates (yg_multi.cu)
int cg_mixed_multi(Lattice &L, const yg_inv_par &par, int nrhs, double *const *xs, double *const *bs, double delta,
                   yg_solve_stats *stats);
// the same with the compressed FP16/FP32 inner operator applied to a tile of systems per
// thread, device-side scalars and one-iteration-late host reads (yg_mrhs.cu)
int cg_mixed_mrhs(Lattice &L, const yg_inv_par &par, int nrhs, double *const *xs, double *const *bs, double delta,
                  yg_solve_stats *stats, const double *masses = nullptr);
void pack_clover_f32(Lattice &L, double mass, void *dst, float *cn);
// the compressed inner operator's matrices (yg_sloppy.cu); formats 32 / 16 / 15, 0 = as prec
void ensure_sloppy(Lattice &L, double mass, int prec, int reals, int lfmt, int cfmt);
void inner_hop_profile(Lattice &L, double mass, int reps, double *ms, double *bytes);
int tune_inner_links(Lattice &L, double mass, double *ms);
int tuned_inner_links(Lattice &L, double mass);

// learned preconditioner: gauge-covariant parallel-transport network (yg_ptc.cu)
constexpr int kPtcMaxLayers = 8;
struct Ptc;
Ptc *ptc_create(Lattice &L, int nl, const int *ch);
void ptc_destroy(Ptc *n);
Lattice &ptc_lattice(Ptc &n);
void ptc_set_weights(Ptc &n, int l, const double *w);
void ptc_get_weights(Ptc &n, int l, double *w);
void ptc_layer(Ptc &n, int l, int adjoint, const float *in, float *out);
void ptc_apply(Ptc &n, double *dst, const double *src);
double ptc_gradient(Ptc &n, int npairs, double *const *r, double *const *e, double *grads);
void ptc_backward(Ptc &n, const double *src, const double *gout, double *grads);
int fgcr(Lattice &L, Ptc *net, const yg_inv_par &par, int restart, double *x, double *b, yg_solve_stats *st);
int solve_learned(Lattice &L, Ptc *net, const yg_inv_par &par, int restart, double *x, double *b,
                  yg_solve_stats *st);

// chronological initial guess (yg_mre.cu)
struct Mre;
Mre *mre_create(Lattice &L, int max, int op, double mass);
void mre_destroy(Mre *m);
void mre_reset(Mre &m);
void mre_store(Mre &m, const double *sol);
void mre_guess(Mre &m, double *dst, const double *src);

}  // namespace yg
