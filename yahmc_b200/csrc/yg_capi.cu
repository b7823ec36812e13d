// extern "C" entry points of include/yahmc_gpu.h: argument checks, exception-to-status
// conversion, and the thin mapping onto the engine functions.
#include <cstdio>
#include <string>
#include <vector>
#include "yg_lattice.h"

using yg::Error;
using yg::Lattice;

static thread_local std::string g_last_error;

namespace yg {
void set_last_error(const char *msg) { g_last_error = msg; }
}

template <typename F>
static int guard(F &&f) {
  try {
    f();
    return YG_OK;
  } catch (const Error &e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return YG_ERR_ARG;
  }
}

template <typename F>
static int guard_status(F &&f) {
  try {
    const int rc = f();
    // a solver status returned rather than thrown: leave a message for yg_last_error()
    if (rc == YG_MAXITER) g_last_error = "the solver reached maxiter before its stopping criterion";
    else if (rc == YG_STALL) g_last_error = "the solver stopped making progress above the requested precision";
    else if (rc == YG_NONFINITE) g_last_error = "a reduction gave a non-finite value";
    else if (rc == YG_TIMEOUT) g_last_error = "a bounded device-side wait gave up";
    return rc;
  } catch (const Error &e) {
    g_last_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return YG_ERR_ARG;
  }
}

static Lattice &lat(yg_lattice *l) {
  if (!l) throw Error(YG_ERR_ARG, "null lattice handle");
  return *reinterpret_cast<Lattice *>(l);
}

static void need(const void *p, const char *what) {
  if (!p) throw Error(YG_ERR_ARG, std::string("null pointer: ") + what);
}

static void range(Lattice &L, int view, long &lo, long &n) { L.view_range(view, lo, n); }

static void need_clover(Lattice &L) {
  if (!L.p.clover) throw Error(YG_ERR_ARG, "this operator needs the clover term (CLOVER_TERM)");
}

extern "C" {

const char *yg_last_error(void) { return g_last_error.c_str(); }

long yg_launch_count(void) { return yg::g_launch_count.load(); }

int yg_set_device(int device) {
  return guard([&] {
    int n = 0;
    YG_CUDA(cudaGetDeviceCount(&n));
    if (device < 0 || device >= n) throw yg::Error(YG_ERR_ARG, "no such CUDA device");
    YG_CUDA(cudaSetDevice(device));
  });
}

int yg_lattice_create(const yg_params *p, yg_lattice **out) {
  return guard([&] {
    need(p, "params");
    need(out, "out");
    *out = reinterpret_cast<yg_lattice *>(yg::lattice_create(*p));
  });
}

void yg_lattice_destroy(yg_lattice *l) { delete reinterpret_cast<Lattice *>(l); }

int yg_lattice_query(const yg_lattice *l, yg_info *out) {
  return guard([&] {
    need(out, "out");
    const Lattice &L = lat(const_cast<yg_lattice *>(l));
    out->volume = L.V;
    out->half_volume = L.Vh;
    out->repr_dim = L.d;
    out->nc = L.nc;
    out->ng = L.ng;
    out->field_doubles = L.field_doubles();
    out->link_doubles = 4L * L.V * 2 * L.d * L.d;
    out->fund_doubles = 4L * L.V * 2 * L.nc * L.nc;
    out->mom_doubles = 4L * L.V * L.ng;
  });
}

int yg_set_stream(yg_lattice *l, void *s) {
  return guard([&] { lat(l).stream = reinterpret_cast<cudaStream_t>(s); });
}

int yg_synchronize(yg_lattice *l) {
  return guard([&] { YG_CUDA(cudaStreamSynchronize(lat(l).stream)); });
}

int yg_field_alloc(yg_lattice *l, double **f) {
  return guard([&] {
    need(f, "out");
    Lattice &L = lat(l);
    YG_CUDA(cudaMalloc(f, L.field_bytes()));
    YG_CUDA(cudaMemsetAsync(*f, 0, L.field_bytes(), L.stream));
  });
}

int yg_field_free(yg_lattice *l, double *f) {
  return guard([&] {
    lat(l);
    if (f) YG_CUDA(cudaFree(f));
  });
}

int yg_field_upload(yg_lattice *l, double *dev, const double *host) {
  return guard([&] { need(dev, "dev"); need(host, "host"); yg::field_upload(lat(l), dev, host); });
}

int yg_field_download(yg_lattice *l, double *host, const double *dev) {
  return guard([&] { need(dev, "dev"); need(host, "host"); yg::field_download(lat(l), host, dev); });
}

int yg_gauge_upload(yg_lattice *l, const double *h) { return guard([&] { need(h, "host"); yg::gauge_upload(lat(l), h); }); }
int yg_gauge_upload_fund(yg_lattice *l, const double *h) {
  return guard([&] { need(h, "host"); yg::gauge_upload_fund(lat(l), h); });
}
int yg_host_register(void *p, size_t bytes) {
  return guard([&] {
    need(p, "host");
    if (bytes == 0) throw Error(YG_ERR_ARG, "yg_host_register: zero bytes");
    YG_CUDA(cudaHostRegister(p, bytes, cudaHostRegisterDefault));
  });
}
int yg_host_unregister(void *p) { return guard([&] { need(p, "host"); YG_CUDA(cudaHostUnregister(p)); }); }
int yg_gauge_download(yg_lattice *l, double *h) { return guard([&] { need(h, "host"); yg::gauge_download(lat(l), h); }); }
int yg_repr_links_download(yg_lattice *l, double *h) { return guard([&] { need(h, "host"); yg::repr_download(lat(l), h); }); }
int yg_clover_term_download(yg_lattice *l, double *h) { return guard([&] { need(h, "host"); yg::clover_download(lat(l), h); }); }
int yg_ldl_download(yg_lattice *l, double m, double *h) { return guard([&] { need(h, "host"); yg::ldl_download(lat(l), m, h); }); }

int yg_Dphi_oe(yg_lattice *l, double *dst, double *src) {
  return guard([&] { need(dst, "dst"); need(src, "src"); yg::hop(lat(l), dst, src, 2, 1.0, false); });
}
int yg_Dphi_eo(yg_lattice *l, double *dst, double *src) {
  return guard([&] { need(dst, "dst"); need(src, "src"); yg::hop(lat(l), dst, src, 1, 1.0, false); });
}
int yg_Dphi_ee(yg_lattice *l, double m, double *dst, double *src) {
  return guard([&] { Lattice &L = lat(l); need_clover(L); need(dst, "dst"); need(src, "src"); yg::clover_apply(L, m, dst, src, 1, false); });
}
int yg_Dphi_oo(yg_lattice *l, double m, double *dst, double *src) {
  return guard([&] { Lattice &L = lat(l); need_clover(L); need(dst, "dst"); need(src, "src"); yg::clover_apply(L, m, dst, src, 2, false); });
}
int yg_Dphi_oo_inv(yg_lattice *l, double m, double *dst, double *src) {
  return guard([&] { Lattice &L = lat(l); need_clover(L); need(dst, "dst"); need(src, "src"); yg::clover_inv_apply(L, m, dst, src, 2, false); });
}
int yg_Dphi(yg_lattice *l, double m, double *dst, double *src) {
  return guard([&] { need(dst, "dst"); need(src, "src"); yg::dphi(lat(l), m, dst, src); });
}
int yg_Hphi(yg_lattice *l, double m, double *dst, double *src) {
  return guard([&] { need(dst, "dst"); need(src, "src"); yg::hphi(lat(l), m, dst, src); });
}
int yg_Hphi_sq(yg_lattice *l, double m, double *dst, double *src) {
  return guard([&] { need(dst, "dst"); need(src, "src"); yg::hphi_sq(lat(l), m, dst, src); });
}
int yg_mvm_get(yg_lattice *l) {
  if (!l) return -1;
  Lattice &L = lat(l);
  return L.p.eo ? (L.mvm >> 1) : L.mvm;    // dirac.cpp:11-18
}
void yg_mvm_reset(yg_lattice *l) {
  if (l) lat(l).mvm = 0;
}

int yg_clover_logdet(yg_lattice *l, double m, double *out) {
  return guard([&] { need(out, "out"); *out = yg::clover_logdet(lat(l), m); });
}

// ---- linalg
int yg_spinor_zero(yg_lattice *l, double *f) {
  return guard([&] { Lattice &L = lat(l); need(f, "f"); yg::blas_zero(L, f, 0, L.V); });
}
int yg_spinor_copy(yg_lattice *l, double *dst, const double *src) {
  return guard([&] { need(dst, "dst"); need(src, "src"); yg::blas_copy(lat(l), dst, src); });
}
int yg_spinor_g5(yg_lattice *l, double *f, int view) {
  return guard([&] { Lattice &L = lat(l); need(f, "f"); long lo, n; range(L, view, lo, n); yg::blas_g5(L, f, lo, n); });
}
int yg_spinor_sqnorm(yg_lattice *l, const double *f, int view, double *out) {
  return guard([&] { Lattice &L = lat(l); need(f, "f"); need(out, "out"); long lo, n; range(L, view, lo, n); *out = yg::blas_sqnorm(L, f, lo, n); });
}
int yg_spinor_product(yg_lattice *l, const double *a, const double *b, int view, double *out) {
  return guard([&] {
    Lattice &L = lat(l); need(a, "a"); need(b, "b"); need(out, "out");
    long lo, n; range(L, view, lo, n);
    double2 v = yg::blas_product(L, a, b, lo, n);
    out[0] = v.x; out[1] = v.y;
  });
}
int yg_spinor_product_re(yg_lattice *l, const double *a, const double *b, int view, double *out) {
  return guard([&] { Lattice &L = lat(l); need(a, "a"); need(b, "b"); need(out, "out"); long lo, n; range(L, view, lo, n); *out = yg::blas_product_re(L, a, b, lo, n); });
}

static int axpby(yg_lattice *l, double *lhs, double2 al, double2 be, const double *rhs, int view, bool need_rhs) {
  return guard([&] {
    Lattice &L = lat(l); need(lhs, "lhs");
    if (need_rhs) need(rhs, "rhs");
    long lo, n; range(L, view, lo, n);
    yg::blas_axpby(L, lhs, al, be, rhs, lo, n);
  });
}
int yg_spinor_add_assign(yg_lattice *l, double *a, const double *b, int v) { return axpby(l, a, make_double2(1, 0), make_double2(1, 0), b, v, true); }
int yg_spinor_sub_assign(yg_lattice *l, double *a, const double *b, int v) { return axpby(l, a, make_double2(1, 0), make_double2(-1, 0), b, v, true); }
int yg_spinor_mulr(yg_lattice *l, double *a, double s, const double *b, int v) { return axpby(l, a, make_double2(0, 0), make_double2(s, 0), b, v, true); }
int yg_spinor_mulc(yg_lattice *l, double *a, double re, double im, const double *b, int v) { return axpby(l, a, make_double2(0, 0), make_double2(re, im), b, v, true); }
int yg_spinor_mulr_assign(yg_lattice *l, double *a, double s, int v) { return axpby(l, a, make_double2(s, 0), make_double2(0, 0), nullptr, v, false); }
int yg_spinor_mulc_assign(yg_lattice *l, double *a, double re, double im, int v) { return axpby(l, a, make_double2(re, im), make_double2(0, 0), nullptr, v, false); }
int yg_spinor_mulr_add_assign(yg_lattice *l, double *a, double s, const double *b, int v) { return axpby(l, a, make_double2(1, 0), make_double2(s, 0), b, v, true); }
int yg_spinor_mulc_add_assign(yg_lattice *l, double *a, double re, double im, const double *b, int v) { return axpby(l, a, make_double2(1, 0), make_double2(re, im), b, v, true); }
int yg_spinor_mulr_sub_assign(yg_lattice *l, double *a, double s, const double *b, int v) { return axpby(l, a, make_double2(1, 0), make_double2(-s, 0), b, v, true); }
int yg_spinor_mulc_sub_assign(yg_lattice *l, double *a, double re, double im, const double *b, int v) { return axpby(l, a, make_double2(1, 0), make_double2(-re, -im), b, v, true); }

// ---- inverters
static void check_par(const yg_inv_par *p) {
  need(p, "par");
  if (p->op < 0 || p->op > 2) throw Error(YG_ERR_ARG, "invalid operator id");
}

int yg_cg_inverter(yg_lattice *l, const yg_inv_par *p, double *x, double *b, int *it) {
  return guard_status([&] { check_par(p); need(x, "x"); need(b, "b"); need(it, "iters"); return yg::cg(lat(l), *p, x, b, it); });
}
int yg_bicgstab_inverter(yg_lattice *l, const yg_inv_par *p, double *x, double *b, int *it) {
  return guard_status([&] { check_par(p); need(x, "x"); need(b, "b"); need(it, "iters"); return yg::bicgstab(lat(l), *p, x, b, it); });
}
int yg_minres_inverter(yg_lattice *l, const yg_inv_par *p, double *x, double *b, int *it) {
  return guard_status([&] { check_par(p); need(x, "x"); need(b, "b"); need(it, "iters"); return yg::minres(lat(l), *p, x, b, it); });
}
int yg_auto_inverter(yg_lattice *l, const yg_inv_par *p, double *x, double *b, int *it) {
  return guard_status([&] { check_par(p); need(x, "x"); need(b, "b"); need(it, "iters"); return yg::auto_inverter(lat(l), *p, x, b, it); });
}
int yg_cg_mshift(yg_lattice *l, const yg_inv_par *p, int num, const double *shifts, double *const *xs, double *b, int *it) {
  return guard_status([&] {
    check_par(p); need(shifts, "shifts"); need(xs, "xs"); need(b, "b"); need(it, "iters");
    for (int i = 0; i < num; i++) need(xs[i], "xs[i]");
    return yg::cg_mshift(lat(l), *p, num, shifts, xs, b, it);
  });
}
int yg_rational_calc(yg_lattice *l, const yg_inv_par *p, double a0, int order, const double *poles,
                     const double *residues, double *x, double *b, int *it) {
  return guard_status([&] {
    check_par(p); need(poles, "poles"); need(residues, "residues"); need(x, "x"); need(b, "b"); need(it, "iters");
    return yg::rational_calc(lat(l), *p, a0, order, poles, residues, x, b, it);
  });
}
int yg_cg_mixed_opts(yg_lattice *l, const yg_inv_par *p, const yg_mixed_opts *o, double *x, double *b,
                     yg_solve_stats *st) {
  return guard_status([&] {
    check_par(p); need(o, "opts"); need(x, "x"); need(b, "b");
    if (o->inner_precision == 0) return yg::cg_mixed(lat(l), *p, x, b, st);
    return yg::cg_mixed_sloppy(lat(l), *p, o->inner_precision, o->link_reals, o->link_storage, o->clover_storage,
                               o->delta, x, b, st, o->escalate != 0);
  });
}
int yg_cg_inverter_multi(yg_lattice *l, const yg_inv_par *p, int nrhs, double *const *xs, double *const *bs,
                         int *iters) {
  return guard_status([&] {
    check_par(p); need(xs, "xs"); need(bs, "bs"); need(iters, "iters");
    for (int i = 0; i < nrhs; i++) { need(xs[i], "xs[i]"); need(bs[i], "bs[i]"); }
    return yg::cg_multi(lat(l), *p, nrhs, xs, bs, iters);
  });
}
int yg_cg_inverter_lattices(int n, yg_lattice *const *lats, const yg_inv_par *pars, double *const *xs,
                            double *const *bs, int *iters) {
  return guard_status([&] {
    need(lats, "lats"); need(pars, "pars"); need(xs, "xs"); need(bs, "bs"); need(iters, "iters");
    if (n < 1 || n > 64) throw yg::Error(YG_ERR_ARG, "1..64 lattices");
    std::vector<yg::Lattice *> L(n);
    for (int i = 0; i < n; i++) {
      check_par(&pars[i]); need(xs[i], "xs[i]"); need(bs[i], "bs[i]");
      L[i] = &lat(lats[i]);
    }
    return yg::cg_lattices(n, L.data(), pars, xs, bs, iters);
  });
}
int yg_cg_inverter_lattices_ex(int n, yg_lattice *const *lats, const yg_inv_par *pars, double *const *xs,
                               double *const *bs, int *iters, long long wait_cycles, int *persistent) {
  return guard_status([&] {
    need(lats, "lats"); need(pars, "pars"); need(xs, "xs"); need(bs, "bs"); need(iters, "iters");
    if (n < 1 || n > 64) throw yg::Error(YG_ERR_ARG, "1..64 lattices");
    std::vector<yg::Lattice *> L(n);
    for (int i = 0; i < n; i++) {
      check_par(&pars[i]); need(xs[i], "xs[i]"); need(bs[i], "bs[i]");
      L[i] = &lat(lats[i]);
    }
    return yg::cg_lattices(n, L.data(), pars, xs, bs, iters, wait_cycles, persistent);
  });
}
int yg_bicgstab_inverter_multi(yg_lattice *l, const yg_inv_par *p, int nrhs, double *const *xs, double *const *bs,
                               int *iters) {
  return guard_status([&] {
    check_par(p); need(xs, "xs"); need(bs, "bs"); need(iters, "iters");
    for (int i = 0; i < nrhs; i++) { need(xs[i], "xs[i]"); need(bs[i], "bs[i]"); }
    return yg::bicgstab_multi(lat(l), *p, nrhs, xs, bs, iters);
  });
}
int yg_cg_mixed_multi(yg_lattice *l, const yg_inv_par *p, int nrhs, double *const *xs, double *const *bs,
                      double delta, yg_solve_stats *stats) {
  return guard_status([&] {
    check_par(p); need(xs, "xs"); need(bs, "bs"); need(stats, "stats");
    for (int i = 0; i < nrhs; i++) { need(xs[i], "xs[i]"); need(bs[i], "bs[i]"); }
    return yg::cg_mixed_mrhs(lat(l), *p, nrhs, xs, bs, delta, stats);
  });
}
int yg_cg_mixed_multi_masses(yg_lattice *l, const yg_inv_par *p, int nrhs, const double *masses,
                             double *const *xs, double *const *bs, double delta, yg_solve_stats *stats) {
  return guard_status([&] {
    check_par(p); need(masses, "masses"); need(xs, "xs"); need(bs, "bs"); need(stats, "stats");
    for (int i = 0; i < nrhs; i++) { need(xs[i], "xs[i]"); need(bs[i], "bs[i]"); }
    return yg::cg_mixed_mrhs(lat(l), *p, nrhs, xs, bs, delta, stats, masses);
  });
}
int yg_inner_hop_profile(yg_lattice *l, double mass, int reps, double *ms, double *bytes) {
  return guard([&] { need(ms, "ms"); need(bytes, "bytes"); yg::inner_hop_profile(lat(l), mass, reps, ms, bytes); });
}
int yg_cg_mixed(yg_lattice *l, const yg_inv_par *p, double *x, double *b, yg_solve_stats *st) {
  return guard_status([&] {
    check_par(p); need(x, "x"); need(b, "b");
    yg::Lattice &L = lat(l);
    // the compressed inner operator where it exists (d = 3, even-odd): FP16 spinors with
    // per-site norms, FP32 links and clover blocks, delta 0.1 -- 16-bit spinors only add
    // noise to each inner step, while 16-bit matrices would change the operator itself; the
    // link format (18, 12 or 8 reals) is the fastest one measured on this lattice at the
    // first call; else the generic FP32 operator
    if (L.d == 3 && L.p.eo) {
      const int reals = yg::tuned_inner_links(L, p->mass);
      return yg::cg_mixed_sloppy(L, *p, 16, reals, 32, 32, 0.1, x, b, st, /*escalate=*/true);
    }
    return yg::cg_mixed(L, *p, x, b, st);
  });
}

int yg_tune_inner_links(yg_lattice *l, double mass, int *link_reals, double *ms_per_hop) {
  return guard([&] {
    yg::Lattice &L = lat(l);
    if (L.d != 3 || !L.p.eo) throw yg::Error(YG_ERR_ARG, "the compressed inner operator needs d = 3 and even-odd");
    const int r = yg::tune_inner_links(L, mass, ms_per_hop);
    if (link_reals) *link_reals = r;
  });
}

// ---- propagators and mesons
int yg_create_point_source(yg_lattice *l, int n, int tau, double *src) {
  return guard([&] { need(src, "src"); yg::create_point_source(lat(l), n, tau, src); });
}
int yg_create_semwall_source(yg_lattice *l, int n, int tau, const double *z2, double *src) {
  return guard([&] { need(src, "src"); yg::create_semwall_source(lat(l), n, tau, z2, src); });
}
int yg_calc_propagator(yg_lattice *l, double mass, double prec, double *dst, double *src, int *iters) {
  return guard_status([&] {
    need(dst, "dst"); need(src, "src");
    int it = 0;
    const int st = yg::calc_propagator(lat(l), mass, prec, dst, src, &it);
    if (iters) *iters = it;
    return st;
  });
}
int yg_calc_propagator_multi(yg_lattice *l, double mass, double prec, int n, double *const *dst, double *const *src,
                             int solver, int *iters) {
  return guard_status([&] {
    need(dst, "dst"); need(src, "src");
    std::vector<int> it(n > 0 ? n : 1, 0);
    const int st = yg::calc_propagator_multi(lat(l), mass, prec, n, dst, src, solver, it.data());
    if (iters)
      for (int i = 0; i < n; i++) iters[i] = it[i];
    return st;
  });
}
int yg_meson_contract(yg_lattice *l, int method, int tau, const double *const *props, int nprops, double *corr) {
  return guard([&] { need(props, "props"); need(corr, "corr"); yg::meson_contract(lat(l), method, tau, props, nprops, corr); });
}

// ---- Wilson and fermion flow
int yg_wf_init(yg_lattice *l) { return guard([&] { yg::wf_init(lat(l)); }); }
int yg_wf_zeta(yg_lattice *l, double alpha) { return guard([&] { yg::wf_zeta(lat(l), alpha); }); }
int yg_wf_update(yg_lattice *l, double val) { return guard([&] { yg::wf_update(lat(l), val); }); }
int yg_wf_iterate(yg_lattice *l, double eps) { return guard([&] { yg::wf_iterate(lat(l), eps); }); }
int yg_wf_observables(yg_lattice *l, double *e_plaq, double *e_sym, double *charge) {
  return guard([&] { yg::wf_observables(lat(l), e_plaq, e_sym, charge); });
}
int yg_wf_fermion_init(yg_lattice *l, int n) { return guard([&] { yg::wf_fermion_init(lat(l), n); }); }
int yg_wf_fermion_iterate(yg_lattice *l, double eps, double *const *phi, int n) {
  return guard([&] {
    need(phi, "phi");
    for (int i = 0; i < n; i++) need(phi[i], "phi[i]");
    yg::wf_fermion_iterate(lat(l), eps, phi, n);
  });
}

// ---- gauge configuration files
int yg_gauge_save_cfg(yg_lattice *l, const char *path, int num_cnfg, int num_accept) {
  return guard([&] { need(path, "path"); yg::gauge_save_cfg(lat(l), path, num_cnfg, num_accept); });
}
int yg_gauge_load_cfg(yg_lattice *l, const char *path, int *num_cnfg, int *num_accept, double *plaq_diff) {
  return guard([&] { need(path, "path"); yg::gauge_load_cfg(lat(l), path, num_cnfg, num_accept, plaq_diff); });
}
int yg_gauge_save_hirep(yg_lattice *l, const char *path) {
  return guard([&] { need(path, "path"); yg::gauge_save_hirep(lat(l), path); });
}
int yg_gauge_load_hirep(yg_lattice *l, const char *path, int *num_cnfg, double *plaq_diff) {
  return guard([&] { need(path, "path"); yg::gauge_load_hirep(lat(l), path, num_cnfg, plaq_diff); });
}

// ---- chronological initial guess
struct yg_mre {
  yg::Mre *m;
};
// ---- learned preconditioner (yg_ptc.cu)
struct yg_ptc {
  yg::Ptc *n;
};
static yg::Ptc &ptc(yg_ptc *h) {
  if (!h || !h->n) throw Error(YG_ERR_ARG, "null network handle");
  return *h->n;
}
int yg_ptc_create(yg_lattice *l, int nlayers, const int *channels, yg_ptc **out) {
  return guard([&] {
    need(out, "out");
    need(channels, "channels");
    *out = nullptr;
    *out = new yg_ptc{yg::ptc_create(lat(l), nlayers, channels)};
  });
}
int yg_ptc_destroy(yg_ptc *h) {
  return guard([&] {
    if (!h) return;
    yg::ptc_destroy(h->n);
    delete h;
  });
}
int yg_ptc_set_weights(yg_ptc *h, int layer, const double *w) {
  return guard([&] { need(w, "w"); yg::ptc_set_weights(ptc(h), layer, w); });
}
int yg_ptc_get_weights(yg_ptc *h, int layer, double *w) {
  return guard([&] { need(w, "w"); yg::ptc_get_weights(ptc(h), layer, w); });
}
int yg_ptc_layer(yg_ptc *h, int layer, int adjoint, const float *in, float *out) {
  return guard([&] {
    need(in, "in");
    need(out, "out");
    yg::Ptc &n = ptc(h);
    yg::ptc_layer(n, layer, adjoint, in, out);
    YG_CUDA(cudaStreamSynchronize(yg::ptc_lattice(n).stream));
  });
}
int yg_ptc_apply(yg_ptc *h, double *dst, const double *src) {
  return guard([&] { need(dst, "dst"); need(src, "src"); yg::ptc_apply(ptc(h), dst, src); });
}
int yg_ptc_gradient(yg_ptc *h, int npairs, double *const *r, double *const *e, double *loss, double *grads) {
  return guard([&] {
    need(r, "r"); need(e, "e"); need(loss, "loss"); need(grads, "grads");
    for (int k = 0; k < npairs; k++) { need(r[k], "r[k]"); need(e[k], "e[k]"); }
    *loss = yg::ptc_gradient(ptc(h), npairs, r, e, grads);
  });
}
int yg_ptc_backward(yg_ptc *h, const double *src, const double *gout, double *grads) {
  return guard([&] { need(src, "src"); need(gout, "gout"); need(grads, "grads"); yg::ptc_backward(ptc(h), src, gout, grads); });
}
int yg_fgcr(yg_lattice *l, yg_ptc *h, const yg_inv_par *p, int restart, double *x, double *b, yg_solve_stats *st) {
  return guard_status([&] {
    check_par(p); need(x, "x"); need(b, "b"); need(st, "stats");
    return yg::fgcr(lat(l), h ? &ptc(h) : nullptr, *p, restart, x, b, st);
  });
}
int yg_solve_learned(yg_lattice *l, yg_ptc *h, const yg_inv_par *p, int restart, double *x, double *b,
                     yg_solve_stats *st) {
  return guard_status([&] {
    check_par(p); need(x, "x"); need(b, "b"); need(st, "stats");
    return yg::solve_learned(lat(l), h ? &ptc(h) : nullptr, *p, restart, x, b, st);
  });
}

int yg_mre_init(yg_lattice *l, int max, int op, double mass, yg_mre **out) {
  return guard([&] {
    need(out, "out");
    *out = nullptr;
    yg_mre *h = new yg_mre{yg::mre_create(lat(l), max, op, mass)};
    *out = h;
  });
}
int yg_mre_store(yg_mre *h, const double *sol) {
  return guard([&] { need(h, "mre"); need(sol, "solution"); yg::mre_store(*h->m, sol); });
}
int yg_mre_guess(yg_mre *h, double *dst, const double *src) {
  return guard([&] { need(h, "mre"); need(dst, "dst"); need(src, "src"); yg::mre_guess(*h->m, dst, src); });
}
int yg_mre_reset(yg_mre *h) { return guard([&] { need(h, "mre"); yg::mre_reset(*h->m); }); }
int yg_mre_free(yg_mre *h) {
  return guard([&] {
    if (!h) return;
    yg::mre_destroy(h->m);
    delete h;
  });
}

// ---- forces
int yg_momenta_upload(yg_lattice *l, const double *h) { return guard([&] { need(h, "host"); yg::momenta_upload(lat(l), h); }); }
int yg_momenta_download(yg_lattice *l, double *h) { return guard([&] { need(h, "host"); yg::momenta_download(lat(l), h); }); }
int yg_momenta_zero(yg_lattice *l) {
  return guard([&] { Lattice &L = lat(l); YG_CUDA(cudaMemsetAsync(L.mom.p, 0, L.mom.bytes, L.stream)); });
}
int yg_clover_force_download(yg_lattice *l, double *h) { return guard([&] { need(h, "host"); yg::clover_force_download(lat(l), h); }); }
int yg_begin_fermion_force(yg_lattice *l) { return guard([&] { yg::begin_fermion_force(lat(l)); }); }
int yg_end_fermion_force(yg_lattice *l, double dt) { return guard([&] { yg::end_fermion_force(lat(l), dt); }); }
int yg_wilson_fermion_force(yg_lattice *l, double dt, double m, double res, double *lhs, double *rhs) {
  return guard([&] { need(lhs, "lhs"); need(rhs, "rhs"); yg::wilson_fermion_force(lat(l), dt, m, res, lhs, rhs); });
}
int yg_wilson_fermion_force_q(yg_lattice *l, double dt, double m, double res, double *rhs) {
  return guard([&] { need(rhs, "rhs"); yg::wilson_fermion_force_q(lat(l), dt, m, res, rhs); });
}
int yg_wilson_fermion_force_q_multi(yg_lattice *l, double dt, double mass, int n, const double *residues,
                                    double *const *rhs) {
  return guard([&] {
    need(residues, "residues");
    need(rhs, "rhs");
    for (int k = 0; k < n; k++) need(rhs[k], "rhs[k]");
    yg::wilson_fermion_force_q_multi(lat(l), dt, mass, n, residues, rhs);
  });
}
int yg_clover_fermion_force(yg_lattice *l, double res, double *lhs, double *rhs) {
  return guard([&] { need(lhs, "lhs"); need(rhs, "rhs"); yg::clover_fermion_force(lat(l), res, lhs, rhs); });
}
int yg_clover_logdet_force(yg_lattice *l, double m, double res) { return guard([&] { yg::clover_logdet_force(lat(l), m, res); }); }
int yg_wilson_gauge_force(yg_lattice *l, double dt, double beta) { return guard([&] { yg::wilson_gauge_force(lat(l), dt, beta); }); }
int yg_avr_plaquette(yg_lattice *l, double *out) { return guard([&] { need(out, "out"); *out = yg::avr_plaquette(lat(l)); }); }

// ---- molecular dynamics
int yg_improved_gauge_force(yg_lattice *l, double dt, double beta, double c0, double c1) {
  return guard([&] { yg::improved_gauge_force(lat(l), dt, beta, c0, c1); });
}
int yg_avr_wilson(yg_lattice *l, int h, int w, double *out) {
  return guard([&] { need(out, "out"); *out = yg::avr_wilson(lat(l), h, w); });
}
int yg_gauge_action(yg_lattice *l, double beta, double c0, double *out) {
  return guard([&] { need(out, "out"); *out = yg::gauge_action(lat(l), beta, c0); });
}
int yg_update_links(yg_lattice *l, double eps) { return guard([&] { yg::update_links(lat(l), eps); }); }
int yg_represent_gauge_field(yg_lattice *l) {
  return guard([&] { yg::Lattice &L = lat(l); yg::represent_and_clover(L); YG_CUDA(cudaStreamSynchronize(L.stream)); });
}
int yg_reunitarize(yg_lattice *l) { return guard([&] { yg::reunitarize(lat(l)); }); }
int yg_momenta_gaussian(yg_lattice *l, unsigned long long seed) { return guard([&] { yg::momenta_gaussian(lat(l), seed); }); }
int yg_momenta_action(yg_lattice *l, double *out) {
  return guard([&] { need(out, "out"); *out = yg::momenta_action(lat(l)); });
}
int yg_gauge_backup(yg_lattice *l) { return guard([&] { yg::gauge_backup(lat(l)); }); }
int yg_gauge_restore(yg_lattice *l) { return guard([&] { yg::gauge_restore(lat(l)); }); }

}  // extern "C"
