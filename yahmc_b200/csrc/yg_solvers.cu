// Inverters (cg.cpp, bicgstab.cpp, minres.cpp, inverter.cpp, rational.cpp) driven from
// the host over device fields, plus the mixed-precision CG with FP64 reliable updates.
//
// The FP64 solvers follow the reference's recurrences step for step, so iteration counts
// and solutions match the reference to rounding; the device work per step is the fused
// operator (yg_dirac.cu) and streaming BLAS passes (yg_blas.cu).  Scalars come back to
// the host once per reduction, as the reference's control flow needs them.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <exception>
#include <thread>
#include <vector>
#include "yg_lattice.h"

namespace yg {

namespace {

// complex arithmetic of include/complex.h (operator/= at :120-130)
struct cx {
  double re, im;
};
inline cx cdiv(cx a, cx b) {
  double sq = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / sq, (a.im * b.re - a.re * b.im) / sq};
}
inline cx cmulx(cx a, cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }

struct Ctx {
  Lattice &L;
  long lo, n;
  explicit Ctx(Lattice &l) : L(l) { L.view_range(YG_VIEW_DEFAULT, lo, n); }
  double sqnorm(const double *a) { return blas_sqnorm(L, a, lo, n); }
  double prod_re(const double *a, const double *b) { return blas_product_re(L, a, b, lo, n); }
  cx prod(const double *a, const double *b) {
    double2 v = blas_product(L, a, b, lo, n);
    return {v.x, v.y};
  }
  // lhs = alpha*lhs + beta*rhs
  void axpby(double *lhs, cx alpha, cx beta, const double *rhs) {
    blas_axpby(L, lhs, make_double2(alpha.re, alpha.im), make_double2(beta.re, beta.im), rhs, lo, n);
  }
  void copy(double *dst, const double *src) { blas_copy(L, dst, src); }
};

void log_line(const yg_inv_par &par, const char *name, int it, double prec) {
  if (par.log) fprintf(stderr, "[INVERTER][30]%s: iterations = %d, precision = %1.4e\n", name, it, prec);
}

void check_finite(double v, const char *what) {
  if (!std::isfinite(v)) throw Error(YG_NONFINITE, std::string("non-finite value in ") + what);
}

}  // namespace

// cg_inverter, cg.cpp:132-202
int cg(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters) {
  Ctx c(L);
  double *r = L.scratch_field(3), *p = L.scratch_field(4), *q = L.scratch_field(5);
  c.copy(p, x);
  apply_op(L, par.op, par.mass, q, p);
  c.copy(r, b);
  c.axpby(r, {1, 0}, {-1, 0}, q);
  c.copy(p, r);
  double norm = c.sqnorm(b);
  double rr = c.sqnorm(r);
  int it = (rr < norm * par.prec) ? -1 : 0;
  int status = YG_OK;
  while (++it) {
    if (par.maxiter > 0 && it > par.maxiter) { it--; status = YG_MAXITER; break; }
    apply_op(L, par.op, par.mass, q, p);
    double atmp = rr;                       // = spinor_sqnorm(r) of cg.cpp:176, unchanged since
    double pq = c.prod_re(p, q);
    check_finite(pq, "cg");
    double alpha = atmp / pq;
    rr = blas_cg_update(L, x, r, p, q, alpha, c.lo, c.n);
    double beta = rr / atmp;
    if (rr < norm * par.prec) break;
    c.axpby(p, {beta, 0}, {1, 0}, r);
  }
  log_line(par, "cg", it, rr / norm);
  *iters = it;
  return status;
}

// No reference counterpart: independent cg_inverter solves on lattices of any sizes at once.
// A small lattice's CG is bound by kernel and reduction latency and leaves most of the GPU
// idle.  Hphi_sq solves on even-odd lattices of one representation dimension d (2, 3, 4, 6;
// all with or all without a clover term; no open/SF boundaries) run as one persistent kernel
// (yg_batch.cu); any other mix runs each lattice's single-lattice cg in its own host thread
// on the lattice's own stream, so the solves overlap on the device.  Iteration counts are
// those of one-at-a-time calls (the persistent kernel's reductions add in another order, so
// a count can differ by one where |r|^2 lands within rounding of the stopping threshold).
// Returns the worst status; *persistent (when given) tells which path ran.
int cg_lattices(int n, Lattice *const *L, const yg_inv_par *par, double *const *xs, double *const *bs, int *iters,
                long long wait_cycles, int *persistent) {
  if (n < 1 || n > 64) throw Error(YG_ERR_ARG, "1..64 lattices");
  for (int i = 0; i < n; i++)
    for (int j = 0; j < i; j++)
      if (L[i] == L[j]) throw Error(YG_ERR_ARG, "each lattice may appear once (its scratch fields are per solve)");
  int cur = 0;
  YG_CUDA(cudaGetDevice(&cur));
  for (int i = 0; i < n; i++)
    if (L[i]->device != cur)
      throw Error(YG_ERR_ARG, "every lattice must belong to the calling thread's current device");
  const bool batch = batch_eligible(n, L, par);
  if (persistent) *persistent = batch ? 1 : 0;
  if (batch) return cg_lattices_persistent(n, L, par, xs, bs, iters, wait_cycles);
  // the scratch fields the solves use, allocated here: a cudaMalloc inside the threads would
  // synchronise the device while the other lattices' solves run
  for (int i = 0; i < n; i++)
    for (int k = 1; k <= 5; k++) L[i]->scratch_field(k);
  int dev = 0;
  YG_CUDA(cudaGetDevice(&dev));
  std::vector<int> st(n, YG_OK);
  std::vector<std::exception_ptr> err(n);
  std::vector<std::thread> th;
  th.reserve(n);
  for (int i = 0; i < n; i++)
    th.emplace_back([&, i] {
      try {
        YG_CUDA(cudaSetDevice(dev));
        st[i] = cg(*L[i], par[i], xs[i], bs[i], &iters[i]);
      } catch (...) {
        err[i] = std::current_exception();
      }
    });
  for (auto &t : th) t.join();
  for (int i = 0; i < n; i++)
    if (err[i]) std::rethrow_exception(err[i]);
  int worst = YG_OK;
  for (int s : st)
    if (s != YG_OK) worst = s;
  return worst;
}

// cg_mshift, cg.cpp:11-130
int cg_mshift(Lattice &L, const yg_inv_par &par, int num, const double *shift, double *const *xs, double *b,
              int *iters) {
  if (num < 1 || num > 50) throw Error(YG_ERR_ARG, "cg_mshift supports 1..50 shifts (cg.cpp:5)");
  Ctx c(L);
  double *r = L.scratch_field(3), *p = L.scratch_field(4), *q = L.scratch_field(5);
  std::vector<double *> k(num);
  for (int n = 0; n < num; n++) k[n] = L.scratch_field(10 + n);
  c.copy(r, b);
  c.copy(p, b);
  for (int n = 0; n < num; n++) {
    blas_zero(L, xs[n], 0, L.V);
    c.copy(k[n], b);
  }
  std::vector<double> c1(num, 1.0), c2(num, 1.0), c3(num, 0.0);
  std::vector<int> flag(num, 0);
  double beta = 1, alpha = 0, btmp = 0;
  double norm = c.sqnorm(b);
  double atmp = c.sqnorm(r);
  int it = 0;
  int status = YG_OK;
  // the per-shift x and k updates of one iteration run as one pass each over all active
  // shifts (blas_mshift_xr / _kp); scalars follow cg.cpp:62-116 in the same order
  std::vector<double *> ax(num), ak(num);
  std::vector<double> abt(num), aat(num), ac3(num);
  while (++it) {
    apply_op(L, par.op, par.mass, q, p);
    double pq = c.prod_re(p, q);
    check_finite(pq, "cg_mshift");
    double beta_old = beta;
    beta = -(atmp / pq);
    int na = 0;
    for (int n = 0; n < num; n++) {
      if (flag[n]) continue;
      c3[n] = c2[n] * c1[n] * beta_old;
      c3[n] /= (beta * alpha * (c1[n] - c2[n])) + (c1[n] * beta_old * (1 - shift[n] * beta));
      ax[na] = xs[n];
      ak[na] = k[n];
      abt[na] = beta * (c3[n] / c2[n]);
      na++;
    }
    btmp = blas_mshift_xr(L, r, q, beta, na, ax.data(), ak.data(), abt.data(), c.lo, c.n);
    alpha = btmp / atmp;
    int notconverged = 0;
    na = 0;
    for (int n = 0; n < num; n++) {
      if (flag[n]) continue;
      aat[na] = alpha * (c3[n] * c3[n]) / (c2[n] * c2[n]);
      ac3[na] = c3[n];
      ak[na] = k[n];
      na++;
      if (btmp * c3[n] * c3[n] < norm * par.prec) flag[n] = 1;
      else notconverged++;
      c1[n] = c2[n];
      c2[n] = c3[n];
    }
    // k_n = at k_n + c3 r for the shifts active in this iteration; p = alpha p + r is only
    // needed when the loop goes on
    bool more = notconverged > 0 && !(par.maxiter > 0 && it >= par.maxiter);
    blas_mshift_kp(L, more ? p : nullptr, r, alpha, na, ak.data(), aat.data(), ac3.data(), c.lo, c.n);
    if (notconverged == 0) break;
    if (par.maxiter > 0 && it >= par.maxiter) { status = YG_MAXITER; break; }
    atmp = btmp;
  }
  log_line(par, "cg_mshift", it, btmp / norm);
  *iters = it;
  return status;
}

// bicgstab_inverter, bicgstab.cpp:9-97
int bicgstab(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters) {
  Ctx c(L);
  double *r = L.scratch_field(3), *r0 = L.scratch_field(4), *v = L.scratch_field(5);
  double *p = L.scratch_field(6), *t = L.scratch_field(7);
  apply_op(L, par.op, par.mass, p, x);
  c.copy(r, b);
  c.axpby(r, {1, 0}, {-1, 0}, p);
  c.copy(r0, r);
  c.copy(p, r);
  double norm = c.sqnorm(b);
  cx rho0 = c.prod(r, r0);
  double residue = rho0.re;
  int it = (residue < norm * par.prec) ? -1 : 0;
  int status = YG_OK;
  while (++it) {
    if (par.maxiter > 0 && it > par.maxiter) { it--; status = YG_MAXITER; break; }
    apply_op(L, par.op, par.mass, v, p);
    cx alpha = cdiv(rho0, c.prod(v, r0));
    check_finite(alpha.re, "bicgstab");
    c.axpby(r, {1, 0}, {-alpha.re, -alpha.im}, v);
    apply_op(L, par.op, par.mass, t, r);
    cx omega = c.prod(r, t);
    double tt = c.sqnorm(t);
    omega = {omega.re / tt, omega.im / tt};
    c.axpby(x, {1, 0}, alpha, p);
    c.axpby(x, {1, 0}, omega, r);
    c.axpby(r, {1, 0}, {-omega.re, -omega.im}, t);
    cx rho1 = c.prod(r, r0);
    cx beta = cmulx(cdiv(rho1, rho0), cdiv(alpha, omega));
    c.axpby(p, beta, {1, 0}, r);
    cx bo = cmulx(beta, omega);
    c.axpby(p, {1, 0}, {-bo.re, -bo.im}, v);
    residue = c.sqnorm(r);
    check_finite(residue, "bicgstab");
    if (residue < norm * par.prec) break;
    rho0 = rho1;
  }
  it *= 2;
  log_line(par, "bicgstab", it, residue / norm);
  *iters = it;
  return status;
}

// minres_inverter, minres.cpp:12-117
int minres(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters) {
  Ctx c(L);
  double *v0 = L.scratch_field(3), *v1 = L.scratch_field(4), *w0 = L.scratch_field(5);
  double *w1 = L.scratch_field(6), *tmp = L.scratch_field(7);
  apply_op(L, par.op, par.mass, tmp, x);
  c.copy(v1, b);
  c.axpby(v1, {1, 0}, {-1, 0}, tmp);
  blas_zero(L, v0, 0, L.V);
  blas_zero(L, w0, 0, L.V);
  blas_zero(L, w1, 0, L.V);
  double g0 = 1, g1 = 1, s0 = 0, s1 = 0;
  double norm = c.sqnorm(b);
  double residue = c.sqnorm(v1);
  double beta0 = std::sqrt(residue), eta = beta0;
  int it = (residue < norm * par.prec) ? -1 : 0;
  int status = YG_OK;
  while (++it) {
    if (par.maxiter > 0 && it > par.maxiter) { it--; status = YG_MAXITER; break; }
    c.axpby(v1, {1.0 / beta0, 0}, {0, 0}, nullptr);
    apply_op(L, par.op, par.mass, tmp, v1);
    double alpha = c.prod_re(v1, tmp);
    check_finite(alpha, "minres");
    c.axpby(tmp, {1, 0}, {-alpha, 0}, v1);
    c.axpby(tmp, {1, 0}, {-beta0, 0}, v0);
    double *ptr = v0; v0 = v1; v1 = tmp; tmp = ptr;
    double beta1 = std::sqrt(c.sqnorm(v1));
    double delta = g1 * alpha - g0 * s1 * beta0;
    double rho1 = std::sqrt(delta * delta + beta1 * beta1);
    double rho2 = s1 * alpha + g0 * g1 * beta0;
    double rho3 = s0 * beta0;
    g0 = g1;
    g1 = delta / rho1;
    s0 = s1;
    s1 = beta1 / rho1;
    c.axpby(tmp, {0, 0}, {1.0 / rho1, 0}, v0);
    c.axpby(tmp, {1, 0}, {-(rho3 / rho1), 0}, w0);
    c.axpby(tmp, {1, 0}, {-(rho2 / rho1), 0}, w1);
    ptr = w0; w0 = w1; w1 = tmp; tmp = ptr;
    c.axpby(x, {1, 0}, {g1 * eta, 0}, w1);
    eta = -s1 * eta;
    beta0 = beta1;
    residue = eta * eta;
    if (residue < norm * par.prec) break;
  }
  log_line(par, "minres", it, residue / norm);
  *iters = it;
  return status;
}

// auto_inverter, inverter.cpp:9-55: BiCGstab on Dphi, gamma5 sandwiches for Hphi / Hphi_sq
int auto_inverter(Lattice &L, const yg_inv_par &par0, double *x, double *b, int *iters) {
  long lo, n;
  L.view_range(YG_VIEW_DEFAULT, lo, n);
  yg_inv_par par = par0;
  int it = 0, st = YG_OK;
  if (par0.op == YG_OP_HPHI_SQ) {
    double *tmp = L.scratch_field(8);
    par.op = YG_OP_DPHI;
    blas_g5(L, b, lo, n);
    int i1 = 0, i2 = 0;
    st = bicgstab(L, par, tmp, b, &i1);
    blas_g5(L, tmp, lo, n);
    if (st == YG_OK) st = bicgstab(L, par, x, tmp, &i2);
    blas_g5(L, b, lo, n);
    it = i1 + i2;
  } else if (par0.op == YG_OP_HPHI) {
    par.op = YG_OP_DPHI;
    blas_g5(L, b, lo, n);
    st = bicgstab(L, par, x, b, &it);
    blas_g5(L, b, lo, n);
  } else if (par0.op == YG_OP_DPHI) {
    st = bicgstab(L, par, x, b, &it);
  } else {
    throw Error(YG_ERR_ARG, "auto: MVM operator not supported");
  }
  *iters = it;
  return st;
}

// rational_calc, rational.cpp:134-166
int rational_calc(Lattice &L, const yg_inv_par &par, double a0, int order, const double *poles,
                  const double *residues, double *x, double *b, int *iters) {
  std::vector<double *> outs(order);
  for (int i = 0; i < order; i++) outs[i] = L.scratch_field(60 + i);
  int st = cg_mshift(L, par, order, poles, outs.data(), b, iters);
  long lo, n;
  L.view_range(YG_VIEW_DEFAULT, lo, n);
  blas_axpby(L, x, make_double2(0, 0), make_double2(a0, 0), b, lo, n);
  for (int i = 0; i < order; i++) blas_axpby(L, x, make_double2(1, 0), make_double2(residues[i], 0), outs[i], lo, n);
  return st;
}

// ---------------------------------------------------------------------------------------
// Mixed precision: CG on A = Hphi_sq (the Hermitian positive operator of the even-odd
// system) with FP32 fields and the FP32 operator for the inner iterations, and FP64
// reliable updates: whenever the iterated residual fell by `delta` since the last update,
// the solution increment is folded into the FP64 x and the residual is recomputed as
// b - A x with the FP64 operator.  The stopping test is on that true FP64 residual, so the
// result meets the same criterion |b - A x|^2 < prec |b|^2 as the reference's cg_inverter.
// A stall (no reduction of the true residual over several updates) falls back to the
// plain FP64 CG from the current x.
int cg_mixed(Lattice &L, const yg_inv_par &par, double *x, double *b, yg_solve_stats *st) {
  auto t0 = std::chrono::steady_clock::now();
  if (par.op != YG_OP_HPHI_SQ) throw Error(YG_ERR_ARG, "cg_mixed solves Hphi_sq systems");
  if (!L.p.eo) throw Error(YG_ERR_ARG, "cg_mixed needs even-odd preconditioning");
  Ctx c(L);
  const long cnt = c.n * 4L * L.d;          // complex words of the even block
  double *r = L.scratch_field(3), *Ax = L.scratch_field(4), *xd = L.scratch_field(5);
  // FP32 fields: full-volume layout (the odd block is operator scratch)
  float *fr = reinterpret_cast<float *>(L.scratch_field(40));
  float *fp = reinterpret_cast<float *>(L.scratch_field(41));
  float *fx = reinterpret_cast<float *>(L.scratch_field(42));
  float *fq = reinterpret_cast<float *>(L.scratch_field(43));
  float *ft = reinterpret_cast<float *>(L.scratch_field(44));
  float *fo = reinterpret_cast<float *>(L.scratch_field(45));

  const double delta = 0.1;
  double norm = c.sqnorm(b);
  c.copy(xd, x);
  apply_op(L, YG_OP_HPHI_SQ, par.mass, Ax, xd);
  c.copy(r, b);
  c.axpby(r, {1, 0}, {-1, 0}, Ax);
  double rr = c.sqnorm(r);
  double target = norm * par.prec;
  int it = 0, updates = 0, status = YG_OK;
  double best = rr;
  int stall = 0;
  double *xbest = L.scratch_field(46);      // the iterate with the smallest true residual
  c.copy(xbest, x);
  if (rr >= target) {
    f_from_d(L, fr, r, cnt);
    f_from_d(L, fp, r, cnt);
    YG_CUDA(cudaMemsetAsync(fx, 0, sizeof(float2) * cnt, L.stream));
    double rr_s = rr, maxrr = rr;
    constexpr int kStagnate = 100;    // forced reliable update when |r| stops falling
    double min_cycle = rr;
    int since_min = 0;
    while (true) {
      if (par.maxiter > 0 && it >= par.maxiter) {
        status = YG_MAXITER;
        d_add_f(L, x, fx, cnt);       // keep the progress of the inner iterations
        break;
      }
      it++;
      hphi_float(L, par.mass, (float2 *)ft, (float2 *)fp, (float2 *)fo);
      hphi_float(L, par.mass, (float2 *)fq, (float2 *)ft, (float2 *)fo);
      double pq = f_product_re(L, fp, fq, cnt);
      check_finite(pq, "cg_mixed");
      double alpha = rr_s / pq;
      double rr_new = f_cg_update(L, fx, fr, fp, fq, (float)alpha, cnt);
      if (rr_new < 0.25 * min_cycle) { min_cycle = rr_new; since_min = 0; }
      else since_min++;
      bool update = rr_new < delta * delta * maxrr || rr_new < target || since_min >= kStagnate;
      if (update) {
        // fold the FP32 increment into x and recompute the true residual in FP64
        d_add_f(L, x, fx, cnt);
        YG_CUDA(cudaMemsetAsync(fx, 0, sizeof(float2) * cnt, L.stream));
        c.copy(xd, x);
        apply_op(L, YG_OP_HPHI_SQ, par.mass, Ax, xd);
        c.copy(r, b);
        c.axpby(r, {1, 0}, {-1, 0}, Ax);
        double rr_true = c.sqnorm(r);
        updates++;
        if (rr_true < target) { rr = rr_true; break; }
        if (rr_true < best) c.copy(xbest, x);
        if (rr_true > 100.0 * best) { status = YG_STALL; rr = rr_true; break; }   // diverged
        if (rr_true < 0.5 * best) stall = 0;
        else if (++stall >= 8) { status = YG_STALL; rr = rr_true; break; }
        best = std::min(best, rr_true);
        f_from_d(L, fr, r, cnt);
        double beta = rr_true / rr_s;
        f_xpay(L, fp, (float)beta, fr, cnt);
        rr_s = rr_true;
        maxrr = rr_true;
        min_cycle = rr_true;
        since_min = 0;
        rr = rr_true;
        continue;
      }
      double beta = rr_new / rr_s;
      f_xpay(L, fp, (float)beta, fr, cnt);
      rr_s = rr_new;
    }
  }
  int fallback = 0;
  if (status != YG_OK) {
    // plain FP64 CG (the reference's solver) from the best iterate, restarted until the
    // true residual meets prec (its recursive residual can stop above the true one)
    c.copy(x, xbest);
    yg_inv_par p64 = par;
    p64.log = 0;
    fallback = 1;
    for (int attempt = 0; attempt < 3; attempt++) {
      int it64 = 0;
      status = cg(L, p64, x, b, &it64);
      it += it64;
      c.copy(xd, x);
      apply_op(L, YG_OP_HPHI_SQ, par.mass, Ax, xd);
      c.copy(r, b);
      c.axpby(r, {1, 0}, {-1, 0}, Ax);
      rr = c.sqnorm(r);
      if (status != YG_OK || rr < target) break;
    }
    if (status == YG_OK && rr >= target) status = YG_STALL;
  }
  YG_CUDA(cudaStreamSynchronize(L.stream));
  if (st) {
    st->iterations = it;
    st->reliable_updates = updates;
    st->fallback = fallback;
    st->true_residual = rr / norm;
    st->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  log_line(par, "cg_mixed", it, rr / norm);
  return status;
}

}  // namespace yg
