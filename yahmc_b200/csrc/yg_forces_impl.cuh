// Device code of the fermion forces and the gauge-side support kernels (included by the
// yg_inst_*_aux.cu units).
//
//   clover_fermion_force   forces.cpp:122-172   sigma_{mu nu} gamma5 outer products -> cl_force
//   hopping force          forces.cpp:175-227   Proj_TA[ U(x,mu) fmat ] -> momenta
//   compute_clover_force   clover.cpp:170-279   coeff * A_oo^-1 columns from the LDL -> cl_force
//   clover_force_core      forces.cpp:33-106    6-link assembly of cl_force -> momenta
//   wilson_gauge_force     forces.cpp:262-283   plaquette staples -> momenta
//   avr_wilson(1,1)        wilsonloop.cpp:116-133
// Momenta keep the reference's host layout afield_momenta[4*id+mu].av[NG]; FP64 throughout.
#pragma once

#include "yg_kernels.h"

namespace yg {

template <int D>
__device__ __forceinline__ void ld_spinor64(double2 (&s)[4][D], const double2 *f, const Geom &g, int id) {
#pragma unroll
  for (int sp = 0; sp < 4; sp++) {
    YG_UNROLL_DF
    for (int c = 0; c < D; c++) s[sp][c] = f[fidx(g, id, sp * D + c, 4 * D)];
  }
}

// Spinor::g5_sigma(mu,nu) for the clover-force slot order (0,1),(0,2),(1,2),(0,3),(1,3),(2,3)
// (spinor.cpp:266-438, forces.cpp:130-170)
template <int D>
__device__ __forceinline__ void g5_sigma(double2 (&o)[4][D], const double2 (&s)[4][D], int slot) {
  YG_UNROLL_DF
  for (int c = 0; c < D; c++) {
    switch (slot) {
      case 0: o[0][c] = ctimesmi(s[1][c]); o[1][c] = ctimesmi(s[0][c]); o[2][c] = ctimesmi(s[3][c]); o[3][c] = ctimesmi(s[2][c]); break;
      case 1: o[0][c] = cscale(s[1][c], -1.0); o[1][c] = s[0][c]; o[2][c] = cscale(s[3][c], -1.0); o[3][c] = s[2][c]; break;
      case 2: o[0][c] = ctimesi(s[0][c]); o[1][c] = ctimesmi(s[1][c]); o[2][c] = ctimesmi(s[2][c]); o[3][c] = ctimesi(s[3][c]); break;
      case 3: o[0][c] = ctimesmi(s[0][c]); o[1][c] = ctimesi(s[1][c]); o[2][c] = ctimesmi(s[2][c]); o[3][c] = ctimesi(s[3][c]); break;
      case 4: o[0][c] = cscale(s[1][c], -1.0); o[1][c] = s[0][c]; o[2][c] = s[3][c]; o[3][c] = cscale(s[2][c], -1.0); break;
      default: o[0][c] = ctimesi(s[1][c]); o[1][c] = ctimesi(s[0][c]); o[2][c] = ctimesmi(s[3][c]); o[3][c] = ctimesmi(s[2][c]); break;
    }
  }
}

// gamma5 (1 - gamma_mu) (Spinor::g5_one_minus_gamma, spinor.cpp:440-500)
template <int D>
__device__ __forceinline__ void g5_omg(double2 (&o)[4][D], const double2 (&s)[4][D], int mu) {
  YG_UNROLL_DF
  for (int c = 0; c < D; c++) {
    double2 a, b;
    switch (mu) {
      case 0: a = cadd(s[0][c], s[2][c]); b = cadd(s[1][c], s[3][c]);
        o[0][c] = a; o[1][c] = b; o[2][c] = cscale(a, -1.0); o[3][c] = cscale(b, -1.0); break;
      case 1: o[0][c] = cadd(s[0][c], ctimesi(s[3][c])); o[1][c] = cadd(s[1][c], ctimesi(s[2][c]));
        o[2][c] = csub(ctimesi(s[1][c]), s[2][c]); o[3][c] = csub(ctimesi(s[0][c]), s[3][c]); break;
      case 2: o[0][c] = cadd(s[0][c], s[3][c]); o[1][c] = csub(s[1][c], s[2][c]);
        o[2][c] = csub(s[1][c], s[2][c]); o[3][c] = cscale(cadd(s[3][c], s[0][c]), -1.0); break;
      default: o[0][c] = cadd(s[0][c], ctimesi(s[2][c])); o[1][c] = csub(s[1][c], ctimesi(s[3][c]));
        o[2][c] = csub(ctimesi(s[0][c]), s[2][c]); o[3][c] = cscale(cadd(s[3][c], ctimesi(s[1][c])), -1.0); break;
    }
  }
}

// fmat[i][j] += sum_k a[k][i] conj(b[k][j])  (fmat_create, forces.cpp:13-30)
template <int D>
__device__ __forceinline__ void outer_acc(double2 (&f)[D * D], const double2 (&a)[4][D], const double2 (&b)[4][D]) {
  YG_UNROLL_DF
  for (int i = 0; i < D; i++) {
    YG_UNROLL_DF
    for (int j = 0; j < D; j++) {
#pragma unroll
      for (int k = 0; k < 4; k++) cfma(f[i * D + j], a[k][i], cconj(b[k][j]));
    }
  }
}

// av[a] += coeff/(-TF) * Re tr(iT[a] m)   (algebra_project, suNa.cpp:91-111), TF = 2
template <int D>
__device__ __forceinline__ void project_add(double *mom, const double2 (&m)[D * D], const double2 *gens, int ng,
                                            double coeff) {
  double c = coeff / -2.0;
  for (int a = 0; a < ng; a++) {
    double tr = 0;
    for (int i = 0; i < D; i++)
      for (int k = 0; k < D; k++) {
        double2 t = gens[(a * D + i) * D + k];
        double2 v = m[k * D + i];
        tr += t.x * v.x - t.y * v.y;
      }
    mom[a] += c * tr;
  }
}

template <int D>
__device__ __forceinline__ void ld_mat(double2 (&m)[D * D], const double2 *base, const Geom &g, int id, int slot,
                                       int nslots) {
  YG_UNROLL_DF
  for (int k = 0; k < D * D; k++) m[k] = base[fidx(g, id, slot * D * D + k, nslots * D * D)];
}

template <int D>
__device__ __forceinline__ void mat_mul(double2 (&c)[D * D], const double2 (&a)[D * D], const double2 (&b)[D * D]) {
  YG_UNROLL_DF
  for (int i = 0; i < D; i++) {
    YG_UNROLL_DF
    for (int j = 0; j < D; j++) {
      double2 s = make_double2(0, 0);
      YG_UNROLL_DF
      for (int k = 0; k < D; k++) cfma(s, a[i * D + k], b[k * D + j]);
      c[i * D + j] = s;
    }
  }
}

template <int D>
__device__ __forceinline__ void dag(double2 (&c)[D * D], const double2 (&a)[D * D]) {
  YG_UNROLL_DF
  for (int i = 0; i < D; i++) {
    YG_UNROLL_DF
    for (int j = 0; j < D; j++) c[i * D + j] = cconj(a[j * D + i]);
  }
}

// ---- clover_fermion_force, forces.cpp:122-172 (all sites)
template <int D>
__global__ void k_clover_fermion_force(double2 *clf, const double2 *lhs, const double2 *rhs, Geom g, double residue) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.V) return;
  double2 l[4][D], r[4][D];
  ld_spinor64<D>(l, lhs, g, id);
  ld_spinor64<D>(r, rhs, g, id);
#pragma unroll 1
  for (int slot = 0; slot < 6; slot++) {
    double2 sl[4][D], sr[4][D];
    g5_sigma<D>(sl, l, slot);
    g5_sigma<D>(sr, r, slot);
    double2 f[D * D];
    YG_UNROLL_DF
    for (int k = 0; k < D * D; k++) f[k] = make_double2(0, 0);
    outer_acc<D>(f, sl, r);
    outer_acc<D>(f, sr, l);
    YG_UNROLL_DF
    for (int k = 0; k < D * D; k++) {
      long ix = fidx(g, id, slot * D * D + k, 6 * D * D);
      double2 o = clf[ix];
      o.x += residue * f[k].x;
      o.y += residue * f[k].y;
      clf[ix] = o;
    }
  }
}

// ---- hopping force, forces.cpp:200-223 (all sites, all mu)
template <int D>
__global__ void k_hopping_force(double *mom, const double2 *lhs, const double2 *rhs, const double2 *U, Geom g,
                                const double2 *itrepr, int ng, double coeff) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  int id = (int)(t >> 2), mu = (int)(t & 3);
  int c[4];
  coords_of(g, id, c);
  int fw = neighbour(g, c, mu, +1);
  double2 a[4][D], b[4][D], tl[4][D], tr[4][D];
  ld_spinor64<D>(a, lhs, g, fw);
  g5_omg<D>(tl, a, mu);
  ld_spinor64<D>(a, rhs, g, fw);
  g5_omg<D>(tr, a, mu);
  ld_spinor64<D>(a, rhs, g, id);
  ld_spinor64<D>(b, lhs, g, id);
  double2 f[D * D];
  YG_UNROLL_DF
  for (int k = 0; k < D * D; k++) f[k] = make_double2(0, 0);
  outer_acc<D>(f, tl, a);
  outer_acc<D>(f, tr, b);
  double2 u[D * D], m[D * D];
  ld_mat<D>(u, U, g, id, mu, 4);
  mat_mul<D>(m, u, f);
  project_add<D>(mom + (4L * id + mu) * ng, m, itrepr, ng, coeff);
}

// ---- _compute_clover_force, clover.cpp:170-262 (sites of block 1)
template <int D>
__global__ void k_clover_ldl_force(double2 *clf, const double2 *ldl, Geom g, double coeff) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= g.Vh) return;
  int id = g.Vh + h;
  constexpr int N = 2 * D, P = D * (2 * D + 1);
  double2 A[2][N][N];
  for (int blk = 0; blk < 2; blk++) {
    const double2 *Lb = ldl + (long)blk * P * g.Vh + h;
    for (int n = 0; n < N; n++) {
      for (int i = 0; i < N; i++) A[blk][i][n] = make_double2(i == n ? coeff : 0.0, 0.0);
      for (int i = n; i < N; i++)
        for (int k = 0; k < i; k++)
          A[blk][i][n] = csub(A[blk][i][n], cmul(Lb[(long)(i * (i + 1) / 2 + k) * g.Vh], A[blk][k][n]));
      for (int i = N - 1; i >= n; i--) {
        A[blk][i][n] = cscale(A[blk][i][n], 1.0 / Lb[(long)(i * (i + 1) / 2 + i) * g.Vh].x);
        for (int k = i + 1; k < N; k++)
          A[blk][i][n] = csub(A[blk][i][n], cmulc(Lb[(long)(k * (k + 1) / 2 + i) * g.Vh], A[blk][k][n]));
      }
    }
  }
  const double2(&a)[N][N] = A[0];
  const double2(&b)[N][N] = A[1];
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) {
      double2 a21 = a[i + D][j], a12 = cconj(a[j + D][i]), a43 = b[i + D][j], a34 = cconj(b[j + D][i]);
      double2 a11, a22, a33, a44;
      if (i < j) {
        a11 = cconj(a[j][i]); a22 = cconj(a[j + D][i + D]); a33 = cconj(b[j][i]); a44 = cconj(b[j + D][i + D]);
      } else {
        a11 = a[i][j]; a22 = a[i + D][j + D]; a33 = b[i][j]; a44 = b[i + D][j + D];
      }
      double2 F[6];
      F[0] = make_double2(a12.y + a21.y - a34.y - a43.y, -a12.x - a21.x + a34.x + a43.x);   // X_01
      F[1] = make_double2(a12.x - a21.x + a43.x - a34.x, a12.y - a21.y + a43.y - a34.y);    // X_02
      F[2] = make_double2(a22.y - a11.y + a44.y - a33.y, a11.x - a22.x + a33.x - a44.x);    // X_12
      F[3] = make_double2(a11.y - a22.y + a44.y - a33.y, a22.x - a11.x + a33.x - a44.x);    // X_03
      F[4] = make_double2(a12.x - a21.x + a34.x - a43.x, a12.y - a21.y + a34.y - a43.y);    // X_13
      F[5] = make_double2(-a12.y - a21.y - a34.y - a43.y, a12.x + a21.x + a34.x + a43.x);   // X_23
      for (int s = 0; s < 6; s++) {
        long ix = fidx(g, id, s * D * D + i * D + j, 6 * D * D);
        clf[ix] = cadd(clf[ix], F[s]);
      }
    }
}

// ---- clover_force_core, forces.cpp:33-106
template <int D>
__global__ void k_clover_force_core(double *mom, const double2 *clf, const double2 *U, Geom g, const double2 *itrepr,
                                    int ng, double coeff) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  int id = (int)(t >> 2), mu = (int)(t & 3);
  int c[4], cc[4];
  coords_of(g, id, c);
#pragma unroll 1
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    int o1 = neighbour(g, c, mu, +1);
    int o2 = neighbour(g, c, nu, +1);
    int o3 = neighbour(g, c, nu, -1);
    coords_of(g, o3, cc);
    int o4 = neighbour(g, cc, mu, +1);
    coords_of(g, o2, cc);
    int o5 = neighbour(g, cc, mu, +1);
    int num, sign;
    if (mu < nu) { num = nu * (nu - 1) / 2 + mu; sign = 1; }
    else { num = mu * (mu - 1) / 2 + nu; sign = -1; }
    double2 W0[D * D], W1[D * D], W2[D * D], W3[D * D], W4[D * D], W5[D * D], W6[D * D], W7[D * D], W8[D * D];
    double2 X[D * D], Y[D * D], Z[D * D], F[D * D];
    ld_mat<D>(X, U, g, o3, mu, 4); dag<D>(W0, X);
    ld_mat<D>(W1, U, g, o3, nu, 4);
    ld_mat<D>(W2, U, g, o1, nu, 4);
    ld_mat<D>(X, U, g, o2, mu, 4); dag<D>(W3, X);
    ld_mat<D>(X, U, g, id, nu, 4); dag<D>(W4, X);
    ld_mat<D>(X, U, g, o4, nu, 4); dag<D>(W5, X);
    mat_mul<D>(W6, W0, W1);
    mat_mul<D>(W7, W2, W3);
    mat_mul<D>(X, W7, W4);
    mat_mul<D>(Y, W5, W6);
    for (int k = 0; k < D * D; k++) W8[k] = csub(X[k], Y[k]);
    // F = W8 Z0 + Z1 W8
    ld_mat<D>(Z, clf, g, id, num, 6); mat_mul<D>(F, W8, Z);
    ld_mat<D>(Z, clf, g, o1, num, 6); mat_mul<D>(X, Z, W8);
    for (int k = 0; k < D * D; k++) F[k] = cadd(F[k], X[k]);
    // F -= W5 (W0 Z2 W1 + Z3 W6)
    ld_mat<D>(Z, clf, g, o3, num, 6); mat_mul<D>(X, W0, Z); mat_mul<D>(Y, X, W1);
    ld_mat<D>(Z, clf, g, o4, num, 6); mat_mul<D>(X, Z, W6);
    for (int k = 0; k < D * D; k++) Y[k] = cadd(Y[k], X[k]);
    mat_mul<D>(X, W5, Y);
    for (int k = 0; k < D * D; k++) F[k] = csub(F[k], X[k]);
    // F += (W2 Z4 W3 + W7 Z5) W4
    ld_mat<D>(Z, clf, g, o5, num, 6); mat_mul<D>(X, W2, Z); mat_mul<D>(Y, X, W3);
    ld_mat<D>(Z, clf, g, o2, num, 6); mat_mul<D>(X, W7, Z);
    for (int k = 0; k < D * D; k++) Y[k] = cadd(Y[k], X[k]);
    mat_mul<D>(X, Y, W4);
    for (int k = 0; k < D * D; k++) F[k] = cadd(F[k], X[k]);
    ld_mat<D>(X, U, g, id, mu, 4);
    mat_mul<D>(Y, X, F);
    project_add<D>(mom + (4L * id + mu) * ng, Y, itrepr, ng, sign * coeff);
  }
}

// ---- the same two forces summed over the poles of a rational approximation
// (rhmc.cpp:86-106 calls wilson_fermion_force_q once per pole): one thread per (site, slot)
// accumulates sum_n w_n fmat_n in registers and updates cl_force once; one thread per
// (site, mu) accumulates sum_n c_n fmat_n, multiplies by U once and projects once.  The
// projection is linear, so the result equals the sum of the per-pole forces up to rounding.
template <int D>
__global__ void k_clover_fermion_force_multi(double2 *clf, PoleSet ps, Geom g) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 6L * g.V) return;
  const int id = (int)(t / 6), slot = (int)(t % 6);
  double2 f[D * D];
  YG_UNROLL_DF
  for (int k = 0; k < D * D; k++) f[k] = make_double2(0, 0);
#pragma unroll 1
  for (int n = 0; n < ps.n; n++) {
    double2 l[4][D], r[4][D], sl[4][D], sr[4][D], fn[D * D];
    ld_spinor64<D>(l, ps.lhs[n], g, id);
    ld_spinor64<D>(r, ps.rhs[n], g, id);
    g5_sigma<D>(sl, l, slot);
    g5_sigma<D>(sr, r, slot);
    YG_UNROLL_DF
    for (int k = 0; k < D * D; k++) fn[k] = make_double2(0, 0);
    outer_acc<D>(fn, sl, r);
    outer_acc<D>(fn, sr, l);
    YG_UNROLL_DF
    for (int k = 0; k < D * D; k++) {
      f[k].x += ps.w[n] * fn[k].x;
      f[k].y += ps.w[n] * fn[k].y;
    }
  }
  YG_UNROLL_DF
  for (int k = 0; k < D * D; k++) {
    long ix = fidx(g, id, slot * D * D + k, 6 * D * D);
    double2 o = clf[ix];
    o.x += f[k].x;
    o.y += f[k].y;
    clf[ix] = o;
  }
}

template <int D>
__global__ void k_hopping_force_multi(double *mom, PoleSet ps, const double2 *U, Geom g, const double2 *itrepr,
                                      int ng) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  int id = (int)(t >> 2), mu = (int)(t & 3);
  int c[4];
  coords_of(g, id, c);
  int fw = neighbour(g, c, mu, +1);
  double2 f[D * D];
  YG_UNROLL_DF
  for (int k = 0; k < D * D; k++) f[k] = make_double2(0, 0);
#pragma unroll 1
  for (int n = 0; n < ps.n; n++) {
    double2 a[4][D], b[4][D], tl[4][D], tr[4][D], fn[D * D];
    ld_spinor64<D>(a, ps.lhs[n], g, fw);
    g5_omg<D>(tl, a, mu);
    ld_spinor64<D>(a, ps.rhs[n], g, fw);
    g5_omg<D>(tr, a, mu);
    ld_spinor64<D>(a, ps.rhs[n], g, id);
    ld_spinor64<D>(b, ps.lhs[n], g, id);
    YG_UNROLL_DF
    for (int k = 0; k < D * D; k++) fn[k] = make_double2(0, 0);
    outer_acc<D>(fn, tl, a);
    outer_acc<D>(fn, tr, b);
    YG_UNROLL_DF
    for (int k = 0; k < D * D; k++) {
      f[k].x += ps.w[n] * fn[k].x;
      f[k].y += ps.w[n] * fn[k].y;
    }
  }
  double2 u[D * D], m[D * D];
  ld_mat<D>(u, U, g, id, mu, 4);
  mat_mul<D>(m, u, f);
  project_add<D>(mom + (4L * id + mu) * ng, m, itrepr, ng, 1.0);
}

// ------------------------------------------------------------------ launchers
template <int D>
void DK<D>::clover_fermion_force_multi(double2 *clf, const PoleSet &ps, Geom g, cudaStream_t s) {
  k_clover_fermion_force_multi<D><<<nblk(6L * g.V, 64), 64, 0, s>>>(clf, ps, g);
}

template <int D>
void DK<D>::hopping_force_multi(double *mom, const PoleSet &ps, const double2 *U, Geom g, const double2 *itrepr,
                                int ng, cudaStream_t s) {
  k_hopping_force_multi<D><<<nblk(4L * g.V, 64), 64, 0, s>>>(mom, ps, U, g, itrepr, ng);
}

template <int D>
void DK<D>::clover_fermion_force(double2 *clf, const double2 *lhs, const double2 *rhs, Geom g, double residue,
                                 cudaStream_t s) {
  k_clover_fermion_force<D><<<nblk(g.V, 64), 64, 0, s>>>(clf, lhs, rhs, g, residue);
}

template <int D>
void DK<D>::hopping_force(double *mom, const double2 *lhs, const double2 *rhs, const double2 *U, Geom g,
                          const double2 *itrepr, int ng, double coeff, cudaStream_t s) {
  k_hopping_force<D><<<nblk(4L * g.V, 64), 64, 0, s>>>(mom, lhs, rhs, U, g, itrepr, ng, coeff);
}

template <int D>
void DK<D>::clover_ldl_force(double2 *clf, const double2 *ldl, Geom g, double coeff, cudaStream_t s) {
  k_clover_ldl_force<D><<<nblk(g.Vh, 64), 64, 0, s>>>(clf, ldl, g, coeff);
}

template <int D>
void DK<D>::clover_force_core(double *mom, const double2 *clf, const double2 *U, Geom g, const double2 *itrepr, int ng,
                              double coeff, cudaStream_t s) {
  k_clover_force_core<D><<<nblk(4L * g.V, 64), 64, 0, s>>>(mom, clf, U, g, itrepr, ng, coeff);
}

}  // namespace yg
