// Device code of the representation map and of the clover-term build (included by the
// yg_inst_*_aux.cu units).
//
//   represent_links          repr.cpp:107-263     fund N x N -> fermion-representation D x D
//   AP sign                  bcs.cpp:264-272      U_0(t=0) *= -1 on the represented links
//   clover_repr              wilsonloop.cpp:5-31  four plaquette leaves, each represented
//   _compute_clover_term     clover.cpp:120-168   the blocks A0..A3 with coefficient -csw/16
//   _bcs_clover_term         clover.cpp:93-118    open / SF boundary slices zeroed
#pragma once

#include "yg_kernels.h"

namespace yg {

template <int N>
__device__ __forceinline__ void rk_load(double2 (&m)[N * N], const double2 *base, const Geom &g, int id, int mu) {
#pragma unroll
  for (int k = 0; k < N * N; k++) m[k] = base[fidx(g, id, mu * N * N + k, 4 * N * N)];
}

template <int N>
__device__ __forceinline__ void rk_mm(double2 (&c)[N * N], const double2 (&a)[N * N], const double2 (&b)[N * N]) {
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < N; k++) cfma(s, a[i * N + k], b[k * N + j]);
      c[i * N + j] = s;
    }
}

// c = a b^dag
template <int N>
__device__ __forceinline__ void rk_mmd(double2 (&c)[N * N], const double2 (&a)[N * N], const double2 (&b)[N * N]) {
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < N; k++) cfma(s, a[i * N + k], cconj(b[j * N + k]));
      c[i * N + j] = s;
    }
}

// c = a^dag b
template <int N>
__device__ __forceinline__ void rk_mdm(double2 (&c)[N * N], const double2 (&a)[N * N], const double2 (&b)[N * N]) {
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < N; k++) cfmac(s, a[k * N + i], b[k * N + j]);
      c[i * N + j] = s;
    }
}

// Representation map of one fundamental matrix.  Fundamental: copy.  Otherwise
// R_nm = tr(b_n^dag U b_m W) with W = U^T (two-index representations, U acting as
// S -> U S U^T) or W = U^dag (adjoint, X -> U X U^dag), in the orthonormal basis b of
// repr.cpp:25-59; this is the map the explicit formulas of repr.cpp:114-259 evaluate.
// The adjoint map is real and its imaginary part is set to zero, as in the reference.
template <int NC, int D>
__device__ void represent_one(double2 (&r)[D * D], const double2 (&u)[NC * NC], const double2 *basis, int rep) {
  if (rep == YG_REPR_FUNDAMENTAL) {
#pragma unroll
    for (int k = 0; k < D * D; k++) r[k] = (k < NC * NC) ? u[k] : make_double2(0, 0);
    return;
  }
#pragma unroll 1
  for (int m = 0; m < D; m++) {
    double2 ub[NC * NC];                      // U b_m
#pragma unroll
    for (int i = 0; i < NC; i++)
#pragma unroll
      for (int j = 0; j < NC; j++) {
        double2 s = make_double2(0, 0);
#pragma unroll
        for (int k = 0; k < NC; k++) cfma(s, u[i * NC + k], basis[m * NC * NC + k * NC + j]);
        ub[i * NC + j] = s;
      }
#pragma unroll 1
    for (int n = 0; n < D; n++) {
      double2 tr = make_double2(0, 0);
#pragma unroll
      for (int a = 0; a < NC; a++)
#pragma unroll
        for (int b = 0; b < NC; b++) {
          double2 bn = basis[n * NC * NC + a * NC + b];
          if (bn.x == 0.0 && bn.y == 0.0) continue;
          double2 x = make_double2(0, 0);     // (U b_m W)[a][b]
#pragma unroll
          for (int k = 0; k < NC; k++) {
            double2 w = (rep == YG_REPR_ADJOINT) ? cconj(u[b * NC + k]) : u[b * NC + k];
            cfma(x, ub[a * NC + k], w);
          }
          cfmac(tr, bn, x);
        }
      if (rep == YG_REPR_ADJOINT) tr.y = 0.0;
      r[n * D + m] = tr;
    }
  }
}

template <int NC, int D>
__global__ void k_represent(double2 *links, const double2 *fund, Geom g, const double2 *basis, int rep) {
  long r = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (r >= 4L * g.V) return;
  int id = (int)(r >> 2), mu = (int)(r & 3);
  double2 u[NC * NC];
  rk_load<NC>(u, fund, g, id, mu);
  double2 R[D * D];
  represent_one<NC, D>(R, u, basis, rep);
  int c[4];
  coords_of(g, id, c);
  double sgn = (g.bc == YG_BC_ANTIPERIODIC && mu == 0 && c[0] == 0) ? -1.0 : 1.0;   // bcs.cpp:264-272
  for (int k = 0; k < D * D; k++) links[fidx(g, id, mu * D * D + k, 4 * D * D)] = cscale(R[k], sgn);
}

// clover_repr(id,mu,nu) (wilsonloop.cpp:5-31) in the fermion representation
template <int NC, int D>
__device__ void clover_leaves(double2 (&out)[D * D], const double2 *fund, const Geom &g, const int c[4], int id,
                              int mu, int nu, const double2 *basis, int rep) {
  double2 A[NC * NC], B[NC * NC], P[NC * NC], Q[NC * NC], R[D * D];
  for (int k = 0; k < D * D; k++) out[k] = make_double2(0, 0);
  int cc[4];
#pragma unroll 1
  for (int leaf = 0; leaf < 4; leaf++) {
    if (leaf == 0) {         // U(x,mu) U(x+mu,nu) [U(x,nu) U(x+nu,mu)]^dag
      int a = neighbour(g, c, mu, +1), b = neighbour(g, c, nu, +1);
      rk_load<NC>(A, fund, g, id, mu); rk_load<NC>(B, fund, g, a, nu); rk_mm<NC>(P, A, B);
      rk_load<NC>(A, fund, g, id, nu); rk_load<NC>(B, fund, g, b, mu); rk_mm<NC>(Q, A, B);
      rk_mmd<NC>(A, P, Q);
    } else if (leaf == 1) {  // U(x,nu) [U(x-mu,nu) U(x-mu+nu,mu)]^dag U(x-mu,mu)
      int a = neighbour(g, c, mu, -1);
      coords_of(g, a, cc);
      int b = neighbour(g, cc, nu, +1);
      rk_load<NC>(A, fund, g, a, nu); rk_load<NC>(B, fund, g, b, mu); rk_mm<NC>(Q, A, B);
      rk_load<NC>(A, fund, g, id, nu); rk_mmd<NC>(P, A, Q);
      rk_load<NC>(B, fund, g, a, mu); rk_mm<NC>(A, P, B);
    } else if (leaf == 2) {  // [U(x-mu-nu,nu) U(x-mu,mu)]^dag U(x-mu-nu,mu) U(x-nu,nu)
      int a = neighbour(g, c, mu, -1), b = neighbour(g, c, nu, -1);
      coords_of(g, a, cc);
      int ci = neighbour(g, cc, nu, -1);
      rk_load<NC>(A, fund, g, ci, nu); rk_load<NC>(B, fund, g, a, mu); rk_mm<NC>(Q, A, B);
      rk_load<NC>(A, fund, g, ci, mu); rk_mdm<NC>(P, Q, A);
      rk_load<NC>(B, fund, g, b, nu); rk_mm<NC>(A, P, B);
    } else {                 // U(x-nu,nu)^dag U(x-nu,mu) U(x-nu+mu,nu) U(x,mu)^dag
      int a = neighbour(g, c, nu, -1);
      coords_of(g, a, cc);
      int b = neighbour(g, cc, mu, +1);
      rk_load<NC>(A, fund, g, a, nu); rk_load<NC>(B, fund, g, a, mu); rk_mdm<NC>(P, A, B);
      rk_load<NC>(B, fund, g, b, nu); rk_mm<NC>(Q, P, B);
      rk_load<NC>(B, fund, g, id, mu); rk_mmd<NC>(A, Q, B);
    }
    represent_one<NC, D>(R, A, basis, rep);
    for (int k = 0; k < D * D; k++) out[k] = cadd(out[k], R[k]);
  }
}

// _compute_clover_term (clover.cpp:120-168) incl. the boundary zeroing (:93-118)
template <int NC, int D>
__global__ void k_clover_term(double2 *cl, const double2 *fund, Geom g, const double2 *basis, int rep, double csw_in) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.V) return;
  int c[4];
  coords_of(g, id, c);
  int t = c[0], T = g.dim[0];
  bool zero = (g.bc == YG_BC_SF && (t == 0 || t == T - 1 || t == T - 2)) ||
              (g.bc == YG_BC_OPEN && (t == 0 || t == T - 1));
  if (zero) {
    for (int k = 0; k < 4 * D * D; k++) cl[fidx(g, id, k, 4 * D * D)] = make_double2(0, 0);
    return;
  }
  const double csw = -csw_in / 16.0;
  const int pm[6][2] = {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 3}};
  double2 tmp[6][D * D];
#pragma unroll 1
  for (int q = 0; q < 6; q++) clover_leaves<NC, D>(tmp[q], fund, g, c, id, pm[q][0], pm[q][1], basis, rep);
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) {
      int ij = i * D + j, ji = j * D + i;
      double a_re = tmp[2][ij].y + tmp[2][ji].y;
      double a_im = tmp[2][ji].x - tmp[2][ij].x;
      double b_re = tmp[3][ij].y + tmp[3][ji].y;
      double b_im = tmp[3][ij].x - tmp[3][ji].x;
      double c_re = tmp[0][ij].y + tmp[0][ji].y - tmp[1][ij].x + tmp[1][ji].x;
      double c_im = tmp[0][ji].x - tmp[0][ij].x - tmp[1][ij].y - tmp[1][ji].y;
      double d_re = tmp[4][ij].x - tmp[4][ji].x + tmp[5][ij].y + tmp[5][ji].y;
      double d_im = tmp[4][ij].y + tmp[4][ji].y - tmp[5][ij].x + tmp[5][ji].x;
      cl[fidx(g, id, 0 * D * D + ij, 4 * D * D)] = make_double2(csw * (a_re - b_re), csw * (a_im + b_im));
      cl[fidx(g, id, 1 * D * D + ij, 4 * D * D)] = make_double2(csw * (c_re - d_re), csw * (c_im - d_im));
      cl[fidx(g, id, 2 * D * D + ij, 4 * D * D)] = make_double2(-csw * (a_re + b_re), csw * (b_im - a_im));
      cl[fidx(g, id, 3 * D * D + ij, 4 * D * D)] = make_double2(-csw * (c_re + d_re), -csw * (c_im + d_im));
    }
}

template <int NC, int D>
void RK<NC, D>::represent(double2 *links, const double2 *fund, Geom g, const double2 *basis, int rep, cudaStream_t s) {
  k_represent<NC, D><<<nblk(4L * g.V, 128), 128, 0, s>>>(links, fund, g, basis, rep);
}

template <int NC, int D>
void RK<NC, D>::clover_term(double2 *cl, const double2 *fund, Geom g, const double2 *basis, int rep, double csw,
                            cudaStream_t s) {
  k_clover_term<NC, D><<<nblk(g.V, 64), 64, 0, s>>>(cl, fund, g, basis, rep, csw);
}

}  // namespace yg
