// Device code of the Wilson-clover Dirac operator (included by the yg_inst_*_op.cu units).
//
//  hop (dirac_kernel, dirac.cpp:227-704):
//      out(x) = -sign/2 * sum_mu [ (1-g_mu) U(x,mu) psi(x+mu) + (1+g_mu) U(x-mu,mu)^dag psi(x-mu) ]
//    in the chiral basis of spinor.cpp:191-264, followed by apply_bcs_on_spinor_field
//    (bcs.cpp:139-164).  One thread per output site; each direction spin-projects the
//    neighbour to a half spinor (2 x d), multiplies by the d x d link and reconstructs the
//    other two spin components.  The antiperiodic sign sits in the links (set at upload,
//    bcs.cpp:264-272).
//  Epilogues fused into the hop (the even-odd Schur operator of dirac.cpp:738-765):
//    CLOVINV  tmp_o = A_oo^-1 (hop)           (clover_inv_kernel, dirac.cpp:109-225)
//    CLOVADD  dst_e = A_ee src_e + hop [g5]    (clover_kernel, dirac.cpp:25-107; Hphi :769-773)
//    AXPY     dst   = a*src + hop [g5]         (dirac.cpp:755-765, no clover term)
//  Compute type R = double (the FP64 operator) or float (the inner operator of the
//  mixed-precision solver); storage is cplx<R>.
#pragma once

#include "yg_kernels.h"

namespace yg {

template <typename T>
__device__ __forceinline__ T ld(const T *p, long i) { return __ldg(p + i); }

template <int D, typename R>
__device__ __forceinline__ void load_spinor(cplx<R> (&s)[4][D], const cplx<R> *f, const Geom &g, int id) {
#pragma unroll
  for (int sp = 0; sp < 4; sp++) {
    YG_UNROLL_D
    for (int c = 0; c < D; c++) s[sp][c] = ld(f, fidx(g, id, sp * D + c, 4 * D));
  }
}

template <int D, typename R>
__device__ __forceinline__ void store_spinor(cplx<R> *f, const cplx<R> (&s)[4][D], const Geom &g, int id) {
#pragma unroll
  for (int sp = 0; sp < 4; sp++) {
    YG_UNROLL_D
    for (int c = 0; c < D; c++) f[fidx(g, id, sp * D + c, 4 * D)] = s[sp][c];
  }
}

// chi = U h (DAG=false) or U^dag h (DAG=true), U = link (id, mu)
template <int D, typename R, bool DAG>
__device__ __forceinline__ void link_mul(cplx<R> (&chi)[2][D], const cplx<R> (&h)[2][D], const cplx<R> *U,
                                         const Geom &g, int id, int mu) {
  YG_UNROLL_D
  for (int i = 0; i < D; i++) {
    cplx<R> s0 = mk<R>(0, 0), s1 = mk<R>(0, 0);
    YG_UNROLL_D
    for (int j = 0; j < D; j++) {
      cplx<R> u = ld(U, fidx(g, id, mu * D * D + (DAG ? j * D + i : i * D + j), 4 * D * D));
      if (DAG) { cfmac(s0, u, h[0][j]); cfmac(s1, u, h[1][j]); }
      else { cfma(s0, u, h[0][j]); cfma(s1, u, h[1][j]); }
    }
    chi[0][i] = s0;
    chi[1][i] = s1;
  }
}

// One direction: SIG = -1 for the forward term (1-g_mu), +1 for the backward term (1+g_mu).
template <int D, typename R, int MU, int SIG>
__device__ __forceinline__ void hop_dir(cplx<R> (&acc)[4][D], const cplx<R> *src, const cplx<R> *U,
                                        const Geom &g, int nid, int lid) {
  cplx<R> h[2][D];
  YG_UNROLL_D
  for (int c = 0; c < D; c++) {
    cplx<R> p0 = ld(src, fidx(g, nid, 0 * D + c, 4 * D));
    cplx<R> p1 = ld(src, fidx(g, nid, 1 * D + c, 4 * D));
    cplx<R> p2 = ld(src, fidx(g, nid, 2 * D + c, 4 * D));
    cplx<R> p3 = ld(src, fidx(g, nid, 3 * D + c, 4 * D));
    if (MU == 0) {
      h[0][c] = SIG < 0 ? cadd(p0, p2) : csub(p0, p2);
      h[1][c] = SIG < 0 ? cadd(p1, p3) : csub(p1, p3);
    } else if (MU == 1) {
      h[0][c] = SIG < 0 ? cadd(p0, ctimesi(p3)) : csub(p0, ctimesi(p3));
      h[1][c] = SIG < 0 ? cadd(p1, ctimesi(p2)) : csub(p1, ctimesi(p2));
    } else if (MU == 2) {
      h[0][c] = SIG < 0 ? cadd(p0, p3) : csub(p0, p3);
      h[1][c] = SIG < 0 ? csub(p1, p2) : cadd(p1, p2);
    } else {
      h[0][c] = SIG < 0 ? cadd(p0, ctimesi(p2)) : csub(p0, ctimesi(p2));
      h[1][c] = SIG < 0 ? csub(p1, ctimesi(p3)) : cadd(p1, ctimesi(p3));
    }
  }
  cplx<R> chi[2][D];
  link_mul<D, R, (SIG > 0)>(chi, h, U, g, lid, MU);
  YG_UNROLL_D
  for (int c = 0; c < D; c++) {
    acc[0][c] = cadd(acc[0][c], chi[0][c]);
    acc[1][c] = cadd(acc[1][c], chi[1][c]);
    if (MU == 0) {
      acc[2][c] = SIG < 0 ? cadd(acc[2][c], chi[0][c]) : csub(acc[2][c], chi[0][c]);
      acc[3][c] = SIG < 0 ? cadd(acc[3][c], chi[1][c]) : csub(acc[3][c], chi[1][c]);
    } else if (MU == 1) {
      acc[2][c] = SIG < 0 ? cadd(acc[2][c], ctimesmi(chi[1][c])) : cadd(acc[2][c], ctimesi(chi[1][c]));
      acc[3][c] = SIG < 0 ? cadd(acc[3][c], ctimesmi(chi[0][c])) : cadd(acc[3][c], ctimesi(chi[0][c]));
    } else if (MU == 2) {
      acc[2][c] = SIG < 0 ? csub(acc[2][c], chi[1][c]) : cadd(acc[2][c], chi[1][c]);
      acc[3][c] = SIG < 0 ? cadd(acc[3][c], chi[0][c]) : csub(acc[3][c], chi[0][c]);
    } else {
      acc[2][c] = SIG < 0 ? cadd(acc[2][c], ctimesmi(chi[0][c])) : cadd(acc[2][c], ctimesi(chi[0][c]));
      acc[3][c] = SIG < 0 ? cadd(acc[3][c], ctimesi(chi[1][c])) : cadd(acc[3][c], ctimesmi(chi[1][c]));
    }
  }
}

template <int D, typename R>
__device__ __forceinline__ void hop_site(cplx<R> (&acc)[4][D], const cplx<R> *src, const cplx<R> *U, const Geom &g,
                                         int id, const int c[4]) {
#pragma unroll
  for (int s = 0; s < 4; s++) {
    YG_UNROLL_D
    for (int k = 0; k < D; k++) acc[s][k] = mk<R>(0, 0);
  }
  int f, b;
  f = neighbour(g, c, 0, +1); hop_dir<D, R, 0, -1>(acc, src, U, g, f, id);
  b = neighbour(g, c, 0, -1); hop_dir<D, R, 0, +1>(acc, src, U, g, b, b);
  f = neighbour(g, c, 1, +1); hop_dir<D, R, 1, -1>(acc, src, U, g, f, id);
  b = neighbour(g, c, 1, -1); hop_dir<D, R, 1, +1>(acc, src, U, g, b, b);
  f = neighbour(g, c, 2, +1); hop_dir<D, R, 2, -1>(acc, src, U, g, f, id);
  b = neighbour(g, c, 2, -1); hop_dir<D, R, 2, +1>(acc, src, U, g, b, b);
  f = neighbour(g, c, 3, +1); hop_dir<D, R, 3, -1>(acc, src, U, g, f, id);
  b = neighbour(g, c, 3, -1); hop_dir<D, R, 3, +1>(acc, src, U, g, b, b);
}

// (4+m+cf) psi + [[A0,A1],[A1^dag,-A0]] (psi0,psi1) (+) [[A2,A3],[A3^dag,-A2]] (psi2,psi3)
template <int D, typename R>
__device__ __forceinline__ void clover_site(cplx<R> (&out)[4][D], const cplx<R> (&s)[4][D], const cplx<R> *cl,
                                            const Geom &g, int id, R diag) {
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    const int s0 = 2 * blk, s1 = 2 * blk + 1;
    const int m0 = 2 * blk, m1 = 2 * blk + 1;
    YG_UNROLL_D
    for (int i = 0; i < D; i++) {
      cplx<R> o0 = cscale(s[s0][i], diag), o1 = cscale(s[s1][i], diag);
      YG_UNROLL_D
      for (int j = 0; j < D; j++) {
        cplx<R> a0 = ld(cl, fidx(g, id, m0 * D * D + i * D + j, 4 * D * D));
        cplx<R> a1 = ld(cl, fidx(g, id, m1 * D * D + i * D + j, 4 * D * D));
        cplx<R> a1t = ld(cl, fidx(g, id, m1 * D * D + j * D + i, 4 * D * D));
        cfma(o0, a0, s[s0][j]);
        cfma(o0, a1, s[s1][j]);
        cfmac(o1, a1t, s[s0][j]);
        o1 = csub(o1, cmul(a0, s[s1][j]));
      }
      out[s0][i] = o0;
      out[s1][i] = o1;
    }
  }
}

// acc += A psi for the psi stored at src2 (A as in clover_site), one spin block at a time
// so that only two spins of psi are live next to the accumulator
template <int D, typename R>
__device__ __forceinline__ void clover_add_site(cplx<R> (&acc)[4][D], const cplx<R> *src2, const cplx<R> *cl,
                                                const Geom &g, int id, R diag) {
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    const int s0 = 2 * blk, s1 = 2 * blk + 1;
    const int m0 = 2 * blk, m1 = 2 * blk + 1;
    cplx<R> p0[D], p1[D];
#pragma unroll
    for (int c = 0; c < D; c++) {
      p0[c] = ld(src2, fidx(g, id, s0 * D + c, 4 * D));
      p1[c] = ld(src2, fidx(g, id, s1 * D + c, 4 * D));
    }
#pragma unroll
    for (int i = 0; i < D; i++) {
      cplx<R> o0 = cadd(acc[s0][i], cscale(p0[i], diag)), o1 = cadd(acc[s1][i], cscale(p1[i], diag));
#pragma unroll
      for (int j = 0; j < D; j++) {
        cplx<R> a0 = ld(cl, fidx(g, id, m0 * D * D + i * D + j, 4 * D * D));
        cplx<R> a1 = ld(cl, fidx(g, id, m1 * D * D + i * D + j, 4 * D * D));
        cplx<R> a1t = ld(cl, fidx(g, id, m1 * D * D + j * D + i, 4 * D * D));
        cfma(o0, a0, p0[j]);
        cfma(o0, a1, p1[j]);
        cfmac(o1, a1t, p0[j]);
        o1 = csub(o1, cmul(a0, p1[j]));
      }
      acc[s0][i] = o0;
      acc[s1][i] = o1;
    }
  }
}

// A^-1 psi through the packed LDL factors of the site: forward substitution, D^-1, back
// substitution with conj(L) (clover_inv_kernel, dirac.cpp:135-212)
template <int D, typename R>
__device__ __forceinline__ void ldl_site(cplx<R> (&out)[4][D], const cplx<R> (&s)[4][D], const double2 *ldl,
                                         int h, int Vh) {
  constexpr int N = 2 * D, P = D * (2 * D + 1);
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    const double2 *Lb = ldl + (long)blk * P * Vh + h;
    double2 x[N];
    #pragma unroll
    for (int i = 0; i < D; i++) {
      x[i] = make_double2((double)s[2 * blk][i].x, (double)s[2 * blk][i].y);
      x[i + D] = make_double2((double)s[2 * blk + 1][i].x, (double)s[2 * blk + 1][i].y);
    }
    #pragma unroll
    for (int i = 1; i < N; i++) {
      #pragma unroll
      for (int k = 0; k < i; k++) x[i] = csub(x[i], cmul(__ldg(Lb + (long)(i * (i + 1) / 2 + k) * Vh), x[k]));
    }
    #pragma unroll
    for (int i = N - 1; i >= 0; i--) {
      double dii = __ldg(Lb + (long)(i * (i + 1) / 2 + i) * Vh).x;
      x[i] = cscale(x[i], 1.0 / dii);
      #pragma unroll
      for (int k = i + 1; k < N; k++) x[i] = csub(x[i], cmulc(__ldg(Lb + (long)(k * (k + 1) / 2 + i) * Vh), x[k]));
    }
    #pragma unroll
    for (int i = 0; i < D; i++) {
      out[2 * blk][i] = mk<R>((R)x[i].x, (R)x[i].y);
      out[2 * blk + 1][i] = mk<R>((R)x[i + D].x, (R)x[i + D].y);
    }
  }
}

// A^-1 psi with explicit (2d x 2d) inverse blocks per site (FP32 inner operator)
template <int D, typename R>
__device__ __forceinline__ void cinv_site(cplx<R> (&out)[4][D], const cplx<R> (&s)[4][D], const cplx<R> *cinv,
                                          int h, int Vh) {
  constexpr int N = 2 * D;
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    YG_UNROLL_D
    for (int i = 0; i < N; i++) {
      cplx<R> acc = mk<R>(0, 0);
      YG_UNROLL_D
      for (int j = 0; j < N; j++) {
        cplx<R> a = ld(cinv, ((long)blk * N * N + i * N + j) * Vh + h);
        cplx<R> v = j < D ? s[2 * blk][j] : s[2 * blk + 1][j - D];
        cfma(acc, a, v);
      }
      if (i < D) out[2 * blk][i] = acc;
      else out[2 * blk + 1][i - D] = acc;
    }
  }
}

// A^-1 psi with the packed Hermitian inverse blocks of the FP64 path: per block of
// N = 2d rows, N real diagonal entries (two per double2 word) then the N(N-1)/2 complex
// lower-triangle entries (1,0),(2,0),(2,1),... one per word; word w of block b of the
// site h lives at (b*2d^2 + w)*Vh + h.  The upper triangle is the conjugate transpose.
template <int D, typename R>
__device__ __forceinline__ void cpk_site(cplx<R> (&out)[4][D], const cplx<R> (&s)[4][D], const double2 *cpk,
                                         int h, int Vh) {
  constexpr int N = 2 * D, W = 2 * D * D;
#pragma unroll
  for (int blk = 0; blk < 2; blk++) {
    const double2 *Cb = cpk + (long)blk * W * Vh + h;
    double2 x[N], y[N];
    #pragma unroll
    for (int i = 0; i < D; i++) {
      x[i] = make_double2((double)s[2 * blk][i].x, (double)s[2 * blk][i].y);
      x[i + D] = make_double2((double)s[2 * blk + 1][i].x, (double)s[2 * blk + 1][i].y);
    }
    #pragma unroll
    for (int w = 0; w < D; w++) {
      double2 dd = __ldg(Cb + (long)w * Vh);
      y[2 * w] = cscale(x[2 * w], dd.x);
      y[2 * w + 1] = cscale(x[2 * w + 1], dd.y);
    }
    #pragma unroll
    for (int i = 1; i < N; i++) {
      #pragma unroll
      for (int j = 0; j < i; j++) {
        double2 m = __ldg(Cb + (long)(D + i * (i - 1) / 2 + j) * Vh);
        cfma(y[i], m, x[j]);
        cfmac(y[j], m, x[i]);
      }
    }
    #pragma unroll
    for (int i = 0; i < D; i++) {
      out[2 * blk][i] = mk<R>((R)y[i].x, (R)y[i].y);
      out[2 * blk + 1][i] = mk<R>((R)y[i + D].x, (R)y[i + D].y);
    }
  }
}

template <int D, typename R, int EPI>
__device__ __forceinline__ void hop_body(const HopArgs<R> &a, int t) {
  const Geom &g = a.g;
  int id = a.lo + t;
  int c[4];
  coords_of(g, id, c);
  bool bnd = spinor_zeroed(g, c[0]);
  cplx<R> acc[4][D];
  hop_site<D, R>(acc, a.src, a.U, g, id, c);
#pragma unroll
  for (int s = 0; s < 4; s++) {
    YG_UNROLL_D
    for (int k = 0; k < D; k++) acc[s][k] = bnd ? mk<R>(0, 0) : cscale(acc[s][k], a.coeff);
  }

  if (EPI == EPI_PLAIN) {
    if (a.assign && !bnd) {
      cplx<R> old[4][D];
      load_spinor<D, R>(old, a.dst, g, id);
#pragma unroll
      for (int s = 0; s < 4; s++) {
        YG_UNROLL_D
        for (int k = 0; k < D; k++) acc[s][k] = cadd(acc[s][k], old[s][k]);
      }
    }
    store_spinor<D, R>(a.dst, acc, g, id);
  } else if (EPI == EPI_CLOVINV || EPI == EPI_CLOVPK) {
    if (a.dst2) store_spinor<D, R>(a.dst2, acc, g, id);
    cplx<R> out[4][D];
    if (EPI == EPI_CLOVPK) cpk_site<D, R>(out, acc, a.cpk, id - g.Vh, g.Vh);
    else if (sizeof(R) == sizeof(double)) ldl_site<D, R>(out, acc, a.ldl, id - g.Vh, g.Vh);
    else cinv_site<D, R>(out, acc, a.cinv, id - g.Vh, g.Vh);
    store_spinor<D, R>(a.dst, out, g, id);
  } else {
    bool zero_add = bnd && a.zero_add_at_boundary;
    if (EPI == EPI_CLOVADD) {
      R diag = a.diag + ((c[0] == g.Ta || c[0] == g.Tb) ? a.cfm1 : (R)0);
      if (!zero_add) clover_add_site<D, R>(acc, a.src2, a.cl, g, id, diag);
    } else {
      cplx<R> s2[4][D];
      load_spinor<D, R>(s2, a.src2, g, id);
#pragma unroll
      for (int s = 0; s < 4; s++) {
        YG_UNROLL_D
        for (int k = 0; k < D; k++) acc[s][k] = zero_add ? acc[s][k] : cadd(acc[s][k], cscale(s2[s][k], a.diag));
      }
    }
    if (a.g5) {
      YG_UNROLL_D
      for (int k = 0; k < D; k++) {
        acc[2][k] = cscale(acc[2][k], (R)-1);
        acc[3][k] = cscale(acc[3][k], (R)-1);
      }
    }
    store_spinor<D, R>(a.dst, acc, g, id);
  }
}

template <int D, typename R, int EPI>
__global__ void __launch_bounds__(128) k_hop(HopArgs<R> a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < a.n) hop_body<D, R, EPI>(a, t);
}

// clover_kernel (dirac.cpp:25-107) standalone: dst (=|+=) A psi over [lo, lo+n)
template <int D>
__global__ void __launch_bounds__(128) k_clover(double2 *dst, const double2 *src, const double2 *cl, Geom g,
                                                double mass4, double cfm1, int lo, int n, int assign) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  int id = lo + t;
  int c[4];
  coords_of(g, id, c);
  double diag = mass4 + ((c[0] == g.Ta || c[0] == g.Tb) ? cfm1 : 0.0);
  double2 s[4][D], o[4][D];
  load_spinor<D, double>(s, src, g, id);
  clover_site<D, double>(o, s, cl, g, id, diag);
  if (assign) {
    double2 old[4][D];
    load_spinor<D, double>(old, dst, g, id);
#pragma unroll
    for (int a = 0; a < 4; a++) {
      YG_UNROLL_D
      for (int k = 0; k < D; k++) o[a][k] = cadd(o[a][k], old[a][k]);
    }
  }
  store_spinor<D, double>(dst, o, g, id);
}

// clover_inv_kernel (dirac.cpp:109-225) standalone, sites of block 1
template <int D>
__global__ void __launch_bounds__(128) k_clover_inv(double2 *dst, const double2 *src, const double2 *ldl, Geom g,
                                                    int assign) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= g.Vh) return;
  int id = g.Vh + h;
  double2 s[4][D], o[4][D];
  load_spinor<D, double>(s, src, g, id);
  ldl_site<D, double>(o, s, ldl, h, g.Vh);
  if (assign) {
    double2 old[4][D];
    load_spinor<D, double>(old, dst, g, id);
#pragma unroll
    for (int a = 0; a < 4; a++) {
      YG_UNROLL_D
      for (int k = 0; k < D; k++) o[a][k] = cadd(o[a][k], old[a][k]);
    }
  }
  store_spinor<D, double>(dst, o, g, id);
}

// _compute_ldl_decomp (clover.cpp:25-91) with ldl() of solver.cpp:97-117, one thread per
// site of block 1 (the odd sites with even-odd ordering; odd_sites_for in geometry.h:18-19)
template <int D>
__global__ void k_ldl(double2 *ldl, const double2 *cl, Geom g, double sigma, double cf_in, int boundary_term) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= g.Vh) return;
  int id = g.Vh + h;
  constexpr int N = 2 * D;
  constexpr int P = D * (2 * D + 1);
  double cf = 0;
  if (boundary_term) {
    int c[4];
    coords_of(g, id, c);
    if (c[0] == g.Ta || c[0] == g.Tb) cf = cf_in - 1.0;
  }
  for (int blk = 0; blk < 2; blk++) {
    double2 A[N * N];
    for (int k = 0; k < N * N; k++) A[k] = make_double2(0, 0);
    int m0 = blk ? 2 : 0, m1 = blk ? 3 : 1;
    for (int i = 0; i < D; i++)
      for (int j = 0; j < D; j++) {
        A[(i + D) * N + j] = cconj(cl[fidx(g, id, m1 * D * D + j * D + i, 4 * D * D)]);
        if (i >= j) {
          double2 a = cl[fidx(g, id, m0 * D * D + i * D + j, 4 * D * D)];
          A[i * N + j] = a;
          A[(i + D) * N + D + j] = make_double2(-a.x, -a.y);
          if (i == j) {
            A[i * N + j].x += sigma + cf;
            A[(i + D) * N + D + j].x += sigma + cf;
          }
        }
      }
    for (int i = 0; i < N; i++) {
      for (int k = 0; k < i; k++)
        A[i * N + i].x -= (A[i * N + k].x * A[i * N + k].x + A[i * N + k].y * A[i * N + k].y) * A[k * N + k].x;
      for (int j = i + 1; j < N; j++) {
        for (int k = 0; k < i; k++) {
          double2 t = cmul(A[j * N + k], cconj(A[i * N + k]));
          A[j * N + i] = csub(A[j * N + i], cscale(t, A[k * N + k].x));
        }
        A[j * N + i] = cscale(A[j * N + i], 1.0 / A[i * N + i].x);
      }
    }
    int k = 0;
    for (int i = 0; i < N; i++)
      for (int j = 0; j <= i; j++, k++) ldl[((long)blk * P + k) * g.Vh + h] = A[i * N + j];
  }
}

// explicit inverse of both clover blocks in FP32, from the FP64 LDL factors
template <int D>
__global__ void k_cinv_float(float2 *cinv, const double2 *ldl, int Vh) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= Vh) return;
  constexpr int N = 2 * D, P = D * (2 * D + 1);
  for (int blk = 0; blk < 2; blk++) {
    const double2 *Lb = ldl + (long)blk * P * Vh + h;
    for (int col = 0; col < N; col++) {
      double2 x[N];
      for (int i = 0; i < N; i++) x[i] = make_double2(i == col ? 1.0 : 0.0, 0.0);
      for (int i = 1; i < N; i++)
        for (int k = 0; k < i; k++) x[i] = csub(x[i], cmul(Lb[(long)(i * (i + 1) / 2 + k) * Vh], x[k]));
      for (int i = N - 1; i >= 0; i--) {
        x[i] = cscale(x[i], 1.0 / Lb[(long)(i * (i + 1) / 2 + i) * Vh].x);
        for (int k = i + 1; k < N; k++) x[i] = csub(x[i], cmulc(Lb[(long)(k * (k + 1) / 2 + i) * Vh], x[k]));
      }
      for (int i = 0; i < N; i++)
        cinv[((long)blk * N * N + i * N + col) * Vh + h] = make_float2((float)x[i].x, (float)x[i].y);
    }
  }
}

// packed Hermitian FP64 inverse of both clover blocks (layout of cpk_site), from the LDL
// factors: column j of A^-1 by forward substitution, D^-1 and back substitution
template <int D>
__global__ void k_cinv_packed64(double2 *cpk, const double2 *ldl, int Vh) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= Vh) return;
  constexpr int N = 2 * D, P = D * (2 * D + 1), W = 2 * D * D;
  for (int blk = 0; blk < 2; blk++) {
    const double2 *Lb = ldl + (long)blk * P * Vh + h;
    double2 *Cb = cpk + (long)blk * W * Vh + h;
    for (int col = 0; col < N; col++) {
      double2 x[N];
      for (int i = 0; i < N; i++) x[i] = make_double2(i == col ? 1.0 : 0.0, 0.0);
      for (int i = 1; i < N; i++)
        for (int k = 0; k < i; k++) x[i] = csub(x[i], cmul(Lb[(long)(i * (i + 1) / 2 + k) * Vh], x[k]));
      for (int i = N - 1; i >= 0; i--) {
        x[i] = cscale(x[i], 1.0 / Lb[(long)(i * (i + 1) / 2 + i) * Vh].x);
        for (int k = i + 1; k < N; k++) x[i] = csub(x[i], cmulc(Lb[(long)(k * (k + 1) / 2 + i) * Vh], x[k]));
      }
      // diagonal entry (col, col): real part into its half of word col/2
      double *dw = reinterpret_cast<double *>(Cb + (long)(col / 2) * Vh);
      dw[col & 1] = x[col].x;
      for (int i = col + 1; i < N; i++) Cb[(long)(D + i * (i - 1) / 2 + col) * Vh] = x[i];
    }
  }
}

// log prod_n D_nn of both blocks per site (clover_logdet, clover.cpp:281-305)
template <int D>
__global__ void k_logdet(double *out, const double2 *ldl, int Vh) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= Vh) return;
  constexpr int N = 2 * D, P = D * (2 * D + 1);
  double prod = 1;
  for (int n = 0; n < N; n++) {
    prod *= ldl[((long)0 * P + n * (n + 1) / 2 + n) * Vh + h].x;
    prod *= ldl[((long)1 * P + n * (n + 1) / 2 + n) * Vh + h].x;
  }
  out[h] = log(prod);
}

// ------------------------------------------------------------------ DK<D> launchers
template <int D, typename R>
static void launch_hop_epi(const HopArgs<R> &a, int epi, cudaStream_t s) {
  const int t = 128;
  switch (epi) {
    case EPI_PLAIN: k_hop<D, R, EPI_PLAIN><<<nblk(a.n, t), t, 0, s>>>(a); break;
    case EPI_CLOVINV: k_hop<D, R, EPI_CLOVINV><<<nblk(a.n, t), t, 0, s>>>(a); break;
    case EPI_CLOVADD: k_hop<D, R, EPI_CLOVADD><<<nblk(a.n, t), t, 0, s>>>(a); break;
    case EPI_CLOVPK: k_hop<D, R, EPI_CLOVPK><<<nblk(a.n, t), t, 0, s>>>(a); break;
    default: k_hop<D, R, EPI_AXPY><<<nblk(a.n, t), t, 0, s>>>(a); break;
  }
}

template <int D>
void DK<D>::hop(const HopArgs<double> &a, int epi, cudaStream_t s) { launch_hop_epi<D, double>(a, epi, s); }

template <int D>
void DK<D>::hop(const HopArgs<float> &a, int epi, cudaStream_t s) { launch_hop_epi<D, float>(a, epi, s); }

template <int D>
void DK<D>::clover(double2 *dst, const double2 *src, const double2 *cl, Geom g, double mass4, double cfm1, int lo,
                   int n, int assign, cudaStream_t s) {
  k_clover<D><<<nblk(n, 128), 128, 0, s>>>(dst, src, cl, g, mass4, cfm1, lo, n, assign);
}

template <int D>
void DK<D>::clover_inv(double2 *dst, const double2 *src, const double2 *ldl, Geom g, int assign, cudaStream_t s) {
  k_clover_inv<D><<<nblk(g.Vh, 128), 128, 0, s>>>(dst, src, ldl, g, assign);
}

template <int D>
void DK<D>::ldl(double2 *ldl, const double2 *cl, Geom g, double sigma, double cf, int boundary_term, cudaStream_t s) {
  k_ldl<D><<<nblk(g.Vh, 64), 64, 0, s>>>(ldl, cl, g, sigma, cf, boundary_term);
}

template <int D>
void DK<D>::cinv_float(float2 *cinv, const double2 *ldl, int Vh, cudaStream_t s) {
  k_cinv_float<D><<<nblk(Vh, 64), 64, 0, s>>>(cinv, ldl, Vh);
}

template <int D>
void DK<D>::cinv_packed64(double2 *cpk, const double2 *ldl, int Vh, cudaStream_t s) {
  k_cinv_packed64<D><<<nblk(Vh, 64), 64, 0, s>>>(cpk, ldl, Vh);
}

template <int D>
void DK<D>::logdet(double *out, const double2 *ldl, int Vh, cudaStream_t s) {
  k_logdet<D><<<nblk(Vh, 128), 128, 0, s>>>(out, ldl, Vh);
}

}  // namespace yg
