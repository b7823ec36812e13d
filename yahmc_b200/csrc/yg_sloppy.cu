// Inner ("sloppy") operator of the mixed-precision solver for d = 3 representations.
//
// The FP64 engine (yg_dirac.cu) keeps the reference's layouts and arithmetic; the inner
// iterations of cg_mixed only need an approximation of the same operator, so they read
// compressed copies built once per gauge field and mass:
//   * spinors in FP32 (2 complex per 16-byte word) or FP16 (4 complex per 16-byte word,
//     scaled by a per-site FP32 norm = max |component|);
//   * links with 18 reals (9 complex) or, for SU(3) fundamental, 12 reals (rows 0 and 1;
//     row 2 = conj(row0 x row1), times the antiperiodic sign the stored rows carry);
//   * the clover term as two packed Hermitian 6x6 blocks per site (6 real diagonal entries
//     + 15 complex lower-triangle entries each): M_e = (4+m+cf) + A on even sites and the
//     explicit inverse M_o^-1 on odd sites, so that the Schur operator of dirac.cpp:738-751
//     is   t_o = M_o^-1 (1/2 H psi_e),   out_e = gamma5 (M_e psi_e - 1/2 H t_o).
//     Without a clover term M_o^-1 = 1 and M_e = (4+m)^2 (dirac.cpp:755-765).
// Arithmetic is FP32 throughout; FP16 is a storage format only.
#include <cuda_fp16.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <thread>
#include "yg_lattice.h"
#include "yg_kernels.h"
#include "yg_sloppy_impl.cuh"

namespace yg {

// one direction: SIG = -1 forward (1 - gamma_mu), +1 backward (1 + gamma_mu); as hop_dir
// in yg_dirac_impl.cuh (dirac.cpp:258-697)
template <int P, int LP, int K, int MU, int SIG>
__device__ __forceinline__ void shop_dir(float2 (&acc)[12], const SHopArgs &a, int nid, int lid, int lt) {
  const Geom &g = a.g;
  float2 p[12];
  int nb = nid >= g.Vh, nh = nid - nb * g.Vh;
  sload_raw<P>(p, a.src, nb, nh, g.Vh);          // the site norm multiplies chi below (linear)
  const float pn = snorm<P>(a.src_norm, nb, nh, g.Vh);
  float2 hh[2][3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    float2 p0 = p[c], p1 = p[3 + c], p2 = p[6 + c], p3 = p[9 + c];
    if (MU == 0) {
      hh[0][c] = SIG < 0 ? cadd(p0, p2) : csub(p0, p2);
      hh[1][c] = SIG < 0 ? cadd(p1, p3) : csub(p1, p3);
    } else if (MU == 1) {
      hh[0][c] = SIG < 0 ? cadd(p0, ctimesi(p3)) : csub(p0, ctimesi(p3));
      hh[1][c] = SIG < 0 ? cadd(p1, ctimesi(p2)) : csub(p1, ctimesi(p2));
    } else if (MU == 2) {
      hh[0][c] = SIG < 0 ? cadd(p0, p3) : csub(p0, p3);
      hh[1][c] = SIG < 0 ? csub(p1, p2) : cadd(p1, p2);
    } else {
      hh[0][c] = SIG < 0 ? cadd(p0, ctimesi(p2)) : csub(p0, ctimesi(p2));
      hh[1][c] = SIG < 0 ? csub(p1, ctimesi(p3)) : cadd(p1, ctimesi(p3));
    }
  }
  int lb = lid >= g.Vh, lh = lid - lb * g.Vh;
  float sgn = (g.bc == YG_BC_ANTIPERIODIC && MU == 0 && lt == 0) ? -1.f : 1.f;
  float2 u[9];
  link_load<LP, K>(u, a.U, lb, lh, g.Vh, MU, sgn);
  float2 chi[2][3];
#pragma unroll
  for (int i = 0; i < 3; i++) {
    float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
#pragma unroll
    for (int j = 0; j < 3; j++) {
      if (SIG > 0) { cfmac(s0, u[j * 3 + i], hh[0][j]); cfmac(s1, u[j * 3 + i], hh[1][j]); }
      else { cfma(s0, u[i * 3 + j], hh[0][j]); cfma(s1, u[i * 3 + j], hh[1][j]); }
    }
    chi[0][i] = P == 16 ? cscale(s0, pn) : s0;
    chi[1][i] = P == 16 ? cscale(s1, pn) : s1;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    acc[c] = cadd(acc[c], chi[0][c]);
    acc[3 + c] = cadd(acc[3 + c], chi[1][c]);
    if (MU == 0) {
      acc[6 + c] = SIG < 0 ? cadd(acc[6 + c], chi[0][c]) : csub(acc[6 + c], chi[0][c]);
      acc[9 + c] = SIG < 0 ? cadd(acc[9 + c], chi[1][c]) : csub(acc[9 + c], chi[1][c]);
    } else if (MU == 1) {
      acc[6 + c] = SIG < 0 ? cadd(acc[6 + c], ctimesmi(chi[1][c])) : cadd(acc[6 + c], ctimesi(chi[1][c]));
      acc[9 + c] = SIG < 0 ? cadd(acc[9 + c], ctimesmi(chi[0][c])) : cadd(acc[9 + c], ctimesi(chi[0][c]));
    } else if (MU == 2) {
      acc[6 + c] = SIG < 0 ? csub(acc[6 + c], chi[1][c]) : cadd(acc[6 + c], chi[1][c]);
      acc[9 + c] = SIG < 0 ? cadd(acc[9 + c], chi[0][c]) : csub(acc[9 + c], chi[0][c]);
    } else {
      acc[6 + c] = SIG < 0 ? cadd(acc[6 + c], ctimesmi(chi[0][c])) : cadd(acc[6 + c], ctimesi(chi[0][c]));
      acc[9 + c] = SIG < 0 ? cadd(acc[9 + c], ctimesi(chi[1][c])) : cadd(acc[9 + c], ctimesmi(chi[1][c]));
    }
  }
}

// STEP 1 (odd output):  out = M_o^-1 (coeff * hop(src))
// STEP 2 (even output): out = gamma5 (M_e src2 + coeff * hop(src))
// (zero on the sites a boundary condition zeroes)
template <int P, int LP, int CP, int K, int STEP>
__device__ __forceinline__ void shop_out(float2 (&out)[12], const SHopArgs &a, int id, const SiteNbr &n) {
  const Geom &g = a.g;
  const int T = g.dim[0], t0 = n.c[0];
  float2 acc[12];
#pragma unroll
  for (int k = 0; k < 12; k++) acc[k] = make_float2(0.f, 0.f);
  shop_dir<P, LP, K, 0, -1>(acc, a, n.f[0], id, t0);
  shop_dir<P, LP, K, 0, +1>(acc, a, n.b[0], n.b[0], t0 == 0 ? T - 1 : t0 - 1);
  shop_dir<P, LP, K, 1, -1>(acc, a, n.f[1], id, t0);
  shop_dir<P, LP, K, 1, +1>(acc, a, n.b[1], n.b[1], t0);
  shop_dir<P, LP, K, 2, -1>(acc, a, n.f[2], id, t0);
  shop_dir<P, LP, K, 2, +1>(acc, a, n.b[2], n.b[2], t0);
  shop_dir<P, LP, K, 3, -1>(acc, a, n.f[3], id, t0);
  shop_dir<P, LP, K, 3, +1>(acc, a, n.b[3], n.b[3], t0);
  int blk = id >= g.Vh, h = id - blk * g.Vh;
  bool bnd = spinor_zeroed(g, t0);
  float cl[72];
  cload<CP>(cl, a.C, a.Cn, blk, h, g.Vh);
  if (STEP == 1) {
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = cscale(acc[k], a.coeff);
    clover_packed(out, cl, acc);
  } else {
    float2 s2[12];
    sload<P>(s2, a.src2, a.src2_norm, blk, h, g.Vh);
    clover_packed(out, cl, s2);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      out[k] = cadd(out[k], cscale(acc[k], a.coeff));
      if (k >= 6) out[k] = cscale(out[k], -1.f);            // gamma5
    }
  }
  if (bnd) {
#pragma unroll
    for (int k = 0; k < 12; k++) out[k] = make_float2(0.f, 0.f);
  }
}

// dst = out of the site; returns |dst|^2 (before FP16 rounding)
template <int P, int LP, int CP, int K, int STEP>
__device__ __forceinline__ float shop_site(const SHopArgs &a, int id, const SiteNbr &n) {
  float2 out[12];
  shop_out<P, LP, CP, K, STEP>(out, a, id, n);
  float n2 = 0.f;
#pragma unroll
  for (int k = 0; k < 12; k++) n2 = fmaf(out[k].x, out[k].x, fmaf(out[k].y, out[k].y, n2));
  const int blk = id >= a.g.Vh;
  sstore<P>(a.dst, a.dst_norm, out, blk, id - blk * a.g.Vh, a.g.Vh);
  return n2;
}

// NRM = 1 (first Hphi of a CG iteration, t = Hphi p): also the per-block partials of
// <p, A p> = |t|^2 (Hphi is Hermitian and A = Hphi^2); a grid-stride loop over a grid of
// resident blocks keeps the number of partials small
template <int P, int LP, int CP, int K, int STEP, int NRM>
__device__ __forceinline__ void shop_body(const SHopArgs &a) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (!NRM) {
    SiteNbr n;
    if (t < a.n) site_nbr(n, a.g, a.lo + t);
    griddep_wait();
    if (t < a.n) shop_site<P, LP, CP, K, STEP>(a, a.lo + t, n);
    griddep_launch();
    return;
  }
  griddep_wait();
  double n2 = 0.0;
  for (; t < a.n; t += gridDim.x * blockDim.x) {
    SiteNbr n;
    site_nbr(n, a.g, a.lo + t);
    n2 += (double)shop_site<P, LP, CP, K, STEP>(a, a.lo + t, n);
  }
  n2 = block_total(n2);
  if (threadIdx.x == 0) a.part[blockIdx.x] = n2;
  griddep_launch();
}

template <int P, int LP, int CP, int K, int STEP, int NRM>
__global__ void __launch_bounds__(128) k_shop(SHopArgs a) {
  shop_body<P, LP, CP, K, STEP, NRM>(a);
}

// step 2 with the <p, A p> partials, registers cut for MINB resident blocks per SM (the tuner
// chooses between this and the compiler's own register count)
template <int P, int LP, int CP, int K, int MINB>
__global__ void __launch_bounds__(128, MINB) k_shop_nrm_min(SHopArgs a) {
  shop_body<P, LP, CP, K, 2, 1>(a);
}

// The plain step 1 in another block shape (TPB threads per block, registers cut for MINB
// resident blocks per SM), for the tuner to choose; one site per thread as k_shop.
template <int P, int LP, int CP, int K, int TPB, int MINB>
__global__ void __launch_bounds__(TPB, MINB) k_shop_shaped(SHopArgs a) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  SiteNbr n;
  if (t < a.n) site_nbr(n, a.g, a.lo + t);
  griddep_wait();
  if (t < a.n) shop_site<P, LP, CP, K, 1>(a, a.lo + t, n);
  griddep_launch();
}

// The last Schur step of the iteration's second Hphi with the residual update as its
// epilogue: q = Hphi t stays in registers, alpha = |r|^2 / <p, A p> (every block sums the
// partials of the NRM hop in the same order), r -= alpha q on the site, and the per-block
// partials of the new |r|^2 go to part_r.  q is never stored; x += alpha p is left to the
// p = r + beta p pass, which reads p anyway.  Resident grid, grid-stride.
struct SCgArgs {
  float2 *r;                      // FP32 even-site words
  double *scal;
  const double *part_pq;
  int n_pq;
  double *part_r;
  int par;
};

template <int P, int LP, int CP, int K>
__device__ __forceinline__ void shop_cg_body(const SHopArgs &a, const SCgArgs &c) {
  griddep_wait();
  const double pq = sum_partials(c.part_pq, c.n_pq);
  const double alpha = c.scal[S_RR0 + c.par] / pq;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    c.scal[S_PQ] = pq;
    c.scal[S_ALPHA] = alpha;
  }
  const float al = (float)alpha;
  const int Vh = a.g.Vh;
  double acc = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < a.n; t += gridDim.x * blockDim.x) {
    SiteNbr n;
    site_nbr(n, a.g, a.lo + t);
    float2 q[12];
    shop_out<P, LP, CP, K, 2>(q, a, a.lo + t, n);
    float s = 0.f;
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const long i = (long)k * Vh + t;
      float2 ri = c.r[i];
      ri.x = fmaf(-al, q[k].x, ri.x);
      ri.y = fmaf(-al, q[k].y, ri.y);
      c.r[i] = ri;
      s = fmaf(ri.x, ri.x, fmaf(ri.y, ri.y, s));
    }
    acc += s;
  }
  acc = block_total(acc);
  if (threadIdx.x == 0) c.part_r[blockIdx.x] = acc;
  griddep_launch();
}

template <int P, int LP, int CP, int K>
__global__ void __launch_bounds__(128) k_shop_cg(SHopArgs a, SCgArgs c) {
  shop_cg_body<P, LP, CP, K>(a, c);
}

template <int P, int LP, int CP, int K, int MINB>
__global__ void __launch_bounds__(128, MINB) k_shop_cg_min(SHopArgs a, SCgArgs c) {
  shop_cg_body<P, LP, CP, K>(a, c);
}

// ------------------------------------------------------------------ builds (once per gauge field / mass)
template <int LP>
__device__ __forceinline__ void lstore(void *base, long i, double2 v) {
  if (LP == ST_F32) reinterpret_cast<float2 *>(base)[i] = make_float2((float)v.x, (float)v.y);
  else if (LP == ST_F16) reinterpret_cast<unsigned *>(base)[i] = f2h(make_float2((float)v.x, (float)v.y));
  else reinterpret_cast<unsigned *>(base)[i] = f2s((float)v.x, (float)v.y);
}

// links: the first K complex entries (row-major) of each FP64 represented link
template <int LP, int K>
__global__ void k_pack_links(void *dst, const double2 *links, Geom g) {
  long r = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (r >= 4L * g.V) return;
  int id = (int)(r >> 2), mu = (int)(r & 3);
  int blk = id >= g.Vh, h = id - blk * g.Vh;
  if (K != 4) {
    for (int k = 0; k < K; k++)
      lstore<LP>(dst, ((long)(blk * 4 + mu) * K + k) * g.Vh + h, links[fidx(g, id, mu * 9 + k, 36)]);
    return;
  }
  // 8 reals (FP32): W = s V with s = sign det V (the antiperiodic sign), columns shifted
  // cyclically so that a0 is the largest entry of row 0 (|a0|^2 >= 1/3), then the smaller
  // of b0, c0 stored in full and the phases of a0 and of the other one (link_load)
  double2 V[9];
  for (int k = 0; k < 9; k++) V[k] = links[fidx(g, id, mu * 9 + k, 36)];
  auto m = [](double2 x, double2 y) { return make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x); };
  auto sb = [](double2 x, double2 y) { return make_double2(x.x - y.x, x.y - y.y); };
  const double2 d0 = m(V[0], sb(m(V[4], V[8]), m(V[5], V[7])));
  const double2 d1 = m(V[1], sb(m(V[5], V[6]), m(V[3], V[8])));
  const double2 d2 = m(V[2], sb(m(V[3], V[7]), m(V[4], V[6])));
  const double s = (d0.x + d1.x + d2.x) < 0.0 ? -1.0 : 1.0;
  double best = -1.0;
  int shift = 0;
  for (int j = 0; j < 3; j++) {
    const double a = V[j].x * V[j].x + V[j].y * V[j].y;
    if (a > best) { best = a; shift = j; }
  }
  double2 R[9];                               // R[i][k] = W[i][(k + shift) mod 3]
  for (int i = 0; i < 3; i++)
    for (int k = 0; k < 3; k++) {
      const double2 v = V[i * 3 + (k + shift) % 3];
      R[i * 3 + k] = make_double2(s * v.x, s * v.y);
    }
  const double b2n = R[3].x * R[3].x + R[3].y * R[3].y, c2n = R[6].x * R[6].x + R[6].y * R[6].y;
  const bool cstored = c2n < b2n;
  const double2 other = cstored ? R[3] : R[6], kept = cstored ? R[6] : R[3];
  const float pa = __uint_as_float((__float_as_uint((float)atan2(R[0].y, R[0].x)) & ~1u) | (cstored ? 1u : 0u));
  const float po = __uint_as_float((__float_as_uint((float)atan2(other.y, other.x)) & ~3u) | (unsigned)shift);
  float2 *f = reinterpret_cast<float2 *>(dst);
  const long base = (long)(blk * 4 + mu) * 4;
  f[(base + 0) * g.Vh + h] = make_float2(pa, po);
  f[(base + 1) * g.Vh + h] = make_float2((float)R[1].x, (float)R[1].y);
  f[(base + 2) * g.Vh + h] = make_float2((float)R[2].x, (float)R[2].y);
  f[(base + 3) * g.Vh + h] = make_float2((float)kept.x, (float)kept.y);
}

template <int CP>
__device__ __forceinline__ void cstore(void *base, float *cn, const float (&c)[72], int blk, int h, int Vh) {
  if (CP == ST_F32) {
    float4 *f = reinterpret_cast<float4 *>(base);
    for (int w = 0; w < 18; w++)
      f[(long)(blk * 18 + w) * Vh + h] = make_float4(c[4 * w], c[4 * w + 1], c[4 * w + 2], c[4 * w + 3]);
  } else if (CP == ST_F16) {
    uint4 *f = reinterpret_cast<uint4 *>(base);
    for (int w = 0; w < 9; w++) {
      uint4 v;
      v.x = f2h(make_float2(c[8 * w], c[8 * w + 1]));
      v.y = f2h(make_float2(c[8 * w + 2], c[8 * w + 3]));
      v.z = f2h(make_float2(c[8 * w + 4], c[8 * w + 5]));
      v.w = f2h(make_float2(c[8 * w + 6], c[8 * w + 7]));
      f[(long)(blk * 9 + w) * Vh + h] = v;
    }
  } else {
    float m = 0.f;
    for (int k = 0; k < 72; k++) m = fmaxf(m, fabsf(c[k]));
    const float inv = m > 0.f ? 1.f / m : 0.f;
    uint4 *f = reinterpret_cast<uint4 *>(base);
    for (int w = 0; w < 9; w++) {
      uint4 v;
      v.x = f2s(c[8 * w] * inv, c[8 * w + 1] * inv);
      v.y = f2s(c[8 * w + 2] * inv, c[8 * w + 3] * inv);
      v.z = f2s(c[8 * w + 4] * inv, c[8 * w + 5] * inv);
      v.w = f2s(c[8 * w + 6] * inv, c[8 * w + 7] * inv);
      f[(long)(blk * 9 + w) * Vh + h] = v;
    }
    cn[(long)blk * Vh + h] = m;
  }
}

// pack a Hermitian 6x6 block (full matrix M in double2) into 36 reals at c
__device__ __forceinline__ void pack_block(float *c, const double2 (&M)[36]) {
  for (int i = 0; i < 6; i++) c[i] = (float)M[i * 6 + i].x;
  int k = 6;
  for (int i = 1; i < 6; i++)
    for (int j = 0; j < i; j++, k += 2) {
      c[k] = (float)M[i * 6 + j].x;
      c[k + 1] = (float)M[i * 6 + j].y;
    }
}

// even sites: M_e = diag + [[A0,A1],[A1^dag,-A0]] (+) [[A2,A3],[A3^dag,-A2]] (clover_kernel,
// dirac.cpp:25-107) with diag = 4+m+cf(t); without a clover term, diag = (4+m)^2 alone
template <int CP>
__global__ void k_pack_clover_even(void *dst, float *cn, const double2 *cl, Geom g, double diag, double cfm1,
                                   int clover) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= g.Vh) return;
  int id = h;
  int c4[4];
  coords_of(g, id, c4);
  double dg = diag + ((clover && (c4[0] == g.Ta || c4[0] == g.Tb)) ? cfm1 : 0.0);
  float c[72];
  for (int b = 0; b < 2; b++) {
    double2 M[36];
    for (int k = 0; k < 36; k++) M[k] = make_double2(0, 0);
    for (int i = 0; i < 6; i++) M[i * 6 + i].x = dg;
    if (clover) {
      int m0 = 2 * b, m1 = 2 * b + 1;
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          double2 a0 = cl[fidx(g, id, m0 * 9 + i * 3 + j, 36)];
          double2 a1 = cl[fidx(g, id, m1 * 9 + i * 3 + j, 36)];
          M[i * 6 + j] = cadd(M[i * 6 + j], a0);
          M[(i + 3) * 6 + (j + 3)] = csub(M[(i + 3) * 6 + (j + 3)], a0);
          M[i * 6 + (j + 3)] = a1;
          M[(j + 3) * 6 + i] = cconj(a1);
        }
    }
    pack_block(c + 36 * b, M);
  }
  cstore<CP>(dst, cn, c, 0, h, g.Vh);
}

// odd sites: the explicit inverse M_o^-1 from the FP64 LDL factors (identity without clover)
template <int CP>
__global__ void k_pack_clover_odd(void *dst, float *cn, const double2 *ldl, Geom g, int clover) {
  int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= g.Vh) return;
  constexpr int N = 6, Pk = 21;
  float c[72];
  for (int b = 0; b < 2; b++) {
    double2 M[36];
    for (int k = 0; k < 36; k++) M[k] = make_double2(0, 0);
    if (!clover) {
      for (int i = 0; i < 6; i++) M[i * 6 + i].x = 1.0;
    } else {
      const double2 *Lb = ldl + (long)b * Pk * g.Vh + h;
      for (int col = 0; col < N; col++) {
        double2 x[N];
        for (int i = 0; i < N; i++) x[i] = make_double2(i == col ? 1.0 : 0.0, 0.0);
        for (int i = 1; i < N; i++)
          for (int k = 0; k < i; k++) x[i] = csub(x[i], cmul(Lb[(long)(i * (i + 1) / 2 + k) * g.Vh], x[k]));
        for (int i = N - 1; i >= 0; i--) {
          x[i] = cscale(x[i], 1.0 / Lb[(long)(i * (i + 1) / 2 + i) * g.Vh].x);
          for (int k = i + 1; k < N; k++) x[i] = csub(x[i], cmulc(Lb[(long)(k * (k + 1) / 2 + i) * g.Vh], x[k]));
        }
        for (int i = 0; i < N; i++) M[i * 6 + col] = x[i];
      }
    }
    pack_block(c + 36 * b, M);
  }
  cstore<CP>(dst, cn, c, 1, h, g.Vh);
}

// ------------------------------------------------------------------ sloppy vector kernels
// FP32 vectors x, r use the FP64 field order (complex k = spin*3+colour at [k*Vh + h],
// even block); sloppy vectors p, q use the formats above.

// sloppy <- FP64 block 0 (even sites)
template <int P>
__global__ void __launch_bounds__(256) k_s_from_d(void *dst, float *dn, const double2 *src, int Vh) {
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += gridDim.x * blockDim.x) {
    float2 s[12];
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double2 v = src[(long)k * Vh + h];
      s[k] = make_float2((float)v.x, (float)v.y);
    }
    sstore<P>(dst, dn, s, 0, h, Vh);
  }
}

// |r|^2 from the update's partials, beta = |r|^2 / |r_old|^2, x += alpha p, p = r + beta p
// (x and p in one pass: the p it reads is the direction of this iteration); block 0
// stores |r|^2 for the next iteration and into *hist, then counts the iteration (S_ITER)
// and stores the count into *seq (hist and seq are mapped host memory, which the host polls
// one iteration later).  Nothing in the arguments changes between iterations of the same
// parity, so an iteration can be replayed as a CUDA graph.
template <int P>
__global__ void __launch_bounds__(256) k_s_xpay(void *p, float *pn, double *scal, const double *part_r, int n_r,
                                                int par, double *hist, unsigned long long *seq, const float2 *r,
                                                float2 *x, int Vh) {
  griddep_wait();
  const double rr = sum_partials(part_r, n_r);
  const float b = (float)(rr / scal[S_RR0 + par]);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    scal[S_RR0 + (par ^ 1)] = rr;
    const double done = scal[S_ITER] + 1.0;
    scal[S_ITER] = done;
    *reinterpret_cast<volatile double *>(hist) = rr;
    __threadfence_system();
    *reinterpret_cast<volatile unsigned long long *>(seq) = (unsigned long long)done;
  }
  const float al = (float)scal[S_ALPHA];
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += gridDim.x * blockDim.x) {
    float2 pp[12];
    sload<P>(pp, p, pn, 0, h, Vh);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const long i = (long)k * Vh + h;
      const float2 ri = r[i];
      float2 xi = x[i];
      xi.x = fmaf(al, pp[k].x, xi.x);                 // x += alpha p with the p of this iteration
      xi.y = fmaf(al, pp[k].y, xi.y);
      x[i] = xi;
      pp[k] = make_float2(fmaf(b, pp[k].x, ri.x), fmaf(b, pp[k].y, ri.y));
    }
    sstore<P>(p, pn, pp, 0, h, Vh);
  }
  griddep_launch();
}

__global__ void k_s_set(double *scal, int i, double v) { scal[i] = v; }

// ------------------------------------------------------------------ host side
// sloppy fields live in the lattice's scratch fields (each one FP64 field in size, which
// holds a sloppy spinor plus its norms: FP32 96 B/site, FP16 48 + 4 B/site)
struct SField {
  void *data;
  float *norm;
};

static SField sfield(Lattice &L, int slot) {
  char *base = reinterpret_cast<char *>(L.scratch_field(slot));
  SField f;
  f.data = base;
  f.norm = reinterpret_cast<float *>(base + (size_t)L.V * 96);   // after the largest (FP32) payload
  return f;
}

static int sgrid(long n) {
  long g = (n + 255) / 256;
  const long cap = 148 * 16;
  return (int)(g < cap ? g : cap);
}

// run-time storage formats -> template arguments: SP spinor, SL links, SC clover, SK complex
// words stored per link.  The combinations built: FP32 throughout; FP32 spinors with int16
// links (and FP32 or int16 clover); FP16 spinors with FP32, FP16 or int16 matrices.
#define YG_SLOPPY_ONE(P_, L_, C_, ...)                                                        \
  if (prec_ == P_ && lf_ == L_ && cf_ == C_) {                                               \
    constexpr int SP = P_, SL = L_, SC = C_;                                                 \
    if (reals_ == 12) { constexpr int SK = 6; __VA_ARGS__; }                                 \
    else if (reals_ == 8) {                                                                  \
      if constexpr (L_ == 32) { constexpr int SK = 4; __VA_ARGS__; }                         \
    }                                                                                        \
    else { constexpr int SK = 9; __VA_ARGS__; }                                              \
    done_ = true;                                                                            \
  }
#define YG_SLOPPY_DISPATCH(PREC, LF, CF, REALS, ...)                                           \
  do {                                                                                       \
    const int prec_ = (PREC), lf_ = (LF), cf_ = (CF), reals_ = (REALS);                      \
    bool done_ = false;                                                                      \
    YG_SLOPPY_ONE(32, 32, 32, __VA_ARGS__)                                                   \
    else YG_SLOPPY_ONE(32, 15, 32, __VA_ARGS__)                                              \
    else YG_SLOPPY_ONE(32, 15, 15, __VA_ARGS__)                                              \
    else YG_SLOPPY_ONE(16, 16, 16, __VA_ARGS__)                                              \
    else YG_SLOPPY_ONE(16, 32, 32, __VA_ARGS__)                                              \
    else YG_SLOPPY_ONE(16, 15, 15, __VA_ARGS__)                                              \
    if (!done_) throw Error(YG_ERR_ARG, "unsupported combination of inner storage formats");  \
  } while (0)

// spinor format only (the inner CG's vector kernels)
#define YG_SPINOR_DISPATCH(PREC, ...)                                                         \
  do {                                                                                       \
    if ((PREC) == 32) { constexpr int SP = 32; __VA_ARGS__; }                                \
    else if ((PREC) == 16) { constexpr int SP = 16; __VA_ARGS__; }                           \
    else throw Error(YG_ERR_ARG, "inner precision must be 32 or 16");                         \
  } while (0)

// 0 (automatic) -> the spinor format; 15 is the int16 fixed-point format
static int matrix_format(int requested, int prec) { return requested == 0 ? prec : requested; }

void ensure_sloppy(Lattice &L, double mass, int prec, int reals, int lfmt, int cfmt) {
  lfmt = matrix_format(lfmt, prec);
  cfmt = matrix_format(cfmt, prec);
  if ((prec != 32 && prec != 16) || (reals != 18 && reals != 12 && reals != 8))
    throw Error(YG_ERR_ARG, "inner precision must be 32 or 16 and link reals 18, 12 or 8");
  if (reals == 8 && matrix_format(lfmt, prec) != ST_F32)
    throw Error(YG_ERR_ARG, "8-real links are stored FP32");
  if (reals == 8 && L.p.bc != YG_BC_PERIODIC && L.p.bc != YG_BC_ANTIPERIODIC)
    throw Error(YG_ERR_ARG, "8-real links need periodic or antiperiodic boundaries (open and SF boundary links are "
                            "not of the parametrised form)");
  for (int f : {lfmt, cfmt})
    if (f != ST_F32 && f != ST_F16 && f != ST_I16) throw Error(YG_ERR_ARG, "matrix storage must be 32, 16 or 15");
  if (L.d != 3) throw Error(YG_ERR_ARG, "the compressed inner operator exists for d = 3 representations");
  if (reals != 18 && !(L.nc == 3 && L.p.repr == YG_REPR_FUNDAMENTAL))
    throw Error(YG_ERR_ARG, "12- and 8-real links need SU(3) fundamental links");
  if (!L.p.eo) throw Error(YG_ERR_ARG, "the mixed-precision solver needs even-odd preconditioning");
  if (!L.sl_hist) {
    // mapped host words: [0], [1] the |r|^2 of the last two iterations, [4] their counter
    YG_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&L.sl_hist), 8 * sizeof(double), cudaHostAllocMapped));
    L.sl_scal.alloc(S_WORDS * sizeof(double));
    YG_CUDA(cudaMemsetAsync(L.sl_scal.p, 0, S_WORDS * sizeof(double), L.stream));
  }
  if (L.sl_valid && L.sl_prec == prec && L.sl_reals == reals && L.sl_lfmt == lfmt && L.sl_cfmt == cfmt &&
      L.sl_mass == mass)
    return;
  {
    // resident-grid sizes of the reduction kernels, and room for their partials
    int dev = 0, sms = 0, per_vec = 0;
    int per_nrm[kStep2Shapes] = {0, 0, 0}, per_cg[kStep2Shapes] = {0, 0, 0};
    YG_CUDA(cudaGetDevice(&dev));
    YG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    YG_SLOPPY_DISPATCH(prec, lfmt, cfmt, reals, {
      YG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_nrm[0], k_shop<SP, SL, SC, SK, 2, 1>, 128, 0));
      YG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_cg[0], k_shop_cg<SP, SL, SC, SK>, 128, 0));
      if constexpr (SP == 16 && SL == 32 && SC == 32) {
        YG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_nrm[1], k_shop_nrm_min<SP, SL, SC, SK, 5>, 128, 0));
        YG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_nrm[2], k_shop_nrm_min<SP, SL, SC, SK, 6>, 128, 0));
        YG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_cg[1], k_shop_cg_min<SP, SL, SC, SK, 5>, 128, 0));
        YG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_cg[2], k_shop_cg_min<SP, SL, SC, SK, 6>, 128, 0));
      }
      YG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_vec, k_s_xpay<SP>, 256, 0));
    });
    int gmax = 0;
    for (int v = 0; v < kStep2Shapes; v++) {
      L.sl_gnrm[v] = (int)std::min<long>((long)sms * std::max(per_nrm[v], 1), nblk(L.Vh, 128));
      L.sl_gcg[v] = (int)std::min<long>((long)sms * std::max(per_cg[v], 1), nblk(L.Vh, 128));
      gmax = std::max({gmax, L.sl_gnrm[v], L.sl_gcg[v]});
    }
    L.sl_grid_vec = (int)std::min<long>((long)sms * std::max(per_vec, 1), nblk(L.Vh, 256));
    L.sl_part_off = gmax;
    L.sl_part.alloc(sizeof(double) * (size_t)(2 * gmax));
  }
  const int K = reals / 2;
  L.sl_links.alloc((lfmt == ST_F32 ? 8 : 4) * (size_t)K * 4 * L.V);
  L.sl_clover.alloc((cfmt == ST_F32 ? 4 : 2) * 72 * (size_t)L.V);
  L.sl_cnorm.alloc(sizeof(float) * (size_t)L.V);
  if (L.p.clover) ensure_ldl(L, 4.0 + mass);
  int clover = L.p.clover ? 1 : 0;
  double diag = clover ? 4.0 + mass : (4.0 + mass) * (4.0 + mass);
  YG_SLOPPY_DISPATCH(prec, lfmt, cfmt, reals, {
    k_pack_links<SL, SK><<<nblk(4 * L.V, 128), 128, 0, L.stream>>>(L.sl_links.p, L.links.as<double2>(), L.g);
    YG_LAUNCHED();
    k_pack_clover_even<SC><<<nblk(L.Vh, 64), 64, 0, L.stream>>>(L.sl_clover.p, L.sl_cnorm.as<float>(),
                                                                 L.clover.as<double2>(), L.g, diag, L.p.cf - 1.0,
                                                                 clover);
    YG_LAUNCHED();
    k_pack_clover_odd<SC><<<nblk(L.Vh, 64), 64, 0, L.stream>>>(L.sl_clover.p, L.sl_cnorm.as<float>(),
                                                                L.ldl.as<double2>(), L.g, clover);
    YG_LAUNCHED();
  });
  L.sl_prec = prec;
  L.sl_reals = reals;
  L.sl_lfmt = lfmt;
  L.sl_cfmt = cfmt;
  L.sl_mass = mass;
  L.sl_valid = true;
}

// FP32 packed clover blocks of another mass (M_e = (4+m+cf) + A on even sites, M_o^-1 on odd
// sites; without a clover term 1 and (4+m)^2) into dst, for inner operators that carry one
// block set per system.  cn receives the per-site norms of the packing (unused for FP32).
void pack_clover_f32(Lattice &L, double mass, void *dst, float *cn) {
  if (L.p.clover) ensure_ldl(L, 4.0 + mass);
  const int clover = L.p.clover ? 1 : 0;
  const double diag = clover ? 4.0 + mass : (4.0 + mass) * (4.0 + mass);
  k_pack_clover_even<ST_F32><<<nblk(L.Vh, 64), 64, 0, L.stream>>>(dst, cn, L.clover.as<double2>(), L.g, diag,
                                                                   L.p.cf - 1.0, clover);
  YG_LAUNCHED();
  k_pack_clover_odd<ST_F32><<<nblk(L.Vh, 64), 64, 0, L.stream>>>(dst, cn, L.ldl.as<double2>(), L.g, clover);
  YG_LAUNCHED();
}

// launch with programmatic stream serialisation (the kernel waits for its predecessor
// itself, griddep_wait)
template <typename... KArgs, typename... Args>
static void launch_pdl(void (*kern)(KArgs...), int grid, int block, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  YG_CUDA(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...));
}

// Block shapes of the step-1 hop the tuner chooses among (threads per block, resident blocks
// per SM the registers are cut for; 0 = the compiler's own choice): the default, 128-thread
// blocks cut for 6 per SM, 256-thread blocks cut for 3, 64-thread blocks cut for 10.  Only the
// default storage (FP16 spinors, FP32 matrices) has the variants; other formats always use
// the first.
constexpr int kShapes[4][2] = {{128, 0}, {128, 6}, {256, 3}, {64, 10}};
// the step-2 kernels (resident grids) tried with the compiler's registers, and cut for 5 and 6
// resident blocks per SM
constexpr int kStep2Min[kStep2Shapes] = {0, 5, 6};

template <int SP, int SL, int SC, int SK>
static void launch_step1(int shape, cudaStream_t s, const SHopArgs &a) {
  if constexpr (SP == 16 && SL == 32 && SC == 32) {
    switch (shape) {
      case 1: launch_pdl(k_shop_shaped<SP, SL, SC, SK, 128, 6>, nblk(a.n, 128), 128, s, a); return;
      case 2: launch_pdl(k_shop_shaped<SP, SL, SC, SK, 256, 3>, nblk(a.n, 256), 256, s, a); return;
      case 3: launch_pdl(k_shop_shaped<SP, SL, SC, SK, 64, 10>, nblk(a.n, 64), 64, s, a); return;
      default: break;
    }
  }
  launch_pdl(k_shop<SP, SL, SC, SK, 1, 0>, nblk(a.n, 128), 128, s, a);
}

static double *dscal(Lattice &L) { return L.sl_scal.as<double>(); }
static unsigned long long *hist_seq(Lattice &L) { return reinterpret_cast<unsigned long long *>(L.sl_hist + 4); }
static double *part_pq(Lattice &L) { return L.sl_part.as<double>(); }
static double *part_r(Lattice &L) { return L.sl_part.as<double>() + L.sl_part_off; }

// the step-2 shapes in use: the tuned ones for the default storage, the compiler's otherwise
static bool default_storage(const Lattice &L) { return L.sl_prec == 16 && L.sl_lfmt == ST_F32 && L.sl_cfmt == ST_F32; }
static int shape_nrm(const Lattice &L) { return default_storage(L) ? L.sl_shape_n : 0; }
static int shape_cg(const Lattice &L) { return default_storage(L) ? L.sl_shape_c : 0; }

// dst = Hphi(src) with the compressed operator; tmp receives the odd-site intermediate.
// nrm: also the partials of |dst|^2 = <p, A p> (the first Hphi of a CG iteration)
static void sloppy_hphi(Lattice &L, SField dst, SField src, SField tmp, bool nrm) {
  SHopArgs a{};
  a.g = L.g;
  a.U = L.sl_links.p;
  a.C = L.sl_clover.p;
  a.Cn = L.sl_cnorm.as<float>();
  a.src = src.data; a.src_norm = src.norm;
  a.dst = tmp.data; a.dst_norm = tmp.norm;
  a.coeff = 0.5f;
  a.lo = (int)L.Vh; a.n = (int)L.Vh;
  SHopArgs b = a;
  b.src = tmp.data; b.src_norm = tmp.norm;
  b.src2 = src.data; b.src2_norm = src.norm;
  b.dst = dst.data; b.dst_norm = dst.norm;
  b.coeff = -0.5f;
  b.lo = 0;
  b.part = part_pq(L);
  YG_SLOPPY_DISPATCH(L.sl_prec, L.sl_lfmt, L.sl_cfmt, L.sl_reals, {
    launch_step1<SP, SL, SC, SK>(L.sl_shape, L.stream, a);
    YG_LAUNCHED();
    if (nrm) {
      const int v = shape_nrm(L);
      const int grid = L.sl_gnrm[v];
      if constexpr (SP == 16 && SL == 32 && SC == 32) {
        if (v == 1) launch_pdl(k_shop_nrm_min<SP, SL, SC, SK, 5>, grid, 128, L.stream, b);
        else if (v == 2) launch_pdl(k_shop_nrm_min<SP, SL, SC, SK, 6>, grid, 128, L.stream, b);
        else launch_pdl(k_shop<SP, SL, SC, SK, 2, 1>, grid, 128, L.stream, b);
      } else {
        launch_pdl(k_shop<SP, SL, SC, SK, 2, 1>, grid, 128, L.stream, b);
      }
    } else {
      launch_pdl(k_shop<SP, SL, SC, SK, 2, 0>, nblk(b.n, 128), 128, L.stream, b);
    }
    YG_LAUNCHED();
  });
  L.mvm += 2;
}

// q = Hphi(t) with the residual update fused into its last step: r -= alpha q and the
// partials of the new |r|^2 (par = iteration parity, selecting the |r|^2 slot)
static void sloppy_hphi_cg(Lattice &L, SField t, SField tmp, float *r, int par) {
  SHopArgs a{};
  a.g = L.g;
  a.U = L.sl_links.p;
  a.C = L.sl_clover.p;
  a.Cn = L.sl_cnorm.as<float>();
  a.src = t.data; a.src_norm = t.norm;
  a.dst = tmp.data; a.dst_norm = tmp.norm;
  a.coeff = 0.5f;
  a.lo = (int)L.Vh; a.n = (int)L.Vh;
  SHopArgs b = a;
  b.src = tmp.data; b.src_norm = tmp.norm;
  b.src2 = t.data; b.src2_norm = t.norm;
  b.dst = nullptr; b.dst_norm = nullptr;
  b.coeff = -0.5f;
  b.lo = 0;
  SCgArgs c{};
  c.r = reinterpret_cast<float2 *>(r);
  c.scal = dscal(L);
  c.part_pq = part_pq(L);
  c.n_pq = L.sl_gnrm[shape_nrm(L)];
  c.part_r = part_r(L);
  c.par = par;
  YG_SLOPPY_DISPATCH(L.sl_prec, L.sl_lfmt, L.sl_cfmt, L.sl_reals, {
    launch_step1<SP, SL, SC, SK>(L.sl_shape, L.stream, a);
    YG_LAUNCHED();
    const int v = shape_cg(L);
    const int grid = L.sl_gcg[v];
    if constexpr (SP == 16 && SL == 32 && SC == 32) {
      if (v == 1) launch_pdl(k_shop_cg_min<SP, SL, SC, SK, 5>, grid, 128, L.stream, b, c);
      else if (v == 2) launch_pdl(k_shop_cg_min<SP, SL, SC, SK, 6>, grid, 128, L.stream, b, c);
      else launch_pdl(k_shop_cg<SP, SL, SC, SK>, grid, 128, L.stream, b, c);
    } else {
      launch_pdl(k_shop_cg<SP, SL, SC, SK>, grid, 128, L.stream, b, c);
    }
    YG_LAUNCHED();
  });
  L.mvm += 2;
}

static void sloppy_xpay(Lattice &L, SField p, const float *r, float *x, int par, double *hist) {
  YG_SPINOR_DISPATCH(L.sl_prec, {
    launch_pdl(k_s_xpay<SP>, L.sl_grid_vec, 256, L.stream, p.data, p.norm, dscal(L), part_r(L), L.sl_gcg[shape_cg(L)],
               par,
               hist, hist_seq(L), (const float2 *)r, (float2 *)x, (int)L.Vh);
    YG_LAUNCHED();
  });
}

// wait until the GPU has finished inner iteration `iter` (its xpay wrote the counter);
// a GPU error or a counter that stops advancing for 30 s ends the wait with an error
static void wait_iteration(Lattice &L, unsigned long long iter) {
  volatile unsigned long long *seq = hist_seq(L);
  if (*seq >= iter) return;
  auto t0 = std::chrono::steady_clock::now();
  while (*seq < iter) {
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (dt > 1e-3) std::this_thread::yield();
    if (dt > 30.0) {
      YG_CUDA(cudaStreamSynchronize(L.stream));
      if (*seq < iter) throw Error(YG_TIMEOUT, "cg_mixed: the inner iteration counter stopped advancing");
      return;
    }
  }
}

static void sloppy_from_d(Lattice &L, SField dst, const double *src) {
  YG_SPINOR_DISPATCH(L.sl_prec, {
    k_s_from_d<SP><<<sgrid(L.Vh), 256, 0, L.stream>>>(dst.data, dst.norm, (const double2 *)src, (int)L.Vh);
    YG_LAUNCHED();
  });
}

static void set_scalar(Lattice &L, int i, double v) {
  k_s_set<<<1, 1, 0, L.stream>>>(dscal(L), i, v);
  YG_LAUNCHED();
}

// CUDA graphs of the inner iteration (YG_CUDA_GRAPH=0 turns them off)
static bool use_graphs() {
  const char *e = std::getenv("YG_CUDA_GRAPH");
  return !(e && e[0] == '0');
}

// The two parities of the inner iteration as instantiated graphs.  Capture records the
// launches without running them: the launch counter and the MVM counter are restored after
// the capture and advanced at every replay instead.  A capture that fails (a driver that
// cannot record a launch form) is ended and discarded, and the solver issues the launches
// one by one as without graphs.
struct IterGraphs {
  cudaGraphExec_t exec[2] = {nullptr, nullptr};
  long launches[2] = {0, 0};
  int mvm[2] = {0, 0};
  bool failed = false;
  bool ready() const { return !failed && exec[0] && exec[1]; }
  template <typename F>
  void capture(Lattice &L, int par, F &&issue) {
    if (failed) return;
    const long n0 = g_launch_count.load();
    const int m0 = L.mvm;
    cudaGraph_t g = nullptr;
    bool ok = cudaStreamBeginCapture(L.stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      try {
        issue();
      } catch (const Error &) {
        ok = false;
      }
      ok = (cudaStreamEndCapture(L.stream, &g) == cudaSuccess) && ok && g;
    }
    launches[par] = g_launch_count.load() - n0;
    g_launch_count -= launches[par];
    mvm[par] = L.mvm - m0;
    L.mvm = m0;
    if (ok) ok = cudaGraphInstantiate(&exec[par], g, 0) == cudaSuccess;
    if (g) cudaGraphDestroy(g);
    if (!ok) {
      failed = true;
      (void)cudaGetLastError();              // the failed capture's error is not sticky
    }
  }
  void launch(Lattice &L, int par) {
    YG_CUDA(cudaGraphLaunch(exec[par], L.stream));
    g_launch_count += launches[par];
    L.mvm += mvm[par];
  }
  ~IterGraphs() {
    for (cudaGraphExec_t &e : exec)
      if (e) cudaGraphExecDestroy(e);
  }
};

// Mixed-precision CG on Hphi_sq with the compressed inner operator.  x and r of the inner
// iterations are FP32, p and Hphi p are in the inner storage format, A p = Hphi Hphi p stays
// in registers: the r update is the epilogue of the operator's last step, the x update rides
// with p = r + beta p.  alpha and beta live on the device, so an inner iteration is five
// launches (four operator steps and x += alpha p, p = r + beta p), replayed as one CUDA graph
// per iteration, and no host synchronisation; the host
// reads each iteration's |r|^2 one iteration late (while the next one runs) and then
// decides on a reliable update: b - A x is recomputed with the FP64 operator whenever the
// iterated |r| fell below delta times its value at the last update, r is replaced by it
// and the search direction is kept.  The solve stops only on the true FP64 squared
// residual |b - A x|^2 < prec |b|^2; a stall falls back to the FP64 CG.
int cg_mixed_sloppy(Lattice &L, const yg_inv_par &par, int prec, int reals, int lfmt, int cfmt, double delta,
                    double *x, double *b, yg_solve_stats *st, bool escalate);

}  // namespace yg

namespace yg {

int cg(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters);

static void tune_shape(Lattice &L, double mass, int reals);

int cg_mixed_sloppy(Lattice &L, const yg_inv_par &par, int prec, int reals, int lfmt, int cfmt, double delta,
                    double *x, double *b, yg_solve_stats *st, bool escalate) {
  auto t0 = std::chrono::steady_clock::now();
  if (par.op != YG_OP_HPHI_SQ) throw Error(YG_ERR_ARG, "cg_mixed solves Hphi_sq systems");
  if (!(delta > 0.0 && delta < 1.0)) throw Error(YG_ERR_ARG, "reliable-update delta must lie in (0,1)");
  if (prec == 16 && matrix_format(lfmt, prec) == ST_F32 && matrix_format(cfmt, prec) == ST_F32 && reals != 8)
    tune_shape(L, par.mass, reals);         // the block shape of the step-1 hop, once per lattice
  ensure_sloppy(L, par.mass, prec, reals, lfmt, cfmt);
  long lo, n;
  L.view_range(YG_VIEW_DEFAULT, lo, n);
  const long cnt = n * 4L * L.d;
  double *r = L.scratch_field(3), *Ax = L.scratch_field(4), *xd = L.scratch_field(5);
  float *fr = reinterpret_cast<float *>(L.scratch_field(40));
  float *fx = reinterpret_cast<float *>(L.scratch_field(42));
  SField p = sfield(L, 41), t = sfield(L, 44), o = sfield(L, 45);
  volatile double *hist = L.sl_hist;
  *hist_seq(L) = 0;                 // no GPU work of this lattice is in flight here
  set_scalar(L, S_ITER, 0.0);       // the device's count of finished inner iterations

  auto residual = [&]() {           // r = b - A x in FP64, returns |r|^2
    blas_copy(L, xd, x);
    apply_op(L, YG_OP_HPHI_SQ, par.mass, Ax, xd);
    blas_copy(L, r, b);
    blas_axpby(L, r, make_double2(1, 0), make_double2(-1, 0), Ax, lo, n);
    return blas_sqnorm(L, r, lo, n);
  };

  double norm = blas_sqnorm(L, b, lo, n);
  double rr = residual();
  double target = norm * par.prec;
  int it = 0, updates = 0, status = YG_OK, stall = 0;
  double best = rr;
  double *xbest = L.scratch_field(46);      // the iterate with the smallest true residual
  blas_copy(L, xbest, x);

  // the inner CG from the current x until the true residual meets prec (YG_OK), maxiter,
  // or a stall / divergence of the true residual (YG_STALL)
  auto run_inner = [&]() -> int {
    f_from_d(L, fr, r, cnt);
    sloppy_from_d(L, p, r);
    YG_CUDA(cudaMemsetAsync(fx, 0, sizeof(float2) * cnt, L.stream));
    set_scalar(L, S_RR0 + (it & 1), rr);      // the slot the first iteration reads
    double maxrr = rr;
    const double d2 = delta * delta;
    bool pending = false;           // an enqueued iteration whose |r|^2 is still to be read
    // The iterated |r| of a low-precision inner solve levels off near the storage precision
    // times |r| at the last update; if it has not halved for kStagnate iterations a
    // reliable update is forced, so a delta below that floor cannot keep the loop going.
    constexpr int kStagnate = 100;
    double min_cycle = rr;
    int since_min = 0;
    stall = 0;
    // an inner iteration is the same five launches with the same arguments for every
    // iteration of one parity; with graphs on, each parity is captured once per inner run and
    // replayed as one CUDA graph launch
    IterGraphs graphs;
    if (use_graphs()) {
      for (int gp = 0; gp < 2; gp++)
        graphs.capture(L, gp, [&] {
          sloppy_hphi(L, t, p, o, true);
          sloppy_hphi_cg(L, t, o, fr, gp);
          sloppy_xpay(L, p, fr, fx, gp, const_cast<double *>(hist) + gp);
        });
    }
    while (true) {
      if (par.maxiter > 0 && it >= par.maxiter) {
        d_add_f(L, x, fx, cnt);     // keep the progress of the inner iterations
        return YG_MAXITER;
      }
      int slot = it & 1;
      if (graphs.ready()) {
        graphs.launch(L, slot);
      } else {
        sloppy_hphi(L, t, p, o, true);
        sloppy_hphi_cg(L, t, o, fr, slot);
        sloppy_xpay(L, p, fr, fx, slot, const_cast<double *>(hist) + slot);
      }
      it++;
      if (!pending) { pending = true; continue; }
      // the previous iteration's |r|^2, read while this one runs
      wait_iteration(L, (unsigned long long)it - 1);
      double rr_prev = hist[slot ^ 1];
      if (!std::isfinite(rr_prev)) throw Error(YG_NONFINITE, "non-finite value in cg_mixed");
      if (rr_prev < 0.25 * min_cycle) { min_cycle = rr_prev; since_min = 0; }
      else since_min++;
      if (rr_prev < d2 * maxrr || rr_prev < target || since_min >= kStagnate) {
        // reliable update on the state after the iteration just enqueued
        d_add_f(L, x, fx, cnt);
        YG_CUDA(cudaMemsetAsync(fx, 0, sizeof(float2) * cnt, L.stream));
        double rr_true = residual();
        updates++;
        rr = rr_true;
        if (rr_true < target) return YG_OK;
        if (rr_true < best) blas_copy(L, xbest, x);
        if (rr_true > 100.0 * best) return YG_STALL;               // the inner solve diverged
        if (rr_true < 0.5 * best) stall = 0;
        else if (++stall >= 8) return YG_STALL;
        best = std::min(best, rr_true);
        f_from_d(L, fr, r, cnt);
        set_scalar(L, S_RR0 + (it & 1), rr_true); // the slot the next iteration reads
        maxrr = rr_true;
        min_cycle = rr_true;
        since_min = 0;
        pending = false;            // the enqueued |r|^2 predates the update
      }
    }
  };

  int raised = 0;
  if (rr >= target) {
    status = run_inner();
    if (status == YG_STALL && escalate && prec == 16) {
      // FP16 spinors (or matrices) too coarse for this system: restart the inner CG with
      // FP32 storage from the best iterate before handing over to the FP64 CG
      raised = 1;
      ensure_sloppy(L, par.mass, 32, reals, 32, 32);
      blas_copy(L, x, xbest);
      rr = residual();
      status = rr < target ? YG_OK : run_inner();
    }
  }
  int fallback = raised ? 2 : 0;
  if (status != YG_OK) {
    // plain FP64 CG (the reference's solver) from the best iterate; its recursive residual
    // can stop above the true one, so it restarts until the true residual meets prec
    blas_copy(L, x, xbest);
    yg_inv_par p64 = par;
    p64.log = 0;
    fallback |= 1;
    for (int attempt = 0; attempt < 3; attempt++) {
      int it64 = 0;
      status = cg(L, p64, x, b, &it64);
      it += it64;
      rr = residual();
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
  if (par.log)
    fprintf(stderr, "[INVERTER][30]cg_mixed(fp%d, %d-real): iterations = %d, precision = %1.4e\n", prec, reals, it,
            rr / norm);
  return status;
}

// Measurement support: mean time of `reps` launches of step 1 of the compressed inner
// operator (the kernel that dominates cg_mixed) with the solver's default storage, timed
// with CUDA events on the lattice's stream, and the compulsory bytes one launch moves
// (neighbour spinors read once, links, clover blocks, output spinor).
// mean time of the inner operator's step-1 hop (FP16 spinors, FP32 matrices, `reals` per link)
// in block shape `shape`
static void hop_time(Lattice &L, double mass, int reals, int reps, double *ms, double *bytes, int shape) {
  if (reps < 1) throw Error(YG_ERR_ARG, "reps must be >= 1");
  ensure_sloppy(L, mass, 16, reals, 32, 32);
  SField src = sfield(L, 41), dst = sfield(L, 44);
  sloppy_from_d(L, src, L.scratch_field(3));
  SHopArgs a{};
  a.g = L.g;
  a.U = L.sl_links.p;
  a.C = L.sl_clover.p;
  a.Cn = L.sl_cnorm.as<float>();
  a.src = src.data; a.src_norm = src.norm;
  a.dst = dst.data; a.dst_norm = dst.norm;
  a.coeff = 0.5f;
  a.lo = (int)L.Vh; a.n = (int)L.Vh;
  cudaEvent_t e0, e1;
  YG_CUDA(cudaEventCreate(&e0));
  YG_CUDA(cudaEventCreate(&e1));
  YG_SLOPPY_DISPATCH(L.sl_prec, L.sl_lfmt, L.sl_cfmt, L.sl_reals, {
    for (int w = 0; w < 3; w++) launch_step1<SP, SL, SC, SK>(shape, L.stream, a);
    YG_CUDA(cudaEventRecord(e0, L.stream));
    for (int r = 0; r < reps; r++) launch_step1<SP, SL, SC, SK>(shape, L.stream, a);
    YG_CUDA(cudaEventRecord(e1, L.stream));
    for (int r = 0; r < reps + 3; r++) YG_LAUNCHED();
  });
  YG_CUDA(cudaEventSynchronize(e1));
  float t = 0.f;
  YG_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / reps;
  const double spinor = L.sl_prec == 16 ? 52.0 : 96.0;
  const double link = (reals / 2) * (L.sl_lfmt == ST_F32 ? 8.0 : 4.0);
  const double clov = 72.0 * (L.sl_cfmt == ST_F32 ? 4.0 : 2.0) + (L.sl_cfmt == ST_I16 ? 4.0 : 0.0);
  *bytes = (double)L.Vh * (spinor + 8.0 * link + clov + spinor);
}

// The block shapes of the inner operator for FP16 spinors, FP32 matrices and `reals` link
// reals: each step-1 shape of kShapes timed over 20 hops on this lattice, then each register
// variant of the two step-2 kernels; the fastest of each kept (once per lattice and link
// format).  YG_TUNE_LOG prints the timings.
static void tune_shape(Lattice &L, double mass, int reals) {
  if (L.sl_shape_reals == reals) return;
  L.sl_shape_n = L.sl_shape_c = 0;
  int shape = 0;
  double best_ms = 0.0;
  for (int v = 0; v < 4; v++) {
    double t = 0.0, bytes = 0.0;
    hop_time(L, mass, reals, 20, &t, &bytes, v);
    if (v == 0 || t < best_ms) { best_ms = t; shape = v; }
    if (std::getenv("YG_TUNE_LOG"))
      fprintf(stderr, "yg tune inner hop: %d-real links, %d threads/block, %d blocks/SM: %.4f ms\n", reals,
              kShapes[v][0], kShapes[v][1], t);
  }
  L.sl_shape = shape;
  // the register variants of the two step-2 kernels, each timed over 10 Hphi applications on
  // the solver's own scratch fields (which the solve rewrites before it reads them)
  const int mvm0 = L.mvm;
  SField p = sfield(L, 41), t = sfield(L, 44), o = sfield(L, 45);
  float *fr = reinterpret_cast<float *>(L.scratch_field(40));
  sloppy_from_d(L, p, L.scratch_field(3));
  set_scalar(L, S_RR0, 1.0);
  cudaEvent_t e0, e1;
  YG_CUDA(cudaEventCreate(&e0));
  YG_CUDA(cudaEventCreate(&e1));
  auto timed = [&](auto &&fn) {
    fn();
    YG_CUDA(cudaEventRecord(e0, L.stream));
    for (int r = 0; r < 10; r++) fn();
    YG_CUDA(cudaEventRecord(e1, L.stream));
    YG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    YG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    return ms / 10.f;
  };
  float best_n = 0.f, best_c = 0.f;
  int vn = 0, vc = 0;
  for (int v = 0; v < kStep2Shapes; v++) {
    L.sl_shape_n = v;
    const float ms = timed([&] { sloppy_hphi(L, t, p, o, true); });
    if (v == 0 || ms < best_n) { best_n = ms; vn = v; }
    if (std::getenv("YG_TUNE_LOG"))
      fprintf(stderr, "yg tune inner Hphi with <p,Ap>: step 2 cut for %d blocks/SM: %.4f ms\n", kStep2Min[v], ms);
  }
  L.sl_shape_n = vn;
  sloppy_hphi(L, t, p, o, true);            // the <p, A p> partials the update kernel reads
  for (int v = 0; v < kStep2Shapes; v++) {
    L.sl_shape_c = v;
    const float ms = timed([&] { sloppy_hphi_cg(L, t, o, fr, 0); });
    if (v == 0 || ms < best_c) { best_c = ms; vc = v; }
    if (std::getenv("YG_TUNE_LOG"))
      fprintf(stderr, "yg tune inner Hphi with the CG update: step 2 cut for %d blocks/SM: %.4f ms\n", kStep2Min[v],
              ms);
  }
  L.sl_shape_c = vc;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  L.mvm = mvm0;
  L.sl_shape_reals = reals;
}

// the step-1 hop of the default solve in the lattice's tuned block shape
void inner_hop_profile(Lattice &L, double mass, int reps, double *ms, double *bytes) {
  const int reals = L.sl_tuned_reals ? L.sl_tuned_reals : (L.nc == 3 && L.p.repr == YG_REPR_FUNDAMENTAL) ? 12 : 18;
  hop_time(L, mass, reals, reps, ms, bytes, L.sl_shape);
}

// No reference counterpart: the link format and block shape of the default mixed solve chosen
// by measurement.  The link candidates carry FP32 matrices (the formats whose rounding leaves
// the operator accurate enough on rough fields): 18 reals always, 12 for SU(3) fundamental
// links, 8 in addition on periodic / antiperiodic lattices.  Each is timed over 20 step-1 hops
// on this lattice in the default block shape; then the fastest format is timed in every block
// shape of kShapes.  Both choices are kept for the lattice (ms[0..2] = 18, 12, 8 real, 0 where
// not a candidate).  YG_TUNE_LOG prints the block-shape timings.
int tune_inner_links(Lattice &L, double mass, double *ms) {
  const bool su3 = L.nc == 3 && L.p.repr == YG_REPR_FUNDAMENTAL;
  const bool pbc = L.p.bc == YG_BC_PERIODIC || L.p.bc == YG_BC_ANTIPERIODIC;
  const int cand[3] = {18, 12, 8};
  const bool ok[3] = {true, su3, su3 && pbc};
  int best = 18;
  double best_ms = 0.0;
  for (int k = 0; k < 3; k++) {
    double t = 0.0, bytes = 0.0;
    if (ok[k]) {
      hop_time(L, mass, cand[k], 20, &t, &bytes, 0);
      if (best_ms == 0.0 || t < best_ms) { best_ms = t; best = cand[k]; }
    }
    if (ms) ms[k] = t;
  }
  L.sl_tuned_reals = best;
  tune_shape(L, mass, best);
  return best;
}

int tuned_inner_links(Lattice &L, double mass) {
  return L.sl_tuned_reals ? L.sl_tuned_reals : tune_inner_links(L, mass, nullptr);
}

}  // namespace yg
