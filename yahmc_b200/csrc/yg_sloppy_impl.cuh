// Device-side pieces of the compressed inner operator shared by the single-system mixed
// CG (yg_sloppy.cu) and the multi-right-hand-side one (yg_mrhs.cu): storage formats of
// spinors, links and packed clover blocks, their loads and stores, the packed Hermitian
// block product, deterministic block sums, programmatic-dependent-launch controls, and a
// site's neighbour table.
#pragma once
#include <cuda_fp16.h>
#include "yg_kernels.h"

namespace yg {

// ------------------------------------------------------------------ storage formats
// Spinor word w of site (blk, h): FP32 -> float4 F[(blk*6 + w)*Vh + h], 6 words, complex 2w, 2w+1
//                                 FP16 -> uint4  F[(blk*3 + w)*Vh + h], 3 words, complex 4w..4w+3
// complex index k = spin*3 + colour (as the FP64 layout)
template <int P> struct SpinorFmt;
template <> struct SpinorFmt<32> {
  using word = float4;
  static constexpr int words = 6;
};
template <> struct SpinorFmt<16> {
  using word = uint4;
  static constexpr int words = 3;
};

__device__ __forceinline__ float2 h2f(unsigned v) {
  __half2 h = *reinterpret_cast<__half2 *>(&v);
  return __half22float2(h);
}
__device__ __forceinline__ unsigned f2h(float2 f) {
  __half2 h = __float22half2_rn(f);
  return *reinterpret_cast<unsigned *>(&h);
}

// unscaled components; FP16 words are stored divided by the site norm (snorm)
template <int P>
__device__ __forceinline__ void sload_raw(float2 (&s)[12], const void *base, int blk, int h, int Vh) {
  if (P == 32) {
    const float4 *f = reinterpret_cast<const float4 *>(base);
#pragma unroll
    for (int w = 0; w < 6; w++) {
      float4 v = __ldg(f + (long)(blk * 6 + w) * Vh + h);
      s[2 * w] = make_float2(v.x, v.y);
      s[2 * w + 1] = make_float2(v.z, v.w);
    }
  } else {
    const uint4 *f = reinterpret_cast<const uint4 *>(base);
#pragma unroll
    for (int w = 0; w < 3; w++) {
      uint4 v = __ldg(f + (long)(blk * 3 + w) * Vh + h);
      s[4 * w + 0] = h2f(v.x);
      s[4 * w + 1] = h2f(v.y);
      s[4 * w + 2] = h2f(v.z);
      s[4 * w + 3] = h2f(v.w);
    }
  }
}

template <int P>
__device__ __forceinline__ float snorm(const float *norm, int blk, int h, int Vh) {
  return P == 32 ? 1.f : __ldg(norm + (long)blk * Vh + h);
}

template <int P>
__device__ __forceinline__ void sload(float2 (&s)[12], const void *base, const float *norm, int blk, int h, int Vh) {
  sload_raw<P>(s, base, blk, h, Vh);
  if (P == 16) {
    float n = snorm<P>(norm, blk, h, Vh);
#pragma unroll
    for (int k = 0; k < 12; k++) s[k] = cscale(s[k], n);
  }
}

template <int P>
__device__ __forceinline__ void sstore(void *base, float *norm, const float2 (&s)[12], int blk, int h, int Vh) {
  if (P == 32) {
    float4 *f = reinterpret_cast<float4 *>(base);
#pragma unroll
    for (int w = 0; w < 6; w++)
      f[(long)(blk * 6 + w) * Vh + h] = make_float4(s[2 * w].x, s[2 * w].y, s[2 * w + 1].x, s[2 * w + 1].y);
  } else {
    float m = 0.f;
#pragma unroll
    for (int k = 0; k < 12; k++) m = fmaxf(m, fmaxf(fabsf(s[k].x), fabsf(s[k].y)));
    float inv = m > 0.f ? 1.f / m : 0.f;
    uint4 *f = reinterpret_cast<uint4 *>(base);
#pragma unroll
    for (int w = 0; w < 3; w++) {
      uint4 v;
      v.x = f2h(make_float2(s[4 * w].x * inv, s[4 * w].y * inv));
      v.y = f2h(make_float2(s[4 * w + 1].x * inv, s[4 * w + 1].y * inv));
      v.z = f2h(make_float2(s[4 * w + 2].x * inv, s[4 * w + 2].y * inv));
      v.w = f2h(make_float2(s[4 * w + 3].x * inv, s[4 * w + 3].y * inv));
      f[(long)(blk * 3 + w) * Vh + h] = v;
    }
    norm[(long)blk * Vh + h] = m;
  }
}

// Storage formats of the inner operator's matrices (links and clover blocks):
//   ST_F32  FP32;  ST_F16  FP16;  ST_I16  16-bit fixed point (value = int16 / 32767 times a
//   scale: 1 for links, whose entries lie in [-1, 1], and a per-site max |entry| for the
//   clover blocks), 15 significant bits against FP16's 11.
constexpr int ST_F32 = 32, ST_F16 = 16, ST_I16 = 15;
constexpr float kI16 = 32767.f;

__device__ __forceinline__ float2 s2f(unsigned v) {          // two int16 -> two float (unscaled)
  return make_float2((float)(short)(v & 0xffffu), (float)(short)(v >> 16));
}
__device__ __forceinline__ unsigned f2s(float a, float b) {   // two floats in [-1,1] -> two int16
  int ia = __float2int_rn(fminf(fmaxf(a, -1.f), 1.f) * kI16);
  int ib = __float2int_rn(fminf(fmaxf(b, -1.f), 1.f) * kI16);
  return ((unsigned)ia & 0xffffu) | ((unsigned)ib << 16);
}

// Links: complex word k of link (site blk,h ; mu): FP32 float2, FP16 half2 or int16 pair at
//   U[((blk*4 + mu)*K + k)*Vh + h], K = 9 (18 reals, row-major) or 6 (rows 0,1)
template <int LP>
__device__ __forceinline__ float2 lload(const void *base, long i) {
  if (LP == ST_F32) return __ldg(reinterpret_cast<const float2 *>(base) + i);
  unsigned v = __ldg(reinterpret_cast<const unsigned *>(base) + i);
  if (LP == ST_F16) return h2f(v);
  return cscale(s2f(v), 1.f / kI16);
}

template <int LP, int K>
__device__ __forceinline__ void link_load(float2 (&u)[9], const void *U, int blk, int h, int Vh, int mu, float sgn) {
#pragma unroll
  for (int k = 0; k < K; k++) u[k] = lload<LP>(U, ((long)(blk * 4 + mu) * K + k) * Vh + h);
  if (K == 6) {
    // row 2 = conj(row0 x row1); the stored rows carry the antiperiodic sign s, and
    // (s r0) x (s r1) = r0 x r1, so the reconstructed row is multiplied by s again
    float2 a0 = u[0], a1 = u[1], a2 = u[2], b0 = u[3], b1 = u[4], b2 = u[5];
    u[6] = cscale(cconj(csub(cmul(a1, b2), cmul(a2, b1))), sgn);
    u[7] = cscale(cconj(csub(cmul(a2, b0), cmul(a0, b2))), sgn);
    u[8] = cscale(cconj(csub(cmul(a0, b1), cmul(a1, b0))), sgn);
  }
  if (K == 4) {
    // 8 reals of an SU(3) link W (FP32 only), see k_pack_links: word 0 = (phase of a0 with
    // the b0/c0 choice in its lowest mantissa bit, phase of the other first-column entry
    // with the column shift in its two lowest bits), words 1-3 = a1, a2 and the smaller of
    // b0, c0 in full.  Rows from |row 0| = |column 0| = 1, then b1, b2 from unitarity and
    // det = 1, c = conj(a x b); finally the columns are shifted back and the sign applied.
    const float2 w = u[0], a1 = u[1], a2 = u[2], st = u[3];
    const bool cstored = (__float_as_uint(w.x) & 1u) != 0u;
    const int shift = (int)(__float_as_uint(w.y) & 3u);
    const float n = a1.x * a1.x + a1.y * a1.y + a2.x * a2.x + a2.y * a2.y;
    float sa, ca, so, co;                     // |phase| <= pi: the SFU forms are accurate to ~4e-7
    __sincosf(w.x, &sa, &ca);
    __sincosf(w.y, &so, &co);
    const float ma = sqrtf(fmaxf(1.f - n, 0.f)), mo = sqrtf(fmaxf(n - (st.x * st.x + st.y * st.y), 0.f));
    const float2 a0 = make_float2(ma * ca, ma * sa), oth = make_float2(mo * co, mo * so);
    const float2 b0 = cstored ? oth : st, c0 = cstored ? st : oth;
    const float inv = n > 0.f ? __frcp_rn(n) : 0.f;
    const float2 b1 = cscale(cadd(cmul(cmulc(a0, a1), b0), cmulc(a2, cconj(c0))), -inv);
    const float2 b2 = cscale(csub(cmulc(a1, cconj(c0)), cmul(cmulc(a0, a2), b0)), inv);
    const float2 c1 = cconj(csub(cmul(a2, b0), cmul(a0, b2)));
    const float2 c2 = cconj(csub(cmul(a0, b1), cmul(a1, b0)));
    const float2 r[3][3] = {{a0, a1, a2}, {b0, b1, b2}, {c0, c1, c2}};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int k = 0; k < 3; k++) {
        // W[i][k] = R[i][(k - shift) mod 3]
        const float2 v = shift == 0 ? r[i][k] : shift == 1 ? r[i][(k + 2) % 3] : r[i][(k + 1) % 3];
        u[i * 3 + k] = cscale(v, sgn);
      }
  }
}

// Packed Hermitian blocks: 72 reals per site (block b: 6 diagonal reals, then the 15
// complex lower-triangle entries (1,0),(2,0),(2,1),...,(5,4)), FP32 as 18 float4, FP16 or
// int16 as 9 uint4 at C[(blk*W + w)*Vh + h]; int16 records scale by cn[blk*Vh + h] / 32767.
template <int CP>
__device__ __forceinline__ void cload(float (&c)[72], const void *base, const float *cn, int blk, int h, int Vh) {
  if (CP == ST_F32) {
    const float4 *f = reinterpret_cast<const float4 *>(base);
#pragma unroll
    for (int w = 0; w < 18; w++) {
      float4 v = __ldg(f + (long)(blk * 18 + w) * Vh + h);
      c[4 * w] = v.x; c[4 * w + 1] = v.y; c[4 * w + 2] = v.z; c[4 * w + 3] = v.w;
    }
  } else {
    const uint4 *f = reinterpret_cast<const uint4 *>(base);
    const float sc = CP == ST_I16 ? __ldg(cn + (long)blk * Vh + h) * (1.f / kI16) : 1.f;
#pragma unroll
    for (int w = 0; w < 9; w++) {
      uint4 v = __ldg(f + (long)(blk * 9 + w) * Vh + h);
      float2 a, b, cc, d;
      if (CP == ST_F16) { a = h2f(v.x); b = h2f(v.y); cc = h2f(v.z); d = h2f(v.w); }
      else { a = cscale(s2f(v.x), sc); b = cscale(s2f(v.y), sc); cc = cscale(s2f(v.z), sc); d = cscale(s2f(v.w), sc); }
      c[8 * w + 0] = a.x; c[8 * w + 1] = a.y; c[8 * w + 2] = b.x; c[8 * w + 3] = b.y;
      c[8 * w + 4] = cc.x; c[8 * w + 5] = cc.y; c[8 * w + 6] = d.x; c[8 * w + 7] = d.y;
    }
  }
}

// y = M x for the Hermitian 6x6 block b of a packed site record
__device__ __forceinline__ void herm_apply(float2 (&y)[6], const float *c, const float2 (&x)[6]) {
#pragma unroll
  for (int i = 0; i < 6; i++) y[i] = cscale(x[i], c[i]);
  int k = 6;
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++, k += 2) {
      float2 m = make_float2(c[k], c[k + 1]);      // M[i][j], and M[j][i] = conj(M[i][j])
      cfma(y[i], m, x[j]);
      cfmac(y[j], m, x[i]);
    }
}

// apply both blocks: spins (0,1) use block 0, spins (2,3) block 1
__device__ __forceinline__ void clover_packed(float2 (&out)[12], const float (&c)[72], const float2 (&s)[12]) {
#pragma unroll
  for (int b = 0; b < 2; b++) {
    float2 x[6], y[6];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      x[i] = s[(2 * b) * 3 + i];
      x[i + 3] = s[(2 * b + 1) * 3 + i];
    }
    herm_apply(y, c + 36 * b, x);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      out[(2 * b) * 3 + i] = y[i];
      out[(2 * b + 1) * 3 + i] = y[i + 3];
    }
  }
}

// ------------------------------------------------------------------ the sloppy hop
struct SHopArgs {
  Geom g;
  const void *src;          // hop input (sloppy spinor)
  const float *src_norm;
  const void *src2;         // STEP2: psi_e for the clover term
  const float *src2_norm;
  void *dst;
  float *dst_norm;
  const void *U;            // sloppy links
  const void *C;            // packed clover blocks
  const float *Cn;          // their per-site scales (int16 storage)
  float coeff;              // +1/2 (step 1) or -1/2 (step 2)
  int lo, n;                // output sites [lo, lo+n): the odd block (step 1) or even (step 2)
  double *part;             // NRM: one partial sum of |dst|^2 per block
};

// ------------------------------------------------------------------ device-side reductions
// Device scalars of the inner CG (sl_scal): |r|^2 in two slots that alternate between
// iterations (iteration k reads slot k&1 and writes slot (k+1)&1, so no block overwrites
// a value another block of the same launch still reads), alpha, <p, A p> for inspection,
// and the count of finished inner iterations (S_ITER, the value the host polls).  Grid sums are two-phase: a producer launch stores one partial per block,
// and every block of the consumer launch adds all of them in index order, so the result
// is deterministic and no block ever waits for another.
enum { S_RR0 = 0, S_RR1 = 1, S_ALPHA = 2, S_PQ = 3, S_ITER = 4, S_WORDS = 8 };

// block total of v, returned to every thread (blockDim a multiple of 32, at most 1024)
__device__ __forceinline__ double block_total(double v) {
  __shared__ double sh[33];
  __syncthreads();                       // a previous call may still be reading sh
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (lane < (int)(blockDim.x >> 5)) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh[32] = v;
  }
  __syncthreads();
  return sh[32];
}

// sum of n partials written by the previous launch, identical in every block
__device__ __forceinline__ double sum_partials(const double *part, int n) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += part[i];
  return block_total(acc);
}

// Programmatic dependent launch: a kernel launched with programmatic stream serialisation
// may start while its predecessor drains; it computes what needs no predecessor data
// (coordinates, neighbour indices), then waits for the predecessor grid to complete and its
// memory to be visible.  Each kernel signals its successor once its block has stored its
// results.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch() { asm volatile("griddepcontrol.launch_dependents;" :::); }

// the neighbours of a site: f[mu] = x+mu, b[mu] = x-mu
struct SiteNbr {
  int c[4];
  int f[4], b[4];
};

__device__ __forceinline__ void site_nbr(SiteNbr &n, const Geom &g, int id) {
  coords_of(g, id, n.c);
#pragma unroll
  for (int mu = 0; mu < 4; mu++) {
    n.f[mu] = neighbour(g, n.c, mu, +1);
    n.b[mu] = neighbour(g, n.c, mu, -1);
  }
}

}  // namespace yg
