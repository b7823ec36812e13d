// Learned preconditioner: a gauge-covariant parallel-transport convolution network ("PTC")
// with its forward, adjoint and weight-gradient passes on the tensor cores.
//
// One layer maps a field of Ci channels to one of Co channels (spinor fields of the
// representation, d = 3 colours, 4 spins, on the whole lattice):
//     out[x, o] = sum_p sum_i W[p, o, i] (T_p in_i)(x),
// nine paths p: 0 the site itself, 1..4 the hop forward along mu = p - 1,
// (T f)(x) = U_mu(x) f(x + mu), and 5..8 the hop backward, (T f)(x) = U_mu(x - mu)^dag f(x - mu),
// through the represented links the Dirac operator uses (boundary signs included).  W[p, o, i]
// is a complex 4x4 matrix on the spin index and never touches colour, so the layer commutes
// with gauge transformations exactly.  The adjoint layer (the input gradient) is a layer with
// conjugate-transposed weights and reversed paths, packed on the host.
//
// Per tile of 64 sites and per path the transported inputs are formed on the CUDA cores in
// FP32 and written to shared memory as BF16 (the B operand, one row per (colour, site), one
// column per (input channel, spin) with real parts before imaginary parts), and the complex
// product with the weights is a real BF16 GEMM with FP32 accumulation on the tensor cores:
//     [Y_re; Y_im] (2 Co 4 x N) += [[W_re, -W_im]; [W_im, W_re]] (2 Co 4 x 2 Ci 4) [X_re; X_im],
// issued with tcgen05.mma (cta_group::1, kind::f16, M = 128, N = 192) by one thread, operands
// in shared memory in the canonical K-major layout without swizzle (8-row x 16-byte core
// matrices), accumulator in tensor memory, read back with tcgen05.ld.  The weight gradient
//     dW[p, o, i][s, s'] = sum_{x, c} g[x, o, c, s] conj((T_p in_i)[x, c, s'])
// is the same kind of product with the sites as the reduction dimension.
//
// Activations are FP32 site blocks: channel ch of site id (the reference's site order) is 24
// floats at (ch * V + id) * 24, float (spin * 3 + colour) * 2 + re/im.  Every wait on the tensor core
// is bounded; a wait that runs out sets an error word, frees the tensor memory and returns.
#include <cuda_bf16.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include "yg_lattice.h"
#include "yg_kernels.h"

namespace yg {

namespace {

constexpr int kPaths = 9;
constexpr int kTileSites = 64;              // sites per CTA tile
constexpr int kN = 3 * kTileSites;          // GEMM columns per tile: (colour, site)
constexpr int kM = 128;                     // GEMM rows (tcgen05 M)
constexpr int kThreads = 128;
constexpr int kTmemCols = 256;              // >= kN, a power of two
constexpr long kSpinLimit = 1L << 26;       // bounded waits
constexpr int kStageLd = kN + 1;            // row stride of the epilogue's staging tile (floats)

// ---- shared-memory operand layout: K-major, no swizzle.  Element (r, k) of an R x K tile
// lives at byte (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2 with SBO = K / 8 * 128:
// each 8 x 8 block of BF16 is one 128-byte core matrix, the K-direction core matrices of a row
// group are adjacent (LBO = 128), row groups follow each other (SBO).
__host__ __device__ __forceinline__ uint32_t kmajor_off(int r, int k, int K) {
  return (uint32_t)((r >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, int K) {
  const uint64_t lbo = 128 >> 4, sbo = (uint64_t)((K >> 3) * 128) >> 4;
  return (uint64_t)((saddr >> 4) & 0x3fff) | (lbo << 16) | (sbo << 32) | (1ull << 46);   // version 1, no swizzle
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
}

// waits for phase `phase` of the barrier; false if the bounded wait ran out
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (long i = 0; i < kSpinLimit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t slot_saddr, int cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_saddr), "r"(cols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, int cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols));
}

// 32 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes 32w..32w+31)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

struct PtcArgs {
  Geom g;
  const double2 *U;         // represented FP64 links (the engine's layout, boundary signs folded in)
  const float *in;          // Ci channels of activation planes
  float *out;               // Co channels
  const __nv_bfloat16 *A;   // forward: 9 packed A chunks (kM x Kp each)
  const float *gin;         // wgrad: Co channels of output gradient planes
  float *part;              // wgrad: per-CTA partial weight gradients
  int *err;                 // bounded-wait failures
  int V;
};

// site id and its neighbour along path p (p = 0 itself), and the link that transports from it
__device__ __forceinline__ int path_site(const Geom &g, int id, int p) {
  if (p == 0) return id;
  int c[4];
  coords_of(g, id, c);
  return p <= 4 ? neighbour(g, c, p - 1, +1) : neighbour(g, c, p - 5, -1);
}

// the 3x3 link that transports along path p to site id: U_mu(x) (forward) or U_mu(x - mu)^dag
__device__ __forceinline__ void path_link(const PtcArgs &a, int id, int nid, int p, float2 (&u)[9]) {
  const Geom &g = a.g;
  const int mu = p <= 4 ? p - 1 : p - 5;
  const int lid = p <= 4 ? id : nid;
  const int lb = lid >= g.Vh, lh = lid - lb * g.Vh;
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const double2 v = __ldg(a.U + ((long)(lb * 4 + mu) * 9 + (p <= 4 ? i * 3 + j : j * 3 + i)) * g.Vh + lh);
      u[i * 3 + j] = p <= 4 ? make_float2((float)v.x, (float)v.y) : make_float2((float)v.x, -(float)v.y);
    }
}

__device__ __forceinline__ void put_bf16(unsigned char *base, uint32_t off, float v) {
  *reinterpret_cast<__nv_bfloat16 *>(base + off) = __float2bfloat16_rn(v);
}

// four consecutive BF16 (one 8-byte store): k-columns k0..k0+3 of row r, k0 a multiple of 4
__device__ __forceinline__ void put_bf16x4(unsigned char *base, uint32_t off, float v0, float v1, float v2, float v3) {
  __nv_bfloat162 lo = __floats2bfloat162_rn(v0, v1), hi = __floats2bfloat162_rn(v2, v3);
  uint2 w;
  w.x = *reinterpret_cast<uint32_t *>(&lo);
  w.y = *reinterpret_cast<uint32_t *>(&hi);
  *reinterpret_cast<uint2 *>(base + off) = w;
}

// Activations are site blocks: channel ch of site id is 24 floats at (ch * V + id) * 24, float
// k2 = (spin * 3 + colour) * 2 + re/im.  A thread gathers whole blocks with 16-byte loads.
struct Block {
  float4 w[6];
};

__device__ __forceinline__ void load_block(Block &b, const float *act, long base) {
  const float4 *p = reinterpret_cast<const float4 *>(act + base * 24);
#pragma unroll
  for (int i = 0; i < 6; i++) b.w[i] = __ldg(p + i);
}

__device__ __forceinline__ float2 blk_c(const Block &b, int s, int a) {   // complex (spin s, colour a)
  const int k = (s * 3 + a) * 2;
  const float4 &w = b.w[k >> 2];
  return (k & 2) ? make_float2(w.z, w.w) : make_float2(w.x, w.y);
}

// the transported spin-colour block y[s][a] = sum_b u[a][b] f[s][b] (IDENT: y = f)
template <bool IDENT>
__device__ __forceinline__ void transport_block(float2 (&y)[4][3], const Block &f, const float2 (&u)[9]) {
#pragma unroll
  for (int s = 0; s < 4; s++) {
    float2 v[3];
#pragma unroll
    for (int b = 0; b < 3; b++) v[b] = blk_c(f, s, b);
#pragma unroll
    for (int a = 0; a < 3; a++) {
      if (IDENT) {
        y[s][a] = v[a];
      } else {
        float2 acc = make_float2(0.f, 0.f);
#pragma unroll
        for (int b = 0; b < 3; b++) cfma(acc, u[a * 3 + b], v[b]);
        y[s][a] = acc;
      }
    }
  }
}

// ---------------------------------------------------------------- forward layer
// grid: one CTA per tile of 64 sites.  CI input channels (1 or a multiple of 2), CO output
// channels (2 * CO * 4 <= 128 rows).  KP = columns of one path's chunk (2 CI 4, padded to 16).
template <int CI, int CO>
__global__ void __launch_bounds__(kThreads, 1) k_ptc_layer(PtcArgs a) {
  constexpr int KP = ((2 * CI * 4 + 15) / 16) * 16;
  constexpr int PAIRS = CI * 4;                          // (channel, spin) pairs per site
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *sA = sm;                                // kM x KP
  unsigned char *sB = sm + kM * KP * 2;                  // kN x KP
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + kN * KP * 2);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
  __shared__ int s_site[kTileSites], s_nbr[kTileSites];

  const int tid = threadIdx.x, warp = tid >> 5;
  const int t0 = blockIdx.x * kTileSites;
  if (warp == 0) tmem_alloc(smem_u32(tslot), kTmemCols);
  if (tid == 0) mbar_init(smem_u32(mbar));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  bool ok = true;

  // zero the padding columns of B once (CI = 1: columns 8..15 stay zero)
  if constexpr (KP > 2 * PAIRS) {
    for (int e = tid; e < kN * (KP - 2 * PAIRS); e += kThreads) {
      const int r = e / (KP - 2 * PAIRS), k = 2 * PAIRS + e % (KP - 2 * PAIRS);
      put_bf16(sB, kmajor_off(r, k, KP), 0.f);
    }
  }

  for (int p = 0; p < kPaths && ok; p++) {
    // A chunk of path p: a straight copy of the packed operand
    {
      const uint4 *src = reinterpret_cast<const uint4 *>(a.A + (long)p * kM * KP);
      uint4 *dst = reinterpret_cast<uint4 *>(sA);
      for (int e = tid; e < kM * KP * 2 / 16; e += kThreads) dst[e] = __ldg(src + e);
    }
    // B chunk: the transported inputs of the tile's sites.  Thread (site j, part) takes the
    // channels part, part + NPART, ...; a one-channel input is split by spin pairs instead.
    if (tid < kTileSites) {
      const int id = t0 + tid;
      s_site[tid] = id < a.V ? id : -1;
      s_nbr[tid] = id < a.V ? path_site(a.g, id, p) : -1;
    }
    __syncthreads();
    {
      constexpr int NPART = kThreads / kTileSites;
      const int j = tid % kTileSites, part = tid / kTileSites;
      const int id = s_site[j], nid = s_nbr[j];
      float2 u[9];
      if (id >= 0 && p > 0) path_link(a, id, nid, p, u);
      constexpr int NCH = CI >= NPART ? CI / NPART : 1;     // channels per thread
      constexpr int CB = NCH < 4 ? NCH : 4;                  // gathered together
#pragma unroll 1
      for (int c0 = 0; c0 < NCH; c0 += CB) {
        Block f[CB];
#pragma unroll
        for (int q = 0; q < CB; q++) {
          const int ch = CI >= NPART ? part + NPART * (c0 + q) : 0;
          if (id >= 0) load_block(f[q], a.in, (long)ch * a.V + nid);
          else
#pragma unroll
            for (int i = 0; i < 6; i++) f[q].w[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int q = 0; q < CB; q++) {
          const int ch = CI >= NPART ? part + NPART * (c0 + q) : 0;
          float2 y[4][3];
          if (p == 0) transport_block<true>(y, f[q], u);
          else transport_block<false>(y, f[q], u);
          if (CI >= NPART) {
#pragma unroll
            for (int c = 0; c < 3; c++) {
              const int r = c * kTileSites + j;
              put_bf16x4(sB, kmajor_off(r, ch * 4, KP), y[0][c].x, y[1][c].x, y[2][c].x, y[3][c].x);
              put_bf16x4(sB, kmajor_off(r, PAIRS + ch * 4, KP), y[0][c].y, y[1][c].y, y[2][c].y, y[3][c].y);
            }
          } else if (part == 0) {
            // one input channel: columns 0..3 real, 4..7 imaginary, written by part 0
#pragma unroll
            for (int c = 0; c < 3; c++) {
              const int r = c * kTileSites + j;
              put_bf16x4(sB, kmajor_off(r, 0, KP), y[0][c].x, y[1][c].x, y[2][c].x, y[3][c].x);
              put_bf16x4(sB, kmajor_off(r, 4, KP), y[0][c].y, y[1][c].y, y[2][c].y, y[3][c].y);
            }
          }
        }
      }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t aa = smem_u32(sA), bb = smem_u32(sB);
#pragma unroll
      for (int kk = 0; kk < KP / 16; kk++)
        mma_bf16(tmem, smem_desc(aa + kk * 256, KP), smem_desc(bb + kk * 256, KP), idesc_bf16(kM, kN),
                 (p > 0 || kk > 0) ? 1u : 0u);
      mma_commit(smem_u32(mbar));
    }
    ok = mbar_wait(smem_u32(mbar), (uint32_t)(p & 1));
    if (!ok && tid == 0) atomicExch(a.err, 1);
    tc_fence_after();
    ok = __syncthreads_and(ok);
  }

  if (ok) {
    // epilogue: accumulator row m = (o, s) real part (m < 4 CO) or imaginary part
    // (4 CO <= m < 8 CO), column n = (colour, site); staged through shared memory (the operand
    // buffers are free now), then every thread writes whole 96-byte site blocks
    float *stage = reinterpret_cast<float *>(sm);
    const int m = warp * 32 + (tid & 31);
    if (warp * 32 < 8 * CO) {
#pragma unroll 1
      for (int cb = 0; cb < kN / 32; cb++) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + cb * 32, v);
#pragma unroll
        for (int i = 0; i < 32; i++) stage[m * kStageLd + cb * 32 + i] = v[i];
      }
    }
    __syncthreads();
    for (int e = tid; e < kTileSites * CO; e += kThreads) {
      const int j = e % kTileSites, o = e / kTileSites;
      if (t0 + j >= a.V) continue;
      float4 w[6];
      float *wf = reinterpret_cast<float *>(w);
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          wf[(s * 3 + c) * 2] = stage[(o * 4 + s) * kStageLd + c * kTileSites + j];
          wf[(s * 3 + c) * 2 + 1] = stage[(4 * CO + o * 4 + s) * kStageLd + c * kTileSites + j];
        }
      float4 *dst = reinterpret_cast<float4 *>(a.out + ((long)o * a.V + t0 + j) * 24);
#pragma unroll
      for (int i = 0; i < 6; i++) dst[i] = w[i];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, kTmemCols);
}

// ---------------------------------------------------------------- weight gradient
// dW_p^T[(i, s'), (o, s)] = sum_n X_p[(i, s'), n] conj(G[(o, s), n]) as a real product
//   [C_re | C_im] = [X_re | X_im] [[G_re^T, -G_im^T]; [G_im^T, G_re^T]]
// A (rows (i, s'), padded to 128; columns (n re | n im), 2 kN) and B (rows the 2 CO 4 columns
// of [C_re | C_im], padded to NB; same K) in shared memory; the CTA accumulates its tiles for
// a group of paths in tensor memory (NB columns per path) and writes one partial per path.
template <int CI, int CO, int PG>
__global__ void __launch_bounds__(kThreads, 1) k_ptc_wgrad(PtcArgs a, int ntiles) {
  constexpr int KW = 2 * kN;                              // reduction columns per tile
  constexpr int NB = ((2 * CO * 4 + 15) / 16) * 16;       // GEMM columns per path
  constexpr int PAIRS = CI * 4, OPAIRS = CO * 4;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char *sA = sm;                                 // kM x KW (transported inputs)
  unsigned char *sB = sm + kM * KW * 2;                   // NB x KW (output gradients)
  uint64_t *mbar = reinterpret_cast<uint64_t *>(sB + NB * KW * 2);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
  __shared__ int s_site[kTileSites], s_nbr[kTileSites];
  constexpr int cols = NB * PG <= 32 ? 32 : NB * PG <= 64 ? 64 : NB * PG <= 128 ? 128 : NB * PG <= 256 ? 256 : 512;
  static_assert(NB * PG <= 512, "tensor memory columns");

  const int tid = threadIdx.x, warp = tid >> 5;
  const int p0 = blockIdx.y * PG;
  if (warp == 0) tmem_alloc(smem_u32(tslot), cols);
  if (tid == 0) mbar_init(smem_u32(mbar));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  // rows of A beyond the input pairs stay zero
  for (int e = tid; e < (kM - PAIRS) * KW; e += kThreads) put_bf16(sA, kmajor_off(PAIRS + e / KW, e % KW, KW), 0.f);
  for (int e = tid; e < (NB - 2 * OPAIRS) * KW; e += kThreads)
    put_bf16(sB, kmajor_off(2 * OPAIRS + e / KW, e % KW, KW), 0.f);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  bool ok = true;
  uint32_t phase = 0;
  bool first = true;

  for (int tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const int t0 = tile * kTileSites;
    // B: the output gradients of the tile (the same for every path), site blocks of gin
    for (int e = tid; e < kTileSites * CO; e += kThreads) {
      const int j = e % kTileSites, o = e / kTileSites, id = t0 + j;
      Block gb;
      if (id < a.V) load_block(gb, a.gin, (long)o * a.V + id);
      else
#pragma unroll
        for (int i = 0; i < 6; i++) gb.w[i] = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int sp = 0; sp < 4; sp++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const float2 gv = blk_c(gb, sp, c);
          const int os = o * 4 + sp, n = c * kTileSites + j;
          put_bf16(sB, kmajor_off(os, n, KW), gv.x);
          put_bf16(sB, kmajor_off(os, kN + n, KW), gv.y);
          put_bf16(sB, kmajor_off(OPAIRS + os, n, KW), -gv.y);
          put_bf16(sB, kmajor_off(OPAIRS + os, kN + n, KW), gv.x);
        }
    }
    for (int pp = 0; pp < PG && ok; pp++) {
      const int p = p0 + pp;
      if (tid < kTileSites) {
        const int id = t0 + tid;
        s_site[tid] = id < a.V ? id : -1;
        s_nbr[tid] = id < a.V ? path_site(a.g, id, p) : -1;
      }
      __syncthreads();
      {
        constexpr int NPART = kThreads / kTileSites;
        const int j = tid % kTileSites, part = tid / kTileSites;
        const int id = s_site[j], nid = s_nbr[j];
        float2 u[9];
        if (id >= 0 && p > 0) path_link(a, id, nid, p, u);
        constexpr int NCH = CI >= NPART ? CI / NPART : 1;
        constexpr int CB = NCH < 4 ? NCH : 4;
#pragma unroll 1
        for (int c0 = 0; c0 < NCH; c0 += CB) {
          Block f[CB];
#pragma unroll
          for (int q = 0; q < CB; q++) {
            const int ch = CI >= NPART ? part + NPART * (c0 + q) : 0;
            if (id >= 0) load_block(f[q], a.in, (long)ch * a.V + nid);
            else
#pragma unroll
              for (int i = 0; i < 6; i++) f[q].w[i] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
#pragma unroll
          for (int q = 0; q < CB; q++) {
            const int ch = CI >= NPART ? part + NPART * (c0 + q) : 0;
            if (CI < NPART && part != 0) continue;
            float2 y[4][3];
            if (p == 0) transport_block<true>(y, f[q], u);
            else transport_block<false>(y, f[q], u);
#pragma unroll
            for (int sp = 0; sp < 4; sp++)
#pragma unroll
              for (int c = 0; c < 3; c++) {
                const int n = c * kTileSites + j, row = ch * 4 + sp;
                put_bf16(sA, kmajor_off(row, n, KW), y[sp][c].x);
                put_bf16(sA, kmajor_off(row, kN + n, KW), y[sp][c].y);
              }
          }
        }
      }
      fence_async_smem();
      tc_fence_before();
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        const uint32_t aa = smem_u32(sA), bb = smem_u32(sB);
#pragma unroll 4
        for (int kk = 0; kk < KW / 16; kk++)
          mma_bf16(tmem + pp * NB, smem_desc(aa + kk * 256, KW), smem_desc(bb + kk * 256, KW), idesc_bf16(kM, NB),
                   (!first || kk > 0) ? 1u : 0u);
        mma_commit(smem_u32(mbar));
      }
      ok = mbar_wait(smem_u32(mbar), phase);
      phase ^= 1u;
      if (!ok && tid == 0) atomicExch(a.err, 1);
      tc_fence_after();
      ok = __syncthreads_and(ok);
      if (pp == PG - 1) first = false;
    }
    // the first tile initialised each path's accumulator (first flips after the last path)
  }

  if (ok) {
    // row m = (i, s') (m < PAIRS), column pp * NB + j: j < 4 CO the real part of dW^T[(i,s'), (o,s)],
    // 4 CO <= j < 8 CO its imaginary part.  part[(blockIdx.x * 9 + p) * kM * NB + m * NB + j]
    const int m = warp * 32 + (tid & 31);
    for (int pp = 0; pp < PG; pp++) {
      for (int cb = 0; cb < (NB + 31) / 32; cb++) {
        float v[32];
        tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + pp * NB + cb * 32, v);
        if (m < PAIRS) {
          float *dst = a.part + ((long)blockIdx.x * kPaths + p0 + pp) * kM * NB + (long)m * NB + cb * 32;
#pragma unroll
          for (int i = 0; i < 32; i++)
            if (cb * 32 + i < NB) dst[i] = v[i];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, cols);
}

// even sites of an FP64 engine field (F[k * Vh + h], complex word k = spin * 3 + colour)
// -> channel 0 of the activations (site blocks), scaled; odd sites zero
__global__ void k_ptc_from_field(float *act, const double2 *f, int V, int Vh, double scale) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= V) return;
  float *dst = act + (long)id * 24;
#pragma unroll
  for (int k = 0; k < 12; k++) {
    const double2 v = id < Vh ? f[(long)k * Vh + id] : make_double2(0.0, 0.0);
    dst[2 * k] = (float)(v.x * scale);
    dst[2 * k + 1] = (float)(v.y * scale);
  }
}

// channel 0 of the activations on the even sites -> FP64 engine field, scaled
__global__ void k_ptc_to_field(double2 *f, const float *act, int V, int Vh, double scale) {
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= Vh) return;
  const float *src = act + (long)h * 24;
#pragma unroll
  for (int k = 0; k < 12; k++) f[(long)k * Vh + h] = make_double2(src[2 * k] * scale, src[2 * k + 1] * scale);
}

// output gradient of the loss term |y - e|^2 / |e|^2 on channel 0's even sites:
// g = (y - e) / |e|^2 (odd sites zero); partials of |y - e|^2 per block
__global__ void k_ptc_loss_grad(float *g, double *part, const float *y, const double2 *e, int V, int Vh, double inv_ne,
                                double escale) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  if (id < V) {
#pragma unroll
    for (int k = 0; k < 12; k++) {
      double dr = 0.0, di = 0.0;
      if (id < Vh) {
        const double2 ev = e[(long)k * Vh + id];
        dr = (double)y[(long)id * 24 + 2 * k] - ev.x * escale;
        di = (double)y[(long)id * 24 + 2 * k + 1] - ev.y * escale;
        acc += dr * dr + di * di;
      }
      g[(long)id * 24 + 2 * k] = (float)(dr * inv_ne);
      g[(long)id * 24 + 2 * k + 1] = (float)(di * inv_ne);
    }
  }
  __shared__ double sh[256];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// sum of the per-CTA weight-gradient partials in CTA order (FP64): out[e] = sum_b part[b * n + e]
__global__ void k_ptc_sum_parts(double *out, const float *part, int nparts, long n) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= n) return;
  double acc = 0.0;
  for (int b = 0; b < nparts; b++) acc += (double)part[(long)b * n + e];
  out[e] = acc;
}

}  // namespace

// ---------------------------------------------------------------- host side
struct Ptc {
  Lattice *L = nullptr;
  int nl = 0;
  int ch[kPtcMaxLayers + 1] = {};
  std::vector<std::vector<double>> W;   // per layer: [9][Co][Ci][4][4] complex as (re, im)
  DevBuf Af[kPtcMaxLayers], Aa[kPtcMaxLayers];
  DevBuf act[kPtcMaxLayers + 1];        // forward activations
  DevBuf g[2];                          // gradient ping-pong
  DevBuf part, err, dpart, wsum;
  int maxc = 1;
};

namespace {

int kp_of(int ci) { return ((2 * ci * 4 + 15) / 16) * 16; }

// packed BF16 A operand of a layer: 9 chunks of kM x Kp, row m = (re|im, o, s), col k = (re|im, i, s')
std::vector<uint16_t> pack_forward(const std::vector<double> &w, int ci, int co) {
  const int kp = kp_of(ci), mc = 4 * co, pairs = 4 * ci;
  std::vector<uint16_t> out((size_t)kPaths * kM * kp, 0);
  auto bf16 = [](double v) {
    float f = (float)v;
    uint32_t u;
    std::memcpy(&u, &f, 4);
    u += 0x7fffu + ((u >> 16) & 1u);      // round to nearest even
    return (uint16_t)(u >> 16);
  };
  for (int p = 0; p < kPaths; p++)
    for (int m = 0; m < 2 * mc; m++)
      for (int k = 0; k < 2 * pairs; k++) {
        const int os = m % mc, is = k % pairs;
        const int o = os >> 2, s = os & 3, i = is >> 2, t = is & 3;
        const size_t idx = ((((size_t)p * co + o) * ci + i) * 4 + s) * 4 + t;
        const double wr = w[2 * idx], wi = w[2 * idx + 1];
        const bool im_out = m >= mc, im_in = k >= pairs;
        const double v = !im_out ? (!im_in ? wr : -wi) : (!im_in ? wi : wr);
        out[(size_t)p * kM * kp + kmajor_off(m, k, kp) / 2] = bf16(v);
      }
  return out;
}

// weights of the adjoint layer: W'[p'][i][o] = W[p][o][i]^dag, p' the reversed path
std::vector<double> adjoint_weights(const std::vector<double> &w, int ci, int co) {
  std::vector<double> a(w.size());
  for (int p = 0; p < kPaths; p++) {
    const int q = p == 0 ? 0 : (p <= 4 ? p + 4 : p - 4);
    for (int o = 0; o < co; o++)
      for (int i = 0; i < ci; i++)
        for (int s = 0; s < 4; s++)
          for (int t = 0; t < 4; t++) {
            const size_t src = ((((size_t)p * co + o) * ci + i) * 4 + s) * 4 + t;
            const size_t dst = ((((size_t)q * ci + i) * co + o) * 4 + t) * 4 + s;
            a[2 * dst] = w[2 * src];
            a[2 * dst + 1] = -w[2 * src + 1];
          }
  }
  return a;
}

// at least 100 KiB of shared memory per CTA (the epilogue's staging tile needs 96.5 KiB) keeps
// two CTAs per SM at most, so their tensor memory (256 columns each) always fits the SM's 512
// columns and no allocation has to wait
constexpr size_t kMinSmem = 100 * 1024;
template <int CI, int CO>
size_t layer_smem() { return std::max(kMinSmem, (size_t)kM * kp_of(CI) * 2 + (size_t)kN * kp_of(CI) * 2 + 16); }
template <int CI, int CO>
size_t wgrad_smem() { return (size_t)kM * 2 * kN * 2 + (size_t)(((2 * CO * 4 + 15) / 16) * 16) * 2 * kN * 2 + 16; }

template <int CI, int CO>
void run_layer(Lattice &L, const PtcArgs &a) {
  const size_t sm = layer_smem<CI, CO>();
  YG_CUDA(cudaFuncSetAttribute(k_ptc_layer<CI, CO>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_ptc_layer<CI, CO><<<nblk(L.V, kTileSites), kThreads, sm, L.stream>>>(a);
  YG_LAUNCHED();
}

constexpr int kPathGroup = 3;   // paths per wgrad CTA (3 x 128 accumulator columns)

template <int CI, int CO>
int run_wgrad(Lattice &L, const PtcArgs &a, int sms) {
  const size_t sm = wgrad_smem<CI, CO>();
  YG_CUDA(cudaFuncSetAttribute(k_ptc_wgrad<CI, CO, kPathGroup>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int ntiles = nblk(L.V, kTileSites);
  const int gx = std::min(ntiles, sms);
  k_ptc_wgrad<CI, CO, kPathGroup><<<dim3(gx, kPaths / kPathGroup), kThreads, sm, L.stream>>>(a, ntiles);
  YG_LAUNCHED();
  return gx;
}

// dispatch on (Ci, Co) in {(1, C), (C, C), (C, 1)}, C in {8, 16}
#define YG_PTC_DISPATCH(CI_, CO_, ...)                                                          \
  do {                                                                                          \
    const int ci_ = (CI_), co_ = (CO_);                                                         \
    if (ci_ == 1 && co_ == 8) { constexpr int CI = 1, CO = 8; __VA_ARGS__; }                    \
    else if (ci_ == 8 && co_ == 8) { constexpr int CI = 8, CO = 8; __VA_ARGS__; }               \
    else if (ci_ == 8 && co_ == 1) { constexpr int CI = 8, CO = 1; __VA_ARGS__; }               \
    else if (ci_ == 1 && co_ == 16) { constexpr int CI = 1, CO = 16; __VA_ARGS__; }             \
    else if (ci_ == 16 && co_ == 16) { constexpr int CI = 16, CO = 16; __VA_ARGS__; }           \
    else if (ci_ == 16 && co_ == 1) { constexpr int CI = 16, CO = 1; __VA_ARGS__; }             \
    else throw Error(YG_ERR_ARG, "PTC layers: channels 1 -> C -> ... -> C -> 1 with C = 8 or 16"); \
  } while (0)

PtcArgs base_args(Ptc &n) {
  PtcArgs a{};
  a.g = n.L->g;
  a.U = n.L->links.as<double2>();
  a.err = n.err.as<int>();
  a.V = (int)n.L->V;
  return a;
}

void check_err(Ptc &n) {
  int e = 0;
  YG_CUDA(cudaMemcpyAsync(&e, n.err.p, sizeof(int), cudaMemcpyDeviceToHost, n.L->stream));
  YG_CUDA(cudaStreamSynchronize(n.L->stream));
  if (e) {
    YG_CUDA(cudaMemsetAsync(n.err.p, 0, sizeof(int), n.L->stream));
    throw Error(YG_TIMEOUT, "PTC layer: a bounded wait on the tensor core ran out");
  }
}

size_t planes_bytes(const Lattice &L, int c) { return sizeof(float) * 24 * (size_t)c * L.V; }

}  // namespace

Ptc *ptc_create(Lattice &L, int nl, const int *ch) {
  if (L.d != 3) throw Error(YG_ERR_ARG, "the PTC network is built for d = 3 representations");
  if (nl < 1 || nl > kPtcMaxLayers) throw Error(YG_ERR_ARG, "1..8 layers");
  if (ch[0] != 1 || ch[nl] != 1) throw Error(YG_ERR_ARG, "the network maps one channel to one channel");
  auto *n = new Ptc();
  n->L = &L;
  n->nl = nl;
  for (int l = 0; l <= nl; l++) {
    n->ch[l] = ch[l];
    n->maxc = std::max(n->maxc, ch[l]);
  }
  for (int l = 0; l < nl; l++) {
    int ci = ch[l], co = ch[l + 1];
    YG_PTC_DISPATCH(ci, co, (void)CI; (void)CO);
    n->W.emplace_back((size_t)2 * kPaths * ci * co * 16, 0.0);
    n->Af[l].alloc((size_t)kPaths * kM * kp_of(ci) * 2);
    n->Aa[l].alloc((size_t)kPaths * kM * kp_of(co) * 2);
    YG_CUDA(cudaMemsetAsync(n->Af[l].p, 0, n->Af[l].bytes, L.stream));     // zero weights until set
    YG_CUDA(cudaMemsetAsync(n->Aa[l].p, 0, n->Aa[l].bytes, L.stream));
  }
  for (int l = 0; l <= nl; l++) n->act[l].alloc(planes_bytes(L, ch[l]));
  n->g[0].alloc(planes_bytes(L, n->maxc));
  n->g[1].alloc(planes_bytes(L, n->maxc));
  n->err.alloc(sizeof(int));
  YG_CUDA(cudaMemsetAsync(n->err.p, 0, sizeof(int), L.stream));
  n->dpart.alloc(sizeof(double) * nblk(L.V, 256));
  return n;
}

Lattice &ptc_lattice(Ptc &n) { return *n.L; }

void ptc_destroy(Ptc *n) {
  if (!n) return;
  for (auto &b : n->Af) b.release();
  for (auto &b : n->Aa) b.release();
  for (auto &b : n->act) b.release();
  for (auto &b : n->g) b.release();
  n->part.release();
  n->wsum.release();
  n->err.release();
  n->dpart.release();
  delete n;
}

void ptc_set_weights(Ptc &n, int l, const double *w) {
  if (l < 0 || l >= n.nl) throw Error(YG_ERR_ARG, "layer index");
  const int ci = n.ch[l], co = n.ch[l + 1];
  std::memcpy(n.W[l].data(), w, sizeof(double) * n.W[l].size());
  std::vector<uint16_t> af = pack_forward(n.W[l], ci, co);
  std::vector<uint16_t> aa = pack_forward(adjoint_weights(n.W[l], ci, co), co, ci);
  YG_CUDA(cudaMemcpyAsync(n.Af[l].p, af.data(), af.size() * 2, cudaMemcpyHostToDevice, n.L->stream));
  YG_CUDA(cudaMemcpyAsync(n.Aa[l].p, aa.data(), aa.size() * 2, cudaMemcpyHostToDevice, n.L->stream));
  YG_CUDA(cudaStreamSynchronize(n.L->stream));
}

void ptc_get_weights(Ptc &n, int l, double *w) {
  if (l < 0 || l >= n.nl) throw Error(YG_ERR_ARG, "layer index");
  std::memcpy(w, n.W[l].data(), sizeof(double) * n.W[l].size());
}

// one layer on activation planes (adjoint: the input-gradient layer, Co -> Ci channels)
void ptc_layer(Ptc &n, int l, int adjoint, const float *in, float *out) {
  if (l < 0 || l >= n.nl) throw Error(YG_ERR_ARG, "layer index");
  PtcArgs a = base_args(n);
  a.in = in;
  a.out = out;
  const int ci = adjoint ? n.ch[l + 1] : n.ch[l], co = adjoint ? n.ch[l] : n.ch[l + 1];
  a.A = (adjoint ? n.Aa[l] : n.Af[l]).as<__nv_bfloat16>();
  YG_PTC_DISPATCH(ci, co, run_layer<CI, CO>(*n.L, a));
}

// forward through all layers from act[0]; act[l] keeps every layer's input
static void forward(Ptc &n) {
  for (int l = 0; l < n.nl; l++) ptc_layer(n, l, 0, n.act[l].as<float>(), n.act[l + 1].as<float>());
}

void ptc_apply(Ptc &n, double *dst, const double *src) {
  Lattice &L = *n.L;
  long lo, cnt;
  L.view_range(YG_VIEW_EVEN, lo, cnt);
  const double nrm = std::sqrt(blas_sqnorm(L, src, lo, cnt));
  if (!(nrm > 0.0)) {
    blas_zero(L, dst, lo, cnt);
    return;
  }
  k_ptc_from_field<<<nblk(L.V, 256), 256, 0, L.stream>>>(n.act[0].as<float>(), (const double2 *)src, (int)L.V,
                                                          (int)L.Vh, 1.0 / nrm);
  YG_LAUNCHED();
  forward(n);
  k_ptc_to_field<<<nblk(L.Vh, 256), 256, 0, L.stream>>>((double2 *)dst, n.act[n.nl].as<float>(), (int)L.V,
                                                        (int)L.Vh, nrm);
  YG_LAUNCHED();
  check_err(n);
}

// weight gradient of layer l from the output gradient planes gin and the layer input act[l],
// added into grads (complex, the layer's W layout)
static void wgrad(Ptc &n, int l, const float *gin, std::vector<double> &grads) {
  Lattice &L = *n.L;
  int dev = 0, sms = 0;
  YG_CUDA(cudaGetDevice(&dev));
  YG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int ci = n.ch[l], co = n.ch[l + 1];
  const int nb = ((2 * co * 4 + 15) / 16) * 16;
  const size_t need = sizeof(float) * (size_t)sms * kPaths * kM * nb;
  if (n.part.bytes < need) {
    n.part.release();
    n.part.alloc(need);
  }
  PtcArgs a = base_args(n);
  a.in = n.act[l].as<float>();
  a.gin = gin;
  a.part = n.part.as<float>();
  int gx = 0;
  YG_PTC_DISPATCH(ci, co, gx = run_wgrad<CI, CO>(L, a, sms));
  // C[(i, s'), (o, s)] summed over the CTAs in order on the device; dW[p][o][i][s][s'] = conj(C)
  const long per = (long)kPaths * kM * nb;
  if (n.wsum.bytes < sizeof(double) * per) {
    n.wsum.release();
    n.wsum.alloc(sizeof(double) * per);
  }
  k_ptc_sum_parts<<<nblk(per, 256), 256, 0, L.stream>>>(n.wsum.as<double>(), n.part.as<float>(), gx, per);
  YG_LAUNCHED();
  std::vector<double> sum(per);
  YG_CUDA(cudaMemcpyAsync(sum.data(), n.wsum.p, sizeof(double) * per, cudaMemcpyDeviceToHost, L.stream));
  check_err(n);
  for (int p = 0; p < kPaths; p++)
    for (int i = 0; i < ci; i++)
      for (int t = 0; t < 4; t++)
        for (int o = 0; o < co; o++)
          for (int s = 0; s < 4; s++) {
            const int m = i * 4 + t, j = o * 4 + s;
            const double *c = sum.data() + ((size_t)p * kM + m) * nb;
            const size_t idx = ((((size_t)p * co + o) * ci + i) * 4 + s) * 4 + t;
            grads[2 * idx] += c[j];
            grads[2 * idx + 1] -= c[4 * co + j];
          }
}

// weight gradients for a loss whose derivative with respect to conj(N(src)) on the even sites
// is gout (an FP64 even-site field): the network runs forward on src / |src| (it is linear,
// N(src) = |src| N(src / |src|)), and the backward pass starts from |src| gout
void ptc_backward(Ptc &n, const double *src, const double *gout, double *grads_out) {
  Lattice &L = *n.L;
  long lo, cnt;
  L.view_range(YG_VIEW_EVEN, lo, cnt);
  const double nr = std::sqrt(blas_sqnorm(L, src, lo, cnt));
  if (!(nr > 0.0)) throw Error(YG_ERR_ARG, "ptc_backward: zero input");
  k_ptc_from_field<<<nblk(L.V, 256), 256, 0, L.stream>>>(n.act[0].as<float>(), (const double2 *)src, (int)L.V,
                                                          (int)L.Vh, 1.0 / nr);
  YG_LAUNCHED();
  forward(n);
  float *gcur = n.g[0].as<float>(), *gnext = n.g[1].as<float>();
  YG_CUDA(cudaMemsetAsync(gcur, 0, planes_bytes(L, n.maxc), L.stream));
  k_ptc_from_field<<<nblk(L.V, 256), 256, 0, L.stream>>>(gcur, (const double2 *)gout, (int)L.V, (int)L.Vh, nr);
  YG_LAUNCHED();
  std::vector<std::vector<double>> grads(n.nl);
  for (int l = 0; l < n.nl; l++) grads[l].assign(n.W[l].size(), 0.0);
  for (int l = n.nl - 1; l >= 0; l--) {
    wgrad(n, l, gcur, grads[l]);
    if (l > 0) {
      ptc_layer(n, l, 1, gcur, gnext);
      std::swap(gcur, gnext);
    }
  }
  check_err(n);
  size_t off = 0;
  for (int l = 0; l < n.nl; l++) {
    std::memcpy(grads_out + off, grads[l].data(), sizeof(double) * grads[l].size());
    off += grads[l].size();
  }
}

double ptc_gradient(Ptc &n, int npairs, double *const *r, double *const *e, double *grads_out) {
  Lattice &L = *n.L;
  long lo, cnt;
  L.view_range(YG_VIEW_EVEN, lo, cnt);
  std::vector<std::vector<double>> grads(n.nl);
  for (int l = 0; l < n.nl; l++) grads[l].assign(n.W[l].size(), 0.0);
  double loss = 0.0;
  const int nbk = nblk(L.V, 256);
  std::vector<double> part(nbk);
  for (int k = 0; k < npairs; k++) {
    const double nr = std::sqrt(blas_sqnorm(L, r[k], lo, cnt));
    const double ne2 = blas_sqnorm(L, e[k], lo, cnt);
    if (!(nr > 0.0) || !(ne2 > 0.0)) throw Error(YG_ERR_ARG, "training pairs must be nonzero");
    // the network is linear: N(r) = |r| N(r / |r|); in units of |r| the target is e / |r|
    k_ptc_from_field<<<nblk(L.V, 256), 256, 0, L.stream>>>(n.act[0].as<float>(), (const double2 *)r[k], (int)L.V,
                                                            (int)L.Vh, 1.0 / nr);
    YG_LAUNCHED();
    forward(n);
    const double inv_ne = nr * nr / ne2;            // 1 / |e / |r||^2
    float *gcur = n.g[0].as<float>(), *gnext = n.g[1].as<float>();
    YG_CUDA(cudaMemsetAsync(gcur, 0, planes_bytes(L, n.maxc), L.stream));
    k_ptc_loss_grad<<<nbk, 256, 0, L.stream>>>(gcur, n.dpart.as<double>(), n.act[n.nl].as<float>(),
                                               (const double2 *)e[k], (int)L.V, (int)L.Vh, inv_ne, 1.0 / nr);
    YG_LAUNCHED();
    YG_CUDA(cudaMemcpyAsync(part.data(), n.dpart.p, sizeof(double) * nbk, cudaMemcpyDeviceToHost, L.stream));
    YG_CUDA(cudaStreamSynchronize(L.stream));
    double d2 = 0.0;
    for (double v : part) d2 += v;
    loss += d2 * inv_ne;
    for (int l = n.nl - 1; l >= 0; l--) {
      wgrad(n, l, gcur, grads[l]);
      if (l > 0) {
        ptc_layer(n, l, 1, gcur, gnext);
        std::swap(gcur, gnext);
      }
    }
    check_err(n);
  }
  size_t off = 0;
  for (int l = 0; l < n.nl; l++) {
    std::memcpy(grads_out + off, grads[l].data(), sizeof(double) * grads[l].size());
    off += grads[l].size();
  }
  return loss;
}

// ---------------------------------------------------------------- flexible GCR
// Right-preconditioned flexible GCR on the even-odd Schur operator Dphi (dirac.cpp:738-751):
// z = M r (the network, or z = r without one), w = D z made orthogonal to the previous w's
// with the same combination applied to the z's, then x += a z, r -= a w, a = <w, r> / <w, w>;
// restarted every `restart` directions with r recomputed as b - D x.  The recursive residual
// decides when to check the true one, and only the true FP64 residual |b - D x|^2 < prec |b|^2
// ends the solve.  If the residual has not halved over 4 restart cycles (a preconditioner that
// does not help), the plain even-odd CG takes over from the current iterate on the normal
// equations Hphi_sq x = Hphi gamma5 b, restarted until the true residual meets prec.
static constexpr int kGcrSlot = 300;      // scratch fields used here: 300 .. 300 + 2 restart + 3

int fgcr(Lattice &L, Ptc *net, const yg_inv_par &par, int restart, double *x, double *b, yg_solve_stats *st) {
  auto t0 = std::chrono::steady_clock::now();
  if (par.op != YG_OP_DPHI) throw Error(YG_ERR_ARG, "fgcr solves Dphi systems");
  if (restart < 1 || restart > 64) throw Error(YG_ERR_ARG, "restart must lie in 1..64");
  if (!L.p.eo) throw Error(YG_ERR_ARG, "fgcr works on the even-odd system");
  if (net && net->L != &L) throw Error(YG_ERR_ARG, "the network belongs to another lattice");
  long lo, n;
  L.view_range(YG_VIEW_DEFAULT, lo, n);
  double *r = L.scratch_field(kGcrSlot), *t = L.scratch_field(kGcrSlot + 1), *u = L.scratch_field(kGcrSlot + 2);
  std::vector<double *> Z(restart), Wv(restart);
  for (int j = 0; j < restart; j++) {
    Z[j] = L.scratch_field(kGcrSlot + 3 + 2 * j);
    Wv[j] = L.scratch_field(kGcrSlot + 4 + 2 * j);
  }
  std::vector<double> wn(restart);
  const double norm = blas_sqnorm(L, b, lo, n);
  const double target = par.prec * norm;
  auto true_residual = [&]() {             // r = b - D x
    blas_copy(L, u, x);
    apply_op(L, YG_OP_DPHI, par.mass, t, u);
    blas_copy(L, r, b);
    blas_axpby(L, r, make_double2(1, 0), make_double2(-1, 0), t, lo, n);
    return blas_sqnorm(L, r, lo, n);
  };
  double rr = norm > 0.0 ? true_residual() : 0.0;
  int it = 0, k = 0, status = YG_OK, fallback = 0, cycles_flat = 0;
  double cycle_start = rr;
  while (rr >= target && norm > 0.0) {
    if (par.maxiter > 0 && it >= par.maxiter) { status = YG_MAXITER; break; }
    if (net) ptc_apply(*net, Z[k], r);
    else blas_copy(L, Z[k], r);
    apply_op(L, YG_OP_DPHI, par.mass, Wv[k], Z[k]);
    for (int j = 0; j < k; j++) {
      const double2 pw = blas_product(L, Wv[k], Wv[j], lo, n);     // <w_j, w_k> = sum conj(w_j) w_k
      const double2 beta = make_double2(pw.x / wn[j], pw.y / wn[j]);
      blas_axpby(L, Wv[k], make_double2(1, 0), make_double2(-beta.x, -beta.y), Wv[j], lo, n);
      blas_axpby(L, Z[k], make_double2(1, 0), make_double2(-beta.x, -beta.y), Z[j], lo, n);
    }
    wn[k] = blas_sqnorm(L, Wv[k], lo, n);
    if (!std::isfinite(wn[k])) throw Error(YG_NONFINITE, "non-finite value in fgcr");
    if (!(wn[k] > 0.0)) { status = YG_STALL; break; }
    const double2 pr = blas_product(L, r, Wv[k], lo, n);            // <w, r> = sum conj(w) r
    const double2 a = make_double2(pr.x / wn[k], pr.y / wn[k]);
    blas_axpby(L, x, make_double2(1, 0), a, Z[k], lo, n);
    blas_axpby(L, r, make_double2(1, 0), make_double2(-a.x, -a.y), Wv[k], lo, n);
    rr = blas_sqnorm(L, r, lo, n);
    it++;
    k++;
    if (rr < target || k == restart) {
      rr = true_residual();               // restart (or confirm convergence) from the true residual
      k = 0;
      if (rr < 0.5 * cycle_start) { cycle_start = rr; cycles_flat = 0; }
      else if (++cycles_flat >= 4) { status = YG_STALL; break; }
    }
  }
  if (status == YG_STALL) {
    // the plain even-odd CG on Hphi_sq x = Hphi gamma5 b from the current iterate
    fallback = 1;
    double *c = L.scratch_field(kGcrSlot + 1);   // t: Hphi (gamma5 b)
    blas_copy(L, u, b);
    blas_g5(L, u, lo, n);
    apply_op(L, YG_OP_HPHI, par.mass, c, u);
    yg_inv_par p2 = par;
    p2.op = YG_OP_HPHI_SQ;
    p2.log = 0;
    double *cb = L.scratch_field(kGcrSlot + 2);
    blas_copy(L, cb, c);
    const double cn = blas_sqnorm(L, cb, lo, n);
    for (int attempt = 0; attempt < 3; attempt++) {
      // the normal-equation residual that gives |b - D x|^2 < prec |b|^2 in the worst case is
      // not known in advance: tighten until the true residual is met
      p2.prec = par.prec * std::pow(1e-2, attempt + 1) * (norm / std::max(cn, 1e-300));
      int it2 = 0;
      status = cg(L, p2, x, cb, &it2);
      it += it2;
      rr = true_residual();
      if (status != YG_OK || rr < target) break;
    }
    if (status == YG_OK && rr >= target) status = YG_STALL;
  }
  YG_CUDA(cudaStreamSynchronize(L.stream));
  if (st) {
    st->iterations = it;
    st->reliable_updates = 0;
    st->fallback = fallback;
    st->true_residual = norm > 0.0 ? rr / norm : 0.0;
    st->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return status;
}

// Hphi_sq x = b through two Dphi solves, as auto_inverter does (inverter.cpp:27-34):
// Hphi_sq = gamma5 D gamma5 D, so D y = gamma5 b, then D x = gamma5 y; each with fgcr and the
// network (prec tightened by 1e-4 for the composition), then the true Hphi_sq residual is the
// judge: if it is above prec the FP64 CG on Hphi_sq finishes from x.
int solve_learned(Lattice &L, Ptc *net, const yg_inv_par &par, int restart, double *x, double *b,
                  yg_solve_stats *st) {
  auto t0 = std::chrono::steady_clock::now();
  if (par.op != YG_OP_HPHI_SQ) throw Error(YG_ERR_ARG, "the learned solve is for Hphi_sq systems");
  long lo, n;
  L.view_range(YG_VIEW_DEFAULT, lo, n);
  double *gb = L.scratch_field(kGcrSlot + 140), *y = L.scratch_field(kGcrSlot + 141);
  double *Ax = L.scratch_field(kGcrSlot + 142), *xc = L.scratch_field(kGcrSlot + 143);
  yg_inv_par pd = par;
  pd.op = YG_OP_DPHI;
  pd.prec = par.prec * 1e-4;
  yg_solve_stats s1{}, s2{};
  blas_copy(L, gb, b);
  blas_g5(L, gb, lo, n);
  blas_zero(L, y, lo, n);
  int st1 = fgcr(L, net, pd, restart, y, gb, &s1);
  blas_g5(L, y, lo, n);
  blas_zero(L, x, lo, n);
  int st2 = fgcr(L, net, pd, restart, x, y, &s2);
  const double norm = blas_sqnorm(L, b, lo, n);
  auto residual = [&]() {
    blas_copy(L, xc, x);
    apply_op(L, YG_OP_HPHI_SQ, par.mass, Ax, xc);
    blas_axpby(L, Ax, make_double2(-1, 0), make_double2(1, 0), b, lo, n);
    return blas_sqnorm(L, Ax, lo, n);
  };
  double rr = residual();
  int it = s1.iterations + s2.iterations, fb = s1.fallback | s2.fallback, status = (st1 != YG_OK) ? st1 : st2;
  if (rr >= par.prec * norm) {
    yg_inv_par p2 = par;
    p2.log = 0;
    int it2 = 0;
    status = cg(L, p2, x, b, &it2);
    it += it2;
    fb |= 2;
    rr = residual();
  }
  if (status == YG_OK && rr >= par.prec * norm) status = YG_STALL;
  YG_CUDA(cudaStreamSynchronize(L.stream));
  if (st) {
    st->iterations = it;
    st->reliable_updates = 0;
    st->fallback = fb;
    st->true_residual = rr / norm;
    st->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return status;
}

}  // namespace yg
