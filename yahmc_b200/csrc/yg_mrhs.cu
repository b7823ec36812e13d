// Several right-hand sides of the mixed-precision CG sharing every inner operator launch.
//
// cg_inverter (cg.cpp:132-202) solves one system at a time and so reads the links and the
// clover term once per right-hand side and operator application.  The inner operator of
// the mixed CG reads, per output site, 384 B of links (8 x 12 FP32 reals), 288 B of packed
// clover blocks and 2 x 52 B of FP16 spinor (with its norm): for n systems solved one at a
// time that is n x 776 B.  Here one thread takes one site and a tile of up to R systems:
// it loads each link once, rebuilds its third row once, and applies it to the R spinors
// before moving on, so n systems cost 672 + n x 104 B per site (1920 B for n = 12, a
// quarter of 12 x 776).  Tiles of the same sites sit in consecutive blocks, so when n > R
// the other tiles find the links in L2.
//
// Every system keeps its own fields in the single-system formats (FP16 spinors with per-site
// norms for p, Hphi p and the intermediates; FP32 x and r; A p = Hphi Hphi p is never stored:
// r -= alpha A p and the |r|^2 partials are the epilogue of the operator's last step, and
// x += alpha p rides with p = r + beta p), its own device scalars (|r|^2 in two alternating
// slots, alpha, beta), its own mass (the packed clover blocks are per launch slot, so the HMC
// and Hasenbusch monomials' solves at m + dm and m share the launches), and the
// single-system rules: reliable updates with the FP64 operator when |r| has fallen by delta or
// stagnates, a stop on the TRUE FP64 residual |b - A x|^2 < prec |b|^2, and a fall-back to the
// FP64 CG on a stall.  All reductions are deterministic: per-block partials summed in index
// order by one warp per system.  The host reads each iteration's |r|^2 values one iteration
// late from mapped memory while the next iteration runs, as the single-system solver does.
#include <cuda_fp16.h>
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>
#include "yg_lattice.h"
#include "yg_kernels.h"
#include "yg_sloppy_impl.cuh"

namespace yg {

namespace {

constexpr int kMR = 16;       // systems per call (kMaxRhs of the batched solvers)
constexpr int kMaxMasses = 4; // distinct masses per call
constexpr int kHopThreads = 128;
constexpr int kVecThreads = 256;

// FP16 spinor words and per-site norms of one field per system
struct MSpin {
  void *d[kMR];
  float *n[kMR];
};

struct MHopArgs {
  Geom g;
  MSpin src, src2, dst;
  const void *U;            // FP32 links, K complex words each
  const void *C[kMR];       // FP32 packed clover blocks (M_e even, M_o^-1 odd) of slot j's mass, 18 float4 per site
  float coeff;
  int lo, n;                // output sites [lo, lo + n)
  int nsys, ntile;
  double *part;             // NRM: part[j * nsb + site block] = sum of |dst_j|^2 (NRM 1) or of the new
  int nsb;                  //   |r_j|^2 (NRM 2) over the block
  // NRM = 2, the last step of the iteration's second Hphi: the residual update of launch
  // slot j (r_j -= alpha q_j with q_j = the step's output, never stored)
  float2 *r[kMR];           // FP32 even-site words
  const double *scal;
  int sys[kMR];             // global system index of launch slot j (its scalars)
};

// Device scalars of system i: scal[i * kW + M_*] (M_RR0/M_RR1 alternate with the iteration
// parity, as in the single-system solver), plus the next beta.
enum { M_RR0 = 0, M_RR1 = 1, M_ALPHA = 2, M_PQ = 3, M_BETA = 4, kW = 8 };

template <int MU, int SIG>
__device__ __forceinline__ void project(float2 (&hh)[2][3], const float2 (&p)[12]) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float2 p0 = p[c], p1 = p[3 + c], p2 = p[6 + c], p3 = p[9 + c];
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
}

template <int MU, int SIG>
__device__ __forceinline__ void reconstruct(float2 (&acc)[12], const float2 (&chi)[2][3]) {
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

// one direction for the rc <= R systems of the thread's tile: the link is loaded (and its
// third row rebuilt) once, then applied to every system's projected neighbour spinor
template <int K, int R, int MU, int SIG>
__device__ __forceinline__ void mhop_dir(float2 (&acc)[R][12], const MHopArgs &a, int s0, int rc, int nid, int lid,
                                         int lt) {
  const Geom &g = a.g;
  const int nbk = nid >= g.Vh, nh = nid - nbk * g.Vh;
  const int lb = lid >= g.Vh, lh = lid - lb * g.Vh;
  const float sgn = (g.bc == YG_BC_ANTIPERIODIC && MU == 0 && lt == 0) ? -1.f : 1.f;
  float2 u[9];
  link_load<ST_F32, K>(u, a.U, lb, lh, g.Vh, MU, sgn);
#pragma unroll
  for (int r = 0; r < R; r++) {
    if (r < rc) {
      float2 p[12];
      sload_raw<16>(p, a.src.d[s0 + r], nbk, nh, g.Vh);
      const float pn = __ldg(a.src.n[s0 + r] + (long)nbk * g.Vh + nh);
      float2 hh[2][3];
      project<MU, SIG>(hh, p);
      float2 chi[2][3];
#pragma unroll
      for (int i = 0; i < 3; i++) {
        float2 c0 = make_float2(0.f, 0.f), c1 = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 3; j++) {
          if (SIG > 0) { cfmac(c0, u[j * 3 + i], hh[0][j]); cfmac(c1, u[j * 3 + i], hh[1][j]); }
          else { cfma(c0, u[i * 3 + j], hh[0][j]); cfma(c1, u[i * 3 + j], hh[1][j]); }
        }
        chi[0][i] = cscale(c0, pn);
        chi[1][i] = cscale(c1, pn);
      }
      reconstruct<MU, SIG>(acc[r], chi);
    }
  }
}

// y = M x for block b (spins 2b, 2b+1) of a site's packed FP32 record, read from memory
__device__ __forceinline__ void herm_block(float2 (&y)[6], const float4 *C, int blk, int h, int Vh, int b,
                                           const float2 (&x)[6]) {
  float c[36];
#pragma unroll
  for (int w = 0; w < 9; w++) {
    const float4 v = __ldg(C + (long)(blk * 18 + 9 * b + w) * Vh + h);
    c[4 * w] = v.x; c[4 * w + 1] = v.y; c[4 * w + 2] = v.z; c[4 * w + 3] = v.w;
  }
#pragma unroll
  for (int i = 0; i < 6; i++) y[i] = cscale(x[i], c[i]);
  int k = 6;
#pragma unroll
  for (int i = 1; i < 6; i++)
#pragma unroll
    for (int j = 0; j < i; j++, k += 2) {
      const float2 m = make_float2(c[k], c[k + 1]);
      cfma(y[i], m, x[j]);
      cfmac(y[j], m, x[i]);
    }
}

// STEP 1 (odd output):  dst_j = M_o^-1 (coeff hop(src_j))
// STEP 2 (even output): dst_j = gamma5 (M_e src2_j + coeff hop(src_j))
// the single-system compressed operator (shop_site of yg_sloppy.cu) for a tile of systems
// resident blocks per SM the register budget is cut for: 6 (R = 1), 4 (R = 2), 3 (R = 4)
template <int R> struct MinBlocks { static constexpr int value = R == 1 ? 6 : R == 2 ? 4 : 3; };

// SPLIT = 2: two neighbouring threads share a site, one taking the directions mu = 0, 1 and the
// other mu = 2, 3; their accumulators are added with one shuffle per word and each then finishes
// half of the tile's systems.  Twice the threads per site hide the latency of the gathers of a
// register-heavy tile.
template <int K, int R, int STEP, int NRM, int SPLIT>
__global__ void __launch_bounds__(kHopThreads, MinBlocks<R>::value) k_mhop(MHopArgs a) {
  constexpr int SITES = kHopThreads / SPLIT;              // sites per block
  const int tile = blockIdx.x % a.ntile, sb = blockIdx.x / a.ntile;
  const int s0 = tile * R;
  const int rc = min(R, a.nsys - s0);
  const int part = SPLIT == 2 ? (threadIdx.x & 1) : 0;
  const int t = sb * SITES + threadIdx.x / SPLIT;
  const Geom &g = a.g;
  float n2[R];
#pragma unroll
  for (int r = 0; r < R; r++) n2[r] = 0.f;
  const bool live = t < a.n;
  const int id = a.lo + (live ? t : 0);
  SiteNbr nb;
  site_nbr(nb, g, id);
  const int T = g.dim[0], t0 = nb.c[0];
  float2 acc[R][12];
#pragma unroll
  for (int r = 0; r < R; r++)
#pragma unroll
    for (int k = 0; k < 12; k++) acc[r][k] = make_float2(0.f, 0.f);
  if (live) {
    if (SPLIT == 1 || part == 0) {
      mhop_dir<K, R, 0, -1>(acc, a, s0, rc, nb.f[0], id, t0);
      mhop_dir<K, R, 0, +1>(acc, a, s0, rc, nb.b[0], nb.b[0], t0 == 0 ? T - 1 : t0 - 1);
      mhop_dir<K, R, 1, -1>(acc, a, s0, rc, nb.f[1], id, t0);
      mhop_dir<K, R, 1, +1>(acc, a, s0, rc, nb.b[1], nb.b[1], t0);
    }
    if (SPLIT == 1 || part == 1) {
      mhop_dir<K, R, 2, -1>(acc, a, s0, rc, nb.f[2], id, t0);
      mhop_dir<K, R, 2, +1>(acc, a, s0, rc, nb.b[2], nb.b[2], t0);
      mhop_dir<K, R, 3, -1>(acc, a, s0, rc, nb.f[3], id, t0);
      mhop_dir<K, R, 3, +1>(acc, a, s0, rc, nb.b[3], nb.b[3], t0);
    }
  }
  if (SPLIT == 2) {
    // every lane takes part (the pair of a dead site holds zeros)
#pragma unroll
    for (int r = 0; r < R; r++)
#pragma unroll
      for (int k = 0; k < 12; k++) {
        acc[r][k].x += __shfl_xor_sync(0xffffffffu, acc[r][k].x, 1);
        acc[r][k].y += __shfl_xor_sync(0xffffffffu, acc[r][k].y, 1);
      }
  }
  if (live) {
    const int blk = id >= g.Vh, h = id - blk * g.Vh;
    const bool bnd = spinor_zeroed(g, t0);
#pragma unroll
    for (int r = 0; r < R; r++) {
      if (r < rc && (SPLIT == 1 || (r & 1) == part)) {
        const float4 *C = reinterpret_cast<const float4 *>(a.C[s0 + r]);
        float2 in[12], out[12];
        if (STEP == 1) {
#pragma unroll
          for (int k = 0; k < 12; k++) in[k] = cscale(acc[r][k], a.coeff);
        } else {
          sload<16>(in, a.src2.d[s0 + r], a.src2.n[s0 + r], blk, h, g.Vh);
        }
#pragma unroll
        for (int b = 0; b < 2; b++) {
          float2 x[6], y[6];
#pragma unroll
          for (int i = 0; i < 3; i++) {
            x[i] = in[(2 * b) * 3 + i];
            x[i + 3] = in[(2 * b + 1) * 3 + i];
          }
          herm_block(y, C, blk, h, g.Vh, b, x);
#pragma unroll
          for (int i = 0; i < 3; i++) {
            out[(2 * b) * 3 + i] = y[i];
            out[(2 * b + 1) * 3 + i] = y[i + 3];
          }
        }
        float sq = 0.f;
#pragma unroll
        for (int k = 0; k < 12; k++) {
          if (STEP == 2) {
            out[k] = cadd(out[k], cscale(acc[r][k], a.coeff));
            if (k >= 6) out[k] = cscale(out[k], -1.f);      // gamma5
          }
          if (bnd) out[k] = make_float2(0.f, 0.f);
          if (NRM != 2) sq = fmaf(out[k].x, out[k].x, fmaf(out[k].y, out[k].y, sq));
        }
        if constexpr (NRM == 2) {
          // r -= alpha q on the (even) site, |r|^2 of the site (x += alpha p rides with
          // p = r + beta p in k_m_xpay, which reads p anyway)
          const float al = (float)a.scal[a.sys[s0 + r] * kW + M_ALPHA];
          float2 *rs = a.r[s0 + r];
#pragma unroll
          for (int k = 0; k < 12; k++) {
            const long i = (long)k * g.Vh + h;
            float2 ri = rs[i];
            ri.x = fmaf(-al, out[k].x, ri.x);
            ri.y = fmaf(-al, out[k].y, ri.y);
            rs[i] = ri;
            sq = fmaf(ri.x, ri.x, fmaf(ri.y, ri.y, sq));
          }
        } else {
          sstore<16>(a.dst.d[s0 + r], a.dst.n[s0 + r], out, blk, h, g.Vh);
        }
        n2[r] = sq;
      }
    }
  }
  if (NRM) {
#pragma unroll
    for (int r = 0; r < R; r++) {
      const double v = block_total((double)n2[r]);
      if (threadIdx.x == 0 && r < rc) a.part[(long)(s0 + r) * a.nsb + sb] = v;
    }
  }
}

// ---- per-system vectors and scalars

struct MVec {
  float2 *x[kMR];           // FP32 inner solution increments
  float2 *r[kMR];           // FP32 iterated residuals
  MSpin p;
  int sys[kMR];             // global system index of launch slot j
  int nsys;
};

// one warp per launch slot: the slot's n partials summed in index order
__device__ __forceinline__ double warp_sum(const double *part, int n) {
  const int lane = threadIdx.x & 31;
  double v = 0.0;
  for (int i = lane; i < n; i += 32) v += part[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// alpha_i = |r_i|^2 / <p_i, A p_i> from the NRM hop's partials
__global__ void k_m_alpha(double *scal, const double *part, int nsb, MVec v, int par) {
  const int j = threadIdx.x >> 5;
  if (j >= v.nsys) return;
  const double pq = warp_sum(part + (long)j * nsb, nsb);
  if ((threadIdx.x & 31) == 0) {
    double *s = scal + v.sys[j] * kW;
    s[M_PQ] = pq;
    s[M_ALPHA] = s[M_RR0 + par] / pq;
  }
}

// |r_i|^2 from the update's partials, beta_i = |r_i|^2 / |r_i,old|^2; the values go to the
// next slot, to hist[2 i + (par ^ 1)] (mapped host memory), then the iteration number to *seq
__global__ void k_m_beta(double *scal, const double *part, int n, MVec v, int par, double *hist,
                         unsigned long long *seq, unsigned long long iter) {
  const int j = threadIdx.x >> 5;
  if (j < v.nsys) {
    const double rr = warp_sum(part + (long)j * n, n);
    if ((threadIdx.x & 31) == 0) {
      double *s = scal + v.sys[j] * kW;
      s[M_BETA] = rr / s[M_RR0 + par];
      s[M_RR0 + (par ^ 1)] = rr;
      reinterpret_cast<volatile double *>(hist)[2 * v.sys[j] + (par ^ 1)] = rr;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence_system();
    *reinterpret_cast<volatile unsigned long long *>(seq) = iter;
  }
}

// x_i += alpha_i p_i ; p_i = r_i + beta_i p_i
__global__ void __launch_bounds__(kVecThreads) k_m_xpay(const double *scal, MVec v, int Vh) {
  const int j = blockIdx.y;
  const float b = (float)scal[v.sys[j] * kW + M_BETA];
  const float al = (float)scal[v.sys[j] * kW + M_ALPHA];
  const float2 *r = v.r[j];
  float2 *x = v.x[j];
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += gridDim.x * blockDim.x) {
    float2 pp[12];
    sload<16>(pp, v.p.d[j], v.p.n[j], 0, h, Vh);
#pragma unroll
    for (int k = 0; k < 12; k++) {
      const long i = (long)k * Vh + h;
      const float2 ri = r[i];
      float2 xi = x[i];
      xi.x = fmaf(al, pp[k].x, xi.x);                 // x += alpha p with this iteration's p
      xi.y = fmaf(al, pp[k].y, xi.y);
      x[i] = xi;
      pp[k] = make_float2(fmaf(b, pp[k].x, ri.x), fmaf(b, pp[k].y, ri.y));
    }
    sstore<16>(v.p.d[j], v.p.n[j], pp, 0, h, Vh);
  }
}

// p_i = r_i (FP32 -> FP16 with norms) for the systems of the launch
__global__ void __launch_bounds__(kVecThreads) k_m_p_from_r(MVec v, int Vh) {
  const int j = blockIdx.y;
  const float2 *r = v.r[j];
  for (int h = blockIdx.x * blockDim.x + threadIdx.x; h < Vh; h += gridDim.x * blockDim.x) {
    float2 pp[12];
#pragma unroll
    for (int k = 0; k < 12; k++) pp[k] = r[(long)k * Vh + h];
    sstore<16>(v.p.d[j], v.p.n[j], pp, 0, h, Vh);
  }
}

__global__ void k_m_set(double *scal, int i, double v) { scal[i] = v; }

// an FP16 field of the compressed operator: 3 words of 16 B per site and one FP32 norm
struct HField {
  void *d;
  float *n;
};

// per-system working storage, carved from one allocation kept on the lattice
struct SysBufs {
  float2 *fx, *fr;          // FP32 even-site words (12 complex per site)
  HField p, t, o;           // FP16 fields of the whole lattice (p, t = Hphi p on even sites, o odd)
  double *xbest;            // FP64 copy of the best iterate (whole field)
};

size_t align256(size_t n) { return (n + 255) & ~(size_t)255; }

size_t sys_bytes(const Lattice &L) {
  const size_t vh = (size_t)L.Vh;
  return 2 * align256(96 * vh) + 3 * (align256(96 * vh) + align256(8 * vh)) + align256(L.field_bytes());
}

SysBufs sys_bufs(Lattice &L, int i) {
  char *p = L.mr_work.as<char>() + (size_t)i * sys_bytes(L);
  const size_t vh = (size_t)L.Vh;
  SysBufs b;
  b.fx = reinterpret_cast<float2 *>(p); p += align256(96 * vh);
  b.fr = reinterpret_cast<float2 *>(p); p += align256(96 * vh);
  for (HField *f : {&b.p, &b.t, &b.o}) {
    f->d = p; p += align256(96 * vh);
    f->n = reinterpret_cast<float *>(p); p += align256(8 * vh);
  }
  b.xbest = reinterpret_cast<double *>(p);
  return b;
}

int vec_grid(int sms) { return sms * 4; }

// the two Schur steps of the inner operator for a launch's systems, R systems per thread,
// SPLIT threads per site
// mode of the second step: 0 plain, 1 with the |dst|^2 partials, 2 with the CG update
template <int K, int R, int SPLIT>
void launch_mhop_r(Lattice &L, const MHopArgs &a0, const MHopArgs &b0, int mode) {
  MHopArgs a = a0, b = b0;
  a.nsb = b.nsb = nblk(a.n, kHopThreads / SPLIT);
  const int grid = a.ntile * a.nsb;
  k_mhop<K, R, 1, 0, SPLIT><<<grid, kHopThreads, 0, L.stream>>>(a);
  YG_LAUNCHED();
  if (mode == 1) k_mhop<K, R, 2, 1, SPLIT><<<grid, kHopThreads, 0, L.stream>>>(b);
  else if (mode == 2) k_mhop<K, R, 2, 2, SPLIT><<<grid, kHopThreads, 0, L.stream>>>(b);
  else k_mhop<K, R, 2, 0, SPLIT><<<grid, kHopThreads, 0, L.stream>>>(b);
  YG_LAUNCHED();
}

// the inner-operator variants the tuner chooses among: (systems per thread, threads per site)
constexpr int kVariants[5][2] = {{1, 1}, {2, 1}, {4, 1}, {2, 2}, {4, 2}};

template <int K>
void launch_mhop_k(Lattice &L, int var, const MHopArgs &a, const MHopArgs &b, int mode) {
  switch (var) {
    case 0: launch_mhop_r<K, 1, 1>(L, a, b, mode); break;
    case 1: launch_mhop_r<K, 2, 1>(L, a, b, mode); break;
    case 2: launch_mhop_r<K, 4, 1>(L, a, b, mode); break;
    case 3: launch_mhop_r<K, 2, 2>(L, a, b, mode); break;
    default: launch_mhop_r<K, 4, 2>(L, a, b, mode); break;
  }
}

void launch_mhop(Lattice &L, int reals, int var, const MHopArgs &a, const MHopArgs &b, int mode) {
  if (reals == 12) launch_mhop_k<6>(L, var, a, b, mode);
  else launch_mhop_k<9>(L, var, a, b, mode);
}

}  // namespace

int cg(Lattice &L, const yg_inv_par &par, double *x, double *b, int *iters);

int cg_mixed_mrhs(Lattice &L, const yg_inv_par &par, int nrhs, double *const *xs, double *const *bs, double delta,
                  yg_solve_stats *stats, const double *masses) {
  auto t0 = std::chrono::steady_clock::now();
  if (par.op != YG_OP_HPHI_SQ) throw Error(YG_ERR_ARG, "the multi-system mixed CG solves Hphi_sq systems");
  if (nrhs < 1 || nrhs > kMR) throw Error(YG_ERR_ARG, "1..16 right-hand sides");
  if (!L.p.eo) throw Error(YG_ERR_ARG, "the multi-system mixed CG needs even-odd preconditioning");
  if (L.d != 3) throw Error(YG_ERR_ARG, "the compressed inner operator exists for d = 3 representations");
  if (!(delta > 0.0 && delta < 1.0)) throw Error(YG_ERR_ARG, "reliable-update delta must lie in (0,1)");
  for (int i = 0; i < nrhs; i++) {
    if (xs[i] == bs[i]) throw Error(YG_ERR_ARG, "a solution field must differ from its source");
    for (int k = 0; k < i; k++)
      if (xs[i] == xs[k] || xs[i] == bs[k] || bs[i] == xs[k])
        throw Error(YG_ERR_ARG, "solution fields must be distinct from each other and from the sources");
  }
  const int nb = nrhs;
  const bool su3 = L.nc == 3 && L.p.repr == YG_REPR_FUNDAMENTAL;
  int reals = su3 ? 12 : 18;               // link reals of the inner operator (tuned below for SU(3))
  // the mass of each system (masses == nullptr: par.mass for all); the first one's clover
  // blocks are the lattice's own inner-operator copy, every other distinct mass gets a
  // packed set of its own, rebuilt on each call (a few hop times)
  std::vector<double> mass(nb, par.mass);
  if (masses)
    for (int i = 0; i < nb; i++) {
      if (!std::isfinite(masses[i])) throw Error(YG_ERR_ARG, "masses must be finite");
      mass[i] = masses[i];
    }
  std::vector<double> dist;
  for (double mv : mass)
    if (std::find(dist.begin(), dist.end(), mv) == dist.end()) dist.push_back(mv);
  if ((int)dist.size() > kMaxMasses) throw Error(YG_ERR_ARG, "at most 4 distinct masses per call");
  const size_t clov_bytes = sizeof(float) * 72 * (size_t)L.V;
  if (dist.size() > 1) {
    L.mr_clov.alloc(clov_bytes * (dist.size() - 1) + sizeof(float) * (size_t)L.V);
    for (size_t k = 1; k < dist.size(); k++)
      pack_clover_f32(L, dist[k], L.mr_clov.as<char>() + clov_bytes * (k - 1),
                      reinterpret_cast<float *>(L.mr_clov.as<char>() + clov_bytes * (dist.size() - 1)));
  }
  ensure_sloppy(L, dist[0], 16, reals, 32, 32);
  std::vector<const void *> clov(nb);
  for (int i = 0; i < nb; i++) {
    const size_t k = std::find(dist.begin(), dist.end(), mass[i]) - dist.begin();
    clov[i] = k == 0 ? L.sl_clover.p : L.mr_clov.as<char>() + clov_bytes * (k - 1);
  }

  int dev = 0, sms = 0;
  YG_CUDA(cudaGetDevice(&dev));
  YG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int Vh = (int)L.Vh;
  const int nsb_max = nblk(Vh, kHopThreads / 2);  // partials per system, most for two threads a site
  const int gv = std::min(vec_grid(sms), nblk(Vh, kVecThreads));
  if (L.mr_cap < nb) {
    L.mr_work.release();
    L.mr_work.alloc(sys_bytes(L) * kMR);
    L.mr_cap = kMR;
  }
  if (!L.mr_hist) {
    YG_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&L.mr_hist), (2 * kMR + 8) * sizeof(double),
                          cudaHostAllocMapped));
    L.mr_scal.alloc(sizeof(double) * kMR * kW);
    YG_CUDA(cudaMemsetAsync(L.mr_scal.p, 0, sizeof(double) * kMR * kW, L.stream));
  }
  const size_t part_words = (size_t)kMR * std::max(nsb_max, gv);
  if (L.mr_part.bytes < 2 * part_words * sizeof(double)) {
    L.mr_part.release();
    L.mr_part.alloc(2 * part_words * sizeof(double));
  }
  double *part_pq = L.mr_part.as<double>(), *part_r = part_pq + part_words;
  double *scal = L.mr_scal.as<double>();
  volatile double *hist = L.mr_hist;
  unsigned long long *seq = reinterpret_cast<unsigned long long *>(L.mr_hist + 2 * kMR);
  *reinterpret_cast<volatile unsigned long long *>(seq) = 0;     // nothing of this lattice is in flight here

  long lo, n;
  L.view_range(YG_VIEW_DEFAULT, lo, n);
  const long cnt = n * 4L * L.d;
  std::vector<SysBufs> sb(nb);
  for (int i = 0; i < nb; i++) sb[i] = sys_bufs(L, i);
  double *r64 = L.scratch_field(3), *Ax = L.scratch_field(4), *xd = L.scratch_field(5);

  auto residual = [&](int i) {      // r64 = b_i - A x_i in FP64, returns |r|^2
    blas_copy(L, xd, xs[i]);
    apply_op(L, YG_OP_HPHI_SQ, mass[i], Ax, xd);
    blas_copy(L, r64, bs[i]);
    blas_axpby(L, r64, make_double2(1, 0), make_double2(-1, 0), Ax, lo, n);
    return blas_sqnorm(L, r64, lo, n);
  };
  auto set_scalar = [&](int idx, double v) {
    k_m_set<<<1, 1, 0, L.stream>>>(scal, idx, v);
    YG_LAUNCHED();
  };

  std::vector<double> norm(nb), target(nb), rr(nb), best(nb), maxrr(nb), min_cycle(nb);
  std::vector<int> its(nb, 0), updates(nb, 0), stall(nb, 0), since(nb, 0), skip(nb, 0), fallback(nb, 0);
  std::vector<int> act;
  int it = 0;
  for (int i = 0; i < nb; i++) {
    norm[i] = blas_sqnorm(L, bs[i], lo, n);
    target[i] = norm[i] * par.prec;
    rr[i] = residual(i);
    best[i] = maxrr[i] = min_cycle[i] = rr[i];
    blas_copy(L, sb[i].xbest, xs[i]);
    if (!(rr[i] < target[i])) {
      f_from_d(L, reinterpret_cast<float *>(sb[i].fr), r64, cnt);
      YG_CUDA(cudaMemsetAsync(sb[i].fx, 0, sizeof(float2) * cnt, L.stream));
      set_scalar(i * kW + M_RR0, rr[i]);
      act.push_back(i);
    }
  }

  auto fill = [&](MVec &v) {
    v.nsys = (int)act.size();
    for (int j = 0; j < v.nsys; j++) {
      const SysBufs &b = sb[act[j]];
      v.x[j] = b.fx;
      v.r[j] = b.fr;
      v.p.d[j] = b.p.d; v.p.n[j] = b.p.n;
      v.sys[j] = act[j];
    }
  };
  int var = 2;                                // index into kVariants
  // t = Hphi p (first; mode 1 adds the <p, A p> partials) or Hphi t (second; mode 2 fuses the
  // residual update, r -= alpha Hphi t, with the |r|^2 partials), o the odd sites
  auto hphi = [&](int mode, bool second) {
    MHopArgs a{};
    a.g = L.g;
    a.U = L.sl_links.p;
    a.nsys = (int)act.size();
    const int tile = kVariants[var][0];
    a.ntile = (a.nsys + tile - 1) / tile;
    a.part = mode == 2 ? part_r : part_pq;
    a.scal = scal;
    MHopArgs b = a;
    for (int j = 0; j < a.nsys; j++) {
      const SysBufs &s = sb[act[j]];
      const HField in = second ? s.t : s.p;
      a.src.d[j] = in.d; a.src.n[j] = in.n;
      a.dst.d[j] = s.o.d; a.dst.n[j] = s.o.n;
      b.src.d[j] = s.o.d; b.src.n[j] = s.o.n;
      b.src2.d[j] = in.d; b.src2.n[j] = in.n;
      b.dst.d[j] = second ? nullptr : s.t.d;         // the second Hphi stores no output
      b.dst.n[j] = second ? nullptr : s.t.n;
      a.C[j] = clov[act[j]];
      b.C[j] = clov[act[j]];
      b.r[j] = s.fr;
      b.sys[j] = act[j];
    }
    a.coeff = 0.5f; a.lo = Vh; a.n = Vh;
    b.coeff = -0.5f; b.lo = 0; b.n = Vh;
    launch_mhop(L, reals, var, a, b, mode);
    L.mvm += 2 * a.nsys;
  };
  auto wait_iteration = [&](unsigned long long k) {
    volatile unsigned long long *sq = seq;
    if (*sq >= k) return;
    auto w0 = std::chrono::steady_clock::now();
    while (*sq < k) {
      const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
      if (dt > 1e-3) std::this_thread::yield();
      if (dt > 30.0) {
        YG_CUDA(cudaStreamSynchronize(L.stream));
        if (*sq < k) throw Error(YG_TIMEOUT, "cg_mixed_multi: the inner iteration counter stopped advancing");
        return;
      }
    }
  };

  if (!act.empty()) {
    MVec v{};
    fill(v);
    k_m_p_from_r<<<dim3(gv, v.nsys), kVecThreads, 0, L.stream>>>(v, Vh);
    YG_LAUNCHED();
  }
  // the tile (systems per thread), the threads per site and, for SU(3) fundamental links, the
  // link format (12 reals with the third row rebuilt, or all 18: the operator is bound by
  // instruction issue, so the rebuild can cost more than the bytes it saves): measured once
  // per lattice and system count on the current fields (one Hphi of each candidate, after a
  // warm-up launch).  mr_tile[ns] = variant + 1, plus 8 for 18-real links.
  if (!act.empty()) {
    const int ns = (int)act.size();
    if (L.mr_tile[ns] == 0) {
      cudaEvent_t e0, e1;
      YG_CUDA(cudaEventCreate(&e0));
      YG_CUDA(cudaEventCreate(&e1));
      float best_ms = 0.f;
      int best = 2, best_reals = reals, calls = 0;
      for (int lr : {12, 18}) {
        if (lr == 12 && !su3) continue;
        reals = lr;
        ensure_sloppy(L, dist[0], 16, reals, 32, 32);
        for (int cand = 0; cand < 5; cand++) {
          const int r = kVariants[cand][0];
          if (r > 1 && r >= 2 * ns) continue;
          var = cand;
          calls += 4;
          hphi(0, false);                        // warm-up; t only (p untouched)
          YG_CUDA(cudaEventRecord(e0, L.stream));
          for (int rep = 0; rep < 3; rep++) hphi(0, false);
          YG_CUDA(cudaEventRecord(e1, L.stream));
          YG_CUDA(cudaEventSynchronize(e1));
          float ms = 0.f;
          YG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
          if (best_ms == 0.f || ms < best_ms) { best_ms = ms; best = cand; best_reals = lr; }
          if (std::getenv("YG_TUNE_LOG"))
            std::fprintf(stderr,
                         "yg tune cg_mixed_multi: %d systems, %d-real links, %d per thread, %d-way direction split: "
                         "%.3f ms/Hphi\n", ns, lr, r, kVariants[cand][1], ms / 3.f);
        }
      }
      YG_CUDA(cudaEventDestroy(e0));
      YG_CUDA(cudaEventDestroy(e1));
      L.mvm -= 2 * ns * calls;                   // the timing launches are not MVMs of the solve
      L.mr_tile[ns] = best + 1 + (best_reals == 18 && su3 ? 8 : 0);
    }
    const int code = L.mr_tile[ns] - 1;
    var = code & 7;
    reals = (code & 8) || !su3 ? 18 : 12;
    ensure_sloppy(L, dist[0], 16, reals, 32, 32);
  }
  const double d2 = delta * delta;
  constexpr int kStagnate = 100;   // as the single-system solver: force an update after 100 flat iterations
  int status = YG_OK;
  bool pending = false;
  while (!act.empty()) {
    if (par.maxiter > 0 && it >= par.maxiter) {
      for (int i : act) d_add_f(L, xs[i], reinterpret_cast<float *>(sb[i].fx), cnt);
      status = YG_MAXITER;
      break;
    }
    const int parity = it & 1;
    MVec v{};
    fill(v);
    const int nsb = nblk(Vh, kHopThreads / kVariants[var][1]);     // site blocks of an operator launch
    hphi(1, false);
    k_m_alpha<<<1, 32 * v.nsys, 0, L.stream>>>(scal, part_pq, nsb, v, parity);
    YG_LAUNCHED();
    hphi(2, true);
    k_m_beta<<<1, 32 * v.nsys, 0, L.stream>>>(scal, part_r, nsb, v, parity, const_cast<double *>(hist), seq,
                                              (unsigned long long)it + 1);
    YG_LAUNCHED();
    k_m_xpay<<<dim3(gv, v.nsys), kVecThreads, 0, L.stream>>>(scal, v, Vh);
    YG_LAUNCHED();
    for (int i : act) its[i]++;
    it++;
    if (!pending) { pending = true; continue; }
    // the previous iteration's |r_i|^2, read while this one runs
    wait_iteration((unsigned long long)it - 1);
    std::vector<int> upd;
    for (int i : act) {
      if (skip[i]) { skip[i] = 0; continue; }
      const double rp = hist[2 * i + ((it - 1) & 1)];   // written by iteration it - 2
      if (!std::isfinite(rp)) throw Error(YG_NONFINITE, "non-finite value in cg_mixed_multi");
      if (rp < 0.25 * min_cycle[i]) { min_cycle[i] = rp; since[i] = 0; }
      else since[i]++;
      if (rp < d2 * maxrr[i] || rp < target[i] || since[i] >= kStagnate) upd.push_back(i);
    }
    if (upd.empty()) continue;
    // reliable updates on the state after the iteration just enqueued
    std::vector<int> done;
    for (int i : upd) {
      d_add_f(L, xs[i], reinterpret_cast<float *>(sb[i].fx), cnt);
      YG_CUDA(cudaMemsetAsync(sb[i].fx, 0, sizeof(float2) * cnt, L.stream));
      const double rt = residual(i);
      updates[i]++;
      rr[i] = rt;
      bool stop = false;
      if (rt < target[i]) stop = true;
      else {
        if (rt < best[i]) blas_copy(L, sb[i].xbest, xs[i]);
        if (rt > 100.0 * best[i]) { fallback[i] = 1; stop = true; }          // the inner solve diverged
        else if (rt < 0.5 * best[i]) stall[i] = 0;
        else if (++stall[i] >= 8) { fallback[i] = 1; stop = true; }
        best[i] = std::min(best[i], rt);
      }
      if (stop) { done.push_back(i); continue; }
      f_from_d(L, reinterpret_cast<float *>(sb[i].fr), r64, cnt);
      set_scalar(i * kW + M_RR0 + (it & 1), rt);      // the slot the next iteration reads
      maxrr[i] = min_cycle[i] = rt;
      since[i] = 0;
      skip[i] = 1;                                     // its enqueued |r|^2 predates the update
    }
    for (int i : done) act.erase(std::find(act.begin(), act.end(), i));
  }
  YG_CUDA(cudaStreamSynchronize(L.stream));
  // systems that stalled: the FP64 CG from their best iterate, restarted until the true
  // residual meets prec (its recursive residual can stop above it)
  for (int i = 0; i < nb; i++) {
    if (!fallback[i]) continue;
    blas_copy(L, xs[i], sb[i].xbest);
    yg_inv_par p64 = par;
    p64.log = 0;
    p64.mass = mass[i];
    int st = YG_OK;
    for (int attempt = 0; attempt < 3; attempt++) {
      int it64 = 0;
      st = cg(L, p64, xs[i], bs[i], &it64);
      its[i] += it64;
      rr[i] = residual(i);
      if (st != YG_OK || rr[i] < target[i]) break;
    }
    if (st != YG_OK && status == YG_OK) status = st;
  }
  YG_CUDA(cudaStreamSynchronize(L.stream));
  const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  for (int i = 0; i < nb; i++) {
    if (status == YG_OK && !(rr[i] < target[i])) status = YG_STALL;
    if (stats) {
      stats[i].iterations = its[i];
      stats[i].reliable_updates = updates[i];
      stats[i].fallback = fallback[i];
      stats[i].true_residual = rr[i] / norm[i];
      stats[i].seconds = secs;
    }
    if (par.log)
      fprintf(stderr, "[INVERTER][30]cg_mixed_multi[%d]: iterations = %d, precision = %1.4e\n", i, its[i],
              rr[i] / norm[i]);
  }
  return status;
}

}  // namespace yg
