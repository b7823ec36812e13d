// Several right-hand sides of the same operator advanced together.
//
// cg_inverter (cg.cpp:132-202) solves one system at a time and reads the links and the
// clover term once per right-hand side and operator application.  Here nrhs systems share
// every operator application: a batched field stores the right-hand-side index fastest,
//   B[((blk*4d + k)*Vh + h)*nrhs + i]   (complex word k of site (blk,h) of system i),
// one thread handles one (site, system) pair, and the nrhs threads of a site sit next to
// each other in a warp, so the site's links and clover blocks are fetched once for all of
// them while each thread gathers its own neighbour spinors (contiguous across the site's
// threads).  Every system keeps the reference's CG recurrence, stopping rule and iteration
// count; a converged system stops being updated.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <vector>
#include "yg_dirac_impl.cuh"
#include "yg_lattice.h"

namespace yg {

constexpr int kMaxRhs = 16;

// batched index of complex word k of site id, system i
__device__ __forceinline__ long bidx(const Geom &g, int id, int k, int ncomp, int nb, int i) {
  return fidx(g, id, k, ncomp) * nb + i;
}

struct MultiHopArgs {
  Geom g;
  const double2 *src;     // batched hop input
  const double2 *src2;    // STEP 2: batched psi_e
  double2 *dst;
  const double2 *U;
  const double2 *cpk;     // STEP 1 with clover: packed Hermitian inverse of the odd-site blocks
  const double2 *cl;      // STEP 2 with clover: clover term
  double diag;            // STEP 2: 4+m (clover) or (4+m)^2 (no clover)
  double cfm1;
  double coeff;           // +1/2 (step 1), -1/2 (step 2)
  int lo, n, nb;          // output sites [lo, lo+n), nb systems
  int sites;              // sites per block (blockDim = sites * nb)
  int clover;
  int g5;
};

// Shared memory of a block of S sites, entry-major so that the S sites of one entry are
// consecutive (no bank conflicts between sites; the nb threads of a site broadcast):
//   links  L[(slot*D*D + k)*S + j], slot 0..3 = U(x,mu), 4..7 = U(x-mu,mu)
//   matrix M[e*S + j], e < 4*D*D: packed inverse words (step 1) or clover entries (step 2)
//   nbr    N[slot*S + j]: neighbour site of slot (x+mu for 0..3, x-mu for 4..7)
template <int D>
__host__ __device__ constexpr int multi_smem_entries() { return 12 * D * D; }

template <int D, int MU, int SIG>
__device__ __forceinline__ void bhop_dir_s(double2 (&acc)[4][D], const double2 *src, const double2 *Ls,
                                           const Geom &g, int nid, int S, int j, int nb, int i) {
  double2 h[2][D];
#pragma unroll
  for (int c = 0; c < D; c++) {
    double2 p0 = __ldg(src + bidx(g, nid, 0 * D + c, 4 * D, nb, i));
    double2 p1 = __ldg(src + bidx(g, nid, 1 * D + c, 4 * D, nb, i));
    double2 p2 = __ldg(src + bidx(g, nid, 2 * D + c, 4 * D, nb, i));
    double2 p3 = __ldg(src + bidx(g, nid, 3 * D + c, 4 * D, nb, i));
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
  const int slot = SIG < 0 ? MU : 4 + MU;
  const double2 *Lp = Ls + (long)slot * D * D * S + j;
  double2 chi[2][D];
#pragma unroll
  for (int r = 0; r < D; r++) {
    double2 s0 = make_double2(0, 0), s1 = make_double2(0, 0);
#pragma unroll
    for (int q = 0; q < D; q++) {
      if (SIG > 0) {                                   // U^dag: element (q, r)
        const double2 u = Lp[(q * D + r) * S];
        cfmac(s0, u, h[0][q]);
        cfmac(s1, u, h[1][q]);
      } else {
        const double2 u = Lp[(r * D + q) * S];
        cfma(s0, u, h[0][q]);
        cfma(s1, u, h[1][q]);
      }
    }
    chi[0][r] = s0;
    chi[1][r] = s1;
  }
#pragma unroll
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

// STEP 1 (odd sites): dst = A_oo^-1 (coeff hop src)            (no clover: coeff hop src)
// STEP 2 (even sites): dst = [g5] (A_ee src2 + coeff hop src)   (no clover: diag src2 + ...)
// as schur_step1 / schur_step2 of the single-system operator (dirac.cpp:738-765)
template <int D, int STEP>
__global__ void __launch_bounds__(192) k_hop_multi(MultiHopArgs a) {
  extern __shared__ double2 smem[];
  const int S = a.sites, nb = a.nb;
  double2 *Ls = smem;                                  // 8*D*D*S
  double2 *Ms = smem + 8 * D * D * S;                  // 4*D*D*S
  int *Ns = reinterpret_cast<int *>(smem + 12 * D * D * S);   // 8*S
  const Geom &g = a.g;
  const int j = threadIdx.x / nb, i = threadIdx.x % nb;
  const int s0 = blockIdx.x * S;
  const bool active = s0 + j < a.n;
  const int id = a.lo + s0 + j;
  int c[4] = {0, 0, 0, 0};
  if (active) {
    coords_of(g, id, c);
    for (int slot = i; slot < 8; slot += nb) Ns[slot * S + j] = neighbour(g, c, slot & 3, slot < 4 ? +1 : -1);
  }
  __syncthreads();
  // stage the links and the site matrices of the block's sites, coalesced over sites
  const int nsites = min(S, a.n - s0);
  const int nent = a.clover ? 12 * D * D : 8 * D * D;
  for (int q = threadIdx.x; q < nent * S; q += blockDim.x) {
    const int e = q / S, jj = q - e * S;
    if (jj >= nsites) continue;
    const int sid = a.lo + s0 + jj;
    double2 v;
    if (e < 8 * D * D) {
      const int slot = e / (D * D), k = e - slot * D * D;
      const int lid = slot < 4 ? sid : Ns[slot * S + jj];
      v = __ldg(a.U + fidx(g, lid, (slot & 3) * D * D + k, 4 * D * D));
    } else {
      const int w = e - 8 * D * D;
      if (STEP == 1) v = __ldg(a.cpk + (long)w * g.Vh + (sid - g.Vh));
      else v = __ldg(a.cl + fidx(g, sid, w, 4 * D * D));
    }
    smem[(long)e * S + jj] = v;
  }
  __syncthreads();
  if (!active) return;
  double2 acc[4][D];
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int k = 0; k < D; k++) acc[s][k] = make_double2(0, 0);
  bhop_dir_s<D, 0, -1>(acc, a.src, Ls, g, Ns[0 * S + j], S, j, nb, i);
  bhop_dir_s<D, 0, +1>(acc, a.src, Ls, g, Ns[4 * S + j], S, j, nb, i);
  bhop_dir_s<D, 1, -1>(acc, a.src, Ls, g, Ns[1 * S + j], S, j, nb, i);
  bhop_dir_s<D, 1, +1>(acc, a.src, Ls, g, Ns[5 * S + j], S, j, nb, i);
  bhop_dir_s<D, 2, -1>(acc, a.src, Ls, g, Ns[2 * S + j], S, j, nb, i);
  bhop_dir_s<D, 2, +1>(acc, a.src, Ls, g, Ns[6 * S + j], S, j, nb, i);
  bhop_dir_s<D, 3, -1>(acc, a.src, Ls, g, Ns[3 * S + j], S, j, nb, i);
  bhop_dir_s<D, 3, +1>(acc, a.src, Ls, g, Ns[7 * S + j], S, j, nb, i);
  const bool bnd = spinor_zeroed(g, c[0]);
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int k = 0; k < D; k++) acc[s][k] = bnd ? make_double2(0, 0) : cscale(acc[s][k], a.coeff);
  double2 out[4][D];
  if (STEP == 1) {
    if (a.clover) {
      // packed Hermitian blocks (layout of cpk_site) from shared memory
      constexpr int N = 2 * D, W = 2 * D * D;
#pragma unroll
      for (int blk = 0; blk < 2; blk++) {
        const double2 *Cb = Ms + (long)blk * W * S + j;
        double2 x[N], y[N];
#pragma unroll
        for (int r = 0; r < D; r++) {
          x[r] = acc[2 * blk][r];
          x[r + D] = acc[2 * blk + 1][r];
        }
#pragma unroll
        for (int w = 0; w < D; w++) {
          const double2 dd = Cb[w * S];
          y[2 * w] = cscale(x[2 * w], dd.x);
          y[2 * w + 1] = cscale(x[2 * w + 1], dd.y);
        }
#pragma unroll
        for (int r = 1; r < N; r++)
#pragma unroll
          for (int q = 0; q < r; q++) {
            const double2 m = Cb[(D + r * (r - 1) / 2 + q) * S];
            cfma(y[r], m, x[q]);
            cfmac(y[q], m, x[r]);
          }
#pragma unroll
        for (int r = 0; r < D; r++) {
          out[2 * blk][r] = y[r];
          out[2 * blk + 1][r] = y[r + D];
        }
      }
    } else {
#pragma unroll
      for (int s = 0; s < 4; s++)
#pragma unroll
        for (int k = 0; k < D; k++) out[s][k] = acc[s][k];
    }
  } else {
    // the diagonal and clover terms are skipped at zeroed boundary slices, as the
    // single-system operator does (zero_add_at_boundary)
    if (!bnd) {
      if (a.clover) {
        const double diag = a.diag + ((c[0] == g.Ta || c[0] == g.Tb) ? a.cfm1 : 0.0);
#pragma unroll
        for (int blk = 0; blk < 2; blk++) {
          const int s0b = 2 * blk, s1b = 2 * blk + 1;
          double2 p0[D], p1[D];
#pragma unroll
          for (int q = 0; q < D; q++) {
            p0[q] = __ldg(a.src2 + bidx(g, id, s0b * D + q, 4 * D, nb, i));
            p1[q] = __ldg(a.src2 + bidx(g, id, s1b * D + q, 4 * D, nb, i));
          }
#pragma unroll
          for (int r = 0; r < D; r++) {
            double2 o0 = cadd(acc[s0b][r], cscale(p0[r], diag)), o1 = cadd(acc[s1b][r], cscale(p1[r], diag));
#pragma unroll
            for (int q = 0; q < D; q++) {
              const double2 a0 = Ms[(s0b * D * D + r * D + q) * S + j];
              const double2 a1 = Ms[(s1b * D * D + r * D + q) * S + j];
              const double2 a1t = Ms[(s1b * D * D + q * D + r) * S + j];
              cfma(o0, a0, p0[q]);
              cfma(o0, a1, p1[q]);
              cfmac(o1, a1t, p0[q]);
              o1 = csub(o1, cmul(a0, p1[q]));
            }
            acc[s0b][r] = o0;
            acc[s1b][r] = o1;
          }
        }
      } else {
#pragma unroll
        for (int s = 0; s < 4; s++)
#pragma unroll
          for (int k = 0; k < D; k++) {
            double2 v = __ldg(a.src2 + bidx(g, id, s * D + k, 4 * D, nb, i));
            acc[s][k] = cadd(acc[s][k], cscale(v, a.diag));
          }
      }
    }
#pragma unroll
    for (int s = 0; s < 4; s++)
#pragma unroll
      for (int k = 0; k < D; k++) out[s][k] = (a.g5 && s >= 2) ? cscale(acc[s][k], -1.0) : acc[s][k];
  }
#pragma unroll
  for (int s = 0; s < 4; s++)
#pragma unroll
    for (int k = 0; k < D; k++) a.dst[bidx(g, id, s * D + k, 4 * D, nb, i)] = out[s][k];
}

// ---- batched BLAS over the words [w0, w0 + cnt) of every system.  Block size 32*nb, so a
// thread's system index threadIdx.x % nb is the same for all the elements it visits.
struct MultiScalars {
  double a[kMaxRhs];
};

// deterministic per-system block sums: thread t holds the partial of system t % nb
__device__ __forceinline__ void block_partials(double v, double *part, int nb) {
  __shared__ double sh[32 * kMaxRhs];
  sh[threadIdx.x] = v;
  __syncthreads();
  if (threadIdx.x < nb) {
    double s = 0;
    for (int k = threadIdx.x; k < (int)blockDim.x; k += nb) s += sh[k];
    part[(long)blockIdx.x * nb + threadIdx.x] = s;
  }
}

// KIND 0: Re <a_i, b_i> ; 1: |a_i|^2
template <int KIND>
__global__ void k_multi_reduce(double *part, const double2 *a, const double2 *b, long w0, long cnt, int nb) {
  const long n = cnt * nb, base = w0 * nb;
  double acc = 0;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    double2 x = a[base + e];
    if (KIND == 0) {
      double2 y = b[base + e];
      acc = fma(x.x, y.x, fma(x.y, y.y, acc));
    } else {
      acc = fma(x.x, x.x, fma(x.y, x.y, acc));
    }
  }
  block_partials(acc, part, nb);
}

// x_i += alpha_i p_i ; r_i -= alpha_i q_i ; partials of |r_i|^2
__global__ void k_multi_cg_update(double *part, double2 *x, double2 *r, const double2 *p, const double2 *q,
                                  MultiScalars al, long w0, long cnt, int nb) {
  const long n = cnt * nb, base = w0 * nb;
  const double a = al.a[threadIdx.x % nb];
  double acc = 0;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    double2 xv = x[base + e], rv = r[base + e], pv = p[base + e], qv = q[base + e];
    xv.x = fma(a, pv.x, xv.x);
    xv.y = fma(a, pv.y, xv.y);
    rv.x = fma(-a, qv.x, rv.x);
    rv.y = fma(-a, qv.y, rv.y);
    x[base + e] = xv;
    r[base + e] = rv;
    acc = fma(rv.x, rv.x, fma(rv.y, rv.y, acc));
  }
  block_partials(acc, part, nb);
}

// p_i = beta_i p_i + r_i for the systems with beta_i != 0 flagged in `on`
__global__ void k_multi_xpay(double2 *p, const double2 *r, MultiScalars be, MultiScalars on, long w0, long cnt,
                             int nb) {
  const long n = cnt * nb, base = w0 * nb;
  const int i = threadIdx.x % nb;
  if (on.a[i] == 0.0) return;
  const double b = be.a[i];
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    double2 pv = p[base + e], rv = r[base + e];
    p[base + e] = make_double2(fma(b, pv.x, rv.x), fma(b, pv.y, rv.y));
  }
}

// dst_i = b_i - a_i on the words [w0, w0+cnt)
__global__ void k_multi_sub(double2 *dst, const double2 *bvec, const double2 *avec, long w0, long cnt, int nb) {
  const long n = cnt * nb, base = w0 * nb;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    double2 x = bvec[base + e], y = avec[base + e];
    dst[base + e] = make_double2(x.x - y.x, x.y - y.y);
  }
}

// pack (dir = 0) or unpack (dir = 1) the words [w0, w0+cnt) of nb single-system fields
struct FieldPtrs {
  double2 *f[kMaxRhs];
};

__global__ void k_multi_pack(double2 *batch, FieldPtrs fp, long w0, long cnt, int nb, int dir) {
  const long n = cnt * nb;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const long w = w0 + e / nb;
    const int i = (int)(e % nb);
    if (dir == 0) batch[w * nb + i] = fp.f[i][w];
    else fp.f[i][w] = batch[w * nb + i];
  }
}

// zero the spinors of the boundary slices (open / SF) of a batched field, both parities:
// the side effect of the single-system operator on its input (bc_zero_field)
__global__ void k_multi_bc_zero(double2 *batch, Geom g, int words, int nb) {
  const long n = (long)g.V * words * nb;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const long w = e / nb;                        // word index in the single-system layout
    const int blk = (int)(w / ((long)words * g.Vh));
    const int h = (int)(w % g.Vh);
    int c[4];
    coords_of(g, blk * g.Vh + h, c);
    if (spinor_zeroed(g, c[0])) batch[e] = make_double2(0, 0);
  }
}

// ------------------------------------------------------------------ host side
namespace {

struct Multi {
  Lattice &L;
  int nb;
  long w0, cnt;            // complex words of the default view (per system)
  int grid, threads;       // batched BLAS launch shape
  DevBuf part;
  std::vector<double> host;

  Multi(Lattice &l, int n) : L(l), nb(n) {
    long lo, ns;
    L.view_range(YG_VIEW_DEFAULT, lo, ns);
    w0 = lo * 4L * L.d;
    cnt = ns * 4L * L.d;
    threads = 32 * nb;
    long g = (cnt * nb + threads - 1) / threads;
    grid = (int)std::min<long>(g, 148L * 8);
    part.alloc(sizeof(double) * (size_t)grid * nb);
    host.resize((size_t)grid * nb);
  }

  double2 *field() {
    double2 *p = nullptr;
    YG_CUDA(cudaMalloc(&p, sizeof(double2) * (size_t)L.V * 4 * L.d * nb));
    YG_CUDA(cudaMemsetAsync(p, 0, sizeof(double2) * (size_t)L.V * 4 * L.d * nb, L.stream));
    return p;
  }

  // sums of the block partials per system, in block order
  std::vector<double> sums() {
    YG_CUDA(cudaMemcpyAsync(host.data(), part.p, sizeof(double) * (size_t)grid * nb, cudaMemcpyDeviceToHost,
                            L.stream));
    YG_CUDA(cudaStreamSynchronize(L.stream));
    std::vector<double> s(nb, 0.0);
    for (int b = 0; b < grid; b++)
      for (int i = 0; i < nb; i++) s[i] += host[(size_t)b * nb + i];
    return s;
  }

  std::vector<double> dot_re(const double2 *a, const double2 *b) {
    k_multi_reduce<0><<<grid, threads, 0, L.stream>>>(part.as<double>(), a, b, w0, cnt, nb);
    YG_LAUNCHED();
    return sums();
  }
  std::vector<double> sqnorm(const double2 *a) {
    k_multi_reduce<1><<<grid, threads, 0, L.stream>>>(part.as<double>(), a, nullptr, w0, cnt, nb);
    YG_LAUNCHED();
    return sums();
  }
};

}  // namespace

// dst = Hphi src (one Schur operator with gamma5; g5 = 0: Dphi) on batched fields; tmp takes the
// odd sites
static void hphi_multi(Lattice &L, int nb, double mass, double2 *dst, const double2 *src, double2 *tmp,
                       int g5 = 1) {
  if (L.d != 3) throw Error(YG_ERR_ARG, "the batched operator is built for d = 3");
  MultiHopArgs a{};
  a.g = L.g;
  a.U = L.links.as<double2>();
  a.nb = nb;
  a.cfm1 = L.p.cf - 1.0;
  a.clover = L.p.clover ? 1 : 0;
  if (a.clover) {
    ensure_ldl(L, 4.0 + mass);
    a.cpk = L.cpk64.as<double2>();
    a.cl = L.clover.as<double2>();
  }
  MultiHopArgs s1 = a;
  s1.src = src;
  s1.dst = tmp;
  s1.coeff = 0.5;
  s1.lo = (int)L.Vh;
  s1.n = (int)L.Vh;
  MultiHopArgs s2 = a;
  s2.src = tmp;
  s2.src2 = src;
  s2.dst = dst;
  s2.coeff = -0.5;
  s2.lo = 0;
  s2.n = (int)L.Vh;
  s2.g5 = g5;
  s2.diag = a.clover ? 4.0 + mass : (4.0 + mass) * (4.0 + mass);
  // blocks of S sites x nb systems (about 192 threads), shared memory for S sites
  const int S = std::min(24, std::max(1, 192 / nb));      // <= 24 sites: 42 KB of shared memory
  s1.sites = s2.sites = S;
  const size_t smem = sizeof(double2) * (size_t)multi_smem_entries<3>() * S + sizeof(int) * 8 * S;
  const int blocks = nblk(L.Vh, S);
  k_hop_multi<3, 1><<<blocks, S * nb, smem, L.stream>>>(s1);
  YG_LAUNCHED();
  k_hop_multi<3, 2><<<blocks, S * nb, smem, L.stream>>>(s2);
  YG_LAUNCHED();
  L.mvm += 2;
}

static void bc_zero_multi(Lattice &L, int nb, double2 *f) {
  if (L.p.bc != YG_BC_OPEN && L.p.bc != YG_BC_SF) return;
  const long n = L.V * 4L * L.d * nb;
  k_multi_bc_zero<<<(int)std::min<long>(nblk(n, 256), 148L * 16), 256, 0, L.stream>>>(f, L.g, 4 * L.d, nb);
  YG_LAUNCHED();
}

// dst = op(src); like the single-system operator it zeroes the boundary slices of its
// input (dirac.cpp:738-765 with apply_bcs_on_spinor_field)
static void op_multi(Lattice &L, int op, int nb, double mass, double2 *dst, double2 *src, double2 *tmp,
                     double2 *mid) {
  if (op == YG_OP_HPHI) {
    hphi_multi(L, nb, mass, dst, src, tmp);
    bc_zero_multi(L, nb, src);
  } else if (op == YG_OP_HPHI_SQ) {
    hphi_multi(L, nb, mass, mid, src, tmp);
    bc_zero_multi(L, nb, src);
    hphi_multi(L, nb, mass, dst, mid, tmp);
  } else {
    throw Error(YG_ERR_ARG, "the batched CG runs on Hphi or Hphi_sq");
  }
}

// nrhs cg_inverter solves (cg.cpp:132-202) sharing every operator application
int cg_multi(Lattice &L, const yg_inv_par &par, int nrhs, double *const *xs, double *const *bs, int *iters) {
  if (nrhs < 1 || nrhs > kMaxRhs) throw Error(YG_ERR_ARG, "1..16 right-hand sides");
  if (!L.p.eo) throw Error(YG_ERR_ARG, "the batched CG needs even-odd preconditioning");
  if (L.d != 3) throw Error(YG_ERR_ARG, "the batched operator is built for d = 3");
  Multi m(L, nrhs);
  const int nb = nrhs;
  double2 *X = m.field(), *B = m.field(), *R = m.field(), *P = m.field(), *Q = m.field(), *T = m.field(),
          *M = m.field();
  std::vector<double2 *> bufs = {X, B, R, P, Q, T, M};
  int status = YG_OK;
  try {
    FieldPtrs fx{}, fb{};
    for (int i = 0; i < nb; i++) {
      fx.f[i] = (double2 *)xs[i];
      fb.f[i] = (double2 *)bs[i];
    }
    const long wall = (long)L.V * 4 * L.d;        // both blocks: the operator reads odd sites of its input
    k_multi_pack<<<nblk(wall * nb, 256), 256, 0, L.stream>>>(X, fx, 0, wall, nb, 0);
    YG_LAUNCHED();
    k_multi_pack<<<nblk(wall * nb, 256), 256, 0, L.stream>>>(B, fb, 0, wall, nb, 0);
    YG_LAUNCHED();
    // r = b - A x ; p = r
    YG_CUDA(cudaMemcpyAsync(P, X, sizeof(double2) * (size_t)wall * nb, cudaMemcpyDeviceToDevice, L.stream));
    op_multi(L, par.op, nb, par.mass, Q, P, T, M);
    k_multi_sub<<<m.grid, m.threads, 0, L.stream>>>(R, B, Q, m.w0, m.cnt, nb);
    YG_LAUNCHED();
    YG_CUDA(cudaMemcpyAsync(P, R, sizeof(double2) * (size_t)wall * nb, cudaMemcpyDeviceToDevice, L.stream));
    std::vector<double> norm = m.sqnorm(B), rr = m.sqnorm(R);
    std::vector<int> active(nb), it(nb, 0);
    int nactive = 0;
    for (int i = 0; i < nb; i++) {
      active[i] = !(rr[i] < norm[i] * par.prec);   // already converged: 0 iterations
      nactive += active[i];
    }
    int k = 0;
    while (nactive > 0) {
      k++;
      if (par.maxiter > 0 && k > par.maxiter) { status = YG_MAXITER; break; }
      op_multi(L, par.op, nb, par.mass, Q, P, T, M);
      std::vector<double> pq = m.dot_re(P, Q);
      MultiScalars al{}, be{}, on{};
      for (int i = 0; i < nb; i++) {
        if (!active[i]) continue;
        if (!std::isfinite(pq[i])) throw Error(YG_NONFINITE, "non-finite value in cg_multi");
        al.a[i] = rr[i] / pq[i];
      }
      k_multi_cg_update<<<m.grid, m.threads, 0, L.stream>>>(m.part.as<double>(), X, R, P, Q, al, m.w0, m.cnt, nb);
      YG_LAUNCHED();
      std::vector<double> rn = m.sums();
      for (int i = 0; i < nb; i++) {
        if (!active[i]) continue;
        it[i] = k;
        be.a[i] = rn[i] / rr[i];
        rr[i] = rn[i];
        if (rn[i] < norm[i] * par.prec) {      // cg.cpp:186-189: stop before the p update
          active[i] = 0;
          nactive--;
        } else {
          on.a[i] = 1.0;
        }
      }
      if (nactive > 0) {
        k_multi_xpay<<<m.grid, m.threads, 0, L.stream>>>(P, R, be, on, m.w0, m.cnt, nb);
        YG_LAUNCHED();
      }
    }
    // x_i (default view) back into the caller's fields
    k_multi_pack<<<nblk(m.cnt * nb, 256), 256, 0, L.stream>>>(X, fx, m.w0, m.cnt, nb, 1);
    YG_LAUNCHED();
    YG_CUDA(cudaStreamSynchronize(L.stream));
    for (int i = 0; i < nb; i++) iters[i] = it[i];
    if (par.log)
      for (int i = 0; i < nb; i++)
        fprintf(stderr, "[INVERTER][30]cg_multi[%d]: iterations = %d, precision = %1.4e\n", i, it[i],
                rr[i] / norm[i]);
  } catch (...) {
    for (double2 *b : bufs) cudaFree(b);
    throw;
  }
  for (double2 *b : bufs) cudaFree(b);
  return status;
}

// ---- batched BiCGstab (complex per-system scalars)
struct MultiC {
  double2 c[kMaxRhs];
};

// <a_i, b_i> = sum a conj(b): per-system partials of the real and imaginary parts
__global__ void k_multi_cdot(double *part_re, double *part_im, const double2 *a, const double2 *b, long w0, long cnt,
                             int nb) {
  const long n = cnt * nb, base = w0 * nb;
  double re = 0, im = 0;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const double2 x = a[base + e], y = b[base + e];
    re = fma(x.x, y.x, fma(x.y, y.y, re));
    im = fma(x.y, y.x, fma(-x.x, y.y, im));
  }
  block_partials(re, part_re, nb);
  __syncthreads();
  block_partials(im, part_im, nb);
}

// y_i += c_i x_i (c_i = 0 leaves system i alone)
__global__ void k_multi_caxpy(double2 *y, const double2 *x, MultiC c, long w0, long cnt, int nb) {
  const long n = cnt * nb, base = w0 * nb;
  const double2 k = c.c[threadIdx.x % nb];
  if (k.x == 0.0 && k.y == 0.0) return;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const double2 xv = x[base + e];
    double2 yv = y[base + e];
    yv.x = fma(k.x, xv.x, fma(-k.y, xv.y, yv.x));
    yv.y = fma(k.x, xv.y, fma(k.y, xv.x, yv.y));
    y[base + e] = yv;
  }
}

// p_i = beta_i p_i + r_i - (beta_i omega_i) v_i for the systems flagged in `on`
__global__ void k_multi_bicg_p(double2 *p, const double2 *r, const double2 *v, MultiC beta, MultiC bw,
                               MultiScalars on, long w0, long cnt, int nb) {
  const long n = cnt * nb, base = w0 * nb;
  const int i = threadIdx.x % nb;
  if (on.a[i] == 0.0) return;
  const double2 be = beta.c[i], w = bw.c[i];
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const double2 pv = p[base + e], rv = r[base + e], vv = v[base + e];
    double2 o;
    o.x = be.x * pv.x - be.y * pv.y + rv.x - (w.x * vv.x - w.y * vv.y);
    o.y = be.x * pv.y + be.y * pv.x + rv.y - (w.x * vv.y + w.y * vv.x);
    p[base + e] = o;
  }
}

// nrhs bicgstab_inverter solves on Dphi (bicgstab.cpp:9-97, each system with its own complex
// scalars and stopping test) sharing every operator application; iters[i] = 2 x the system's
// iterations, as the reference counts them
int bicgstab_multi(Lattice &L, const yg_inv_par &par, int nrhs, double *const *xs, double *const *bs, int *iters) {
  using zc = std::complex<double>;
  if (nrhs < 1 || nrhs > kMaxRhs) throw Error(YG_ERR_ARG, "1..16 right-hand sides");
  if (!L.p.eo) throw Error(YG_ERR_ARG, "the batched BiCGstab needs even-odd preconditioning");
  if (L.d != 3) throw Error(YG_ERR_ARG, "the batched operator is built for d = 3");
  if (par.op != YG_OP_DPHI) throw Error(YG_ERR_ARG, "the batched BiCGstab solves Dphi systems");
  Multi m(L, nrhs);
  const int nb = nrhs;
  double2 *X = m.field(), *B = m.field(), *R = m.field(), *R0 = m.field(), *P = m.field(), *V = m.field(),
          *T = m.field(), *TMP = m.field();
  std::vector<double2 *> bufs = {X, B, R, R0, P, V, T, TMP};
  DevBuf part_im;
  int status = YG_OK;
  try {
    part_im.alloc(sizeof(double) * (size_t)m.grid * nb);
    auto dphi = [&](double2 *dst, double2 *src) {
      hphi_multi(L, nb, par.mass, dst, src, TMP, 0);
      bc_zero_multi(L, nb, src);
    };
    auto cdot = [&](const double2 *a, const double2 *b) {
      k_multi_cdot<<<m.grid, m.threads, 0, L.stream>>>(m.part.as<double>(), part_im.as<double>(), a, b, m.w0, m.cnt,
                                                       nb);
      YG_LAUNCHED();
      std::vector<double> hi((size_t)m.grid * nb);
      YG_CUDA(cudaMemcpyAsync(hi.data(), part_im.p, sizeof(double) * hi.size(), cudaMemcpyDeviceToHost, L.stream));
      std::vector<double> re = m.sums();          // synchronises the stream
      std::vector<zc> out(nb);
      for (int i = 0; i < nb; i++) {
        double im = 0;
        for (int blk = 0; blk < m.grid; blk++) im += hi[(size_t)blk * nb + i];
        out[i] = zc(re[i], im);
      }
      return out;
    };
    auto caxpy = [&](double2 *y, const double2 *x, const std::vector<zc> &c) {
      MultiC k{};
      for (int i = 0; i < nb; i++) k.c[i] = make_double2(c[i].real(), c[i].imag());
      k_multi_caxpy<<<m.grid, m.threads, 0, L.stream>>>(y, x, k, m.w0, m.cnt, nb);
      YG_LAUNCHED();
    };
    FieldPtrs fx{}, fb{};
    for (int i = 0; i < nb; i++) {
      fx.f[i] = (double2 *)xs[i];
      fb.f[i] = (double2 *)bs[i];
    }
    const long wall = (long)L.V * 4 * L.d;
    k_multi_pack<<<nblk(wall * nb, 256), 256, 0, L.stream>>>(X, fx, 0, wall, nb, 0);
    YG_LAUNCHED();
    k_multi_pack<<<nblk(wall * nb, 256), 256, 0, L.stream>>>(B, fb, 0, wall, nb, 0);
    YG_LAUNCHED();
    // r = b - D x ; r0 = p = r
    dphi(P, X);
    k_multi_sub<<<m.grid, m.threads, 0, L.stream>>>(R, B, P, m.w0, m.cnt, nb);
    YG_LAUNCHED();
    YG_CUDA(cudaMemcpyAsync(R0, R, sizeof(double2) * (size_t)wall * nb, cudaMemcpyDeviceToDevice, L.stream));
    YG_CUDA(cudaMemcpyAsync(P, R, sizeof(double2) * (size_t)wall * nb, cudaMemcpyDeviceToDevice, L.stream));
    std::vector<double> norm = m.sqnorm(B);
    std::vector<zc> rho0 = cdot(R, R0);
    std::vector<int> active(nb), it(nb, 0);
    std::vector<double> res(nb);
    int nactive = 0;
    for (int i = 0; i < nb; i++) {
      res[i] = rho0[i].real();
      active[i] = !(res[i] < norm[i] * par.prec);   // bicgstab.cpp:48-53: 0 iterations
      nactive += active[i];
    }
    int k = 0;
    std::vector<zc> alpha(nb), omega(nb), zero(nb, zc(0, 0));
    while (nactive > 0) {
      k++;
      if (par.maxiter > 0 && k > par.maxiter) { status = YG_MAXITER; break; }
      dphi(V, P);
      std::vector<zc> vr0 = cdot(V, R0);
      for (int i = 0; i < nb; i++) {
        alpha[i] = active[i] ? rho0[i] / vr0[i] : zc(0, 0);
        if (active[i] && !std::isfinite(alpha[i].real())) throw Error(YG_NONFINITE, "non-finite value in bicgstab_multi");
      }
      std::vector<zc> nalpha(nb);
      for (int i = 0; i < nb; i++) nalpha[i] = -alpha[i];
      caxpy(R, V, nalpha);                          // r -= alpha v
      dphi(T, R);
      std::vector<zc> rt = cdot(R, T);
      std::vector<double> tt = m.sqnorm(T);
      for (int i = 0; i < nb; i++) omega[i] = active[i] ? rt[i] / tt[i] : zc(0, 0);
      caxpy(X, P, alpha);                           // x += alpha p + omega r
      caxpy(X, R, omega);
      std::vector<zc> nomega(nb);
      for (int i = 0; i < nb; i++) nomega[i] = -omega[i];
      caxpy(R, T, nomega);                          // r -= omega t
      std::vector<zc> rho1 = cdot(R, R0);
      std::vector<double> rr = m.sqnorm(R);
      MultiC be{}, bw{};
      MultiScalars on{};
      for (int i = 0; i < nb; i++) {
        if (!active[i]) continue;
        it[i] = k;
        const zc beta = (rho1[i] / rho0[i]) * (alpha[i] / omega[i]);
        res[i] = rr[i];
        if (rr[i] < norm[i] * par.prec) {         // bicgstab.cpp:77-81: stop before rho0 = rho1
          active[i] = 0;
          nactive--;
          continue;
        }
        be.c[i] = make_double2(beta.real(), beta.imag());
        const zc w = beta * omega[i];
        bw.c[i] = make_double2(w.real(), w.imag());
        on.a[i] = 1.0;
        rho0[i] = rho1[i];
      }
      if (nactive > 0) {
        k_multi_bicg_p<<<m.grid, m.threads, 0, L.stream>>>(P, R, V, be, bw, on, m.w0, m.cnt, nb);
        YG_LAUNCHED();
      }
    }
    k_multi_pack<<<nblk(m.cnt * nb, 256), 256, 0, L.stream>>>(X, fx, m.w0, m.cnt, nb, 1);
    YG_LAUNCHED();
    YG_CUDA(cudaStreamSynchronize(L.stream));
    for (int i = 0; i < nb; i++) iters[i] = 2 * it[i];
    if (par.log)
      for (int i = 0; i < nb; i++)
        fprintf(stderr, "[INVERTER][30]bicgstab_multi[%d]: iterations = %d, precision = %1.4e\n", i, 2 * it[i],
                res[i] / norm[i]);
  } catch (...) {
    for (double2 *b : bufs) cudaFree(b);
    throw;
  }
  for (double2 *b : bufs) cudaFree(b);
  return status;
}

// ==================================================================== mixed precision
// The batched CG with FP32 inner iterations: FP32 batched fields (float2 words in the
// batched layout), the compressed operator's FP32 matrices (12- or 18-real links, packed
// Hermitian clover blocks M_e / M_o^-1, built by ensure_sloppy) staged per block of sites
// in shared memory, FP64 reliable updates through the batched FP64 operator.

struct MultiFHopArgs {
  Geom g;
  const float2 *src;      // batched FP32 hop input
  const float2 *src2;     // STEP 2: batched psi_e
  float2 *dst;
  const float2 *U;        // FP32 links, K complex words per link
  const float4 *C;        // FP32 packed clover blocks, 18 float4 per site
  float coeff;
  int lo, n, nb, sites;
};

// y = M x for one packed Hermitian 6x6 block (6 diagonal reals, then the lower triangle)
__device__ __forceinline__ void herm6(float2 (&y)[6], const float *c, const float2 (&x)[6]) {
#pragma unroll
  for (int r = 0; r < 6; r++) y[r] = cscale(x[r], c[r]);
  int k = 6;
#pragma unroll
  for (int r = 1; r < 6; r++)
#pragma unroll
    for (int q = 0; q < r; q++, k += 2) {
      const float2 m = make_float2(c[k], c[k + 1]);
      cfma(y[r], m, x[q]);
      cfmac(y[q], m, x[r]);
    }
}

template <int MU, int SIG>
__device__ __forceinline__ void fhop_dir(float2 (&acc)[12], const float2 *src, const float2 *Ls, const Geom &g,
                                         int nid, int S, int j, int nb, int i) {
  float2 h[2][3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const float2 p0 = __ldg(src + bidx(g, nid, 0 * 3 + c, 12, nb, i));
    const float2 p1 = __ldg(src + bidx(g, nid, 1 * 3 + c, 12, nb, i));
    const float2 p2 = __ldg(src + bidx(g, nid, 2 * 3 + c, 12, nb, i));
    const float2 p3 = __ldg(src + bidx(g, nid, 3 * 3 + c, 12, nb, i));
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
  const float2 *Lp = Ls + (SIG < 0 ? MU : 4 + MU) * 9 * S + j;
  float2 chi[2][3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    float2 s0 = make_float2(0.f, 0.f), s1 = make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      if (SIG > 0) {
        const float2 u = Lp[(q * 3 + r) * S];
        cfmac(s0, u, h[0][q]);
        cfmac(s1, u, h[1][q]);
      } else {
        const float2 u = Lp[(r * 3 + q) * S];
        cfma(s0, u, h[0][q]);
        cfma(s1, u, h[1][q]);
      }
    }
    chi[0][r] = s0;
    chi[1][r] = s1;
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

// bytes of shared memory per site: 8 links x 9 float2, 18 float4 clover words, 8 neighbour
// indices and the site's time coordinate
constexpr int kFSiteBytes = 8 * 9 * 8 + 18 * 16 + 9 * 4;

// STEP 1 (odd sites): dst = M_o^-1 (coeff hop src); STEP 2 (even sites): dst = gamma5 (M_e
// src2 + coeff hop src); zero on the spinor boundary slices -- the compressed operator of
// the single-system mixed CG, for nb systems at once
template <int K, int STEP>
__global__ void __launch_bounds__(192) k_fhop_multi(MultiFHopArgs a) {
  extern __shared__ __align__(16) unsigned char fsm[];
  const int S = a.sites, nb = a.nb;
  float2 *Ls = reinterpret_cast<float2 *>(fsm);                       // [8*9][S]
  float4 *Cs = reinterpret_cast<float4 *>(fsm + 8 * 9 * 8 * S);       // [18][S]
  int *Ns = reinterpret_cast<int *>(fsm + (8 * 9 * 8 + 18 * 16) * S);  // [8][S]
  int *Ts = Ns + 8 * S;                                               // [S]
  const Geom &g = a.g;
  const int j = threadIdx.x / nb, i = threadIdx.x % nb;
  const int s0 = blockIdx.x * S;
  const bool active = s0 + j < a.n;
  const int id = a.lo + s0 + j;
  int c[4] = {0, 0, 0, 0};
  if (active) {
    coords_of(g, id, c);
    for (int slot = i; slot < 8; slot += nb) Ns[slot * S + j] = neighbour(g, c, slot & 3, slot < 4 ? +1 : -1);
    if (i == 0) Ts[j] = c[0];
  }
  __syncthreads();
  const int nsites = min(S, a.n - s0);
  const int T = g.dim[0];
  // links: one (site, slot) per thread step; 12-real links get row 2 rebuilt here, with the
  // antiperiodic sign the stored rows carry applied again
  for (int q = threadIdx.x; q < 8 * S; q += blockDim.x) {
    const int slot = q / S, jj = q - slot * S;
    if (jj >= nsites) continue;
    const int sid = a.lo + s0 + jj;
    const int mu = slot & 3;
    const int lid = slot < 4 ? sid : Ns[slot * S + jj];
    const int lb = lid >= g.Vh, lh = lid - lb * g.Vh;
    float2 u[9];
#pragma unroll
    for (int k = 0; k < K; k++) u[k] = __ldg(a.U + ((long)(lb * 4 + mu) * K + k) * g.Vh + lh);
    if (K == 6) {
      const int tl = slot < 4 ? Ts[jj] : (mu == 0 ? (Ts[jj] == 0 ? T - 1 : Ts[jj] - 1) : Ts[jj]);
      const float sgn = (g.bc == YG_BC_ANTIPERIODIC && mu == 0 && tl == 0) ? -1.f : 1.f;
      const float2 a0 = u[0], a1 = u[1], a2 = u[2], b0 = u[3], b1 = u[4], b2 = u[5];
      u[6] = cscale(cconj(csub(cmul(a1, b2), cmul(a2, b1))), sgn);
      u[7] = cscale(cconj(csub(cmul(a2, b0), cmul(a0, b2))), sgn);
      u[8] = cscale(cconj(csub(cmul(a0, b1), cmul(a1, b0))), sgn);
    }
#pragma unroll
    for (int k = 0; k < 9; k++) Ls[(slot * 9 + k) * S + jj] = u[k];
  }
  for (int q = threadIdx.x; q < 18 * S; q += blockDim.x) {
    const int w = q / S, jj = q - w * S;
    if (jj >= nsites) continue;
    const int sid = a.lo + s0 + jj;
    const int blk = sid >= g.Vh, h = sid - blk * g.Vh;
    Cs[w * S + jj] = __ldg(a.C + (long)(blk * 18 + w) * g.Vh + h);
  }
  __syncthreads();
  if (!active) return;
  float2 acc[12];
#pragma unroll
  for (int k = 0; k < 12; k++) acc[k] = make_float2(0.f, 0.f);
  fhop_dir<0, -1>(acc, a.src, Ls, g, Ns[0 * S + j], S, j, nb, i);
  fhop_dir<0, +1>(acc, a.src, Ls, g, Ns[4 * S + j], S, j, nb, i);
  fhop_dir<1, -1>(acc, a.src, Ls, g, Ns[1 * S + j], S, j, nb, i);
  fhop_dir<1, +1>(acc, a.src, Ls, g, Ns[5 * S + j], S, j, nb, i);
  fhop_dir<2, -1>(acc, a.src, Ls, g, Ns[2 * S + j], S, j, nb, i);
  fhop_dir<2, +1>(acc, a.src, Ls, g, Ns[6 * S + j], S, j, nb, i);
  fhop_dir<3, -1>(acc, a.src, Ls, g, Ns[3 * S + j], S, j, nb, i);
  fhop_dir<3, +1>(acc, a.src, Ls, g, Ns[7 * S + j], S, j, nb, i);
  float cl[72];
#pragma unroll
  for (int w = 0; w < 18; w++) {
    const float4 v = Cs[w * S + j];
    cl[4 * w] = v.x; cl[4 * w + 1] = v.y; cl[4 * w + 2] = v.z; cl[4 * w + 3] = v.w;
  }
  float2 in[12];
  if (STEP == 1) {
#pragma unroll
    for (int k = 0; k < 12; k++) in[k] = cscale(acc[k], a.coeff);
  } else {
#pragma unroll
    for (int k = 0; k < 12; k++) in[k] = __ldg(a.src2 + bidx(g, id, k, 12, nb, i));
  }
  float2 out[12];
#pragma unroll
  for (int b = 0; b < 2; b++) {
    float2 x[6], y[6];
#pragma unroll
    for (int r = 0; r < 3; r++) {
      x[r] = in[(2 * b) * 3 + r];
      x[r + 3] = in[(2 * b + 1) * 3 + r];
    }
    herm6(y, cl + 36 * b, x);
#pragma unroll
    for (int r = 0; r < 3; r++) {
      out[(2 * b) * 3 + r] = y[r];
      out[(2 * b + 1) * 3 + r] = y[r + 3];
    }
  }
  if (STEP == 2) {
#pragma unroll
    for (int k = 0; k < 12; k++) {
      out[k] = cadd(out[k], cscale(acc[k], a.coeff));
      if (k >= 6) out[k] = cscale(out[k], -1.f);              // gamma5
    }
  }
  const bool bnd = spinor_zeroed(g, c[0]);
#pragma unroll
  for (int k = 0; k < 12; k++) a.dst[bidx(g, id, k, 12, nb, i)] = bnd ? make_float2(0.f, 0.f) : out[k];
}

// ---- batched FP32 vectors (float2 words, batched layout, the default view from word 0)
template <int KIND>    // 0: Re <a_i, b_i> ; 1: |a_i|^2
__global__ void k_fm_reduce(double *part, const float2 *a, const float2 *b, long cnt, int nb) {
  const long n = cnt * nb;
  double acc = 0;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const float2 x = a[e];
    if (KIND == 0) {
      const float2 y = b[e];
      acc += (double)fmaf(x.x, y.x, x.y * y.y);
    } else {
      acc += (double)fmaf(x.x, x.x, x.y * x.y);
    }
  }
  block_partials(acc, part, nb);
}

// x_i += alpha_i p_i ; r_i -= alpha_i q_i ; partials of |r_i|^2
__global__ void k_fm_update(double *part, float2 *x, float2 *r, const float2 *p, const float2 *q, MultiScalars al,
                            long cnt, int nb) {
  const long n = cnt * nb;
  const float a = (float)al.a[threadIdx.x % nb];
  double acc = 0;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    float2 xv = x[e], rv = r[e];
    const float2 pv = p[e], qv = q[e];
    xv.x = fmaf(a, pv.x, xv.x);
    xv.y = fmaf(a, pv.y, xv.y);
    rv.x = fmaf(-a, qv.x, rv.x);
    rv.y = fmaf(-a, qv.y, rv.y);
    x[e] = xv;
    r[e] = rv;
    acc += (double)fmaf(rv.x, rv.x, rv.y * rv.y);
  }
  block_partials(acc, part, nb);
}

// p_i = r_i + beta_i p_i for the systems flagged in `on`
__global__ void k_fm_xpay(float2 *p, const float2 *r, MultiScalars be, MultiScalars on, long cnt, int nb) {
  const long n = cnt * nb;
  const int i = threadIdx.x % nb;
  if (on.a[i] == 0.0) return;
  const float b = (float)be.a[i];
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const float2 pv = p[e], rv = r[e];
    p[e] = make_float2(fmaf(b, pv.x, rv.x), fmaf(b, pv.y, rv.y));
  }
}

__global__ void k_fm_from_d(float2 *f, const double2 *d, long n) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const double2 v = d[e];
    f[e] = make_float2((float)v.x, (float)v.y);
  }
}

__global__ void k_fm_add_to_d(double2 *d, const float2 *f, long n) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
    const float2 v = f[e];
    double2 w = d[e];
    w.x += (double)v.x;
    w.y += (double)v.y;
    d[e] = w;
  }
}

// dst = Hphi src with the compressed FP32 operator on batched FP32 fields (tmp: odd sites)
static void fhphi_multi(Lattice &L, int nb, float2 *dst, const float2 *src, float2 *tmp) {
  MultiFHopArgs a{};
  a.g = L.g;
  a.U = L.sl_links.as<float2>();
  a.C = L.sl_clover.as<float4>();
  a.nb = nb;
  const int S = std::min(24, std::max(1, 192 / nb));
  a.sites = S;
  MultiFHopArgs s1 = a;
  s1.src = src; s1.dst = tmp; s1.coeff = 0.5f; s1.lo = (int)L.Vh; s1.n = (int)L.Vh;
  MultiFHopArgs s2 = a;
  s2.src = tmp; s2.src2 = src; s2.dst = dst; s2.coeff = -0.5f; s2.lo = 0; s2.n = (int)L.Vh;
  const size_t smem = (size_t)kFSiteBytes * S;
  const int blocks = nblk(L.Vh, S);
  if (L.sl_reals == 12) {
    k_fhop_multi<6, 1><<<blocks, S * nb, smem, L.stream>>>(s1);
    YG_LAUNCHED();
    k_fhop_multi<6, 2><<<blocks, S * nb, smem, L.stream>>>(s2);
  } else {
    k_fhop_multi<9, 1><<<blocks, S * nb, smem, L.stream>>>(s1);
    YG_LAUNCHED();
    k_fhop_multi<9, 2><<<blocks, S * nb, smem, L.stream>>>(s2);
  }
  YG_LAUNCHED();
  L.mvm += 2;
}

// nrhs solves of Hphi_sq with FP32 inner iterations and FP64 reliable updates; each system
// stops on its TRUE FP64 residual |b_i - A x_i|^2 < prec |b_i|^2
int cg_mixed_multi(Lattice &L, const yg_inv_par &par, int nrhs, double *const *xs, double *const *bs, double delta,
                   yg_solve_stats *stats) {
  auto t0 = std::chrono::steady_clock::now();
  if (par.op != YG_OP_HPHI_SQ) throw Error(YG_ERR_ARG, "the batched mixed CG solves Hphi_sq systems");
  if (nrhs < 1 || nrhs > kMaxRhs) throw Error(YG_ERR_ARG, "1..16 right-hand sides");
  if (!L.p.eo) throw Error(YG_ERR_ARG, "the batched CG needs even-odd preconditioning");
  if (L.d != 3) throw Error(YG_ERR_ARG, "the batched operator is built for d = 3");
  if (!(delta > 0.0 && delta < 1.0)) throw Error(YG_ERR_ARG, "reliable-update delta must lie in (0,1)");
  const int nb = nrhs;
  const int reals = (L.nc == 3 && L.p.repr == YG_REPR_FUNDAMENTAL) ? 12 : 18;
  // FP32 matrices of the compressed operator (shared with the single-system solver)
  ensure_sloppy(L, par.mass, 16, reals, 32, 32);
  Multi m(L, nb);
  const long wall = (long)L.V * 4 * L.d;
  const long nview = m.cnt * nb;                 // batched elements of the default view
  std::vector<void *> bufs;
  auto f64 = [&]() { double2 *p = m.field(); bufs.push_back(p); return p; };
  auto f32 = [&]() {
    float2 *p = nullptr;
    YG_CUDA(cudaMalloc(&p, sizeof(float2) * (size_t)wall * nb));
    bufs.push_back(p);
    YG_CUDA(cudaMemsetAsync(p, 0, sizeof(float2) * (size_t)wall * nb, L.stream));
    return p;
  };
  int status = YG_OK;
  try {
    double2 *X = f64(), *B = f64(), *R = f64(), *P64 = f64(), *Q = f64(), *T = f64(), *M = f64();
    float2 *FX = f32(), *FR = f32(), *FP = f32(), *FQ = f32(), *FT = f32(), *FO = f32();
    FieldPtrs fx{}, fb{};
    for (int i = 0; i < nb; i++) {
      fx.f[i] = (double2 *)xs[i];
      fb.f[i] = (double2 *)bs[i];
    }
    k_multi_pack<<<nblk(wall * nb, 256), 256, 0, L.stream>>>(X, fx, 0, wall, nb, 0);
    YG_LAUNCHED();
    k_multi_pack<<<nblk(wall * nb, 256), 256, 0, L.stream>>>(B, fb, 0, wall, nb, 0);
    YG_LAUNCHED();
    const int sg = (int)std::min<long>(nblk(nview, 256), 148L * 16);
    auto residual = [&]() {               // R = B - A X (FP64), per-system |R|^2
      YG_CUDA(cudaMemcpyAsync(P64, X, sizeof(double2) * (size_t)wall * nb, cudaMemcpyDeviceToDevice, L.stream));
      op_multi(L, YG_OP_HPHI_SQ, nb, par.mass, Q, P64, T, M);
      k_multi_sub<<<m.grid, m.threads, 0, L.stream>>>(R, B, Q, m.w0, m.cnt, nb);
      YG_LAUNCHED();
      return m.sqnorm(R);
    };
    auto f_reduce = [&](int kind, const float2 *a, const float2 *b) {
      if (kind == 0) k_fm_reduce<0><<<m.grid, m.threads, 0, L.stream>>>(m.part.as<double>(), a, b, m.cnt, nb);
      else k_fm_reduce<1><<<m.grid, m.threads, 0, L.stream>>>(m.part.as<double>(), a, b, m.cnt, nb);
      YG_LAUNCHED();
      return m.sums();
    };
    const std::vector<double> norm = m.sqnorm(B);
    std::vector<double> rr = residual(), rr_s(nb), maxrr(nb), best(nb), min_cycle(nb);
    std::vector<int> active(nb), it(nb, 0), stall(nb, 0), since(nb, 0);
    int nactive = 0, updates = 0;
    for (int i = 0; i < nb; i++) {
      active[i] = !(rr[i] < norm[i] * par.prec);
      nactive += active[i];
      rr_s[i] = maxrr[i] = best[i] = min_cycle[i] = rr[i];
    }
    k_fm_from_d<<<sg, 256, 0, L.stream>>>(FR, R, nview);
    YG_LAUNCHED();
    YG_CUDA(cudaMemcpyAsync(FP, FR, sizeof(float2) * (size_t)nview, cudaMemcpyDeviceToDevice, L.stream));
    const double d2 = delta * delta;
    constexpr int kStagnate = 100;
    bool fallback = false;
    int k = 0;
    while (nactive > 0) {
      k++;
      if (par.maxiter > 0 && k > par.maxiter) { status = YG_MAXITER; break; }
      fhphi_multi(L, nb, FT, FP, FO);
      fhphi_multi(L, nb, FQ, FT, FO);
      const std::vector<double> pq = f_reduce(0, FP, FQ);
      MultiScalars al{}, be{}, on{};
      for (int i = 0; i < nb; i++) {
        if (!active[i]) continue;
        if (!std::isfinite(pq[i])) throw Error(YG_NONFINITE, "non-finite value in cg_mixed_multi");
        al.a[i] = rr_s[i] / pq[i];
      }
      k_fm_update<<<m.grid, m.threads, 0, L.stream>>>(m.part.as<double>(), FX, FR, FP, FQ, al, m.cnt, nb);
      YG_LAUNCHED();
      const std::vector<double> rn = m.sums();
      bool trigger = false;
      for (int i = 0; i < nb; i++) {
        if (!active[i]) continue;
        it[i] = k;
        be.a[i] = rn[i] / rr_s[i];
        on.a[i] = 1.0;
        rr_s[i] = rn[i];
        if (rn[i] < 0.25 * min_cycle[i]) { min_cycle[i] = rn[i]; since[i] = 0; }
        else since[i]++;
        if (rn[i] < d2 * maxrr[i] || rn[i] < norm[i] * par.prec || since[i] >= kStagnate) trigger = true;
      }
      k_fm_xpay<<<m.grid, m.threads, 0, L.stream>>>(FP, FR, be, on, m.cnt, nb);
      YG_LAUNCHED();
      if (!trigger) continue;
      // reliable update of every system: fold the FP32 increments into X, recompute R
      k_fm_add_to_d<<<sg, 256, 0, L.stream>>>(X, FX, nview);
      YG_LAUNCHED();
      YG_CUDA(cudaMemsetAsync(FX, 0, sizeof(float2) * (size_t)nview, L.stream));
      const std::vector<double> rt = residual();
      updates++;
      for (int i = 0; i < nb; i++) {
        if (!active[i]) continue;
        rr[i] = rt[i];
        if (rt[i] < norm[i] * par.prec) {
          active[i] = 0;
          nactive--;
          continue;
        }
        if (rt[i] > 100.0 * best[i]) fallback = true;             // the inner solve diverged
        if (rt[i] < 0.5 * best[i]) stall[i] = 0;
        else if (++stall[i] >= 8) fallback = true;
        best[i] = std::min(best[i], rt[i]);
        rr_s[i] = maxrr[i] = min_cycle[i] = rt[i];
        since[i] = 0;
      }
      if (fallback) break;
      k_fm_from_d<<<sg, 256, 0, L.stream>>>(FR, R, nview);
      YG_LAUNCHED();
    }
    if (status == YG_MAXITER) {
      k_fm_add_to_d<<<sg, 256, 0, L.stream>>>(X, FX, nview);
      YG_LAUNCHED();
    }
    k_multi_pack<<<nblk(nview, 256), 256, 0, L.stream>>>(X, fx, m.w0, m.cnt, nb, 1);
    YG_LAUNCHED();
    YG_CUDA(cudaStreamSynchronize(L.stream));
    std::vector<int> fb_flag(nb, 0);
    if (fallback) {
      // the systems still open continue with the batched FP64 CG from their iterates
      std::vector<double *> ox, ob;
      std::vector<int> idx;
      for (int i = 0; i < nb; i++)
        if (active[i]) { ox.push_back(xs[i]); ob.push_back(bs[i]); idx.push_back(i); }
      for (void *b : bufs) cudaFree(b);
      bufs.clear();
      std::vector<int> its(idx.size());
      yg_inv_par p64 = par;
      p64.log = 0;
      status = cg_multi(L, p64, (int)idx.size(), ox.data(), ob.data(), its.data());
      for (size_t q = 0; q < idx.size(); q++) {
        it[idx[q]] += its[q];
        fb_flag[idx[q]] = 1;
      }
      // true residuals of the fallback systems
      Multi m2(L, nb);
      double2 *X2 = m2.field(), *B2 = m2.field(), *R2 = m2.field(), *Q2 = m2.field(), *T2 = m2.field(),
              *M2 = m2.field();
      bufs = {X2, B2, R2, Q2, T2, M2};
      k_multi_pack<<<nblk(wall * nb, 256), 256, 0, L.stream>>>(X2, fx, 0, wall, nb, 0);
      YG_LAUNCHED();
      k_multi_pack<<<nblk(wall * nb, 256), 256, 0, L.stream>>>(B2, fb, 0, wall, nb, 0);
      YG_LAUNCHED();
      op_multi(L, YG_OP_HPHI_SQ, nb, par.mass, Q2, X2, T2, M2);
      k_multi_sub<<<m2.grid, m2.threads, 0, L.stream>>>(R2, B2, Q2, m2.w0, m2.cnt, nb);
      YG_LAUNCHED();
      rr = m2.sqnorm(R2);
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int i = 0; i < nb; i++) {
      if (status == YG_OK && rr[i] >= norm[i] * par.prec) status = YG_STALL;
      if (stats) {
        stats[i].iterations = it[i];
        stats[i].reliable_updates = updates;
        stats[i].fallback = fb_flag[i];
        stats[i].true_residual = rr[i] / norm[i];
        stats[i].seconds = secs;
      }
    }
    if (par.log)
      for (int i = 0; i < nb; i++)
        fprintf(stderr, "[INVERTER][30]cg_mixed_multi[%d]: iterations = %d, precision = %1.4e\n", i, it[i],
                rr[i] / norm[i]);
  } catch (...) {
    for (void *b : bufs) cudaFree(b);
    throw;
  }
  for (void *b : bufs) cudaFree(b);
  return status;
}

}  // namespace yg
