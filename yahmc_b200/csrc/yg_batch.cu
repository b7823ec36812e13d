// Persistent uneven-volume batch: independent cg_inverter solves (cg.cpp:132-202) of Hphi_sq on
// several even-odd lattices of different sizes in ONE cooperative kernel launch.
//
// A small lattice's CG is bound by launch and reduction latency: a 8^4 or 12^4 operator step
// fills a few SMs for a few microseconds, and the reference's recurrence needs two host
// round trips per iteration (<p,q> for alpha, |r|^2 for beta and the stopping test).  Here
// the grid is split into one group of blocks per lattice, sized in proportion to the
// lattice's even volume (at least one block each), and every group runs its lattice's whole
// CG loop on the device:
//
//   P1  o = A_oo^-1 (1/2 H p)              (odd sites)
//   P2  t = g5 (A_ee p - 1/2 H o)          (even sites)          t = Hphi p
//   P3  o = A_oo^-1 (1/2 H t)
//   P4  q = g5 (A_ee t - 1/2 H o), <p,q>   (even sites)          q = Hphi_sq p
//   P5  x += alpha p, r -= alpha q, |r|^2
//   P6  p = beta p + r
//
// with a barrier of the group after each phase.  The operator steps are the FP64 Schur steps
// of the single-lattice path (hop_body of yg_dirac_impl.cuh with the same epilogues), and the
// scalars are the reference's: alpha = rr / <p,q>, beta = rr_new / rr, stop when
// rr_new < prec |b|^2, iteration count as cg_inverter's.  Reductions are deterministic: one
// partial per block, which every block of the group adds in block order after the barrier,
// so all blocks of a group hold the same alpha and beta.  Groups never wait for each other:
// a lattice that converges early just ends its blocks.
//
// Barriers: a counter and a generation word per group in global memory.  Every wait is
// bounded by a cycle limit; a block whose wait runs out sets the launch's error flag and
// returns, every other block returns at its next barrier once the flag is set, and the host
// reports YG_TIMEOUT.  The launch is cooperative, so all blocks are resident and in a healthy
// run every barrier completes; the limit is the guard against anything else.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>
#include "yg_lattice.h"
#include "yg_kernels.h"
#include "yg_dirac_impl.cuh"

namespace yg {

namespace {

constexpr int kThreads = 128;
constexpr long long kDefaultWait = 20000000000LL;   // cycles (about 10 s at 2 GHz)

struct BLat {
  HopArgs<double> s1a, s2a, s1b, s2b;   // P1, P2, P3, P4
  double2 *x, *r, *p, *q;              // even-site words of the whole-field layout
  int b0, nb;                          // the group's blocks [b0, b0 + nb)
  int maxiter, it0;                    // it0 = -1: solved by the initial guess, no iteration
  double target, rr0;                  // prec |b|^2, |r|^2 of the initial residual
};

struct BOut {
  int iters, status;
  double rr;
};

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[kThreads / 32];
  __syncthreads();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int w = 0; w < kThreads / 32; w++) s += sh[w];
  return s;
}

// sum of the group's partials in block order (the same value in every block of the group)
__device__ __forceinline__ double group_total(const double *part, int b0, int nb) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += kThreads) acc += part[b0 + i];
  return block_sum(acc);
}

// barrier of the nb blocks of a group; false when this block's wait ran out or another
// block of the launch gave up (the error flag is set), in which case the block returns
__device__ __forceinline__ bool group_sync(unsigned *cnt, unsigned *gen, unsigned nb, int *err, long long limit) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int good = 1;
    volatile unsigned *vgen = gen;
    volatile int *verr = err;
    const unsigned g0 = *vgen;
    __threadfence();                                   // this block's stores before its arrival
    if (atomicAdd(cnt, 1u) == nb - 1) {
      atomicExch(cnt, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      const long long t0 = clock64();
      while (*vgen == g0) {
        if (*verr) { good = 0; break; }
        if (clock64() - t0 > limit) { atomicExch(err, 1); good = 0; break; }
        __nanosleep(100);
      }
    }
    __threadfence();
    if (*verr) good = 0;
    ok = good;
  }
  __syncthreads();
  return ok != 0;
}

// the two Schur steps as called functions, one body each however often the loop calls them
template <int D, int EPI>
__device__ __noinline__ void step(const HopArgs<double> &a, int t) {
  hop_body<D, double, EPI>(a, t);
}

// CLOV = 1: A_oo^-1 from the packed inverse blocks and A_ee from the clover term (d <= 6);
// CLOV = 0: no clover term, A_oo = 1 and the (4+m)^2 diagonal.  Registers are capped for 3
// resident CTAs per SM, so that a 16^4 lattice's group covers its 32768 even sites in one
// pass of the grid (one site per thread).
template <int D, int CLOV>
__global__ void __launch_bounds__(kThreads, 3) k_cg_batch(const BLat *lats, int n, double *part_pq, double *part_rr,
                                                       unsigned *sync, int *err, BOut *out, long long limit) {
  constexpr int E1 = CLOV ? EPI_CLOVPK : EPI_PLAIN, E2 = CLOV ? EPI_CLOVADD : EPI_AXPY;
  int li = 0;
  while (li + 1 < n && (int)blockIdx.x >= lats[li + 1].b0) li++;
  const BLat &L = lats[li];
  const int lb = blockIdx.x - L.b0;
  const int first = lb * kThreads + threadIdx.x, stride = L.nb * kThreads;
  const int Vh = L.s2a.g.Vh;
  constexpr int NC = 4 * D;                          // complex words per site
  unsigned *cnt = sync + 2 * li, *gen = cnt + 1;
  double rr = L.rr0;
  int it = 0, status = YG_OK;
  // cg.cpp:151-153: a system solved by its initial guess returns 0 iterations
  while (L.it0 == 0) {
    ++it;
    if (L.maxiter > 0 && it > L.maxiter) { it--; status = YG_MAXITER; break; }
    for (int t = first; t < Vh; t += stride) step<D, E1>(L.s1a, t);
    if (!group_sync(cnt, gen, L.nb, err, limit)) { status = YG_TIMEOUT; break; }
    for (int t = first; t < Vh; t += stride) step<D, E2>(L.s2a, t);
    if (!group_sync(cnt, gen, L.nb, err, limit)) { status = YG_TIMEOUT; break; }
    for (int t = first; t < Vh; t += stride) step<D, E1>(L.s1b, t);
    if (!group_sync(cnt, gen, L.nb, err, limit)) { status = YG_TIMEOUT; break; }
    double acc = 0.0;
    for (int t = first; t < Vh; t += stride) {
      step<D, E2>(L.s2b, t);
      double s = 0.0;                                // Re <p, q> of the site just written
#pragma unroll 4
      for (int k = 0; k < NC; k++) {
        const long i = (long)k * Vh + t;
        const double2 pv = L.p[i], qv = L.q[i];
        s = fma(pv.x, qv.x, fma(pv.y, qv.y, s));
      }
      acc += s;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part_pq[blockIdx.x] = acc;
    if (!group_sync(cnt, gen, L.nb, err, limit)) { status = YG_TIMEOUT; break; }
    const double pq = group_total(part_pq, L.b0, L.nb);
    if (!isfinite(pq)) { status = YG_NONFINITE; break; }
    const double alpha = rr / pq;
    acc = 0.0;
    for (int t = first; t < Vh; t += stride) {
      double s = 0.0;
#pragma unroll 4
      for (int k = 0; k < NC; k++) {
        const long i = (long)k * Vh + t;
        const double2 pv = L.p[i], qv = L.q[i];
        double2 xv = L.x[i], rv = L.r[i];
        xv.x = fma(alpha, pv.x, xv.x);
        xv.y = fma(alpha, pv.y, xv.y);
        rv.x = fma(-alpha, qv.x, rv.x);
        rv.y = fma(-alpha, qv.y, rv.y);
        L.x[i] = xv;
        L.r[i] = rv;
        s = fma(rv.x, rv.x, fma(rv.y, rv.y, s));
      }
      acc += s;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part_rr[blockIdx.x] = acc;
    if (!group_sync(cnt, gen, L.nb, err, limit)) { status = YG_TIMEOUT; break; }
    const double rrn = group_total(part_rr, L.b0, L.nb);
    if (!isfinite(rrn)) { status = YG_NONFINITE; break; }
    const double beta = rrn / rr;
    rr = rrn;
    if (rr < L.target) break;
    for (int t = first; t < Vh; t += stride) {
#pragma unroll 4
      for (int k = 0; k < NC; k++) {
        const long i = (long)k * Vh + t;
        const double2 pv = L.p[i], rv = L.r[i];
        L.p[i] = make_double2(fma(beta, pv.x, rv.x), fma(beta, pv.y, rv.y));
      }
    }
    if (!group_sync(cnt, gen, L.nb, err, limit)) { status = YG_TIMEOUT; break; }
  }
  if (lb == 0 && threadIdx.x == 0) {
    out[li].iters = it;
    out[li].status = status;
    out[li].rr = rr;
  }
}

template <int D, int CLOV>
void launch_batch(int grid, cudaStream_t s, const BLat *lats, int n, double *part_pq, double *part_rr,
                  unsigned *sync, int *err, BOut *out, long long limit) {
  void *args[] = {(void *)&lats, (void *)&n, (void *)&part_pq, (void *)&part_rr, (void *)&sync, (void *)&err,
                  (void *)&out, (void *)&limit};
  YG_CUDA(cudaLaunchCooperativeKernel((const void *)k_cg_batch<D, CLOV>, dim3(grid), dim3(kThreads), args, 0, s));
  YG_LAUNCHED();
}

template <int D, int CLOV>
int resident_blocks() {
  int dev = 0, sms = 0, per = 0;
  YG_CUDA(cudaGetDevice(&dev));
  YG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  YG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cg_batch<D, CLOV>, kThreads, 0));
  return sms * per;
}

// the representation dimensions of the persistent batch: SU(2) fundamental (2), SU(3)
// fundamental and SU(2) adjoint (3), SU(4) fundamental (4), SU(3) sextet and SU(4)
// antisymmetric (6)
#define YG_BATCH_D(DV, CV, ...)                                                                                    \
  do {                                                                                                            \
    const bool cv_ = (CV);                                                                                        \
    switch (DV) {                                                                                                 \
      case 2: if (cv_) { constexpr int BD = 2, BC = 1; __VA_ARGS__; } else { constexpr int BD = 2, BC = 0; __VA_ARGS__; } break; \
      case 3: if (cv_) { constexpr int BD = 3, BC = 1; __VA_ARGS__; } else { constexpr int BD = 3, BC = 0; __VA_ARGS__; } break; \
      case 4: if (cv_) { constexpr int BD = 4, BC = 1; __VA_ARGS__; } else { constexpr int BD = 4, BC = 0; __VA_ARGS__; } break; \
      case 6: if (cv_) { constexpr int BD = 6, BC = 1; __VA_ARGS__; } else { constexpr int BD = 6, BC = 0; __VA_ARGS__; } break; \
      default: throw Error(YG_ERR_ARG, "the persistent batch exists for d = 2, 3, 4, 6");                        \
    }                                                                                                             \
  } while (0)

HopArgs<double> step_args(Lattice &L, bool first_step, double mass, const double *src, double *dst,
                          const double *src2) {
  HopArgs<double> a{};
  a.g = L.g;
  a.cfm1 = L.p.cf - 1.0;
  a.U = L.links.as<double2>();
  a.src = (const double2 *)src;
  a.dst = (double2 *)dst;
  a.n = (int)L.Vh;
  if (first_step) {                          // schur_step1: odd output, A_oo^-1 (1/2 H src)
    a.lo = (int)L.Vh;
    a.coeff = 0.5;
    if (L.p.clover) a.cpk = L.cpk64.as<double2>();
  } else {                                   // schur_step2: even output, g5 (A_ee src2 - 1/2 H src)
    a.lo = 0;
    a.src2 = (const double2 *)src2;
    a.coeff = -0.5;
    a.g5 = 1;
    a.zero_add_at_boundary = 1;
    if (L.p.clover) { a.cl = L.clover.as<double2>(); a.diag = 4.0 + mass; }
    else a.diag = (4.0 + mass) * (4.0 + mass);
  }
  return a;
}

}  // namespace

bool batch_eligible(int n, Lattice *const *L, const yg_inv_par *par) {
  const int d = L[0]->d;
  if (d != 2 && d != 3 && d != 4 && d != 6) return false;
  for (int i = 0; i < n; i++) {
    const Lattice &l = *L[i];
    if (par[i].op != YG_OP_HPHI_SQ || !l.p.eo || l.d != d || l.p.clover != L[0]->p.clover) return false;
    if (l.p.bc == YG_BC_OPEN || l.p.bc == YG_BC_SF) return false;   // spinor boundary slices
  }
  return true;
}

// The cg_inverter prologue on every lattice (cg.cpp:134-150: r = b - A x, p = r, |b|^2, |r|^2)
// with the engine's ordinary launches, then one persistent launch for all iterations.
int cg_lattices_persistent(int n, Lattice *const *L, const yg_inv_par *par, double *const *xs, double *const *bs,
                           int *iters, long long wait_cycles) {
  if (n < 1 || n > 64) throw Error(YG_ERR_ARG, "1..64 lattices");
  if (!batch_eligible(n, L, par))
    throw Error(YG_ERR_ARG, "the persistent batch solves Hphi_sq on even-odd lattices of one d (2, 3, 4 or 6), "
                            "all with or all without a clover term, without open/SF boundaries");
  const int d = L[0]->d;
  const bool clov = L[0]->p.clover;
  std::vector<BLat> h(n);
  long vol = 0;
  for (int i = 0; i < n; i++) vol += L[i]->Vh;
  int grid_max = 0;
  YG_BATCH_D(d, clov, grid_max = resident_blocks<BD, BC>());
  if (grid_max < n) throw Error(YG_ERR_ARG, "more lattices than resident blocks");
  int b0 = 0;
  for (int i = 0; i < n; i++) {
    Lattice &l = *L[i];
    const double mass = par[i].mass;
    double *r = l.scratch_field(3), *p = l.scratch_field(4), *q = l.scratch_field(5);
    double *t = l.scratch_field(2), *o = l.scratch_field(1);
    long lo, cnt;
    l.view_range(YG_VIEW_DEFAULT, lo, cnt);
    blas_copy(l, p, xs[i]);
    apply_op(l, YG_OP_HPHI_SQ, mass, q, p);    // also builds the clover inverse for this mass
    blas_copy(l, r, bs[i]);
    blas_axpby(l, r, make_double2(1, 0), make_double2(-1, 0), q, lo, cnt);
    blas_copy(l, p, r);
    const double norm = blas_sqnorm(l, bs[i], lo, cnt);
    const double rr = blas_sqnorm(l, r, lo, cnt);
    BLat &b = h[i];
    b.s1a = step_args(l, true, mass, p, o, nullptr);
    b.s2a = step_args(l, false, mass, o, t, p);
    b.s1b = step_args(l, true, mass, t, o, nullptr);
    b.s2b = step_args(l, false, mass, o, q, t);
    b.x = (double2 *)xs[i];
    b.r = (double2 *)r;
    b.p = (double2 *)p;
    b.q = (double2 *)q;
    b.maxiter = par[i].maxiter;
    b.target = norm * par[i].prec;
    b.rr0 = rr;
    b.it0 = rr < b.target ? -1 : 0;
    // blocks in proportion to the even volume, at least one, at most one per 128 sites
    const long share = (long)((double)grid_max * (double)l.Vh / (double)vol);
    b.nb = (int)std::max<long>(1, std::min<long>(share, nblk(l.Vh, kThreads)));
    b.b0 = b0;
    b0 += b.nb;
    YG_CUDA(cudaStreamSynchronize(l.stream));
  }
  const int grid = b0;
  if (grid > grid_max) throw Error(YG_ERR_ARG, "block groups exceed the resident grid");
  // one device allocation: lattice records, partials, barrier words, error flag, results
  const size_t off_part = ((sizeof(BLat) * n + 255) / 256) * 256;
  const size_t off_sync = off_part + 2 * sizeof(double) * grid;
  const size_t off_err = off_sync + ((sizeof(unsigned) * 2 * n + 15) / 16) * 16;
  const size_t off_out = off_err + 16;
  const size_t bytes = off_out + sizeof(BOut) * n;
  DevBuf buf;
  buf.alloc(bytes);
  char *base = buf.as<char>();
  cudaStream_t s = L[0]->stream;
  int err = 0;
  std::vector<BOut> res(n);
  try {
    YG_CUDA(cudaMemsetAsync(base, 0, bytes, s));
    YG_CUDA(cudaMemcpyAsync(base, h.data(), sizeof(BLat) * n, cudaMemcpyHostToDevice, s));
    const long long limit = wait_cycles > 0 ? wait_cycles : kDefaultWait;
    double *part = reinterpret_cast<double *>(base + off_part);
    YG_BATCH_D(d, clov, launch_batch<BD, BC>(grid, s, reinterpret_cast<const BLat *>(base), n, part, part + grid,
                                             reinterpret_cast<unsigned *>(base + off_sync),
                                             reinterpret_cast<int *>(base + off_err),
                                             reinterpret_cast<BOut *>(base + off_out), limit));
    YG_CUDA(cudaMemcpyAsync(res.data(), base + off_out, sizeof(BOut) * n, cudaMemcpyDeviceToHost, s));
    YG_CUDA(cudaMemcpyAsync(&err, base + off_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    YG_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    cudaStreamSynchronize(s);
    buf.release();
    throw;
  }
  buf.release();
  int worst = YG_OK;
  for (int i = 0; i < n; i++) {
    iters[i] = res[i].iters;
    L[i]->mvm += 4 * res[i].iters;
    if (par[i].log)
      fprintf(stderr, "[INVERTER][30]cg: iterations = %d, precision = %1.4e\n", res[i].iters,
              res[i].rr / (h[i].target / par[i].prec));
    if (res[i].status != YG_OK && worst == YG_OK) worst = res[i].status;
  }
  if (err) return YG_TIMEOUT;
  return worst;
}

}  // namespace yg
