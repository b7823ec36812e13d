// Spinor-field linear algebra (linalg.cpp:29-270) on the device.
//
// A view of a field is a contiguous range of complex words in the device layout
// (yg_core.cuh): block 0 (even) then block 1 (odd), each 4d*Vh words, so every
// operation here is a flat streaming pass.  Reductions are deterministic: a fixed
// grid of blocks each reduces its slice by a fixed tree (warp shuffles, then shared
// memory) into one FP64 partial, and a single block sums the partials in index order.
// That replaces the OpenMP reduction + mp_global_sum of linalg.cpp:55-270.
#include <vector>
#include "yg_lattice.h"
#include "yg_kernels.h"

namespace yg {

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// block-wide sum of a double2, result valid in thread 0
__device__ __forceinline__ double2 block_sum2(double2 v) {
  __shared__ double2 sh[32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum2(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? sh[threadIdx.x] : make_double2(0, 0);
  if (w == 0) v = warp_sum2(v);
  return v;
}

// kind 0: sum |a|^2 ; 1: sum a*conj(b) ; 2: Re sum a*conj(b)
template <int KIND>
__global__ void __launch_bounds__(256) k_reduce(double2 *partial, const double2 *a, const double2 *b, long n) {
  double2 acc = make_double2(0, 0);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double2 x = a[i];
    if (KIND == 0) {
      acc.x = fma(x.x, x.x, acc.x);
      acc.x = fma(x.y, x.y, acc.x);
    } else {
      double2 y = b[i];
      acc.x = fma(x.x, y.x, acc.x);
      acc.x = fma(x.y, y.y, acc.x);
      if (KIND == 1) {
        acc.y = fma(x.y, y.x, acc.y);
        acc.y = fma(-x.x, y.y, acc.y);
      }
    }
  }
  acc = block_sum2(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(1024) k_reduce_final(double2 *result, const double2 *partial, int nparts) {
  double2 acc = make_double2(0, 0);
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) {
    acc.x += partial[i].x;
    acc.y += partial[i].y;
  }
  acc = block_sum2(acc);
  if (threadIdx.x == 0) *result = acc;
}

static int red_grid(Lattice &L, long n) {
  int g = nblk(n, 256);
  return g < L.red_blocks ? g : L.red_blocks;
}

double2 reduce_partials(Lattice &L, int grid) {
  k_reduce_final<<<1, 1024, 0, L.stream>>>(L.red_result.as<double2>(), L.red_partial.as<double2>(), grid);
  YG_LAUNCHED();
  YG_CUDA(cudaMemcpyAsync(L.host_result, L.red_result.p, sizeof(double2), cudaMemcpyDeviceToHost, L.stream));
  YG_CUDA(cudaStreamSynchronize(L.stream));
  return make_double2(L.host_result[0], L.host_result[1]);
}

static inline long woff(const Lattice &L, long lo) { return lo * 4L * L.d; }   // site -> complex word
static inline long wcnt(const Lattice &L, long n) { return n * 4L * L.d; }

double blas_sqnorm(Lattice &L, const double *a, long lo, long n) {
  long cnt = wcnt(L, n);
  int grid = red_grid(L, cnt);
  k_reduce<0><<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), (const double2 *)a + woff(L, lo), nullptr, cnt);
  YG_LAUNCHED();
  return reduce_partials(L, grid).x;
}

double2 blas_product(Lattice &L, const double *a, const double *b, long lo, long n) {
  long cnt = wcnt(L, n);
  int grid = red_grid(L, cnt);
  k_reduce<1><<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), (const double2 *)a + woff(L, lo),
                                           (const double2 *)b + woff(L, lo), cnt);
  YG_LAUNCHED();
  return reduce_partials(L, grid);
}

double blas_product_re(Lattice &L, const double *a, const double *b, long lo, long n) {
  long cnt = wcnt(L, n);
  int grid = red_grid(L, cnt);
  k_reduce<2><<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), (const double2 *)a + woff(L, lo),
                                           (const double2 *)b + woff(L, lo), cnt);
  YG_LAUNCHED();
  return reduce_partials(L, grid).x;
}

// lhs = alpha*lhs + beta*rhs  (alpha == 0 does not read lhs; rhs == null drops the term)
__global__ void __launch_bounds__(256) k_axpby(double2 *lhs, double2 alpha, double2 beta, const double2 *rhs,
                                               long n, int read_lhs) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double2 r = make_double2(0, 0);
    if (read_lhs) r = cmul(alpha, lhs[i]);
    if (rhs) cfma(r, beta, rhs[i]);
    lhs[i] = r;
  }
}

static int stream_grid(long n) {
  int g = nblk(n, 256);
  const int cap = 148 * 16;
  return g < cap ? g : cap;
}

void blas_axpby(Lattice &L, double *lhs, double2 alpha, double2 beta, const double *rhs, long lo, long n) {
  long cnt = wcnt(L, n);
  int read_lhs = !(alpha.x == 0.0 && alpha.y == 0.0);
  k_axpby<<<stream_grid(cnt), 256, 0, L.stream>>>((double2 *)lhs + woff(L, lo), alpha, beta,
                                                    rhs ? (const double2 *)rhs + woff(L, lo) : nullptr, cnt, read_lhs);
  YG_LAUNCHED();
}

__global__ void __launch_bounds__(256) k_neg(double2 *f, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double2 v = f[i];
    f[i] = make_double2(-v.x, -v.y);
  }
}

// gamma5 = diag(1,1,-1,-1) (spinor.cpp:255-264): spins 2,3 are the upper half of each block
void blas_g5(Lattice &L, double *f, long lo, long n) {
  long per_blk = 4L * L.d * L.Vh;
  for (long blk = lo / L.Vh; blk * L.Vh < lo + n; blk++) {
    double2 *base = (double2 *)f + blk * per_blk + 2L * L.d * L.Vh;
    long cnt = 2L * L.d * L.Vh;
    k_neg<<<stream_grid(cnt), 256, 0, L.stream>>>(base, cnt);
    YG_LAUNCHED();
  }
}

void blas_copy(Lattice &L, double *dst, const double *src) {
  if (dst == src) return;
  YG_CUDA(cudaMemcpyAsync(dst, src, L.field_bytes(), cudaMemcpyDeviceToDevice, L.stream));
}

void blas_zero(Lattice &L, double *f, long lo, long n) {
  YG_CUDA(cudaMemsetAsync((double2 *)f + woff(L, lo), 0, sizeof(double2) * wcnt(L, n), L.stream));
}

// x += a p ; r -= a q ; partial |r|^2   (cg.cpp:181-186 in one pass)
__global__ void __launch_bounds__(256) k_cg_update(double2 *partial, double2 *x, double2 *r, const double2 *p,
                                                   const double2 *q, double a, long n) {
  double2 acc = make_double2(0, 0);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double2 pi = p[i], qi = q[i], xi = x[i], ri = r[i];
    xi.x = fma(a, pi.x, xi.x);
    xi.y = fma(a, pi.y, xi.y);
    ri.x = fma(-a, qi.x, ri.x);
    ri.y = fma(-a, qi.y, ri.y);
    x[i] = xi;
    r[i] = ri;
    acc.x = fma(ri.x, ri.x, acc.x);
    acc.x = fma(ri.y, ri.y, acc.x);
  }
  acc = block_sum2(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

double blas_cg_update(Lattice &L, double *x, double *r, const double *p, const double *q, double a, long lo, long n) {
  long cnt = wcnt(L, n);
  int grid = red_grid(L, cnt);
  long o = woff(L, lo);
  k_cg_update<<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), (double2 *)x + o, (double2 *)r + o,
                                           (const double2 *)p + o, (const double2 *)q + o, a, cnt);
  YG_LAUNCHED();
  return reduce_partials(L, grid).x;
}

// sum of n doubles (per-site partials of logdet / plaquette), deterministic
__global__ void __launch_bounds__(256) k_sum_partial(double2 *partial, const double *v, long n) {
  double2 acc = make_double2(0, 0);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) acc.x += v[i];
  acc = block_sum2(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

double sum_device(Lattice &L, const double *v, long n) {
  int grid = red_grid(L, n);
  k_sum_partial<<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), v, n);
  YG_LAUNCHED();
  return reduce_partials(L, grid).x;
}

// ---------------------------------------------------------------- FP32 helpers (mixed solver)
__global__ void k_d2f(float2 *dst, const double2 *src, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}

__global__ void k_f2d_add(double2 *dst, const float2 *src, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double2 v = dst[i];
    v.x += (double)src[i].x;
    v.y += (double)src[i].y;
    dst[i] = v;
  }
}

template <int KIND>
__global__ void __launch_bounds__(256) k_reduce_f(double2 *partial, const float2 *a, const float2 *b, long n) {
  double2 acc = make_double2(0, 0);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float2 x = a[i];
    if (KIND == 0) {
      acc.x += (double)x.x * x.x + (double)x.y * x.y;
    } else {
      float2 y = b[i];
      acc.x += (double)x.x * y.x + (double)x.y * y.y;
    }
  }
  acc = block_sum2(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// x += a p ; r -= a q (FP32 storage, FP32 arithmetic) ; partial |r|^2 in FP64
__global__ void __launch_bounds__(256) k_cg_update_f(double2 *partial, float2 *x, float2 *r, const float2 *p,
                                                     const float2 *q, float a, long n) {
  double2 acc = make_double2(0, 0);
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float2 pi = p[i], qi = q[i], xi = x[i], ri = r[i];
    xi.x = fmaf(a, pi.x, xi.x);
    xi.y = fmaf(a, pi.y, xi.y);
    ri.x = fmaf(-a, qi.x, ri.x);
    ri.y = fmaf(-a, qi.y, ri.y);
    x[i] = xi;
    r[i] = ri;
    acc.x += (double)ri.x * ri.x + (double)ri.y * ri.y;
  }
  acc = block_sum2(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// p = b*p + r
__global__ void k_xpay_f(float2 *p, float b, const float2 *r, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    float2 pi = p[i], ri = r[i];
    pi.x = fmaf(b, pi.x, ri.x);
    pi.y = fmaf(b, pi.y, ri.y);
    p[i] = pi;
  }
}

void f_from_d(Lattice &L, float *dst, const double *src, long cnt) {
  k_d2f<<<stream_grid(cnt), 256, 0, L.stream>>>((float2 *)dst, (const double2 *)src, cnt);
  YG_LAUNCHED();
}

void d_add_f(Lattice &L, double *dst, const float *src, long cnt) {
  k_f2d_add<<<stream_grid(cnt), 256, 0, L.stream>>>((double2 *)dst, (const float2 *)src, cnt);
  YG_LAUNCHED();
}

double f_sqnorm(Lattice &L, const float *a, long cnt) {
  int grid = red_grid(L, cnt);
  k_reduce_f<0><<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), (const float2 *)a, nullptr, cnt);
  YG_LAUNCHED();
  return reduce_partials(L, grid).x;
}

double f_product_re(Lattice &L, const float *a, const float *b, long cnt) {
  int grid = red_grid(L, cnt);
  k_reduce_f<2><<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), (const float2 *)a, (const float2 *)b, cnt);
  YG_LAUNCHED();
  return reduce_partials(L, grid).x;
}

double f_cg_update(Lattice &L, float *x, float *r, const float *p, const float *q, float a, long cnt) {
  int grid = red_grid(L, cnt);
  k_cg_update_f<<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), (float2 *)x, (float2 *)r,
                                             (const float2 *)p, (const float2 *)q, a, cnt);
  YG_LAUNCHED();
  return reduce_partials(L, grid).x;
}

void f_xpay(Lattice &L, float *p, float b, const float *r, long cnt) {
  k_xpay_f<<<stream_grid(cnt), 256, 0, L.stream>>>((float2 *)p, b, (const float2 *)r, cnt);
  YG_LAUNCHED();
}

// ---- cg_mshift updates of all shifts in one pass each (cg.cpp:62-116)
// Launch parameters carry the per-shift fields and coefficients of the active shifts.
struct MshiftArgs {
  double2 *x[kMaxShifts];
  double2 *k[kMaxShifts];
  double c_x[kMaxShifts];     // x_n -= c_x[n] k_n
  double c_kk[kMaxShifts];    // k_n = c_kk[n] k_n + c_kr[n] r
  double c_kr[kMaxShifts];
  int num;
};

// r += beta q (partial |r|^2) and x_n -= bt_n k_n for every active shift, one pass
__global__ void __launch_bounds__(256) k_mshift_xr(double2 *partial, double2 *r, const double2 *q, double beta,
                                                   MshiftArgs a, long n) {
  double acc = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    double2 v = r[i], w = q[i];
    v.x = fma(beta, w.x, v.x);
    v.y = fma(beta, w.y, v.y);
    r[i] = v;
    acc = fma(v.x, v.x, fma(v.y, v.y, acc));
    for (int s = 0; s < a.num; s++) {
      double2 xv = a.x[s][i], kv = a.k[s][i];
      xv.x = fma(-a.c_x[s], kv.x, xv.x);
      xv.y = fma(-a.c_x[s], kv.y, xv.y);
      a.x[s][i] = xv;
    }
  }
  double2 t = block_sum2(make_double2(acc, 0.0));
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

// k_n = at_n k_n + c3_n r for every active shift, and p = alpha p + r, one pass
__global__ void __launch_bounds__(256) k_mshift_kp(double2 *p, const double2 *r, double alpha, MshiftArgs a, long n) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const double2 rv = r[i];
    for (int s = 0; s < a.num; s++) {
      double2 kv = a.k[s][i];
      kv.x = fma(a.c_kr[s], rv.x, a.c_kk[s] * kv.x);
      kv.y = fma(a.c_kr[s], rv.y, a.c_kk[s] * kv.y);
      a.k[s][i] = kv;
    }
    if (p) {
      double2 pv = p[i];
      p[i] = make_double2(fma(alpha, pv.x, rv.x), fma(alpha, pv.y, rv.y));
    }
  }
}

static MshiftArgs mshift_args(const Lattice &L, int num, double *const *x, double *const *k, const double *c1,
                              const double *c2, const double *c3, long lo) {
  if (num < 0 || num > kMaxShifts) throw Error(YG_ERR_ARG, "too many shifts");
  MshiftArgs a{};
  a.num = num;
  const long o = woff(L, lo);
  for (int s = 0; s < num; s++) {
    a.x[s] = x ? (double2 *)x[s] + o : nullptr;
    a.k[s] = (double2 *)k[s] + o;
    a.c_x[s] = c1 ? c1[s] : 0.0;
    a.c_kk[s] = c2 ? c2[s] : 0.0;
    a.c_kr[s] = c3 ? c3[s] : 0.0;
  }
  return a;
}

double blas_mshift_xr(Lattice &L, double *r, const double *q, double beta, int num, double *const *x,
                      double *const *k, const double *bt, long lo, long n) {
  long cnt = wcnt(L, n);
  int grid = red_grid(L, cnt);
  MshiftArgs a = mshift_args(L, num, x, k, bt, nullptr, nullptr, lo);
  k_mshift_xr<<<grid, 256, 0, L.stream>>>(L.red_partial.as<double2>(), (double2 *)r + woff(L, lo),
                                           (const double2 *)q + woff(L, lo), beta, a, cnt);
  YG_LAUNCHED();
  return reduce_partials(L, grid).x;
}

void blas_mshift_kp(Lattice &L, double *p, const double *r, double alpha, int num, double *const *k,
                    const double *at, const double *c3, long lo, long n) {
  long cnt = wcnt(L, n);
  MshiftArgs a = mshift_args(L, num, nullptr, k, nullptr, at, c3, lo);
  k_mshift_kp<<<stream_grid(cnt), 256, 0, L.stream>>>(p ? (double2 *)p + woff(L, lo) : nullptr,
                                                       (const double2 *)r + woff(L, lo), alpha, a, cnt);
  YG_LAUNCHED();
}

}  // namespace yg
