// Allocation-free squared norm of a device field.
//
// yg_spinor_sqnorm needs a lattice handle, and creating one allocates device memory (the
// gauge field, the clover term and the reduction scratch).  Some callers cannot allocate:
// a host application that reserved the whole device for its own pools before it calls us,
// or code that must not call cudaMalloc because it would synchronise the device while
// other streams are busy.  yg_field_sqnorm_noalloc gives them the same reduction with no
// allocation at all: its per-block partial sums live in the file-scope array below, which
// every GPU that loads this library holds until the process exits.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "../../include/yahmc_gpu.h"

namespace {

constexpr int kThreads = 256;                 // threads per block
constexpr int kWordsPerThread = 8;            // complex words each thread sums
constexpr int kWordsPerBlock = kThreads * kWordsPerThread;
constexpr int kMaxBlocks = 8192;              // 8192 x 16 B = 128 KiB of scratch
constexpr long kMaxWords = (long)kMaxBlocks * kWordsPerBlock;   // 16,777,216 complex words

// One FP64 partial per block.  Every call writes all the partials it later reads, so
// nothing needs clearing between calls; calls that overlap on the GPU race on it.
static __device__ __align__(256) double noalloc_partials[kMaxBlocks];

// Device address of noalloc_partials, per device, looked up at the first call on that
// device.  Atomic because several host threads may make their first call at once; they
// all store the same address, so whichever store lands last is correct.
constexpr int kMaxDevices = 64;
std::atomic<double *> g_scratch[kMaxDevices] = {};

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = v;
  __syncthreads();
  v = (threadIdx.x < kThreads / 32) ? sh[threadIdx.x] : 0.0;
  if (w == 0) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  }
  return v;
}

__global__ void __launch_bounds__(kThreads) k_partials(double *partials, const double2 *a, long n) {
  long base = (long)blockIdx.x * kWordsPerBlock + threadIdx.x;
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j < kWordsPerThread; j++) {
    long i = base + (long)j * kThreads;
    if (i < n) {
      double2 x = a[i];
      acc = fma(x.x, x.x, acc);
      acc = fma(x.y, x.y, acc);
    }
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void __launch_bounds__(kThreads) k_final(double *out, const double *partials, int nparts) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += kThreads) acc += partials[i];
  acc = block_sum(acc);
  if (threadIdx.x == 0) *out = acc;
}

}  // namespace

namespace yg {
void set_last_error(const char *msg);   // yg_capi.cu: the message yg_last_error() returns
}

static int fail(int code, const char *msg) {
  yg::set_last_error(msg);
  return code;
}

// Sum of |a_i|^2 over n complex FP64 words at dev_words (a view of a field: the even
// half of a spinor field is its first 4*d*V/2 words), written to the device double
// *dev_out on `stream`.  Allocates nothing.  dev_words must be 16-byte aligned and dev_out
// 8-byte aligned (YG_ERR_ARG otherwise, checked before any launch).  The first call on a
// device looks up the device address of the scratch array with that device current and
// caches it for the process; make that first call before any stream capture.
extern "C" int yg_field_sqnorm_noalloc(const double *dev_words, long n_words, double *dev_out, void *stream) {
  if (!dev_words || !dev_out) return fail(YG_ERR_ARG, "yg_field_sqnorm_noalloc: null pointer");
  if (n_words < 1) return fail(YG_ERR_ARG, "yg_field_sqnorm_noalloc: n_words must be >= 1");
  if (n_words > kMaxWords)
    return fail(YG_ERR_ARG, "yg_field_sqnorm_noalloc: n_words exceeds the 16,777,216-word scratch limit");
  // The kernel reads the words as 16-byte double2 and writes one double: a view that starts
  // an odd number of doubles into a buffer is rejected here, before anything is launched.
  if (reinterpret_cast<std::uintptr_t>(dev_words) % 16 != 0)
    return fail(YG_ERR_ARG, "yg_field_sqnorm_noalloc: dev_words must be 16-byte aligned");
  if (reinterpret_cast<std::uintptr_t>(dev_out) % 8 != 0)
    return fail(YG_ERR_ARG, "yg_field_sqnorm_noalloc: dev_out must be 8-byte aligned");
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return fail(YG_ERR_CUDA, "yg_field_sqnorm_noalloc: no usable current device");
  double *scratch = g_scratch[dev].load(std::memory_order_acquire);
  if (!scratch) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, noalloc_partials) != cudaSuccess || !p)
      return fail(YG_ERR_CUDA, "yg_field_sqnorm_noalloc: cudaGetSymbolAddress failed");
    scratch = static_cast<double *>(p);
    g_scratch[dev].store(scratch, std::memory_order_release);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int blocks = (int)((n_words + kWordsPerBlock - 1) / kWordsPerBlock);
  k_partials<<<blocks, kThreads, 0, s>>>(scratch, reinterpret_cast<const double2 *>(dev_words), n_words);
  if (cudaGetLastError() != cudaSuccess) return fail(YG_ERR_CUDA, "yg_field_sqnorm_noalloc: launch failed");
  k_final<<<1, kThreads, 0, s>>>(dev_out, scratch, blocks);
  if (cudaGetLastError() != cudaSuccess) return fail(YG_ERR_CUDA, "yg_field_sqnorm_noalloc: launch failed");
  return YG_OK;
}
