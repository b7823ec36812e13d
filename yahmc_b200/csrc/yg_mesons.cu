// Propagator sources, the even-odd propagator solve and the meson contractions on the
// device: observables/propagator.cpp:22-166 and observables/mesons.cpp:55-128.
//
// The contraction reads each propagator component of a site once: for every source index x
// and colour y it loads the 4 x 4 spin block q[c][b] = P[c*NS + x](spin b, colour y) into
// registers and adds, for all sixteen channels at once,
//     Re sum_{a,c} v1[a] v2[c] q[c][col1[a]] conj(q[col2[c]][a]),
// with the g5*Gamma tables (mesons.cpp:12-27) folded in at compile time.  A block covers 128
// sites of one time slice; the slice sums are formed in a fixed order (warp shuffles, then
// the block, then the blocks of the slice), so the result does not depend on scheduling.
#include <cmath>
#include <vector>
#include "yg_kernels.h"
#include "yg_lattice.h"

namespace yg {

namespace {

// g5*Gamma as signed spin permutations: row a has its one entry in column gcol(g, a).
// g = 0 ID, 1 G1, 2 G2, 3 G3, 4 G5, 5 G5G1, 6 G5G2, 7 G5G3, 8 G0G1, 9 G0G2, 10 G0G3,
// 11 G0G5, 12 G0G5G1, 13 G0G5G2, 14 G0G5G3 (mesons.cpp:12-27).
__host__ __device__ constexpr int gcol(int g, int a) {
  return (g == 0 || g == 4 || g == 10 || g == 14) ? a
         : (g == 1 || g == 2 || g == 5 || g == 6) ? 3 - a
         : (g == 3 || g == 7 || g == 11) ? (a ^ 2)
                                         : (a ^ 1);
}

// the entry's value as a code: 0 = +1, 1 = -1, 2 = +i, 3 = -i
__host__ __device__ constexpr int gcode(int g, int a) {
  constexpr signed char k[15][4] = {
      {0, 0, 1, 1},  // ID
      {3, 3, 3, 3},  // G1
      {1, 0, 1, 0},  // G2
      {3, 2, 3, 2},  // G3
      {0, 0, 0, 0},  // G5
      {3, 3, 2, 2},  // G5G1
      {1, 0, 0, 1},  // G5G2
      {3, 2, 2, 3},  // G5G3
      {3, 3, 3, 3},  // G0G1
      {1, 0, 1, 0},  // G0G2
      {3, 2, 3, 2},  // G0G3
      {0, 0, 0, 0},  // G0G5
      {2, 2, 3, 3},  // G0G5G1
      {0, 1, 1, 0},  // G0G5G2
      {2, 3, 3, 2},  // G0G5G3
  };
  return k[g][a];
}
__host__ __device__ constexpr int code_re(int c) { return c == 0 ? 1 : c == 1 ? -1 : 0; }
__host__ __device__ constexpr int code_im(int c) { return c == 2 ? 1 : c == 3 ? -1 : 0; }

// the gamma pair of channel ch (MESON order id, g1, ..., g0g5g3, g5_g0g5)
__host__ __device__ constexpr int chan_g1(int ch) { return ch < 15 ? ch : 11; }
__host__ __device__ constexpr int chan_g2(int ch) { return ch < 15 ? ch : 4; }

constexpr int kChannels = 16, kMesonThreads = 128, kMaxProps = 60;

struct MesonArgs {
  const double2 *P[kMaxProps];
  Geom g;
  int vol3, bps;      // sites per slice, blocks per slice
  double *partial;    // [T * bps][16]
};

template <int D, int NS>
__global__ void __launch_bounds__(kMesonThreads) k_meson(MesonArgs a) {
  const int t = blockIdx.x / a.bps, j = blockIdx.x % a.bps;
  const int s = j * kMesonThreads + threadIdx.x;
  double acc[kChannels];
#pragma unroll
  for (int ch = 0; ch < kChannels; ch++) acc[ch] = 0.0;
  if (s < a.vol3) {
    const int Z = a.g.dim[3], Y = a.g.dim[2];
    const int z = s % Z, y = (s / Z) % Y, x = s / (Z * Y);
    const int id = id_of(a.g, t, x, y, z);
#pragma unroll 1
    for (int xs = 0; xs < NS; xs++) {
#pragma unroll 1
      for (int col = 0; col < D; col++) {
        double2 q[4][4];
#pragma unroll
        for (int c = 0; c < 4; c++)
#pragma unroll
          for (int b = 0; b < 4; b++) q[c][b] = a.P[c * NS + xs][fidx(a.g, id, b * D + col, 4 * D)];
#pragma unroll
        for (int ch = 0; ch < kChannels; ch++)
#pragma unroll
          for (int ar = 0; ar < 4; ar++)
#pragma unroll
            for (int cr = 0; cr < 4; cr++) {
              const int c1 = gcode(chan_g1(ch), ar), c2 = gcode(chan_g2(ch), cr);
              const int wr = code_re(c1) * code_re(c2) - code_im(c1) * code_im(c2);
              const int wi = code_re(c1) * code_im(c2) + code_im(c1) * code_re(c2);
              const double2 u = q[cr][gcol(chan_g1(ch), ar)], v = q[gcol(chan_g2(ch), cr)][ar];
              // m = u * conj(v)
              const double mr = u.x * v.x + u.y * v.y, mi = u.y * v.x - u.x * v.y;
              if (wr) acc[ch] += wr * mr;
              if (wi) acc[ch] -= wi * mi;
            }
      }
    }
  }
  __shared__ double sh[kMesonThreads / 32][kChannels];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int ch = 0; ch < kChannels; ch++) {
    double v = acc[ch];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sh[warp][ch] = v;
  }
  __syncthreads();
  if (threadIdx.x < kChannels) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kMesonThreads / 32; w++) v += sh[w][threadIdx.x];
    a.partial[(long)blockIdx.x * kChannels + threadIdx.x] = v;
  }
}

// out[ch * T + (t - tau) mod T] = sum over the slice's blocks, in block order
__global__ void k_meson_slices(const double *partial, double *out, int T, int bps, int tau) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kChannels * T) return;
  const int ch = i % kChannels, t = i / kChannels;
  double v = 0.0;
  for (int j = 0; j < bps; j++) v += partial[((long)t * bps + j) * kChannels + ch];
  out[ch * T + (t - tau + T) % T] = v;
}

__global__ void k_set_component(double2 *f, long idx, double re) { f[idx] = make_double2(re, 0.0); }

// spin 0 of the slice sites from the z2 noise; k = rank of the site among the slice's sites
// by increasing site id (even sites first with even-odd order: rank p * vol3/2 + s/2)
__global__ void k_semwall_fill(double2 *f, const double *z2, Geom g, int tau, int vol3, int d) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= vol3) return;
  const int Z = g.dim[3], Y = g.dim[2];
  const int z = s % Z, y = (s / Z) % Y, x = s / (Z * Y);
  const int id = id_of(g, tau, x, y, z);
  const int k = g.eo ? ((tau + x + y + z) & 1) * (vol3 / 2) + s / 2 : s;
  for (int i = 0; i < d; i++) f[fidx(g, id, 0 * d + i, 4 * d)] = make_double2(z2[(long)k * 2 * d + 2 * i], z2[(long)k * 2 * d + 2 * i + 1]);
}

// spin n-1 -> spin n on every site (create_semwall_source, n > 0)
__global__ void k_semwall_shift(double2 *f, Geom g, int n, int d) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= (long)g.V * d) return;
  const int id = (int)(i / d), c = (int)(i % d);
  const long from = fidx(g, id, (n - 1) * d + c, 4 * d), to = fidx(g, id, n * d + c, 4 * d);
  f[to] = f[from];
  f[from] = make_double2(0.0, 0.0);
}

int vol3_of(const Lattice &L) { return L.p.dims[1] * L.p.dims[2] * L.p.dims[3]; }

void check_tau(const Lattice &L, int tau) {
  if (tau < 0 || tau >= L.p.dims[0]) throw Error(YG_ERR_ARG, "time slice out of range");
}

// the odd half of a field is the second half of its buffer: F[(blk*4d + k)*Vh + h]
double *odd_half(const Lattice &L, double *f) { return f + 8L * L.d * L.Vh; }
const double *odd_half(const Lattice &L, const double *f) { return f + 8L * L.d * L.Vh; }

constexpr int kPropTmp = 120, kPropEo = 121, kPropPool = 124;

}  // namespace

// create_point_source, propagator.cpp:58-73
void create_point_source(Lattice &L, int n, int tau, double *src) {
  check_tau(L, tau);
  if (n < 0 || n >= 4 * L.d) throw Error(YG_ERR_ARG, "point source index out of range");
  YG_CUDA(cudaMemsetAsync(src, 0, L.field_bytes(), L.stream));
  const int id = id_of(L.g, tau, 0, 0, 0);
  k_set_component<<<1, 1, 0, L.stream>>>((double2 *)src, fidx(L.g, id, (n / L.d) * L.d + n % L.d, 4 * L.d), 1.0);
  YG_LAUNCHED();
}

// create_semwall_source, propagator.cpp:22-56
void create_semwall_source(Lattice &L, int n, int tau, const double *z2, double *src) {
  check_tau(L, tau);
  if (n < 0 || n > 3) throw Error(YG_ERR_ARG, "semwall source index out of range");
  if (n == 0) {
    if (!z2) throw Error(YG_ERR_ARG, "z2 noise required for n = 0");
    const int vol3 = vol3_of(L);
    double *noise = L.scratch_field(kPropTmp);
    YG_CUDA(cudaMemcpyAsync(noise, z2, sizeof(double) * 2 * L.d * vol3, cudaMemcpyHostToDevice, L.stream));
    YG_CUDA(cudaMemsetAsync(src, 0, L.field_bytes(), L.stream));
    k_semwall_fill<<<nblk(vol3, 128), 128, 0, L.stream>>>((double2 *)src, noise, L.g, tau, vol3, L.d);
    YG_LAUNCHED();
    YG_CUDA(cudaStreamSynchronize(L.stream));   // the noise buffer is scratch
  } else {
    k_semwall_shift<<<nblk(L.V * L.d, 256), 256, 0, L.stream>>>((double2 *)src, L.g, n, L.d);
    YG_LAUNCHED();
  }
}

namespace {

template <int D>
void launch_meson(const MesonArgs &a, bool point, int grid, cudaStream_t s) {
  if (point)
    k_meson<D, D><<<grid, kMesonThreads, 0, s>>>(a);
  else
    k_meson<D, 1><<<grid, kMesonThreads, 0, s>>>(a);
}

// the even-site system of calc_propagator into eo (clover: b_e - D_eo D_oo^-1 b_o; Wilson:
// (4+m) b_e - D_eo b_o), as propagator.cpp:90-95 and 126-129
void eo_source(Lattice &L, double mass, double *eo, double *src, double *tmp) {
  const size_t half = sizeof(double) * 8L * L.d * L.Vh;
  if (L.p.clover) {
    clover_inv_apply(L, mass, tmp, src, 2, false);
    hop(L, tmp, tmp, 1, 1.0, false);
    YG_CUDA(cudaMemcpyAsync(eo, src, half, cudaMemcpyDeviceToDevice, L.stream));
    blas_axpby(L, eo, make_double2(1, 0), make_double2(-1, 0), tmp, 0, L.Vh);
  } else {
    hop(L, tmp, src, 1, 1.0, false);
    YG_CUDA(cudaMemcpyAsync(eo, src, half, cudaMemcpyDeviceToDevice, L.stream));
    blas_axpby(L, eo, make_double2(4.0 + mass, 0), make_double2(0, 0), nullptr, 0, L.Vh);
    blas_axpby(L, eo, make_double2(1, 0), make_double2(-1, 0), tmp, 0, L.Vh);
  }
}

// x_o from x_e, propagator.cpp:100-113 and 134-145
void odd_sites(Lattice &L, double mass, double *dst, const double *src, double *tmp) {
  const size_t half = sizeof(double) * 8L * L.d * L.Vh;
  hop(L, tmp, dst, 2, 1.0, false);
  YG_CUDA(cudaMemcpyAsync(odd_half(L, dst), odd_half(L, src), half, cudaMemcpyDeviceToDevice, L.stream));
  if (L.p.clover) {
    blas_axpby(L, dst, make_double2(1, 0), make_double2(-1, 0), tmp, L.Vh, L.Vh);
    clover_inv_apply(L, mass, dst, dst, 2, false);
  } else {
    const double r = 1.0 / (4.0 + mass);
    blas_axpby(L, dst, make_double2(r, 0), make_double2(0, 0), nullptr, L.Vh, L.Vh);
    blas_axpby(L, dst, make_double2(1, 0), make_double2(-r, 0), tmp, L.Vh, L.Vh);
  }
}

}  // namespace

// contract_all_correlators, mesons.cpp:105-128, for one source time slice: corr[ch*T + t]
// += the slice sums of the sixteen channels (raw, before print_correlator's sign and norm)
void meson_contract(Lattice &L, int method, int tau, const double *const *props, int nprops, double *corr) {
  check_tau(L, tau);
  if (method != YG_MESON_SEMWALL && method != YG_MESON_POINT) throw Error(YG_ERR_ARG, "unknown meson method");
  const bool point = method == YG_MESON_POINT;
  const int need = point ? 4 * L.d : 4;
  if (nprops != need) throw Error(YG_ERR_ARG, point ? "POINT needs 4*d propagators" : "SEMWALL needs 4 propagators");
  MesonArgs a{};
  for (int i = 0; i < nprops; i++) {
    if (!props[i]) throw Error(YG_ERR_ARG, "null propagator");
    a.P[i] = (const double2 *)props[i];
  }
  const int T = L.p.dims[0];
  a.g = L.g;
  a.vol3 = vol3_of(L);
  a.bps = nblk(a.vol3, kMesonThreads);
  double *buf = L.scratch_field(kPropEo);
  a.partial = buf;
  double *out = buf + (long)T * a.bps * kChannels;
  const int grid = T * a.bps;
  switch (L.d) {
    case 1: launch_meson<1>(a, point, grid, L.stream); break;
    case 2: launch_meson<2>(a, point, grid, L.stream); break;
    case 3: launch_meson<3>(a, point, grid, L.stream); break;
    case 4: launch_meson<4>(a, point, grid, L.stream); break;
    case 6: launch_meson<6>(a, point, grid, L.stream); break;
    case 8: launch_meson<8>(a, point, grid, L.stream); break;
    case 10: launch_meson<10>(a, point, grid, L.stream); break;
    case 15: launch_meson<15>(a, point, grid, L.stream); break;
    default: throw Error(YG_ERR_ARG, "unsupported representation dimension");
  }
  YG_LAUNCHED();
  k_meson_slices<<<nblk(kChannels * T, 128), 128, 0, L.stream>>>(buf, out, T, a.bps, tau);
  YG_LAUNCHED();
  std::vector<double> h((size_t)kChannels * T);
  YG_CUDA(cudaMemcpyAsync(h.data(), out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, L.stream));
  YG_CUDA(cudaStreamSynchronize(L.stream));
  for (size_t i = 0; i < h.size(); i++) corr[i] += h[i];
}

// calc_propagator, propagator.cpp:75-166: auto_inverter on the even-site system, then the
// odd sites; without even-odd preconditioning a direct solve.  dst holds the initial guess.
int calc_propagator(Lattice &L, double mass, double prec, double *dst, double *src, int *iters) {
  yg_inv_par par{};
  par.op = YG_OP_DPHI;
  par.mass = mass;
  par.prec = prec;
  if (!L.p.eo) return auto_inverter(L, par, dst, src, iters);
  double *tmp = L.scratch_field(kPropTmp), *eo = L.scratch_field(kPropEo);
  eo_source(L, mass, eo, src, tmp);
  const int st = auto_inverter(L, par, dst, eo, iters);
  odd_sites(L, mass, dst, src, tmp);
  return st;
}

// No reference counterpart: the n propagators of one source time slice solved together, with
// every operator application shared.  solver 0: BiCGstab on the even-site system D x_e = b'
// (the reference's recurrence per system, dst as the initial guess); 1, 2: CG on Hphi_sq y = g5 b'
// with x_e = Hphi y (Hphi = g5 D is Hermitian), mixed precision (1) or FP64 (2), from zero.  All
// stop on |r|^2 / |b'|^2 < prec; the odd sites follow as in calc_propagator.
int calc_propagator_multi(Lattice &L, double mass, double prec, int n, double *const *dst, double *const *src,
                          int solver, int *iters) {
  if (!L.p.eo) throw Error(YG_ERR_ARG, "the batched propagator needs even-odd preconditioning");
  if (n < 1 || n > 16) throw Error(YG_ERR_ARG, "1..16 propagators");
  if (solver < 0 || solver > 2) throw Error(YG_ERR_ARG, "solver: 0 BiCGstab, 1 mixed CG, 2 FP64 CG");
  double *tmp = L.scratch_field(kPropTmp);
  std::vector<double *> rhs(n), y(n);
  for (int i = 0; i < n; i++) {
    if (!dst[i] || !src[i]) throw Error(YG_ERR_ARG, "null field");
    rhs[i] = L.scratch_field(kPropPool + i);
    eo_source(L, mass, rhs[i], src[i], tmp);
  }
  yg_inv_par par{};
  par.mass = mass;
  par.prec = prec;
  int st;
  if (solver == 0) {
    par.op = YG_OP_DPHI;
    st = bicgstab_multi(L, par, n, dst, rhs.data(), iters);
  } else {
    for (int i = 0; i < n; i++) {
      y[i] = L.scratch_field(kPropPool + 16 + i);
      blas_g5(L, rhs[i], 0, L.Vh);
      blas_zero(L, y[i], 0, L.V);
    }
    par.op = YG_OP_HPHI_SQ;
    if (solver == 1) {
      std::vector<yg_solve_stats> ss(n);
      st = cg_mixed_mrhs(L, par, n, y.data(), rhs.data(), 0.1, ss.data());
      if (iters)
        for (int i = 0; i < n; i++) iters[i] = ss[i].iterations;
    } else {
      st = cg_multi(L, par, n, y.data(), rhs.data(), iters);
    }
    for (int i = 0; i < n; i++) hphi(L, mass, dst[i], y[i]);
  }
  for (int i = 0; i < n; i++) odd_sites(L, mass, dst[i], src[i], tmp);
  return st;
}

}  // namespace yg
