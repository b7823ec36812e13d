// Core device types and layout of the B200 fermion engine.
//
// Device layout (structure of arrays, one complex number per 8/16-byte word):
//   The reference's site index id (geometry.cpp:756-878; even-odd order
//   id = (parity*V + lex)/2, or id = lex without even-odd preconditioning) is
//   split into two half-volume blocks: blk = id / Vh, h = id % Vh.
//   spinor field  F[(blk*4d + k)*Vh + h],  k = spin*d + colour
//   links         U[((blk*4 + mu)*d*d + i*d + j)*Vh + h]      (U(x,mu) stored at x)
//   clover term   C[((blk*4 + m)*d*d + i*d + j)*Vh + h]       (the 4 blocks A0..A3, clover.h:12-13)
//   LDL factors   L[(b*P + k)*Vh + h], b = upper/lower spin block, P = d(2d+1), for blk 1
// Consecutive threads take consecutive h, so every component load of the
// own site is one fully coalesced 128-byte line per 8 (FP64) threads.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

// Unrolling of loops over colour indices.  YG_UNROLL_D (operator kernels) unrolls fully
// for every representation: a build that kept the d >= 8 loops of the fused hop
// epilogues rolled gave wrong results while the same device functions were exact in
// stand-alone kernels, so those stay fully unrolled.  YG_UNROLL_DF (force kernels) keeps
// d >= 8 loops rolled to bound the build time; the parity tests cover every d.
#define YG_STR_(x) #x
#define YG_STR(x) YG_STR_(x)
#define YG_UNROLL_D _Pragma(YG_STR(unroll 64))
#define YG_UNROLL_DF _Pragma(YG_STR(unroll (D <= 6 ? 64 : 1)))

namespace yg {

// ------------------------------------------------------------------ complex
template <typename R> struct C2;
template <> struct C2<double> { using t = double2; };
template <> struct C2<float> { using t = float2; };
template <typename R> using cplx = typename C2<R>::t;

template <typename R> __host__ __device__ __forceinline__ cplx<R> mk(R a, R b) { cplx<R> c; c.x = a; c.y = b; return c; }
template <typename T> __host__ __device__ __forceinline__ T cadd(T a, T b) { a.x += b.x; a.y += b.y; return a; }
template <typename T> __host__ __device__ __forceinline__ T csub(T a, T b) { a.x -= b.x; a.y -= b.y; return a; }
template <typename T> __host__ __device__ __forceinline__ T cmul(T a, T b) { T c; c.x = a.x * b.x - a.y * b.y; c.y = a.x * b.y + a.y * b.x; return c; }
// conj(a) * b
template <typename T> __host__ __device__ __forceinline__ T cmulc(T a, T b) { T c; c.x = a.x * b.x + a.y * b.y; c.y = a.x * b.y - a.y * b.x; return c; }
template <typename T, typename R> __host__ __device__ __forceinline__ T cscale(T a, R s) { a.x *= s; a.y *= s; return a; }
template <typename T> __host__ __device__ __forceinline__ T ctimesi(T a) { T c; c.x = -a.y; c.y = a.x; return c; }      // i*a
template <typename T> __host__ __device__ __forceinline__ T ctimesmi(T a) { T c; c.x = a.y; c.y = -a.x; return c; }     // -i*a
template <typename T> __host__ __device__ __forceinline__ T cconj(T a) { a.y = -a.y; return a; }
// acc += a*b
template <typename T> __host__ __device__ __forceinline__ void cfma(T &acc, T a, T b) {
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(a.y, b.x, acc.y);
}
// acc += conj(a)*b
template <typename T> __host__ __device__ __forceinline__ void cfmac(T &acc, T a, T b) {
  acc.x = fma(a.x, b.x, acc.x); acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y); acc.y = fma(-a.y, b.x, acc.y);
}

// ------------------------------------------------------------------ geometry
struct Geom {
  int dim[4];     // T, X, Y, Z
  int V, Vh;
  int eo;         // 1: even-odd site order (UPDATE_EO), 0: lexicographic
  int bc;         // 0 periodic, 1 antiperiodic, 2 open, 3 sf
  int zt[3];      // time slices whose spinors the boundary conditions zero (-1 = unused)
  int Ta, Tb;     // time slices of the Dirac boundary term (open / sf), -1 otherwise
};

__host__ __device__ __forceinline__ int lex_of(const Geom &g, int t, int x, int y, int z) {
  return ((t * g.dim[1] + x) * g.dim[2] + y) * g.dim[3] + z;
}

__host__ __device__ __forceinline__ int id_of(const Geom &g, int t, int x, int y, int z) {
  int lex = lex_of(g, t, x, y, z);
  if (!g.eo) return lex;
  int p = (t + x + y + z) & 1;
  return (p * g.V + lex) >> 1;
}

// coordinates (t,x,y,z) of site id
__host__ __device__ __forceinline__ void coords_of(const Geom &g, int id, int c[4]) {
  int lex;
  if (g.eo) {
    int p = id >= g.Vh;
    lex = 2 * (id - p * g.Vh);
    int z = lex % g.dim[3];
    int r = lex / g.dim[3];
    int y = r % g.dim[2];
    r /= g.dim[2];
    int x = r % g.dim[1];
    int t = r / g.dim[1];
    if (((t + x + y + z) & 1) != p) z += 1;   // dims are even: lex 2h and 2h+1 differ in z only
    c[0] = t; c[1] = x; c[2] = y; c[3] = z;
    return;
  }
  lex = id;
  c[3] = lex % g.dim[3];
  int r = lex / g.dim[3];
  c[2] = r % g.dim[2];
  r /= g.dim[2];
  c[1] = r % g.dim[1];
  c[0] = r / g.dim[1];
}

__host__ __device__ __forceinline__ int neighbour(const Geom &g, const int c[4], int mu, int dir) {
  int n[4] = {c[0], c[1], c[2], c[3]};
  int L = g.dim[mu];
  n[mu] = dir > 0 ? (n[mu] + 1 == L ? 0 : n[mu] + 1) : (n[mu] == 0 ? L - 1 : n[mu] - 1);
  return id_of(g, n[0], n[1], n[2], n[3]);
}

__host__ __device__ __forceinline__ bool spinor_zeroed(const Geom &g, int t) {
  return t == g.zt[0] || t == g.zt[1] || t == g.zt[2];
}

// ------------------------------------------------------------------ field views
// Index of component k of site id in a field with `ncomp` complex components per site.
__host__ __device__ __forceinline__ long fidx(const Geom &g, int id, int k, int ncomp) {
  int blk = id >= g.Vh;
  int h = id - blk * g.Vh;
  return ((long)blk * ncomp + k) * g.Vh + h;
}

}  // namespace yg
