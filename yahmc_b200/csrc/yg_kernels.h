// Kernel sets, instantiated once per representation dimension D (and per N where the
// fundamental links enter) in separate translation units (yg_inst_*.cu) so that the
// sm_100a builds of the large representations compile in parallel.  Host orchestration
// code includes only these declarations and dispatches on the run-time (N, D).
#pragma once

#include "yg_core.cuh"
#include "../../include/yahmc_gpu.h"

namespace yg {

// CLOVINV applies the LDL factors (FP64) or the explicit inverse (FP32); CLOVPK the packed
// Hermitian FP64 inverse
enum { EPI_PLAIN = 0, EPI_CLOVINV = 1, EPI_CLOVADD = 2, EPI_AXPY = 3, EPI_CLOVPK = 4 };

template <typename R>
struct HopArgs {
  Geom g;
  const cplx<R> *src;
  const cplx<R> *U;
  cplx<R> *dst;
  cplx<R> *dst2;          // CLOVINV: also store the raw hop here (the reference's in-place write)
  const cplx<R> *src2;    // CLOVADD / AXPY: psi at the output site
  const cplx<R> *cl;      // clover term (4 d x d per site)
  const double2 *ldl;     // LDL factors (FP64 path)
  const cplx<R> *cinv;    // explicit inverse clover blocks (FP32 path): 2 x (2d)^2 per site
  const double2 *cpk;     // packed Hermitian inverse clover blocks (FP64 path, d <= 6): 2 x 2d^2 words per site
  R coeff;                // -sign/2
  R diag;                 // 4+m (CLOVADD) or the AXPY coefficient
  R cfm1;                 // cf-1 (Dirac boundary term at t = Ta, Tb)
  int lo, n;              // output sites [lo, lo+n)
  int assign;
  int g5;
  int zero_add_at_boundary;
};

// The fields of several pseudo-fermion poles for one batched force launch
constexpr int kMaxPoles = 32;
struct PoleSet {
  const double2 *lhs[kMaxPoles];
  const double2 *rhs[kMaxPoles];
  double w[kMaxPoles];       // per-pole coefficient
  int n;
};

// Dirac-operator and force kernels of representation dimension D
template <int D>
struct DK {
  static void hop(const HopArgs<double> &a, int epi, cudaStream_t s);
  static void hop(const HopArgs<float> &a, int epi, cudaStream_t s);
  static void clover(double2 *dst, const double2 *src, const double2 *cl, Geom g, double mass4, double cfm1, int lo,
                     int n, int assign, cudaStream_t s);
  static void clover_inv(double2 *dst, const double2 *src, const double2 *ldl, Geom g, int assign, cudaStream_t s);
  static void ldl(double2 *ldl, const double2 *cl, Geom g, double sigma, double cf, int boundary_term, cudaStream_t s);
  static void cinv_float(float2 *cinv, const double2 *ldl, int Vh, cudaStream_t s);
  static void cinv_packed64(double2 *cpk, const double2 *ldl, int Vh, cudaStream_t s);
  static void logdet(double *out, const double2 *ldl, int Vh, cudaStream_t s);
  static void clover_fermion_force(double2 *clf, const double2 *lhs, const double2 *rhs, Geom g, double residue,
                                   cudaStream_t s);
  static void hopping_force(double *mom, const double2 *lhs, const double2 *rhs, const double2 *U, Geom g,
                            const double2 *itrepr, int ng, double coeff, cudaStream_t s);
  static void clover_ldl_force(double2 *clf, const double2 *ldl, Geom g, double coeff, cudaStream_t s);
  // sums over the poles of a PoleSet, one read-modify-write of cl_force / the momenta
  static void clover_fermion_force_multi(double2 *clf, const PoleSet &ps, Geom g, cudaStream_t s);
  static void hopping_force_multi(double *mom, const PoleSet &ps, const double2 *U, Geom g, const double2 *itrepr,
                                  int ng, cudaStream_t s);
  static void clover_force_core(double *mom, const double2 *clf, const double2 *U, Geom g, const double2 *itrepr,
                                int ng, double coeff, cudaStream_t s);
};

// Representation map and clover-term build: fundamental N x N links -> D x D
template <int NC, int D>
struct RK {
  static void represent(double2 *links, const double2 *fund, Geom g, const double2 *basis, int rep, cudaStream_t s);
  static void clover_term(double2 *cl, const double2 *fund, Geom g, const double2 *basis, int rep, double csw,
                          cudaStream_t s);
};


// run-time D -> DK<D>
#define YG_DISPATCH_D(DV, CALL)                                                              \
  do {                                                                                       \
    switch (DV) {                                                                            \
      case 1: { using K = ::yg::DK<1>; CALL; } break;                                        \
      case 2: { using K = ::yg::DK<2>; CALL; } break;                                        \
      case 3: { using K = ::yg::DK<3>; CALL; } break;                                        \
      case 4: { using K = ::yg::DK<4>; CALL; } break;                                        \
      case 6: { using K = ::yg::DK<6>; CALL; } break;                                        \
      case 8: { using K = ::yg::DK<8>; CALL; } break;                                        \
      case 10: { using K = ::yg::DK<10>; CALL; } break;                                      \
      case 15: { using K = ::yg::DK<15>; CALL; } break;                                      \
      default: throw ::yg::Error(YG_ERR_ARG, "unsupported representation dimension");        \
    }                                                                                        \
  } while (0)

// run-time (N, D) -> RK<N, D>
#define YG_DISPATCH_ND(NCV, DV, CALL)                                                        \
  do {                                                                                       \
    if (NCV == 2 && DV == 1) { using K = ::yg::RK<2, 1>; CALL; }                             \
    else if (NCV == 2 && DV == 2) { using K = ::yg::RK<2, 2>; CALL; }                        \
    else if (NCV == 2 && DV == 3) { using K = ::yg::RK<2, 3>; CALL; }                        \
    else if (NCV == 3 && DV == 3) { using K = ::yg::RK<3, 3>; CALL; }                        \
    else if (NCV == 3 && DV == 6) { using K = ::yg::RK<3, 6>; CALL; }                        \
    else if (NCV == 3 && DV == 8) { using K = ::yg::RK<3, 8>; CALL; }                        \
    else if (NCV == 4 && DV == 4) { using K = ::yg::RK<4, 4>; CALL; }                        \
    else if (NCV == 4 && DV == 6) { using K = ::yg::RK<4, 6>; CALL; }                        \
    else if (NCV == 4 && DV == 10) { using K = ::yg::RK<4, 10>; CALL; }                      \
    else if (NCV == 4 && DV == 15) { using K = ::yg::RK<4, 15>; CALL; }                      \
    else throw ::yg::Error(YG_ERR_ARG, "unsupported (N, representation) pair");              \
  } while (0)

static inline int nblk(long n, int t) { return (int)((n + t - 1) / t); }

}  // namespace yg
