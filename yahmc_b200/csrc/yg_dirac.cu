// Host orchestration of the Wilson-clover Dirac operator (dirac.cpp:706-781): the hop
// with its fused epilogues (device code in yg_dirac_impl.cuh), the standalone clover /
// clover-inverse kernels, the even-odd Schur operator Dphi / Hphi / Hphi_sq with the
// reference's side effects on its source field, and the FP32 mirror used by the
// mixed-precision solver.
#include "yg_lattice.h"
#include "yg_kernels.h"

namespace yg {

// apply_bcs_on_spinor_field (bcs.cpp:139-164): zero every site of the listed time slices
__global__ void k_bc_zero(double2 *f, Geom g, int ncomp) {
  int vol3 = g.dim[1] * g.dim[2] * g.dim[3];
  int t_ = blockIdx.x * blockDim.x + threadIdx.x;
  if (t_ >= 3 * vol3) return;
  int slice = g.zt[t_ / vol3];
  if (slice < 0) return;
  int r = t_ % vol3;
  int z = r % g.dim[3]; r /= g.dim[3];
  int y = r % g.dim[2];
  int x = r / g.dim[2];
  int id = id_of(g, slice, x, y, z);
  for (int k = 0; k < ncomp; k++) f[fidx(g, id, k, ncomp)] = make_double2(0, 0);
}

static void part_range(const Lattice &L, int part, int &lo, int &n) {
  if (part == 1) { lo = 0; n = (int)L.Vh; }
  else if (part == 2) { lo = (int)L.Vh; n = (int)L.Vh; }
  else { lo = 0; n = (int)L.V; }
}

static bool has_spinor_bcs(const Lattice &L) { return L.p.bc == YG_BC_OPEN || L.p.bc == YG_BC_SF; }

void bc_zero_field(Lattice &L, double *f) {
  if (!has_spinor_bcs(L)) return;
  int vol3 = L.g.dim[1] * L.g.dim[2] * L.g.dim[3];
  k_bc_zero<<<nblk(3L * vol3, 128), 128, 0, L.stream>>>((double2 *)f, L.g, 4 * L.d);
  YG_LAUNCHED();
}

template <typename R>
static HopArgs<R> base_args(const Lattice &L) {
  HopArgs<R> a{};
  a.g = L.g;
  a.cfm1 = (R)(L.p.cf - 1.0);
  return a;
}

template <int EPI, typename R>
static void launch_hop(Lattice &L, const HopArgs<R> &a) {
  YG_DISPATCH_D(L.d, K::hop(a, EPI, L.stream));
  YG_LAUNCHED();
}

void hop(Lattice &L, double *dst, const double *src, int part, double sign, bool assign) {
  L.mvm++;
  auto a = base_args<double>(L);
  part_range(L, part, a.lo, a.n);
  a.src = (const double2 *)src;
  a.U = L.links.as<double2>();
  a.dst = (double2 *)dst;
  a.coeff = -0.5 * sign;
  a.assign = assign;
  launch_hop<EPI_PLAIN>(L, a);
  bc_zero_field(L, dst);
}

void clover_apply(Lattice &L, double mass, double *dst, const double *src, int part, bool assign) {
  if (!L.p.clover) throw Error(YG_ERR_ARG, "clover term disabled");
  int lo, n;
  part_range(L, part, lo, n);
  YG_DISPATCH_D(L.d, K::clover((double2 *)dst, (const double2 *)src, L.clover.as<double2>(), L.g, 4.0 + mass,
                                L.p.cf - 1.0, lo, n, assign, L.stream));
  YG_LAUNCHED();
}

void clover_inv_apply(Lattice &L, double mass, double *dst, const double *src, int part, bool assign) {
  if (!L.p.clover) throw Error(YG_ERR_ARG, "clover term disabled");
  if (part != 2) throw Error(YG_ERR_ARG, "the clover inverse is stored for the odd block only");
  ensure_ldl(L, 4.0 + mass);
  YG_DISPATCH_D(L.d, K::clover_inv((double2 *)dst, (const double2 *)src, L.ldl.as<double2>(), L.g, assign, L.stream));
  YG_LAUNCHED();
}

void schur_step1(Lattice &L, double mass, double *tmp, const double *src, double *clob) {
  ensure_ldl(L, 4.0 + mass);
  L.mvm++;
  auto a = base_args<double>(L);
  a.lo = (int)L.Vh;
  a.n = (int)L.Vh;
  a.src = (const double2 *)src;
  a.U = L.links.as<double2>();
  a.dst = (double2 *)tmp;
  a.dst2 = (double2 *)clob;
  a.coeff = 0.5;                      // dirac_kernel(sptr, sptr, ODD, -1): -(-1)/2
  if (L.d <= kPackedInverseMaxD) {
    a.cpk = L.cpk64.as<double2>();
    launch_hop<EPI_CLOVPK>(L, a);
  } else {
    a.ldl = L.ldl.as<double2>();
    launch_hop<EPI_CLOVINV>(L, a);
  }
}

void schur_step2(Lattice &L, double mass, double *dst, const double *tmp, const double *src, bool g5) {
  L.mvm++;
  auto a = base_args<double>(L);
  a.lo = 0;
  a.n = (int)L.Vh;
  a.src = (const double2 *)tmp;
  a.U = L.links.as<double2>();
  a.dst = (double2 *)dst;
  a.src2 = (const double2 *)src;
  a.coeff = -0.5;
  a.g5 = g5;
  a.zero_add_at_boundary = 1;
  if (L.p.clover) {
    a.cl = L.clover.as<double2>();
    a.diag = 4.0 + mass;
    launch_hop<EPI_CLOVADD>(L, a);
  } else {
    a.diag = (4.0 + mass) * (4.0 + mass);
    launch_hop<EPI_AXPY>(L, a);
  }
}

// Dphi with the reference's side effects (dirac.cpp:738-765)
static void dphi_impl(Lattice &L, double mass, double *dst, double *src, bool g5) {
  if (L.p.eo) {
    if (L.p.clover) {
      double *tmp = L.scratch_field(1);
      schur_step1(L, mass, tmp, src, src);        // src_o = 1/2 H src_e (in place, as the reference)
      schur_step2(L, mass, dst, tmp, src, g5);
    } else {
      auto a = base_args<double>(L);
      L.mvm++;
      a.lo = (int)L.Vh; a.n = (int)L.Vh;
      a.src = (const double2 *)src; a.U = L.links.as<double2>(); a.dst = (double2 *)src; a.coeff = 0.5;
      // in-place is safe: the odd output block is disjoint from the even input block
      launch_hop<EPI_PLAIN>(L, a);
      schur_step2(L, mass, dst, src, src, g5);
    }
    bc_zero_field(L, src);
    bc_zero_field(L, dst);
    return;
  }
  // without even-odd preconditioning: hop on all sites, then + clover (or + (4+m)) psi.
  // The reference zeroes dst's boundary slices right after the hop and adds the diagonal
  // term afterwards, so boundary sites end up as (diagonal term) psi: the kernel zeroes only
  // the hop part there (zero_add_at_boundary = 0).
  L.mvm++;
  auto a = base_args<double>(L);
  a.lo = 0; a.n = (int)L.V;
  a.src = (const double2 *)src; a.U = L.links.as<double2>(); a.dst = (double2 *)dst; a.src2 = (const double2 *)src;
  a.coeff = -0.5; a.g5 = g5; a.zero_add_at_boundary = 0;
  if (L.p.clover) {
    a.cl = L.clover.as<double2>();
    a.diag = 4.0 + mass;
    launch_hop<EPI_CLOVADD>(L, a);
  } else {
    a.diag = 4.0 + mass;
    launch_hop<EPI_AXPY>(L, a);
  }
}

void dphi(Lattice &L, double mass, double *dst, double *src) { dphi_impl(L, mass, dst, src, false); }
void hphi(Lattice &L, double mass, double *dst, double *src) { dphi_impl(L, mass, dst, src, true); }

void hphi_sq(Lattice &L, double mass, double *dst, double *src) {
  double *tmp = L.scratch_field(2);
  hphi(L, mass, tmp, src);
  hphi(L, mass, dst, tmp);
}

void apply_op(Lattice &L, int op, double mass, double *dst, double *src) {
  switch (op) {
    case YG_OP_DPHI: dphi(L, mass, dst, src); return;
    case YG_OP_HPHI: hphi(L, mass, dst, src); return;
    case YG_OP_HPHI_SQ: hphi_sq(L, mass, dst, src); return;
  }
  throw Error(YG_ERR_ARG, "invalid operator id");
}

// ------------------------------------------------------------------ FP32 inner operator
// Single-precision mirrors: links and clover term converted from the FP64 copies, odd-site
// clover inverse formed explicitly from the FP64 LDL factors.
__global__ void k_to_float(float2 *dst, const double2 *src, long n) {
  long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}

static void ensure_float_operator(Lattice &L, double mass) {
  long nl = 4L * L.V * L.d * L.d;
  if (!L.links_f_valid) {
    L.links_f.alloc(sizeof(float2) * nl);
    k_to_float<<<nblk(nl, 256), 256, 0, L.stream>>>(L.links_f.as<float2>(), L.links.as<double2>(), nl);
    YG_LAUNCHED();
    if (L.p.clover) {
      L.clover_f.alloc(sizeof(float2) * nl);
      k_to_float<<<nblk(nl, 256), 256, 0, L.stream>>>(L.clover_f.as<float2>(), L.clover.as<double2>(), nl);
      YG_LAUNCHED();
    }
    L.links_f_valid = true;
  }
  if (L.p.clover && !(L.cinv_f_valid && L.cinv_f_sigma == 4.0 + mass)) {
    ensure_ldl(L, 4.0 + mass);
    long n = 2L * (2 * L.d) * (2 * L.d) * L.Vh;
    L.cinv_f.alloc(sizeof(float2) * n);
    YG_DISPATCH_D(L.d, K::cinv_float(L.cinv_f.as<float2>(), L.ldl.as<double2>(), (int)L.Vh, L.stream));
    YG_LAUNCHED();
    L.cinv_f_sigma = 4.0 + mass;
    L.cinv_f_valid = true;
  }
}

// Hphi (gamma5 times the even-odd Schur operator) in FP32 on FP32 fields; writes only the
// odd block of tmp and the even block of dst.  Used by the inner iterations of yg_cg_mixed.
void hphi_float(Lattice &L, double mass, float2 *dst, float2 *src, float2 *tmp) {
  if (!L.p.eo) throw Error(YG_ERR_ARG, "the mixed-precision solver needs even-odd preconditioning");
  ensure_float_operator(L, mass);
  auto a = base_args<float>(L);
  a.U = L.links_f.as<float2>();
  a.lo = (int)L.Vh; a.n = (int)L.Vh; a.src = src; a.dst = tmp; a.coeff = 0.5f;
  auto b = base_args<float>(L);
  b.U = L.links_f.as<float2>();
  b.lo = 0; b.n = (int)L.Vh; b.src = tmp; b.dst = dst; b.src2 = src; b.coeff = -0.5f; b.g5 = 1;
  b.zero_add_at_boundary = 1;
  if (L.p.clover) {
    a.cinv = L.cinv_f.as<float2>();
    launch_hop<EPI_CLOVINV>(L, a);
    b.cl = L.clover_f.as<float2>();
    b.diag = (float)(4.0 + mass);
    launch_hop<EPI_CLOVADD>(L, b);
  } else {
    launch_hop<EPI_PLAIN>(L, a);
    b.diag = (float)((4.0 + mass) * (4.0 + mass));
    launch_hop<EPI_AXPY>(L, b);
  }
  L.mvm += 2;
}

}  // namespace yg
