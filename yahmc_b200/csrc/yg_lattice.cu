// Lattice state on the device: geometry, representation tables, link upload and
// representation, clover term, LDL factors, and the host<->device field layout
// conversion.
//
// Reference counterparts: geometry_init (geometry.cpp:1032-1191), repr_init and
// represent_links (repr.cpp:17-263), represent_gauge_field (repr.cpp:265-280),
// bcs_init / apply_bcs_on_represented_gauge_field (bcs.cpp:11-137, 264-272),
// compute_clover_term (clover.cpp:93-168, 330-347), clover_repr
// (wilsonloop.cpp:5-31), compute_ldl_decomp + ldl (clover.cpp:25-91, 307-328,
// solver.cpp:97-142).  The device kernels live in yg_repr_impl.cuh / yg_dirac_impl.cuh.
#include <complex>
#include <cstring>
#include <cmath>
#include "yg_lattice.h"
#include "yg_kernels.h"

namespace yg {

std::atomic<long> g_launch_count{0};

void check_cuda(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    int code = (e == cudaErrorMemoryAllocation) ? YG_ERR_OOM : YG_ERR_CUDA;
    throw Error(code, std::string(what) + ": " + cudaGetErrorString(e));
  }
}

void DevBuf::alloc(size_t n) {
  if (p && bytes >= n) return;
  release();
  if (n == 0) return;
  YG_CUDA(cudaMalloc(&p, n));
  bytes = n;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
}

Lattice::~Lattice() {
  for (double *s : scratch) if (s) cudaFree(s);
  if (host_result) cudaFreeHost(host_result);
  if (sl_hist) cudaFreeHost(sl_hist);
  if (mr_hist) cudaFreeHost(mr_hist);
  for (cudaEvent_t e : sl_ev) if (e) cudaEventDestroy(e);
  if (stream) {
    cudaStreamSynchronize(stream);
    cudaStreamDestroy(stream);
  }
  for (DevBuf *b : {&fund, &links, &clover, &ldl, &cl_force, &mom, &tables, &red_partial, &red_result, &links_f,
                    &clover_f, &cinv_f, &sl_links, &sl_clover, &cpk64, &sl_part, &sl_scal, &fund_backup, &sl_cnorm,
                    &mr_work, &mr_scal, &mr_part, &mr_clov})
    b->release();
}

double *Lattice::scratch_field(int i) {
  while ((int)scratch.size() <= i) scratch.push_back(nullptr);
  if (!scratch[i]) {
    YG_CUDA(cudaMalloc(&scratch[i], field_bytes()));
    YG_CUDA(cudaMemsetAsync(scratch[i], 0, field_bytes(), stream));
  }
  return scratch[i];
}

void Lattice::view_range(int view, long &lo, long &n) const {
  switch (view) {
    case YG_VIEW_EVEN: lo = 0; n = Vh; return;
    case YG_VIEW_ODD: lo = Vh; n = Vh; return;
    case YG_VIEW_FULL: lo = 0; n = V; return;
    case YG_VIEW_DEFAULT:
      if (p.eo) { lo = 0; n = Vh; } else { lo = 0; n = V; }
      return;
    default: throw Error(YG_ERR_ARG, "invalid view");
  }
}

// ------------------------------------------------------------------ host tables
using cd = std::complex<double>;

// suNg(suNa&) of suNg.cpp:15-58 for the unit algebra vector e_which
static std::vector<cd> su_generator(int nc, int which) {
  std::vector<cd> out(nc * nc, 0.0);
  int n = 0;
  for (int i = 0; i < nc; i++)
    for (int j = 0; j < nc; j++) {
      double a;
      if (i > j) {
        a = (n == which); out[i * nc + j] += cd(0, a); out[j * nc + i] += cd(0, a); n++;
      } else if (i < j) {
        a = (n == which); out[i * nc + j] += a; out[j * nc + i] -= a; n++;
      } else if (i > 0) {
        a = (n == which);
        double v = std::sqrt(2.0 / (i * (i + 1)));
        for (int k = 0; k < i; k++) out[k * nc + k] += cd(0, v * a);
        out[i * nc + i] -= cd(0, i * v * a);
        n++;
      }
    }
  return out;
}

static int repr_dim(int nc, int rep) {
  switch (rep) {
    case YG_REPR_FUNDAMENTAL: return nc;
    case YG_REPR_ADJOINT: return nc * nc - 1;
    case YG_REPR_SYMMETRIC: return nc * (nc + 1) / 2;
    case YG_REPR_ANTISYMMETRIC: return nc * (nc - 1) / 2;
  }
  return -1;
}

// basis b_n of the representation space, repr.cpp:25-59 (fundamental: unused)
static std::vector<cd> repr_basis(int nc, int rep, int d) {
  std::vector<cd> b(d * nc * nc, 0.0);
  const double s = 1.0 / std::sqrt(2.0);
  int n = 0;
  if (rep == YG_REPR_SYMMETRIC) {
    for (int i = 0; i < nc; i++)
      for (int j = 0; j <= i; j++, n++) {
        if (i == j) b[n * nc * nc + i * nc + i] = 1.0;
        else { b[n * nc * nc + i * nc + j] = s; b[n * nc * nc + j * nc + i] = s; }
      }
  } else if (rep == YG_REPR_ANTISYMMETRIC) {
    for (int i = 0; i < nc; i++)
      for (int j = 0; j < i; j++, n++) {
        b[n * nc * nc + j * nc + i] = s;
        b[n * nc * nc + i * nc + j] = -s;
      }
  } else if (rep == YG_REPR_ADJOINT) {
    for (n = 0; n < nc * nc - 1; n++) {
      auto g = su_generator(nc, n);
      for (int k = 0; k < nc * nc; k++) b[n * nc * nc + k] = cd(0, -s) * g[k];
    }
  }
  return b;
}

static std::vector<cd> matmul(const std::vector<cd> &a, const std::vector<cd> &b, int n) {
  std::vector<cd> c(n * n, 0.0);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < n; k++)
      for (int j = 0; j < n; j++) c[i * n + j] += a[i * n + k] * b[k * n + j];
  return c;
}

static std::vector<cd> transpose(const std::vector<cd> &a, int n, bool conjugate) {
  std::vector<cd> c(n * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) c[i * n + j] = conjugate ? std::conj(a[j * n + i]) : a[j * n + i];
  return c;
}

// iTrepr of repr.cpp:73-104
static std::vector<cd> repr_generators(int nc, int rep, int d, const std::vector<cd> &basis) {
  int ng = nc * nc - 1;
  std::vector<cd> out(ng * d * d, 0.0);
  for (int k = 0; k < ng; k++) {
    auto t = su_generator(nc, k);
    if (rep == YG_REPR_FUNDAMENTAL) {
      for (int q = 0; q < d * d; q++) out[k * d * d + q] = t[q];
      continue;
    }
    for (int i = 0; i < d; i++)
      for (int j = 0; j < d; j++) {
        std::vector<cd> bi(basis.begin() + i * nc * nc, basis.begin() + (i + 1) * nc * nc);
        std::vector<cd> bj(basis.begin() + j * nc * nc, basis.begin() + (j + 1) * nc * nc);
        std::vector<cd> m1, m2;
        if (rep == YG_REPR_ADJOINT) {
          m1 = matmul(matmul(bj, bi, nc), t, nc);
          m2 = matmul(matmul(bi, bj, nc), transpose(t, nc, true), nc);
        } else if (rep == YG_REPR_SYMMETRIC) {
          m1 = matmul(matmul(bj, bi, nc), t, nc);
          m2 = matmul(matmul(bi, bj, nc), transpose(t, nc, false), nc);
        } else {
          auto bit = transpose(bi, nc, false);
          m1 = matmul(matmul(bj, bit, nc), t, nc);
          m2 = matmul(matmul(bit, bj, nc), transpose(t, nc, false), nc);
        }
        cd tr = 0;
        for (int a = 0; a < nc; a++) tr += m1[a * nc + a] + m2[a * nc + a];
        out[k * d * d + i * d + j] = tr;
      }
  }
  return out;
}

// ------------------------------------------------------------------ layout kernels
// Host AoS record (re block, then im block; `rec` complex entries) <-> device SoA
__global__ void k_aos_to_soa(double2 *dst, const double *src, Geom g, int rec, int per_site, long nrec) {
  long r = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  int id = (int)(r / per_site);
  int sub = (int)(r % per_site);
  const double *s = src + r * 2 * rec;
  for (int k = 0; k < rec; k++)
    dst[fidx(g, id, sub * rec + k, per_site * rec)] = make_double2(s[k], s[rec + k]);
}

__global__ void k_soa_to_aos(double *dst, const double2 *src, Geom g, int rec, int per_site, long nrec) {
  long r = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (r >= nrec) return;
  int id = (int)(r / per_site);
  int sub = (int)(r % per_site);
  double *s = dst + r * 2 * rec;
  for (int k = 0; k < rec; k++) {
    double2 v = src[fidx(g, id, sub * rec + k, per_site * rec)];
    s[k] = v.x;
    s[rec + k] = v.y;
  }
}

// Spinor{re[d][4], im[d][4]} (colour-major) <-> device k = spin*d + colour
__global__ void k_spinor_to_dev(double2 *dst, const double *src, Geom g, int d) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.V) return;
  const double *s = src + (long)id * 8 * d;
  for (int c = 0; c < d; c++)
    for (int sp = 0; sp < 4; sp++)
      dst[fidx(g, id, sp * d + c, 4 * d)] = make_double2(s[c * 4 + sp], s[4 * d + c * 4 + sp]);
}

__global__ void k_spinor_to_host(double *dst, const double2 *src, Geom g, int d) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.V) return;
  double *s = dst + (long)id * 8 * d;
  for (int c = 0; c < d; c++)
    for (int sp = 0; sp < 4; sp++) {
      double2 v = src[fidx(g, id, sp * d + c, 4 * d)];
      s[c * 4 + sp] = v.x;
      s[4 * d + c * 4 + sp] = v.y;
    }
}

// ------------------------------------------------------------------ gauge field
void represent_and_clover(Lattice &L) {
  YG_DISPATCH_ND(L.nc, L.d, K::represent(L.links.as<double2>(), L.fund.as<double2>(), L.g, L.rt.basis, L.p.repr, L.stream));
  YG_LAUNCHED();
  if (L.p.clover) {
    YG_DISPATCH_ND(L.nc, L.d, K::clover_term(L.clover.as<double2>(), L.fund.as<double2>(), L.g, L.rt.basis, L.p.repr,
                                              L.p.csw, L.stream));
    YG_LAUNCHED();
  }
  L.ldl_valid = false;          // cl_sigma = 0xF00F, clover.cpp:337
  L.cinv_f_valid = false;
  L.links_f_valid = false;
  L.sl_valid = false;
}

void ensure_ldl(Lattice &L, double sigma) {
  if (!L.p.clover) return;
  if (L.ldl_valid && L.ldl_sigma == sigma) return;    // clover.cpp:314-321
  int boundary_term = (L.p.bc == YG_BC_OPEN || L.p.bc == YG_BC_SF);
  YG_DISPATCH_D(L.d, K::ldl(L.ldl.as<double2>(), L.clover.as<double2>(), L.g, sigma, L.p.cf, boundary_term, L.stream));
  YG_LAUNCHED();
  if (L.d <= kPackedInverseMaxD) {
    // the Schur step of the FP64 operator applies this explicit inverse (a Hermitian
    // mat-vec) instead of the LDL substitutions: same matrix, no serial divide chain
    L.cpk64.alloc(sizeof(double2) * 2 * 2 * (size_t)L.d * L.d * L.Vh);
    YG_DISPATCH_D(L.d, K::cinv_packed64(L.cpk64.as<double2>(), L.ldl.as<double2>(), (int)L.Vh, L.stream));
    YG_LAUNCHED();
  }
  L.ldl_sigma = sigma;
  L.ldl_valid = true;
}

// ------------------------------------------------------------------ lifecycle
Lattice *lattice_create(const yg_params &p) {
  for (int mu = 0; mu < 4; mu++)
    if (p.dims[mu] < 2 || (p.dims[mu] & 1)) throw Error(YG_ERR_ARG, "lattice dimensions must be even and >= 2");
  if (p.nc < 2 || p.nc > 4) throw Error(YG_ERR_ARG, "nc must be 2, 3 or 4");
  if (p.repr < 0 || p.repr > 3) throw Error(YG_ERR_ARG, "invalid representation");
  if (p.bc < 0 || p.bc > 3) throw Error(YG_ERR_ARG, "invalid boundary condition");
  if (p.bc == YG_BC_SF && p.nc > 3) throw Error(YG_ERR_ARG, "SF boundary conditions exist for N=2,3 only (bcs.cpp:210-222)");
  int d = repr_dim(p.nc, p.repr);
  if (d < 1) throw Error(YG_ERR_ARG, "representation dimension < 1");
  long V = (long)p.dims[0] * p.dims[1] * p.dims[2] * p.dims[3];
  if (V >= (1L << 30)) throw Error(YG_ERR_ARG, "lattice too large for 32-bit site indices");
  int dev_count = 0;
  YG_CUDA(cudaGetDeviceCount(&dev_count));
  Lattice *L = new Lattice();
  try {
    // the lattice's own stream; a blocking stream, so work on the legacy default stream
    // (and events recorded there) still orders with it
    YG_CUDA(cudaStreamCreateWithFlags(&L->stream, cudaStreamDefault));
    YG_CUDA(cudaGetDevice(&L->device));
    L->p = p;
    L->d = d;
    L->nc = p.nc;
    L->ng = p.nc * p.nc - 1;
    L->V = V;
    L->Vh = V / 2;
    Geom &g = L->g;
    for (int mu = 0; mu < 4; mu++) g.dim[mu] = p.dims[mu];
    g.V = (int)V;
    g.Vh = (int)(V / 2);
    g.eo = p.eo ? 1 : 0;
    g.bc = p.bc;
    g.zt[0] = g.zt[1] = g.zt[2] = -1;
    g.Ta = g.Tb = -1;
    int T = p.dims[0];
    if (p.bc == YG_BC_OPEN) { g.zt[0] = 0; g.zt[1] = T - 1; g.Ta = 1; g.Tb = T - 2; }                 // bcs.cpp:33-70
    if (p.bc == YG_BC_SF) { g.zt[0] = 0; g.zt[1] = T - 2; g.zt[2] = T - 1; g.Ta = 1; g.Tb = T - 3; } // bcs.cpp:73-133

    int nc = p.nc, ng = L->ng;
    L->fund.alloc(sizeof(double2) * 4 * V * nc * nc);
    L->links.alloc(sizeof(double2) * 4 * V * d * d);
    YG_CUDA(cudaMemset(L->fund.p, 0, L->fund.bytes));
    YG_CUDA(cudaMemset(L->links.p, 0, L->links.bytes));
    if (p.clover) {
      L->clover.alloc(sizeof(double2) * 4 * V * d * d);
      L->ldl.alloc(sizeof(double2) * 2 * (long)d * (2 * d + 1) * (V / 2));
      L->cl_force.alloc(sizeof(double2) * 6 * V * d * d);
      YG_CUDA(cudaMemset(L->clover.p, 0, L->clover.bytes));
      YG_CUDA(cudaMemset(L->cl_force.p, 0, L->cl_force.bytes));
    }
    L->mom.alloc(sizeof(double) * 4 * V * ng);
    YG_CUDA(cudaMemset(L->mom.p, 0, L->mom.bytes));

    auto basis = repr_basis(nc, p.repr, d);
    auto itr = repr_generators(nc, p.repr, d, basis);
    std::vector<cd> itf(ng * nc * nc);
    for (int k = 0; k < ng; k++) {
      auto t = su_generator(nc, k);
      for (int q = 0; q < nc * nc; q++) itf[k * nc * nc + q] = t[q];
    }
    size_t nb = basis.size(), nr = itr.size(), nf = itf.size();
    L->tables.alloc(sizeof(double2) * (nb + nr + nf));
    std::vector<double2> host(nb + nr + nf);
    for (size_t i = 0; i < nb; i++) host[i] = make_double2(basis[i].real(), basis[i].imag());
    for (size_t i = 0; i < nr; i++) host[nb + i] = make_double2(itr[i].real(), itr[i].imag());
    for (size_t i = 0; i < nf; i++) host[nb + nr + i] = make_double2(itf[i].real(), itf[i].imag());
    YG_CUDA(cudaMemcpy(L->tables.p, host.data(), sizeof(double2) * host.size(), cudaMemcpyHostToDevice));
    L->rt.basis = L->tables.as<double2>();
    L->rt.itrepr = L->rt.basis + nb;
    L->rt.itfund = L->rt.itrepr + nr;

    // reduction scratch: one partial (double2) per block + result
    L->red_blocks = 148 * 8;
    L->red_partial.alloc(sizeof(double2) * L->red_blocks);
    L->red_result.alloc(sizeof(double2) * 4);
    YG_CUDA(cudaMallocHost(&L->host_result, sizeof(double) * 8));

    // unit gauge field (gauge_field_set_unit, gaugefield.cpp:200-215)
    std::vector<double> unit((size_t)4 * V * 2 * nc * nc, 0.0);
    for (long r = 0; r < 4 * V; r++)
      for (int i = 0; i < nc; i++) unit[r * 2 * nc * nc + i * nc + i] = 1.0;
    DevBuf tmp;
    tmp.alloc(unit.size() * sizeof(double));
    YG_CUDA(cudaMemcpy(tmp.p, unit.data(), unit.size() * sizeof(double), cudaMemcpyHostToDevice));
    k_aos_to_soa<<<nblk(4 * V, 128), 128, 0, L->stream>>>(L->fund.as<double2>(), tmp.as<double>(), g, nc * nc, 4, 4 * V);
    YG_LAUNCHED();
    represent_and_clover(*L);
    YG_CUDA(cudaStreamSynchronize(L->stream));
    tmp.release();
  } catch (...) {
    delete L;
    throw;
  }
  return L;
}

// ---- host <-> device conversions
static void upload_records(Lattice &L, DevBuf &dst, const double *host, int rec, int per_site) {
  long nrec = (long)L.V * per_site;
  size_t bytes = sizeof(double) * nrec * 2 * rec;
  DevBuf big;
  double *buf = L.scratch_field(0);
  if (bytes > L.field_bytes()) { big.alloc(bytes); buf = big.as<double>(); }
  YG_CUDA(cudaMemcpyAsync(buf, host, bytes, cudaMemcpyHostToDevice, L.stream));
  k_aos_to_soa<<<nblk(nrec, 128), 128, 0, L.stream>>>(dst.as<double2>(), buf, L.g, rec, per_site, nrec);
  YG_LAUNCHED();
  YG_CUDA(cudaStreamSynchronize(L.stream));
  big.release();
}

static void download_records(Lattice &L, double *host, const void *src, int rec, int per_site) {
  long nrec = (long)L.V * per_site;
  size_t bytes = sizeof(double) * nrec * 2 * rec;
  DevBuf big;
  double *buf = L.scratch_field(0);
  if (bytes > L.field_bytes()) { big.alloc(bytes); buf = big.as<double>(); }
  k_soa_to_aos<<<nblk(nrec, 128), 128, 0, L.stream>>>(buf, (const double2 *)src, L.g, rec, per_site, nrec);
  YG_LAUNCHED();
  YG_CUDA(cudaMemcpyAsync(host, buf, bytes, cudaMemcpyDeviceToHost, L.stream));
  YG_CUDA(cudaStreamSynchronize(L.stream));
  big.release();
}

void gauge_upload(Lattice &L, const double *host) {
  upload_records(L, L.fund, host, L.nc * L.nc, 4);
  represent_and_clover(L);
  YG_CUDA(cudaStreamSynchronize(L.stream));
}

// the fundamental links alone: what the reference's update_links leaves behind on the host
// (update.cpp:228-247) before represent_gauge_field runs; the represented field and the
// clover term keep the state of the last gauge_upload / represent_and_clover
void gauge_upload_fund(Lattice &L, const double *host) {
  upload_records(L, L.fund, host, L.nc * L.nc, 4);
  YG_CUDA(cudaStreamSynchronize(L.stream));
}

// as gauge_field_load does after reading (gaugefield.cpp:146-152): the links, then the
// boundary conditions on them, then the represented field
void gauge_upload_with_bcs(Lattice &L, const double *host) {
  upload_records(L, L.fund, host, L.nc * L.nc, 4);
  apply_gauge_bcs(L);
  represent_and_clover(L);
  YG_CUDA(cudaStreamSynchronize(L.stream));
}

void gauge_download(Lattice &L, double *host) { download_records(L, host, L.fund.p, L.nc * L.nc, 4); }
void repr_download(Lattice &L, double *host) { download_records(L, host, L.links.p, L.d * L.d, 4); }

void clover_download(Lattice &L, double *host) {
  if (!L.p.clover) throw Error(YG_ERR_ARG, "clover term disabled");
  download_records(L, host, L.clover.p, L.d * L.d, 4);
}

void clover_force_download(Lattice &L, double *host) {
  if (!L.p.clover) throw Error(YG_ERR_ARG, "clover term disabled");
  download_records(L, host, L.cl_force.p, L.d * L.d, 6);
}

// ldl_t records (clover.h:30-33): complex upper[P], lower[P] per site; block-1 sites filled
void ldl_download(Lattice &L, double mass, double *host) {
  if (!L.p.clover) throw Error(YG_ERR_ARG, "clover term disabled");
  ensure_ldl(L, 4.0 + mass);
  long P = (long)L.d * (2 * L.d + 1);
  std::vector<double2> dev(2 * P * L.Vh);
  YG_CUDA(cudaMemcpyAsync(dev.data(), L.ldl.p, sizeof(double2) * dev.size(), cudaMemcpyDeviceToHost, L.stream));
  YG_CUDA(cudaStreamSynchronize(L.stream));
  std::memset(host, 0, sizeof(double) * 4 * P * L.V);
  for (long h = 0; h < L.Vh; h++) {
    double *rec = host + (L.Vh + h) * 4 * P;
    for (int b = 0; b < 2; b++)
      for (long k = 0; k < P; k++) {
        double2 v = dev[(b * P + k) * L.Vh + h];
        rec[(b * P + k) * 2] = v.x;
        rec[(b * P + k) * 2 + 1] = v.y;
      }
  }
}

void field_upload(Lattice &L, double *dev, const double *host) {
  double *stage = L.scratch_field(0);
  YG_CUDA(cudaMemcpyAsync(stage, host, L.field_bytes(), cudaMemcpyHostToDevice, L.stream));
  k_spinor_to_dev<<<nblk(L.V, 128), 128, 0, L.stream>>>((double2 *)dev, stage, L.g, L.d);
  YG_LAUNCHED();
}

void field_download(Lattice &L, double *host, const double *dev) {
  double *stage = L.scratch_field(0);
  k_spinor_to_host<<<nblk(L.V, 128), 128, 0, L.stream>>>(stage, (const double2 *)dev, L.g, L.d);
  YG_LAUNCHED();
  YG_CUDA(cudaMemcpyAsync(host, stage, L.field_bytes(), cudaMemcpyDeviceToHost, L.stream));
  YG_CUDA(cudaStreamSynchronize(L.stream));
}

void momenta_upload(Lattice &L, const double *host) {
  YG_CUDA(cudaMemcpyAsync(L.mom.p, host, L.mom.bytes, cudaMemcpyHostToDevice, L.stream));
  YG_CUDA(cudaStreamSynchronize(L.stream));
}

void momenta_download(Lattice &L, double *host) {
  YG_CUDA(cudaMemcpyAsync(host, L.mom.p, L.mom.bytes, cudaMemcpyDeviceToHost, L.stream));
  YG_CUDA(cudaStreamSynchronize(L.stream));
}

}  // namespace yg
