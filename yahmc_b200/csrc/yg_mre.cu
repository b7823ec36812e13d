// Minimal residual extrapolation of the initial guess from past solutions (mre.cpp:15-117,
// with the LU solve of solver.cpp:4-95).  The past solutions stay on the device; every
// vector operation is the engine's BLAS on the default view (even sites with even-odd
// preconditioning), the operator is the solver's, and only the small projected system
// (at most 15 x 15 complex) is solved on the host.
#include <cmath>
#include <complex>
#include <vector>
#include "yg_lattice.h"

namespace yg {

constexpr int kMreMax = 15;                 // MRE_MAX, mre.h:7

struct Mre {
  Lattice *L = nullptr;
  int max = 0, num = 0, op = YG_OP_HPHI_SQ;
  double mass = 0;
  std::vector<double *> s;                  // past solutions, newest first
  double *out = nullptr;                    // operator scratch
  ~Mre() {
    for (double *p : s) if (p) cudaFree(p);
    if (out) cudaFree(out);
  }
};

using zc = std::complex<double>;

// A x = b for a small dense complex system (A row-major, overwritten): LU factorisation
// with partial pivoting on the column, then forward and back substitution.  A pivot below
// 1e-14 means the stored solutions are (numerically) dependent: an error, where the
// reference stops the program (solver.cpp:46-49).
static void lu_solve(int n, std::vector<zc> &A, std::vector<zc> &x, const std::vector<zc> &b) {
  std::vector<int> perm(n);
  for (int i = 0; i < n; i++) perm[i] = i;
  for (int c = 0; c < n; c++) {
    int piv = c;
    double big = std::abs(A[c * n + c]);
    for (int r = c + 1; r < n; r++)
      if (std::abs(A[r * n + c]) > big) { big = std::abs(A[r * n + c]); piv = r; }
    if (big < 1e-14) throw Error(YG_ERR_ARG, "mre_guess: the projected system is singular");
    if (piv != c) {
      for (int k = 0; k < n; k++) std::swap(A[piv * n + k], A[c * n + k]);
      std::swap(perm[piv], perm[c]);
    }
    for (int r = c + 1; r < n; r++) {
      const zc f = A[r * n + c] / A[c * n + c];
      A[r * n + c] = f;
      for (int k = c + 1; k < n; k++) A[r * n + k] -= f * A[c * n + k];
    }
  }
  x.assign(n, zc(0, 0));
  for (int i = 0; i < n; i++) {
    zc v = b[perm[i]];
    for (int k = 0; k < i; k++) v -= A[i * n + k] * x[k];
    x[i] = v;
  }
  for (int i = n - 1; i >= 0; i--) {
    zc v = x[i];
    for (int k = i + 1; k < n; k++) v -= A[i * n + k] * x[k];
    x[i] = v / A[i * n + i];
  }
}

// mre_init, mre.cpp:85-111: max = 0 disables the extrapolation
Mre *mre_create(Lattice &L, int max, int op, double mass) {
  if (max < 0) throw Error(YG_ERR_ARG, "mre: max must be >= 0");
  if (op != YG_OP_DPHI && op != YG_OP_HPHI && op != YG_OP_HPHI_SQ) throw Error(YG_ERR_ARG, "mre: unknown operator");
  Mre *m = new Mre();
  try {
    m->L = &L;
    m->max = max < kMreMax ? max : kMreMax;
    m->op = op;
    m->mass = mass;
    if (m->max > 0) {
      YG_CUDA(cudaMalloc(&m->out, L.field_bytes()));
      for (int k = 0; k < m->max; k++) {
        double *p = nullptr;
        YG_CUDA(cudaMalloc(&p, L.field_bytes()));
        YG_CUDA(cudaMemsetAsync(p, 0, L.field_bytes(), L.stream));
        m->s.push_back(p);
      }
    }
  } catch (...) {
    delete m;
    throw;
  }
  return m;
}

void mre_destroy(Mre *m) { delete m; }

// mre_reset, mre.cpp:113-116
void mre_reset(Mre &m) { m.num = 0; }

// mre_store, mre.cpp:35-51: the oldest buffer becomes slot 0 and takes a copy of the solution
void mre_store(Mre &m, const double *sol) {
  if (m.max == 0) return;
  double *tmp = m.s[m.max - 1];
  for (int k = m.max - 1; k > 0; k--) m.s[k] = m.s[k - 1];
  m.s[0] = tmp;
  blas_copy(*m.L, m.s[0], sol);
  m.num++;
}

// mre_guess, mre.cpp:53-83: dst = sum_k x_k s_k with the stored solutions orthonormalised
// in place (Gram-Schmidt) and x solving <A s_i, s_j> x = <src, s_j>
void mre_guess(Mre &m, double *dst, const double *src) {
  if (m.max == 0) return;
  Lattice &L = *m.L;
  long lo, n;
  L.view_range(YG_VIEW_DEFAULT, lo, n);
  const int k = m.num > m.max ? m.max : m.num;
  blas_zero(L, dst, 0, L.V);
  // gram_schmidt, mre.cpp:14-33
  for (int i = 0; i < k; i++) {
    const double rii = 1.0 / std::sqrt(blas_sqnorm(L, m.s[i], lo, n));
    blas_axpby(L, m.s[i], make_double2(rii, 0), make_double2(0, 0), nullptr, lo, n);
    for (int j = i + 1; j < k; j++) {
      const double2 rij = blas_product(L, m.s[i], m.s[j], lo, n);
      blas_axpby(L, m.s[j], make_double2(1, 0), make_double2(-rij.x, -rij.y), m.s[i], lo, n);
    }
  }
  std::vector<zc> A((size_t)k * k), b(k), x;
  for (int i = 0; i < k; i++) {
    apply_op(L, m.op, m.mass, m.out, m.s[i]);
    for (int j = 0; j < k; j++) {
      const double2 v = blas_product(L, m.out, m.s[j], lo, n);
      A[(size_t)j * k + i] = zc(v.x, v.y);
    }
    const double2 v = blas_product(L, src, m.s[i], lo, n);
    b[i] = zc(v.x, v.y);
  }
  if (k == 0) return;
  lu_solve(k, A, x, b);
  for (int i = 0; i < k; i++)
    blas_axpby(L, dst, make_double2(1, 0), make_double2(x[i].real(), x[i].imag()), m.s[i], lo, n);
}

}  // namespace yg
