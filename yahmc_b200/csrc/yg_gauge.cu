// Gauge-field side of the molecular dynamics, on the fundamental links (FP64):
//   plaquette / rectangle weights of the boundary conditions      bcs.cpp:29-133
//   staples_wilson, staples_symanzik                               staples.cpp:7-107
//   wilson_gauge_force, improved_gauge_force                       forces.cpp:262-309
//   wilson_loop, avr_wilson                                        wilsonloop.cpp:56-133
//   update_links (exp(eps P) U), reunitarize                       update.cpp:228-279, suNa.cpp:113-134,
//                                                                  suNg.cpp:15-58, 171-359
//   apply_bcs_on_momentum_field / _gauge_field                     bcs.cpp:166-262
//   momentum refresh and the momentum part of hamiltonian()        update.cpp:201-226, 254-267
// One thread per link (site, mu) or per site; links and momenta keep the layouts of the
// rest of the engine (links SoA per component, momenta [site][mu][a]).
#include <cmath>
#include "yg_forces_impl.cuh"
#include "yg_lattice.h"

namespace yg {

// ------------------------------------------------------------------ boundary weights
// plaq_weight(id,mu,nu): 0.5 on the spatial planes of the open (t = 0, T-1) and SF
// (t = 0, T-2) boundary slices, 1 elsewhere
__device__ __forceinline__ double plaq_w(const Geom &g, int t, int mu, int nu) {
  if (mu == 0 || nu == 0) return 1.0;
  const int T = g.dim[0];
  if (g.bc == YG_BC_OPEN && (t == 0 || t == T - 1)) return 0.5;
  if (g.bc == YG_BC_SF && (t == 0 || t == T - 2)) return 0.5;
  return 1.0;
}

// rect_weight(id,mu,nu): the plaquette weights for open boundaries (one array there); for
// SF 0 on the planes (1,2),(1,3),(2,3) at t = 0 and T-2, and 1.5 on (0,1),(0,2),(0,3) at
// t = 0 and T-3 (ordered pairs, as the reference fills them)
__device__ __forceinline__ double rect_w(const Geom &g, int t, int mu, int nu) {
  if (g.bc != YG_BC_SF) return plaq_w(g, t, mu, nu);
  const int T = g.dim[0];
  if ((t == 0 || t == T - 2) && mu >= 1 && nu > mu) return 0.0;
  if ((t == 0 || t == T - 3) && mu == 0 && nu >= 1) return 1.5;
  return 1.0;
}

// ------------------------------------------------------------------ small-matrix helpers
// a lattice position: coordinates plus the site index they map to
struct Pos {
  int c[4];
  int id;
};

__device__ __forceinline__ Pos pos_of(const Geom &g, int id) {
  Pos p;
  coords_of(g, id, p.c);
  p.id = id;
  return p;
}

__device__ __forceinline__ Pos step(const Geom &g, Pos p, int mu, int dir) {
  const int L = g.dim[mu];
  p.c[mu] = dir > 0 ? (p.c[mu] + 1 == L ? 0 : p.c[mu] + 1) : (p.c[mu] == 0 ? L - 1 : p.c[mu] - 1);
  p.id = id_of(g, p.c[0], p.c[1], p.c[2], p.c[3]);
  return p;
}

template <int N>
__device__ __forceinline__ void ldU(double2 (&m)[N * N], const double2 *U, const Geom &g, const Pos &p, int mu) {
  ld_mat<N>(m, U, g, p.id, mu, 4);
}

// c = a b^dag
template <int N>
__device__ __forceinline__ void mul_dag(double2 (&c)[N * N], const double2 (&a)[N * N], const double2 (&b)[N * N]) {
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < N; k++) cfmac(s, b[j * N + k], a[i * N + k]);
      c[i * N + j] = s;
    }
}

// c = a^dag b
template <int N>
__device__ __forceinline__ void dag_mul(double2 (&c)[N * N], const double2 (&a)[N * N], const double2 (&b)[N * N]) {
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int k = 0; k < N; k++) cfmac(s, a[k * N + i], b[k * N + j]);
      c[i * N + j] = s;
    }
}

template <int N>
__device__ __forceinline__ void add_scaled(double2 (&s)[N * N], const double2 (&a)[N * N], double w) {
#pragma unroll
  for (int k = 0; k < N * N; k++) s[k] = make_double2(fma(w, a[k].x, s[k].x), fma(w, a[k].y, s[k].y));
}

// ------------------------------------------------------------------ staples and forces
// plaquette staples of link (x, mu): sum over nu of the two weighted 3-link paths
template <int N>
__device__ void staple_plaq(double2 (&st)[N * N], const double2 *U, const Geom &g, const Pos &x, int mu) {
  double2 A[N * N], B[N * N], P[N * N], Q[N * N];
#pragma unroll 1
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    // U(x+mu, nu) [U(x, nu) U(x+nu, mu)]^dag
    Pos o1 = step(g, x, mu, +1), o2 = step(g, x, nu, +1);
    ldU<N>(A, U, g, x, nu); ldU<N>(B, U, g, o2, mu); mat_mul<N>(P, A, B);
    ldU<N>(A, U, g, o1, nu); mul_dag<N>(Q, A, P);
    add_scaled<N>(st, Q, plaq_w(g, x.c[0], mu, nu));
    // [U(x-nu, mu) U(x-nu+mu, nu)]^dag U(x-nu, nu)
    Pos b1 = step(g, x, nu, -1), b2 = step(g, b1, mu, +1);
    ldU<N>(A, U, g, b1, mu); ldU<N>(B, U, g, b2, nu); mat_mul<N>(P, A, B);
    ldU<N>(A, U, g, b1, nu); dag_mul<N>(Q, P, A);
    add_scaled<N>(st, Q, plaq_w(g, b1.c[0], nu, mu));
  }
}

// R = a (b c d)^dag e f  style products of the rectangle staples, with the three links
// under the dagger multiplied first
template <int N>
__device__ __forceinline__ void prod3(double2 (&r)[N * N], const double2 *U, const Geom &g, const Pos &p0, int m0,
                                      const Pos &p1, int m1, const Pos &p2, int m2) {
  double2 A[N * N], B[N * N], C[N * N];
  ldU<N>(A, U, g, p0, m0); ldU<N>(B, U, g, p1, m1); mat_mul<N>(C, A, B);
  ldU<N>(A, U, g, p2, m2); mat_mul<N>(r, C, A);
}

// rectangle (2x1) staples of link (x, mu), staples_symanzik: for each nu the six paths
// that close a 2x1 loop with the link
template <int N>
__device__ void staple_rect(double2 (&st)[N * N], const double2 *U, const Geom &g, const Pos &x, int mu) {
  double2 H[N * N], D2[N * N], P[N * N], Q[N * N], A[N * N];
#pragma unroll 1
  for (int nu = 0; nu < 4; nu++) {
    if (nu == mu) continue;
    {  // U(x+mu,nu) U(x+mu+nu,nu) [U(x,nu) U(x+nu,nu) U(x+2nu,mu)]^dag
      Pos o1 = step(g, x, mu, +1), o2 = step(g, o1, nu, +1), o3 = step(g, x, nu, +1), o4 = step(g, o3, nu, +1);
      prod3<N>(H, U, g, x, nu, o3, nu, o4, mu);
      ldU<N>(A, U, g, o1, nu); ldU<N>(D2, U, g, o2, nu); mat_mul<N>(P, A, D2);
      mul_dag<N>(Q, P, H);
      add_scaled<N>(st, Q, rect_w(g, x.c[0], mu, nu));
    }
    {  // [U(y,mu) U(y+mu,nu) U(y+mu+nu,nu)]^dag U(y,nu) U(y+nu,nu),  y = x-2nu
      Pos o1 = step(g, x, nu, -1), o2 = step(g, o1, nu, -1), o3 = step(g, o2, mu, +1), o4 = step(g, o3, nu, +1);
      prod3<N>(H, U, g, o2, mu, o3, nu, o4, nu);
      ldU<N>(A, U, g, o2, nu); ldU<N>(D2, U, g, o1, nu); mat_mul<N>(P, A, D2);
      dag_mul<N>(Q, H, P);
      add_scaled<N>(st, Q, rect_w(g, o2.c[0], mu, nu));
    }
    {  // U(x+mu,mu) [U(y,mu) U(y+mu,mu) U(y+2mu,nu)]^dag U(y,nu),  y = x-nu
      Pos o1 = step(g, x, nu, -1), o2 = step(g, o1, mu, +1), o3 = step(g, o2, mu, +1), o4 = step(g, x, mu, +1);
      prod3<N>(H, U, g, o1, mu, o2, mu, o3, nu);
      ldU<N>(A, U, g, o4, mu); mul_dag<N>(P, A, H);
      ldU<N>(A, U, g, o1, nu); mat_mul<N>(Q, P, A);
      add_scaled<N>(st, Q, rect_w(g, o1.c[0], nu, mu));
    }
    {  // U(x+mu,mu) U(x+2mu,nu) [U(x,nu) U(x+nu,mu) U(x+nu+mu,mu)]^dag
      Pos o1 = step(g, x, mu, +1), o2 = step(g, o1, mu, +1), o3 = step(g, x, nu, +1), o4 = step(g, o3, mu, +1);
      prod3<N>(H, U, g, x, nu, o3, mu, o4, mu);
      ldU<N>(A, U, g, o1, mu); ldU<N>(D2, U, g, o2, nu); mat_mul<N>(P, A, D2);
      mul_dag<N>(Q, P, H);
      add_scaled<N>(st, Q, rect_w(g, x.c[0], nu, mu));
    }
    {  // [U(y,mu) U(y+mu,mu) U(y+2mu,nu)]^dag U(y,nu) U(y+nu,mu),  y = x-mu-nu
      Pos o1 = step(g, x, mu, -1), o2 = step(g, o1, nu, -1), o3 = step(g, o2, mu, +1), o4 = step(g, o3, mu, +1);
      prod3<N>(H, U, g, o2, mu, o3, mu, o4, nu);
      ldU<N>(A, U, g, o2, nu); ldU<N>(D2, U, g, o1, mu); mat_mul<N>(P, A, D2);
      dag_mul<N>(Q, H, P);
      add_scaled<N>(st, Q, rect_w(g, o2.c[0], nu, mu));
    }
    {  // U(x+mu,nu) [U(y,nu) U(y+nu,mu) U(y+nu+mu,mu)]^dag U(y,mu),  y = x-mu
      Pos o1 = step(g, x, mu, -1), o2 = step(g, o1, nu, +1), o3 = step(g, o2, mu, +1), o4 = step(g, x, mu, +1);
      prod3<N>(H, U, g, o1, nu, o2, mu, o3, mu);
      ldU<N>(A, U, g, o4, nu); mul_dag<N>(P, A, H);
      ldU<N>(A, U, g, o1, mu); mat_mul<N>(Q, P, A);
      add_scaled<N>(st, Q, rect_w(g, o1.c[0], nu, mu));
    }
  }
}

// mom(x,mu) -= algebra_project(U(x,mu) (c0 S_plaq + c1 S_rect), coeff); IMP = 0 skips the
// rectangles (wilson_gauge_force, c0 = 1)
template <int N, int IMP>
__global__ void __launch_bounds__(64) k_gauge_force(double *mom, const double2 *U, Geom g, const double2 *itfund,
                                                    double coeff, double c0, double c1) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  const int id = (int)(t >> 2), mu = (int)(t & 3);
  const Pos x = pos_of(g, id);
  double2 sw[N * N], F[N * N], A[N * N];
#pragma unroll
  for (int k = 0; k < N * N; k++) sw[k] = make_double2(0, 0);
  staple_plaq<N>(sw, U, g, x, mu);
  if (IMP) {
    double2 sr[N * N];
#pragma unroll
    for (int k = 0; k < N * N; k++) {
      sr[k] = make_double2(0, 0);
      sw[k] = make_double2(c0 * sw[k].x, c0 * sw[k].y);
    }
    staple_rect<N>(sr, U, g, x, mu);
    add_scaled<N>(sw, sr, c1);
  }
  ldU<N>(A, U, g, x, mu);
  mat_mul<N>(F, A, sw);
  project_add<N>(mom + (4L * id + mu) * (N * N - 1), F, itfund, N * N - 1, -coeff);
}

// ------------------------------------------------------------------ Wilson loops
// Re tr of the height x width loop in the (mu, nu) plane starting at x, weighted as
// wilson_loop does for 1x1, 1x2 and 2x1
template <int N>
__device__ double wilson_loop(const double2 *U, const Geom &g, const Pos &x, int mu, int nu, int height, int width) {
  double2 one[N * N], two[N * N], A[N * N], B[N * N];
  ldU<N>(one, U, g, x, mu);
  ldU<N>(two, U, g, x, nu);
  Pos p = x;
  for (int k = 1; k < height; k++) {
    p = step(g, p, mu, +1);
    ldU<N>(A, U, g, p, mu); mat_mul<N>(B, one, A);
#pragma unroll
    for (int q = 0; q < N * N; q++) one[q] = B[q];
  }
  p = step(g, p, mu, +1);
  ldU<N>(A, U, g, p, nu); mat_mul<N>(B, one, A);
#pragma unroll
  for (int q = 0; q < N * N; q++) one[q] = B[q];
  for (int k = 1; k < width; k++) {
    p = step(g, p, nu, +1);
    ldU<N>(A, U, g, p, nu); mat_mul<N>(B, one, A);
#pragma unroll
    for (int q = 0; q < N * N; q++) one[q] = B[q];
  }
  p = x;
  for (int k = 1; k < width; k++) {
    p = step(g, p, nu, +1);
    ldU<N>(A, U, g, p, nu); mat_mul<N>(B, two, A);
#pragma unroll
    for (int q = 0; q < N * N; q++) two[q] = B[q];
  }
  p = step(g, p, nu, +1);
  ldU<N>(A, U, g, p, mu); mat_mul<N>(B, two, A);
#pragma unroll
  for (int q = 0; q < N * N; q++) two[q] = B[q];
  for (int k = 1; k < height; k++) {
    p = step(g, p, mu, +1);
    ldU<N>(A, U, g, p, mu); mat_mul<N>(B, two, A);
#pragma unroll
    for (int q = 0; q < N * N; q++) two[q] = B[q];
  }
  double tr = 0;                      // Re tr(one two^dag) = sum Re(one_ik conj(two_ik))
#pragma unroll
  for (int q = 0; q < N * N; q++) tr += one[q].x * two[q].x + one[q].y * two[q].y;
  if (height == 1 && width == 1) tr *= plaq_w(g, x.c[0], mu, nu);
  else if (height == 1 && width == 2) tr *= rect_w(g, x.c[0], mu, nu);
  else if (height == 2 && width == 1) tr *= rect_w(g, x.c[0], nu, mu);
  return tr;
}

// per-site sum over the six planes (1,0),(2,0),(2,1),(3,0),(3,1),(3,2)
template <int N>
__global__ void __launch_bounds__(128) k_wilson_loops(double *out, const double2 *U, Geom g, int height, int width) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.V) return;
  const Pos x = pos_of(g, id);
  double s = 0;
#pragma unroll 1
  for (int mu = 1; mu < 4; mu++)
#pragma unroll 1
    for (int nu = 0; nu < mu; nu++) s += wilson_loop<N>(U, g, x, mu, nu, height, width);
  out[id] = s;
}

// ------------------------------------------------------------------ exp and reunitarize
// anti-Hermitian matrix of the algebra coordinates av (suNg(suNa&), suNg.cpp:15-58):
// off-diagonal pairs i > j take i*av at (i,j) and (j,i); pairs i < j take +av at (i,j) and
// -av at (j,i); the diagonal generators follow in the order the pairs are visited
template <int N>
__device__ __forceinline__ void algebra_matrix(double2 (&X)[N * N], const double *av) {
#pragma unroll
  for (int k = 0; k < N * N; k++) X[k] = make_double2(0, 0);
  int n = 0;
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++) {
      if (i > j) {
        X[i * N + j].y = av[n];
        X[j * N + i].y = av[n];
        n++;
      } else if (i < j) {
        X[i * N + j].x = av[n];
        X[j * N + i].x = -av[n];
        n++;
      } else if (i > 0) {
        const double v = sqrt(2.0 / (i * (i + 1)));
#pragma unroll
        for (int k = 0; k < i; k++) X[k * N + k].y += v * av[n];
        X[i * N + i].y -= i * v * av[n];
        n++;
      }
    }
}

// projection back onto SU(N): the rows are orthonormalised in order; for N = 2, 3 the last
// row is rebuilt from the others (conjugate cross product for N = 3), for larger N the last
// row takes the phase that makes the determinant one.  A matrix whose first row vanishes
// (a zero boundary link) is left unchanged.
template <int N>
__device__ void reunitarize_mat(double2 (&u)[N * N]) {
  double n0 = 0;
#pragma unroll
  for (int k = 0; k < N; k++) n0 += u[k].x * u[k].x + u[k].y * u[k].y;
  n0 = sqrt(n0);
  if (n0 == 0) return;
  if (N == 2) {
#pragma unroll
    for (int k = 0; k < 2; k++) u[k] = make_double2(u[k].x / n0, u[k].y / n0);
    u[2] = make_double2(-u[1].x, u[1].y);
    u[3] = make_double2(u[0].x, -u[0].y);
    return;
  }
  const int last = (N == 3) ? 2 : N;        // rows orthonormalised explicitly
  for (int i = 0; i < last; i++) {
    double nr = 0;
#pragma unroll
    for (int k = 0; k < N; k++) nr += u[i * N + k].x * u[i * N + k].x + u[i * N + k].y * u[i * N + k].y;
    nr = sqrt(nr);
    if (nr == 0) return;
#pragma unroll
    for (int k = 0; k < N; k++) u[i * N + k] = make_double2(u[i * N + k].x / nr, u[i * N + k].y / nr);
    for (int j = i + 1; j < last; j++) {
      double2 c = make_double2(0, 0);                      // <row i, row j>
#pragma unroll
      for (int k = 0; k < N; k++) cfmac(c, u[i * N + k], u[j * N + k]);
#pragma unroll
      for (int k = 0; k < N; k++) u[j * N + k] = csub(u[j * N + k], cmul(c, u[i * N + k]));
    }
  }
  if (N == 3) {
    const double2 a0 = u[0], a1 = u[1], a2 = u[2], b0 = u[3], b1 = u[4], b2 = u[5];
    u[6] = cconj(csub(cmul(a1, b2), cmul(a2, b1)));
    u[7] = cconj(csub(cmul(a2, b0), cmul(a0, b2)));
    u[8] = cconj(csub(cmul(a0, b1), cmul(a1, b0)));
    return;
  }
  // determinant by Gaussian elimination on a copy, then the last row times exp(-i arg det)
  double2 m[N * N];
#pragma unroll
  for (int k = 0; k < N * N; k++) m[k] = u[k];
  double2 det = make_double2(1, 0);
  for (int i = 0; i < N; i++) {
    const double2 piv = m[i * N + i];
    det = cmul(det, piv);
    const double pn = piv.x * piv.x + piv.y * piv.y;
    if (pn == 0) break;
    const double2 inv = make_double2(piv.x / pn, -piv.y / pn);
    for (int r = i + 1; r < N; r++) {
      const double2 f = cmul(m[r * N + i], inv);
      for (int k = i; k < N; k++) m[r * N + k] = csub(m[r * N + k], cmul(f, m[i * N + k]));
    }
  }
  const double ph = atan2(det.y, det.x);
  double s, c;
  sincos(ph, &s, &c);
  const double2 rot = make_double2(c, -s);
#pragma unroll
  for (int k = 0; k < N; k++) u[(N - 1) * N + k] = cmul(u[(N - 1) * N + k], rot);
}

// exp(eps X) by its Taylor series, each term (eps/k) X^(k-1)/... X added until the last
// added term has squared norm <= 1e-24 (at most 64 terms), then reunitarised
template <int N>
__device__ void exp_algebra(double2 (&E)[N * N], const double2 (&X)[N * N], double eps) {
  double2 Xk[N * N], T[N * N];
#pragma unroll
  for (int k = 0; k < N * N; k++) {
    Xk[k] = make_double2(0, 0);
    E[k] = make_double2(0, 0);
  }
#pragma unroll
  for (int i = 0; i < N; i++) {
    Xk[i * N + i] = make_double2(1, 0);
    E[i * N + i] = make_double2(1, 0);
  }
  double err = 1;
  for (int k = 1; err > 1e-24 && k <= 64; k++) {
    mat_mul<N>(T, Xk, X);
    const double f = eps / k;
    err = 0;
#pragma unroll
    for (int q = 0; q < N * N; q++) {
      Xk[q] = make_double2(f * T[q].x, f * T[q].y);
      E[q] = cadd(E[q], Xk[q]);
      err += Xk[q].x * Xk[q].x + Xk[q].y * Xk[q].y;
    }
  }
  reunitarize_mat<N>(E);
}

// the link boundary values of apply_bcs_on_gauge_field for link (t, mu); returns false
// when the link is free.  SF boundary fields are diagonal: sf1, sf2 hold their entries.
struct SFLinks {
  double2 c1[4], c2[4];
};

template <int N>
__device__ __forceinline__ bool gauge_bc(double2 (&u)[N * N], const Geom &g, int t, int mu, const SFLinks &sf) {
  const int T = g.dim[0];
  if (g.bc == YG_BC_OPEN) {
    if (t == T - 1 && mu == 0) {
#pragma unroll
      for (int k = 0; k < N * N; k++) u[k] = make_double2(0, 0);
      return true;
    }
    return false;
  }
  if (g.bc != YG_BC_SF) return false;
  const double2 *diag = nullptr;
  bool zero = false;
  if (t == 0 && mu >= 1) diag = sf.c1;
  else if (t == T - 2) { if (mu == 0) zero = true; else diag = sf.c2; }
  else if (t == T - 1) zero = true;
  if (!zero && !diag) return false;
#pragma unroll
  for (int k = 0; k < N * N; k++) u[k] = make_double2(0, 0);
  if (diag) {
#pragma unroll
    for (int i = 0; i < N; i++) u[i * N + i] = diag[i];
  }
  return true;
}

// U(x,mu) <- exp(eps P(x,mu)) U(x,mu), then the link boundary values
template <int N>
__global__ void __launch_bounds__(64) k_update_links(double2 *U, const double *mom, Geom g, double eps, SFLinks sf) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  const int id = (int)(t >> 2), mu = (int)(t & 3);
  int c[4];
  coords_of(g, id, c);
  double2 u[N * N];
  if (!gauge_bc<N>(u, g, c[0], mu, sf)) {
    double av[N * N - 1];
#pragma unroll
    for (int a = 0; a < N * N - 1; a++) av[a] = mom[(4L * id + mu) * (N * N - 1) + a];
    double2 X[N * N], E[N * N], V0[N * N];
    algebra_matrix<N>(X, av);
    exp_algebra<N>(E, X, eps);
    ld_mat<N>(V0, U, g, id, mu, 4);
    mat_mul<N>(u, E, V0);
  }
#pragma unroll
  for (int k = 0; k < N * N; k++) U[fidx(g, id, mu * N * N + k, 4 * N * N)] = u[k];
}

// apply_bcs_on_gauge_field alone (bcs.cpp:201-262): the boundary links take their fixed values
template <int N>
__global__ void __launch_bounds__(64) k_gauge_bcs(double2 *U, Geom g, SFLinks sf) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  const int id = (int)(t >> 2), mu = (int)(t & 3);
  int c[4];
  coords_of(g, id, c);
  double2 u[N * N];
  if (gauge_bc<N>(u, g, c[0], mu, sf)) {
#pragma unroll
    for (int k = 0; k < N * N; k++) U[fidx(g, id, mu * N * N + k, 4 * N * N)] = u[k];
  }
}

template <int N>
__global__ void __launch_bounds__(64) k_reunitarize(double2 *U, Geom g) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  const int id = (int)(t >> 2), mu = (int)(t & 3);
  double2 u[N * N];
  ld_mat<N>(u, U, g, id, mu, 4);
  reunitarize_mat<N>(u);
#pragma unroll
  for (int k = 0; k < N * N; k++) U[fidx(g, id, mu * N * N + k, 4 * N * N)] = u[k];
}

// ------------------------------------------------------------------ momenta
// apply_bcs_on_momentum_field: open zeroes P(t = T-1, 0); SF zeroes P(0, mu >= 1) and all
// momenta of t = T-2 and T-1
__global__ void k_mom_bcs(double *mom, Geom g, int ng) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  const int id = (int)(t >> 2), mu = (int)(t & 3);
  int c[4];
  coords_of(g, id, c);
  const int T = g.dim[0];
  bool zero = false;
  if (g.bc == YG_BC_OPEN) zero = (c[0] == T - 1 && mu == 0);
  else if (g.bc == YG_BC_SF) zero = (c[0] == 0 && mu >= 1) || c[0] == T - 2 || c[0] == T - 1;
  if (zero)
    for (int a = 0; a < ng; a++) mom[(4L * id + mu) * ng + a] = 0.0;
}

// per-site sum over mu and a of P^2
__global__ void k_mom_sqnorm(double *out, const double *mom, int V, int ng) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= V) return;
  double s = 0;
  for (int k = 0; k < 4 * ng; k++) {
    const double v = mom[(long)id * 4 * ng + k];
    s = fma(v, v, s);
  }
  out[id] = s;
}

// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC11): ten rounds of two 32x32->64 multiplications with
// the round keys bumped by the Weyl constants
__device__ __forceinline__ uint4 philox4x32(uint4 ctr, uint2 key) {
  const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    const unsigned hi0 = __umulhi(M0, ctr.x), lo0 = M0 * ctr.x;
    const unsigned hi1 = __umulhi(M1, ctr.z), lo1 = M1 * ctr.z;
    ctr = make_uint4(hi1 ^ ctr.y ^ key.x, lo1, hi0 ^ ctr.w ^ key.y, lo0);
    key.x += W0;
    key.y += W1;
  }
  return ctr;
}

// uniform in (0, 1] from 32 random bits
__device__ __forceinline__ double u01(unsigned v) { return (v + 1.0) * (1.0 / 4294967296.0); }

// momentum(id,mu).random(): every algebra component Gaussian with standard deviation
// 1/sqrt(2) (rand_gaussian, random.h:15), by Box-Muller on Philox output keyed by the seed
// and counted by (link, component pair)
__global__ void k_mom_gaussian(double *mom, long nlinks, int ng, unsigned long long seed) {
  long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= nlinks) return;
  const uint2 key = make_uint2((unsigned)seed, (unsigned)(seed >> 32));
  for (int a = 0; a < ng; a += 2) {
    const uint4 r = philox4x32(make_uint4((unsigned)t, (unsigned)(t >> 32), (unsigned)a, 0x4d4f4d21u), key);
    const double rad = sqrt(-log(u01(r.x)));           // sqrt(-2 ln u) / sqrt(2)
    double s, c;
    sincospi(2.0 * u01(r.y), &s, &c);
    mom[t * ng + a] = rad * c;
    if (a + 1 < ng) mom[t * ng + a + 1] = rad * s;
  }
}

// ------------------------------------------------------------------ host side
template <int N>
static void launch_gauge_force(Lattice &L, double coeff, double c0, double c1, bool improved) {
  const long n = 4L * L.V;
  if (improved)
    k_gauge_force<N, 1><<<nblk(n, 64), 64, 0, L.stream>>>(L.mom.as<double>(), L.fund.as<double2>(), L.g, L.rt.itfund,
                                                           coeff, c0, c1);
  else
    k_gauge_force<N, 0><<<nblk(n, 64), 64, 0, L.stream>>>(L.mom.as<double>(), L.fund.as<double2>(), L.g, L.rt.itfund,
                                                           coeff, 1.0, 0.0);
  YG_LAUNCHED();
}

#define YG_GAUGE_N(NCV, ...)                                                                 \
  do {                                                                                       \
    if (NCV == 2) { constexpr int GN = 2; __VA_ARGS__; }                                     \
    else if (NCV == 3) { constexpr int GN = 3; __VA_ARGS__; }                                \
    else if (NCV == 4) { constexpr int GN = 4; __VA_ARGS__; }                                \
    else throw Error(YG_ERR_ARG, "gauge kernels are built for N = 2, 3, 4");                 \
  } while (0)

// wilson_gauge_force, forces.cpp:262-283
void wilson_gauge_force(Lattice &L, double dt, double beta) {
  YG_GAUGE_N(L.nc, launch_gauge_force<GN>(L, dt * (beta / L.nc), 1.0, 0.0, false));
}

// improved_gauge_force, forces.cpp:285-309
void improved_gauge_force(Lattice &L, double dt, double beta, double c0, double c1) {
  YG_GAUGE_N(L.nc, launch_gauge_force<GN>(L, dt * (beta / L.nc), c0, c1, true));
}

// the global `volume` of the gauge action (bcs.cpp:32, 76)
static double gauge_volume(const Lattice &L) {
  const long v3 = L.V / L.p.dims[0];
  if (L.p.bc == YG_BC_OPEN) return (double)(L.p.dims[0] - 1) * v3;
  if (L.p.bc == YG_BC_SF) return (double)(L.p.dims[0] - 2) * v3;
  return (double)L.V;
}

// avr_wilson, wilsonloop.cpp:116-133
double avr_wilson(Lattice &L, int height, int width) {
  if (height < 1 || width < 1 || height > 8 || width > 8) throw Error(YG_ERR_ARG, "loop extent must be 1..8");
  double *tmp = L.scratch_field(0);
  YG_GAUGE_N(L.nc, k_wilson_loops<GN><<<nblk(L.V, 128), 128, 0, L.stream>>>(tmp, L.fund.as<double2>(), L.g, height,
                                                                            width));
  YG_LAUNCHED();
  return sum_device(L, tmp, L.V) / (L.nc * 6.0 * gauge_volume(L));
}

double avr_plaquette(Lattice &L) { return avr_wilson(L, 1, 1); }

// MonomialGauge::action, monomials/gauge.cpp:21-40 (c1 = (1 - c0)/8)
double gauge_action(Lattice &L, double beta, double c0) {
  const double c1 = (1.0 - c0) / 8.0;
  double v;
  if (std::fabs(c1) > 1e-8) v = c0 * avr_wilson(L, 1, 1) + c1 * (avr_wilson(L, 2, 1) + avr_wilson(L, 1, 2));
  else v = avr_wilson(L, 1, 1);
  return -beta * v * 6.0 * gauge_volume(L);
}

static void momenta_bcs(Lattice &L) {
  if (L.p.bc != YG_BC_OPEN && L.p.bc != YG_BC_SF) return;
  k_mom_bcs<<<nblk(4L * L.V, 128), 128, 0, L.stream>>>(L.mom.as<double>(), L.g, L.ng);
  YG_LAUNCHED();
}

// the SF boundary fields C1, C2 = diag exp(i v_k / L) (bcs.cpp:211-245)
static SFLinks sf_links(const Lattice &L) {
  SFLinks s{};
  if (L.p.bc != YG_BC_SF) return s;
  double v1[3], v2[3], len;
  if (L.nc == 2) {
    v1[0] = -M_PI; v1[1] = M_PI; v2[0] = -3 * M_PI; v2[1] = 3 * M_PI; len = 4.0 * L.p.dims[1];
  } else if (L.nc == 3) {
    v1[0] = -M_PI; v1[1] = 0; v1[2] = M_PI; v2[0] = -5 * M_PI; v2[1] = 2 * M_PI; v2[2] = 3 * M_PI;
    len = 6.0 * L.p.dims[1];
  } else {
    throw Error(YG_ERR_ARG, "SF boundary fields exist for N = 2 and 3");
  }
  for (int i = 0; i < L.nc; i++) {
    s.c1[i] = make_double2(std::cos(v1[i] / len), std::sin(v1[i] / len));
    s.c2[i] = make_double2(std::cos(v2[i] / len), std::sin(v2[i] / len));
  }
  return s;
}

// update_links, update.cpp:228-247: the represented field is left to represent_gauge_field
void update_links(Lattice &L, double eps) {
  momenta_bcs(L);
  const SFLinks sf = sf_links(L);
  YG_GAUGE_N(L.nc, k_update_links<GN><<<nblk(4L * L.V, 64), 64, 0, L.stream>>>(L.fund.as<double2>(),
                                                                               L.mom.as<double>(), L.g, eps, sf));
  YG_LAUNCHED();
}

// apply_bcs_on_gauge_field, bcs.cpp:201-262 (nothing to do for periodic / antiperiodic)
void apply_gauge_bcs(Lattice &L) {
  if (L.p.bc != YG_BC_OPEN && L.p.bc != YG_BC_SF) return;
  const SFLinks sf = sf_links(L);
  YG_GAUGE_N(L.nc, k_gauge_bcs<GN><<<nblk(4L * L.V, 64), 64, 0, L.stream>>>(L.fund.as<double2>(), L.g, sf));
  YG_LAUNCHED();
}

// reunitarize, update.cpp:269-279
void reunitarize(Lattice &L) {
  YG_GAUGE_N(L.nc, k_reunitarize<GN><<<nblk(4L * L.V, 64), 64, 0, L.stream>>>(L.fund.as<double2>(), L.g));
  YG_LAUNCHED();
}

// reset_variables, momentum part (update.cpp:254-267)
void momenta_gaussian(Lattice &L, unsigned long long seed) {
  k_mom_gaussian<<<nblk(4L * L.V, 128), 128, 0, L.stream>>>(L.mom.as<double>(), 4L * L.V, L.ng, seed);
  YG_LAUNCHED();
}

// hamiltonian(), momentum part (update.cpp:201-220): (TF/2) sum P^2 after the momentum
// boundary conditions (applied in place, as there); TF = 2
double momenta_action(Lattice &L) {
  momenta_bcs(L);
  double *tmp = L.scratch_field(0);
  k_mom_sqnorm<<<nblk(L.V, 128), 128, 0, L.stream>>>(tmp, L.mom.as<double>(), (int)L.V, L.ng);
  YG_LAUNCHED();
  return 2.0 / 2.0 * sum_device(L, tmp, L.V);
}

// gauge_field_backup / gauge_field_restore, gaugefield.cpp:32-42
void gauge_backup(Lattice &L) {
  L.fund_backup.alloc(L.fund.bytes);
  YG_CUDA(cudaMemcpyAsync(L.fund_backup.p, L.fund.p, L.fund.bytes, cudaMemcpyDeviceToDevice, L.stream));
}

void gauge_restore(Lattice &L) {
  if (!L.fund_backup.p) throw Error(YG_ERR_ARG, "no gauge field backup");
  YG_CUDA(cudaMemcpyAsync(L.fund.p, L.fund_backup.p, L.fund.bytes, cudaMemcpyDeviceToDevice, L.stream));
}

// ------------------------------------------------------------------ Wilson and fermion flow
// observables/wilsonflow.cpp:8-157 (the gradient flow of the Wilson action, third-order
// Runge-Kutta, with the plaquette and clover energy densities and the clover charge) and
// observables/fermionflow.cpp:11-97 (fields flowed with the gauge-covariant Laplacian).

__global__ void k_scale(double *v, long n, double s) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) v[i] *= s;
}

// clover_fund(id, mu, nu), wilsonloop.cpp:33-54: the four plaquette leaves at x, summed
template <int N>
__device__ __noinline__ void clover_fund(double2 (&C)[N * N], const double2 *U, const Geom &g, const Pos &x, int mu, int nu) {
  double2 A[N * N], B[N * N], P[N * N], Q[N * N];
  const Pos xm = step(g, x, mu, +1), xn = step(g, x, nu, +1);
  const Pos bm = step(g, x, mu, -1), bn = step(g, x, nu, -1);
  const Pos bmn = step(g, bm, nu, +1), bmbn = step(g, bm, nu, -1), bnm = step(g, bn, mu, +1);
  // U(x,mu) U(x+mu,nu) [U(x,nu) U(x+nu,mu)]^dag
  ldU<N>(A, U, g, x, mu); ldU<N>(B, U, g, xm, nu); mat_mul<N>(P, A, B);
  ldU<N>(A, U, g, x, nu); ldU<N>(B, U, g, xn, mu); mat_mul<N>(Q, A, B);
  mul_dag<N>(C, P, Q);
  // U(x,nu) [U(x-mu,nu) U(x-mu+nu,mu)]^dag U(x-mu,mu)
  ldU<N>(A, U, g, bm, nu); ldU<N>(B, U, g, bmn, mu); mat_mul<N>(Q, A, B);
  ldU<N>(A, U, g, x, nu); mul_dag<N>(P, A, Q);
  ldU<N>(A, U, g, bm, mu); mat_mul<N>(Q, P, A);
#pragma unroll
  for (int k = 0; k < N * N; k++) C[k] = make_double2(C[k].x + Q[k].x, C[k].y + Q[k].y);
  // [U(x-mu-nu,nu) U(x-mu,mu)]^dag U(x-mu-nu,mu) U(x-nu,nu)
  ldU<N>(A, U, g, bmbn, nu); ldU<N>(B, U, g, bm, mu); mat_mul<N>(P, A, B);
  ldU<N>(A, U, g, bmbn, mu); dag_mul<N>(Q, P, A);
  ldU<N>(A, U, g, bn, nu); mat_mul<N>(P, Q, A);
#pragma unroll
  for (int k = 0; k < N * N; k++) C[k] = make_double2(C[k].x + P[k].x, C[k].y + P[k].y);
  // U(x-nu,nu)^dag U(x-nu,mu) U(x-nu+mu,nu) U(x,mu)^dag
  ldU<N>(A, U, g, bn, nu); ldU<N>(B, U, g, bn, mu); dag_mul<N>(P, A, B);
  ldU<N>(A, U, g, bnm, nu); mat_mul<N>(Q, P, A);
  ldU<N>(A, U, g, x, mu); mul_dag<N>(P, Q, A);
#pragma unroll
  for (int k = 0; k < N * N; k++) C[k] = make_double2(C[k].x + P[k].x, C[k].y + P[k].y);
}

// algebra_project(clover_fund(x, mu, nu), sqrt(2 TF)) into av
template <int N>
__device__ __forceinline__ void clover_algebra(double (&av)[N * N - 1], const double2 *U, const Geom &g, const Pos &x,
                                               int mu, int nu, const double2 *itfund) {
  double2 C[N * N];
  clover_fund<N>(C, U, g, x, mu, nu);
#pragma unroll
  for (int a = 0; a < N * N - 1; a++) av[a] = 0.0;
  project_add<N>(av, C, itfund, N * N - 1, 2.0);      // sqrt(2 TF) = 2
}

// per-site terms of wf_e_plaq (sum of N - w Re tr P over the six planes), wf_e_sym (sum of
// |algebra_project(clover, sqrt(2 TF))|^2 over the six planes) and wf_charge (the three
// products of dual planes): out[id], out[V + id], out[2V + id]
template <int N>
__global__ void __launch_bounds__(64) k_wf_densities(double *out, const double2 *U, Geom g, const double2 *itfund) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= g.V) return;
  const Pos x = pos_of(g, id);
  double ep = 0.0, es = 0.0, tc = 0.0;
#pragma unroll 1
  for (int mu = 1; mu < 4; mu++)
#pragma unroll 1
    for (int nu = 0; nu < mu; nu++) {
      ep += N - wilson_loop<N>(U, g, x, mu, nu, 1, 1);
      double av[N * N - 1];
      clover_algebra<N>(av, U, g, x, mu, nu, itfund);
#pragma unroll
      for (int a = 0; a < N * N - 1; a++) es += av[a] * av[a];
    }
  const int pairs[3][4] = {{0, 3, 1, 2}, {0, 2, 3, 1}, {0, 1, 2, 3}};
#pragma unroll 1
  for (int k = 0; k < 3; k++) {
    double a1[N * N - 1], a2[N * N - 1];
    clover_algebra<N>(a1, U, g, x, pairs[k][0], pairs[k][1], itfund);
    clover_algebra<N>(a2, U, g, x, pairs[k][2], pairs[k][3], itfund);
#pragma unroll
    for (int a = 0; a < N * N - 1; a++) tc += a1[a] * a2[a];
  }
  out[id] = ep;
  out[(long)g.V + id] = es;
  out[2L * g.V + id] = tc;
}

// wf_laplacian, fermionflow.cpp:11-26: dst(x) = -8 src(x) + sum_mu U(x,mu) src(x+mu)
// + U(x-mu,mu)^dag src(x-mu) with the represented links, on every site; one thread per
// (site, spin)
template <int D>
__global__ void __launch_bounds__(128) k_wf_laplacian(double2 *dst, const double2 *src, const double2 *U, Geom g) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= 4L * g.V) return;
  const int id = (int)(t >> 2), sp = (int)(t & 3);
  int c[4];
  coords_of(g, id, c);
  double2 acc[D], v[D];
#pragma unroll
  for (int i = 0; i < D; i++) {
    const double2 s = src[fidx(g, id, sp * D + i, 4 * D)];
    acc[i] = make_double2(-8.0 * s.x, -8.0 * s.y);
  }
#pragma unroll 1
  for (int mu = 0; mu < 4; mu++) {
    const int fw = neighbour(g, c, mu, +1), bk = neighbour(g, c, mu, -1);
#pragma unroll
    for (int j = 0; j < D; j++) v[j] = src[fidx(g, fw, sp * D + j, 4 * D)];
#pragma unroll
    for (int i = 0; i < D; i++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int j = 0; j < D; j++) cfma(s, U[fidx(g, id, mu * D * D + i * D + j, 4 * D * D)], v[j]);
      acc[i] = make_double2(acc[i].x + s.x, acc[i].y + s.y);
    }
#pragma unroll
    for (int j = 0; j < D; j++) v[j] = src[fidx(g, bk, sp * D + j, 4 * D)];
#pragma unroll
    for (int i = 0; i < D; i++) {
      double2 s = make_double2(0, 0);
#pragma unroll
      for (int j = 0; j < D; j++) cfmac(s, U[fidx(g, bk, mu * D * D + j * D + i, 4 * D * D)], v[j]);
      acc[i] = make_double2(acc[i].x + s.x, acc[i].y + s.y);
    }
  }
#pragma unroll
  for (int i = 0; i < D; i++) dst[fidx(g, id, sp * D + i, 4 * D)] = acc[i];
}

template <int D>
static void launch_wf_laplacian(Lattice &L, double *dst, const double *src) {
  k_wf_laplacian<D><<<nblk(4L * L.V, 128), 128, 0, L.stream>>>((double2 *)dst, (const double2 *)src,
                                                                L.links.as<double2>(), L.g);
}

// wf_init, wilsonflow.cpp:149-157
void wf_init(Lattice &L) { YG_CUDA(cudaMemsetAsync(L.mom.p, 0, L.mom.bytes, L.stream)); }

// wf_zeta, wilsonflow.cpp:8-23: P -= algebra_project(U staple, alpha), which is
// wilson_gauge_force with dt = alpha and beta = N
void wf_zeta(Lattice &L, double alpha) { wilson_gauge_force(L, alpha, (double)L.nc); }

// wf_update, wilsonflow.cpp:25-41: U <- exp(P) U (no momentum boundary conditions), then
// P <- val P; the boundary links take their fixed values
void wf_update(Lattice &L, double val) {
  const SFLinks sf = sf_links(L);
  YG_GAUGE_N(L.nc, k_update_links<GN><<<nblk(4L * L.V, 64), 64, 0, L.stream>>>(L.fund.as<double2>(),
                                                                               L.mom.as<double>(), L.g, 1.0, sf));
  YG_LAUNCHED();
  const long n = 4L * L.V * L.ng;
  k_scale<<<nblk(n, 256) < 1184 ? nblk(n, 256) : 1184, 256, 0, L.stream>>>(L.mom.as<double>(), n, val);
  YG_LAUNCHED();
}

// wf_iterate, wilsonflow.cpp:43-53: one Runge-Kutta step of size eps
void wf_iterate(Lattice &L, double eps) {
  wf_zeta(L, eps / 4.0);
  wf_update(L, -17.0 / 9.0);
  wf_zeta(L, 8.0 * eps / 9.0);
  wf_update(L, -1.0);
  wf_zeta(L, 3.0 * eps / 4.0);
  wf_update(L, 0.0);
}

// wf_e_plaq, wf_e_sym, wf_charge (wilsonflow.cpp:55-147) from one pass over the sites
void wf_observables(Lattice &L, double *e_plaq, double *e_sym, double *charge) {
  double *tmp = L.scratch_field(kFlowDensities);
  YG_GAUGE_N(L.nc, k_wf_densities<GN><<<nblk(L.V, 64), 64, 0, L.stream>>>(tmp, L.fund.as<double2>(), L.g, L.rt.itfund));
  YG_LAUNCHED();
  const double V = (double)L.V;
  const double ep = sum_device(L, tmp, L.V), es = sum_device(L, tmp + L.V, L.V), tc = sum_device(L, tmp + 2 * L.V, L.V);
  if (e_plaq) *e_plaq = 2 * ep / V;
  if (e_sym) *e_sym = (2 * es) / (16 * 4 * V);
  if (charge) *charge = (2 * tc) / (16 * 16 * M_PI * M_PI);
}

// wf_laplacian on the represented links
void wf_laplacian(Lattice &L, double *dst, const double *src) {
  switch (L.d) {
    case 1: launch_wf_laplacian<1>(L, dst, src); break;
    case 2: launch_wf_laplacian<2>(L, dst, src); break;
    case 3: launch_wf_laplacian<3>(L, dst, src); break;
    case 4: launch_wf_laplacian<4>(L, dst, src); break;
    case 6: launch_wf_laplacian<6>(L, dst, src); break;
    case 8: launch_wf_laplacian<8>(L, dst, src); break;
    case 10: launch_wf_laplacian<10>(L, dst, src); break;
    case 15: launch_wf_laplacian<15>(L, dst, src); break;
    default: throw Error(YG_ERR_ARG, "unsupported representation dimension");
  }
  YG_LAUNCHED();
}

// wf_fermion_init, fermionflow.cpp:76-92: the stage fields start at zero, the momenta too
void wf_fermion_init(Lattice &L, int n) {
  if (n < 1 || n > kFlowMaxFields) throw Error(YG_ERR_ARG, "1..32 flowed fields");
  for (int i = 0; i < n; i++) {
    blas_zero(L, L.scratch_field(kFlowPhi1 + i), 0, L.V);
    blas_zero(L, L.scratch_field(kFlowPhi2 + i), 0, L.V);
  }
  wf_init(L);
}

// wf_fermion_iterate, fermionflow.cpp:28-74: the fields phi0[i] and the gauge field flow
// together.  As in the reference, spinor_copy copies whole fields (linalg.cpp:71-76) while
// the other vector updates cover the default view (the even sites with even-odd
// preconditioning); the Laplacian covers all sites.
void wf_fermion_iterate(Lattice &L, double eps, double *const *phi0, int n) {
  if (n < 1 || n > kFlowMaxFields) throw Error(YG_ERR_ARG, "1..32 flowed fields");
  long lo, cnt;
  L.view_range(YG_VIEW_DEFAULT, lo, cnt);
  double *dphi = L.scratch_field(kFlowDphi);
  const double2 one = make_double2(1, 0), zero = make_double2(0, 0);
  auto re = [](double v) { return make_double2(v, 0); };
  represent_and_clover(L);
  for (int i = 0; i < n; i++) {
    double *p1 = L.scratch_field(kFlowPhi1 + i);
    wf_laplacian(L, dphi, phi0[i]);
    blas_copy(L, p1, phi0[i]);
    blas_axpby(L, p1, one, re(eps / 4.0), dphi, lo, cnt);
  }
  wf_zeta(L, eps / 4.0);
  wf_update(L, -17.0 / 9.0);
  represent_and_clover(L);
  for (int i = 0; i < n; i++) {
    double *p1 = L.scratch_field(kFlowPhi1 + i), *p2 = L.scratch_field(kFlowPhi2 + i);
    wf_laplacian(L, dphi, p1);
    blas_axpby(L, p2, zero, re(-8.0 / 9.0), p1, lo, cnt);
    blas_axpby(L, p2, one, re(17.0 / 9.0), phi0[i], lo, cnt);
    blas_axpby(L, p2, one, re(8.0 * eps / 9.0), dphi, lo, cnt);
  }
  wf_zeta(L, 8.0 * eps / 9.0);
  wf_update(L, -1.0);
  represent_and_clover(L);
  for (int i = 0; i < n; i++) {
    double *p1 = L.scratch_field(kFlowPhi1 + i), *p2 = L.scratch_field(kFlowPhi2 + i);
    wf_laplacian(L, dphi, p2);
    blas_copy(L, phi0[i], p1);
    blas_axpby(L, phi0[i], one, re(3.0 * eps / 4.0), dphi, lo, cnt);
  }
  wf_zeta(L, 3.0 * eps / 4.0);
  wf_update(L, 0.0);
}

}  // namespace yg
