// Host orchestration of the fermion forces (forces.cpp) and of the gauge-side support
// (wilson_gauge_force, plaquette, clover logdet); device code in yg_forces_impl.cuh.
#include <cmath>
#include <vector>
#include "yg_lattice.h"
#include "yg_kernels.h"

namespace yg {

void clover_fermion_force(Lattice &L, double residue, double *lhs, double *rhs) {
  if (!L.p.clover) return;
  YG_DISPATCH_D(L.d, K::clover_fermion_force(L.cl_force.as<double2>(), (const double2 *)lhs, (const double2 *)rhs,
                                             L.g, residue, L.stream));
  YG_LAUNCHED();
}

// wilson_fermion_force, forces.cpp:175-227
void wilson_fermion_force(Lattice &L, double dt, double mass, double residue, double *lhs, double *rhs) {
  double coeff = dt * residue;
  if (L.p.eo) {
    hop(L, rhs, rhs, 2, 1.0, false);      // Dphi_oe(rhs, rhs)
    hop(L, lhs, lhs, 2, 1.0, false);
    if (L.p.clover) {
      clover_inv_apply(L, mass, rhs, rhs, 2, false);    // Dphi_oo_inv(mass, rhs, rhs)
      clover_inv_apply(L, mass, lhs, lhs, 2, false);
    }
    coeff = -coeff;
  }
  if (L.p.clover) clover_fermion_force(L, residue, lhs, rhs);
  YG_DISPATCH_D(L.d, K::hopping_force(L.mom.as<double>(), (const double2 *)lhs, (const double2 *)rhs,
                                      L.links.as<double2>(), L.g, L.rt.itrepr, L.ng, coeff, L.stream));
  YG_LAUNCHED();
}

// wilson_fermion_force_q, forces.cpp:230-236
void wilson_fermion_force_q(Lattice &L, double dt, double mass, double residue, double *rhs) {
  double *tmp = L.scratch_field(9);
  hphi(L, mass, tmp, rhs);
  wilson_fermion_force(L, dt, mass, residue, tmp, rhs);
}

// the loop of MonomialRHMC::update (rhmc.cpp:100-103) over the poles of a rational
// approximation, as one batched force: for every pole n the fields of
// wilson_fermion_force_q(dt, mass, residue_n, rhs_n) are formed (tmp_n = Hphi rhs_n, and with
// even-odd preconditioning the odd halves of both replaced by A_oo^-1 H_oe, in place like the
// reference), then the clover force and the hopping force of all poles are summed in one
// launch each, reading the links and writing cl_force and the momenta once
static constexpr int kPoleSlot = 400;   // scratch fields kPoleSlot .. kPoleSlot + n - 1

void wilson_fermion_force_q_multi(Lattice &L, double dt, double mass, int n, const double *residue,
                                  double *const *rhs) {
  if (n < 1 || n > kMaxPoles) throw Error(YG_ERR_ARG, "1..32 poles");
  PoleSet ps{};
  ps.n = n;
  for (int k = 0; k < n; k++) {
    double *tmp = L.scratch_field(kPoleSlot + k);
    hphi(L, mass, tmp, rhs[k]);
    if (L.p.eo) {
      hop(L, rhs[k], rhs[k], 2, 1.0, false);
      hop(L, tmp, tmp, 2, 1.0, false);
      if (L.p.clover) {
        clover_inv_apply(L, mass, rhs[k], rhs[k], 2, false);
        clover_inv_apply(L, mass, tmp, tmp, 2, false);
      }
    }
    ps.lhs[k] = (const double2 *)tmp;
    ps.rhs[k] = (const double2 *)rhs[k];
  }
  if (L.p.clover) {
    for (int k = 0; k < n; k++) ps.w[k] = residue[k];
    YG_DISPATCH_D(L.d, K::clover_fermion_force_multi(L.cl_force.as<double2>(), ps, L.g, L.stream));
    YG_LAUNCHED();
  }
  for (int k = 0; k < n; k++) ps.w[k] = (L.p.eo ? -1.0 : 1.0) * dt * residue[k];
  YG_DISPATCH_D(L.d, K::hopping_force_multi(L.mom.as<double>(), ps, L.links.as<double2>(), L.g, L.rt.itrepr, L.ng,
                                            L.stream));
  YG_LAUNCHED();
}

void begin_fermion_force(Lattice &L) {
  if (!L.p.clover) return;
  YG_CUDA(cudaMemsetAsync(L.cl_force.p, 0, L.cl_force.bytes, L.stream));
}

void clover_logdet_force(Lattice &L, double mass, double residue) {
  if (!L.p.clover) return;
  ensure_ldl(L, 4.0 + mass);
  YG_DISPATCH_D(L.d, K::clover_ldl_force(L.cl_force.as<double2>(), L.ldl.as<double2>(), L.g, residue, L.stream));
  YG_LAUNCHED();
}

void end_fermion_force(Lattice &L, double dt) {
  if (!L.p.clover) return;
  double coeff = L.p.csw * dt / 8.0;
  YG_DISPATCH_D(L.d, K::clover_force_core(L.mom.as<double>(), L.cl_force.as<double2>(), L.links.as<double2>(), L.g,
                                          L.rt.itrepr, L.ng, coeff, L.stream));
  YG_LAUNCHED();
}

double clover_logdet(Lattice &L, double mass) {
  if (!L.p.clover) return 0.0;
  ensure_ldl(L, 4.0 + mass);
  double *tmp = L.scratch_field(0);
  YG_DISPATCH_D(L.d, K::logdet(tmp, L.ldl.as<double2>(), (int)L.Vh, L.stream));
  YG_LAUNCHED();
  return sum_device(L, tmp, L.Vh);
}

}  // namespace yg
