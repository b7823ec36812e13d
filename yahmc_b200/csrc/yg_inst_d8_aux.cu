// Instantiation unit: force, representation and gauge kernels for d = 8
// (declarations in yg_kernels.h, device code in yg_forces_impl.cuh / yg_repr_impl.cuh).
#include "yg_forces_impl.cuh"
#include "yg_repr_impl.cuh"

namespace yg {
template void DK<8>::clover_fermion_force(double2 *, const double2 *, const double2 *, Geom, double, cudaStream_t);
template void DK<8>::hopping_force(double *, const double2 *, const double2 *, const double2 *, Geom, const double2 *, int, double, cudaStream_t);
template void DK<8>::clover_ldl_force(double2 *, const double2 *, Geom, double, cudaStream_t);
template void DK<8>::clover_fermion_force_multi(double2 *, const PoleSet &, Geom, cudaStream_t);
template void DK<8>::hopping_force_multi(double *, const PoleSet &, const double2 *, Geom, const double2 *, int, cudaStream_t);
template void DK<8>::clover_force_core(double *, const double2 *, const double2 *, Geom, const double2 *, int, double, cudaStream_t);
template struct RK<3, 8>;
}  // namespace yg
