// Instantiation unit: Dirac-operator kernels of representation dimension d = 6
// (declarations in yg_kernels.h, device code in yg_dirac_impl.cuh).
#include "yg_dirac_impl.cuh"

namespace yg {
template void DK<6>::hop(const HopArgs<double> &, int, cudaStream_t);
template void DK<6>::hop(const HopArgs<float> &, int, cudaStream_t);
template void DK<6>::clover(double2 *, const double2 *, const double2 *, Geom, double, double, int, int, int, cudaStream_t);
template void DK<6>::clover_inv(double2 *, const double2 *, const double2 *, Geom, int, cudaStream_t);
template void DK<6>::ldl(double2 *, const double2 *, Geom, double, double, int, cudaStream_t);
template void DK<6>::cinv_float(float2 *, const double2 *, int, cudaStream_t);
template void DK<6>::cinv_packed64(double2 *, const double2 *, int, cudaStream_t);
template void DK<6>::logdet(double *, const double2 *, int, cudaStream_t);
}  // namespace yg
