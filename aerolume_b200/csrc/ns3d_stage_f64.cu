// The double instantiations of the 3D eddy-viscosity and stage kernels.
#include "ns3d_stage.cuh"

namespace aero {

template size_t stage_smem_bytes<double>();
template cudaError_t launch_stage<double>(const StageParams<double> &, cudaStream_t);
template cudaError_t launch_nu<double>(const NuParams<double> &, cudaStream_t);

}  // namespace aero
