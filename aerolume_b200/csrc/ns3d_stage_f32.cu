// The float instantiations of the 3D eddy-viscosity and stage kernels.
#include "ns3d_stage.cuh"

namespace aero {

template size_t stage_smem_bytes<float>();
template cudaError_t launch_stage<float>(const StageParams<float> &, cudaStream_t);
template cudaError_t launch_nu<float>(const NuParams<float> &, cudaStream_t);

}  // namespace aero
