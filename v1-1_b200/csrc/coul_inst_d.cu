// Explicit instantiations of the Coulomb passes for a group of FFT lengths
// (split across files so that nvcc compiles them in parallel).
#include "coulomb_kernels.cuh"
namespace sincgpu {
SINCGPU_INSTANTIATE_LAUNCH(126, 14, 9)
SINCGPU_INSTANTIATE_LAUNCH(144, 12, 12)
SINCGPU_INSTANTIATE_LAUNCH(162, 18, 9)
}  // namespace sincgpu
