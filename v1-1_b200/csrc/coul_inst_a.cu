// Explicit instantiations of the Coulomb passes for a group of FFT lengths
// (split across files so that nvcc compiles them in parallel).
#include "coulomb_kernels.cuh"
namespace sincgpu {
SINCGPU_INSTANTIATE_LAUNCH(16, 4, 4)
SINCGPU_INSTANTIATE_LAUNCH(20, 5, 4)
SINCGPU_INSTANTIATE_LAUNCH(24, 6, 4)
SINCGPU_INSTANTIATE_LAUNCH(27, 9, 3)
SINCGPU_INSTANTIATE_LAUNCH(32, 8, 4)
SINCGPU_INSTANTIATE_LAUNCH(36, 6, 6)
}  // namespace sincgpu
