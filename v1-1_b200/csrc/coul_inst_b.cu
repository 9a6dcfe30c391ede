// Explicit instantiations of the Coulomb passes for a group of FFT lengths
// (split across files so that nvcc compiles them in parallel).
#include "coulomb_kernels.cuh"
namespace sincgpu {
SINCGPU_INSTANTIATE_LAUNCH(42, 7, 6)
SINCGPU_INSTANTIATE_LAUNCH(48, 8, 6)
SINCGPU_INSTANTIATE_LAUNCH(54, 9, 6)
SINCGPU_INSTANTIATE_LAUNCH(64, 8, 8)
SINCGPU_INSTANTIATE_LAUNCH(72, 9, 8)
}  // namespace sincgpu
