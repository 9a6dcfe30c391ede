// Explicit instantiations of the Coulomb passes for a group of FFT lengths
// (split across files so that nvcc compiles them in parallel).
#include "coulomb_kernels.cuh"
namespace sincgpu {
SINCGPU_INSTANTIATE_LAUNCH(81, 9, 9)
SINCGPU_INSTANTIATE_LAUNCH(90, 10, 9)
SINCGPU_INSTANTIATE_LAUNCH(100, 10, 10)
SINCGPU_INSTANTIATE_LAUNCH(108, 12, 9)
SINCGPU_INSTANTIATE_LAUNCH(120, 12, 10)
}  // namespace sincgpu
