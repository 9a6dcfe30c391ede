// Explicit instantiations of the Coulomb passes for a group of FFT lengths
// (split across files so that nvcc compiles them in parallel).
#include "coulomb_kernels.cuh"
namespace sincgpu {
SINCGPU_INSTANTIATE_LAUNCH(180, 15, 12)
SINCGPU_INSTANTIATE_LAUNCH(192, 16, 12)
SINCGPU_INSTANTIATE_LAUNCH(216, 18, 12)
}  // namespace sincgpu
