// Explicit instantiations of the Coulomb passes for a group of FFT lengths
// (split across files so that nvcc compiles them in parallel).
#include "coulomb_kernels.cuh"
namespace sincgpu {
SINCGPU_INSTANTIATE_LAUNCH(240, 16, 15)
SINCGPU_INSTANTIATE_LAUNCH(256, 16, 16)
}  // namespace sincgpu
