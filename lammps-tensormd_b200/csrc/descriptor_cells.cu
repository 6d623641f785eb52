// descriptor_cells.cu -- descriptor kernels of multi-cell batches (each
// atom's images use the box of its own cell), one radial kind per function.
#include "descriptor_impl.cuh"

namespace tmd {
void launch_descriptor_gauss_cells(const DescArgs &a, cudaStream_t st) {
  launch_descriptor_rk<kRadGauss, true>(a, st);
}
}  // namespace tmd
