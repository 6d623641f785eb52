// force_cells.cu -- pair-force kernels of multi-cell batches (each atom's
// images use the box of its own cell), Gaussian radial basis.
#include "force_impl.cuh"

namespace tmd {
void launch_force_gauss_cells(const ForceArgs &a, cudaStream_t st) {
  launch_force_rk<kRadGauss, true>(a, st);
}
}  // namespace tmd
