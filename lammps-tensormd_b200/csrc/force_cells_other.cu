// force_cells_other.cu -- pair-force kernels of multi-cell batches,
// rational-table and power-exponential / Morse / density radial bases.
#include "force_impl.cuh"

namespace tmd {
void launch_force_table_cells(const ForceArgs &a, cudaStream_t st) {
  launch_force_rk<kRadTable, true>(a, st);
}
void launch_force_generic_cells(const ForceArgs &a, cudaStream_t st) {
  launch_force_rk<kRadGeneric, true>(a, st);
}
}  // namespace tmd
