// descriptor_cells_other.cu -- descriptor kernels of multi-cell batches,
// rational-table and power-exponential / Morse / density radial bases.
#include "descriptor_impl.cuh"

namespace tmd {
void launch_descriptor_table_cells(const DescArgs &a, cudaStream_t st) {
  launch_descriptor_rk<kRadTable, true>(a, st);
}
void launch_descriptor_generic_cells(const DescArgs &a, cudaStream_t st) {
  launch_descriptor_rk<kRadGeneric, true>(a, st);
}
}  // namespace tmd
