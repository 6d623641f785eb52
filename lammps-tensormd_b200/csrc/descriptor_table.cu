// descriptor_table.cu -- descriptor kernel, rational-table radial basis.
#include "descriptor_impl.cuh"

namespace tmd {
void launch_descriptor_table(const DescArgs &a, cudaStream_t st) {
  launch_descriptor_rk<kRadTable, false>(a, st);
}
}  // namespace tmd
