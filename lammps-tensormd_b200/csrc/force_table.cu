// force_table.cu -- pair-force kernel, rational-table radial basis.
#include "force_impl.cuh"

namespace tmd {
void launch_force_table(const ForceArgs &a, cudaStream_t st) {
  launch_force_rk<kRadTable, false>(a, st);
}
}  // namespace tmd
