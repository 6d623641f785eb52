// descriptor_generic.cu -- descriptor kernel, power-exponential / Morse /
// density radial bases.
#include "descriptor_impl.cuh"

namespace tmd {
void launch_descriptor_generic(const DescArgs &a, cudaStream_t st) {
  launch_descriptor_rk<kRadGeneric, false>(a, st);
}
}  // namespace tmd
