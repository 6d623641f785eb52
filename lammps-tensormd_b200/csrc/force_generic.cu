// force_generic.cu -- pair-force kernel, power-exponential / Morse / density
// radial bases.
#include "force_impl.cuh"

namespace tmd {
void launch_force_generic(const ForceArgs &a, cudaStream_t st) {
  launch_force_rk<kRadGeneric, false>(a, st);
}
}  // namespace tmd
