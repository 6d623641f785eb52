// descriptor.cu -- dispatch of the descriptor kernel on the radial kind.
// The Gaussian kind is instantiated here; the table and generic analytic kinds
// live in descriptor_table.cu and descriptor_generic.cu (parallel builds).
#include "descriptor_impl.cuh"

namespace tmd {

void launch_descriptor_table(const DescArgs &a, cudaStream_t st);
void launch_descriptor_generic(const DescArgs &a, cudaStream_t st);

void launch_descriptor(const DescArgs &a, cudaStream_t st, long &launches) {
  switch (radial_kind(a.kp)) {
    case kRadTable: launch_descriptor_table(a, st); break;
    case kRadGauss: launch_descriptor_rk<kRadGauss>(a, st); break;
    default: launch_descriptor_generic(a, st); break;
  }
  launches += 1;
}

}  // namespace tmd
