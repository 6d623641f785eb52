// descriptor.cu -- dispatch of the descriptor kernel on the radial kind and
// the box mode.  The single-box Gaussian kind is instantiated here; the other
// variants live in descriptor_table.cu, descriptor_generic.cu,
// descriptor_cells.cu and descriptor_cells_other.cu (parallel builds).
#include "descriptor_impl.cuh"

namespace tmd {

void launch_descriptor_table(const DescArgs &a, cudaStream_t st);
void launch_descriptor_generic(const DescArgs &a, cudaStream_t st);
void launch_descriptor_gauss_cells(const DescArgs &a, cudaStream_t st);
void launch_descriptor_table_cells(const DescArgs &a, cudaStream_t st);
void launch_descriptor_generic_cells(const DescArgs &a, cudaStream_t st);

void launch_descriptor(const DescArgs &a, cudaStream_t st, long &launches) {
  const bool cells = a.cbox != nullptr;
  switch (radial_kind(a.kp)) {
    case kRadTable:
      if (cells) launch_descriptor_table_cells(a, st); else launch_descriptor_table(a, st);
      break;
    case kRadGauss:
      if (cells) launch_descriptor_gauss_cells(a, st); else launch_descriptor_rk<kRadGauss, false>(a, st);
      break;
    default:
      if (cells) launch_descriptor_generic_cells(a, st); else launch_descriptor_generic(a, st);
      break;
  }
  if (a.variant == kDescSplit) {
    launches += 2;  // k_pair_geo + k_descriptor_c (G formed inside)
  } else if (a.variant != kDescFilter4) {
    launches += 1;  // G formed inside k_descriptor_w
  } else {
    launch_invariants(a, st);
    launches += 2;
  }
}

}  // namespace tmd
