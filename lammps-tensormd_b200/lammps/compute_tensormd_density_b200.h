/* compute_tensormd_density_b200.h -- per-atom descriptors of pair_style
 * tensormd/b200.
 *
 *   compute ID group-ID tensormd/density/b200
 *
 * Same output as compute tensormd/density
 * (src/ML-TENSORMD/compute_tensormd_density.cpp:129-200): a per-atom array
 * with one column per MLP input (b*k*m), row i holding local atom i's G row
 * at the current positions.  The reference builds its own potential and an
 * occasional full list; here the pair style's device system evaluates the
 * descriptor (include/tmd_b200.h, tmd_get_descriptors), so the pair style
 * must be tensormd/b200 and its pair_coeff sets the columns.
 */
#ifdef COMPUTE_CLASS
// clang-format off
ComputeStyle(tensormd/density/b200,ComputeTensorMDDensityB200);
// clang-format on
#else

#ifndef LMP_COMPUTE_TENSORMD_DENSITY_B200_H
#define LMP_COMPUTE_TENSORMD_DENSITY_B200_H

#include "compute.h"

#include <vector>

namespace LAMMPS_NS {

class ComputeTensorMDDensityB200 : public Compute {
 public:
  ComputeTensorMDDensityB200(class LAMMPS *, int, char **);
  ~ComputeTensorMDDensityB200() override;
  void init() override;
  void compute_peratom() override;
  double memory_usage() override;

 private:
  class PairTensorMDB200 *pair;
  int nmax;
  double **G;
  std::vector<double> gbuf;
};

}    // namespace LAMMPS_NS

#endif
#endif
