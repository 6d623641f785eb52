/* pair_tensormd_b200.h -- LAMMPS pair style "tensormd/b200".
 *
 * Same input grammar as pair_style tensormd (src/ML-TENSORMD/pair_tensormd.h:16-83):
 *   pair_style tensormd/b200
 *   pair_coeff * * file.npz El1 El2 ... [interp dx] [cmax exact|default]
 *              [precision fp32|tf32x3|bf16|bf16x3|fp8]
 * The force evaluation runs in libtmd_b200.so (include/tmd_b200.h), which
 * builds its own neighbor list.  On one MPI rank the device handles the
 * periodic images and the style writes forces on local atoms; on several
 * ranks it hands local and ghost atoms over and writes forces on both, for
 * LAMMPS's reverse communication.
 */
#ifdef PAIR_CLASS
// clang-format off
PairStyle(tensormd/b200,PairTensorMDB200);
// clang-format on
#else

#ifndef LMP_PAIR_TENSORMD_B200_H
#define LMP_PAIR_TENSORMD_B200_H

#include "pair.h"

#include <string>
#include <vector>

struct tmd_model;
struct tmd_system;

namespace LAMMPS_NS {

class PairTensorMDB200 : public Pair {
 public:
  PairTensorMDB200(class LAMMPS *);
  ~PairTensorMDB200() override;
  void compute(int, int) override;
  void settings(int, char **) override;
  void coeff(int, char **) override;
  void init_style() override;
  double init_one(int, int) override;
  void *extract(const char *, int &) override;
  double memory_usage() override;

  // compute tensormd/density/b200: G rows of the local atoms at the current
  // positions (G[nlocal][descriptor_width()])
  int descriptor_width();
  void descriptors(double *G);

  // temperature-dependent potentials (tdnp = 1), as PairTensorMD: the
  // electron temperature in eV (pair_coeff etemp, fix tensormd/etemp through
  // extract("etemp")), and the entropy and free energy of the last compute
  double etemp, eentropy, free_energy;

 private:
  tmd_model *model;
  tmd_system *sys;
  double cutmax;
  double skin;
  double **scale;
  int natoms_cap;
  int last_nlocal, last_nall;
  bool ghost_mode;
  int last_box_stamp;
  double last_etemp;
  double last_box[9];
  std::vector<double> xbuf, fbuf, ebuf, vbuf;
  std::vector<int> tbuf;

  void allocate();
  void check(int rc, const char *what);
  void upload();
};

}    // namespace LAMMPS_NS

#endif
#endif
