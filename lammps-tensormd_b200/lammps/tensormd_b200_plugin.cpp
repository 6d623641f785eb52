/* tensormd_b200_plugin.cpp -- run-time plugin registration of the pair style
 * and of compute tensormd/density/b200 (LAMMPS PLUGIN package,
 * src/lammpsplugin.h).  Load with
 *   plugin load tensormd_b200_plugin.so
 */
#include "lammpsplugin.h"
#include "version.h"

#include "compute_tensormd_density_b200.h"
#include "pair_tensormd_b200.h"

using namespace LAMMPS_NS;

static Pair *tensormd_b200_creator(LAMMPS *lmp)
{
  return new PairTensorMDB200(lmp);
}

static Compute *tensormd_density_b200_creator(LAMMPS *lmp, int argc, char **argv)
{
  return new ComputeTensorMDDensityB200(lmp, argc, argv);
}

extern "C" void lammpsplugin_init(void *lmp, void *handle, void *regfunc)
{
  lammpsplugin_t plugin;
  lammpsplugin_regfunc register_plugin = (lammpsplugin_regfunc) regfunc;
  plugin.version = LAMMPS_VERSION;
  plugin.style = "pair";
  plugin.name = "tensormd/b200";
  plugin.info = "tensor-moment ML potential on B200 (sm_100a)";
  plugin.author = "tmd-b200";
  plugin.creator.v1 = (lammpsplugin_factory1 *) &tensormd_b200_creator;
  plugin.handle = handle;
  (*register_plugin)(&plugin, lmp);

  plugin.style = "compute";
  plugin.name = "tensormd/density/b200";
  plugin.info = "per-atom descriptors of pair_style tensormd/b200";
  plugin.creator.v2 = (lammpsplugin_factory2 *) &tensormd_density_b200_creator;
  (*register_plugin)(&plugin, lmp);
}
