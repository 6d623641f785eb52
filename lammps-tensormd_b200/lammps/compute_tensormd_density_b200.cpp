/* compute_tensormd_density_b200.cpp -- compute tensormd/density/b200: the
 * per-atom descriptors G (the MLP input rows) of pair_style tensormd/b200,
 * as compute tensormd/density exports them
 * (src/ML-TENSORMD/compute_tensormd_density.cpp:129-200: array_atom[i][j] =
 * G row of local atom i, column j in b*k*m order; atoms outside the group
 * are zero here, the reference fills every local atom).
 */
#include "compute_tensormd_density_b200.h"

#include "atom.h"
#include "error.h"
#include "force.h"
#include "memory.h"
#include "update.h"

#include "pair_tensormd_b200.h"

#include <cstring>

using namespace LAMMPS_NS;

ComputeTensorMDDensityB200::ComputeTensorMDDensityB200(LAMMPS *lmp, int narg, char **arg) :
    Compute(lmp, narg, arg), pair(nullptr), nmax(0), G(nullptr)
{
  if (narg != 3) error->all(FLERR, "Illegal compute tensormd/density/b200 command");
  pair = dynamic_cast<PairTensorMDB200 *>(force->pair_match("tensormd/b200", 1, 0));
  if (pair == nullptr)
    error->all(FLERR, "compute tensormd/density/b200 requires pair_style tensormd/b200");
  size_peratom_cols = pair->descriptor_width();
  if (size_peratom_cols < 1)
    error->all(FLERR, "compute tensormd/density/b200 needs pair_coeff to be set first");
  peratom_flag = 1;
  timeflag = 1;
}

ComputeTensorMDDensityB200::~ComputeTensorMDDensityB200()
{
  memory->destroy(G);
}

void ComputeTensorMDDensityB200::init()
{
  pair = dynamic_cast<PairTensorMDB200 *>(force->pair_match("tensormd/b200", 1, 0));
  if (pair == nullptr)
    error->all(FLERR, "compute tensormd/density/b200 requires pair_style tensormd/b200");
}

void ComputeTensorMDDensityB200::compute_peratom()
{
  invoked_peratom = update->ntimestep;
  if (atom->nmax > nmax) {
    memory->destroy(G);
    nmax = atom->nmax;
    memory->create(G, nmax, size_peratom_cols, "tensormd/density/b200:G");
    array_atom = G;
  }
  const int nlocal = atom->nlocal;
  const int nc = size_peratom_cols;
  gbuf.resize((size_t)nlocal * nc);
  pair->descriptors(gbuf.data());
  const int *mask = atom->mask;
  for (int i = 0; i < nlocal; i++) {
    if (mask[i] & groupbit)
      std::memcpy(G[i], gbuf.data() + (size_t)i * nc, nc * sizeof(double));
    else
      std::memset(G[i], 0, nc * sizeof(double));
  }
}

double ComputeTensorMDDensityB200::memory_usage()
{
  return (double) nmax * size_peratom_cols * sizeof(double) +
      (double) gbuf.capacity() * sizeof(double);
}
