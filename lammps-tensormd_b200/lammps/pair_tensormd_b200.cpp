/* pair_tensormd_b200.cpp -- LAMMPS pair style "tensormd/b200" over the C ABI
 * of libtmd_b200.so.
 *
 * Mirrors PairTensorMD (src/ML-TENSORMD/pair_tensormd.cpp): settings() takes
 * no arguments (:205-208); coeff() takes "* * file.npz El1 ... [keywords]"
 * (:214-317) and sets the per-type masses from the potential file (:303-312);
 * init_style() requires newton_pair on (:323-330); init_one() returns the
 * cutoff (:336-341); extract("scale") exposes the fix-adapt scale (:415-425),
 * of which compute() uses scale[1][1] for every type, as the reference does
 * (:168-170).  compute() runs in one of two modes:
 *   one MPI rank   the local atoms and the periodic box go to the device,
 *                  which builds its own periodic list (periodic images on the
 *                  device, ghosts unused); forces on local atoms only;
 *   several ranks  the ghost-aware mode: local and ghost atoms go to the
 *                  device (tmd_system_set_atoms_ghost), which evaluates the
 *                  local atoms over the same neighbor set as LAMMPS's full
 *                  list and returns forces on local and ghost atoms, which
 *                  LAMMPS's reverse communication sums (newton_pair on), as
 *                  the reference does (kernel.cu:1760-1789).
 * No LAMMPS neighbor list is requested: the device builds the list itself,
 * and LAMMPS sets its neighbor and ghost cutoff to the pair cutoff + skin
 * whether or not a list is requested (neighbor.cpp:337-376), so the ghost
 * shell the device needs is always there; a full list would cost a host
 * build at every reneighboring for nothing.  The virial comes from the pair
 * separations on the device (no fdotr), energy and virial per rank.
 */
#include "pair_tensormd_b200.h"

#include "atom.h"
#include "comm.h"
#include "domain.h"
#include "error.h"
#include "force.h"
#include "memory.h"
#include "neighbor.h"
#include "utils.h"

#include "tmd_b200.h"

#include <cstring>
#include <string>

using namespace LAMMPS_NS;

PairTensorMDB200::PairTensorMDB200(LAMMPS *lmp) : Pair(lmp)
{
  single_enable = 0;
  restartinfo = 0;
  one_coeff = 1;
  manybody_flag = 1;
  no_virial_fdotr_compute = 1;
  centroidstressflag = CENTROID_NOTAVAIL;
  model = nullptr;
  sys = nullptr;
  cutmax = 0.0;
  skin = 1.0;
  scale = nullptr;
  natoms_cap = 0;
  last_nlocal = -1;
  last_nall = -1;
  last_box_stamp = -1;
  ghost_mode = false;
  etemp = eentropy = free_energy = 0.0;
  last_etemp = -1.0;
}

PairTensorMDB200::~PairTensorMDB200()
{
  if (sys) tmd_system_free(sys);
  if (model) tmd_model_free(model);
  if (allocated) {
    memory->destroy(setflag);
    memory->destroy(cutsq);
    memory->destroy(scale);
  }
}

void PairTensorMDB200::check(int rc, const char *what)
{
  if (rc == TMD_OK) return;
  char buf[512];
  tmd_last_error(buf, sizeof(buf));
  error->one(FLERR, std::string("pair tensormd/b200: ") + what + ": " + buf);
}

void PairTensorMDB200::allocate()
{
  allocated = 1;
  int n = atom->ntypes;
  memory->create(setflag, n + 1, n + 1, "pair:setflag");
  memory->create(cutsq, n + 1, n + 1, "pair:cutsq");
  memory->create(scale, n + 1, n + 1, "pair:scale");
  map = new int[n + 1];
  for (int i = 0; i <= n; i++) map[i] = -1;
}

void PairTensorMDB200::settings(int narg, char ** /*arg*/)
{
  if (narg != 0) error->all(FLERR, "Illegal pair_style command");
}

void PairTensorMDB200::coeff(int narg, char **arg)
{
  if (!allocated) allocate();
  if (narg < 4) error->all(FLERR, "Incorrect args for pair coefficients");
  if (strcmp(arg[0], "*") != 0 || strcmp(arg[1], "*") != 0)
    error->all(FLERR, "Incorrect args for pair coefficients");
  std::string args;
  for (int i = 2; i < narg; i++) {
    if (i > 2) args += " ";
    args += arg[i];
    // electron temperature in K, kept in eV (pair_tensormd.cpp:33,245-246)
    if (strcmp(arg[i], "etemp") == 0 && i + 1 < narg)
      etemp = utils::numeric(FLERR, arg[i + 1], false, lmp) / 11604.522060401008;
  }
  if (sys) { tmd_system_free(sys); sys = nullptr; }
  if (model) { tmd_model_free(model); model = nullptr; }
  check(tmd_model_load(args.c_str(), 0, &model), "pair_coeff");
  int ntypes_mapped = 0;
  check(tmd_model_info(model, &cutmax, nullptr, &ntypes_mapped, nullptr, nullptr, nullptr),
        "model info");
  int n = atom->ntypes;
  if (ntypes_mapped != n)
    error->all(FLERR, "Number of elements in pair_coeff must equal the number of atom types");
  std::vector<int> tmap(n + 1);
  std::vector<double> tmass(n + 1);
  check(tmd_model_type_map(model, tmap.data(), tmass.data()), "type map");
  int count = 0;
  for (int i = 1; i <= n; i++) {
    map[i] = tmap[i];
    for (int j = i; j <= n; j++) {
      setflag[i][j] = (tmap[i] >= 0 && tmap[j] >= 0) ? 1 : 0;
      scale[i][j] = 1.0;
      if (setflag[i][j]) count++;
    }
    if (tmap[i] >= 0) atom->set_mass(FLERR, i, tmass[i]);
  }
  if (count == 0) error->all(FLERR, "Incorrect args for pair coefficients");
  last_nlocal = -1;
  last_box_stamp = -1;
}

void PairTensorMDB200::init_style()
{
  if (force->newton_pair == 0) error->all(FLERR, "Pair style tensormd/b200 requires newton pair on");
  skin = neighbor->skin;
  ghost_mode = comm->nprocs > 1;
  last_nlocal = -1;
  last_box_stamp = -1;
  // one scale for all types, as PairTensorMD::compute (pair_tensormd.cpp:168-170)
  const int n = atom->ntypes;
  for (int i = 1; i <= n; i++)
    for (int j = i; j <= n; j++)
      if (setflag[i][j] && scale[i][j] != scale[1][1] && comm->me == 0)
        error->warning(FLERR, "pair tensormd/b200 uses scale[1][1] for every type pair");
}

double PairTensorMDB200::init_one(int i, int j)
{
  if (setflag[i][j] == 0) scale[i][j] = 1.0;
  scale[j][i] = scale[i][j];
  return cutmax;
}

// Hand the current atoms to the device: the first call after LAMMPS
// reneighbored (atoms migrated, re-sorted, ghosts rebuilt) uploads types and
// order, the others positions only.
void PairTensorMDB200::upload()
{
  const int nlocal = atom->nlocal;
  const int nall = ghost_mode ? nlocal + atom->nghost : nlocal;
  if (!sys || nall > natoms_cap) {
    if (sys) tmd_system_free(sys);
    natoms_cap = nall + nall / 5 + 64;
    check(tmd_system_create(model, natoms_cap, skin, &sys), "system");
    last_nlocal = -1;
    last_box_stamp = -1;
    last_etemp = -1.0;
  }
  xbuf.assign(atom->x[0], atom->x[0] + 3 * (size_t)nall);
  const bool reneighbored = nall != last_nall || nlocal != last_nlocal || neighbor->ago == 0;
  if (ghost_mode) {
    if (reneighbored) {
      tbuf.assign(atom->type, atom->type + nall);
      check(tmd_system_set_atoms_ghost(sys, nlocal, nall - nlocal, xbuf.data(), tbuf.data()),
            "local and ghost atoms");
    } else {
      check(tmd_system_set_positions(sys, xbuf.data()), "positions");
    }
  } else {
    double box[9] = {domain->boxlo[0], domain->boxlo[1], domain->boxlo[2],
                     domain->xprd,     domain->yprd,     domain->zprd,
                     domain->xy,       domain->xz,       domain->yz};
    int pbc[3] = {domain->xperiodic, domain->yperiodic, domain->zperiodic};
    bool box_changed = last_box_stamp < 0;
    for (int c = 0; c < 9 && !box_changed; c++) box_changed = box[c] != last_box[c];
    if (box_changed) {
      check(tmd_system_set_box(sys, box, pbc), "box");
      memcpy(last_box, box, sizeof(box));
      last_box_stamp = 1;
    }
    if (reneighbored || box_changed) {
      tbuf.assign(atom->type, atom->type + nlocal);
      check(tmd_system_set_atoms(sys, nlocal, xbuf.data(), tbuf.data(), nullptr), "atoms");
    } else {
      check(tmd_system_set_positions(sys, xbuf.data()), "positions");
    }
  }
  last_nlocal = nlocal;
  last_nall = nall;
}

void PairTensorMDB200::compute(int eflag, int vflag)
{
  ev_init(eflag, vflag);
  upload();
  // forces (and per-atom virials) on every atom the device holds: the local
  // ones, and in the ghost-aware mode the ghosts for reverse communication
  const int n = last_nall;
  fbuf.resize(3 * (size_t)n);
  double e = 0.0, v6[6] = {0, 0, 0, 0, 0, 0};
  double *ea = nullptr, *va = nullptr;
  if (eflag_atom) { ebuf.resize(n); ea = ebuf.data(); }
  if (vflag_atom) { vbuf.resize(6 * (size_t)n); va = vbuf.data(); }
  if (etemp != last_etemp) {
    check(tmd_system_set_etemp(sys, etemp), "electron temperature");
    last_etemp = etemp;
  }
  check(tmd_compute(sys, eflag, vflag, scale[1][1], &e, v6, fbuf.data(), ea, va), "compute");
  // TDNP potentials: entropy and free energy (zero otherwise)
  if (tmd_system_tdnp_energies(sys, &eentropy, &free_energy) != TMD_OK)
    eentropy = free_energy = 0.0;
  double **f = atom->f;
  for (int i = 0; i < n; i++) {
    f[i][0] += fbuf[3 * i];
    f[i][1] += fbuf[3 * i + 1];
    f[i][2] += fbuf[3 * i + 2];
  }
  if (eflag_global) eng_vdwl += e;
  if (vflag_global)
    for (int c = 0; c < 6; c++) virial[c] += v6[c];
  if (eflag_atom)
    for (int i = 0; i < n; i++) eatom[i] += ebuf[i];
  if (vflag_atom)
    for (int i = 0; i < n; i++)
      for (int c = 0; c < 6; c++) vatom[i][c] += vbuf[6 * i + c];
}

int PairTensorMDB200::descriptor_width()
{
  int nd = 0;
  if (model) check(tmd_model_info(model, nullptr, nullptr, nullptr, &nd, nullptr, nullptr), "model info");
  return nd;
}

void PairTensorMDB200::descriptors(double *G)
{
  upload();
  check(tmd_get_descriptors(sys, G), "descriptors");
}

void *PairTensorMDB200::extract(const char *str, int &dim)
{
  if (strcmp(str, "scale") == 0) {
    dim = 2;
    return (void *) scale;
  }
  if (strcmp(str, "etemp") == 0) {
    dim = 0;
    return (void *) &etemp;
  }
  return nullptr;
}

double PairTensorMDB200::memory_usage()
{
  return (double) (xbuf.capacity() + fbuf.capacity() + ebuf.capacity() + vbuf.capacity()) *
      sizeof(double);
}
