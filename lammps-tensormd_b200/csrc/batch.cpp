// batch.cpp -- multi-cell batches: many small periodic systems (cells) in one
// set of device arrays, each cell with its own box, evaluated by the same
// kernels in one launch per kernel.
//
// Cells are concatenated: atoms of cell c are coff[c]..coff[c+1]-1, every
// atom records its cell, and a pair never leaves its cell (images are taken
// in the cell's own box).  The neighbor build bins every cell in its own grid
// of fractional-coordinate bins and walks a stencil of bins and image shifts
// around each atom; the descriptor, MLP, force and gather kernels are the
// single-system kernels with the box read per atom.  Energies and virials are summed per cell in a
// fixed order.  The reference evaluates one LAMMPS system per process
// (pair_tensormd.cpp:141-184); a batch of C cells gives the same per-cell
// results as C separate systems.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "system.h"

using namespace tmd;

struct tmd_batch {
  tmd_system *s = nullptr;
};

namespace tmd {

int cells_alloc(tmd_system *s, int max_cells) {
  cudaError_t e = dalloc(&s->cbox, max_cells);
  if (e == cudaSuccess) e = dalloc(&s->cgeom, max_cells);
  if (e == cudaSuccess) e = dalloc(&s->acell, s->natoms_cap);
  if (e == cudaSuccess) e = dalloc(&s->coff, max_cells + 1);
  if (e == cudaSuccess) e = dalloc(&s->cell_out, 8 * (size_t)max_cells);
  if (e == cudaSuccess) e = dalloc(&s->cflag, max_cells);
  if (e == cudaSuccess) e = cudaMemset(s->cflag, 0, sizeof(int) * (size_t)max_cells);
  if (e != cudaSuccess)
    return fail(TMD_ERR_CUDA, std::string("batch allocation: ") + cudaGetErrorString(e));
  s->max_cells = max_cells;
  return TMD_OK;
}

int cells_layout(tmd_system *s, int ncells, const int *natoms) {
  if (ncells < 1 || ncells > s->max_cells)
    return fail(TMD_ERR_CAPACITY, "cell count outside the batch capacity");
  long total = 0;
  for (int c = 0; c < ncells; c++) {
    if (natoms[c] < 0) return fail(TMD_ERR_ARG, "negative atom count");
    total += natoms[c];
  }
  if (total > s->natoms_cap) return fail(TMD_ERR_CAPACITY, "atoms exceed the batch capacity");
  drop_graph(s);
  s->ncells = ncells;
  s->h_coff.assign(ncells + 1, 0);
  s->h_acell.resize(total);
  for (int c = 0; c < ncells; c++) {
    s->h_coff[c + 1] = s->h_coff[c] + natoms[c];
    for (int a = s->h_coff[c]; a < s->h_coff[c + 1]; a++) s->h_acell[a] = c;
  }
  if (total > 0)
    TMD_CUDA(cudaMemcpyAsync(s->acell, s->h_acell.data(), total * sizeof(int),
                             cudaMemcpyHostToDevice, s->st));
  TMD_CUDA(cudaMemcpyAsync(s->coff, s->h_coff.data(), (ncells + 1) * sizeof(int),
                           cudaMemcpyHostToDevice, s->st));
  TMD_CUDA(cudaStreamSynchronize(s->st));
  return TMD_OK;
}

int cell_setup(const tmd_system *s, const double bx[9], const int pbc[3], BoxP &b,
               CellGeom &g, std::string &why) {
  const double cut = s->m->h.rmax + s->skin;
  if (!(bx[3] > 0 && bx[4] > 0 && bx[5] > 0)) {
    why = "box lengths must be > 0";
    return TMD_ERR_ARG;
  }
  box_setup(b, bx, pbc);
  g = CellGeom{};
  widths(b, g.w);
  for (int a = 0; a < 3; a++) {
    g.m[a] = 0;
    if (!b.pbc[a]) continue;
    // the largest shift whose slab can come within cut of an atom
    g.m[a] = (int)std::ceil(cut * (1.0 + 1e-9) / g.w[a] + 1e-6);
    if (g.m[a] > kShiftR) {
      why = "too small for the cutoff: more than 3 images per axis would be needed";
      return TMD_ERR_ARG;
    }
  }
  return TMD_OK;
}

void cell_bins(const BoxP &b, int natoms, double cut, CellGeom &g) {
  // bins slightly wider than cut/2 (as the single-box grid), at most about
  // two per atom so a sparse cell does not hold a large empty grid
  for (int a = 0; a < 3; a++) {
    int nb = (int)std::floor(g.w[a] / (0.5 * cut * (1.0 + 1e-6)));
    g.nb[a] = std::max(1, std::min(nb, 1024));
  }
  const long most = std::max(8L, 2L * natoms);
  while ((long)g.nb[0] * g.nb[1] * g.nb[2] > most) {
    const int a = (g.nb[0] >= g.nb[1] && g.nb[0] >= g.nb[2]) ? 0 : (g.nb[1] >= g.nb[2] ? 1 : 2);
    g.nb[a] = (g.nb[a] + 1) / 2;
  }
  for (int a = 0; a < 3; a++) {
    int ns = (int)std::ceil(cut * (1.0 + 1e-9) / (g.w[a] / g.nb[a]));
    if (!b.pbc[a] && ns > g.nb[a]) ns = g.nb[a];
    g.ns[a] = std::max(ns, 1);
  }
}

int cells_geometry(tmd_system *s, const double *boxes, const int *pbc) {
  const int C = s->ncells;
  const double cut = s->m->h.rmax + s->skin;
  std::vector<BoxP> hb(C);
  std::vector<CellGeom> hg(C);
  std::string why;
  long nbins = 0;
  for (int c = 0; c < C; c++) {
    int rc = cell_setup(s, boxes + 9 * (size_t)c, pbc + 3 * (size_t)c, hb[c], hg[c], why);
    if (rc) return fail(rc, "cell " + std::to_string(c) + ": " + why);
    cell_bins(hb[c], s->h_coff[c + 1] - s->h_coff[c], cut, hg[c]);
    hg[c].bin0 = (int)nbins;
    nbins += (long)hg[c].nb[0] * hg[c].nb[1] * hg[c].nb[2];
  }
  if (nbins > (1L << 30)) return fail(TMD_ERR_CAPACITY, "too many neighbor bins");
  drop_graph(s);
  if (nbins > s->ncell_alloc) {
    // with headroom: a server's layouts grow a little at a time
    const long alloc = std::min(nbins + nbins / 2 + 1024, 1L << 30);
    dfree(s->cell_count); dfree(s->cell_start); dfree(s->cell_cursor);
    s->ncell_alloc = 0;
    TMD_CUDA(dalloc(&s->cell_count, alloc));
    TMD_CUDA(dalloc(&s->cell_start, alloc + 1));
    TMD_CUDA(dalloc(&s->cell_cursor, alloc));
    s->ncell_alloc = (int)alloc;
  }
  s->nbins = (int)nbins;
  TMD_CUDA(cudaMemcpyAsync(s->cbox, hb.data(), C * sizeof(BoxP), cudaMemcpyHostToDevice, s->st));
  TMD_CUDA(cudaMemcpyAsync(s->cgeom, hg.data(), C * sizeof(CellGeom), cudaMemcpyHostToDevice,
                           s->st));
  TMD_CUDA(cudaStreamSynchronize(s->st));
  s->h_cbox = hb;
  s->have_box = true;
  s->forces_valid = false;
  return TMD_OK;
}

}  // namespace tmd

namespace {

int batch_ok(const tmd_batch *b) {
  if (!b || !b->s) return fail(TMD_ERR_ARG, "null batch");
  return TMD_OK;
}

}  // namespace

extern "C" {

int tmd_batch_create(const tmd_model *m, int ncells, const int *natoms, double skin,
                     tmd_batch **out) {
  if (!m || !natoms || !out || ncells < 1) return fail(TMD_ERR_ARG, "bad batch arguments");
  *out = nullptr;
  long total = 0;
  for (int c = 0; c < ncells; c++) {
    if (natoms[c] < 0) return fail(TMD_ERR_ARG, "negative atom count");
    total += natoms[c];
  }
  if (total < 1) return fail(TMD_ERR_ARG, "a batch needs at least one atom");
  if (total > kMaxAtoms) return fail(TMD_ERR_CAPACITY, "too many atoms for one batch");
  tmd_system *s = nullptr;
  int rc = tmd_system_create(m, (int)total, skin, &s);
  if (rc) return rc;
  rc = cells_alloc(s, ncells);
  if (!rc) rc = cells_layout(s, ncells, natoms);
  if (rc) {
    tmd_system_free(s);
    return rc;
  }
  tmd_batch *b = new tmd_batch();
  b->s = s;
  *out = b;
  return TMD_OK;
}

void tmd_batch_free(tmd_batch *b) {
  if (!b) return;
  tmd_system_free(b->s);
  delete b;
}

int tmd_batch_system(tmd_batch *b, tmd_system **sys) {
  if (int rc = batch_ok(b)) return rc;
  if (!sys) return fail(TMD_ERR_ARG, "null argument");
  *sys = b->s;
  return TMD_OK;
}

int tmd_batch_set_cells(tmd_batch *b, const double *boxes, const int *pbc) {
  if (int rc = batch_ok(b)) return rc;
  if (!boxes || !pbc) return fail(TMD_ERR_ARG, "null argument");
  tmd_system *s = b->s;
  TMD_CUDA(cudaSetDevice(s->m->device));
  int rc = cells_geometry(s, boxes, pbc);
  if (rc) return rc;
  if (s->have_atoms) {
    int cap = initial_cap(s);
    if (cap > s->cap) {
      rc = alloc_neighbors(s, cap);
      if (rc) return rc;
    }
    return rebuild_now(s);
  }
  return TMD_OK;
}

int tmd_batch_set_atoms(tmd_batch *b, const double *x, const int *type, const double *v) {
  if (int rc = batch_ok(b)) return rc;
  return tmd_system_set_atoms(b->s, b->s->h_coff[b->s->ncells], x, type, v);
}

int tmd_batch_get(tmd_batch *b, double *x, double *v, double *f, int *image) {
  if (int rc = batch_ok(b)) return rc;
  return tmd_system_get(b->s, x, v, f, image);
}

int tmd_batch_compute(tmd_batch *b, double *energy, double *virial, double *f) {
  if (int rc = batch_ok(b)) return rc;
  tmd_system *s = b->s;
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms before compute");
  TMD_CUDA(cudaSetDevice(s->m->device));
  const int C = s->ncells, n = s->n;
  launch_force_eval(s, 1.0f, false);
  launch_cell_sum(C, s->coff, s->E, 1, 1.0, s->cell_out, 8, s->st, s->launches);
  launch_cell_sum(C, s->coff, s->wv, 6, 1.0, s->cell_out + 1, 8, s->st, s->launches);
  launch_check_finite(n, s->f, nullptr, s->status, s->st, s->launches);
  TMD_CUDA(cudaGetLastError());
  std::vector<double> out(8 * (size_t)C);
  TMD_CUDA(cudaMemcpyAsync(out.data(), s->cell_out, out.size() * sizeof(double),
                           cudaMemcpyDeviceToHost, s->st));
  if (f) TMD_CUDA(cudaMemcpyAsync(f, s->f, 3 * (size_t)n * sizeof(double),
                                  cudaMemcpyDeviceToHost, s->st));
  int rc = read_status(s);
  if (rc) return rc;
  const int st = s->h_status[0];
  if (st & kStatusOverflow) {
    rc = rebuild_now(s);
    if (rc) return rc;
    return tmd_batch_compute(b, energy, virial, f);
  }
  if (st & kStatusTimeout) return fail(TMD_ERR_TIMEOUT, "a tensor-core wait timed out");
  if (st & kStatusLaunch) return fail(TMD_ERR_CUDA, "neighbor build launched without its shared memory");
  if (st & kStatusShift) return fail(TMD_ERR_ARG, "a cell is too small for the cutoff");
  if (st & kStatusOutside) return fail(TMD_ERR_ARG, "atom outside a non-periodic boundary");
  for (int c = 0; c < C; c++) {
    if (energy) energy[c] = out[8 * (size_t)c];
    if (virial)
      for (int k = 0; k < 6; k++) virial[6 * (size_t)c + k] = out[8 * (size_t)c + 1 + k];
  }
  s->forces_valid = true;
  if (st & kStatusNonfinite) return fail(TMD_ERR_NONFINITE, "non-finite energy or force");
  return TMD_OK;
}

int tmd_batch_nve_run(tmd_batch *b, int nsteps, double dt, int thermo_every,
                      double *thermo) {
  if (int rc = batch_ok(b)) return rc;
  tmd_system *s = b->s;
  if (nsteps < 0 || !(dt > 0)) return fail(TMD_ERR_ARG, "bad nve arguments");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms before nve_run");
  if (thermo && thermo_every < 1) return fail(TMD_ERR_ARG, "thermo_every must be >= 1");
  const long rows = thermo ? 1 + nsteps / thermo_every + ((nsteps % thermo_every) ? 1 : 0) : 0;
  // row r: (potential, kinetic) energy of every cell
  auto row_fn = [](tmd_system *q, int r) {
    double *o = q->thermo_d + 2 * (size_t)r * q->ncells;
    launch_cell_sum(q->ncells, q->coff, q->E, 1, 1.0, o, 2, q->st, q->launches);
    launch_kinetic(q->n, q->v, q->elem, q->m->d_mass, q->ke, q->st, q->launches);
    launch_cell_sum(q->ncells, q->coff, q->ke, 1, 1.0, o + 1, 2, q->st, q->launches);
  };
  return run_md(s, nsteps, dt, nullptr, thermo ? thermo_every : 0, row_fn, thermo,
                2 * rows * s->ncells);
}

int tmd_batch_nvt_run(tmd_batch *b, int nsteps, double dt, const double *t_start,
                      const double *t_stop, double t_damp, int thermo_every, double *thermo) {
  if (int rc = batch_ok(b)) return rc;
  tmd_system *s = b->s;
  if (nsteps < 0 || !(dt > 0) || !t_start || !t_stop)
    return fail(TMD_ERR_ARG, "bad nvt arguments");
  for (int c = 0; c < s->ncells; c++)
    if (!(t_start[c] > 0) || !(t_stop[c] > 0))
      return fail(TMD_ERR_ARG, "fix nvt needs t_start and t_stop > 0 in every cell");
  if (!(t_damp > 0)) return fail(TMD_ERR_ARG, "fix nvt needs t_damp > 0");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms before nvt_run");
  if (thermo && thermo_every < 1) return fail(TMD_ERR_ARG, "thermo_every must be >= 1");
  const long rows = thermo ? 1 + nsteps / thermo_every + ((nsteps % thermo_every) ? 1 : 0) : 0;
  auto row_fn = [](tmd_system *q, int r) {
    double *o = q->thermo_d + 2 * (size_t)r * q->ncells;
    launch_cell_sum(q->ncells, q->coff, q->E, 1, 1.0, o, 2, q->st, q->launches);
    launch_kinetic(q->n, q->v, q->elem, q->m->d_mass, q->ke, q->st, q->launches);
    launch_cell_sum(q->ncells, q->coff, q->ke, 1, 1.0, o + 1, 2, q->st, q->launches);
  };
  const NvtSpec nvt{t_start, t_stop, t_damp};
  return run_md(s, nsteps, dt, &nvt, thermo ? thermo_every : 0, row_fn, thermo,
                2 * rows * s->ncells);
}

}  // extern "C"
