// server.cpp -- the serving loop: continuous batching of independent small
// systems (single-point energies, NVE runs, FIRE relaxations) on one GPU.
//
// Callers submit jobs from any thread (tmd_server_submit) and collect results
// (tmd_server_wait).  One worker thread owns the device: it keeps every job
// in flight as a cell of one multi-cell system (batch.cpp) and repeats ticks:
//   1. retire finished cells and admit queued jobs (single-point jobs first,
//      then FIFO, up to the atom and cell budget), re-laying the cells out on
//      the device: continuing cells move with their state and neighbor lists,
//      new jobs come from a staging upload and get their lists built;
//   2. one force evaluation: single-point jobs are finished by it and leave
//      before the steps (FIRE jobs test convergence only after an iteration,
//      as LAMMPS does);
//   3. steps_per_tick steps of the mixed integrator (server_kernels.cu) for the rest;
//   4. per-cell status to the host; finished NVE / FIRE jobs are copied out.
// A job waits at most one tick before it enters the batch, and every step
// advances all jobs in flight with one launch per kernel.  LAMMPS runs one
// system per process (pair_tensormd.cpp:141-184); the batch gives each cell
// the results that system would give.
#include <algorithm>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "system.h"

using namespace tmd;
using Clock = std::chrono::steady_clock;

namespace {

struct Job {
  long id = 0;
  int kind = kJobEnergy;
  int n = 0;
  std::vector<double> x, v;
  std::vector<int> elem;
  std::vector<int> ecount;  // atoms per potential element
  double box[9];
  int pbc[3];
  int nsteps = 0;
  double dt = 0.001, fmax = 0.01;
  Clock::time_point t_submit, t_done;
  // results
  bool done = false;
  int status = TMD_OK;
  std::string err;
  double energy = 0.0, virial[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> xo, vo, fo;
  int steps = 0;
};

using JobP = std::shared_ptr<Job>;

}  // namespace

struct tmd_server {
  const tmd_model *m = nullptr;
  tmd_system *s = nullptr;
  int max_atoms = 0, max_cells = 0, steps_per_tick = 8;
  int max_cap = 0;  // > 0: longest neighbor row the HBM budget allows (byte-budget servers)
  // shared with callers
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::deque<JobP> queue;
  std::unordered_map<long, JobP> jobs;
  long next_id = 1;
  long submitted = 0, completed = 0;
  double atom_steps = 0.0, busy_s = 0.0;
  long active_atoms = 0;
  std::string fatal;  // worker error: every later job fails with it
  double t_phase[4] = {0, 0, 0, 0};  // relayout, admission evaluation, steps, results
  // worker-owned
  std::thread worker;
  std::vector<JobP> active;            // cell order
  std::vector<CellCtl> h_ctl;          // host copy of the cells' control blocks
  std::vector<double> h_cell;          // [cells][8] energy, virial
  // second copies of the per-atom arrays a relayout moves into
  double *x2 = nullptr, *v2 = nullptr, *f2 = nullptr, *xb2 = nullptr;
  int *img2 = nullptr, *elem2 = nullptr, *boff2 = nullptr;
  int *rev2 = nullptr;  // natoms x cap, allocated with the rows
  double *stage_x = nullptr, *stage_v = nullptr;
  int *stage_e = nullptr;
  int *src = nullptr, *fresh = nullptr, *estart = nullptr;
  CellCtl *ctl = nullptr;
  double *pw = nullptr, *pm = nullptr, *csum = nullptr, *cmax = nullptr, *fsq = nullptr,
         *cfmax = nullptr;
};

namespace {

void finish(tmd_server *sv, const JobP &j, int status, const std::string &err) {
  std::lock_guard<std::mutex> lk(sv->mu);
  j->status = status;
  j->err = err;
  j->done = true;
  j->t_done = Clock::now();
  sv->completed++;
  sv->cv_done.notify_all();
}

CellCtl initial_ctl(const Job &j) {
  CellCtl q{};
  q.mode = j.kind;
  q.left = j.kind == kJobEnergy ? 0 : j.nsteps;
  q.dt = j.dt;
  q.dtmax = 10.0 * j.dt;   // min_style fire tmax 10
  q.dtmin = 0.02 * j.dt;   // tmin 0.02
  q.alpha = 0.25;          // alpha0
  q.fmax2 = j.fmax * j.fmax;
  return q;
}

// Device bytes per atom of a server whose neighbor rows hold `cap` entries:
// the system's and the server's per-atom arrays, cap x 64 B of rows (tmp,
// nbr, rev and the relayout copy of rev: 4 B each; pair forces 16 B; pair
// geometry 32 B) and the neighbor bins (at most about two per atom).
size_t server_bytes_per_atom(const tmd_model *m, int cap) {
  const HostModel &h = m->h;
  const size_t B = h.nelt, nin = h.nin;
  size_t a = 4 * 24 + 12 + 4;          // x, v, f, xbuild; image; element
  a += 3 * 4;                          // bin of atom, binned atoms, raw row length
  a += 4 * (B + 1) + 4 * B;            // row block offsets, active pairs per block
  a += 4 * B * h.K * h.D + 2 * 4 * nin;  // P; G and dE/dG
  a += 8 + 48 + 8 + 48 + 8 + 4 + 4;    // E, virial partials, eatom, vatom, ke, perm, cell
  a += 4 * 24 + 12 + 4 + 4 * (B + 1);  // relayout copies: x v f xbuild, image, element, offsets
  a += 48 + 4 + 40 + 8;                // staging x v, staging element, FIRE power and maxima, |F|^2
  a += 2 * 12;                         // bins: count, start, cursor
  a += (size_t)cap * 64;
  return a;
}

// Row length (a multiple of 32) a job of n atoms in box volume vol needs.
int job_cap(const tmd_server *sv, int n, double vol) {
  return (cap_for_density(sv->s, n / vol) + 31) / 32 * 32;
}

// Move every atom into the layout described by sv->src / sv->fresh (already
// on the device, with acell and coff) with neighbor rows of cap1 entries, and
// swap the moved arrays in.  Rows of the same length go through the build
// scratch (tmp) and sv->rev2; longer rows get new arrays.
int move_cells(tmd_server *sv, int n, int cap1) {
  tmd_system *s = sv->s;
  if (cap1 > 4096) return fail(TMD_ERR_CAPACITY, "more than 4096 neighbors per atom");
  if (sv->max_cap > 0 && cap1 > sv->max_cap)
    return fail(TMD_ERR_CAPACITY, "neighbor rows beyond the server's HBM budget");
  const bool same = cap1 == s->cap && s->nbr && s->tmp && sv->rev2;
  uint32_t *nbr2 = same ? s->tmp : nullptr;
  int *rev2 = same ? sv->rev2 : nullptr;
  if (!same) {
    const size_t tot = (size_t)s->natoms_cap * cap1;
    cudaError_t e = dalloc(&nbr2, tot);
    if (e == cudaSuccess) e = dalloc(&rev2, tot);
    if (e != cudaSuccess) {
      dfree(nbr2);
      dfree(rev2);
      return fail(TMD_ERR_CUDA, std::string("neighbor rows: ") + cudaGetErrorString(e));
    }
  }
  SrvMove m{};
  m.n = n;
  m.B = s->m->h.nelt;
  m.cap0 = s->cap > 0 ? s->cap : 1;
  m.cap1 = cap1;
  m.acell = s->acell; m.coff = s->coff; m.src = sv->src; m.fresh = sv->fresh;
  m.x = s->x; m.v = s->v; m.f = s->f; m.xb = s->xbuild;
  m.img = s->image; m.elem = s->elem; m.boff = s->boff; m.rev = s->rev; m.nbr = s->nbr;
  m.sx = sv->stage_x; m.sv = sv->stage_v; m.selem = sv->stage_e;
  m.x2 = sv->x2; m.v2 = sv->v2; m.f2 = sv->f2; m.xb2 = sv->xb2;
  m.img2 = sv->img2; m.elem2 = sv->elem2; m.boff2 = sv->boff2; m.rev2 = rev2; m.nbr2 = nbr2;
  launch_srv_move(m, s->st, s->launches);
  TMD_CUDA(cudaGetLastError());
  std::swap(s->x, sv->x2);
  std::swap(s->v, sv->v2);
  std::swap(s->f, sv->f2);
  std::swap(s->xbuild, sv->xb2);
  std::swap(s->image, sv->img2);
  std::swap(s->elem, sv->elem2);
  std::swap(s->boff, sv->boff2);
  if (same) {
    std::swap(s->nbr, s->tmp);
    std::swap(s->rev, sv->rev2);
    return TMD_OK;
  }
  int rc = adopt_rows(s, cap1, nbr2, rev2);  // synchronises, frees the old rows
  if (rc) return rc;
  dfree(sv->rev2);
  TMD_CUDA(dalloc(&sv->rev2, (size_t)s->natoms_cap * cap1));
  return TMD_OK;
}

// Neighbor lists of the fresh cells (the others kept theirs).  An overflow
// lengthens every row in place (each cell moves onto itself) and builds the
// fresh cells again.
int build_fresh(tmd_server *sv) {
  tmd_system *s = sv->s;
  for (int attempt = 0; attempt < 4; attempt++) {
    int rc = clear_status(s);
    if (rc) return rc;
    launch_srv_mark(s->ncells, sv->fresh, s->cflag, s->flag, s->st, s->launches);
    launch_neighbor_build(nb_args(s), s->st, s->launches);
    TMD_CUDA(cudaGetLastError());
    rc = read_status(s);
    if (rc) return rc;
    const int st = s->h_status[0];
    if (st & kStatusShift) return fail(TMD_ERR_ARG, "periodic cell is too small for the cutoff");
    if (st & kStatusOutside) return fail(TMD_ERR_ARG, "atom outside a non-periodic boundary");
    if (!(st & kStatusOverflow)) return TMD_OK;
    const int need = s->h_status[1];
    const int cap1 = (need + need / 4 + 32 + 31) / 32 * 32;
    std::vector<int> self(s->h_coff.begin(), s->h_coff.end() - 1);
    TMD_CUDA(cudaMemcpyAsync(sv->src, self.data(), self.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s->st));
    rc = move_cells(sv, s->n, cap1);
    if (rc) return rc;
  }
  return fail(TMD_ERR_CAPACITY, "neighbor list did not fit after resizing");
}

// Lay the cells of `next` out on the device: continuing jobs move from the
// current layout with their neighbor lists (a cell's list is rebuilt only
// when its own atoms trigger it, as for a separate system), new ones come
// from staging and get their lists built.  Host work is per cell; per-atom
// work (cell index, element grouping) runs on the device.
int relayout(tmd_server *sv, const std::vector<JobP> &next) {
  tmd_system *s = sv->s;
  const int C = (int)next.size();
  if (C == 0) {  // nothing in flight: keep the arrays, launch nothing
    sv->active.clear();
    sv->h_ctl.clear();
    s->n = 0;
    return TMD_OK;
  }
  const int B = s->m->h.nelt, tr = s->m->mlp_tr;
  std::unordered_map<const Job *, int> old_cell;
  for (size_t c = 0; c < sv->active.size(); c++) old_cell[sv->active[c].get()] = (int)c;
  std::vector<int> coff(C + 1, 0), srcv(C), fresh(C, 0), total(B, 0), selem;
  std::vector<double> boxes(9 * (size_t)C), sx, svel;
  std::vector<int> pbc(3 * (size_t)C);
  std::vector<CellCtl> ctl(C);
  int staged = 0;
  for (int c = 0; c < C; c++) {
    const Job &j = *next[c];
    coff[c + 1] = coff[c] + j.n;
    std::memcpy(&boxes[9 * (size_t)c], j.box, sizeof j.box);
    std::memcpy(&pbc[3 * (size_t)c], j.pbc, sizeof j.pbc);
    for (int e = 0; e < B; e++) total[e] += j.ecount[e];
    auto it = old_cell.find(&j);
    if (it != old_cell.end()) {
      srcv[c] = s->h_coff[it->second];
      ctl[c] = sv->h_ctl[it->second];
    } else {
      srcv[c] = -staged - 1;
      sx.insert(sx.end(), j.x.begin(), j.x.end());
      svel.insert(svel.end(), j.v.begin(), j.v.end());
      selem.insert(selem.end(), j.elem.begin(), j.elem.end());
      staged += j.n;
      ctl[c] = initial_ctl(j);
      fresh[c] = 1;
    }
  }
  const int n = coff[C];
  if (n > s->natoms_cap) return fail(TMD_ERR_CAPACITY, "atoms exceed the batch capacity");
  // MLP element grouping (set_elements' order): element e from start[e],
  // cell by cell; tiles of up to mlp_tr atoms of one element
  std::vector<int> cur(B, 0), estart((size_t)C * B), tiles;
  for (int e = 1; e < B; e++) cur[e] = cur[e - 1] + total[e - 1];
  for (int e = 0; e < B; e++)
    for (int o = 0; o < total[e]; o += tr) {
      tiles.push_back(e);
      tiles.push_back(cur[e] + o);
      tiles.push_back(std::min(tr, total[e] - o));
    }
  for (int c = 0; c < C; c++)
    for (int e = 0; e < B; e++) {
      estart[(size_t)c * B + e] = cur[e];
      cur[e] += next[c]->ecount[e];
    }
  s->ncells = C;
  s->h_coff = coff;
  s->h_acell.clear();
  int rc = cells_geometry(s, boxes.data(), pbc.data());
  if (rc) return rc;
  TMD_CUDA(cudaMemcpyAsync(s->coff, coff.data(), (C + 1) * sizeof(int), cudaMemcpyHostToDevice,
                           s->st));
  TMD_CUDA(cudaMemcpyAsync(sv->src, srcv.data(), C * sizeof(int), cudaMemcpyHostToDevice,
                           s->st));
  TMD_CUDA(cudaMemcpyAsync(sv->fresh, fresh.data(), C * sizeof(int), cudaMemcpyHostToDevice,
                           s->st));
  TMD_CUDA(cudaMemcpyAsync(sv->ctl, ctl.data(), C * sizeof(CellCtl), cudaMemcpyHostToDevice,
                           s->st));
  TMD_CUDA(cudaMemcpyAsync(sv->estart, estart.data(), estart.size() * sizeof(int),
                           cudaMemcpyHostToDevice, s->st));
  if (!tiles.empty())
    TMD_CUDA(cudaMemcpyAsync(s->tiles, tiles.data(), tiles.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s->st));
  if (staged > 0) {
    TMD_CUDA(cudaMemcpyAsync(sv->stage_x, sx.data(), sx.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s->st));
    TMD_CUDA(cudaMemcpyAsync(sv->stage_v, svel.data(), svel.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s->st));
    TMD_CUDA(cudaMemcpyAsync(sv->stage_e, selem.data(), selem.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s->st));
  }
  launch_srv_acell(C, s->coff, s->acell, s->st, s->launches);
  // row length: the current one unless a fresh cell is denser than it allows
  // (a byte-budget server holds rows of its full length from the start)
  int cap1 = std::max(s->cap, sv->max_cap);
  if (staged > 0) {
    double dens = 0.0;
    for (int c = 0; c < C; c++)
      if (fresh[c]) {
        const BoxP &bx = s->h_cbox[c];
        dens = std::max(dens, (coff[c + 1] - coff[c]) / (bx.xprd * bx.yprd * bx.zprd));
      }
    cap1 = std::max(cap1, (cap_for_density(s, dens) + 31) / 32 * 32);
  }
  rc = move_cells(sv, n, cap1);
  if (rc) return rc;
  launch_srv_perm(C, B, s->coff, s->elem, sv->estart, s->perm, s->st, s->launches);
  TMD_CUDA(cudaGetLastError());
  s->n = n;
  s->ntiles = (int)tiles.size() / 3;
  s->h_elem.clear();
  s->have_atoms = true;
  s->forces_valid = false;
  s->nhc_valid = false;
  sv->active = next;
  sv->h_ctl = ctl;
  if (staged > 0) return build_fresh(sv);  // synchronises
  TMD_CUDA(cudaStreamSynchronize(s->st));
  return TMD_OK;
}

// Per-cell energy/virial sums and control blocks to the host.
int read_cells(tmd_server *sv) {
  tmd_system *s = sv->s;
  const int C = s->ncells;
  launch_cell_sum(C, s->coff, s->E, 1, 1.0, s->cell_out, 8, s->st, s->launches);
  launch_cell_sum(C, s->coff, s->wv, 6, 1.0, s->cell_out + 1, 8, s->st, s->launches);
  launch_check_finite(s->n, s->f, nullptr, s->status, s->st, s->launches);
  sv->h_cell.resize(8 * (size_t)C);
  sv->h_ctl.resize(C);
  TMD_CUDA(cudaMemcpyAsync(sv->h_cell.data(), s->cell_out, 8 * (size_t)C * sizeof(double),
                           cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaMemcpyAsync(sv->h_ctl.data(), sv->ctl, C * sizeof(CellCtl),
                           cudaMemcpyDeviceToHost, s->st));
  int rc = read_status(s);  // synchronises
  if (rc) return rc;
  const int st = s->h_status[0];
  if (st & kStatusOverflow) return fail(TMD_ERR_CAPACITY, "neighbor list overflow");
  if (st & kStatusTimeout) return fail(TMD_ERR_TIMEOUT, "a tensor-core wait timed out");
  if (st & kStatusLaunch) return fail(TMD_ERR_CUDA, "neighbor build launched without its shared memory");
  if (st & kStatusShift) return fail(TMD_ERR_ARG, "a cell is too small for the cutoff");
  return TMD_OK;
}

// Copy the results of cell c to its job and finish it.
int take_results(tmd_server *sv, int c) {
  tmd_system *s = sv->s;
  Job &j = *sv->active[c];
  const size_t a0 = (size_t)s->h_coff[c], n = (size_t)j.n;
  j.xo.resize(3 * n);
  j.fo.resize(3 * n);
  j.vo.resize(3 * n);
  TMD_CUDA(cudaMemcpyAsync(j.xo.data(), s->x + 3 * a0, 3 * n * sizeof(double),
                           cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaMemcpyAsync(j.fo.data(), s->f + 3 * a0, 3 * n * sizeof(double),
                           cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaMemcpyAsync(j.vo.data(), s->v + 3 * a0, 3 * n * sizeof(double),
                           cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaStreamSynchronize(s->st));
  j.energy = sv->h_cell[8 * (size_t)c];
  for (int k = 0; k < 6; k++) j.virial[k] = sv->h_cell[8 * (size_t)c + 1 + k];
  const CellCtl &q = sv->h_ctl[c];
  j.steps = j.kind == kJobEnergy ? 0 : (j.kind == kJobNve ? j.nsteps - q.left : q.it);
  bool finite = std::isfinite(j.energy);
  for (double fv : j.fo) finite = finite && std::isfinite(fv);
  finish(sv, sv->active[c], finite ? TMD_OK : TMD_ERR_NONFINITE,
         finite ? "" : "non-finite energy or force");
  return TMD_OK;
}

bool cell_done(const Job &j, const CellCtl &q) {
  if (j.kind == kJobEnergy) return true;
  if (j.kind == kJobNve) return q.left <= 0;
  return q.conv || q.left <= 0;
}

// Jobs of `sv->active` not finished, in order.
std::vector<JobP> survivors(tmd_server *sv, const std::vector<char> &gone) {
  std::vector<JobP> out;
  for (size_t c = 0; c < sv->active.size(); c++)
    if (!gone[c]) out.push_back(sv->active[c]);
  return out;
}

int tick(tmd_server *sv) {
  tmd_system *s = sv->s;
  // 1. admission within the budget: queued single-point jobs first (they
  // hold atoms only for the tick that evaluates them), then the others FIFO;
  // jobs finished by the last tick's steps leave with the same relayout
  std::vector<JobP> next;
  long atoms = 0;
  for (auto &j : sv->active)
    if (!j->done) {
      next.push_back(j);
      atoms += j->n;
    }
  const bool retired = next.size() != sv->active.size();
  size_t nadm = 0;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto fits = [&](const Job &j) {
      return atoms + j.n <= sv->max_atoms && (int)next.size() < sv->max_cells;
    };
    std::deque<JobP> rest;
    for (auto &j : sv->queue) {
      if (j->kind == kJobEnergy && fits(*j)) {
        atoms += j->n;
        next.push_back(j);
        nadm++;
      } else {
        rest.push_back(j);
      }
    }
    sv->queue.swap(rest);
    while (!sv->queue.empty() && fits(*sv->queue.front())) {
      atoms += sv->queue.front()->n;
      next.push_back(sv->queue.front());
      sv->queue.pop_front();
      nadm++;
    }
    sv->active_atoms = atoms;
  }
  int rc = TMD_OK;
  std::vector<char> gone;
  bool any = false;
  auto t0 = Clock::now();
  auto lap = [&](double &acc) {
    auto t1 = Clock::now();
    acc += std::chrono::duration<double>(t1 - t0).count();
    t0 = t1;
  };
  if (retired || nadm > 0) {
    rc = relayout(sv, next);
    if (rc) return rc;
    lap(sv->t_phase[0]);
    if (sv->active.empty()) return TMD_OK;
  }
  if (nadm > 0) {
    // 2. new jobs need forces: one evaluation; the jobs it finishes leave now
    launch_force_eval(s, 1.0f, false);
    launch_srv_post(s->n, s->ncells, s->acell, s->coff, sv->ctl, s->v, s->f, s->elem,
                    s->m->d_mass, sv->fsq, sv->cfmax, 0, 0, s->st, s->launches);
    rc = read_cells(sv);
    if (rc) return rc;
    sv->atom_steps += s->n;
    lap(sv->t_phase[1]);
    gone.assign(sv->active.size(), 0);
    for (size_t c = 0; c < sv->active.size(); c++)
      if (cell_done(*sv->active[c], sv->h_ctl[c])) {
        rc = take_results(sv, (int)c);
        if (rc) return rc;
        gone[c] = 1;
        any = true;
      }
    lap(sv->t_phase[3]);
    if (any) {
      rc = relayout(sv, survivors(sv, gone));
      if (rc) return rc;
      lap(sv->t_phase[0]);
    }
  }
  if (sv->active.empty()) return TMD_OK;
  // 3. steps of the mixed integrator
  const double half = 0.5 * s->skin;
  for (int k = 0; k < sv->steps_per_tick; k++) {
    launch_srv_pre(s->n, s->ncells, s->acell, s->coff, sv->ctl, s->x, s->v, s->f, s->elem,
                   s->m->d_mass, sv->pw, sv->pm, sv->csum, sv->cmax, s->st, s->launches);
    launch_neighbor_check(s->n, s->x, s->xbuild, half * half, s->flag, s->st, s->launches,
                          s->acell, s->cflag);
    launch_neighbor_build(nb_args(s), s->st, s->launches);
    launch_force_eval(s, 1.0f, false);
    launch_srv_post(s->n, s->ncells, s->acell, s->coff, sv->ctl, s->v, s->f, s->elem,
                    s->m->d_mass, sv->fsq, sv->cfmax, 1, 1, s->st, s->launches);
    sv->atom_steps += s->n;
  }
  TMD_CUDA(cudaGetLastError());
  rc = read_cells(sv);
  if (rc) return rc;
  lap(sv->t_phase[2]);
  // 4. finished NVE / FIRE jobs are copied out; they leave the batch with the
  // next tick's relayout
  for (size_t c = 0; c < sv->active.size(); c++)
    if (!sv->active[c]->done && cell_done(*sv->active[c], sv->h_ctl[c])) {
      rc = take_results(sv, (int)c);
      if (rc) return rc;
    }
  lap(sv->t_phase[3]);
  return TMD_OK;
}

void worker_main(tmd_server *sv) {
  cudaSetDevice(sv->m->device);
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->cv_work.wait(lk, [&] { return sv->stop || !sv->queue.empty() || !sv->active.empty(); });
      if (sv->stop) break;
    }
    auto t0 = Clock::now();
    int rc = sv->fatal.empty() ? tick(sv) : TMD_OK;
    auto t1 = Clock::now();
    std::vector<JobP> failed;
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      sv->busy_s += std::chrono::duration<double>(t1 - t0).count();
      if (rc != TMD_OK && sv->fatal.empty()) {
        char buf[512];
        tmd_last_error(buf, sizeof buf);
        sv->fatal = buf;
      }
      if (!sv->fatal.empty()) {
        failed.assign(sv->active.begin(), sv->active.end());
        failed.insert(failed.end(), sv->queue.begin(), sv->queue.end());
        sv->queue.clear();
      }
    }
    if (!failed.empty()) {
      for (auto &j : failed)
        if (!j->done) finish(sv, j, TMD_ERR_CUDA, "server stopped: " + sv->fatal);
      sv->active.clear();
    }
  }
}

int server_create(const tmd_model *m, int max_atoms, int max_cells, double skin,
                  int steps_per_tick, int row_cap, tmd_server **out);

}  // namespace

extern "C" {

int tmd_server_create(const tmd_model *m, int max_atoms, int max_cells, double skin,
                      int steps_per_tick, tmd_server **out) {
  return server_create(m, max_atoms, max_cells, skin, steps_per_tick, 0, out);
}

}  // extern "C"

namespace {

// row_cap > 0: neighbor rows of exactly this length for the server's life
// (byte-budget servers); 0: rows for jobs up to 0.09 atoms/A^3, longer when
// a denser job comes
int server_create(const tmd_model *m, int max_atoms, int max_cells, double skin,
                  int steps_per_tick, int row_cap, tmd_server **out) {
  if (!m || !out || max_atoms < 1 || max_cells < 1 || steps_per_tick < 1)
    return fail(TMD_ERR_ARG, "bad server arguments");
  *out = nullptr;
  tmd_system *s = nullptr;
  int rc = tmd_system_create(m, max_atoms, skin, &s);
  if (rc) return rc;
  rc = cells_alloc(s, max_cells);
  if (rc) {
    tmd_system_free(s);
    return rc;
  }
  tmd_server *sv = new tmd_server();
  sv->m = m;
  sv->s = s;
  sv->max_atoms = max_atoms;
  sv->max_cells = max_cells;
  sv->steps_per_tick = steps_per_tick;
  const size_t N = max_atoms, C = max_cells;
  cudaError_t e = dalloc(&sv->x2, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->v2, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->f2, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->img2, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->xb2, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->elem2, N);
  if (e == cudaSuccess) e = dalloc(&sv->boff2, N * (m->h.nelt + 1));
  if (e == cudaSuccess) e = dalloc(&sv->stage_x, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->stage_v, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->stage_e, N);
  if (e == cudaSuccess) e = dalloc(&sv->src, C);
  if (e == cudaSuccess) e = dalloc(&sv->fresh, C);
  if (e == cudaSuccess) e = dalloc(&sv->estart, C * m->h.nelt);
  if (e == cudaSuccess) e = dalloc(&sv->ctl, C);
  if (e == cudaSuccess) e = dalloc(&sv->pw, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->pm, 2 * N);
  if (e == cudaSuccess) e = dalloc(&sv->csum, 4 * C);
  if (e == cudaSuccess) e = dalloc(&sv->cmax, 2 * C);
  if (e == cudaSuccess) e = dalloc(&sv->fsq, N);
  if (e == cudaSuccess) e = dalloc(&sv->cfmax, C);
  if (e != cudaSuccess) {
    tmd_server_free(sv);
    return fail(TMD_ERR_CUDA, std::string("server allocation: ") + cudaGetErrorString(e));
  }
  s->have_box = true;
  // neighbor rows up front, so that admissions move data instead of
  // allocating it
  sv->max_cap = row_cap;
  rc = move_cells(sv, 0, row_cap > 0 ? row_cap : (cap_for_density(s, 0.09) + 31) / 32 * 32);
  if (rc) {
    tmd_server_free(sv);
    return rc;
  }
  sv->worker = std::thread(worker_main, sv);
  *out = sv;
  return TMD_OK;
}

}  // namespace

extern "C" {

int tmd_server_create_bytes(const tmd_model *m, size_t hbm_bytes, double max_density,
                            int max_cells, double skin, int steps_per_tick, tmd_server **out) {
  if (!m || !out || !(max_density > 0) || !(skin >= 0) || max_cells < 1)
    return fail(TMD_ERR_ARG, "bad server arguments");
  *out = nullptr;
  // the row length of the densest admissible job, then as many atoms as fit
  const double cut = m->h.rmax + skin;
  const double est = max_density * 4.0 / 3.0 * M_PI * cut * cut * cut;
  int cap = std::max((int)std::ceil(1.3 * est) + 32, 64);
  cap = (cap + 31) / 32 * 32;
  if (cap > 4096) return fail(TMD_ERR_CAPACITY, "density needs more than 4096 neighbors per atom");
  const size_t per = server_bytes_per_atom(m, cap);
  const size_t cell_bytes = (size_t)max_cells * 160;  // boxes, geometry, sums, controls
  if (hbm_bytes <= cell_bytes + per) return fail(TMD_ERR_CAPACITY, "HBM budget below one atom");
  const size_t atoms = (hbm_bytes - cell_bytes) / per;
  if (atoms > (size_t)kMaxAtoms) return fail(TMD_ERR_CAPACITY, "HBM budget beyond the atom index range");
  return server_create(m, (int)atoms, max_cells, skin, steps_per_tick, cap, out);
}

int tmd_server_footprint(const tmd_server *sv, size_t *device_bytes, int *max_atoms,
                         int *row_length) {
  if (!sv) return fail(TMD_ERR_ARG, "null server");
  const int cap = std::max(sv->s->cap, sv->max_cap);
  if (device_bytes)
    *device_bytes = (size_t)sv->max_atoms * server_bytes_per_atom(sv->m, cap) +
                    (size_t)sv->max_cells * 160;
  if (max_atoms) *max_atoms = sv->max_atoms;
  if (row_length) *row_length = cap;
  return TMD_OK;
}

void tmd_server_free(tmd_server *sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  if (sv->worker.joinable()) sv->worker.join();
  if (sv->s) cudaSetDevice(sv->s->m->device);
  dfree(sv->x2); dfree(sv->v2); dfree(sv->f2); dfree(sv->img2);
  dfree(sv->xb2); dfree(sv->elem2); dfree(sv->boff2); dfree(sv->rev2);
  dfree(sv->stage_x); dfree(sv->stage_v); dfree(sv->stage_e); dfree(sv->src);
  dfree(sv->fresh); dfree(sv->estart); dfree(sv->ctl);
  dfree(sv->pw); dfree(sv->pm); dfree(sv->csum); dfree(sv->cmax); dfree(sv->fsq);
  dfree(sv->cfmax);
  tmd_system_free(sv->s);
  delete sv;
}

int tmd_server_submit(tmd_server *sv, int kind, int n, const double *x, const int *type,
                      const double *v, const double box[9], const int pbc[3], int nsteps,
                      double dt, double fmax, long *ticket) {
  if (!sv || !x || !type || !box || !pbc || !ticket || n < 1)
    return fail(TMD_ERR_ARG, "bad job arguments");
  if (kind != kJobEnergy && kind != kJobNve && kind != kJobFire)
    return fail(TMD_ERR_ARG, "unknown job kind");
  if (kind != kJobEnergy && (nsteps < 1 || !(dt > 0)))
    return fail(TMD_ERR_ARG, "NVE and FIRE jobs need nsteps >= 1 and dt > 0");
  if (kind == kJobFire && !(fmax > 0)) return fail(TMD_ERR_ARG, "FIRE jobs need fmax > 0");
  if (n > sv->max_atoms) return fail(TMD_ERR_CAPACITY, "job larger than the server's atom budget");
  {
    BoxP b;
    CellGeom g;
    std::string why;
    int rc = cell_setup(sv->s, box, pbc, b, g, why);
    if (rc) return fail(rc, "job box: " + why);
    if (sv->max_cap > 0 && job_cap(sv, n, b.xprd * b.yprd * b.zprd) > sv->max_cap)
      return fail(TMD_ERR_CAPACITY, "job denser than the server's HBM budget allows");
  }
  auto j = std::make_shared<Job>();
  j->kind = kind;
  j->n = n;
  j->x.assign(x, x + 3 * (size_t)n);
  j->v.assign(3 * (size_t)n, 0.0);
  // FIRE starts from v = 0 (MinFire::setup_style); the caller's v is ignored
  if (v && kind != kJobFire) j->v.assign(v, v + 3 * (size_t)n);
  int rc = map_types(sv->m, n, type, j->elem);
  if (rc) return rc;
  j->ecount.assign(sv->m->h.nelt, 0);
  for (int e : j->elem) j->ecount[e]++;
  std::memcpy(j->box, box, sizeof j->box);
  std::memcpy(j->pbc, pbc, sizeof j->pbc);
  j->nsteps = nsteps;
  j->dt = dt;
  j->fmax = fmax;
  j->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (!sv->fatal.empty()) return fail(TMD_ERR_STATE, "server stopped: " + sv->fatal);
    j->id = sv->next_id++;
    sv->jobs[j->id] = j;
    sv->queue.push_back(j);
    sv->submitted++;
  }
  sv->cv_work.notify_one();
  *ticket = j->id;
  return TMD_OK;
}

int tmd_server_wait(tmd_server *sv, long ticket, double timeout_s, double *energy,
                    double *virial, double *x, double *v, double *f, int *steps,
                    double *latency_s) {
  if (!sv) return fail(TMD_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->jobs.find(ticket);
  if (it == sv->jobs.end()) return fail(TMD_ERR_ARG, "unknown ticket");
  JobP j = it->second;
  auto ready = [&] { return j->done; };
  if (timeout_s < 0) {
    sv->cv_done.wait(lk, ready);
  } else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    return fail(TMD_ERR_TIMEOUT, "job not finished yet");
  }
  sv->jobs.erase(it);
  lk.unlock();
  if (latency_s) *latency_s = std::chrono::duration<double>(j->t_done - j->t_submit).count();
  if (j->status != TMD_OK && j->status != TMD_ERR_NONFINITE) return fail(j->status, j->err);
  const size_t m = 3 * (size_t)j->n;
  if (energy) *energy = j->energy;
  if (virial) std::memcpy(virial, j->virial, sizeof j->virial);
  if (x && j->xo.size() == m) std::memcpy(x, j->xo.data(), m * sizeof(double));
  if (v && j->vo.size() == m) std::memcpy(v, j->vo.data(), m * sizeof(double));
  if (f && j->fo.size() == m) std::memcpy(f, j->fo.data(), m * sizeof(double));
  if (steps) *steps = j->steps;
  if (j->status != TMD_OK) return fail(j->status, j->err);
  return TMD_OK;
}

int tmd_server_timing(tmd_server *sv, double *seconds) {
  if (!sv || !seconds) return fail(TMD_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(sv->mu);
  for (int k = 0; k < 4; k++) seconds[k] = sv->t_phase[k];
  return TMD_OK;
}

int tmd_server_stats(tmd_server *sv, long *submitted, long *completed, long *active_atoms,
                     double *atom_steps, double *busy_s) {
  if (!sv) return fail(TMD_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(sv->mu);
  if (submitted) *submitted = sv->submitted;
  if (completed) *completed = sv->completed;
  if (active_atoms) *active_atoms = sv->active_atoms;
  if (atom_steps) *atom_steps = sv->atom_steps;
  if (busy_s) *busy_s = sv->busy_s;
  return TMD_OK;
}

}  // extern "C"
