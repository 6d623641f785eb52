// server.cpp -- the serving loop: continuous batching of independent small
// systems (single-point energies, NVE runs, FIRE relaxations) on one GPU.
//
// Callers submit jobs from any thread (tmd_server_submit) and collect results
// (tmd_server_wait).  One worker thread owns the device: it keeps every job
// in flight as a cell of one multi-cell system (batch.cpp) and repeats ticks:
//   1. retire finished cells and admit queued jobs (FIFO, up to the atom and
//      cell budget), re-laying the cells out on the device (positions,
//      velocities, forces and image counters of continuing cells gathered
//      into the new order, new jobs appended from a staging upload), then a
//      neighbor rebuild;
//   2. one force evaluation: single-point jobs are finished by it, FIRE jobs
//      that already satisfy fmax too; these leave before the steps;
//   3. steps_per_tick steps of the mixed integrator (server_kernels.cu) for the rest;
//   4. per-cell status to the host; finished NVE / FIRE jobs are copied out.
// A job waits at most one tick before it enters the batch, and every step
// advances all jobs in flight with one launch per kernel.  LAMMPS runs one
// system per process (pair_tensormd.cpp:141-184); the batch gives each cell
// the results that system would give.
#include <algorithm>
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
  double *x2 = nullptr, *v2 = nullptr, *f2 = nullptr;
  int *img2 = nullptr;
  double *stage_x = nullptr, *stage_v = nullptr;
  int *src = nullptr;
  CellCtl *ctl = nullptr;
  double *pw = nullptr, *csum = nullptr, *fsq = nullptr, *cfmax = nullptr;
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
  q.dtmax = 10.0 * j.dt;
  q.alpha = 0.1;
  q.fmax2 = j.fmax * j.fmax;
  return q;
}

// Lay the cells of `next` out on the device (continuing jobs gathered from
// the current layout, new ones from staging), then rebuild the lists.
int relayout(tmd_server *sv, const std::vector<JobP> &next) {
  tmd_system *s = sv->s;
  const int C = (int)next.size();
  if (C == 0) {  // nothing in flight: keep the arrays, launch nothing
    sv->active.clear();
    sv->h_ctl.clear();
    s->n = 0;
    return TMD_OK;
  }
  std::unordered_map<const Job *, int> old_cell;
  for (size_t c = 0; c < sv->active.size(); c++) old_cell[sv->active[c].get()] = (int)c;
  const std::vector<int> old_off = s->h_coff;
  std::vector<int> natoms(C), srcv(C), elem;
  std::vector<double> boxes(9 * (size_t)C), sx, svel;
  std::vector<int> pbc(3 * (size_t)C);
  std::vector<CellCtl> ctl(C);
  int staged = 0;
  for (int c = 0; c < C; c++) {
    const Job &j = *next[c];
    natoms[c] = j.n;
    std::memcpy(&boxes[9 * (size_t)c], j.box, sizeof j.box);
    std::memcpy(&pbc[3 * (size_t)c], j.pbc, sizeof j.pbc);
    elem.insert(elem.end(), j.elem.begin(), j.elem.end());
    auto it = old_cell.find(&j);
    if (it != old_cell.end()) {
      srcv[c] = old_off[it->second];
      ctl[c] = sv->h_ctl[it->second];
    } else {
      srcv[c] = -staged - 1;
      sx.insert(sx.end(), j.x.begin(), j.x.end());
      svel.insert(svel.end(), j.v.begin(), j.v.end());
      staged += j.n;
      ctl[c] = initial_ctl(j);
    }
  }
  if (staged > 0) {
    TMD_CUDA(cudaMemcpyAsync(sv->stage_x, sx.data(), sx.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s->st));
    TMD_CUDA(cudaMemcpyAsync(sv->stage_v, svel.data(), svel.size() * sizeof(double),
                             cudaMemcpyHostToDevice, s->st));
  }
  TMD_CUDA(cudaMemcpyAsync(sv->src, srcv.data(), C * sizeof(int), cudaMemcpyHostToDevice,
                           s->st));
  TMD_CUDA(cudaMemcpyAsync(sv->ctl, ctl.data(), C * sizeof(CellCtl), cudaMemcpyHostToDevice,
                           s->st));
  int rc = cells_layout(s, C, natoms.data());  // new acell/coff (synchronises)
  if (rc) return rc;
  const int n = s->h_coff[C];
  launch_srv_gather(n, s->acell, s->coff, sv->src, s->x, s->v, s->f, s->image, sv->stage_x,
                    sv->stage_v, sv->x2, sv->v2, sv->f2, sv->img2, s->st, s->launches);
  TMD_CUDA(cudaGetLastError());
  std::swap(s->x, sv->x2);
  std::swap(s->v, sv->v2);
  std::swap(s->f, sv->f2);
  std::swap(s->image, sv->img2);
  rc = cells_geometry(s, boxes.data(), pbc.data());
  if (rc) return rc;
  rc = set_elements(s, n, elem.data());
  if (rc) return rc;
  sv->active = next;
  sv->h_ctl = ctl;
  s->have_atoms = true;
  int cap = initial_cap(s);
  if (cap > s->cap) {
    rc = alloc_neighbors(s, cap);
    if (rc) return rc;
  }
  return rebuild_now(s);
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
  // 1. admission (FIFO within the budget); jobs finished by the last tick's
  // steps leave with the same relayout
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
    while (!sv->queue.empty()) {
      const JobP &j = sv->queue.front();
      if (atoms + j->n > sv->max_atoms || (int)next.size() >= sv->max_cells) break;
      atoms += j->n;
      next.push_back(j);
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
                   s->m->d_mass, sv->pw, sv->csum, s->st, s->launches);
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

}  // namespace

extern "C" {

int tmd_server_create(const tmd_model *m, int max_atoms, int max_cells, double skin,
                      int steps_per_tick, tmd_server **out) {
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
  if (e == cudaSuccess) e = dalloc(&sv->stage_x, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->stage_v, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->src, C);
  if (e == cudaSuccess) e = dalloc(&sv->ctl, C);
  if (e == cudaSuccess) e = dalloc(&sv->pw, 3 * N);
  if (e == cudaSuccess) e = dalloc(&sv->csum, 4 * C);
  if (e == cudaSuccess) e = dalloc(&sv->fsq, N);
  if (e == cudaSuccess) e = dalloc(&sv->cfmax, C);
  if (e != cudaSuccess) {
    tmd_server_free(sv);
    return fail(TMD_ERR_CUDA, std::string("server allocation: ") + cudaGetErrorString(e));
  }
  s->have_box = true;
  sv->worker = std::thread(worker_main, sv);
  *out = sv;
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
  dfree(sv->stage_x); dfree(sv->stage_v); dfree(sv->src); dfree(sv->ctl);
  dfree(sv->pw); dfree(sv->csum); dfree(sv->fsq); dfree(sv->cfmax);
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
  if (!(box[3] > 0 && box[4] > 0 && box[5] > 0)) return fail(TMD_ERR_ARG, "box lengths must be > 0");
  auto j = std::make_shared<Job>();
  j->kind = kind;
  j->n = n;
  j->x.assign(x, x + 3 * (size_t)n);
  j->v.assign(3 * (size_t)n, 0.0);
  if (v) j->v.assign(v, v + 3 * (size_t)n);
  int rc = map_types(sv->m, n, type, j->elem);
  if (rc) return rc;
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
