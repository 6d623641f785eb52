// abi.cpp -- the C ABI of include/tmd_b200.h.
//
// Host orchestration of one force evaluation (PairTensorMD::compute,
// pair_tensormd.cpp:141-184, and TensorMD::calc_tensor_density/run,
// tensormd.cpp:369-615) and of the NVE loop (Verlet::run + FixNVE,
// verlet.cpp:229-349, fix_nve.cpp:64-141) on one stream, with every array
// resident in device memory:
//
//   [nve initial] -> rebuild check -> (rebuild: bin, build, sort, partners)
//   -> descriptor (P, G) -> MLP forward/backward (E, dE/dG) -> pair forces
//   -> gather (f, FP64) -> [nve final] -> FP64 energy / virial sums
//
// The reference copies the neighbor list and positions to the device and the
// forces back every step with ~15 device synchronisations
// (kernel.cu:1500-1541,1760-1789); here the host synchronises only to return
// requested results.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "system.h"

using namespace tmd;

namespace {
thread_local std::string g_err;
}  // namespace

namespace tmd {
// error message of calls implemented in other translation units
void set_last_error(const std::string &msg) { g_err = msg; }

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}

void drop_graph(tmd_system *s) {
  if (s->step_exec) cudaGraphExecDestroy(s->step_exec);
  s->step_exec = nullptr;
  if (s->pos_exec) cudaGraphExecDestroy(s->pos_exec);
  s->pos_exec = nullptr;
}

// Rebuild kernels counted for the set_positions graphs launched since the
// last read of the device rebuild counter (rb: its current value).
void account_pos_rebuilds(tmd_system *s, int rb) {
  if (s->pos_pending) s->launches += (long)(rb - s->rb_seen) * s->pos_rebuild_launches;
  s->pos_pending = false;
  s->rb_seen = rb;
}

namespace {

cudaEvent_t prof_event(tmd_system *s) {
  if (!s->ev_pool.empty()) {
    cudaEvent_t e = s->ev_pool.back();
    s->ev_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

void prof_begin(tmd_system *s) {
  if (!s->prof) return;
  s->cur_start = prof_event(s);
  cudaEventRecord(s->cur_start, s->st);
}

void prof_end(tmd_system *s, int fam) {
  if (!s->prof) return;
  cudaEvent_t e = prof_event(s);
  cudaEventRecord(e, s->st);
  s->ev_pending.push_back({fam, {s->cur_start, e}});
  if (s->ev_pending.size() > 4096) {  // resolve to bound the pool
    cudaEventSynchronize(e);
    for (auto &p : s->ev_pending) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, p.second.first, p.second.second);
      s->prof_n[p.first]++;
      s->prof_ms[p.first] += ms;
      s->ev_pool.push_back(p.second.first);
      s->ev_pool.push_back(p.second.second);
    }
    s->ev_pending.clear();
  }
}

}  // namespace

void box_setup(BoxP &b, const double bx[9], const int pbc[3]) {
  b.lo[0] = bx[0]; b.lo[1] = bx[1]; b.lo[2] = bx[2];
  b.xprd = bx[3]; b.yprd = bx[4]; b.zprd = bx[5];
  b.xy = bx[6]; b.xz = bx[7]; b.yz = bx[8];
  b.pbc[0] = pbc[0] ? 1 : 0; b.pbc[1] = pbc[1] ? 1 : 0; b.pbc[2] = pbc[2] ? 1 : 0;
  b.triclinic = (b.xy != 0.0 || b.xz != 0.0 || b.yz != 0.0) ? 1 : 0;
  // inverse of h = [[xprd, xy, xz], [0, yprd, yz], [0, 0, zprd]]
  b.hinv[0] = 1.0 / b.xprd;
  b.hinv[1] = 1.0 / b.yprd;
  b.hinv[2] = 1.0 / b.zprd;
  b.hinv[3] = -b.xy / (b.xprd * b.yprd);
  b.hinv[4] = (b.xy * b.yz - b.yprd * b.xz) / (b.xprd * b.yprd * b.zprd);
  b.hinv[5] = -b.yz / (b.yprd * b.zprd);
}

// Perpendicular widths of the cell (distance between opposite faces).
void widths(const BoxP &b, double w[3]) {
  double a[3] = {b.xprd, 0, 0}, bb[3] = {b.xy, b.yprd, 0}, c[3] = {b.xz, b.yz, b.zprd};
  auto cross = [](const double *u, const double *v, double *o) {
    o[0] = u[1] * v[2] - u[2] * v[1];
    o[1] = u[2] * v[0] - u[0] * v[2];
    o[2] = u[0] * v[1] - u[1] * v[0];
  };
  double V = b.xprd * b.yprd * b.zprd;
  double t[3];
  cross(bb, c, t); w[0] = V / std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  cross(c, a, t); w[1] = V / std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
  cross(a, bb, t); w[2] = V / std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
}

namespace {
int bin_setup(tmd_system *s) {
  drop_graph(s);
  double cut = s->m->h.rmax + s->skin;
  double w[3];
  widths(s->box, w);
  BinP b{};
  long ncell = 1;
  for (int a = 0; a < 3; a++) {
    // bins slightly wider than cut/2 so a +-2 stencil covers the cutoff with
    // a margin far above rounding of the fractional coordinates
    int nb = (int)std::floor(w[a] / (0.5 * cut * (1.0 + 1e-6)));
    if (nb < 1) nb = 1;
    if (nb > 1024) nb = 1024;
    b.nb[a] = nb;
    int ns = (int)std::ceil(cut * (1.0 + 1e-9) / (w[a] / nb));
    if (!s->box.pbc[a] && ns > nb) ns = nb;
    if (ns < 1) ns = 1;
    if (s->box.pbc[a] && (ns + nb - 1) / nb > kShiftR + 1)
      return fail(TMD_ERR_ARG, "periodic cell is too small for the cutoff: more than "
                               "3 images per axis would be needed");
    b.ns[a] = ns;
    ncell *= nb;
  }
  while (ncell > (1 << 22)) {  // keep the cell arrays modest
    int a = (b.nb[0] >= b.nb[1] && b.nb[0] >= b.nb[2]) ? 0 : (b.nb[1] >= b.nb[2] ? 1 : 2);
    b.nb[a] = (b.nb[a] + 1) / 2;
    b.ns[a] = (int)std::ceil(cut * (1.0 + 1e-9) / (w[a] / b.nb[a]));
    ncell = (long)b.nb[0] * b.nb[1] * b.nb[2];
  }
  b.ncell = (int)ncell;
  s->bin = b;
  if (b.ncell > s->ncell_alloc) {
    dfree(s->cell_count); dfree(s->cell_start); dfree(s->cell_cursor);
    TMD_CUDA(dalloc(&s->cell_count, b.ncell));
    TMD_CUDA(dalloc(&s->cell_start, b.ncell + 1));
    TMD_CUDA(dalloc(&s->cell_cursor, b.ncell));
    s->ncell_alloc = b.ncell;
  }
  return TMD_OK;
}

int pow2_at_least(int v) {
  int p = 32;
  while (p < v) p <<= 1;
  return p;
}
}  // namespace

int alloc_neighbors(tmd_system *s, int cap) {
  drop_graph(s);
  cap = (cap + 31) / 32 * 32;
  if (cap > 4096) return fail(TMD_ERR_CAPACITY, "more than 4096 neighbors per atom");
  dfree(s->tmp); dfree(s->nbr); dfree(s->rev); dfree(s->pdf); dfree(s->pgeo);
  size_t tot = (size_t)s->natoms_cap * cap;
  TMD_CUDA(dalloc(&s->tmp, tot));
  TMD_CUDA(dalloc(&s->nbr, tot));
  TMD_CUDA(dalloc(&s->rev, tot));
  TMD_CUDA(dalloc(&s->pdf, tot));
  TMD_CUDA(dalloc(&s->pgeo, 2 * tot));
  s->cap = cap;
  s->capp = pow2_at_least(cap);
  return TMD_OK;
}

int adopt_rows(tmd_system *s, int cap, uint32_t *nbr, int *rev) {
  if (cap > 4096) return fail(TMD_ERR_CAPACITY, "more than 4096 neighbors per atom");
  TMD_CUDA(cudaStreamSynchronize(s->st));  // the rows were filled on s->st
  drop_graph(s);
  dfree(s->tmp); dfree(s->nbr); dfree(s->rev); dfree(s->pdf); dfree(s->pgeo);
  s->nbr = nbr;
  s->rev = rev;
  size_t tot = (size_t)s->natoms_cap * cap;
  TMD_CUDA(dalloc(&s->tmp, tot));
  TMD_CUDA(dalloc(&s->pdf, tot));
  TMD_CUDA(dalloc(&s->pgeo, 2 * tot));
  s->cap = cap;
  s->capp = pow2_at_least(cap);
  return TMD_OK;
}

int cap_for_density(const tmd_system *s, double dens) {
  double cut = s->m->h.rmax + s->skin;
  double est = dens * 4.0 / 3.0 * M_PI * cut * cut * cut;
  int cap = (int)std::ceil(1.3 * est) + 32;
  if (cap < 64) cap = 64;
  return cap;
}

int initial_cap(tmd_system *s) {
  double dens = 0.0;
  if (s->ncells > 0) {
    for (int c = 0; c < s->ncells; c++) {
      const BoxP &b = s->h_cbox[c];
      double nc = s->h_coff[c + 1] - s->h_coff[c];
      dens = std::max(dens, nc / (b.xprd * b.yprd * b.zprd));
    }
  } else {
    dens = s->n / (s->box.xprd * s->box.yprd * s->box.zprd);
  }
  return cap_for_density(s, dens);
}

NbArgs nb_args(tmd_system *s) {
  NbArgs a{};
  a.n = s->n; a.B = s->m->h.nelt; a.cap = s->cap; a.capp = s->capp;
  a.kp = s->m->kp; a.box = s->box; a.bin = s->bin;
  double cut = s->m->h.rmax + s->skin;
  a.cutsq = cut * cut;
  a.x = s->x; a.image = s->image; a.elem = s->elem;
  a.cell_of = s->cell_of; a.cell_count = s->cell_count; a.cell_start = s->cell_start;
  a.cell_cursor = s->cell_cursor; a.cell_atoms = s->cell_atoms;
  a.tmp = s->tmp; a.nraw = s->nraw; a.nbr = s->nbr; a.boff = s->boff; a.rev = s->rev;
  // status[0]: status bits; status[1]: the longest row a build needed (read
  // back and cleared together by read_status)
  a.xbuild = s->xbuild; a.flag = s->flag; a.status = s->status; a.maxneed = s->status + 1;
  a.ncells = s->ncells; a.cbox = s->cbox; a.cgeom = s->cgeom; a.acell = s->acell;
  a.coff = s->coff;
  a.cflag = s->ncells ? s->cflag : nullptr;
  a.nlocal = s->n - s->nghost; a.pdf = s->pdf; a.wv = s->wv;
  return a;
}

// Read the status words and clear them for the next kernels.
int read_status(tmd_system *s) {
  TMD_CUDA(cudaMemcpyAsync(s->h_status, s->status, 2 * sizeof(int),
                           cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaMemcpyAsync(s->h_status + 2, s->flag + 1, sizeof(int),
                           cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaMemsetAsync(s->status, 0, 2 * sizeof(int), s->st));
  TMD_CUDA(cudaStreamSynchronize(s->st));
  account_pos_rebuilds(s, s->h_status[2]);
  return TMD_OK;
}

// The graph of set_positions' rebuild: a one-thread kernel sets an IF node
// from the displacement check's flag; the node's body is the rebuild.
int ensure_pos_graph(tmd_system *s) {
  if (s->pos_exec) return TMD_OK;
  if (!s->st_aux) TMD_CUDA(cudaStreamCreateWithFlags(&s->st_aux, cudaStreamNonBlocking));
  long lcount = 0, lb = 0;
  cudaError_t e = cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return fail(TMD_ERR_CUDA, cudaGetErrorString(e));
  cudaStreamCaptureStatus cs;
  cudaGraph_t cg = nullptr;
  const cudaGraphNode_t *deps = nullptr;
  size_t ndeps = 0;
  cudaGraphConditionalHandle ch;
  cudaGraphNode_t cn = nullptr;
  e = cudaStreamGetCaptureInfo(s->st, &cs, nullptr, &cg, &deps, &ndeps);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&ch, cg, 0, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    launch_rebuild_cond(ch, s->flag, s->st, lcount);
    e = cudaStreamGetCaptureInfo(s->st, &cs, nullptr, &cg, &deps, &ndeps);
  }
  cudaGraphNodeParams cp = {};
  if (e == cudaSuccess) {
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = ch;
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    e = cudaGraphAddNode(&cn, cg, deps, ndeps, &cp);
  }
  if (e == cudaSuccess)
    e = cudaStreamBeginCaptureToGraph(s->st_aux, cp.conditional.phGraph_out[0], nullptr, nullptr,
                                      0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    launch_neighbor_build(nb_args(s), s->st_aux, lb);
    cudaGraph_t body;
    e = cudaStreamEndCapture(s->st_aux, &body);
  }
  if (e == cudaSuccess)
    e = cudaStreamUpdateCaptureDependencies(s->st, &cn, 1, cudaStreamSetCaptureDependencies);
  cudaGraph_t g = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(s->st, &g);
  if (e == cudaSuccess) e = ee;
  if (e == cudaSuccess) e = cudaGraphInstantiate(&s->pos_exec, g, 0);
  if (g) cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    s->pos_exec = nullptr;
    cudaGetLastError();  // a refused capture leaves no sticky error
    return fail(TMD_ERR_CUDA, cudaGetErrorString(e));
  }
  s->pos_rebuild_launches = lb;
  return TMD_OK;
}

int clear_status(tmd_system *s) {
  TMD_CUDA(cudaMemsetAsync(s->status, 0, 2 * sizeof(int), s->st));
  return TMD_OK;
}

// Rebuild the list now (flag forced), growing the capacity until it fits.
int rebuild_now(tmd_system *s) {
  for (int attempt = 0; attempt < 4; attempt++) {
    int rc = clear_status(s);
    if (rc) return rc;
    launch_set_flag(s->flag, s->st, s->launches);
    launch_neighbor_build(nb_args(s), s->st, s->launches);
    TMD_CUDA(cudaGetLastError());
    rc = read_status(s);
    if (rc) return rc;
    int st = s->h_status[0];
    if (st & kStatusShift)
      return fail(TMD_ERR_ARG, "periodic cell is too small for the cutoff");
    if (st & kStatusOutside)
      return fail(TMD_ERR_ARG, "atom outside a non-periodic boundary");
    if (!(st & kStatusOverflow)) return TMD_OK;
    int need = s->h_status[1];
    rc = alloc_neighbors(s, need + need / 4 + 32);
    if (rc) return rc;
  }
  return fail(TMD_ERR_CAPACITY, "neighbor list did not fit after resizing");
}

// Force evaluation on the current (valid) list.
DescArgs desc_args(tmd_system *s, int variant) {
  DescArgs d{};
  d.n = s->n - s->nghost; d.cap = s->cap; d.kp = s->m->kp; d.box = s->box; d.x = s->x;
  d.elem = s->elem; d.nbr = s->nbr; d.boff = s->boff; d.P = s->P; d.G = s->G;
  d.cbox = s->ncells ? s->cbox : nullptr; d.acell = s->acell;
  d.variant = variant;
  d.pdf = s->pdf; d.pgeo = s->pgeo; d.pcnt = s->pcnt;
  return d;
}

int default_desc_variant(const tmd_model *m) {
  // measured on the B200 (tmd_system_autotune): the wide form is 1.25-1.33x
  // faster at K = 16 and equal at K = 32
  (void)m;
  return kDescWide;
}

int default_force_variant(const tmd_model *m) {
  // measured on the B200 (tmd_system_autotune): whole pairs per lane beat 4
  // filters per lane by 1.3-2x; 8 lanes per atom up to 16 filters, 16 lanes
  // above (the per-atom dE/dP staging grows with K)
  return m->kp.K <= 16 ? kForcePairLane8 : kForcePairLane16;
}

ForceArgs force_args(tmd_system *s, float scale, int variant) {
  ForceArgs fa{};
  fa.n = s->n - s->nghost; fa.cap = s->cap; fa.kp = s->m->kp; fa.box = s->box; fa.scale = scale;
  fa.x = s->x; fa.elem = s->elem; fa.nbr = s->nbr; fa.boff = s->boff;
  fa.P = s->P; fa.G = s->G; fa.dEdG = s->dEdG;
  fa.pdf = s->pdf; fa.wv = s->wv;
  fa.cbox = s->ncells ? s->cbox : nullptr; fa.acell = s->acell;
  fa.variant = variant;
  fa.pgeo = s->pgeo; fa.pcnt = s->pcnt;
  return fa;
}

void launch_force_eval(tmd_system *s, float scale, bool want_vatom) {
  const tmd_model *m = s->m;
  const DescArgs d = desc_args(s, s->desc_variant);
  prof_begin(s);
  launch_descriptor(d, s->st, s->launches);
  prof_end(s, 1);
  MlpArgs ma{};
  ma.nl = m->h.nl; ma.actfn = m->h.actfn; ma.resnet = m->h.resnet; ma.nin = m->h.nin;
  int maxh = 1;
  for (int l = 1; l < m->h.nl; l++) maxh = std::max(maxh, m->h.sizes[l]);
  ma.maxh = maxh; ma.tr = m->mlp_tr; ma.smem = m->mlp_smem; ma.resident = m->mlp_resident;
  ma.warped = m->mlp_warped;
  ma.streamed = m->mlp_streamed; ma.stages = m->mlp_stages; ma.status = s->status;
  ma.ntiles = s->ntiles; ma.tiles = s->tiles; ma.perm = s->perm; ma.G = s->G;
  ma.dEdG = s->dEdG; ma.E = s->E; ma.layers = m->d_layers;
  prof_begin(s);
  if (m->h.tdnp) {
    TdnpArgs td{};
    td.n = s->n - s->nghost; td.nin = m->h.nin; td.ydim = m->h.ydim; td.maxw = m->tdnp_maxw;
    td.nelt = m->h.nelt;
    td.nl[0] = m->h.tH.nl; td.nl[1] = m->h.tU.nl; td.nl[2] = m->h.tS.nl;
    td.actfn[0] = m->h.tH.actfn; td.actfn[1] = m->h.tU.actfn; td.actfn[2] = m->h.tS.actfn;
    td.resnet[0] = m->h.tH.resnet; td.resnet[1] = m->h.tU.resnet; td.resnet[2] = m->h.tS.resnet;
    td.layers = m->d_tdnp; td.elem = s->elem; td.G = s->G; td.dEdG = s->dEdG;
    td.E = s->E; td.Sa = s->tdnp_s; td.Aa = s->tdnp_a;
    td.T = (float)s->etemp;
    td.c = (float)(m->h.sommerfeld ? s->etemp * s->etemp : s->etemp);
    td.sommerfeld = m->h.sommerfeld;
    td.warp_floats = m->tdnp_warp_floats;
    launch_mlp_tdnp(td, s->st, s->launches);
  } else if (m->d_tc_layers) {
    MlpTcArgs ta{};
    ta.nl = m->h.nl; ta.actfn = m->h.actfn; ta.resnet = m->h.resnet; ta.nin = m->h.nin;
    ta.maxh = m->maxh; ta.ntiles = s->ntiles; ta.tiles = s->tiles; ta.perm = s->perm;
    ta.G = s->G; ta.dEdG = s->dEdG; ta.E = s->E; ta.layers = m->d_tc_layers;
    ta.status = s->status; ta.smem = m->tc_smem; ta.dz_bf16 = m->tc_dz_bf16 ? 1 : 0;
    ta.np = m->tc_np;
    ta.persistent = m->tc_persistent; ta.smem_p = m->tc_smem_p;
    ta.dz_bf16_p = m->tc_dz_bf16_p ? 1 : 0;
    ta.streamed = m->tc_streamed; ta.smem_s = m->tc_smem_s; ta.stages = m->tc_stages;
    ta.cps_s = m->tc_cps;
    ta.probe_wait = s->wait_probe;
    ta.tf32 = m->tc_tf32 ? 1 : 0;
    ta.hi2 = m->tc_hi2;
    if (m->tc_fp8) launch_mlp_fp8(ta, s->st, s->launches);
    else launch_mlp_tc(ta, s->st, s->launches);
  } else {
    launch_mlp_fp32(ma, s->st, s->launches);
  }
  prof_end(s, 2);
  const ForceArgs fa = force_args(s, scale, s->force_variant);
  prof_begin(s);
  launch_force(fa, s->st, s->launches);
  prof_end(s, 3);
  GatherArgs ga{};
  ga.n = s->n; ga.cap = s->cap; ga.B = m->h.nelt; ga.boff = s->boff; ga.pdf = s->pdf;
  ga.rev = s->rev; ga.nbr = s->nbr; ga.x = s->x; ga.box = s->box; ga.wv = s->wv;
  ga.f = s->f; ga.vatom = want_vatom ? s->vatom : nullptr;
  ga.cbox = d.cbox; ga.acell = s->acell;
  prof_begin(s);
  launch_gather(ga, s->st, s->launches);
  prof_end(s, 4);
}

int map_types(const tmd_model *m, int n, const int *type, std::vector<int> &elem) {
  const HostModel &h = m->h;
  const int ntypes = (int)h.type_elements.size();
  elem.resize(n);
  for (int i = 0; i < n; i++) {
    const int t = type[i];
    if (t < 1 || t > ntypes || h.typemap[t] < 0)
      return fail(TMD_ERR_ARG, "atom " + std::to_string(i) + " has type " +
                                   std::to_string(t) + " that pair_coeff did not map");
    elem[i] = h.typemap[t];
  }
  return TMD_OK;
}

int set_elements(tmd_system *s, int n, const int *elem) {
  const HostModel &h = s->m->h;
  s->n = n;
  s->h_elem.assign(elem, elem + n);
  s->nhc_valid = false;  // new atoms: a fresh thermostat
  // atoms grouped by element (TensorMD::calc_tensor_density i2row order),
  // MLP tiles of up to mlp_tr atoms of one element
  // (ghost atoms, the last s->nghost, have no MLP rows)
  const int ne = n - s->nghost;
  std::vector<int> cnt(h.nelt, 0), start(h.nelt + 1, 0);
  for (int i = 0; i < ne; i++) cnt[elem[i]]++;
  for (int e = 0; e < h.nelt; e++) start[e + 1] = start[e] + cnt[e];
  std::vector<int> perm(n > 0 ? n : 1), fill(start.begin(), start.end() - 1);
  for (int i = 0; i < ne; i++) perm[fill[elem[i]]++] = i;
  std::vector<int> tiles;
  for (int e = 0; e < h.nelt; e++)
    for (int o = 0; o < cnt[e]; o += s->m->mlp_tr) {
      tiles.push_back(e);
      tiles.push_back(start[e] + o);
      tiles.push_back(std::min(s->m->mlp_tr, cnt[e] - o));
    }
  s->ntiles = (int)tiles.size() / 3;
  if (n > 0) {
    TMD_CUDA(cudaMemcpyAsync(s->elem, s->h_elem.data(), n * sizeof(int), cudaMemcpyHostToDevice,
                             s->st));
    TMD_CUDA(cudaMemcpyAsync(s->perm, perm.data(), n * sizeof(int), cudaMemcpyHostToDevice, s->st));
    TMD_CUDA(cudaMemcpyAsync(s->tiles, tiles.data(), tiles.size() * sizeof(int),
                             cudaMemcpyHostToDevice, s->st));
    // the copies read host vectors that go out of scope: wait for them
    TMD_CUDA(cudaStreamSynchronize(s->st));
  }
  return TMD_OK;
}

int thermo_reserve(tmd_system *s, long count) {
  if (count > s->thermo_alloc) {
    dfree(s->thermo_d);
    TMD_CUDA(dalloc(&s->thermo_d, (size_t)count));
    s->thermo_alloc = count;
  }
  return TMD_OK;
}

// Device checkpoint of the dynamic state for rolling back a chunk of steps.
int checkpoint_reserve(tmd_system *s) {
  if (!s->ck_x) {
    const size_t N = s->natoms_cap;
    TMD_CUDA(dalloc(&s->ck_x, 3 * N));
    TMD_CUDA(dalloc(&s->ck_v, 3 * N));
    TMD_CUDA(dalloc(&s->ck_f, 3 * N));
    TMD_CUDA(dalloc(&s->ck_img, 3 * N));
  }
  if (s->nhc_alloc > s->ck_nhc_alloc) {
    dfree(s->ck_nhc);
    TMD_CUDA(dalloc(&s->ck_nhc, s->nhc_alloc));
    s->ck_nhc_alloc = s->nhc_alloc;
  }
  return TMD_OK;
}

// save: state -> checkpoint; else checkpoint -> state (stream-ordered).
void checkpoint_copy(tmd_system *s, bool save) {
  const size_t b3 = 3 * (size_t)s->n * sizeof(double), i3 = 3 * (size_t)s->n * sizeof(int);
  auto cp = [&](void *live, void *ck, size_t bytes) {
    if (bytes == 0) return;
    cudaMemcpyAsync(save ? ck : live, save ? live : ck, bytes, cudaMemcpyDeviceToDevice, s->st);
  };
  cp(s->x, s->ck_x, b3);
  cp(s->v, s->ck_v, b3);
  cp(s->f, s->ck_f, b3);
  cp(s->image, s->ck_img, i3);
  if (s->nhc_valid && s->ck_nhc) cp(s->nhc, s->ck_nhc, s->nhc_groups * sizeof(NhcState));
}

// Kinetic energy of every thermostat group into s->nhc_ke.
void group_ke(tmd_system *s) {
  launch_kinetic(s->n, s->v, s->elem, s->m->d_mass, s->ke, s->st, s->launches);
  if (s->ncells > 0)
    launch_cell_sum(s->ncells, s->coff, s->ke, 1, 1.0, s->nhc_ke, 1, s->st, s->launches);
  else
    launch_reduce_f64(s->ke, s->n, 1, s->partial, s->nhc_ke, s->st, s->launches);
}

// Thermostat state for this run: one group per cell (or one for the
// system), eta / eta_dot kept from the previous run of the same layout.
int nhc_prepare(tmd_system *s, const NvtSpec &nvt, int nsteps, double dt) {
  const int G = s->ncells > 0 ? s->ncells : 1;
  if (G > s->nhc_alloc) {
    dfree(s->nhc);
    dfree(s->nhc_ke);
    TMD_CUDA(dalloc(&s->nhc, G));
    TMD_CUDA(dalloc(&s->nhc_ke, G));
    s->nhc_alloc = G;
    s->nhc_valid = false;
  }
  std::vector<NhcState> h(G);
  if (s->nhc_valid && s->nhc_groups == G)
    TMD_CUDA(cudaMemcpy(h.data(), s->nhc, G * sizeof(NhcState), cudaMemcpyDeviceToHost));
  else
    for (auto &c : h) c = NhcState{};
  for (int g = 0; g < G; g++) {
    const int na = s->ncells > 0 ? s->h_coff[g + 1] - s->h_coff[g] : s->n;
    h[g].tdof = 3.0 * na - 3.0;  // compute temp: dof = 3N - dimension
    h[g].t_freq = 1.0 / nvt.t_damp;
    h[g].t_start = nvt.t_start[g];
    h[g].t_stop = nvt.t_stop[g];
    h[g].dt = dt;
    h[g].nsteps = nsteps;
  }
  TMD_CUDA(cudaMemcpyAsync(s->nhc, h.data(), G * sizeof(NhcState), cudaMemcpyHostToDevice,
                           s->st));
  TMD_CUDA(cudaStreamSynchronize(s->st));
  s->nhc_groups = G;
  s->nhc_valid = true;
  return TMD_OK;
}

int run_md(tmd_system *s, int nsteps, double dt, const NvtSpec *nvt, int thermo_every,
           void (*thermo_row)(tmd_system *, int), double *thermo, long thermo_count) {
  TMD_CUDA(cudaSetDevice(s->m->device));
  const int n = s->n;
  if (n == 0) return TMD_OK;
  const double ftm2v = 1.0 / 1.0364269e-4;  // metal units, update.cpp:187-206
  const double dtf = 0.5 * dt * ftm2v;
  const double half = 0.5 * s->skin;
  const double trigsq = half * half;
  const bool want_thermo = thermo && thermo_every > 0;
  if (want_thermo) {
    int rc = thermo_reserve(s, thermo_count);
    if (rc) return rc;
  }
  int rc = clear_status(s);
  if (rc) return rc;
  if (nvt) {
    rc = nhc_prepare(s, *nvt, nsteps, dt);
    if (rc) return rc;
  }
  const int G = s->nhc_groups;
  const int *acell = s->ncells > 0 ? s->acell : nullptr;
  // Verlet::setup: forces of the starting positions (and FixNH::setup)
  launch_force_eval(s, 1.0f, false);
  if (nvt) {
    group_ke(s);
    launch_nhc_setup(G, s->nhc, s->nhc_ke, s->st, s->launches);
  }
  int row = 0;
  if (want_thermo) thermo_row(s, row++);
  auto md_step = [&]() {
    prof_begin(s);
    if (nvt) launch_nhc_half(G, s->nhc, nullptr, n, acell, s->v, s->st, s->launches);
    launch_nve_initial(n, s->x, s->v, s->f, s->elem, s->m->d_mass, dtf, dt, s->st, s->launches);
    launch_neighbor_check(n, s->x, s->xbuild, trigsq, s->flag, s->st, s->launches, s->acell,
                          s->ncells ? s->cflag : nullptr);
    prof_end(s, 5);
    prof_begin(s);
    launch_neighbor_build(nb_args(s), s->st, s->launches);
    prof_end(s, 0);
    launch_force_eval(s, 1.0f, false);
    prof_begin(s);
    launch_nve_final(n, s->v, s->f, s->elem, s->m->d_mass, dtf, s->st, s->launches);
    if (nvt) {
      group_ke(s);
      launch_nhc_half(G, s->nhc, s->nhc_ke, n, acell, s->v, s->st, s->launches);
    }
    prof_end(s, 5);
  };
  // Without kernel timing, the step runs as one captured CUDA graph with its
  // arguments fixed at capture; buffers, box, atom count and dt key the
  // graph.  The rebuild kernels sit in the body of a conditional (IF) node
  // whose value a one-thread kernel sets from the displacement check's flag
  // (cudaGraphSetConditional), so a step without a rebuild launches none of
  // them; where the runtime refuses conditional nodes, every rebuild kernel
  // is captured and returns at once when no rebuild is pending.
  const bool use_graph = !s->prof;
  auto md_step_conditional = [&](cudaGraph_t *g_out) -> cudaError_t {
    long lb = 0;
    cudaError_t e = cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    if (nvt) launch_nhc_half(G, s->nhc, nullptr, n, acell, s->v, s->st, s->launches);
    launch_nve_initial(n, s->x, s->v, s->f, s->elem, s->m->d_mass, dtf, dt, s->st, s->launches);
    launch_neighbor_check(n, s->x, s->xbuild, trigsq, s->flag, s->st, s->launches, s->acell,
                          s->ncells ? s->cflag : nullptr);
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    cudaGraphConditionalHandle ch;
    cudaGraphNode_t cn = nullptr;
    e = cudaStreamGetCaptureInfo(s->st, &cs, nullptr, &cg, &deps, &ndeps);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&ch, cg, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
      launch_rebuild_cond(ch, s->flag, s->st, s->launches);
      e = cudaStreamGetCaptureInfo(s->st, &cs, nullptr, &cg, &deps, &ndeps);
    }
    cudaGraphNodeParams cp = {};
    if (e == cudaSuccess) {
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = ch;
      cp.conditional.type = cudaGraphCondTypeIf;
      cp.conditional.size = 1;
      e = cudaGraphAddNode(&cn, cg, deps, ndeps, &cp);
    }
    if (e == cudaSuccess && !s->st_aux) e = cudaStreamCreateWithFlags(&s->st_aux, cudaStreamNonBlocking);
    if (e == cudaSuccess)
      e = cudaStreamBeginCaptureToGraph(s->st_aux, cp.conditional.phGraph_out[0], nullptr, nullptr,
                                        0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      const long l1 = s->launches;
      launch_neighbor_build(nb_args(s), s->st_aux, s->launches);
      lb = s->launches - l1;
      s->launches = l1;
      cudaGraph_t body;
      e = cudaStreamEndCapture(s->st_aux, &body);
    }
    if (e == cudaSuccess)
      e = cudaStreamUpdateCaptureDependencies(s->st, &cn, 1, cudaStreamSetCaptureDependencies);
    if (e == cudaSuccess) {
      launch_force_eval(s, 1.0f, false);
      launch_nve_final(n, s->v, s->f, s->elem, s->m->d_mass, dtf, s->st, s->launches);
      if (nvt) {
        group_ke(s);
        launch_nhc_half(G, s->nhc, s->nhc_ke, n, acell, s->v, s->st, s->launches);
      }
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s->st, &g);
    if (e == cudaSuccess) e = ee;
    if (e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();  // a refused capture leaves no sticky error
      return e;
    }
    s->rebuild_launches = lb;
    *g_out = g;
    return cudaSuccess;
  };
  auto ensure_graph = [&]() -> int {
    if (!use_graph || (s->step_exec && s->step_dt == dt && s->step_nvt == (nvt != nullptr)))
      return TMD_OK;
    drop_graph(s);
    cudaGraph_t g = nullptr;
    long l0 = s->launches;
    s->rebuild_launches = 0;
    if (md_step_conditional(&g) != cudaSuccess) {
      s->launches = l0;
      s->rebuild_launches = 0;
      TMD_CUDA(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
      md_step();
      TMD_CUDA(cudaStreamEndCapture(s->st, &g));
    }
    cudaError_t ie = cudaGraphInstantiate(&s->step_exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      s->step_exec = nullptr;
      return fail(TMD_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie));
    }
    s->step_launches = s->launches - l0;
    s->launches = l0;
    s->step_dt = dt;
    s->step_nvt = nvt != nullptr;
    return TMD_OK;
  };
  rc = ensure_graph();
  if (rc) return rc;
  // Steps run in chunks from a device checkpoint (x, v, f, image flags,
  // thermostat).  A neighbor row that outgrew its capacity during a chunk
  // truncated that step's list, so the chunk is rolled back, the capacity
  // grown and the chunk run again: the trajectory is the one a large enough
  // list gives.
  constexpr int kChunk = 256;
  rc = checkpoint_reserve(s);
  if (rc) return rc;
  // rebuilds before the run: the conditional rebuild kernels are counted
  // once per rebuild that ran (flag[1])
  int rb0[2] = {0, 0};
  if (use_graph && s->rebuild_launches > 0) {
    TMD_CUDA(cudaMemcpyAsync(rb0, s->flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->st));
    TMD_CUDA(cudaStreamSynchronize(s->st));
    account_pos_rebuilds(s, rb0[1]);
  }
  for (int s0 = 1, retries = 0; s0 <= nsteps;) {
    const int s1 = std::min(nsteps, s0 + kChunk - 1);
    const int row0 = row;
    checkpoint_copy(s, true);
    for (int step = s0; step <= s1; step++) {
      if (use_graph) {
        TMD_CUDA(cudaGraphLaunch(s->step_exec, s->st));
        s->launches += s->step_launches;
      } else {
        md_step();
      }
      if (want_thermo && (step % thermo_every == 0 || step == nsteps)) {
        prof_begin(s);
        thermo_row(s, row++);
        prof_end(s, 6);
      }
    }
    launch_check_finite(n, s->f, nullptr, s->status, s->st, s->launches);
    TMD_CUDA(cudaGetLastError());
    rc = read_status(s);
    if (rc) return rc;
    const int st = s->h_status[0];
    if (st & kStatusOverflow) {
      if (++retries > 8) return fail(TMD_ERR_CAPACITY, "neighbor list kept overflowing");
      // size the rows for the longest one any rebuild of the chunk needed
      // (the restored positions may not need it yet), then rebuild there
      const int need = s->h_status[1];
      checkpoint_copy(s, false);
      rc = alloc_neighbors(s, std::max(need + need / 4 + 32, s->cap + 32));  // drops the graph
      if (rc) return rc;
      rc = rebuild_now(s);
      if (rc) return rc;
      rc = ensure_graph();
      if (rc) return rc;
      row = row0;
      continue;
    }
    if (st & kStatusTimeout) return fail(TMD_ERR_TIMEOUT, "a tensor-core wait timed out");
    if (st & kStatusLaunch) return fail(TMD_ERR_CUDA, "neighbor build launched without its shared memory");
    if (st & kStatusShift) return fail(TMD_ERR_ARG, "periodic cell is too small for the cutoff");
    if (st & kStatusNonfinite) return fail(TMD_ERR_NONFINITE, "non-finite force during the run");
    s0 = s1 + 1;
  }
  if (want_thermo && thermo_count > 0) {
    TMD_CUDA(cudaMemcpyAsync(thermo, s->thermo_d, thermo_count * sizeof(double),
                             cudaMemcpyDeviceToHost, s->st));
    TMD_CUDA(cudaStreamSynchronize(s->st));
  }
  if (use_graph && s->rebuild_launches > 0) {
    int rb1[2] = {0, 0};
    TMD_CUDA(cudaMemcpyAsync(rb1, s->flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->st));
    TMD_CUDA(cudaStreamSynchronize(s->st));
    s->launches += (long)(rb1[1] - rb0[1]) * s->rebuild_launches;
    account_pos_rebuilds(s, rb1[1]);
  }
  s->forces_valid = true;
  return TMD_OK;
}

}  // namespace tmd

extern "C" {

int tmd_last_error(char *buf, int len) {
  if (!buf || len <= 0) return TMD_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", g_err.c_str());
  return TMD_OK;
}

int tmd_model_load(const char *coeff_args, int device, tmd_model **out) {
  if (!coeff_args || !out) return fail(TMD_ERR_ARG, "null argument");
  *out = nullptr;
  tmd_model *m = new tmd_model();
  try {
    m->h = parse_model(coeff_args);
  } catch (const ModelError &e) {
    delete m;
    return fail(TMD_ERR_MODEL, e.what());
  } catch (const std::exception &e) {
    delete m;
    return fail(TMD_ERR_IO, e.what());
  }
  m->device = device;
  cudaError_t ce = cudaSetDevice(device);
  if (ce != cudaSuccess) {
    delete m;
    return fail(TMD_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(ce));
  }
  const HostModel &h = m->h;
  fill_kparams(h, m->kp);
  auto up = [&](const std::vector<float> &v, float **p) -> cudaError_t {
    cudaError_t e = dalloc(p, v.size());
    if (e != cudaSuccess) return e;
    m->d_buf.push_back(*p);
    return cudaMemcpy(*p, v.data(), v.size() * sizeof(float), cudaMemcpyHostToDevice);
  };
  std::vector<MlpLayer> layers((size_t)h.nelt * h.nl);
  cudaError_t e = cudaSuccess;
  if (h.tab_n > 0) {
    e = up(h.table, &m->d_table);
    m->kp.table = m->d_table;
  }
  auto upd = [&](const std::vector<double> &v, double **p) -> cudaError_t {
    cudaError_t e2 = dalloc(p, v.size());
    if (e2 != cudaSuccess) return e2;
    m->d_buf.push_back(reinterpret_cast<float *>(*p));
    return cudaMemcpy(*p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
  };
  for (int el = 0; el < h.nelt && e == cudaSuccess; el++)
    for (int l = 0; l < h.nl && e == cudaSuccess; l++) {
      MlpLayer &L = layers[(size_t)el * h.nl + l];
      L.K = h.sizes[l];
      L.N = h.sizes[l + 1];
      float *w = nullptr, *b = nullptr;
      double *wd = nullptr, *bd = nullptr;
      e = up(h.W[el][l], &w);
      if (e == cudaSuccess && !h.Bs[el][l].empty()) e = up(h.Bs[el][l], &b);
      if (l == h.nl - 1) {
        if (e == cudaSuccess) e = upd(h.Wout[el], &wd);
        if (e == cudaSuccess && !h.Bout[el].empty()) e = upd(h.Bout[el], &bd);
      }
      L.W = w;
      L.b = b;
      L.Wd = wd;
      L.bd = bd;
    }
  if (e == cudaSuccess) e = dalloc(&m->d_layers, layers.size());
  if (e == cudaSuccess)
    e = cudaMemcpy(m->d_layers, layers.data(), layers.size() * sizeof(MlpLayer),
                   cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = dalloc(&m->d_mass, h.nelt);
  if (e == cudaSuccess)
    e = cudaMemcpy(m->d_mass, h.masses.data(), h.nelt * sizeof(double),
                   cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    tmd_model_free(m);
    return fail(TMD_ERR_CUDA, std::string("model upload: ") + cudaGetErrorString(e));
  }
  if (h.tdnp) {
    // the H, U, S nets replace the MLP (k_mlp_tdnp); their layers as
    // [net][element][kMaxLayers], W and W^T in FP32, output row sums of U
    // and S in FP32 and FP64
    const HostModel::Net *nets[3] = {&h.tH, &h.tU, &h.tS};
    std::vector<TdnpLayer> tl((size_t)3 * h.nelt * kMaxLayers);
    int maxw = std::max(h.nin, h.ydim);
    for (int q = 0; q < 3 && e == cudaSuccess; q++)
      for (int el = 0; el < h.nelt && e == cudaSuccess; el++)
        for (int l = 0; l < nets[q]->nl && e == cudaSuccess; l++) {
          const HostModel::Net &t = *nets[q];
          TdnpLayer &L = tl[((size_t)q * h.nelt + el) * kMaxLayers + l];
          L.K = t.sizes[l];
          L.N = t.sizes[l + 1];
          maxw = std::max(maxw, std::max(L.K, L.N));
          const std::vector<double> &W = t.W[el][l];
          std::vector<float> wf(W.begin(), W.end()), wt((size_t)L.K * L.N);
          for (int k = 0; k < L.K; k++)
            for (int n = 0; n < L.N; n++) wt[(size_t)n * L.K + k] = (float)W[(size_t)k * L.N + n];
          float *dw = nullptr, *dwt = nullptr, *db = nullptr, *dwf = nullptr;
          double *dwd = nullptr;
          e = up(wf, &dw);
          if (e == cudaSuccess) e = up(wt, &dwt);
          if (e == cudaSuccess && !t.B[el][l].empty()) {
            std::vector<float> bf(t.B[el][l].begin(), t.B[el][l].end());
            e = up(bf, &db);
          }
          L.W = dw; L.WT = dwt; L.b = db; L.Wf = nullptr; L.Wd = nullptr; L.bd = 0.0;
          if (q > 0 && l == t.nl - 1 && e == cudaSuccess) {
            std::vector<double> rs(L.K, 0.0);
            std::vector<float> rf(L.K, 0.f);
            for (int k = 0; k < L.K; k++)
              for (int n = 0; n < L.N; n++) {
                rs[k] += W[(size_t)k * L.N + n];
                rf[k] += (float)W[(size_t)k * L.N + n];
              }
            e = upd(rs, &dwd);
            if (e == cudaSuccess) e = up(rf, &dwf);
            for (double b : t.B[el][l]) L.bd += b;
            L.Wf = dwf; L.Wd = dwd;
          }
        }
    if (e == cudaSuccess) e = dalloc(&m->d_tdnp, tl.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(m->d_tdnp, tl.data(), tl.size() * sizeof(TdnpLayer), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      tmd_model_free(m);
      return fail(TMD_ERR_CUDA, std::string("TDNP upload: ") + cudaGetErrorString(e));
    }
    const int nl[3] = {h.tH.nl, h.tU.nl, h.tS.nl};
    m->tdnp_maxw = (maxw + 3) / 4 * 4;
    m->tdnp_warp_floats = tdnp_warp_floats(nl, m->tdnp_maxw);
    if (m->tdnp_warp_floats * sizeof(float) * 4 > 227 * 1024) {
      tmd_model_free(m);
      return fail(TMD_ERR_MODEL, "TDNP nets too wide for the shared-memory work space");
    }
    m->mlp_tr = 64;  // element grouping only (the TDNP kernel takes atoms directly)
    *out = m;
    return TMD_OK;
  }
  // MLP: with 64-wide hidden layers and no residual layers the warp-tile
  // form (a warp per 32 atoms, the element's weights in shared memory);
  // else the resident-weight form (one persistent CTA per SM) when the
  // element's hidden weights and a tile's activations fit in shared memory
  // (128-atom tiles, else 64); else the persistent streamed-weight form
  // (64-atom tiles, weight chunks copied through a stage ring); else, for
  // residual MLPs, weights staged per chunk by the threads with 64- or
  // 32-atom tiles
  size_t s64 = mlp_fp32_smem(h.nl, h.sizes.data(), 64);
  size_t s32 = mlp_fp32_smem(h.nl, h.sizes.data(), 32);
  const size_t sres = mlp_fp32r_smem(h.nl, h.sizes.data(), 128);
  const size_t sres64 = mlp_fp32r_smem(h.nl, h.sizes.data(), 64);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  int wt_warps = 0;
  size_t swt = 0;
  for (int nw = 16; nw >= 8 && wt_warps == 0; nw--) {
    swt = mlp_fp32w_smem(h.nl, h.sizes.data(), h.resnet, nw);
    if (swt > 0 && swt <= 227 * 1024) wt_warps = nw;
  }
  if (wt_warps > 0 && nsm > 0) {
    // 64-wide hidden layers: the warp-tile form, one CTA of wt_warps warps
    // per SM, tiles of mlp_fp32w_rows() atoms per warp
    m->mlp_tr = mlp_fp32w_rows() * wt_warps; m->mlp_smem = swt; m->mlp_resident = nsm;
    m->mlp_warped = wt_warps;
  } else if (h.nl >= 2 && sres <= 227 * 1024 && nsm > 0) {
    m->mlp_tr = 128; m->mlp_smem = sres; m->mlp_resident = nsm;
  } else if (h.nl >= 2 && sres64 <= 227 * 1024 && nsm > 0) {
    m->mlp_tr = 64; m->mlp_smem = sres64; m->mlp_resident = nsm;
  } else if (int stages = 0;
             nsm > 0 && (m->mlp_smem = mlp_fp32s_smem(h.nl, h.sizes.data(), h.resnet, &stages)) > 0) {
    // weights streamed through shared memory in chunks (64-atom tiles):
    // pack each hidden layer's W and W^T into the chunk layouts
    m->mlp_tr = 64; m->mlp_streamed = nsm; m->mlp_stages = stages;
    for (int el = 0; el < h.nelt && e == cudaSuccess; el++)
      for (int l = 0; l + 1 < h.nl && e == cudaSuccess; l++) {
        MlpLayer &Ly = layers[(size_t)el * h.nl + l];
        std::vector<float> pf, pb;
        mlp_fp32s_pack(h.W[el][l].data(), h.sizes[l], h.sizes[l + 1], pf, pb);
        float *df = nullptr, *db = nullptr;
        e = up(pf, &df);
        if (e == cudaSuccess) e = up(pb, &db);
        Ly.Wp = df;
        Ly.Wtp = db;
      }
    if (e == cudaSuccess)
      e = cudaMemcpy(m->d_layers, layers.data(), layers.size() * sizeof(MlpLayer),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      tmd_model_free(m);
      return fail(TMD_ERR_CUDA, std::string("model upload: ") + cudaGetErrorString(e));
    }
    mlp_fp32s_prepare(m->mlp_smem);
  } else if (s64 <= 110 * 1024) {
    m->mlp_tr = 64; m->mlp_smem = s64;
  } else if (s32 <= 220 * 1024) {
    m->mlp_tr = 32; m->mlp_smem = s32;
  } else {
    tmd_model_free(m);
    return fail(TMD_ERR_MODEL, "MLP too wide for the shared-memory tile");
  }
  if (m->mlp_warped > 0) mlp_fp32w_prepare(m->mlp_smem);
  else if (m->mlp_streamed == 0) mlp_fp32_prepare(m->mlp_tr, m->mlp_smem, m->mlp_resident > 0);
  for (int l = 1; l < h.nl; l++) m->maxh = std::max(m->maxh, h.sizes[l]);
  if (h.precision == TMD_PREC_TF32X3) {
    // 3xTF32 on tcgen05 (streamed form): W as hi = tf32(W) and lo =
    // tf32(W - hi) planes, 32-column chunks, W^T (forward) and W (backward)
    int stages = 0;
    const size_t ss = mlp_tcs_smem(h.nl, h.sizes.data(), h.resnet, 3, 1, 1, &stages);
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    if (ss == 0 || nsm <= 0) {
      tmd_model_free(m);
      return fail(TMD_ERR_MODEL, "precision tf32x3 needs no residual layers, nelt*k*m and hidden "
                                 "widths that are multiples of 32, hidden widths <= 256 and "
                                 "act' within 512 TMEM columns");
    }
    std::vector<MlpTcLayer> tl((size_t)h.nelt * h.nl);
    for (int el = 0; el < h.nelt && e == cudaSuccess; el++)
      for (int l = 0; l < h.nl && e == cudaSuccess; l++) {
        MlpTcLayer &T = tl[(size_t)el * h.nl + l];
        const MlpLayer &F = layers[(size_t)el * h.nl + l];
        T.K = h.sizes[l];
        T.N = h.sizes[l + 1];
        T.b = F.b;
        T.wd = F.Wd;
        T.bd = F.bd;
        T.wscale = 1.f;
        if (l == h.nl - 1) continue;
        const int K = T.K, N = T.N;
        const size_t nf = (size_t)N * K;
        std::vector<float> pf(2 * nf), pb(2 * nf);
        const std::vector<float> &W = h.W[el][l];
        for (int part = 0; part < 2; part++) {
          pack_core_chunks_tf32(W.data(), N, K, 1, N, part, pf.data() + part * nf);  // W^T
          pack_core_chunks_tf32(W.data(), K, N, N, 1, part, pb.data() + part * nf);  // W
        }
        for (auto *vec : {&pf, &pb}) {
          float *d = nullptr;
          if (e == cudaSuccess) e = dalloc(&d, vec->size());
          if (e == cudaSuccess) {
            m->d_buf.push_back(d);
            e = cudaMemcpy(d, vec->data(), vec->size() * 4, cudaMemcpyHostToDevice);
          }
          if (vec == &pf) T.Wf = d; else T.Wb = d;
        }
      }
    if (e == cudaSuccess) e = dalloc(&m->d_tc_layers, tl.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(m->d_tc_layers, tl.data(), tl.size() * sizeof(MlpTcLayer),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      tmd_model_free(m);
      return fail(TMD_ERR_CUDA, std::string("tensor-core weight upload: ") +
                                    cudaGetErrorString(e));
    }
    m->tc_np = 3;
    m->tc_tf32 = true;
    m->tc_hi2 = mlp_tcs_hi2(h.nl, h.sizes.data(), 3, 1);
    m->tc_streamed = nsm;
    m->tc_smem_s = ss;
    m->tc_stages = stages;
    mlp_tcs_prepare(ss, 3, 1, 1);
    m->mlp_tr = 128;
  }
  if (h.precision == TMD_PREC_BF16 || h.precision == TMD_PREC_BF16X3 ||
      h.precision == TMD_PREC_FP8) {
    const bool fp8 = h.precision == TMD_PREC_FP8;
    const int np = h.precision == TMD_PREC_BF16X3 ? 3 : 1;
    m->tc_np = np;
    m->tc_fp8 = fp8;
    // tcgen05 MLP: 128-atom tiles, widths in multiples of the 64-column chunk
    bool shape_ok = h.nin % 64 == 0 && h.nin <= 1024;
    for (int l = 1; l < h.nl; l++) shape_ok = shape_ok && h.sizes[l] % 64 == 0 && h.sizes[l] <= 128;
    if (!shape_ok) {
      tmd_model_free(m);
      return fail(TMD_ERR_MODEL, "precision bf16/fp8 needs nelt*k*m and hidden widths that "
                                 "are multiples of 64, hidden widths <= 128");
    }
    size_t sm32 = fp8 ? mlp_fp8_smem(h.nl, m->maxh, h.resnet, false)
                      : mlp_tc_smem(h.nl, m->maxh, h.resnet, false, np);
    size_t sm16 = fp8 ? mlp_fp8_smem(h.nl, m->maxh, h.resnet, true)
                      : mlp_tc_smem(h.nl, m->maxh, h.resnet, true, np);
    const size_t kSmemMax = 227 * 1024;
    if (sm32 <= kSmemMax / 2 || (sm32 <= kSmemMax && sm16 > kSmemMax / 2)) {
      m->tc_smem = sm32; m->tc_dz_bf16 = false;
    } else if (sm16 <= kSmemMax) {
      m->tc_smem = sm16; m->tc_dz_bf16 = true;
    } else {
      tmd_model_free(m);
      return fail(TMD_ERR_MODEL, "MLP too large for the tensor-core tile");
    }
    std::vector<MlpTcLayer> tl((size_t)h.nelt * h.nl);
    for (int el = 0; el < h.nelt && e == cudaSuccess; el++)
      for (int l = 0; l < h.nl && e == cudaSuccess; l++) {
        MlpTcLayer &T = tl[(size_t)el * h.nl + l];
        const MlpLayer &F = layers[(size_t)el * h.nl + l];
        T.K = h.sizes[l];
        T.N = h.sizes[l + 1];
        T.b = F.b;
        T.wd = F.Wd;
        T.bd = F.bd;
        T.wscale = 1.f;
        if (l < h.nl - 1 && fp8) {
          // one scale per layer: s_w = 448 / max|W| (e4m3 range)
          const int K = T.K, N = T.N;
          const std::vector<float> &W = h.W[el][l];
          float wmax = 0.f;
          for (float w : W) wmax = std::max(wmax, std::fabs(w));
          T.wscale = wmax > 0.f ? 448.f / wmax : 1.f;
          std::vector<uint8_t> pf((size_t)N * K), pb((size_t)K * N);
          pack_core_chunks_fp8(W.data(), N, K, 1, N, T.wscale, pf.data());  // W^T
          pack_core_chunks_fp8(W.data(), K, N, N, 1, T.wscale, pb.data());  // W
          for (auto *vec : {&pf, &pb}) {
            uint8_t *d = nullptr;
            if (e == cudaSuccess) e = dalloc(&d, vec->size());
            if (e == cudaSuccess) {
              m->d_buf.push_back(reinterpret_cast<float *>(d));
              e = cudaMemcpy(d, vec->data(), vec->size(), cudaMemcpyHostToDevice);
            }
            if (vec == &pf) T.Wf = d; else T.Wb = d;
          }
        } else if (l < h.nl - 1) {
          const int K = T.K, N = T.N;
          const size_t nf = (size_t)N * K, nbk = (size_t)K * N;
          std::vector<uint16_t> pf(nf * np), pb(nbk * np);
          // hi part, then (split form) lo = W - bf16(W)
          const std::vector<float> &Wh = h.W[el][l];
          std::vector<float> Wlo(Wh.size());
          for (size_t q = 0; q < Wh.size(); q++) {
            __nv_bfloat16 hb = __float2bfloat16_rn(Wh[q]);
            Wlo[q] = Wh[q] - __bfloat162float(hb);
          }
          pack_core_chunks(Wh.data(), N, K, 1, N, pf.data());   // W^T
          pack_core_chunks(Wh.data(), K, N, N, 1, pb.data());   // W
          if (np == 3) {
            pack_core_chunks(Wlo.data(), N, K, 1, N, pf.data() + nf);
            pack_core_chunks(Wlo.data(), K, N, N, 1, pb.data() + nbk);
          }
          for (auto *vec : {&pf, &pb}) {
            uint16_t *d = nullptr;
            if (e == cudaSuccess) e = dalloc(&d, vec->size());
            if (e == cudaSuccess) {
              m->d_buf.push_back(reinterpret_cast<float *>(d));
              e = cudaMemcpy(d, vec->data(), vec->size() * 2, cudaMemcpyHostToDevice);
            }
            if (vec == &pf) T.Wf = d; else T.Wb = d;
          }
        }
      }
    if (e == cudaSuccess) e = dalloc(&m->d_tc_layers, tl.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(m->d_tc_layers, tl.data(), tl.size() * sizeof(MlpTcLayer),
                     cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      tmd_model_free(m);
      return fail(TMD_ERR_CUDA, std::string("tensor-core weight upload: ") +
                                    cudaGetErrorString(e));
    }
    if (fp8) mlp_fp8_prepare(m->tc_smem, m->tc_dz_bf16);
    else mlp_tc_prepare(m->tc_smem, m->tc_dz_bf16, np);
    // weight-resident persistent form when the hidden weights, one tile's
    // operands and act' fit in shared memory (next to ~3 KB of static data)
    if (!fp8) {
      // act' in FP32; the BF16 form falls back to BF16 act' when that is what fits
      const size_t kLimit = 227 * 1024 - 3 * 1024;
      size_t sp = mlp_tcp_smem(h.nl, h.sizes.data(), h.resnet, np, false);
      bool dzb = false;
      if ((sp == 0 || sp > kLimit) && np == 1) {
        sp = mlp_tcp_smem(h.nl, h.sizes.data(), h.resnet, np, true);
        dzb = true;
      }
      int nsm = 0;
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
      if (sp > 0 && sp <= kLimit && nsm > 0) {
        // two CTAs per SM where both fit (228 KB per SM, 1 KB reserved and
        // ~3 KB of static data per CTA): one CTA's epilogue and barriers
        // overlap the other's MMAs
        m->tc_persistent = 2 * (sp + 4 * 1024) <= 228 * 1024 ? 2 * nsm : nsm;
        m->tc_smem_p = sp;
        m->tc_dz_bf16_p = dzb;
        mlp_tcp_prepare(sp, np, dzb);
      }
      // weights too large to stay resident: the streamed-weight form, the
      // BF16 form as two CTAs per SM where they fit
      int stages = 0, cps = 2;
      size_t ss = np == 1 ? mlp_tcs_smem(h.nl, h.sizes.data(), h.resnet, np, 0, 2, &stages) : 0;
      if (ss == 0) {
        cps = 1;
        ss = mlp_tcs_smem(h.nl, h.sizes.data(), h.resnet, np, 0, 1, &stages);
      }
      if (m->tc_persistent == 0 && ss > 0 && nsm > 0) {
        m->tc_streamed = cps * nsm;
        m->tc_cps = cps;
        m->tc_smem_s = ss;
        m->tc_stages = stages;
        mlp_tcs_prepare(ss, np, 0, cps);
      }
    }
    m->mlp_tr = 128;
  }
  *out = m;
  return TMD_OK;
}

void tmd_model_free(tmd_model *m) {
  if (!m) return;
  if (m->nsys > 0) {  // systems still use it: the last tmd_system_free releases it
    m->released = true;
    return;
  }
  for (float *p : m->d_buf) cudaFree(p);
  if (m->d_layers) cudaFree(m->d_layers);
  if (m->d_tc_layers) cudaFree(m->d_tc_layers);
  if (m->d_tdnp) cudaFree(m->d_tdnp);
  if (m->d_mass) cudaFree(m->d_mass);
  delete m;
}

int tmd_model_info(const tmd_model *m, double *cutmax, int *nelt, int *ntypes,
                   int *n_desc, int *num_filters, int *mmax) {
  if (!m) return fail(TMD_ERR_ARG, "null model");
  if (cutmax) *cutmax = m->h.rmax;
  if (nelt) *nelt = m->h.nelt;
  if (ntypes) *ntypes = (int)m->h.type_elements.size();
  if (n_desc) *n_desc = m->h.nin;
  if (num_filters) *num_filters = m->h.K;
  if (mmax) *mmax = m->h.M;
  return TMD_OK;
}

int tmd_model_type_map(const tmd_model *m, int *map, double *mass) {
  if (!m) return fail(TMD_ERR_ARG, "null model");
  for (size_t t = 0; t < m->h.typemap.size(); t++) {
    if (map) map[t] = m->h.typemap[t];
    if (mass) mass[t] = m->h.typemass[t];
  }
  return TMD_OK;
}

int tmd_system_create(const tmd_model *m, int natoms_cap, double skin,
                      tmd_system **out) {
  if (!m || !out || natoms_cap < 1) return fail(TMD_ERR_ARG, "bad system arguments");
  if (natoms_cap > kMaxAtoms) return fail(TMD_ERR_CAPACITY, "too many atoms for one system");
  if (!(skin >= 0)) return fail(TMD_ERR_ARG, "skin must be >= 0");
  *out = nullptr;
  TMD_CUDA(cudaSetDevice(m->device));
  tmd_system *s = new tmd_system();
  s->m = m;
  s->natoms_cap = natoms_cap;
  s->skin = skin;
  s->force_variant = default_force_variant(m);
  s->desc_variant = default_desc_variant(m);
  s->etemp = m->h.etemp;
  const HostModel &h = m->h;
  size_t N = natoms_cap;
  cudaError_t e = cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking);
#define A(p, cnt) if (e == cudaSuccess) e = dalloc(&s->p, (cnt))
  A(x, 3 * N); A(v, 3 * N); A(f, 3 * N); A(xbuild, 3 * N);
  A(image, 3 * N); A(elem, N);
  A(cell_of, N); A(cell_atoms, N);
  A(nraw, N); A(boff, N * (h.nelt + 1)); A(pcnt, N * h.nelt);
  A(P, N * h.nelt * h.K * h.D); A(G, N * h.nin); A(dEdG, N * h.nin); A(E, N);
  A(wv, 6 * N); A(eatom, N); A(vatom, 6 * N); A(ke, N);
  if (h.tdnp) { A(tdnp_s, N); A(tdnp_a, N); A(tdnp_tot, 2); }
  A(partial, 1024 * 8); A(scal, 8);
  A(flag, 2); A(status, 2);  // flag[0] rebuild pending, flag[1] rebuilds done
  A(perm, N); A(tiles, 3 * (N / 32 + h.nelt + 1));
#undef A
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&s->h_scal), 8 * sizeof(double));
  if (e == cudaSuccess) e = cudaMallocHost(reinterpret_cast<void **>(&s->h_status), 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(s->v, 0, 3 * N * sizeof(double));
  if (e == cudaSuccess) e = cudaMemset(s->image, 0, 3 * N * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(s->status, 0, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(s->flag, 0, 2 * sizeof(int));
  if (e != cudaSuccess) {
    tmd_system_free(s);
    return fail(TMD_ERR_CUDA, std::string("system allocation: ") + cudaGetErrorString(e));
  }
  const_cast<tmd_model *>(m)->nsys++;
  *out = s;
  return TMD_OK;
}

void tmd_system_free(tmd_system *s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  drop_graph(s);
  dfree(s->x); dfree(s->v); dfree(s->f); dfree(s->xbuild); dfree(s->image); dfree(s->elem);
  dfree(s->cell_of); dfree(s->cell_count); dfree(s->cell_start); dfree(s->cell_cursor);
  dfree(s->cell_atoms); dfree(s->tmp); dfree(s->nbr); dfree(s->nraw); dfree(s->boff);
  dfree(s->rev); dfree(s->P); dfree(s->G); dfree(s->dEdG); dfree(s->E); dfree(s->pdf);
  dfree(s->pgeo); dfree(s->pcnt);
  dfree(s->wv); dfree(s->eatom); dfree(s->vatom); dfree(s->ke); dfree(s->partial);
  dfree(s->scal); dfree(s->flag); dfree(s->status); dfree(s->perm);
  dfree(s->tdnp_s); dfree(s->tdnp_a); dfree(s->tdnp_tot);
  dfree(s->tiles); dfree(s->thermo_d);
  dfree(s->cbox); dfree(s->cgeom); dfree(s->acell); dfree(s->coff); dfree(s->cell_out);
  dfree(s->cflag);
  dfree(s->nhc); dfree(s->nhc_ke);
  dfree(s->ck_x); dfree(s->ck_v); dfree(s->ck_f); dfree(s->ck_img); dfree(s->ck_nhc);
  if (s->h_scal) cudaFreeHost(s->h_scal);
  if (s->h_status) cudaFreeHost(s->h_status);
  for (auto &p : s->ev_pending) {
    cudaEventDestroy(p.second.first);
    cudaEventDestroy(p.second.second);
  }
  for (cudaEvent_t e : s->ev_pool) cudaEventDestroy(e);
  if (s->st) cudaStreamDestroy(s->st);
  if (s->st_aux) cudaStreamDestroy(s->st_aux);
  if (s->m) {
    tmd_model *m = const_cast<tmd_model *>(s->m);
    if (--m->nsys == 0 && m->released) tmd_model_free(m);
  }
  delete s;
}

int tmd_system_set_box(tmd_system *s, const double bx[9], const int pbc[3]) {
  if (!s || !bx || !pbc) return fail(TMD_ERR_ARG, "null argument");
  if (!(bx[3] > 0 && bx[4] > 0 && bx[5] > 0)) return fail(TMD_ERR_ARG, "box lengths must be > 0");
  if (s->ncells > 0)
    return fail(TMD_ERR_STATE, "a batch takes one box per cell (tmd_batch_set_cells)");
  TMD_CUDA(cudaSetDevice(s->m->device));
  box_setup(s->box, bx, pbc);
  s->have_box = true;
  int rc = bin_setup(s);
  if (rc) return rc;
  s->forces_valid = false;
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

int tmd_system_set_atoms(tmd_system *s, int n, const double *x, const int *type,
                         const double *v) {
  if (!s || !x || !type || n < 0) return fail(TMD_ERR_ARG, "null argument");
  if (n > s->natoms_cap) return fail(TMD_ERR_CAPACITY, "n exceeds the system capacity");
  if (!s->have_box) return fail(TMD_ERR_STATE, "set the box before the atoms");
  if (s->ncells > 0 && n != s->h_coff[s->ncells])
    return fail(TMD_ERR_ARG, "a batch takes exactly the atoms of its cells");
  TMD_CUDA(cudaSetDevice(s->m->device));
  drop_graph(s);
  std::vector<int> elem;
  int rc = map_types(s->m, n, type, elem);
  if (rc) return rc;
  s->nghost = 0;
  rc = set_elements(s, n, elem.data());
  if (rc) return rc;
  if (n > 0) {
    TMD_CUDA(cudaMemcpyAsync(s->x, x, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s->st));
    if (v) {
      TMD_CUDA(cudaMemcpyAsync(s->v, v, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s->st));
    } else {
      TMD_CUDA(cudaMemsetAsync(s->v, 0, 3 * n * sizeof(double), s->st));
    }
    TMD_CUDA(cudaMemsetAsync(s->image, 0, 3 * n * sizeof(int), s->st));
  }
  TMD_CUDA(cudaStreamSynchronize(s->st));
  s->have_atoms = true;
  s->forces_valid = false;
  if (n == 0) return TMD_OK;
  int cap = initial_cap(s);
  if (cap > s->cap) {
    rc = alloc_neighbors(s, cap);
    if (rc) return rc;
  }
  return rebuild_now(s);
}

int tmd_system_set_atoms_ghost(tmd_system *s, int nlocal, int nghost, const double *x,
                               const int *type) {
  if (!s || !x || !type || nlocal < 0 || nghost < 0) return fail(TMD_ERR_ARG, "null argument");
  const long nall = (long)nlocal + nghost;
  if (nall > s->natoms_cap) return fail(TMD_ERR_CAPACITY, "nlocal + nghost exceeds the system capacity");
  if (s->ncells > 0) return fail(TMD_ERR_STATE, "a batch has no ghost atoms");
  TMD_CUDA(cudaSetDevice(s->m->device));
  drop_graph(s);
  const int n = (int)nall;
  // a non-periodic box around every atom: the bounding box of the atoms with
  // a margin of cutoff + skin on each side (atoms move less than skin/2
  // between LAMMPS's reneighborings, when the caller sets the atoms anew)
  double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {1.0, 1.0, 1.0};
  for (int a = 0; a < 3 && n > 0; a++) {
    lo[a] = hi[a] = x[a];
    for (int i = 1; i < n; i++) {
      lo[a] = std::min(lo[a], x[3 * (size_t)i + a]);
      hi[a] = std::max(hi[a], x[3 * (size_t)i + a]);
    }
  }
  const double margin = s->m->h.rmax + s->skin;
  const double bx[9] = {lo[0] - margin, lo[1] - margin, lo[2] - margin,
                        hi[0] - lo[0] + 2 * margin, hi[1] - lo[1] + 2 * margin,
                        hi[2] - lo[2] + 2 * margin, 0.0, 0.0, 0.0};
  const int pbc[3] = {0, 0, 0};
  box_setup(s->box, bx, pbc);
  s->have_box = true;
  int rc = bin_setup(s);
  if (rc) return rc;
  std::vector<int> elem;
  rc = map_types(s->m, n, type, elem);
  if (rc) return rc;
  s->nghost = nghost;
  rc = set_elements(s, n, elem.data());
  if (rc) return rc;
  if (n > 0) {
    TMD_CUDA(cudaMemcpyAsync(s->x, x, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, s->st));
    TMD_CUDA(cudaMemsetAsync(s->v, 0, 3 * (size_t)n * sizeof(double), s->st));
    TMD_CUDA(cudaMemsetAsync(s->image, 0, 3 * (size_t)n * sizeof(int), s->st));
  }
  TMD_CUDA(cudaStreamSynchronize(s->st));
  s->have_atoms = true;
  s->forces_valid = false;
  if (n == 0) return TMD_OK;
  // rows for the density inside the atoms' own bounding box
  double vol = 1.0;
  for (int a = 0; a < 3; a++) vol *= std::max(hi[a] - lo[a], 1.0);
  const int cap = cap_for_density(s, n / vol);
  if (cap > s->cap) {
    rc = alloc_neighbors(s, cap);
    if (rc) return rc;
  }
  return rebuild_now(s);
}

int tmd_system_set_positions(tmd_system *s, const double *x) {
  if (!s || !x) return fail(TMD_ERR_ARG, "null argument");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms first");
  if (s->n == 0) return TMD_OK;
  TMD_CUDA(cudaMemcpyAsync(s->x, x, 3 * s->n * sizeof(double), cudaMemcpyHostToDevice, s->st));
  launch_nearest_image(s->n, s->x, s->xbuild, s->box, s->ncells ? s->cbox : nullptr, s->acell,
                       s->st, s->launches);
  s->forces_valid = false;
  double half = 0.5 * s->skin;
  launch_neighbor_check(s->n, s->x, s->xbuild, half * half, s->flag, s->st, s->launches,
                        s->acell, s->ncells ? s->cflag : nullptr);
  // the rebuild only when the check asks for it (conditional graph node);
  // where the graph cannot be made, every rebuild kernel is launched and
  // returns at once when no rebuild is pending
  if (!s->prof && ensure_pos_graph(s) == TMD_OK) {
    TMD_CUDA(cudaGraphLaunch(s->pos_exec, s->st));
    s->launches += 1;
    s->pos_pending = true;
  } else {
    launch_neighbor_build(nb_args(s), s->st, s->launches);
  }
  return TMD_OK;
}

int tmd_system_get(tmd_system *s, double *x, double *v, double *f, int *image) {
  if (!s) return fail(TMD_ERR_ARG, "null system");
  int n = s->n;
  if (n == 0) return TMD_OK;
  if (x) TMD_CUDA(cudaMemcpyAsync(x, s->x, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (v) TMD_CUDA(cudaMemcpyAsync(v, s->v, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (f) TMD_CUDA(cudaMemcpyAsync(f, s->f, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (image) TMD_CUDA(cudaMemcpyAsync(image, s->image, 3 * n * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaStreamSynchronize(s->st));
  return TMD_OK;
}

int tmd_compute(tmd_system *s, int eflag, int vflag, double scale, double *energy,
                double *virial, double *f, double *eatom, double *vatom) {
  if (!s) return fail(TMD_ERR_ARG, "null system");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms before compute");
  TMD_CUDA(cudaSetDevice(s->m->device));
  int n = s->n;
  if (n == 0) {
    if (energy) *energy = 0;
    if (virial) for (int c = 0; c < 6; c++) virial[c] = 0;
    return TMD_OK;
  }
  int rc;
  bool want_vatom = vatom != nullptr;
  // energies and virial partials belong to the evaluated (local) atoms;
  // forces and per-atom virials to every atom, ghosts included
  const int nl = n - s->nghost;
  launch_force_eval(s, (float)scale, want_vatom);
  if (eflag || energy)
    launch_reduce_scaled(s->E, nl, s->partial, s->scal, scale, s->st, s->launches);
  if (s->m->h.tdnp) {
    // entropy and free energy totals of the temperature-dependent model
    // (TensorMD::run, tensormd.cpp:491-492: S and A times the pair scale)
    launch_reduce_scaled(s->tdnp_s, nl, s->partial, s->tdnp_tot, scale, s->st, s->launches);
    launch_reduce_scaled(s->tdnp_a, nl, s->partial, s->tdnp_tot + 1, scale, s->st, s->launches);
  }
  if (vflag || virial)
    launch_reduce_f64(s->wv, nl, 6, s->partial, s->scal + 1, s->st, s->launches);
  launch_check_finite(n, s->f, (eflag || energy) ? s->scal : nullptr, s->status, s->st,
                      s->launches);
  TMD_CUDA(cudaGetLastError());
  if (eatom && nl > 0) launch_scale_copy(s->E, nl, scale, s->eatom, s->st, s->launches);
  TMD_CUDA(cudaMemcpyAsync(s->h_scal, s->scal, 7 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (f) TMD_CUDA(cudaMemcpyAsync(f, s->f, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  if (eatom) {
    if (nl > 0)
      TMD_CUDA(cudaMemcpyAsync(eatom, s->eatom, nl * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    for (int i = nl; i < n; i++) eatom[i] = 0.0;  // ghosts carry no energy
  }
  if (vatom) TMD_CUDA(cudaMemcpyAsync(vatom, s->vatom, 6 * n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
  rc = read_status(s);
  if (rc) return rc;
  int st = s->h_status[0];
  if (st & kStatusOverflow) {
    // positions moved enough to overflow the list: rebuild larger and redo
    rc = rebuild_now(s);
    if (rc) return rc;
    return tmd_compute(s, eflag, vflag, scale, energy, virial, f, eatom, vatom);
  }
  if (st & kStatusTimeout) return fail(TMD_ERR_TIMEOUT, "a tensor-core wait timed out");
  if (st & kStatusLaunch) return fail(TMD_ERR_CUDA, "neighbor build launched without its shared memory");
  if (st & kStatusShift) return fail(TMD_ERR_ARG, "periodic cell is too small for the cutoff");
  if (st & kStatusOutside) return fail(TMD_ERR_ARG, "atom outside a non-periodic boundary");
  if (energy) *energy = s->h_scal[0];
  if (virial) for (int c = 0; c < 6; c++) virial[c] = s->h_scal[1 + c];
  if (s->m->h.tdnp) {
    double t2[2] = {0.0, 0.0};
    TMD_CUDA(cudaMemcpyAsync(t2, s->tdnp_tot, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    TMD_CUDA(cudaStreamSynchronize(s->st));
    s->tdnp_S = t2[0];
    s->tdnp_A = t2[1];
  }
  s->forces_valid = true;
  if (st & kStatusNonfinite) return fail(TMD_ERR_NONFINITE, "non-finite energy or force");
  return TMD_OK;
}

int tmd_nve_run(tmd_system *s, int nsteps, double dt, int thermo_every, double *thermo) {
  if (!s || nsteps < 0 || !(dt > 0)) return fail(TMD_ERR_ARG, "bad nve arguments");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms before nve_run");
  if (s->nghost > 0) return fail(TMD_ERR_STATE, "ghost atoms: the caller integrates");
  if (thermo && thermo_every < 1) return fail(TMD_ERR_ARG, "thermo_every must be >= 1");
  int rows = thermo ? 1 + nsteps / thermo_every + ((nsteps % thermo_every) ? 1 : 0) : 0;
  // row r: potential energy, kinetic energy of the whole system
  auto row_fn = [](tmd_system *q, int r) {
    launch_reduce_scaled(q->E, q->n, q->partial, q->thermo_d + 2 * r, 1.0, q->st, q->launches);
    launch_kinetic(q->n, q->v, q->elem, q->m->d_mass, q->ke, q->st, q->launches);
    launch_reduce_f64(q->ke, q->n, 1, q->partial, q->thermo_d + 2 * r + 1, q->st, q->launches);
  };
  return run_md(s, nsteps, dt, nullptr, thermo ? thermo_every : 0, row_fn, thermo, 2L * rows);
}

int tmd_nvt_run(tmd_system *s, int nsteps, double dt, double t_start, double t_stop,
                double t_damp, int thermo_every, double *thermo) {
  if (!s || nsteps < 0 || !(dt > 0)) return fail(TMD_ERR_ARG, "bad nvt arguments");
  if (!(t_start > 0) || !(t_stop > 0) || !(t_damp > 0))
    return fail(TMD_ERR_ARG, "fix nvt needs t_start, t_stop and t_damp > 0");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms before nvt_run");
  if (s->nghost > 0) return fail(TMD_ERR_STATE, "ghost atoms: the caller integrates");
  if (s->ncells > 0) return fail(TMD_ERR_STATE, "a batch runs nvt through tmd_batch_nvt_run");
  if (thermo && thermo_every < 1) return fail(TMD_ERR_ARG, "thermo_every must be >= 1");
  int rows = thermo ? 1 + nsteps / thermo_every + ((nsteps % thermo_every) ? 1 : 0) : 0;
  auto row_fn = [](tmd_system *q, int r) {
    launch_reduce_scaled(q->E, q->n, q->partial, q->thermo_d + 2 * r, 1.0, q->st, q->launches);
    launch_kinetic(q->n, q->v, q->elem, q->m->d_mass, q->ke, q->st, q->launches);
    launch_reduce_f64(q->ke, q->n, 1, q->partial, q->thermo_d + 2 * r + 1, q->st, q->launches);
  };
  const NvtSpec nvt{&t_start, &t_stop, t_damp};
  return run_md(s, nsteps, dt, &nvt, thermo ? thermo_every : 0, row_fn, thermo, 2L * rows);
}

int tmd_nvt_energy(tmd_system *s, double *energy) {
  if (!s || !energy) return fail(TMD_ERR_ARG, "null argument");
  if (!s->nhc_valid) return fail(TMD_ERR_STATE, "no nvt run on these atoms");
  TMD_CUDA(cudaSetDevice(s->m->device));
  std::vector<NhcState> h(s->nhc_groups);
  TMD_CUDA(cudaStreamSynchronize(s->st));
  TMD_CUDA(cudaMemcpy(h.data(), s->nhc, h.size() * sizeof(NhcState), cudaMemcpyDeviceToHost));
  const double boltz = 8.617343e-5;
  for (size_t g = 0; g < h.size(); g++) {  // FixNH::compute_scalar (fix_nh.cpp:1447-1473)
    const NhcState &c = h[g];
    double e = c.ke_target * c.eta[0] + 0.5 * c.eta_mass[0] * c.eta_dot[0] * c.eta_dot[0];
    for (int k = 1; k < kNhcChain; k++)
      e += boltz * c.t_target * c.eta[k] + 0.5 * c.eta_mass[k] * c.eta_dot[k] * c.eta_dot[k];
    energy[g] = e;
  }
  return TMD_OK;
}

int tmd_neighbor_list(tmd_system *s, double cut, int *counts, int *entries, long cap,
                      long *total) {
  if (!s || !counts || !total) return fail(TMD_ERR_ARG, "null argument");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "no atoms");
  if (cut > s->m->h.rmax + s->skin) return fail(TMD_ERR_ARG, "cut exceeds cutmax + skin");
  int n = s->n;
  int B = s->m->h.nelt;
  std::vector<uint32_t> nb((size_t)n * s->cap);
  std::vector<int> bo((size_t)n * (B + 1));
  std::vector<double> x(3 * (size_t)n);
  if (n > 0) {
    TMD_CUDA(cudaMemcpyAsync(nb.data(), s->nbr, nb.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s->st));
    TMD_CUDA(cudaMemcpyAsync(bo.data(), s->boff, bo.size() * sizeof(int), cudaMemcpyDeviceToHost, s->st));
    TMD_CUDA(cudaMemcpyAsync(x.data(), s->x, x.size() * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    TMD_CUDA(cudaStreamSynchronize(s->st));
  }
  double cutsq = cut * cut;
  long tot = 0;
  for (int i = 0; i < n; i++) {
    int cnt = 0;
    int m = bo[(size_t)i * (B + 1) + B];
    for (int t = 0; t < m; t++) {
      uint32_t e = nb[(size_t)i * s->cap + t];
      int j = e & kAtomMask, sx, sy, sz;
      shift_decode(int(e >> kAtomBits), sx, sy, sz);
      double gx, gy, gz;
      const BoxP &bx = s->ncells ? s->h_cbox[s->h_acell[i]] : s->box;
      image_of(bx, x[3 * j], x[3 * j + 1], x[3 * j + 2], sx, sy, sz, gx, gy, gz);
      double dx = x[3 * i] - gx, dy = x[3 * i + 1] - gy, dz = x[3 * i + 2] - gz;
      double rsq = dx * dx + dy * dy + dz * dz;
      if (rsq <= cutsq) {
        if (entries && tot < cap) {
          entries[4 * tot] = j;
          entries[4 * tot + 1] = sx;
          entries[4 * tot + 2] = sy;
          entries[4 * tot + 3] = sz;
        }
        tot++;
        cnt++;
      }
    }
    counts[i] = cnt;
  }
  *total = tot;
  if (entries && tot > cap) return fail(TMD_ERR_CAPACITY, "entries buffer too small");
  return TMD_OK;
}

int tmd_get_descriptors(tmd_system *s, double *G) {
  if (!s || !G) return fail(TMD_ERR_ARG, "null argument");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms before get_descriptors");
  TMD_CUDA(cudaSetDevice(s->m->device));
  const int nl = s->n - s->nghost;
  size_t cnt = (size_t)nl * s->m->h.nin;
  if (cnt == 0) return TMD_OK;
  // the descriptor of the current positions (compute tensormd/density runs
  // between force evaluations, after LAMMPS moved the atoms)
  for (int attempt = 0; attempt < 2; attempt++) {
    launch_descriptor(desc_args(s, s->desc_variant), s->st, s->launches);
    TMD_CUDA(cudaGetLastError());
    int rc = read_status(s);
    if (rc) return rc;
    if (!(s->h_status[0] & kStatusOverflow)) break;
    rc = rebuild_now(s);  // positions outgrew the rows: rebuild larger, redo
    if (rc) return rc;
  }
  if (s->h_status[0] & kStatusOutside) return fail(TMD_ERR_ARG, "atom outside a non-periodic boundary");
  std::vector<float> tmp(cnt);
  TMD_CUDA(cudaMemcpyAsync(tmp.data(), s->G, cnt * sizeof(float), cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaStreamSynchronize(s->st));
  for (size_t i = 0; i < cnt; i++) G[i] = tmp[i];
  return TMD_OK;
}

namespace {
int family_forms(int family) {
  return family == TMD_TUNE_FORCE ? kForceVariants
                                  : (family == TMD_TUNE_DESCRIPTOR ? kDescVariants : 0);
}
int &family_slot(tmd_system *s, int family) {
  return family == TMD_TUNE_FORCE ? s->force_variant : s->desc_variant;
}
}  // namespace

int tmd_system_set_variant(tmd_system *s, int family, int variant) {
  if (!s) return fail(TMD_ERR_ARG, "null system");
  if (family_forms(family) == 0) return fail(TMD_ERR_ARG, "unknown kernel family");
  if (variant < 0 || variant >= family_forms(family)) return fail(TMD_ERR_ARG, "unknown variant");
  if (variant != family_slot(s, family)) {
    TMD_CUDA(cudaStreamSynchronize(s->st));
    drop_graph(s);  // the captured step holds the old kernel
    family_slot(s, family) = variant;
  }
  return TMD_OK;
}

int tmd_system_get_variant(tmd_system *s, int family, int *variant) {
  if (!s || !variant) return fail(TMD_ERR_ARG, "null argument");
  if (family_forms(family) == 0) return fail(TMD_ERR_ARG, "unknown kernel family");
  *variant = family_slot(s, family);
  return TMD_OK;
}

int tmd_system_autotune(tmd_system *s, int family, int reps, double *ms) {
  if (!s) return fail(TMD_ERR_ARG, "null system");
  const int nforms = family_forms(family);
  if (nforms == 0) return fail(TMD_ERR_ARG, "unknown kernel family");
  if (!s->have_atoms) return fail(TMD_ERR_STATE, "set_atoms before autotune");
  if (reps < 1) reps = 1;
  TMD_CUDA(cudaSetDevice(s->m->device));
  // a full evaluation leaves the list, P, G and dE/dG current for either loop
  int rc = tmd_compute(s, 0, 0, 1.0, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (rc) return rc;
  cudaEvent_t e0, e1;
  TMD_CUDA(cudaEventCreate(&e0));
  TMD_CUDA(cudaEventCreate(&e1));
  int best = family_slot(s, family);
  float best_ms = 0.f;
  cudaError_t err = cudaSuccess;
  for (int v = 0; v < nforms && err == cudaSuccess; v++) {
    auto launch = [&]() {
      if (family == TMD_TUNE_FORCE) launch_force(force_args(s, 1.0f, v), s->st, s->launches);
      else launch_descriptor(desc_args(s, v), s->st, s->launches);
    };
    launch();  // warm-up
    err = cudaEventRecord(e0, s->st);
    for (int r = 0; r < reps && err == cudaSuccess; r++) launch();
    if (err == cudaSuccess) err = cudaEventRecord(e1, s->st);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    if (err == cudaSuccess) err = cudaGetLastError();
    float t = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
    t /= reps;
    if (ms) ms[v] = t;
    if (err == cudaSuccess && (v == 0 || t < best_ms)) { best = v; best_ms = t; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (err != cudaSuccess)
    return fail(TMD_ERR_CUDA, std::string("autotune: ") + cudaGetErrorString(err));
  rc = tmd_system_set_variant(s, family, best);
  if (rc) return rc;
  // results of the chosen form (the forms round differently)
  return tmd_compute(s, 0, 0, 1.0, nullptr, nullptr, nullptr, nullptr, nullptr);
}

int tmd_system_stream(tmd_system *s, void **stream) {
  if (!s || !stream) return fail(TMD_ERR_ARG, "null argument");
  *stream = (void *)s->st;
  return TMD_OK;
}

long tmd_system_launches(const tmd_system *s) { return s ? s->launches : 0; }

int tmd_system_set_etemp(tmd_system *s, double etemp_ev) {
  if (!s || !(etemp_ev >= 0)) return fail(TMD_ERR_ARG, "electron temperature must be >= 0");
  if (etemp_ev != s->etemp) drop_graph(s);  // a captured step holds the old value
  s->etemp = etemp_ev;
  return TMD_OK;
}

int tmd_system_tdnp_energies(tmd_system *s, double *entropy, double *free_energy) {
  if (!s) return fail(TMD_ERR_ARG, "null system");
  if (!s->m->h.tdnp) return fail(TMD_ERR_STATE, "the potential is not temperature-dependent");
  if (entropy) *entropy = s->tdnp_S;
  if (free_energy) *free_energy = s->tdnp_A;
  return TMD_OK;
}

int tmd_system_set_wait_probe(tmd_system *s, long long cycles) {
  if (!s || cycles < 0) return fail(TMD_ERR_ARG, "bad wait probe");
  drop_graph(s);  // a captured step holds the old kernel parameters
  s->wait_probe = cycles;
  return TMD_OK;
}

int tmd_system_rebuilds(tmd_system *s, long *count) {
  if (!s || !count) return fail(TMD_ERR_ARG, "null argument");
  int h[2] = {0, 0};
  TMD_CUDA(cudaMemcpyAsync(h, s->flag, 2 * sizeof(int), cudaMemcpyDeviceToHost, s->st));
  TMD_CUDA(cudaStreamSynchronize(s->st));
  *count = h[1];
  return TMD_OK;
}

int tmd_profile_enable(tmd_system *s, int enable) {
  if (!s) return fail(TMD_ERR_ARG, "null system");
  s->prof = enable != 0;
  return TMD_OK;
}

int tmd_profile_read(tmd_system *s, long *launches, double *ms, int reset) {
  if (!s) return fail(TMD_ERR_ARG, "null system");
  TMD_CUDA(cudaStreamSynchronize(s->st));
  for (auto &p : s->ev_pending) {
    float t = 0.f;
    TMD_CUDA(cudaEventElapsedTime(&t, p.second.first, p.second.second));
    s->prof_n[p.first]++;
    s->prof_ms[p.first] += t;
    s->ev_pool.push_back(p.second.first);
    s->ev_pool.push_back(p.second.second);
  }
  s->ev_pending.clear();
  for (int k = 0; k < TMD_NPROF; k++) {
    if (launches) launches[k] = s->prof_n[k];
    if (ms) ms[k] = s->prof_ms[k];
    if (reset) { s->prof_n[k] = 0; s->prof_ms[k] = 0; }
  }
  return TMD_OK;
}

}  // extern "C"
