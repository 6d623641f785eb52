// system.h -- host-side state behind the opaque handles of tmd_b200.h, shared
// by the translation units of the C ABI (abi.cpp: model, system, NVE;
// batch.cpp: multi-cell batches).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/tmd_b200.h"
#include "model.h"
#include "tmd_kernels.h"

struct tmd_model {
  int device = 0;
  tmd::HostModel h;
  tmd::KParams kp;
  float *d_table = nullptr;
  std::vector<float *> d_buf;   // weights and biases
  tmd::MlpLayer *d_layers = nullptr;
  tmd::MlpTcLayer *d_tc_layers = nullptr;  // tensor-core MLP (precision bf16)
  size_t tc_smem = 0;
  bool tc_dz_bf16 = false;
  int tc_np = 1;
  bool tc_fp8 = false;   // FP8 (e4m3) tensor-core MLP
  bool tc_tf32 = false;  // 3xTF32 tensor-core MLP (streamed form)
  int tc_hi2 = 0;        // its second hi accumulator (TMEM permitting)
  int tc_persistent = 0; // > 0: weight-resident persistent tensor-core MLP (grid size)
  size_t tc_smem_p = 0;
  bool tc_dz_bf16_p = false;
  int tc_streamed = 0;   // > 0: streamed-weight persistent tensor-core MLP (grid size)
  size_t tc_smem_s = 0;
  int tc_stages = 0;
  int tc_cps = 1;        // its CTAs per SM
  int maxh = 1;
  double *d_mass = nullptr;     // per element
  int mlp_tr = 64;
  size_t mlp_smem = 0;
  int mlp_resident = 0;    // > 0: resident-weight MLP, persistent grid size
  int mlp_warped = 0;      // > 0: warp-tile MLP, warps per CTA (grid mlp_resident)
  int mlp_streamed = 0;    // > 0: streamed-weight FP32 MLP, persistent grid size
  int mlp_stages = 0;
  // temperature-dependent model (tdnp = 1): the nets' layers on the device
  tmd::TdnpLayer *d_tdnp = nullptr;
  size_t tdnp_warp_floats = 0;
  int tdnp_maxw = 0;
  int nsys = 0;            // systems created from this model and not yet freed
  bool released = false;   // tmd_model_free called while nsys > 0
};

struct tmd_system {
  const tmd_model *m = nullptr;
  cudaStream_t st = nullptr;
  long launches = 0;
  int natoms_cap = 0, n = 0;
  // ghost-aware mode (tmd_system_set_atoms_ghost): the last nghost of the n
  // atoms are LAMMPS ghosts, partners only (rows built, never evaluated)
  int nghost = 0;
  double skin = 1.0;
  bool have_box = false, have_atoms = false, have_v = false;
  bool forces_valid = false;
  tmd::BoxP box{};
  tmd::BinP bin{};
  int cap = 0, capp = 0;  // neighbor entries per atom, pow2 >= cap
  int ncell_alloc = 0;
  // multi-cell batch (ncells > 0): cell c holds atoms coff[c]..coff[c+1]-1
  // in its own periodic box; box/bin above are unused
  int ncells = 0, max_cells = 0;
  int nbins = 0;  // neighbor bins of all cells (CellGeom::bin0 numbering)
  std::vector<int> h_coff, h_acell;
  std::vector<tmd::BoxP> h_cbox;
  tmd::BoxP *cbox = nullptr;
  tmd::CellGeom *cgeom = nullptr;
  int *acell = nullptr, *coff = nullptr;
  double *cell_out = nullptr;  // [ncells][8]: energy, virial[6], spare
  int *cflag = nullptr;        // [max_cells] cells whose list must be rebuilt
  // device state
  double *x = nullptr, *v = nullptr, *f = nullptr, *xbuild = nullptr;
  int *image = nullptr, *elem = nullptr;
  int *cell_of = nullptr, *cell_count = nullptr, *cell_start = nullptr,
      *cell_cursor = nullptr, *cell_atoms = nullptr;
  uint32_t *tmp = nullptr, *nbr = nullptr;
  int *nraw = nullptr, *boff = nullptr, *rev = nullptr;
  float *P = nullptr, *G = nullptr, *dEdG = nullptr;
  double *E = nullptr;
  float4 *pdf = nullptr;
  float4 *pgeo = nullptr;   // [natoms_cap][cap][2] active-pair geometry (descriptor step)
  int *pcnt = nullptr;      // [natoms_cap][B] active pairs per (atom, element block)
  double *wv = nullptr, *eatom = nullptr, *vatom = nullptr, *ke = nullptr;
  double *partial = nullptr, *scal = nullptr;  // scal: [0] pe, [1..6] virial, [7] ke
  int *flag = nullptr, *status = nullptr;  // status[0] bits, status[1] longest row needed
  int *perm = nullptr, *tiles = nullptr;
  int ntiles = 0;
  double *thermo_d = nullptr;
  long thermo_alloc = 0;
  // host
  std::vector<int> h_elem;
  double *h_scal = nullptr;  // pinned [8]
  int *h_status = nullptr;   // pinned [2]
  // kernel form of the pair-force loop (kForce*), set by the default rule,
  // tmd_system_set_variant or tmd_system_autotune
  int force_variant = 0;
  int desc_variant = 0;    // kDesc*, the same way
  long long wait_probe = 0;  // tmd_system_set_wait_probe (failure-detection tests)
  // temperature-dependent model: electron temperature (eV), per-atom
  // entropy and free energy, and their totals of the last compute
  double etemp = 0.0;
  double *tdnp_s = nullptr, *tdnp_a = nullptr, *tdnp_tot = nullptr;  // tot: [2]
  double tdnp_S = 0.0, tdnp_A = 0.0;
  // kernel timing
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
  long prof_n[TMD_NPROF] = {0};
  double prof_ms[TMD_NPROF] = {0};
  cudaEvent_t cur_start = nullptr;
  // captured MD step (velocity Verlet + rebuild check/rebuild + force)
  cudaGraphExec_t step_exec = nullptr;
  double step_dt = 0.0;
  bool step_nvt = false;
  long step_launches = 0;
  long rebuild_launches = 0;      // kernels of the conditional rebuild body
  cudaStream_t st_aux = nullptr;  // captures the rebuild body
  // tmd_system_set_positions: the list rebuild in a conditional graph node,
  // launched only when the displacement check asks for it.  Its kernels are
  // counted once per rebuild that ran, from the device rebuild counter
  // (flag[1]) read with the status words.
  cudaGraphExec_t pos_exec = nullptr;
  long pos_rebuild_launches = 0;
  bool pos_pending = false;  // launched since the rebuild counter was last read
  int rb_seen = 0;           // the rebuild counter at that read
  // fix nvt: one Nose-Hoover chain per group (cell, or the whole system);
  // kept between runs of the same atoms like the fix's state in LAMMPS
  tmd::NhcState *nhc = nullptr;
  double *nhc_ke = nullptr;
  int nhc_alloc = 0, nhc_groups = 0;
  bool nhc_valid = false;
  // checkpoint of the dynamic state at the start of each chunk of MD steps
  double *ck_x = nullptr, *ck_v = nullptr, *ck_f = nullptr;
  int *ck_img = nullptr;
  tmd::NhcState *ck_nhc = nullptr;
  int ck_nhc_alloc = 0;
};

namespace tmd {

// Record msg as the thread's last error and return code.
int fail(int code, const std::string &msg);

#define TMD_CUDA(call)                                                        \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess)                                                    \
      return ::tmd::fail(TMD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  return cudaMalloc(reinterpret_cast<void **>(p), count * sizeof(T));
}

template <typename T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

void drop_graph(tmd_system *s);
void box_setup(BoxP &b, const double bx[9], const int pbc[3]);
void widths(const BoxP &b, double w[3]);
int alloc_neighbors(tmd_system *s, int cap);
// Take nbr/rev (natoms_cap x cap entries, filled on s->st) as the neighbor
// rows and re-allocate the per-entry scratch arrays (tmp, pdf, pgeo) at cap.
int adopt_rows(tmd_system *s, int cap, uint32_t *nbr, int *rev);
int initial_cap(tmd_system *s);
// Neighbor entries per atom for a number density (atoms / A^3): the atoms in
// the (rc + skin) sphere with a 30% margin plus 32, at least 64.
int cap_for_density(const tmd_system *s, double dens);
int read_status(tmd_system *s);
int clear_status(tmd_system *s);
int rebuild_now(tmd_system *s);
void launch_force_eval(tmd_system *s, float scale, bool want_vatom);
ForceArgs force_args(tmd_system *s, float scale, int variant);
DescArgs desc_args(tmd_system *s, int variant);
int default_desc_variant(const tmd_model *m);
// Kernel form of the force loop used when nothing chose one.
int default_force_variant(const tmd_model *m);
NbArgs nb_args(tmd_system *s);
// LAMMPS types (1-based) -> potential elements; TMD_ERR_ARG for unmapped types.
int map_types(const tmd_model *m, int n, const int *type, std::vector<int> &elem);
// Set n atoms' elements: host mirror, device elem[], MLP element grouping
// (perm, tiles).  Synchronises the stream.
int set_elements(tmd_system *s, int n, const int *elem);
// Multi-cell mode (batch.cpp): device arrays for up to max_cells cells, the
// cell layout (atoms per cell, concatenated), per-cell boxes.
int cells_alloc(tmd_system *s, int max_cells);
int cells_layout(tmd_system *s, int ncells, const int *natoms);
// Needs ncells and h_coff of the layout (bins per cell scale with its atoms).
int cells_geometry(tmd_system *s, const double *boxes, const int *pbc);
// Box and image-shift range of one cell; TMD_ERR_ARG with the reason in `why`
// for a degenerate box or one too small for the cutoff.
int cell_setup(const tmd_system *s, const double bx[9], const int pbc[3], BoxP &b,
               CellGeom &g, std::string &why);
// Make sure s->thermo_d holds count doubles.
int thermo_reserve(tmd_system *s, long count);
// fix nvt parameters, one target ramp per thermostat group (cell or system).
struct NvtSpec {
  const double *t_start, *t_stop;
  double t_damp;
};
// Velocity Verlet for nsteps on the device (graph-captured step), with the
// Nose-Hoover chain of fix nvt when nvt is given.  thermo_row(r) enqueues
// thermo row r; it is called for the starting state (r = 0) and every
// thermo_every steps and at the last step when thermo_every > 0.  On success
// the first thermo_count doubles of s->thermo_d are copied to thermo.
int run_md(tmd_system *s, int nsteps, double dt, const NvtSpec *nvt, int thermo_every,
           void (*thermo_row)(tmd_system *, int), double *thermo, long thermo_count);

}  // namespace tmd
