// tmd_kernels.h -- launch interfaces of the device kernels.
#pragma once

#include <vector>

#include "tmd_internal.h"

namespace tmd {

// status word bits set by kernels (read by the host after a step)
constexpr int kStatusOverflow = 1;   // neighbor row longer than cap
constexpr int kStatusShift = 2;      // image shift beyond +-3 cells
constexpr int kStatusOutside = 4;    // atom outside a non-periodic boundary
constexpr int kStatusNonfinite = 8;  // NaN/Inf energy or force
constexpr int kStatusTimeout = 16;   // a bounded device wait gave up
constexpr int kStatusLaunch = 32;    // a kernel launched without its shared memory

// Per-cell constants of the multi-cell neighbor build: perpendicular widths,
// the largest image shift per axis (0 on non-periodic axes) and the cell's
// grid of bins in fractional coordinates: nb bins per axis, a +-ns stencil
// reaching the cutoff, bins numbered from bin0 in the batch-wide bin arrays.
struct CellGeom {
  double w[3];
  int m[3];
  int nb[3];
  int ns[3];
  int bin0;
};

struct NbArgs {
  int n, B, cap, capp;
  KParams kp;
  BoxP box;
  BinP bin;
  double cutsq;
  double *x;
  int *image;
  const int *elem;
  int *cell_of, *cell_count, *cell_start, *cell_cursor, *cell_atoms;
  uint32_t *tmp;
  int *nraw;
  uint32_t *nbr;
  // multi-cell mode (ncells > 0): atoms of cell c are coff[c]..coff[c+1]-1,
  // each cell periodic in its own box with its own bins (CellGeom)
  int ncells;
  const BoxP *cbox;
  const CellGeom *cgeom;
  const int *acell, *coff;
  int *boff;
  int *rev;
  double *xbuild;
  int *flag, *status, *maxneed;
  // ghost-aware mode: atoms nlocal..n-1 are never evaluated; a build zeroes
  // their pair forces and virial partials (read by the gather as partners)
  int nlocal;
  float4 *pdf;
  double *wv;
  int *cflag;  // multi-cell mode: cells to rebuild (k_nbc_check), else nullptr
};

void launch_neighbor_build(const NbArgs &a, cudaStream_t st, long &launches);
// Displacement check: sets flag when an atom moved more than sqrt(trigsq)
// since the last build; in multi-cell mode (cflag) also marks the atom's cell.
void launch_neighbor_check(int n, const double *x, const double *xbuild,
                           double trigsq, int *flag, cudaStream_t st,
                           long &launches, const int *acell = nullptr, int *cflag = nullptr);
void launch_set_flag(int *flag, cudaStream_t st, long &launches);
// One thread: sets an IF node's condition of a captured graph to flag[0] != 0.
void launch_rebuild_cond(cudaGraphConditionalHandle h, const int *flag, cudaStream_t st,
                         long &launches);
// Positions from a caller's frame: each atom to the periodic image nearest its
// position at the last list build (cbox/acell in multi-cell mode, else box).
void launch_nearest_image(int n, double *x, const double *xbuild, const BoxP &box,
                          const BoxP *cbox, const int *acell, cudaStream_t st, long &launches);

// Descriptor: P[n][B][K][D], G[n][B*K*M].
// Kernel forms: K/4 lanes per atom with 4 filters each (k_descriptor), or
// min(K, 32) lanes per atom with K/min(K, 32) filters each and the monomials
// of each pair computed once (k_descriptor_w).
constexpr int kDescFilter4 = 0;
constexpr int kDescWide = 1;
constexpr int kDescWide2 = 2;  // two pair streams per atom, 2+ filters per lane
constexpr int kDescSplit = 3;  // geometry kernel + contraction kernel
constexpr int kDescVariants = 4;
struct DescArgs {
  int n, cap;
  KParams kp;
  BoxP box;
  const double *x;
  const int *elem;
  const uint32_t *nbr;
  const int *boff;
  float *P, *G;
  const BoxP *cbox;   // multi-cell mode: box of each cell, else nullptr
  const int *acell;   // multi-cell mode: cell of each atom
  int variant;        // kDesc*
  // per-pair outputs for the force step: zero pair force of every list entry
  // beyond rc (pdf[n][cap]), compact geometry of the active pairs
  // (pgeo[n][cap][2], element block by element block) and their number per
  // (atom, block) (pcnt[n][B])
  float4 *pdf, *pgeo;
  int *pcnt;
};
void launch_descriptor(const DescArgs &a, cudaStream_t st, long &launches);

// MLP forward + backward over element-grouped tiles.
struct MlpLayer {
  int K, N;
  const float *W;  // [K][N] row-major (npz weights_e_l)
  const float *b;  // [N] or nullptr
  // output layer only: FP64 copies, the atomic energy is formed in FP64
  const double *Wd;
  const double *bd;
  // streamed-weight form only (hidden layers): W packed [N/128][K][128] and
  // W^T packed [K/128][N][128] (mlp_fp32s_pack)
  const float *Wp;
  const float *Wtp;
};
struct MlpArgs {
  int nl, actfn, resnet, nin, maxh;
  int tr;             // atoms per tile (32 or 64 streamed, 64 or 128 resident)
  size_t smem;        // dynamic shared memory bytes
  int resident;       // > 0: resident-weight form, persistent grid of this many CTAs
  int warped;         // > 0: warp-tile form, this many warps per CTA (tiles of 32 per warp)
  int streamed;       // > 0: streamed-weight form, persistent grid of this many CTAs
  int stages;         // its weight-chunk stages
  int *status;        // timeout bit of the streamed form's bounded waits
  int ntiles;
  const int *tiles;   // [ntiles][3] = (element, start, count) into perm
  const int *perm;    // atom indices grouped by element
  const float *G;     // [n][nin]
  float *dEdG;        // [n][nin]
  double *E;          // [n] atomic energies (FP64 output layer)
  // per element, per layer (host table copied into a device param block)
  const MlpLayer *layers;  // [nelt][nl] device array
};
void launch_mlp_fp32(const MlpArgs &a, cudaStream_t st, long &launches);
size_t mlp_fp32_smem(int nl, const int *sizes, int tr);
// Resident-weight form: shared memory per CTA for tiles of tr atoms (128
// atoms on 512 threads, or 64 on 256 when the wider tile does not fit).
size_t mlp_fp32r_smem(int nl, const int *sizes, int tr);
// Warp-tile form (64-wide hidden layers, no residual layers): shared memory
// per CTA of `warps` warps, 0 if the form does not apply.
size_t mlp_fp32w_smem(int nl, const int *sizes, int resnet, int warps);
int mlp_fp32w_rows();  // atoms per warp tile
void mlp_fp32w_prepare(size_t smem);
void mlp_fp32_prepare(int tr, size_t smem, bool resident);
// Streamed-weight form (weights too large for shared memory): dynamic shared
// memory and weight stages, 0 if unsupported (residual layers, widths not
// multiples of 32); host packing of one layer's W into its chunk layouts.
size_t mlp_fp32s_smem(int nl, const int *sizes, int resnet, int *stages);
void mlp_fp32s_pack(const float *W, int K, int N, std::vector<float> &fwd,
                    std::vector<float> &bwd);
void mlp_fp32s_prepare(size_t smem);

// Tensor-core (tcgen05) MLP, BF16 operands (TF32 in the 3xTF32 streamed
// form).  Weights are packed on the host in chunks of the K-major
// core-matrix layout: 64 BF16 columns (pack_core_chunks) or 32 TF32 columns
// (pack_core_chunks_tf32).
struct MlpTcLayer {
  int K, N;
  const void *Wf;    // forward B = W^T: N rows x K cols (bf16, packed; the lo
                     // block of the split form follows the hi block)
  const void *Wb;    // backward B = W: K rows x N cols (bf16, packed, same)
  const float *b;    // [N] bias (hidden layers)
  const double *wd;  // output layer weights (FP64), last layer only
  const double *bd;  // output bias (FP64) or nullptr, last layer only
  float wscale;      // FP8 form: packed weights are e4m3(W * wscale); 1 otherwise
};
struct MlpTcArgs {
  int nl, actfn, resnet, nin, maxh, ntiles;
  const int *tiles, *perm;
  const float *G;
  float *dEdG;
  double *E;
  const MlpTcLayer *layers;  // [nelt][nl] device array
  int *status;
  size_t smem;
  int dz_bf16;
  int np;  // 1: BF16 products; 3: split BF16 (hi*hi + hi*lo + lo*hi)
  int tf32;  // 1: split TF32 operands (3xTF32, np = 3; streamed form only)
  int hi2;   // 3xTF32: a second accumulator for the odd K steps' hi products
  int persistent;     // > 0: weight-resident persistent form on this many CTAs
  size_t smem_p;      // its dynamic shared memory
  int dz_bf16_p;      // its act' in BF16 (BF16 form only, when FP32 does not fit)
  int streamed;       // > 0: streamed-weight persistent form on this many CTAs
  size_t smem_s;      // its dynamic shared memory
  int stages;         // its weight-chunk stages
  int cps_s;          // its CTAs per SM (2: 256 threads, act' as packed BF16 in TMEM)
  // > 0: failure-detection hook (tmd_system_set_wait_probe): every CTA first
  // waits at most this many cycles on one of its mbarriers before issuing any
  // MMA or copy; nothing arrives on it, so the kernel takes its timeout path
  // with no asynchronous work in flight and reports kStatusTimeout
  long long probe_wait;
};
void launch_mlp_tc(const MlpTcArgs &a, cudaStream_t st, long &launches);

// ---- temperature-dependent model (tdnp.cu) ----
// One layer of a TDNP net: W (K x N), WT (N x K), b (N or null); for the
// last layer of U and S also Wf (FP32) / Wd (FP64) row sums over the outputs
// and bd the summed bias (FP64).
struct TdnpLayer {
  int K, N;
  const float *W, *WT, *b, *Wf;
  const double *Wd;
  double bd;
};
struct TdnpArgs {
  int n, nin, ydim, maxw, nelt;
  int nl[3], actfn[3], resnet[3];    // H, U, S
  const TdnpLayer *layers;           // [net][element][kMaxLayers]
  const int *elem;
  const float *G;
  float *dEdG;
  double *E, *Sa, *Aa;               // per atom: u, s, u - T s
  float T, c;                        // electron temperature (eV); T or T^2 (Sommerfeld)
  int sommerfeld;
  size_t warp_floats;                // shared memory per warp (floats)
};
size_t tdnp_warp_floats(const int nl[3], int maxw);
// 0, or -1 when the nets need more shared memory than a CTA has.
int launch_mlp_tdnp(const TdnpArgs &a, cudaStream_t st, long &launches);
size_t mlp_tc_smem(int nl, int maxh, int resnet, bool dz_bf16, int np);
void mlp_tc_prepare(size_t smem, bool dz_bf16, int np);
// Persistent form: dynamic shared memory for sizes[0..nl], 0 if unsupported
// (residual layers).
size_t mlp_tcp_smem(int nl, const int *sizes, int resnet, int np, bool dz_bf16);
void mlp_tcp_prepare(size_t smem, int np, bool dz_bf16);
// Streamed-weight persistent form (weights too large to stay in shared
// memory): dynamic shared memory and weight stages, 0 if unsupported
// (residual layers, widths not multiples of the chunk (64 BF16 / 32 TF32
// columns) or above 256, act' beyond 512 TMEM columns).  tf32 = 1: the
// 3xTF32 operand format.
size_t mlp_tcs_smem(int nl, const int *sizes, int resnet, int np, int tf32, int cps,
                    int *stages);
void mlp_tcs_prepare(size_t smem, int np, int tf32, int cps);
// 3xTF32: 1 when TMEM holds a second hi accumulator (MlpTcArgs::hi2).
int mlp_tcs_hi2(int nl, const int *sizes, int np, int tf32);

// Host: pack a rows x cols matrix (element (r, k) = src[r * ld_r + k * ld_k])
// into 64-column chunks of 8x8 BF16 core matrices, K-major.
void pack_core_chunks(const float *src, int rows, int cols, long ld_r, long ld_k,
                      uint16_t *dst);
// Host: the same into 32-column chunks of 8x4 TF32 core matrices; part 0 =
// hi = tf32(v), part 1 = lo = tf32(v - hi) (round to nearest, ties away).
void pack_core_chunks_tf32(const float *src, int rows, int cols, long ld_r, long ld_k, int part,
                           float *dst);
float tf32_round_host(float v);

// FP8 (e4m3) form of the tensor-core MLP (mlp_fp8.cu): same arguments, packed
// weights e4m3(W * wscale) in 8x16 core matrices, per-row operand scales.
void launch_mlp_fp8(const MlpTcArgs &a, cudaStream_t st, long &launches);
size_t mlp_fp8_smem(int nl, int maxh, int resnet, bool dz_bf16);
void mlp_fp8_prepare(size_t smem, bool dz_bf16);
void pack_core_chunks_fp8(const float *src, int rows, int cols, long ld_r, long ld_k,
                          float scale, uint8_t *dst);

// Force: per-pair dE_i/dx_j into pdf, per-atom virial partials.
// Kernel forms: K/4 lanes per atom with 4 filters each (k_force), or W lanes
// per atom with whole pairs per lane (k_force_pl, W = 8, 16, 32).
constexpr int kForceFilterLane = 0;
constexpr int kForcePairLane8 = 1;
constexpr int kForcePairLane16 = 2;
constexpr int kForcePairLane32 = 3;
constexpr int kForceVariants = 4;
struct ForceArgs {
  int n, cap;
  KParams kp;
  BoxP box;
  float scale;
  const double *x;
  const int *elem;
  const uint32_t *nbr;
  const int *boff;
  // S = dE/dP is formed per (atom, block) from the descriptor moments P
  // [n][B][K][D] and the MLP rows G, dE/dG [n*B*K][M] (dedp_row)
  const float *P, *G, *dEdG;
  float4 *pdf;
  double *wv;  // [n][6] per-atom sum of -r_ij (x) df over own pairs
  const BoxP *cbox;   // multi-cell mode (as DescArgs)
  const int *acell;
  int variant;        // kForce*
  const float4 *pgeo;  // active pairs from the descriptor step (pair-lane forms)
  const int *pcnt;
};
void launch_force(const ForceArgs &a, cudaStream_t st, long &launches);

// Gather: f_i = sum_t pdf[t] - pdf[rev[t]] (FP64), optional per-atom virial.
struct GatherArgs {
  int n, cap, B;
  const int *boff;
  const float4 *pdf;
  const int *rev;
  const uint32_t *nbr;
  const double *x;
  BoxP box;
  const double *wv;
  double *f;
  double *vatom;   // nullable
  const BoxP *cbox;   // multi-cell mode (as DescArgs)
  const int *acell;
};
void launch_gather(const GatherArgs &a, cudaStream_t st, long &launches);

// Deterministic FP64 reductions: out[c] = sum_i in[i*ncomp + c] (in FP64 or
// FP32 input).  partial has >= 1024*ncomp doubles.
void launch_reduce_f64(const double *in, int n, int ncomp, double *partial,
                       double *out, cudaStream_t st, long &launches);
void launch_reduce_scaled(const double *in, int n, double *partial, double *out,
                          double scale, cudaStream_t st, long &launches);
// Per-cell sums in a fixed order: out[c*ostride + k] = scale * sum over the
// atoms a of cell c of in[a*ncomp + k].
void launch_cell_sum(int ncells, const int *coff, const double *in, int ncomp,
                     double scale, double *out, int ostride, cudaStream_t st,
                     long &launches);
void launch_scale_copy(const double *in, int n, double scale, double *out,
                       cudaStream_t st, long &launches);

// ---- serving: per-cell control of mixed jobs in one multi-cell system ----
constexpr int kJobEnergy = 0;  // one force evaluation, atoms fixed
constexpr int kJobNve = 1;     // velocity Verlet, `left` steps
constexpr int kJobFire = 2;    // FIRE relaxation until max |F| < fmax or `left` runs out

struct CellCtl {
  int mode;      // kJob*
  int left;      // NVE steps / FIRE iterations still to run
  int nneg;      // FIRE: iterations in a row with P = F.v <= 0
  int conv;      // FIRE: converged (max |F|^2 < fmax2) or stopped
  int it;        // FIRE: iterations begun
  int phase;     // FIRE: 1 = stepped back, forces of the new positions pending
  int last_neg;  // FIRE: last iteration with P <= 0
  int plan;      // FIRE: move of the current step (kFirePlan*)
  double dt;     // NVE step; FIRE current step (ps)
  double dtmax, dtmin;  // FIRE step limits
  double alpha;  // FIRE mixing parameter
  double fmax2;  // FIRE convergence threshold, (eV/A)^2
  double mix1, mix2;  // FIRE velocity mixing of the current step
  double dtv;    // FIRE step of the current move after the dmax limit
};

// FIRE moves of one step of a cell (server_kernels.cu)
constexpr int kFirePlanNone = 0;
constexpr int kFirePlanMix = 1;    // P > 0: Euler kick, mix, drift
constexpr int kFirePlanBack = 2;   // P <= 0: half step back, v = 0 (forces re-evaluated)
constexpr int kFirePlanReset = 3;  // after a reset: v = dt F / m, drift


// New layout of a server batch: atom a of new cell c comes from old atom
// src[c] + (a - coff[c]) when src[c] >= 0, else from staging slot
// -src[c] - 1 + (a - coff[c]) (new requests; image counters start at 0).
// A moved cell keeps its neighbor list: rows (cap0 entries per atom in the
// old arrays, cap1 in the new ones) are copied with their atom indices and
// partner slots re-based to the new offsets, unless fresh[c] is set (the
// cell is about to be rebuilt).
struct SrvMove {
  int n, B, cap0, cap1;
  const int *acell, *coff, *src, *fresh;
  const double *x, *v, *f, *xb;
  const int *img, *elem, *boff, *rev;
  const uint32_t *nbr;
  const double *sx, *sv;
  const int *selem;
  double *x2, *v2, *f2, *xb2;
  int *img2, *elem2, *boff2, *rev2;
  uint32_t *nbr2;
};
void launch_srv_move(const SrvMove &m, cudaStream_t st, long &launches);
// acell[a] = c for every atom of cell c.
void launch_srv_acell(int ncells, const int *coff, int *acell, cudaStream_t st,
                      long &launches);
// MLP element grouping of a batch: perm lists the atoms of element 0 in cell
// order, then element 1, ...; estart[c*B + e] is where cell c's atoms of
// element e begin (the order a counting sort over all atoms gives).
void launch_srv_perm(int ncells, int B, const int *coff, const int *elem, const int *estart,
                     int *perm, cudaStream_t st, long &launches);
// Rebuild request for the fresh cells: cflag[c] = fresh[c], *flag = 1.
void launch_srv_mark(int ncells, const int *fresh, int *cflag, int *flag, cudaStream_t st,
                     long &launches);
// One serving step, before the force evaluation: FIRE power (F.v, v.v, F.F)
// summed per cell and the largest velocity and force/mass components per
// cell, the FIRE plan of each cell, then the position update of NVE (half
// kick + drift) and FIRE (mix + Euler, or step back) cells.  pw: 3 doubles
// per atom, pm: 2 per atom, csum: 4 per cell, cmax: 2 per cell.
void launch_srv_pre(int n, int ncells, const int *acell, const int *coff, CellCtl *ctl,
                    double *x, double *v, const double *f, const int *elem,
                    const double *mass_e, double *pw, double *pm, double *csum,
                    double *cmax, cudaStream_t st, long &launches);
// After the force evaluation: NVE second half kick (kick != 0), per-cell
// max |F|^2, step bookkeeping (count != 0) and FIRE convergence.
void launch_srv_post(int n, int ncells, const int *acell, const int *coff, CellCtl *ctl,
                     double *v, const double *f, const int *elem, const double *mass_e,
                     double *fsq, double *cfmax, int kick, int count, cudaStream_t st,
                     long &launches);

// ---- fix nvt: Nose-Hoover chain thermostat per group of atoms ----
// (FixNH, fix_nh.cpp: chain of 3, one loop, no drag).  A group is a whole
// system or one cell of a batch; goff[g]..goff[g+1]-1 are its atoms.
constexpr int kNhcChain = 3;
struct NhcState {
  double eta[kNhcChain], eta_dot[kNhcChain + 1], eta_dotdot[kNhcChain], eta_mass[kNhcChain];
  double t_current, t_target, ke_target, tdof, t_freq;
  double t_start, t_stop;  // linear ramp of the target over the run
  double dt, factor;       // step; velocity factor of the last chain update
  int step, nsteps;        // steps run in this run / its length
};
// FixNH::setup: temperature from the group's kinetic energy, target, masses.
void launch_nhc_setup(int ngroups, NhcState *st, const double *ke_group, cudaStream_t s,
                      long &launches);
// initial_integrate (step += 1, target of this step) or final_integrate
// (temperature from ke_group): one chain update per group, then v of every
// atom scaled by its group's factor (acell = group of each atom, or nullptr
// for a single group).
void launch_nhc_half(int ngroups, NhcState *st, const double *ke_group, int n,
                     const int *acell, double *v, cudaStream_t s, long &launches);

// Velocity Verlet halves (fix_nve.cpp:64-141).
void launch_nve_initial(int n, double *x, double *v, const double *f,
                        const int *elem, const double *mass_e, double dtf,
                        double dtv, cudaStream_t st, long &launches);
void launch_nve_final(int n, double *v, const double *f, const int *elem,
                      const double *mass_e, double dtf, cudaStream_t st,
                      long &launches);
void launch_kinetic(int n, const double *v, const int *elem,
                    const double *mass_e, double *ke_atom, cudaStream_t st,
                    long &launches);
void launch_check_finite(int n, const double *f, const double *etot,
                         int *status, cudaStream_t st, long &launches);

}  // namespace tmd
