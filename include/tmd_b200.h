/* tmd_b200.h -- C ABI of the B200 (sm_100a) force path of pair_style tensormd.
 *
 * A drop-in for the path PairTensorMD::compute -> TensorMD::calc_tensor_density
 * -> TensorMD::run (src/ML-TENSORMD/pair_tensormd.cpp:141-184,
 * tensormd.cpp:369-615): neighbor list -> tensor-moment descriptor ->
 * per-element MLP and its backward -> forces/virial -> velocity Verlet.
 *
 * Conventions
 *   - Every entry point returns an int status: TMD_OK (0) or a negative code.
 *     Nothing throws across the ABI; tmd_last_error() returns the message of
 *     the last failure on the calling thread.
 *   - The caller owns host arrays; the library owns device memory.  One CUDA
 *     stream per system; a handle is used from one host thread at a time.
 *   - Units are LAMMPS "metal": Angstrom, eV, ps, g/mol.
 *   - box[9] = {xlo, ylo, zlo, xprd, yprd, zprd, xy, xz, yz} (LAMMPS
 *     triclinic convention: a = (xprd,0,0), b = (xy,yprd,0), c = (xz,yz,zprd)).
 *   - virial[6] and vatom rows are ordered xx, yy, zz, xy, xz, yz with
 *     W = -sum_pairs r_ij (x) dE_i/dx_j, the value LAMMPS virial_fdotr_compute
 *     (src/pair.cpp:1735-1776) returns for this pair style.
 */
#ifndef TMD_B200_H
#define TMD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define TMD_OK 0
#define TMD_ERR_ARG (-1)       /* invalid argument */
#define TMD_ERR_CUDA (-2)      /* CUDA runtime error (message has the call) */
#define TMD_ERR_MODEL (-3)     /* potential file missing keys / unsupported */
#define TMD_ERR_CAPACITY (-4)  /* atom or neighbor capacity exceeded */
#define TMD_ERR_NONFINITE (-5) /* NaN/Inf in energies or forces */
#define TMD_ERR_IO (-6)        /* cannot open or parse a file */
#define TMD_ERR_STATE (-7)     /* call order (e.g. compute before set_atoms) */
#define TMD_ERR_TIMEOUT (-8)   /* a bounded device wait gave up */

/* MLP arithmetic of a loaded model.  FP32 is the plain form (FP32 arithmetic,
 * FP64 cutoff test, energy/virial sums and position update). */
#define TMD_PREC_FP32 0
#define TMD_PREC_BF16 1
#define TMD_PREC_FP8 2    /* e4m3 tensor-core MLP, per-layer weight and per-row operand scales */
#define TMD_PREC_BF16X3 3 /* split BF16 products: FP32-class accuracy */
#define TMD_PREC_TF32X3 4 /* split TF32 products (3xTF32) on tcgen05: FP32 accuracy */

typedef struct tmd_model tmd_model;
typedef struct tmd_system tmd_system;

/* pair_coeff arguments after "* *":  "file.npz El1 El2 ... [interp dx]
 * [cmax exact|default] [precision fp32|tf32x3|bf16|bf16x3|fp8]".
 * Replaces PairTensorMD::coeff + read_potential_file + TensorMD::read_npz /
 * setup_global / setup_interpolation (pair_tensormd.cpp:214-317,376-399;
 * tensormd.cpp:109-280,438-446).  The element list maps LAMMPS atom types
 * 1..n to potential elements exactly as PairTensorMD::setup_eltmap
 * (pair_tensormd.cpp:349-370).  `device` is the CUDA ordinal. */
int tmd_model_load(const char *coeff_args, int device, tmd_model **out);

/* Free a model.  If systems created from it are still alive, the model is
 * released when the last of them is freed (any free order is safe). */
void tmd_model_free(tmd_model *model);

/* Model facts: cutmax (PairTensorMD::init_one, pair_tensormd.cpp:336-341),
 * number of elements of the potential, number of LAMMPS types mapped,
 * descriptor width (b*k*m), filters k, moments m.  Any pointer may be NULL. */
int tmd_model_info(const tmd_model *model, double *cutmax, int *nelt,
                   int *ntypes, int *n_desc, int *num_filters, int *mmax);

/* map[t] (t = 1..ntypes) -> potential element index, -1 if unmapped
 * (PairTensorMD::map); mass[t] -> mass the potential file gives that type
 * (PairTensorMD::coeff sets atom->mass from it, pair_tensormd.cpp:303-312).
 * Arrays have ntypes+1 entries; index 0 is unused. */
int tmd_model_type_map(const tmd_model *model, int *map, double *mass);

/* A device-resident periodic cell of up to natoms_cap atoms.  skin is the
 * neighbor skin (LAMMPS `neighbor <skin> bin`); the list cutoff is
 * cutmax + skin. */
int tmd_system_create(const tmd_model *model, int natoms_cap, double skin,
                      tmd_system **out);
void tmd_system_free(tmd_system *sys);

/* Box (see conventions) and periodic flags; forces a neighbor rebuild. */
int tmd_system_set_box(tmd_system *sys, const double box[9], const int pbc[3]);

/* Upload n atoms: x[n*3] positions, type[n] LAMMPS types (1-based, mapped
 * through the pair_coeff element list), v[n*3] velocities (may be NULL).
 * Types are fixed until the next call.  Positions outside the box are
 * wrapped by the next neighbor rebuild as Domain::pbc() does. */
int tmd_system_set_atoms(tmd_system *sys, int n, const double *x,
                         const int *type, const double *v);

/* Replace positions only (same n and types); the cheap per-step upload of
 * the LAMMPS drop-in.  The positions may be in any periodic frame (wrapped by
 * the caller at its own times, or never): each atom takes the periodic image
 * nearest its position at the last neighbor build, so the list stays valid
 * and only real motion (more than skin/2) triggers a rebuild.  The upload,
 * the displacement check and a rebuild are queued on the system's stream and
 * the call returns without waiting (the rebuild sits in a conditional graph
 * node: a call that needs none launches none of its kernels).  From pinned
 * (page-locked) host memory the copy runs asynchronously: keep x unchanged
 * until the next tmd_compute returns. */
int tmd_system_set_positions(tmd_system *sys, const double *x);

/* Ghost-aware mode for domain-decomposed (multi-rank) LAMMPS runs, in place
 * of tmd_system_set_box + tmd_system_set_atoms.  x[nall*3], type[nall] with
 * nall = nlocal + nghost are LAMMPS's atom->x and atom->type: the rank's
 * local atoms first, then its ghosts (copies of other ranks' atoms and
 * periodic images, placed by LAMMPS's border exchange out to the ghost
 * cutoff, which must reach cutmax + skin).  The reference evaluates the
 * local atoms over LAMMPS's full list with ghosts
 * (pair_tensormd.cpp:141-184,321-330) and writes forces on local and ghost
 * atoms for reverse communication (kernel.cu:1760-1789); here the system
 * becomes non-periodic (its box is the atoms' bounding box plus cutmax +
 * skin on each side), neighbor rows are built for all nall atoms (the same
 * neighbor set as LAMMPS's list of the local atoms) and evaluated for the
 * local ones.  tmd_compute then fills f[nall*3] (forces on the ghosts
 * included, for LAMMPS to reverse-communicate), the energy of the local
 * atoms, the virial of their pairs (LAMMPS's fdotr sum over local and ghost
 * atoms), eatom[nall] (ghosts 0) and vatom[nall*6].  Until the next call,
 * tmd_system_set_positions takes nall positions in the same order (LAMMPS's
 * forward communication between reneighborings).  tmd_nve_run and
 * tmd_nvt_run are refused in this mode (LAMMPS integrates); tmd_system_
 * set_atoms leaves it. */
int tmd_system_set_atoms_ghost(tmd_system *sys, int nlocal, int nghost, const double *x,
                               const int *type);

/* Download state; NULL pointers are skipped.  image[n*3] are the periodic
 * image counters accumulated by wrapping (Domain::pbc image flags). */
int tmd_system_get(tmd_system *sys, double *x, double *v, double *f,
                   int *image);

/* One force evaluation: PairTensorMD::compute(eflag, vflag).  Outputs (any
 * may be NULL, which leaves the value on the device): energy (eng_vdwl),
 * virial[6], f[n*3], eatom[n], vatom[n*6].  scale is the pair_coeff scale
 * factor of fix adapt (1.0 normally; PairTensorMD::extract("scale")). */
int tmd_compute(tmd_system *sys, int eflag, int vflag, double scale,
                double *energy, double *virial, double *f, double *eatom,
                double *vatom);

/* nsteps of velocity Verlet (FixNVE initial/final_integrate,
 * fix_nve.cpp:64-141, metal units) driven as Verlet::run does
 * (verlet.cpp:229-349), positions and velocities resident on the device,
 * neighbor rebuild when an atom moved more than skin/2 (neigh_modify every 1
 * delay 0 check yes).  If thermo is not NULL it receives (pe, ke) after
 * every thermo_every-th step and the last one: rows = nsteps/thermo_every
 * (+1 if nsteps % thermo_every != 0).  dt in ps. */
int tmd_nve_run(tmd_system *sys, int nsteps, double dt, int thermo_every,
                double *thermo);

/* nsteps of `fix nvt temp t_start t_stop t_damp` (FixNH, fix_nh.cpp:741-930,
 * 1758-1822): velocity Verlet with a Nose-Hoover chain thermostat of 3
 * (tchain 3, tloop 1, drag 0: the fix's defaults), target temperature ramped
 * linearly from t_start to t_stop over the run, temperature with 3N - 3
 * degrees of freedom (compute temp).  The chain state is kept between runs on
 * the same atoms, as the fix keeps it between LAMMPS runs; set_atoms starts a
 * fresh one.  Temperatures in K, t_damp and dt in ps; thermo as tmd_nve_run. */
int tmd_nvt_run(tmd_system *sys, int nsteps, double dt, double t_start,
                double t_stop, double t_damp, int thermo_every, double *thermo);
/* Energy of the thermostat chain after the last nvt run (what `thermo` prints
 * as f_ID of fix nvt, FixNH::compute_scalar, fix_nh.cpp:1447-1473): one value
 * for a system, one per cell for the system of a batch.  pe + ke + this is
 * the conserved quantity of the thermostatted dynamics. */
int tmd_nvt_energy(tmd_system *sys, double *energy);

/* Export the current full neighbor list with cutoff `cut` (<= cutmax +
 * skin) for parity checks: counts[n]; entries[total*4] = (j, sx, sy, sz)
 * where the neighbor is atom j shifted by sx*a + sy*b + sz*c.  Pass
 * entries = NULL to get the total in *total only.  cap = entries capacity. */
int tmd_neighbor_list(tmd_system *sys, double cut, int *counts, int *entries,
                      long cap, long *total);

/* Per-atom descriptors G[n * n_desc] (compute tensormd/density,
 * compute_tensormd_density.cpp:129-200: array_atom[i] = the atom's MLP input
 * row, b*k*m order) of the current positions, in atom order; the descriptor
 * kernel runs for the call.  In ghost-aware mode, the nlocal local atoms'
 * rows only. */
int tmd_get_descriptors(tmd_system *sys, double *G);

/* Kernel forms of the pair loops.  The reference has one implementation per
 * phase (kernel.cu); here a phase may have several kernels that compute the
 * same quantities with different thread mappings, and the fastest depends on
 * the potential's shape (filters, monomials, elements) and the neighbor
 * count.  Family TMD_TUNE_FORCE (the pair-force loop, kernel.cu:541-631):
 *   0  K/4 lanes per atom, 4 filters per lane, partial forces summed over lanes
 *   1  8 lanes per atom, one whole pair per lane, dE/dP staged in shared memory
 *   2  16 lanes per atom, as 1
 *   3  32 lanes per atom, as 1
 * Family TMD_TUNE_DESCRIPTOR (the moment contraction P = sum H M,
 * kernel.cu:1105, with G = T P^2):
 *   0  K/4 lanes per atom, 4 filters per lane
 *   1  min(K, 32) lanes per atom, K/min(K, 32) filters per lane, monomials of
 *      a pair computed once and shared through shared memory, G formed in
 *      the same kernel
 *   2  as 1, the atom's lanes split into two streams that take alternate
 *      pairs, 2K/min(K, 32) filters per lane (K = 4..64; other K run form 1)
 *   3  split: the pair geometry of every list entry in a kernel of its own
 *      (warp per atom, compact active pairs), then the contraction of form 1
 *      over the compact pairs
 * The forms agree to FP32 rounding (summation order).  set_variant picks one;
 * autotune runs one evaluation, times reps launches of every form of the
 * family on the system's current atoms, keeps the fastest and recomputes the
 * results with it; ms (may be NULL) receives the mean device milliseconds per
 * launch of each form (4 force forms, 4 descriptor forms; at most
 * TMD_TUNE_VARIANTS). */
#define TMD_TUNE_FORCE 0
#define TMD_TUNE_DESCRIPTOR 1
#define TMD_TUNE_VARIANTS 4
int tmd_system_set_variant(tmd_system *sys, int family, int variant);
int tmd_system_get_variant(tmd_system *sys, int family, int *variant);
int tmd_system_autotune(tmd_system *sys, int family, int reps, double *ms);

/* CUDA stream of the system (cudaStream_t as void*), for event timing. */
int tmd_system_stream(tmd_system *sys, void **stream);

/* Number of kernels the library launched since the system was created. */
long tmd_system_launches(const tmd_system *sys);

/* Neighbor-list rebuilds the system has run since it was created (forced
 * ones at set_atoms included, and the displacement-triggered ones inside MD
 * runs: LAMMPS's "Neighbor list builds" count).  Waits for the stream. */
int tmd_system_rebuilds(tmd_system *sys, long *count);

/* Temperature-dependent potentials (tdnp = 1 files, TDNP in tdnp.cpp): the
 * electron temperature in eV (pair_coeff keyword etemp gives it in K, as
 * pair_tensormd.cpp:245-246; fix tensormd/etemp sets pair->etemp between
 * steps, fix_tensormd_etemp.cpp:80-89).  With such a potential tmd_compute's
 * energy is the internal energy U and its forces those of the free energy
 * A = U - T S (tdnp.cpp:167-226); tmd_system_tdnp_energies returns S and A
 * of the last compute (PairTensorMD::eentropy, free_energy), times scale. */
int tmd_system_set_etemp(tmd_system *sys, double etemp_ev);
int tmd_system_tdnp_energies(tmd_system *sys, double *entropy, double *free_energy);

/* Failure-detection hook for tests (no reference counterpart).  With
 * cycles > 0 the system's tensor-core MLP kernels (precision tf32x3, bf16, bf16x3,
 * fp8) start every CTA with a wait of at most `cycles` clock cycles on one
 * of their mbarriers, before any MMA or copy is issued; nothing arrives on
 * it, so each CTA takes its timeout path (no asynchronous work in flight,
 * TMEM freed) and tmd_compute returns TMD_ERR_TIMEOUT with the context still
 * usable.  cycles = 0 (the default) turns it off; the FP32 MLP has no waits. */
int tmd_system_set_wait_probe(tmd_system *sys, long long cycles);

/* Measured FP32 issue peak of a device: a packed-FMA (FFMA2) kernel with
 * eight independent chains per thread on every SM, `reps` timed launches
 * (CUDA events) after one warm-up, best of them, in TFLOP/s (2 FLOP per
 * FMA).  The denominator of the FP32 rooflines; no reference counterpart.
 * Uses its own stream and returns after it has finished. */
int tmd_fp32_peak(int device, int reps, double *tflops);

/* Kernel timing (TensorMDTimer's phase report, tensormd_timer.h:25-46, with
 * CUDA events instead of host clocks).  enable != 0 records an event pair
 * around every kernel family on the system stream during tmd_compute and
 * tmd_nve_run; tmd_profile_read returns, per family, the number of launches
 * and the summed device milliseconds since the last reset.  Families:
 * 0 neighbor build, 1 descriptor, 2 mlp, 3 force, 4 gather, 5 nve+check,
 * 6 reductions, 7 dE/dP (no launches: the force kernels form dE/dP per
 * atom).  Arrays hold TMD_NPROF entries. */
#define TMD_NPROF 8
int tmd_profile_enable(tmd_system *sys, int enable);
int tmd_profile_read(tmd_system *sys, long *launches, double *ms, int reset);

/* Copy the message of the last failed call on this thread into buf. */
int tmd_last_error(char *buf, int len);

/* ---- Multi-cell batches ---------------------------------------------------
 * Many independent small periodic systems ("cells", e.g. 4096 cells of 256
 * atoms) evaluated together: one launch per kernel over all cells.  The
 * reference runs one LAMMPS system per process (pair_tensormd.cpp:141-184);
 * a batch of C cells gives, cell by cell, the results of C separate systems
 * (tmd_system_*), with per-cell energies, virials and thermo.
 *
 * Atom arrays are concatenated cell by cell: cell c holds natoms[c] atoms
 * starting at sum(natoms[0..c-1]).  Each cell has its own box[9] and pbc[3]
 * (conventions above); a cell may be smaller than the cutoff (up to 3 images
 * per axis).  tmd_batch_system() returns the underlying system handle for
 * tmd_system_stream / launches / profile / get / neighbor_list /
 * get_descriptors; its tmd_compute gives the sum over cells. */
typedef struct tmd_batch tmd_batch;
int tmd_batch_create(const tmd_model *model, int ncells, const int *natoms,
                     double skin, tmd_batch **out);
void tmd_batch_free(tmd_batch *batch);
int tmd_batch_system(tmd_batch *batch, tmd_system **sys);
/* boxes[ncells*9], pbc[ncells*3]. */
int tmd_batch_set_cells(tmd_batch *batch, const double *boxes, const int *pbc);
/* x[N*3], type[N], v[N*3] or NULL, N = total atoms of the batch. */
int tmd_batch_set_atoms(tmd_batch *batch, const double *x, const int *type,
                        const double *v);
int tmd_batch_get(tmd_batch *batch, double *x, double *v, double *f, int *image);
/* energy[ncells], virial[ncells*6], f[N*3]; any may be NULL. */
int tmd_batch_compute(tmd_batch *batch, double *energy, double *virial, double *f);
/* As tmd_nve_run for every cell at once; thermo[rows*ncells*2] holds
 * (pe, ke) per cell, row-major by thermo row then cell. */
int tmd_batch_nve_run(tmd_batch *batch, int nsteps, double dt, int thermo_every,
                      double *thermo);
/* As tmd_nvt_run with one thermostat per cell: t_start[ncells], t_stop[ncells]. */
int tmd_batch_nvt_run(tmd_batch *batch, int nsteps, double dt, const double *t_start,
                      const double *t_stop, double t_damp, int thermo_every,
                      double *thermo);

/* ---- Serving ---------------------------------------------------------------
 * A job server on one GPU: callers submit independent small systems from any
 * thread; one library thread keeps every job in flight as a cell of one
 * multi-cell batch and advances all of them together (continuous batching:
 * finished jobs leave and queued jobs join between ticks, single-point jobs
 * ahead of the queue (they hold atoms for one tick only), the others FIFO, within
 * max_atoms / max_cells; each tick runs steps_per_tick steps).  There is no
 * counterpart in the reference, which runs one LAMMPS system per process.
 * Job kinds:
 *   TMD_JOB_ENERGY  one force evaluation (energy, virial, forces)
 *   TMD_JOB_NVE     nsteps of velocity Verlet with step dt (as tmd_nve_run)
 *   TMD_JOB_FIRE    energy minimisation as LAMMPS's min_style fire at its
 *                   defaults (min.cpp:63-72, min_fire.cpp:149-619: Euler
 *                   implicit, half step back, dmax 0.1 A, delaystep 20,
 *                   alpha0 0.25, tmax 10, tmin 0.02; initial step dt, v = 0
 *                   at the start) until max_i |F_i| < fmax after an iteration
 *                   (min_modify norm max) or nsteps iterations ran; a step
 *                   back costs one more force evaluation of its cell
 * tmd_server_submit returns TMD_ERR_ARG for a box that is degenerate or too
 * small for the cutoff (more than 3 images per axis) and TMD_ERR_CAPACITY for
 * a job larger than max_atoms.  A job's results do not depend on the other
 * jobs in flight: when jobs join or leave, the continuing ones move on the
 * device together with their neighbor lists, and a job's list is rebuilt
 * only when its own atoms trigger it, as for a separate system.
 * tmd_server_wait blocks up to timeout_s seconds (< 0: no limit) and returns
 * TMD_ERR_TIMEOUT if the job is not done (the ticket stays valid); on
 * completion it fills the non-NULL outputs: energy, virial[6], final x / v /
 * f [n*3] (positions as wrapped at the job's last neighbor rebuild), steps
 * run, latency from submit to completion, and releases the ticket. */
#define TMD_JOB_ENERGY 0
#define TMD_JOB_NVE 1
#define TMD_JOB_FIRE 2
typedef struct tmd_server tmd_server;
int tmd_server_create(const tmd_model *model, int max_atoms, int max_cells,
                      double skin, int steps_per_tick, tmd_server **out);
/* Admission by HBM footprint: a server sized from a device-memory budget.
 * The neighbor rows are given the length the densest admissible job needs
 * (max_density atoms per A^3, the same 30% + 32 margin as any system), and
 * max_atoms is the number of atoms whose arrays (positions, velocities,
 * forces, descriptors, MLP rows, neighbor rows, relayout copies, bins) fit in
 * hbm_bytes at that length.  Jobs are then admitted while their atoms fit, so
 * the batch never holds more than the budget; tmd_server_submit refuses a job
 * denser than max_density (TMD_ERR_CAPACITY) instead of growing the rows. */
int tmd_server_create_bytes(const tmd_model *model, size_t hbm_bytes, double max_density,
                            int max_cells, double skin, int steps_per_tick,
                            tmd_server **out);
/* Device bytes the server's arrays hold at its current neighbor-row length,
 * its atom capacity and that row length (entries per atom). */
int tmd_server_footprint(const tmd_server *server, size_t *device_bytes, int *max_atoms,
                         int *row_length);
void tmd_server_free(tmd_server *server);
int tmd_server_submit(tmd_server *server, int kind, int n, const double *x,
                      const int *type, const double *v, const double box[9],
                      const int pbc[3], int nsteps, double dt, double fmax,
                      long *ticket);
int tmd_server_wait(tmd_server *server, long ticket, double timeout_s,
                    double *energy, double *virial, double *x, double *v,
                    double *f, int *steps, double *latency_s);
/* Counters since creation: jobs submitted / completed, atoms in flight,
 * atom-steps evaluated (force evaluations x atoms), worker busy seconds. */
int tmd_server_stats(tmd_server *server, long *submitted, long *completed,
                     long *active_atoms, double *atom_steps, double *busy_s);
/* Worker seconds by phase since creation: seconds[0] relayout (admission and
 * retirement: moving the cells, neighbor lists of the new jobs), [1] force
 * evaluations of newly admitted jobs, [2] integrator steps, [3] copying
 * results out. */
int tmd_server_timing(tmd_server *server, double *seconds);

/* Full neighbor list without allocating any memory.  This entry point has no
 * counterpart in the reference.  It is meant for host programs that must not
 * let a library call cudaMalloc: programs that manage every byte of device
 * memory through their own pool, or that reserve the whole device up front,
 * so that an allocation inside the library would fail or escape their
 * accounting.  The call is synchronous: it waits for `stream` to finish and
 * reads a status word back to the host, so it must be made outside any
 * stream capture.
 *
 * x_dev[n*3]: device positions, already inside the periodic cell (no
 * wrapping is done; atoms outside a periodic cell give TMD_ERR_ARG).
 * box/pbc as tmd_system_set_box; cut: list cutoff (<= any cell width * 3).
 * Outputs, device memory owned by the caller: counts_dev[n] and
 * rows_dev[n*cap]; row i holds counts_dev[i] entries (shift_code << 23 | j)
 * with shift_code = (sx+3) + 7*(sy+3) + 49*(sz+3), in no particular order.
 * A row longer than cap gives TMD_ERR_CAPACITY (rows are then incomplete).
 * stream: cudaStream_t or NULL for the default stream; the call returns after
 * the stream has finished the work.
 *
 * Cell binning uses one scratch array of 4 MiB in the library's static device
 * memory, which every GPU that loads the library keeps until the process
 * exits.  Limits: n <= TMD_NOALLOC_MAX_ATOMS and at most TMD_NOALLOC_MAX_CELLS
 * cells (larger requests give TMD_ERR_CAPACITY).  All calls share that one
 * array: calls whose work overlaps on the GPU race and corrupt each other, so
 * serialise them.  The first call on each device looks the array up
 * (cudaGetSymbolAddress) with that device current. */
#define TMD_NOALLOC_MAX_ATOMS 262144
#define TMD_NOALLOC_MAX_CELLS 131072
int tmd_neighbor_list_noalloc(const double *x_dev, int n, const double box[9],
                              const int pbc[3], double cut, int cap,
                              int *counts_dev, unsigned int *rows_dev,
                              void *stream);

#ifdef __cplusplus
}
#endif

#endif /* TMD_B200_H */
