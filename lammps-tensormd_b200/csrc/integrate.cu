// integrate.cu -- velocity Verlet, deterministic FP64 reductions, checks.
//
// FixNVE (src/fix_nve.cpp:64-141): dtfm = dtf / mass[type]; v += dtfm * f;
// x += dtv * v; then after the force v += dtfm * f.  Products and sums are
// rounded separately (no FMA) as the host arithmetic of LAMMPS does.
// Reductions use a fixed grid and a fixed tree, so sums are bitwise
// reproducible run to run.
#include "tmd_kernels.h"

namespace tmd {

namespace {
constexpr int kRedBlocks = 1024;
constexpr int kRedThreads = 256;

__device__ inline double block_sum(double v, double *sh) {
  const int tid = threadIdx.x;
  sh[tid] = v;
  __syncthreads();
  for (int s = kRedThreads / 2; s > 0; s >>= 1) {
    if (tid < s) sh[tid] += sh[tid + s];
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}
}  // namespace

template <typename Tin>
__global__ void k_reduce_partial(const Tin *__restrict__ in, int n, int ncomp,
                                 double scale, double *__restrict__ partial) {
  __shared__ double sh[kRedThreads];
  const int per = (n + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = min(n, i0 + per);
  for (int c = 0; c < ncomp; c++) {
    double s = 0.0;
    for (int i = i0 + threadIdx.x; i < i1; i += blockDim.x)
      s += (double)in[(size_t)i * ncomp + c];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[(size_t)blockIdx.x * ncomp + c] = s * scale;
  }
}

__global__ void k_reduce_final(const double *__restrict__ partial, int nb, int ncomp,
                               double *__restrict__ out) {
  __shared__ double sh[kRedThreads];
  for (int c = 0; c < ncomp; c++) {
    double s = 0.0;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(size_t)b * ncomp + c];
    s = block_sum(s, sh);
    if (threadIdx.x == 0) out[c] = s;
  }
}

static int red_blocks(int n) {
  int b = (n + kRedThreads - 1) / kRedThreads;
  if (b > kRedBlocks) b = kRedBlocks;
  if (b < 1) b = 1;
  return b;
}

void launch_reduce_f64(const double *in, int n, int ncomp, double *partial,
                       double *out, cudaStream_t st, long &launches) {
  int nb = red_blocks(n);
  k_reduce_partial<double><<<nb, kRedThreads, 0, st>>>(in, n, ncomp, 1.0, partial);
  k_reduce_final<<<1, kRedThreads, 0, st>>>(partial, nb, ncomp, out);
  launches += 2;
}

void launch_reduce_scaled(const double *in, int n, double *partial, double *out,
                          double scale, cudaStream_t st, long &launches) {
  int nb = red_blocks(n);
  k_reduce_partial<double><<<nb, kRedThreads, 0, st>>>(in, n, 1, scale, partial);
  k_reduce_final<<<1, kRedThreads, 0, st>>>(partial, nb, 1, out);
  launches += 2;
}

// One block per cell (grid-stride over cells), a fixed tree per block.
__global__ void k_cell_sum(int ncells, const int *__restrict__ coff,
                           const double *__restrict__ in, int ncomp, double scale,
                           double *__restrict__ out, int ostride) {
  __shared__ double sh[kRedThreads];
  for (int c = blockIdx.x; c < ncells; c += gridDim.x) {
    const int a0 = coff[c], a1 = coff[c + 1];
    for (int k = 0; k < ncomp; k++) {
      double s = 0.0;
      for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) s += in[(size_t)a * ncomp + k];
      s = block_sum(s, sh);
      if (threadIdx.x == 0) out[(size_t)c * ostride + k] = s * scale;
    }
  }
}

void launch_cell_sum(int ncells, const int *coff, const double *in, int ncomp,
                     double scale, double *out, int ostride, cudaStream_t st,
                     long &launches) {
  int g = ncells < 148 * 16 ? ncells : 148 * 16;
  if (g < 1) g = 1;
  k_cell_sum<<<g, kRedThreads, 0, st>>>(ncells, coff, in, ncomp, scale, out, ostride);
  launches += 1;
}

__global__ void k_scale_copy(const double *__restrict__ in, int n, double scale,
                             double *__restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] * scale;
}

void launch_scale_copy(const double *in, int n, double scale, double *out,
                       cudaStream_t st, long &launches) {
  k_scale_copy<<<(n + 255) / 256, 256, 0, st>>>(in, n, scale, out);
  launches += 1;
}

__global__ void k_nve_initial(int n, double *__restrict__ x, double *__restrict__ v,
                              const double *__restrict__ f, const int *__restrict__ elem,
                              const double *__restrict__ mass_e, double dtf,
                              double dtv) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dtfm = dtf / mass_e[elem[i]];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    double vv = __dadd_rn(v[3 * i + c], __dmul_rn(dtfm, f[3 * i + c]));
    v[3 * i + c] = vv;
    x[3 * i + c] = __dadd_rn(x[3 * i + c], __dmul_rn(dtv, vv));
  }
}

__global__ void k_nve_final(int n, double *__restrict__ v, const double *__restrict__ f,
                            const int *__restrict__ elem,
                            const double *__restrict__ mass_e, double dtf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dtfm = dtf / mass_e[elem[i]];
#pragma unroll
  for (int c = 0; c < 3; c++)
    v[3 * i + c] = __dadd_rn(v[3 * i + c], __dmul_rn(dtfm, f[3 * i + c]));
}

void launch_nve_initial(int n, double *x, double *v, const double *f,
                        const int *elem, const double *mass_e, double dtf,
                        double dtv, cudaStream_t st, long &launches) {
  k_nve_initial<<<(n + 255) / 256, 256, 0, st>>>(n, x, v, f, elem, mass_e, dtf, dtv);
  launches += 1;
}

void launch_nve_final(int n, double *v, const double *f, const int *elem,
                      const double *mass_e, double dtf, cudaStream_t st,
                      long &launches) {
  k_nve_final<<<(n + 255) / 256, 256, 0, st>>>(n, v, f, elem, mass_e, dtf);
  launches += 1;
}

// ---------------------------------------------------------------------
// fix nvt (FixNH, fix_nh.cpp).  One thread per group runs the chain update;
// the velocity factor is applied by a per-atom kernel.  With the default one
// loop per half step (nc_tchain = 1) this is the same arithmetic as
// nh_v_temp scaling every velocity by factor_eta.
// ---------------------------------------------------------------------
namespace {
constexpr double kBoltz = 8.617343e-5;  // metal units, update.cpp:187-206

// FixNH::nhc_temp_integrate (fix_nh.cpp:1758-1822), nc_tchain = 1, drag = 0
// (the defaults, fix_nh.cpp:78-86), masses kept at the current target.
__device__ void nhc_integrate(NhcState &c) {
  const double dthalf = 0.5 * c.dt, dt4 = 0.25 * c.dt, dt8 = 0.125 * c.dt;
  const double w2 = c.t_freq * c.t_freq;
  double kecurrent = c.tdof * kBoltz * c.t_current;
  c.eta_mass[0] = c.tdof * kBoltz * c.t_target / w2;
  for (int k = 1; k < kNhcChain; k++) c.eta_mass[k] = kBoltz * c.t_target / w2;
  c.eta_dotdot[0] = c.eta_mass[0] > 0.0 ? (kecurrent - c.ke_target) / c.eta_mass[0] : 0.0;
  double expfac;
  for (int k = kNhcChain - 1; k > 0; k--) {
    expfac = exp(-dt8 * c.eta_dot[k + 1]);
    c.eta_dot[k] *= expfac;
    c.eta_dot[k] += c.eta_dotdot[k] * dt4;
    c.eta_dot[k] *= expfac;
  }
  expfac = exp(-dt8 * c.eta_dot[1]);
  c.eta_dot[0] *= expfac;
  c.eta_dot[0] += c.eta_dotdot[0] * dt4;
  c.eta_dot[0] *= expfac;
  const double factor = exp(-dthalf * c.eta_dot[0]);
  c.t_current *= factor * factor;
  kecurrent = c.tdof * kBoltz * c.t_current;
  c.eta_dotdot[0] = c.eta_mass[0] > 0.0 ? (kecurrent - c.ke_target) / c.eta_mass[0] : 0.0;
  for (int k = 0; k < kNhcChain; k++) c.eta[k] += dthalf * c.eta_dot[k];
  c.eta_dot[0] *= expfac;
  c.eta_dot[0] += c.eta_dotdot[0] * dt4;
  c.eta_dot[0] *= expfac;
  for (int k = 1; k < kNhcChain; k++) {
    expfac = exp(-dt8 * c.eta_dot[k + 1]);
    c.eta_dot[k] *= expfac;
    c.eta_dotdot[k] =
        (c.eta_mass[k - 1] * c.eta_dot[k - 1] * c.eta_dot[k - 1] - kBoltz * c.t_target) /
        c.eta_mass[k];
    c.eta_dot[k] += c.eta_dotdot[k] * dt4;
    c.eta_dot[k] *= expfac;
  }
  c.factor = factor;
}
}  // namespace

// FixNH::setup (fix_nh.cpp:741-800) for a thermostat-only fix.
__global__ void k_nhc_setup(int G, NhcState *__restrict__ st, const double *__restrict__ keg) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  NhcState c = st[g];
  c.t_current = c.tdof > 0.0 ? 2.0 * keg[g] / (c.tdof * kBoltz) : 0.0;
  c.t_target = c.t_start;
  c.ke_target = c.tdof * kBoltz * c.t_target;
  const double w2 = c.t_freq * c.t_freq;
  c.eta_mass[0] = c.tdof * kBoltz * c.t_target / w2;
  for (int k = 1; k < kNhcChain; k++) c.eta_mass[k] = kBoltz * c.t_target / w2;
  for (int k = 1; k < kNhcChain; k++)
    c.eta_dotdot[k] =
        (c.eta_mass[k - 1] * c.eta_dot[k - 1] * c.eta_dot[k - 1] - kBoltz * c.t_target) /
        c.eta_mass[k];
  c.step = 0;
  c.factor = 1.0;
  st[g] = c;
}

__global__ void k_nhc_update(int G, NhcState *__restrict__ st, const double *__restrict__ keg) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G) return;
  NhcState c = st[g];
  if (keg == nullptr) {  // initial_integrate: FixNH::compute_temp_target
    c.step++;
    double delta = c.nsteps > 0 ? (double)c.step / (double)c.nsteps : 0.0;
    c.t_target = c.t_start + delta * (c.t_stop - c.t_start);
    c.ke_target = c.tdof * kBoltz * c.t_target;
  } else {  // final_integrate: temperature after the second half kick
    c.t_current = c.tdof > 0.0 ? 2.0 * keg[g] / (c.tdof * kBoltz) : 0.0;
  }
  if (c.tdof > 0.0 && c.t_freq > 0.0 && c.t_target > 0.0)
    nhc_integrate(c);
  else
    c.factor = 1.0;
  st[g] = c;
}

__global__ void k_nhc_scale(int n, const int *__restrict__ acell,
                            const NhcState *__restrict__ st, double *__restrict__ v) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const double f = st[acell ? acell[a] : 0].factor;
  v[3 * a] *= f;
  v[3 * a + 1] *= f;
  v[3 * a + 2] *= f;
}

void launch_nhc_setup(int ngroups, NhcState *st, const double *ke_group, cudaStream_t s,
                      long &launches) {
  k_nhc_setup<<<(ngroups + 127) / 128, 128, 0, s>>>(ngroups, st, ke_group);
  launches += 1;
}

void launch_nhc_half(int ngroups, NhcState *st, const double *ke_group, int n,
                     const int *acell, double *v, cudaStream_t s, long &launches) {
  k_nhc_update<<<(ngroups + 127) / 128, 128, 0, s>>>(ngroups, st, ke_group);
  if (n > 0) k_nhc_scale<<<(n + 255) / 256, 256, 0, s>>>(n, acell, st, v);
  launches += 2;
}

// 0.5 * mvv2e * m * v^2 per atom (compute ke, metal mvv2e = 1.0364269e-4)
__global__ void k_kinetic(int n, const double *__restrict__ v, const int *__restrict__ elem,
                          const double *__restrict__ mass_e, double *__restrict__ ke) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double m = mass_e[elem[i]];
  double s = v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2];
  ke[i] = 0.5 * 1.0364269e-4 * m * s;
}

void launch_kinetic(int n, const double *v, const int *elem, const double *mass_e,
                    double *ke_atom, cudaStream_t st, long &launches) {
  k_kinetic<<<(n + 255) / 256, 256, 0, st>>>(n, v, elem, mass_e, ke_atom);
  launches += 1;
}

__global__ void k_check_finite(int n, const double *__restrict__ f,
                               const double *__restrict__ etot, int *status) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  if (i == 0 && etot && !isfinite(*etot)) bad = true;
  if (i < n)
    bad |= !isfinite(f[3 * i]) || !isfinite(f[3 * i + 1]) || !isfinite(f[3 * i + 2]);
  if (bad) atomicOr(status, kStatusNonfinite);
}

void launch_check_finite(int n, const double *f, const double *etot, int *status,
                         cudaStream_t st, long &launches) {
  int grid = (n + 255) / 256;
  if (grid < 1) grid = 1;
  k_check_finite<<<grid, 256, 0, st>>>(n, f, etot, status);
  launches += 1;
}

}  // namespace tmd
