// server_kernels.cu -- device side of the serving loop: mixed single-point / NVE /
// FIRE jobs advanced together in one multi-cell system.
//
// Every cell carries a CellCtl.  NVE cells follow FixNVE (fix_nve.cpp:64-141,
// metal units, products and sums rounded separately like integrate.cu).
// FIRE cells follow Bitzek et al., PRL 97, 170201 (2006) with a semi-implicit
// Euler step: from the current v and F of the cell, P = F.v; P > 0 mixes
// v <- (1 - a) v + a |v| F/|F| and, after more than Nmin such steps in a row,
// grows dt (x finc, capped at dtmax) and shrinks a (x fa); P <= 0 zeroes v,
// resets a and, past the first Nmin iterations, halves dt.  Then
// v <- v + dt F/m and x <- x + dt v.  Convergence: max_i |F_i| <= fmax.
#include <cmath>

#include "tmd_kernels.h"

namespace tmd {

namespace {
constexpr double kFtm2v = 1.0 / 1.0364269e-4;  // metal units, update.cpp:187-206
constexpr int kFireNmin = 5;
constexpr double kFireFinc = 1.1, kFireFdec = 0.5, kFireAlpha0 = 0.1, kFireFalpha = 0.99;
constexpr int kThreads = 256;

__device__ inline bool fire_active(const CellCtl &c) {
  return c.mode == kJobFire && !c.conv && c.left > 0;
}
}  // namespace

__global__ void k_srv_gather(int n, const int *__restrict__ acell, const int *__restrict__ coff,
                             const int *__restrict__ src, const double *__restrict__ x_old,
                             const double *__restrict__ v_old, const double *__restrict__ f_old,
                             const int *__restrict__ img_old,
                             const double *__restrict__ x_stage,
                             const double *__restrict__ v_stage, double *__restrict__ x,
                             double *__restrict__ v, double *__restrict__ f,
                             int *__restrict__ img) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const int c = acell[a];
  const int k = a - coff[c];
  const int s = src[c];
  for (int d = 0; d < 3; d++) {
    if (s >= 0) {
      const long o = 3L * (s + k) + d;
      x[3L * a + d] = x_old[o];
      v[3L * a + d] = v_old[o];
      f[3L * a + d] = f_old[o];
      img[3L * a + d] = img_old[o];
    } else {
      const long o = 3L * (-s - 1 + k) + d;
      x[3L * a + d] = x_stage[o];
      v[3L * a + d] = v_stage[o];
      f[3L * a + d] = 0.0;
      img[3L * a + d] = 0;
    }
  }
}

void launch_srv_gather(int n, const int *acell, const int *coff, const int *src,
                       const double *x_old, const double *v_old, const double *f_old,
                       const int *img_old, const double *x_stage, const double *v_stage,
                       double *x, double *v, double *f, int *img, cudaStream_t st,
                       long &launches) {
  if (n <= 0) return;
  k_srv_gather<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(
      n, acell, coff, src, x_old, v_old, f_old, img_old, x_stage, v_stage, x, v, f, img);
  launches += 1;
}

// (F.v, v.v, F.F) per atom of active FIRE cells, 0 elsewhere.
__global__ void k_srv_power(int n, const int *__restrict__ acell,
                            const CellCtl *__restrict__ ctl, const double *__restrict__ v,
                            const double *__restrict__ f, double *__restrict__ pw) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  double p = 0, vv = 0, ff = 0;
  if (fire_active(ctl[acell[a]])) {
    for (int d = 0; d < 3; d++) {
      const double vd = v[3L * a + d], fd = f[3L * a + d];
      p += fd * vd;
      vv += vd * vd;
      ff += fd * fd;
    }
  }
  pw[3L * a] = p;
  pw[3L * a + 1] = vv;
  pw[3L * a + 2] = ff;
}

// FIRE state of every active cell from its (P, v.v, F.F) sums.
__global__ void k_srv_fire_update(int ncells, CellCtl *__restrict__ ctl,
                                  const double *__restrict__ csum) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  CellCtl q = ctl[c];
  if (!fire_active(q)) return;
  const double P = csum[4L * c], vv = csum[4L * c + 1], ff = csum[4L * c + 2];
  if (P > 0.0) {
    q.mix1 = 1.0 - q.alpha;
    q.mix2 = ff > 0.0 ? q.alpha * sqrt(vv / ff) : 0.0;
    q.npos++;
    if (q.npos > kFireNmin) {
      q.dt = fmin(q.dt * kFireFinc, q.dtmax);
      q.alpha *= kFireFalpha;
    }
  } else {
    q.mix1 = 0.0;
    q.mix2 = 0.0;
    q.npos = 0;
    q.alpha = kFireAlpha0;
    if (q.it >= kFireNmin) q.dt *= kFireFdec;
  }
  ctl[c] = q;
}

// Position update before the force evaluation.
__global__ void k_srv_initial(int n, const int *__restrict__ acell,
                              const CellCtl *__restrict__ ctl, double *__restrict__ x,
                              double *__restrict__ v, const double *__restrict__ f,
                              const int *__restrict__ elem, const double *__restrict__ mass_e) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const CellCtl q = ctl[acell[a]];
  const double m = mass_e[elem[a]];
  if (q.mode == kJobNve && q.left > 0) {
    const double dtfm = __ddiv_rn(__dmul_rn(0.5 * q.dt, kFtm2v), m);
    for (int d = 0; d < 3; d++) {
      const double vd = __dadd_rn(v[3L * a + d], __dmul_rn(dtfm, f[3L * a + d]));
      v[3L * a + d] = vd;
      x[3L * a + d] = __dadd_rn(x[3L * a + d], __dmul_rn(q.dt, vd));
    }
  } else if (fire_active(q)) {
    const double dtfm = q.dt * kFtm2v / m;
    for (int d = 0; d < 3; d++) {
      const double fd = f[3L * a + d];
      double vd = q.mix1 * v[3L * a + d] + q.mix2 * fd;
      vd += dtfm * fd;
      v[3L * a + d] = vd;
      x[3L * a + d] += q.dt * vd;
    }
  }
}

void launch_srv_pre(int n, int ncells, const int *acell, const int *coff, CellCtl *ctl,
                    double *x, double *v, const double *f, const int *elem,
                    const double *mass_e, double *pw, double *csum, cudaStream_t st,
                    long &launches) {
  if (n <= 0) return;
  const int g = (n + kThreads - 1) / kThreads;
  k_srv_power<<<g, kThreads, 0, st>>>(n, acell, ctl, v, f, pw);
  launch_cell_sum(ncells, coff, pw, 3, 1.0, csum, 4, st, launches);
  k_srv_fire_update<<<(ncells + kThreads - 1) / kThreads, kThreads, 0, st>>>(ncells, ctl,
                                                                             csum);
  k_srv_initial<<<g, kThreads, 0, st>>>(n, acell, ctl, x, v, f, elem, mass_e);
  launches += 3;
}

// NVE second half kick; |F|^2 per atom.
__global__ void k_srv_final(int n, const int *__restrict__ acell,
                            const CellCtl *__restrict__ ctl, double *__restrict__ v,
                            const double *__restrict__ f, const int *__restrict__ elem,
                            const double *__restrict__ mass_e, double *__restrict__ fsq,
                            int kick) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  const CellCtl q = ctl[acell[a]];
  if (kick && q.mode == kJobNve && q.left > 0) {
    const double dtfm = __ddiv_rn(__dmul_rn(0.5 * q.dt, kFtm2v), mass_e[elem[a]]);
    for (int d = 0; d < 3; d++)
      v[3L * a + d] = __dadd_rn(v[3L * a + d], __dmul_rn(dtfm, f[3L * a + d]));
  }
  const double fx = f[3L * a], fy = f[3L * a + 1], fz = f[3L * a + 2];
  fsq[a] = fx * fx + fy * fy + fz * fz;
}

// Per-cell maximum of fsq (one block per cell, grid-stride over cells).
__global__ void k_cell_max(int ncells, const int *__restrict__ coff,
                           const double *__restrict__ in, double *__restrict__ out) {
  __shared__ double sh[kThreads];
  for (int c = blockIdx.x; c < ncells; c += gridDim.x) {
    double mx = 0.0;
    for (int a = coff[c] + threadIdx.x; a < coff[c + 1]; a += blockDim.x) mx = fmax(mx, in[a]);
    sh[threadIdx.x] = mx;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + s]);
      __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = sh[0];
    __syncthreads();
  }
}

__global__ void k_srv_cell_end(int ncells, CellCtl *__restrict__ ctl,
                               const double *__restrict__ cfmax, int count) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  CellCtl q = ctl[c];
  if (q.mode == kJobNve) {
    if (count && q.left > 0) q.left--;
  } else if (q.mode == kJobFire && !q.conv && q.left > 0) {
    if (count) {
      q.left--;
      q.it++;
    }
    if (cfmax[c] <= q.fmax2) q.conv = 1;
  }
  ctl[c] = q;
}

void launch_srv_post(int n, int ncells, const int *acell, const int *coff, CellCtl *ctl,
                     double *v, const double *f, const int *elem, const double *mass_e,
                     double *fsq, double *cfmax, int kick, int count, cudaStream_t st,
                     long &launches) {
  if (n <= 0) return;
  k_srv_final<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(n, acell, ctl, v, f, elem,
                                                                   mass_e, fsq, kick);
  const int gc = ncells < 148 * 16 ? ncells : 148 * 16;
  k_cell_max<<<gc, kThreads, 0, st>>>(ncells, coff, fsq, cfmax);
  k_srv_cell_end<<<(ncells + kThreads - 1) / kThreads, kThreads, 0, st>>>(ncells, ctl, cfmax,
                                                                          count);
  launches += 3;
}

}  // namespace tmd
