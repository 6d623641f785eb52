// server_kernels.cu -- device side of the serving loop: mixed single-point / NVE /
// FIRE jobs advanced together in one multi-cell system.
//
// Every cell carries a CellCtl.  NVE cells follow FixNVE (fix_nve.cpp:64-141,
// metal units, products and sums rounded separately like integrate.cu).
// FIRE cells follow LAMMPS's min_style fire at its defaults (min.cpp:63-72,
// MinFire::run_iterate<EULERIMPLICIT> in min_fire.cpp:149-619): per cell
// P = F.v; P > 0 mixes v <- (1 - a) v + a sqrt(v.v / F.F) F after the Euler
// kick and, more than delaystep (20) iterations after the last P <= 0, grows
// dt by 1.1 (at most 10 dt0) and shrinks a by 0.99; P <= 0 (after the first
// 20 iterations) resets a to 0.25 and halves dt (not below 0.02 dt0), steps
// the atoms back by dt v / 2 and zeroes v, after which the forces of the new
// positions are evaluated (one more force evaluation of the batch) before the
// step continues from v = 0.  The step is limited so that no atom moves more
// than dmax = 0.1 A along an axis; then v += dt F / m and x += dt v.  An
// iteration ends with the force evaluation after its move; the cell has
// converged when max_i |F_i|^2 < fmax^2 (min_modify norm max) at that point.
#include <cmath>

#include "tmd_kernels.h"

namespace tmd {

namespace {
constexpr double kFtm2v = 1.0 / 1.0364269e-4;  // metal units, update.cpp:187-206
// min_style fire defaults (min.cpp:63-72)
constexpr int kFireDelay = 20;
constexpr double kFireGrow = 1.1, kFireShrink = 0.5, kFireAlpha0 = 0.25, kFireAlphaShrink = 0.99;
constexpr double kFireDmax = 0.1;
constexpr int kFireMaxNeg = 2000;  // max_vdotf_negatif
constexpr int kThreads = 256;

__device__ inline bool fire_active(const CellCtl &c) {
  return c.mode == kJobFire && !c.conv && c.left > 0;
}
}  // namespace

// One warp per atom of the new layout.  A moved atom brings its state and,
// unless its cell is about to be rebuilt, its neighbor row: entries keep
// their shift code and move their atom index with the cell (every partner
// of a cell's atom is in the same cell), partner slots j*cap0 + t become
// (j + delta)*cap1 + t.  The row keeps its sorted order since one delta
// moves every index.  A new atom gets an empty row.
__global__ void k_srv_move(SrvMove m) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int B1 = m.B + 1;
  for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < m.n; a += nw) {
    const int c = m.acell[a];
    const int k = a - m.coff[c];
    const int s = m.src[c];
    if (s >= 0) {
      const long o = (long)s + k;
      if (lane < 3) {
        m.x2[3L * a + lane] = m.x[3 * o + lane];
        m.v2[3L * a + lane] = m.v[3 * o + lane];
        m.f2[3L * a + lane] = m.f[3 * o + lane];
        m.xb2[3L * a + lane] = m.xb[3 * o + lane];
        m.img2[3L * a + lane] = m.img[3 * o + lane];
      } else if (lane == 3) {
        m.elem2[a] = m.elem[o];
      }
      if (m.fresh[c]) {
        for (int b = lane; b < B1; b += 32) m.boff2[(long)a * B1 + b] = 0;
        continue;
      }
      for (int b = lane; b < B1; b += 32) m.boff2[(long)a * B1 + b] = m.boff[o * B1 + b];
      int cnt = m.boff[o * B1 + m.B];
      cnt = min(cnt, min(m.cap0, m.cap1));
      const int delta = m.coff[c] - s;
      const uint32_t *row = m.nbr + o * m.cap0;
      const int *rrow = m.rev + o * m.cap0;
      uint32_t *row2 = m.nbr2 + (long)a * m.cap1;
      int *rrow2 = m.rev2 + (long)a * m.cap1;
      for (int t = lane; t < cnt; t += 32) {
        const uint32_t e = row[t];
        row2[t] = (e & ~kAtomMask) | uint32_t((int)(e & kAtomMask) + delta);
        const int r = rrow[t];
        rrow2[t] = r < 0 ? -1 : (int)((long)(r / m.cap0 + delta) * m.cap1 + r % m.cap0);
      }
    } else {
      const long o = (long)(-s - 1) + k;
      if (lane < 3) {
        m.x2[3L * a + lane] = m.sx[3 * o + lane];
        m.v2[3L * a + lane] = m.sv[3 * o + lane];
        m.f2[3L * a + lane] = 0.0;
        m.xb2[3L * a + lane] = m.sx[3 * o + lane];
        m.img2[3L * a + lane] = 0;
      } else if (lane == 3) {
        m.elem2[a] = m.selem[o];
      }
      for (int b = lane; b < B1; b += 32) m.boff2[(long)a * B1 + b] = 0;
    }
  }
}

void launch_srv_move(const SrvMove &m, cudaStream_t st, long &launches) {
  if (m.n <= 0) return;
  long g = ((long)m.n * 32 + kThreads - 1) / kThreads;
  if (g > 148 * 16) g = 148 * 16;
  k_srv_move<<<(int)g, kThreads, 0, st>>>(m);
  launches += 1;
}

__global__ void k_srv_acell(int ncells, const int *__restrict__ coff, int *__restrict__ acell) {
  for (int c = blockIdx.x; c < ncells; c += gridDim.x)
    for (int a = coff[c] + threadIdx.x; a < coff[c + 1]; a += blockDim.x) acell[a] = c;
}

void launch_srv_acell(int ncells, const int *coff, int *acell, cudaStream_t st,
                      long &launches) {
  if (ncells <= 0) return;
  const int g = ncells < 148 * 16 ? ncells : 148 * 16;
  k_srv_acell<<<g, kThreads, 0, st>>>(ncells, coff, acell);
  launches += 1;
}

// One warp per cell: a ballot per 32 atoms and element places the cell's
// atoms of each element at its slots in perm, in atom order.
__global__ void k_srv_perm(int ncells, int B, const int *__restrict__ coff,
                           const int *__restrict__ elem, const int *__restrict__ estart,
                           int *__restrict__ perm) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const unsigned below = (1u << lane) - 1u;
  for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < ncells; c += nw) {
    const int a0 = coff[c], a1 = coff[c + 1];
    for (int e = 0; e < B; e++) {
      int pos = estart[(long)c * B + e];
      for (int ab = a0; ab < a1; ab += 32) {
        const int a = ab + lane;
        const bool hit = a < a1 && elem[a] == e;
        const unsigned bal = __ballot_sync(0xffffffffu, hit);
        if (hit) perm[pos + __popc(bal & below)] = a;
        pos += __popc(bal);
      }
    }
  }
}

void launch_srv_perm(int ncells, int B, const int *coff, const int *elem, const int *estart,
                     int *perm, cudaStream_t st, long &launches) {
  if (ncells <= 0) return;
  long g = ((long)ncells * 32 + kThreads - 1) / kThreads;
  if (g > 148 * 16) g = 148 * 16;
  k_srv_perm<<<(int)g, kThreads, 0, st>>>(ncells, B, coff, elem, estart, perm);
  launches += 1;
}

__global__ void k_srv_mark(int ncells, const int *__restrict__ fresh, int *__restrict__ cflag,
                           int *flag) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x)
    cflag[c] = fresh[c];
  if (blockIdx.x == 0 && threadIdx.x == 0) *flag = 1;
}

void launch_srv_mark(int ncells, const int *fresh, int *cflag, int *flag, cudaStream_t st,
                     long &launches) {
  int g = (ncells + kThreads - 1) / kThreads;
  if (g > 148 * 8) g = 148 * 8;
  if (g < 1) g = 1;
  k_srv_mark<<<g, kThreads, 0, st>>>(ncells, fresh, cflag, flag);
  launches += 1;
}

// Per atom of active FIRE cells (0 elsewhere): (F.v, v.v, F.F) into pw and
// (max_k |v_k|, max_k |F_k| / m) into pm, for the per-cell sums and maxima.
__global__ void k_srv_power(int n, const int *__restrict__ acell,
                            const CellCtl *__restrict__ ctl, const double *__restrict__ v,
                            const double *__restrict__ f, const int *__restrict__ elem,
                            const double *__restrict__ mass_e, double *__restrict__ pw,
                            double *__restrict__ pm) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  double p = 0, vv = 0, ff = 0, vm = 0, fm = 0;
  if (fire_active(ctl[acell[a]])) {
    for (int d = 0; d < 3; d++) {
      const double vd = v[3L * a + d], fd = f[3L * a + d];
      p += vd * fd;
      vv += vd * vd;
      ff += fd * fd;
      vm = fmax(vm, fabs(vd));
      fm = fmax(fm, fabs(fd));
    }
    fm /= mass_e[elem[a]];
  }
  pw[3L * a] = p;
  pw[3L * a + 1] = vv;
  pw[3L * a + 2] = ff;
  pm[2L * a] = vm;
  pm[2L * a + 1] = fm;
}

// Per-cell maxima of two interleaved per-atom values (one block per cell).
__global__ void k_cell_max2(int ncells, const int *__restrict__ coff,
                            const double *__restrict__ in, double *__restrict__ out) {
  __shared__ double sh[2][kThreads];
  for (int c = blockIdx.x; c < ncells; c += gridDim.x) {
    double m0 = 0.0, m1 = 0.0;
    for (int a = coff[c] + threadIdx.x; a < coff[c + 1]; a += blockDim.x) {
      m0 = fmax(m0, in[2L * a]);
      m1 = fmax(m1, in[2L * a + 1]);
    }
    sh[0][threadIdx.x] = m0;
    sh[1][threadIdx.x] = m1;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) {
        sh[0][threadIdx.x] = fmax(sh[0][threadIdx.x], sh[0][threadIdx.x + s]);
        sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + s]);
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      out[2L * c] = sh[0][0];
      out[2L * c + 1] = sh[1][0];
    }
    __syncthreads();
  }
}

// Step limit so that no atom moves more than dmax along an axis, for the
// largest velocity component vmax (min_fire.cpp, dtvone).
__device__ inline double fire_limit(double dt, double vmax) {
  return dt * vmax > kFireDmax ? kFireDmax / vmax : dt;
}

// FIRE plan of every active cell for this step, from its (P, v.v, F.F) sums
// and (max |v_k|, max |F_k| / m) maxima.
__global__ void k_srv_fire_update(int ncells, CellCtl *__restrict__ ctl,
                                  const double *__restrict__ csum,
                                  const double *__restrict__ cmax) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncells) return;
  CellCtl q = ctl[c];
  if (!fire_active(q)) {
    q.plan = kFirePlanNone;
    ctl[c] = q;
    return;
  }
  const double P = csum[4L * c], vv = csum[4L * c + 1], ff = csum[4L * c + 2];
  const double vmax = cmax[2L * c], fmm = cmax[2L * c + 1];
  if (q.phase == 1) {
    // forces of the stepped-back positions are in: v = dt F / m estimates the
    // step limit, then the move starts from v = 0
    q.phase = 0;
    q.plan = kFirePlanReset;
    q.dtv = fire_limit(q.dt, q.dt * kFtm2v * fmm);
  } else {
    q.it++;
    if (P > 0.0) {
      q.nneg = 0;
      q.mix1 = 1.0 - q.alpha;
      q.mix2 = ff <= 1e-20 ? 0.0 : q.alpha * sqrt(vv / ff);
      if (q.it - q.last_neg > kFireDelay) {
        q.dt = fmin(q.dt * kFireGrow, q.dtmax);
        q.alpha *= kFireAlphaShrink;
      }
      q.plan = kFirePlanMix;
      q.dtv = fire_limit(q.dt, vmax);
    } else {
      q.last_neg = q.it;
      if (q.it >= kFireDelay) {
        q.alpha = kFireAlpha0;
        if (q.dt * kFireShrink >= q.dtmin) q.dt *= kFireShrink;
      }
      if (++q.nneg > kFireMaxNeg) {
        q.conv = 2;  // stuck in a basin (LAMMPS: "max iterations with v.f negative")
        q.plan = kFirePlanNone;
      } else if (vv > 0.0) {
        q.plan = kFirePlanBack;
        q.phase = 1;
      } else {
        // v is already zero: the step back moves nothing and the forces in
        // hand are those of the current positions
        q.plan = kFirePlanReset;
        q.dtv = fire_limit(q.dt, q.dt * kFtm2v * fmm);
      }
    }
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
  } else if (q.mode == kJobFire && q.plan == kFirePlanBack) {
    for (int d = 0; d < 3; d++) {
      x[3L * a + d] -= 0.5 * q.dt * v[3L * a + d];
      v[3L * a + d] = 0.0;
    }
  } else if (q.mode == kJobFire && (q.plan == kFirePlanMix || q.plan == kFirePlanReset)) {
    const double dtfm = q.dtv * kFtm2v / m;
    const bool mix = q.plan == kFirePlanMix;
    for (int d = 0; d < 3; d++) {
      const double fd = f[3L * a + d];
      double vd = (mix ? v[3L * a + d] : 0.0) + dtfm * fd;
      if (mix) vd = q.mix1 * vd + q.mix2 * fd;
      v[3L * a + d] = vd;
      x[3L * a + d] += q.dtv * vd;
    }
  }
}

void launch_srv_pre(int n, int ncells, const int *acell, const int *coff, CellCtl *ctl,
                    double *x, double *v, const double *f, const int *elem,
                    const double *mass_e, double *pw, double *pm, double *csum,
                    double *cmax, cudaStream_t st, long &launches) {
  if (n <= 0) return;
  const int g = (n + kThreads - 1) / kThreads;
  k_srv_power<<<g, kThreads, 0, st>>>(n, acell, ctl, v, f, elem, mass_e, pw, pm);
  launch_cell_sum(ncells, coff, pw, 3, 1.0, csum, 4, st, launches);
  const int gc = ncells < 148 * 16 ? ncells : 148 * 16;
  k_cell_max2<<<gc, kThreads, 0, st>>>(ncells, coff, pm, cmax);
  k_srv_fire_update<<<(ncells + kThreads - 1) / kThreads, kThreads, 0, st>>>(ncells, ctl,
                                                                             csum, cmax);
  k_srv_initial<<<g, kThreads, 0, st>>>(n, acell, ctl, x, v, f, elem, mass_e);
  launches += 4;
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
    // an iteration ends with the force evaluation after its move (not after
    // a step back); only then is convergence tested, as LAMMPS does
    if (count && (q.plan == kFirePlanMix || q.plan == kFirePlanReset)) {
      q.left--;
      if (cfmax[c] < q.fmax2) q.conv = 1;
    }
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
