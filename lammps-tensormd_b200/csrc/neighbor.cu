// neighbor.cu -- on-device cell binning and full neighbor list.
//
// Semantics follow LAMMPS NBinStandard::bin_atoms + NPairFullBinAtomonly::build
// (src/nbin_standard.cpp:221-261, src/npair_full_bin_atomonly.cpp:32-92): a
// full list of every image (j, shift) with rsq <= (rc + skin)^2 except the atom
// itself, rsq computed in FP64 without fused multiply-add from the image
// coordinate x_j + shift built hop by hop as AtomVec::pack_border does.  The
// ghost atoms of LAMMPS are represented as (j, shift) entries, so small and
// triclinic periodic cells need no ghost arrays.
//
// Layout (n atoms, cap entries per atom):
//   nbr[i*cap + t]  packed (shift_code << 23 | j), sorted by (element block,
//                   packed key): block 0 = same element as i, then the others
//                   in the order of tensormd.cpp:165-176
//   boff[i*(B+1)+b] start of block b in the row, boff[i*(B+1)+B] = count
//   rev[i*cap + t]  flat slot of the partner entry (j -> i, -shift), -1 if the
//                   partner fell outside the list cutoff by rounding
//
// Every kernel takes `flag` and returns at once when no rebuild is pending, so
// the sequence can sit inside a captured CUDA graph of the MD step.
#include <cmath>

#include "tmd_kernels.h"

namespace tmd {

__global__ void k_nb_check(int n, const double *__restrict__ x,
                           const double *__restrict__ xbuild, double trigsq,
                           int *flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (*flag) return;
  double dx = x[3 * i] - xbuild[3 * i];
  double dy = x[3 * i + 1] - xbuild[3 * i + 1];
  double dz = x[3 * i + 2] - xbuild[3 * i + 2];
  double rsq = dx * dx + dy * dy + dz * dz;
  if (rsq > trigsq) atomicOr(flag, 1);
}

// Multi-cell mode rebuilds only the cells whose atoms moved (cflag[c] set by
// k_nbc_check), as separate systems would; bit 2 of the flag (a forced
// rebuild) rebuilds every cell.  Single-box mode passes cflag = nullptr.
__device__ inline bool nb_rebuild(const int *flag, const int *__restrict__ cflag,
                                  const int *__restrict__ acell, int i) {
  return cflag == nullptr || (*flag & 2) || cflag[acell[i]];
}

__global__ void k_nbc_check(int n, const double *__restrict__ x,
                            const double *__restrict__ xbuild, double trigsq,
                            const int *__restrict__ acell, int *__restrict__ cflag, int *flag) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double dx = x[3 * i] - xbuild[3 * i];
  double dy = x[3 * i + 1] - xbuild[3 * i + 1];
  double dz = x[3 * i + 2] - xbuild[3 * i + 2];
  double rsq = dx * dx + dy * dy + dz * dz;
  if (rsq > trigsq) {
    cflag[acell[i]] = 1;
    atomicOr(flag, 1);
  }
}

__global__ void k_nbc_clear(int ncells, int *__restrict__ cflag, const int *flag) {
  if (!*flag) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncells; c += gridDim.x * blockDim.x)
    cflag[c] = 0;
}

__device__ inline void frac_of(const BoxP &b, double px, double py, double pz,
                               double &fx, double &fy, double &fz) {
  double dx = px - b.lo[0], dy = py - b.lo[1], dz = pz - b.lo[2];
  fz = dz / b.zprd;
  fy = (dy - fz * b.yz) / b.yprd;
  fx = (dx - fy * b.xy - fz * b.xz) / b.xprd;
}

__global__ void k_nb_zero(int ncell, int *cell_count, const int *flag) {
  if (!*flag) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
       c += gridDim.x * blockDim.x)
    cell_count[c] = 0;
}

// Wrap atom i back into the periodic cell (Domain::pbc()), counting the
// crossings in image[]; returns the wrapped position.
__device__ inline void wrap_atom(const BoxP &box, int i, double *__restrict__ x,
                                 int *__restrict__ image, double &px, double &py,
                                 double &pz) {
  px = x[3 * i]; py = x[3 * i + 1]; pz = x[3 * i + 2];
  if (!box.triclinic) {
    double lo[3] = {box.lo[0], box.lo[1], box.lo[2]};
    double prd[3] = {box.xprd, box.yprd, box.zprd};
    double p[3] = {px, py, pz};
    for (int a = 0; a < 3; a++) {
      if (!box.pbc[a]) continue;
      if (p[a] < lo[a]) {
        p[a] += prd[a];
        image[3 * i + a] -= 1;
      }
      if (p[a] >= lo[a] + prd[a]) {
        p[a] -= prd[a];
        p[a] = p[a] < lo[a] ? lo[a] : p[a];
        image[3 * i + a] += 1;
      }
    }
    px = p[0]; py = p[1]; pz = p[2];
  } else {
    double f[3];
    frac_of(box, px, py, pz, f[0], f[1], f[2]);
    int s[3] = {0, 0, 0};
    for (int a = 0; a < 3; a++)
      if (box.pbc[a]) s[a] = (int)floor(f[a]);
    if (s[0] || s[1] || s[2]) {
      image_of(box, px, py, pz, -s[0], -s[1], -s[2], px, py, pz);
      image[3 * i] += s[0];
      image[3 * i + 1] += s[1];
      image[3 * i + 2] += s[2];
    }
  }
  x[3 * i] = px; x[3 * i + 1] = py; x[3 * i + 2] = pz;
}

// Wrap atoms into the cell, then bin them.
__global__ void k_nb_bin(int n, double *__restrict__ x, int *__restrict__ image,
                         BoxP box, BinP bin, int *__restrict__ cell_of,
                         int *__restrict__ cell_count, int *status,
                         const int *flag) {
  if (!*flag) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
  double px, py, pz;
  wrap_atom(box, i, x, image, px, py, pz);
  double f[3];
  frac_of(box, px, py, pz, f[0], f[1], f[2]);
  int c3[3];
  for (int a = 0; a < 3; a++) {
    if (!box.pbc[a] && (f[a] < 0.0 || f[a] > 1.0)) atomicOr(status, kStatusOutside);
    int q = (int)floor(f[a] * bin.nb[a]);
    q = q < 0 ? 0 : (q >= bin.nb[a] ? bin.nb[a] - 1 : q);
    c3[a] = q;
  }
  int c = (c3[2] * bin.nb[1] + c3[1]) * bin.nb[0] + c3[0];
  cell_of[i] = c;
  atomicAdd(&cell_count[c], 1);
  }
}

// Exclusive scan of the cell counts with one block of 1024 threads.
__global__ void k_nb_scan(int ncell, const int *__restrict__ cell_count,
                          int *__restrict__ cell_start,
                          int *__restrict__ cell_cursor, const int *flag) {
  if (!*flag) return;
  __shared__ int warp_sums[32];
  int tid = threadIdx.x;
  int per = (ncell + blockDim.x - 1) / blockDim.x;
  int c0 = tid * per, c1 = min(c0 + per, ncell);
  int local = 0;
  for (int c = c0; c < c1; c++) local += cell_count[c];
  int lane = tid & 31, w = tid >> 5;
  int incl = local;
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warp_sums[w] = incl;
  __syncthreads();
  if (w == 0) {
    int v = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    warp_sums[lane] = v;
  }
  __syncthreads();
  int base = (w > 0 ? warp_sums[w - 1] : 0) + incl - local;
  for (int c = c0; c < c1; c++) {
    cell_start[c] = base;
    cell_cursor[c] = base;
    base += cell_count[c];
  }
  if (tid == blockDim.x - 1) cell_start[ncell] = base;
}

__global__ void k_nb_fill(int n, const int *__restrict__ cell_of,
                          int *__restrict__ cell_cursor,
                          int *__restrict__ cell_atoms, const int *flag) {
  if (!*flag) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    int pos = atomicAdd(&cell_cursor[cell_of[i]], 1);
    cell_atoms[pos] = i;
  }
}

// Order each cell's atoms by index so the build is deterministic.
__global__ void k_nb_cellsort(int ncell, const int *__restrict__ cell_start,
                              int *__restrict__ cell_atoms, const int *flag) {
  if (!*flag) return;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ncell;
       c += gridDim.x * blockDim.x) {
    int s0 = cell_start[c], s1 = cell_start[c + 1];
    for (int a = s0 + 1; a < s1; a++) {
      int v = cell_atoms[a];
      int b = a - 1;
      while (b >= s0 && cell_atoms[b] > v) {
        cell_atoms[b + 1] = cell_atoms[b];
        b--;
      }
      cell_atoms[b + 1] = v;
    }
  }
}

// FP64 squared distance, products and sums rounded separately (no FMA).
__device__ inline double rsq_nofma(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                   __dmul_rn(dz, dz));
}

// One warp per atom; lanes walk stencil cells.  Each lane keeps the passing
// candidates of its cell (up to kNbKeep) in shared memory while it counts
// them, then writes them at its prefix position: the order is deterministic
// (lane order, then cell order) and the distances are computed once; a cell
// with more passing candidates than that is walked a second time.
constexpr int kNbKeep = 16;
constexpr int kNbKeepStride = kNbKeep + 1;  // odd stride: lanes in distinct banks

// Dynamic shared memory a launch of k_nb_build with `threads` threads needs.
size_t nb_build_smem(int threads) { return sizeof(uint32_t) * (size_t)threads * kNbKeepStride; }
__global__ void k_nb_build(int n, const double *__restrict__ x, BoxP box,
                           BinP bin, const int *__restrict__ cell_of,
                           const int *__restrict__ cell_start,
                           const int *__restrict__ cell_atoms, double cutsq,
                           int cap, uint32_t *__restrict__ tmp,
                           int *__restrict__ nraw, int *status, int *maxneed,
                           const int *flag) {
  if (!*flag) return;
  extern __shared__ uint32_t nb_keep[];
  {
    // a launch without the keep buffers (nb_build_smem) would write past the
    // dynamic shared memory: refuse with a status bit instead
    uint32_t dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (dyn < sizeof(uint32_t) * blockDim.x * kNbKeepStride) {
      if (threadIdx.x == 0) atomicOr(status, kStatusLaunch);
      return;
    }
  }
  const int lane = threadIdx.x & 31;
  uint32_t *keep = nb_keep + (size_t)threadIdx.x * kNbKeepStride;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
  const double xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
  const int ci = cell_of[i];
  const int cx = ci % bin.nb[0], cy = (ci / bin.nb[0]) % bin.nb[1],
            cz = ci / (bin.nb[0] * bin.nb[1]);
  const int wx = 2 * bin.ns[0] + 1, wy = 2 * bin.ns[1] + 1, wz = 2 * bin.ns[2] + 1;
  const int S = wx * wy * wz;
  int out = 0;
  uint32_t *row = tmp + (size_t)i * cap;
  for (int base = 0; base < S; base += 32) {
    int s = base + lane;
    int c = -1, sh[3] = {0, 0, 0};
    if (s < S) {
      int o[3] = {s % wx - bin.ns[0], (s / wx) % wy - bin.ns[1],
                  s / (wx * wy) - bin.ns[2]};
      int cc[3] = {cx + o[0], cy + o[1], cz + o[2]};
      int w3[3];
      bool ok = true;
      for (int a = 0; a < 3; a++) {
        int q = cc[a];
        int sa = (q >= 0) ? q / bin.nb[a] : -((-q + bin.nb[a] - 1) / bin.nb[a]);
        w3[a] = q - sa * bin.nb[a];
        sh[a] = sa;
        if (!box.pbc[a] && sa != 0) ok = false;
        if (sa > kShiftR || sa < -kShiftR) {
          ok = false;
          atomicOr(status, kStatusShift);
        }
      }
      if (ok) c = (w3[2] * bin.nb[1] + w3[1]) * bin.nb[0] + w3[0];
    }
    int cnt = 0;
    int a0 = 0, a1 = 0;
    if (c >= 0) {
      a0 = cell_start[c];
      a1 = cell_start[c + 1];
    }
    const bool self_cell = (sh[0] == 0 && sh[1] == 0 && sh[2] == 0);
    const int code = shift_code(sh[0], sh[1], sh[2]);
    for (int p = a0; p < a1; p++) {
      int j = cell_atoms[p];
      if (j == i && self_cell) continue;
      double gx, gy, gz;
      image_of(box, x[3 * j], x[3 * j + 1], x[3 * j + 2], sh[0], sh[1], sh[2],
               gx, gy, gz);
      double r2 = rsq_nofma(xi - gx, yi - gy, zi - gz);
      if (r2 <= cutsq) {
        if (cnt < kNbKeep) keep[cnt] = nb_pack(j, code);
        cnt++;
      }
    }
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    int total = __shfl_sync(0xffffffffu, incl, 31);
    int pos = out + incl - cnt;
    if (cnt > 0 && cnt <= kNbKeep) {
      for (int q = 0; q < cnt; q++)
        if (pos + q < cap) row[pos + q] = keep[q];
    } else if (cnt > kNbKeep) {
      for (int p = a0; p < a1; p++) {
        int j = cell_atoms[p];
        if (j == i && self_cell) continue;
        double gx, gy, gz;
        image_of(box, x[3 * j], x[3 * j + 1], x[3 * j + 2], sh[0], sh[1], sh[2],
                 gx, gy, gz);
        double r2 = rsq_nofma(xi - gx, yi - gy, zi - gz);
        if (r2 <= cutsq) {
          if (pos < cap) row[pos] = nb_pack(j, code);
          pos++;
        }
      }
    }
    out += total;
  }
  if (lane == 0) {
    nraw[i] = out;
    if (out > cap) {
      atomicOr(status, kStatusOverflow);
      atomicMax(maxneed, out);
    }
  }
  }
}

// ---------------------------------------------------------------------
// Multi-cell batches: many small periodic cells, each in its own box.  Atoms
// of cell c are coff[c]..coff[c+1]-1 and see only atoms of their own cell
// and its images.  Every cell has its own grid of bins in fractional
// coordinates (CellGeom: nb bins per axis, at least cut/2 wide, a +-ns
// stencil reaching the cutoff); the bins of all cells share one set of bin
// arrays, cell c's from bin0.  A stencil bin beyond the grid is a bin of an
// image (shift = floor division by nb), so a cell narrower than the cutoff
// is walked under every image shift that can reach it.  The kept set is the
// same (j, shift) set as the single-box binned build, with the same FP64
// image construction and no-FMA rsq.  Only cells flagged for a rebuild are
// zeroed, binned, scanned, sorted and walked: a cell's binned atoms occupy
// its own atom range coff[c].., so the scan runs per cell, and a bin's atoms
// are cell_atoms[cell_start[b] .. cell_cursor[b]) once the fill has advanced
// the cursors (the next bin's start may belong to a cell left as it was).
// ---------------------------------------------------------------------
__device__ inline bool nbc_cell_flagged(const int *flag, const int *__restrict__ cflag, int c) {
  return (*flag & 2) || cflag[c];
}

__device__ inline int nbc_cell_bins(const CellGeom &g) { return g.nb[0] * g.nb[1] * g.nb[2]; }

// One block per flagged cell: zero its bin counts.
__global__ void k_nbc_zero(int ncells, const CellGeom *__restrict__ cgeom,
                           const int *__restrict__ cflag, int *__restrict__ cell_count,
                           const int *flag) {
  if (!*flag) return;
  for (int c = blockIdx.x; c < ncells; c += gridDim.x) {
    if (!nbc_cell_flagged(flag, cflag, c)) continue;
    const CellGeom &g = cgeom[c];
    const int nbc = nbc_cell_bins(g);
    for (int b = threadIdx.x; b < nbc; b += blockDim.x) cell_count[g.bin0 + b] = 0;
  }
}

// One warp per flagged cell: exclusive scan of its bin counts from coff[c].
__global__ void k_nbc_scan(int ncells, const CellGeom *__restrict__ cgeom,
                           const int *__restrict__ coff, const int *__restrict__ cflag,
                           const int *__restrict__ cell_count, int *__restrict__ cell_start,
                           int *__restrict__ cell_cursor, const int *flag) {
  if (!*flag) return;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int c = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; c < ncells; c += nw) {
    if (!nbc_cell_flagged(flag, cflag, c)) continue;
    const CellGeom &g = cgeom[c];
    const int nbc = nbc_cell_bins(g);
    int base = coff[c];
    for (int b0 = 0; b0 < nbc; b0 += 32) {
      const int b = b0 + lane;
      const int v = b < nbc ? cell_count[g.bin0 + b] : 0;
      int incl = v;
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (b < nbc) {
        cell_start[g.bin0 + b] = base + incl - v;
        cell_cursor[g.bin0 + b] = base + incl - v;
      }
      base += __shfl_sync(0xffffffffu, incl, 31);
    }
  }
}

// One block per flagged cell, a thread per bin: order each bin's atoms by
// index so the build is deterministic.
__global__ void k_nbc_cellsort(int ncells, const CellGeom *__restrict__ cgeom,
                               const int *__restrict__ cflag,
                               const int *__restrict__ cell_start,
                               const int *__restrict__ cell_cursor,
                               int *__restrict__ cell_atoms, const int *flag) {
  if (!*flag) return;
  for (int c = blockIdx.x; c < ncells; c += gridDim.x) {
    if (!nbc_cell_flagged(flag, cflag, c)) continue;
    const CellGeom &g = cgeom[c];
    const int nbc = nbc_cell_bins(g);
    for (int b = threadIdx.x; b < nbc; b += blockDim.x) {
      const int s0 = cell_start[g.bin0 + b], s1 = cell_cursor[g.bin0 + b];
      for (int a = s0 + 1; a < s1; a++) {
        const int v = cell_atoms[a];
        int q = a - 1;
        while (q >= s0 && cell_atoms[q] > v) {
          cell_atoms[q + 1] = cell_atoms[q];
          q--;
        }
        cell_atoms[q + 1] = v;
      }
    }
  }
}

__global__ void k_nbc_bin(int n, double *__restrict__ x, int *__restrict__ image,
                          const BoxP *__restrict__ cbox, const CellGeom *__restrict__ cgeom,
                          const int *__restrict__ acell, const int *__restrict__ cflag,
                          int *__restrict__ cell_of, int *__restrict__ cell_count,
                          int *status, const int *flag) {
  if (!*flag) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    if (!nb_rebuild(flag, cflag, acell, i)) continue;
    const int c = acell[i];
    const BoxP &box = cbox[c];
    const CellGeom &g = cgeom[c];
    double px, py, pz, f[3];
    wrap_atom(box, i, x, image, px, py, pz);
    frac_of(box, px, py, pz, f[0], f[1], f[2]);
    int q[3];
    for (int a = 0; a < 3; a++) {
      if (!box.pbc[a] && (f[a] < 0.0 || f[a] > 1.0)) atomicOr(status, kStatusOutside);
      int v = (int)floor(f[a] * g.nb[a]);
      q[a] = v < 0 ? 0 : (v >= g.nb[a] ? g.nb[a] - 1 : v);
    }
    const int bin = g.bin0 + (q[2] * g.nb[1] + q[1]) * g.nb[0] + q[0];
    cell_of[i] = bin;
    atomicAdd(&cell_count[bin], 1);
  }
}

__global__ void k_nbc_fill(int n, const int *__restrict__ cell_of,
                           const int *__restrict__ acell, const int *__restrict__ cflag,
                           int *__restrict__ cell_cursor, int *__restrict__ cell_atoms,
                           const int *flag) {
  if (!*flag) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    if (!nb_rebuild(flag, cflag, acell, i)) continue;
    const int pos = atomicAdd(&cell_cursor[cell_of[i]], 1);
    cell_atoms[pos] = i;
  }
}

// One warp per atom, lanes over the stencil bins with per-lane keep buffers
// (as k_nb_build), the box and grid of the atom's cell.
__global__ void k_nbc_build(int n, const double *__restrict__ x,
                            const BoxP *__restrict__ cbox,
                            const CellGeom *__restrict__ cgeom,
                            const int *__restrict__ acell, const int *__restrict__ cell_of,
                            const int *__restrict__ cell_start,
                            const int *__restrict__ cell_end,
                            const int *__restrict__ cell_atoms, double cutsq, int cap,
                            uint32_t *__restrict__ tmp, int *__restrict__ nraw, int *status,
                            int *maxneed, const int *__restrict__ cflag, const int *flag) {
  if (!*flag) return;
  extern __shared__ uint32_t nb_keep[];
  {
    uint32_t dyn;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
    if (dyn < sizeof(uint32_t) * blockDim.x * kNbKeepStride) {
      if (threadIdx.x == 0) atomicOr(status, kStatusLaunch);
      return;
    }
  }
  const int lane = threadIdx.x & 31;
  uint32_t *keep = nb_keep + (size_t)threadIdx.x * kNbKeepStride;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    if (!nb_rebuild(flag, cflag, acell, i)) continue;
    const int cidx = acell[i];
    const BoxP &box = cbox[cidx];
    const CellGeom &g = cgeom[cidx];
    const double xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
    const int ci = cell_of[i] - g.bin0;
    const int cx = ci % g.nb[0], cy = (ci / g.nb[0]) % g.nb[1], cz = ci / (g.nb[0] * g.nb[1]);
    const int wx = 2 * g.ns[0] + 1, wy = 2 * g.ns[1] + 1, wz = 2 * g.ns[2] + 1;
    const int S = wx * wy * wz;
    int out = 0;
    uint32_t *row = tmp + (size_t)i * cap;
    for (int base = 0; base < S; base += 32) {
      const int sidx = base + lane;
      int c = -1, sh[3] = {0, 0, 0};
      if (sidx < S) {
        const int o[3] = {sidx % wx - g.ns[0], (sidx / wx) % wy - g.ns[1],
                          sidx / (wx * wy) - g.ns[2]};
        const int cc[3] = {cx + o[0], cy + o[1], cz + o[2]};
        int w3[3];
        bool ok = true;
        for (int a = 0; a < 3; a++) {
          const int q = cc[a], nb = g.nb[a];
          const int sa = q >= 0 ? q / nb : -((-q + nb - 1) / nb);
          w3[a] = q - sa * nb;
          sh[a] = sa;
          if (!box.pbc[a] && sa != 0) ok = false;
          if (sa > kShiftR || sa < -kShiftR) {
            ok = false;
            atomicOr(status, kStatusShift);
          }
        }
        if (ok) c = g.bin0 + (w3[2] * g.nb[1] + w3[1]) * g.nb[0] + w3[0];
      }
      int cnt = 0, a0 = 0, a1 = 0;
      if (c >= 0) {
        a0 = cell_start[c];
        a1 = cell_end[c];
      }
      const bool self_img = (sh[0] == 0 && sh[1] == 0 && sh[2] == 0);
      const int code = shift_code(sh[0], sh[1], sh[2]);
      for (int p = a0; p < a1; p++) {
        const int j = cell_atoms[p];
        if (j == i && self_img) continue;
        double gx, gy, gz;
        image_of(box, x[3 * j], x[3 * j + 1], x[3 * j + 2], sh[0], sh[1], sh[2], gx, gy, gz);
        if (rsq_nofma(xi - gx, yi - gy, zi - gz) <= cutsq) {
          if (cnt < kNbKeep) keep[cnt] = nb_pack(j, code);
          cnt++;
        }
      }
      int incl = cnt;
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      int pos = out + incl - cnt;
      if (cnt > 0 && cnt <= kNbKeep) {
        for (int q = 0; q < cnt; q++)
          if (pos + q < cap) row[pos + q] = keep[q];
      } else if (cnt > kNbKeep) {
        for (int p = a0; p < a1; p++) {
          const int j = cell_atoms[p];
          if (j == i && self_img) continue;
          double gx, gy, gz;
          image_of(box, x[3 * j], x[3 * j + 1], x[3 * j + 2], sh[0], sh[1], sh[2], gx, gy,
                   gz);
          if (rsq_nofma(xi - gx, yi - gy, zi - gz) <= cutsq) {
            if (pos < cap) row[pos] = nb_pack(j, code);
            pos++;
          }
        }
      }
      out += total;
    }
    if (lane == 0) {
      nraw[i] = out;
      if (out > cap) {
        atomicOr(status, kStatusOverflow);
        atomicMax(maxneed, out);
      }
    }
  }
}

// One warp per atom: bitonic sort of the row by (block, packed key) in
// shared memory, then block offsets.
__global__ void k_nb_sort(int n, int B, KParams kp, const int *__restrict__ elem,
                          int cap, int capp, const uint32_t *__restrict__ tmp,
                          const int *__restrict__ nraw,
                          uint32_t *__restrict__ nbr, int *__restrict__ boff,
                          const int *__restrict__ acell, const int *__restrict__ cflag,
                          const int *flag) {
  if (!*flag) return;
  extern __shared__ unsigned long long sbuf[];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wpb = blockDim.x >> 5;
  for (int i = blockIdx.x * wpb + wib; i < n; i += gridDim.x * wpb) {
  if (!nb_rebuild(flag, cflag, acell, i)) continue;
  unsigned long long *s = sbuf + (size_t)wib * capp;
  __syncwarp();
  int cnt = min(nraw[i], cap);
  int ei = elem[i];
  const uint32_t *row = tmp + (size_t)i * cap;
  for (int t = lane; t < capp; t += 32) {
    unsigned long long v = ~0ull;
    if (t < cnt) {
      uint32_t e = row[t];
      int j = e & kAtomMask;
      int b = kp.eltij[ei * kMaxElt + elem[j]];
      v = ((unsigned long long)b << 32) | e;
    }
    s[t] = v;
  }
  __syncwarp();
  for (int k = 2; k <= capp; k <<= 1) {
    for (int jj = k >> 1; jj > 0; jj >>= 1) {
      for (int t = lane; t < capp; t += 32) {
        int p = t ^ jj;
        if (p > t) {
          unsigned long long a = s[t], c = s[p];
          bool up = ((t & k) == 0);
          if ((a > c) == up) {
            s[t] = c;
            s[p] = a;
          }
        }
      }
      __syncwarp();
    }
  }
  uint32_t *orow = nbr + (size_t)i * cap;
  for (int t = lane; t < cnt; t += 32) orow[t] = (uint32_t)(s[t] & 0xffffffffu);
  for (int b = 0; b <= B; b++) {
    int c = 0;
    for (int t = lane; t < cnt; t += 32) c += ((int)(s[t] >> 32) < b) ? 1 : 0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) boff[(size_t)i * (B + 1) + b] = c;
  }
  }
}

// The same sort for rows of up to 32*NQ entries, keys in registers: element
// e = q*32 + lane of the row is key q of the lane.  Network stages with a
// stride of 32 or more compare two keys of one lane; smaller strides compare
// with the partner lane through a shuffle (the lower element keeps the
// minimum of an ascending pair).  Same network as k_nb_sort, so the same
// order.
template <int NQ>
__global__ void k_nb_sort_reg(int n, int B, KParams kp, const int *__restrict__ elem,
                              int cap, const uint32_t *__restrict__ tmp,
                              const int *__restrict__ nraw, uint32_t *__restrict__ nbr,
                              int *__restrict__ boff, const int *__restrict__ acell,
                              const int *__restrict__ cflag, const int *flag) {
  if (!*flag) return;
  constexpr int CAPP = 32 * NQ;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
    if (!nb_rebuild(flag, cflag, acell, i)) continue;
    const int cnt = min(nraw[i], cap);
    const int ei = elem[i];
    const uint32_t *row = tmp + (size_t)i * cap;
    unsigned long long v[NQ];
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      const int t = q * 32 + lane;
      v[q] = ~0ull;
      if (t < cnt) {
        const uint32_t e = row[t];
        const int b = kp.eltij[ei * kMaxElt + elem[e & kAtomMask]];
        v[q] = ((unsigned long long)b << 32) | e;
      }
    }
#pragma unroll
    for (int k = 2; k <= CAPP; k <<= 1) {
#pragma unroll
      for (int jj = k >> 1; jj > 0; jj >>= 1) {
        if (jj >= 32) {
#pragma unroll
          for (int q = 0; q < NQ; q++) {
            const int p = q ^ (jj >> 5);
            if (p > q) {
              const bool up = ((q * 32) & k) == 0;
              const unsigned long long a = v[q], c = v[p];
              if ((a > c) == up) { v[q] = c; v[p] = a; }
            }
          }
        } else {
          const bool lower = (lane & jj) == 0;
#pragma unroll
          for (int q = 0; q < NQ; q++) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, v[q], jj);
            const bool up = ((q * 32 + lane) & k) == 0;
            const unsigned long long lo = v[q] < o ? v[q] : o, hi = v[q] < o ? o : v[q];
            v[q] = (lower == up) ? lo : hi;
          }
        }
      }
    }
    uint32_t *orow = nbr + (size_t)i * cap;
#pragma unroll
    for (int q = 0; q < NQ; q++) {
      const int t = q * 32 + lane;
      if (t < cnt) orow[t] = (uint32_t)(v[q] & 0xffffffffu);
    }
    for (int b = 0; b <= B; b++) {
      int c = 0;
#pragma unroll
      for (int q = 0; q < NQ; q++) {
        const int t = q * 32 + lane;
        c += (t < cnt && (int)(v[q] >> 32) < b) ? 1 : 0;
      }
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
      if (lane == 0) boff[(size_t)i * (B + 1) + b] = c;
    }
  }
}

// Partner slot of every entry: (j -> i, -shift) found by binary search in the
// sorted block of atom j.
__global__ void k_nb_rev(int n, int B, KParams kp, const int *__restrict__ elem,
                         int cap, const uint32_t *__restrict__ nbr,
                         const int *__restrict__ boff, int *__restrict__ rev,
                         const int *__restrict__ acell, const int *__restrict__ cflag,
                         const int *flag) {
  if (!*flag) return;
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
  if (!nb_rebuild(flag, cflag, acell, i)) continue;
  int cnt = boff[(size_t)i * (B + 1) + B];
  int ei = elem[i];
  for (int t = lane; t < cnt; t += 32) {
    uint32_t e = nbr[(size_t)i * cap + t];
    int j = e & kAtomMask;
    int code = e >> kAtomBits;
    uint32_t key = nb_pack(i, neg_code(code));
    int bj = kp.eltij[elem[j] * kMaxElt + ei];
    int lo = boff[(size_t)j * (B + 1) + bj], hi = boff[(size_t)j * (B + 1) + bj + 1];
    const uint32_t *rj = nbr + (size_t)j * cap;
    int found = -1;
    while (lo < hi) {
      int mid = (lo + hi) >> 1;
      uint32_t v = rj[mid];
      if (v == key) { found = mid; break; }
      if (v < key) lo = mid + 1; else hi = mid;
    }
    rev[(size_t)i * cap + t] = found >= 0 ? (int)((size_t)j * cap + found) : -1;
  }
  }
}

__global__ void k_nb_finish(int n, const double *__restrict__ x,
                            double *__restrict__ xbuild, const int *__restrict__ acell,
                            const int *__restrict__ cflag, int *flag) {
  if (!*flag) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += gridDim.x * blockDim.x) {
    if (!nb_rebuild(flag, cflag, acell, i)) continue;
    xbuild[3 * i] = x[3 * i];
    xbuild[3 * i + 1] = x[3 * i + 1];
    xbuild[3 * i + 2] = x[3 * i + 2];
  }
}

// Positions handed over by a caller each step (tmd_system_set_positions) are
// in the caller's periodic frame, which wraps atoms at other times than the
// list build does (LAMMPS wraps at its own reneighboring, a caller's
// integrator may never wrap).  Each atom takes the periodic image of its new
// position nearest to its position at the last build, so the list's image
// shifts stay valid and the displacement check sees the atom's motion rather
// than a box vector.  Shifts beyond 3 cells per axis are left alone (the
// check then rebuilds).  Image counters keep counting the device's own wraps.
__global__ void k_nearest_image(int n, double *__restrict__ x,
                                const double *__restrict__ xbuild, BoxP box,
                                const BoxP *__restrict__ cbox, const int *__restrict__ acell) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const BoxP &b = cbox ? cbox[acell[i]] : box;
  double f[3], g[3];
  frac_of(b, x[3 * i], x[3 * i + 1], x[3 * i + 2], f[0], f[1], f[2]);
  frac_of(b, xbuild[3 * i], xbuild[3 * i + 1], xbuild[3 * i + 2], g[0], g[1], g[2]);
  int k[3] = {0, 0, 0};
  for (int a = 0; a < 3; a++) {
    if (!b.pbc[a]) continue;
    const double d = rint(f[a] - g[a]);
    if (fabs(d) <= kShiftR) k[a] = (int)d;
  }
  if (k[0] || k[1] || k[2]) {
    double ox, oy, oz;
    image_of(b, x[3 * i], x[3 * i + 1], x[3 * i + 2], -k[0], -k[1], -k[2], ox, oy, oz);
    x[3 * i] = ox;
    x[3 * i + 1] = oy;
    x[3 * i + 2] = oz;
  }
}

void launch_nearest_image(int n, double *x, const double *xbuild, const BoxP &box,
                          const BoxP *cbox, const int *acell, cudaStream_t st, long &launches) {
  if (n <= 0) return;
  k_nearest_image<<<(n + 255) / 256, 256, 0, st>>>(n, x, xbuild, box, cbox, acell);
  launches += 1;
}

// Ghost-aware mode: rows of ghost atoms are built (their partner slots serve
// the local atoms' gather) but never evaluated, so after a build their pair
// forces and virial partials are set to zero once.
__global__ void k_nb_zero_ghost(int n, int nlocal, int cap, float4 *__restrict__ pdf,
                                double *__restrict__ wv, const int *flag) {
  if (!*flag) return;
  const long e0 = (long)nlocal * cap, e1 = (long)n * cap;
  for (long e = e0 + blockIdx.x * (long)blockDim.x + threadIdx.x; e < e1;
       e += (long)gridDim.x * blockDim.x)
    pdf[e] = make_float4(0.f, 0.f, 0.f, 0.f);
  for (long e = 6L * nlocal + blockIdx.x * (long)blockDim.x + threadIdx.x; e < 6L * n;
       e += (long)gridDim.x * blockDim.x)
    wv[e] = 0.0;
}

// End of the rebuild sequence: count a rebuild that ran (flag[1]) and clear
// the pending flag.
__global__ void k_nb_clear(int *flag) {
  if (flag[0]) flag[1] += 1;
  flag[0] = 0;
}

__global__ void k_set_flag(int *flag) { *flag = 3; }  // rebuild, every cell

// Host driver: the whole rebuild sequence on `st`.  All launches are
// conditional on *flag; `launches` counts them.
void launch_neighbor_build(const NbArgs &a, cudaStream_t st, long &launches) {
  // Grids are capped at a few waves of the 148 SMs and the kernels stride
  // over atoms, so a launch with no rebuild pending costs a few microseconds.
  const int T = 256;
  const int kMaxGrid = 148 * 8;
  auto cap_grid = [&](long g) { return (int)(g < 1 ? 1 : (g > kMaxGrid ? kMaxGrid : g)); };
  int gn = cap_grid((a.n + T - 1) / T);
  int gw = cap_grid(((long)a.n * 32 + T - 1) / T);
  if (a.ncells > 0) {
    const int gc = cap_grid(a.ncells);
    const int gcw = cap_grid(((long)a.ncells * 32 + T - 1) / T);
    k_nbc_zero<<<gc, T, 0, st>>>(a.ncells, a.cgeom, a.cflag, a.cell_count, a.flag);
    k_nbc_bin<<<gn, T, 0, st>>>(a.n, a.x, a.image, a.cbox, a.cgeom, a.acell, a.cflag,
                                a.cell_of, a.cell_count, a.status, a.flag);
    k_nbc_scan<<<gcw, T, 0, st>>>(a.ncells, a.cgeom, a.coff, a.cflag, a.cell_count,
                                  a.cell_start, a.cell_cursor, a.flag);
    k_nbc_fill<<<gn, T, 0, st>>>(a.n, a.cell_of, a.acell, a.cflag, a.cell_cursor,
                                 a.cell_atoms, a.flag);
    k_nbc_cellsort<<<gc, T, 0, st>>>(a.ncells, a.cgeom, a.cflag, a.cell_start, a.cell_cursor,
                                     a.cell_atoms, a.flag);
    k_nbc_build<<<gw, T, nb_build_smem(T), st>>>(
        a.n, a.x, a.cbox, a.cgeom, a.acell, a.cell_of, a.cell_start, a.cell_cursor,
        a.cell_atoms, a.cutsq, a.cap, a.tmp, a.nraw, a.status, a.maxneed, a.cflag, a.flag);
    launches += 6;
  } else {
    int gc = cap_grid((a.bin.ncell + T - 1) / T);
    k_nb_zero<<<gc, T, 0, st>>>(a.bin.ncell, a.cell_count, a.flag);
    k_nb_bin<<<gn, T, 0, st>>>(a.n, a.x, a.image, a.box, a.bin, a.cell_of,
                               a.cell_count, a.status, a.flag);
    k_nb_scan<<<1, 1024, 0, st>>>(a.bin.ncell, a.cell_count, a.cell_start,
                                  a.cell_cursor, a.flag);
    k_nb_fill<<<gn, T, 0, st>>>(a.n, a.cell_of, a.cell_cursor, a.cell_atoms, a.flag);
    k_nb_cellsort<<<gc, T, 0, st>>>(a.bin.ncell, a.cell_start, a.cell_atoms, a.flag);
    k_nb_build<<<gw, T, nb_build_smem(T), st>>>(
        a.n, a.x, a.box, a.bin, a.cell_of, a.cell_start, a.cell_atoms, a.cutsq, a.cap,
        a.tmp, a.nraw, a.status, a.maxneed, a.flag);
    launches += 6;
  }
  if (a.capp <= 256) {
#define TMD_SORT_REG(NQ)                                                                  \
  k_nb_sort_reg<NQ><<<gw, T, 0, st>>>(a.n, a.B, a.kp, a.elem, a.cap, a.tmp, a.nraw, a.nbr, \
                                      a.boff, a.acell, a.cflag, a.flag)
    switch (a.capp) {
      case 32: TMD_SORT_REG(1); break;
      case 64: TMD_SORT_REG(2); break;
      case 128: TMD_SORT_REG(4); break;
      default: TMD_SORT_REG(8); break;
    }
#undef TMD_SORT_REG
  } else {
    int wpb = a.capp >= 1024 ? 1 : (a.capp >= 512 ? 2 : 4);
    size_t smem = (size_t)wpb * a.capp * sizeof(unsigned long long);
    k_nb_sort<<<cap_grid((a.n + wpb - 1) / wpb), 32 * wpb, smem, st>>>(
        a.n, a.B, a.kp, a.elem, a.cap, a.capp, a.tmp, a.nraw, a.nbr, a.boff, a.acell, a.cflag,
        a.flag);
  }
  k_nb_rev<<<gw, T, 0, st>>>(a.n, a.B, a.kp, a.elem, a.cap, a.nbr, a.boff, a.rev, a.acell,
                             a.cflag, a.flag);
  k_nb_finish<<<gn, T, 0, st>>>(a.n, a.x, a.xbuild, a.acell, a.cflag, a.flag);
  if (a.cflag) {
    k_nbc_clear<<<cap_grid((a.ncells + T - 1) / T), T, 0, st>>>(a.ncells, a.cflag, a.flag);
    launches += 1;
  }
  if (a.pdf && a.nlocal < a.n) {
    k_nb_zero_ghost<<<cap_grid(((long)(a.n - a.nlocal) * a.cap + T - 1) / T), T, 0, st>>>(
        a.n, a.nlocal, a.cap, a.pdf, a.wv, a.flag);
    launches += 1;
  }
  k_nb_clear<<<1, 1, 0, st>>>(a.flag);
  launches += 4;
}

void launch_neighbor_check(int n, const double *x, const double *xbuild,
                           double trigsq, int *flag, cudaStream_t st,
                           long &launches, const int *acell, int *cflag) {
  const int T = 256;
  if (cflag)
    k_nbc_check<<<(n + T - 1) / T, T, 0, st>>>(n, x, xbuild, trigsq, acell, cflag, flag);
  else
    k_nb_check<<<(n + T - 1) / T, T, 0, st>>>(n, x, xbuild, trigsq, flag);
  launches += 1;
}

// The MD step graph's rebuild condition: 1 when the displacement check (or a
// forced rebuild) set the flag.
__global__ void k_rebuild_cond(cudaGraphConditionalHandle h, const int *flag) {
  cudaGraphSetConditional(h, flag[0] != 0 ? 1u : 0u);
}

void launch_rebuild_cond(cudaGraphConditionalHandle h, const int *flag, cudaStream_t st,
                         long &launches) {
  k_rebuild_cond<<<1, 1, 0, st>>>(h, flag);
  launches += 1;
}

void launch_set_flag(int *flag, cudaStream_t st, long &launches) {
  k_set_flag<<<1, 1, 0, st>>>(flag);
  launches += 1;
}

}  // namespace tmd
