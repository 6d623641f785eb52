// force.cu -- dispatch of the pair-force kernel on the radial kind and the
// box mode (single-box Gaussian instantiated here; the other variants in
// force_table.cu, force_generic.cu, force_cells.cu and force_cells_other.cu)
// and the atomics-free force gather.
#include "force_impl.cuh"

namespace tmd {

void launch_force_table(const ForceArgs &a, cudaStream_t st);
void launch_force_generic(const ForceArgs &a, cudaStream_t st);
void launch_force_gauss_cells(const ForceArgs &a, cudaStream_t st);
void launch_force_table_cells(const ForceArgs &a, cudaStream_t st);
void launch_force_generic_cells(const ForceArgs &a, cudaStream_t st);

void launch_force(const ForceArgs &a, cudaStream_t st, long &launches) {
  const bool cells = a.cbox != nullptr;
  switch (radial_kind(a.kp)) {
    case kRadTable:
      if (cells) launch_force_table_cells(a, st); else launch_force_table(a, st);
      break;
    case kRadGauss:
      if (cells) launch_force_gauss_cells(a, st); else launch_force_rk<kRadGauss, false>(a, st);
      break;
    default:
      if (cells) launch_force_generic_cells(a, st); else launch_force_generic(a, st);
      break;
  }
  launches += 1;
}

// ---------------------------------------------------------------------
// Gather: f_i = sum over own slots of (df_ij - df_ji), FP64, fixed order.
// df_ji is read from the partner slot rev[t] written by atom j, so every
// atom sums its own row and no two threads write the same force.  8 lanes
// per atom.
// ---------------------------------------------------------------------
template <bool VATOM>
__global__ void k_gather(int n, int cap, int B, const int *__restrict__ boff,
                         const float4 *__restrict__ pdf, const int *__restrict__ rev,
                         const uint32_t *__restrict__ nbr, const double *__restrict__ x,
                         BoxP box, const double *__restrict__ wv,
                         double *__restrict__ f, double *__restrict__ vatom,
                         const BoxP *__restrict__ cbox, const int *__restrict__ acell) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt >> 3, sub = gt & 7;
  if (a >= n) return;
  const unsigned lane = threadIdx.x & 31;
  const unsigned gmask = 0xffu << (lane & ~7u);
  const int cnt = boff[(size_t)a * (B + 1) + B];
  double fx = 0, fy = 0, fz = 0;
  double v6[6] = {0, 0, 0, 0, 0, 0};
  const size_t base = (size_t)a * cap;
  int t0 = sub;
  if (!VATOM) {
    // four of the lane's entries per round: their rev slots and own pair
    // forces, then the partners' pair forces, all in flight together; the
    // sums run in the same order as the one-entry loop below
    for (; t0 + 24 < cnt; t0 += 32) {
      int rv[4];
      float4 p[4], q[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        rv[u] = rev[base + t0 + 8 * u];
        p[u] = pdf[base + t0 + 8 * u];
      }
#pragma unroll
      for (int u = 0; u < 4; u++) q[u] = rv[u] >= 0 ? pdf[rv[u]] : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
      for (int u = 0; u < 4; u++) {
        fx += (double)p[u].x - (double)q[u].x;
        fy += (double)p[u].y - (double)q[u].y;
        fz += (double)p[u].z - (double)q[u].z;
      }
    }
  }
  for (int t = t0; t < cnt; t += 8) {
    float4 p = pdf[base + t];
    int rv = rev[base + t];
    float4 q = rv >= 0 ? pdf[rv] : make_float4(0.f, 0.f, 0.f, 0.f);
    fx += (double)p.x - (double)q.x;
    fy += (double)p.y - (double)q.y;
    fz += (double)p.z - (double)q.z;
    if (VATOM) {
      uint32_t e = nbr[base + t];
      int j = e & kAtomMask;
      int sx, sy, sz;
      shift_decode(int(e >> kAtomBits), sx, sy, sz);
      double gx, gy, gz;
      image_of(cbox ? cbox[acell[a]] : box, x[3 * j], x[3 * j + 1], x[3 * j + 2], sx, sy,
               sz, gx, gy, gz);
      double rx = gx - x[3 * a], ry = gy - x[3 * a + 1], rz = gz - x[3 * a + 2];
      v6[0] += rx * q.x;
      v6[1] += ry * q.y;
      v6[2] += rz * q.z;
      v6[3] += rx * q.y;
      v6[4] += rx * q.z;
      v6[5] += ry * q.z;
    }
  }
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) {
    fx += __shfl_xor_sync(gmask, fx, o, 8);
    fy += __shfl_xor_sync(gmask, fy, o, 8);
    fz += __shfl_xor_sync(gmask, fz, o, 8);
  }
  if (VATOM) {
#pragma unroll
    for (int c = 0; c < 6; c++)
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) v6[c] += __shfl_xor_sync(gmask, v6[c], o, 8);
  }
  if (sub == 0) {
    f[3 * a] = fx;
    f[3 * a + 1] = fy;
    f[3 * a + 2] = fz;
    if (VATOM) {
#pragma unroll
      for (int c = 0; c < 6; c++) vatom[6 * a + c] = 0.5 * (wv[6 * a + c] + v6[c]);
    }
  }
}

void launch_gather(const GatherArgs &a, cudaStream_t st, long &launches) {
  const int T = 256;
  long threads = (long)a.n * 8;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
  if (a.vatom)
    k_gather<true><<<grid, T, 0, st>>>(a.n, a.cap, a.B, a.boff, a.pdf, a.rev, a.nbr, a.x,
                                       a.box, a.wv, a.f, a.vatom, a.cbox, a.acell);
  else
    k_gather<false><<<grid, T, 0, st>>>(a.n, a.cap, a.B, a.boff, a.pdf, a.rev, a.nbr, a.x,
                                        a.box, a.wv, a.f, a.vatom, a.cbox, a.acell);
  launches += 1;
}

}  // namespace tmd
