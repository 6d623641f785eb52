// force.cu -- dE_i/dx_j for every neighbor pair, without atomics.
//
// Reverse mode through the descriptor (tensormd.cpp:563-602):
//   dEdG'[b,k,0] = 0.5 dEdG[b,k,0] / G[b,k,0]   (0 if |G0| < 1e-8)
//   S[b,k,d] = dE/dP = 2 P[b,k,d] sum_m T[m,d] dEdG'[b,k,m]
//                                         (kernel.cu:775-817, tensor_ops.cpp:633-674)
//   U_k = sum_d S[k,d] M_d, V_d = sum_k S[k,d] H_k
//   df = (sum_k U_k dH_k) u + sum_d V_d dM_d/dx_j     (F1 + F2, kernel.cu:541-631,
//                                                       tensor_ops.cpp:126-190,470-535)
// The reference writes U, V, F1 and F2 per padded slot and scatters df with
// FP64 atomics (kernel.cu:1639-1758).  Here S stays in registers (4 filters x D
// per lane, TPA = K/4 lanes per atom), sum_d V_d dM_d/dx_j is evaluated as the
// gradient of the polynomial Q(u) = sum_d V_d M_d(u), and df (times the
// pair_coeff scale) goes to its slot pdf[i*cap + t].  The reaction -df on j is
// summed later by k_gather through the partner slot, in a fixed order.
//
// wv[i] = sum over i's pairs of -r_ij (x) df (xx, yy, zz, xy, xz, yz): the
// per-pair virial of sum_forces_device (kernel.cu:1714-1758); its sum over
// atoms is the global virial.
#include "pair_math.cuh"
#include "tmd_kernels.h"

namespace tmd {

template <int TPA, int D>
__global__ void __launch_bounds__(128)
k_force(KParams kp, BoxP box, int n, int cap, float scale,
        const double *__restrict__ x, const int *__restrict__ elem,
        const uint32_t *__restrict__ nbr, const int *__restrict__ boff,
        const float *__restrict__ P, const float *__restrict__ G,
        const float *__restrict__ dEdG, float4 *__restrict__ pdf,
        double *__restrict__ wv) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt / TPA;
  const int sub = gt % TPA;
  if (a >= n) return;
  const int lane = threadIdx.x & 31;
  const unsigned gmask =
      TPA == 32 ? 0xffffffffu : (((1u << TPA) - 1u) << (lane & ~(TPA - 1)));
  const int B = kp.B, K = kp.K, M = kp.M;
  const int k0 = 4 * sub;
  const double xi = x[3 * a], yi = x[3 * a + 1], zi = x[3 * a + 2];
  const uint32_t *row = nbr + (size_t)a * cap;
  const int *bo = boff + (size_t)a * (B + 1);
  double w6[6] = {0, 0, 0, 0, 0, 0};
  for (int b = 0; b < B; b++) {
    const int s0 = bo[b], s1 = bo[b + 1];
    if (s0 == s1) continue;
    // S = dE/dP for this lane's 4 filters
    float S[4][D];
    {
      const float *Pp = P + (((size_t)a * B + b) * K + k0) * D;
      const float *Gp = G + (size_t)a * kp.nin + ((size_t)b * K + k0) * M;
      const float *dGp = dEdG + (size_t)a * kp.nin + ((size_t)b * K + k0) * M;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        float gp[4] = {0.f, 0.f, 0.f, 0.f};
        for (int m = 0; m < M; m++) gp[m] = dGp[q * M + m];
        float g0 = Gp[q * M];
        gp[0] = fabsf(g0) < 1e-8f ? 0.f : gp[0] / g0 * 0.5f;
#pragma unroll
        for (int d = 0; d < D; d++) {
          float t = 0.f;
          for (int m = 0; m < M; m++) t = fmaf(gp[m], kp.T[m * D + d], t);
          S[q][d] = 2.f * t * Pp[q * D + d];
        }
      }
    }
    for (int t0 = s0; t0 < s1; t0 += TPA) {
      PairGeo mine;
      mine.ti = -1;
      mine.r = mine.ux = mine.uy = mine.uz = mine.fc = mine.dfc = mine.tq = 0.f;
      if (t0 + sub < s1) pair_geometry(kp, box, x, xi, yi, zi, row[t0 + sub], mine);
      const int cnt = min(TPA, s1 - t0);
      for (int c = 0; c < cnt; c++) {
        PairGeo g = shfl_geo(gmask, mine, c, TPA);
        float4 out = make_float4(0.f, 0.f, 0.f, 0.f);
        if (g.ti >= 0) {
          float H[4], dH[4];
          radial4<true>(kp, k0, g, H, dH);
          float Mv[D];
          moments<D>(g.ux, g.uy, g.uz, Mv);
          float f1 = 0.f;
          float V[D];
#pragma unroll
          for (int d = 0; d < D; d++) V[d] = 0.f;
#pragma unroll
          for (int q = 0; q < 4; q++) {
            float U = 0.f;
#pragma unroll
            for (int d = 0; d < D; d++) {
              U = fmaf(S[q][d], Mv[d], U);
              V[d] = fmaf(S[q][d], H[q], V[d]);
            }
            f1 = fmaf(U, dH[q], f1);
          }
          float gq[3], nvm;
          poly_grad<D>(V, g.ux, g.uy, g.uz, gq, nvm);
          const float rinv = 1.f / g.r;
          float fx = f1 * g.ux + (gq[0] - g.ux * nvm) * rinv;
          float fy = f1 * g.uy + (gq[1] - g.uy * nvm) * rinv;
          float fz = f1 * g.uz + (gq[2] - g.uz * nvm) * rinv;
#pragma unroll
          for (int o = TPA >> 1; o > 0; o >>= 1) {
            fx += __shfl_xor_sync(gmask, fx, o, TPA);
            fy += __shfl_xor_sync(gmask, fy, o, TPA);
            fz += __shfl_xor_sync(gmask, fz, o, TPA);
          }
          out = make_float4(fx * scale, fy * scale, fz * scale, 0.f);
          if (sub == 0) {
            double rx = (double)g.ux * g.r, ry = (double)g.uy * g.r,
                   rz = (double)g.uz * g.r;
            w6[0] -= rx * out.x;
            w6[1] -= ry * out.y;
            w6[2] -= rz * out.z;
            w6[3] -= rx * out.y;
            w6[4] -= rx * out.z;
            w6[5] -= ry * out.z;
          }
        }
        if (sub == 0) pdf[(size_t)a * cap + t0 + c] = out;
      }
    }
  }
  if (sub == 0) {
#pragma unroll
    for (int c = 0; c < 6; c++) wv[(size_t)a * 6 + c] = w6[c];
  }
}

template <int TPA>
static void launch_tpa(const ForceArgs &a, cudaStream_t st) {
  const int T = 128;
  long threads = (long)a.n * TPA;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
#define TMD_FORCE_ARGS a.kp, a.box, a.n, a.cap, a.scale, a.x, a.elem, a.nbr, a.boff, a.P, a.G, a.dEdG, a.pdf, a.wv
  switch (a.kp.D) {
    case 1: k_force<TPA, 1><<<grid, T, 0, st>>>(TMD_FORCE_ARGS); break;
    case 4: k_force<TPA, 4><<<grid, T, 0, st>>>(TMD_FORCE_ARGS); break;
    case 10: k_force<TPA, 10><<<grid, T, 0, st>>>(TMD_FORCE_ARGS); break;
    default: k_force<TPA, 20><<<grid, T, 0, st>>>(TMD_FORCE_ARGS); break;
  }
#undef TMD_FORCE_ARGS
}

void launch_force(const ForceArgs &a, cudaStream_t st, long &launches) {
  switch (a.kp.K / 4) {
    case 1: launch_tpa<1>(a, st); break;
    case 2: launch_tpa<2>(a, st); break;
    case 4: launch_tpa<4>(a, st); break;
    case 8: launch_tpa<8>(a, st); break;
    case 16: launch_tpa<16>(a, st); break;
    default: launch_tpa<32>(a, st); break;
  }
  launches += 1;
}

// ---------------------------------------------------------------------
// Gather: f_i = sum over own slots of (df_ij - df_ji), FP64, fixed order.
// 8 lanes per atom.
// ---------------------------------------------------------------------
__global__ void k_gather(int n, int cap, int B, const int *__restrict__ boff,
                         const float4 *__restrict__ pdf, const int *__restrict__ rev,
                         const uint32_t *__restrict__ nbr, const double *__restrict__ x,
                         BoxP box, const double *__restrict__ wv,
                         double *__restrict__ f, double *__restrict__ vatom) {
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt >> 3, sub = gt & 7;
  if (a >= n) return;
  const unsigned lane = threadIdx.x & 31;
  const unsigned gmask = 0xffu << (lane & ~7u);
  const int cnt = boff[(size_t)a * (B + 1) + B];
  double fx = 0, fy = 0, fz = 0;
  double v6[6] = {0, 0, 0, 0, 0, 0};
  const size_t base = (size_t)a * cap;
  for (int t = sub; t < cnt; t += 8) {
    float4 p = pdf[base + t];
    int rv = rev[base + t];
    float4 q = rv >= 0 ? pdf[rv] : make_float4(0.f, 0.f, 0.f, 0.f);
    fx += (double)p.x - (double)q.x;
    fy += (double)p.y - (double)q.y;
    fz += (double)p.z - (double)q.z;
    if (vatom) {
      uint32_t e = nbr[base + t];
      int j = e & kAtomMask;
      int sx, sy, sz;
      shift_decode(int(e >> kAtomBits), sx, sy, sz);
      double gx, gy, gz;
      image_of(box, x[3 * j], x[3 * j + 1], x[3 * j + 2], sx, sy, sz, gx, gy, gz);
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
  if (vatom) {
#pragma unroll
    for (int c = 0; c < 6; c++)
#pragma unroll
      for (int o = 4; o > 0; o >>= 1) v6[c] += __shfl_xor_sync(gmask, v6[c], o, 8);
  }
  if (sub == 0) {
    f[3 * a] = fx;
    f[3 * a + 1] = fy;
    f[3 * a + 2] = fz;
    if (vatom) {
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
  k_gather<<<grid, T, 0, st>>>(a.n, a.cap, a.B, a.boff, a.pdf, a.rev, a.nbr, a.x,
                               a.box, a.wv, a.f, a.vatom);
  launches += 1;
}

}  // namespace tmd
