// descriptor.cu -- tensor-moment descriptor P and rotation invariants G.
//
// For atom i and element block b (tensormd.cpp:165-176):
//   P[b,k,d] = sum_{j in b} H_k(r_ij) M_d(u_ij)       (kernel.cu:1105, cuBLAS
//                                                        strided GEMM there)
//   G[b,k,m] = sum_d T[m,d] P[b,k,d]^2, G[b,k,0] = sign(P0) sqrt(.)
//                                                      (kernel.cu:1028-1096)
// The reference materialises R, M and H per (atom, block, padded slot) and
// runs a batched GEMM; here a group of TPA = K/4 lanes owns one atom, each
// lane accumulates 4 filters x D monomials in registers, and the FP64 pair
// geometry of TPA neighbors at a time is computed once per lane and shared by
// shuffles.  Nothing per pair is written to memory.
//
// Output layout: P[n][B][K][D] (kept for the force kernel), G[n][B*K*M] (the
// MLP input rows, m fastest, as TensorMD::get_G).
#include "pair_math.cuh"
#include "tmd_kernels.h"

namespace tmd {

template <int TPA, int D>
__global__ void __launch_bounds__(128)
k_descriptor(KParams kp, BoxP box, int n, int cap, const double *__restrict__ x,
             const int *__restrict__ elem, const uint32_t *__restrict__ nbr,
             const int *__restrict__ boff, float *__restrict__ P,
             float *__restrict__ G) {
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
  for (int b = 0; b < B; b++) {
    float acc[4][D];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int d = 0; d < D; d++) acc[q][d] = 0.f;
    const int s0 = bo[b], s1 = bo[b + 1];
    for (int t0 = s0; t0 < s1; t0 += TPA) {
      PairGeo mine;
      mine.ti = -1;
      mine.r = mine.ux = mine.uy = mine.uz = mine.fc = mine.dfc = mine.tq = 0.f;
      if (t0 + sub < s1) pair_geometry(kp, box, x, xi, yi, zi, row[t0 + sub], mine);
      const int cnt = min(TPA, s1 - t0);
      for (int c = 0; c < cnt; c++) {
        PairGeo g = shfl_geo(gmask, mine, c, TPA);
        if (g.ti < 0) continue;
        float H[4], dH[4];
        radial4<false>(kp, k0, g, H, dH);
        float Mv[D];
        moments<D>(g.ux, g.uy, g.uz, Mv);
#pragma unroll
        for (int q = 0; q < 4; q++)
#pragma unroll
          for (int d = 0; d < D; d++) acc[q][d] = fmaf(H[q], Mv[d], acc[q][d]);
      }
    }
    // P rows of this lane: 4 filters x D values, contiguous
    float4 *Pp = reinterpret_cast<float4 *>(P + (((size_t)a * B + b) * K + k0) * D);
#pragma unroll
    for (int v = 0; v < D; v++) {
      Pp[v] = make_float4(acc[(4 * v) / D][(4 * v) % D], acc[(4 * v + 1) / D][(4 * v + 1) % D],
                          acc[(4 * v + 2) / D][(4 * v + 2) % D],
                          acc[(4 * v + 3) / D][(4 * v + 3) % D]);
    }
    // G = T P^2 for the 4 filters
    float *Gp = G + (size_t)a * kp.nin + ((size_t)b * K + k0) * M;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      for (int m = 0; m < M; m++) {
        float s = 0.f;
#pragma unroll
        for (int d = 0; d < D; d++) s = fmaf(kp.T[m * D + d], acc[q][d] * acc[q][d], s);
        if (m == 0) s = copysignf(1.f, acc[q][0]) * sqrtf(s);
        Gp[q * M + m] = s;
      }
    }
  }
}

template <int TPA>
static void launch_tpa(const DescArgs &a, cudaStream_t st) {
  const int T = 128;
  long threads = (long)a.n * TPA;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
  switch (a.kp.D) {
    case 1: k_descriptor<TPA, 1><<<grid, T, 0, st>>>(a.kp, a.box, a.n, a.cap, a.x, a.elem, a.nbr, a.boff, a.P, a.G); break;
    case 4: k_descriptor<TPA, 4><<<grid, T, 0, st>>>(a.kp, a.box, a.n, a.cap, a.x, a.elem, a.nbr, a.boff, a.P, a.G); break;
    case 10: k_descriptor<TPA, 10><<<grid, T, 0, st>>>(a.kp, a.box, a.n, a.cap, a.x, a.elem, a.nbr, a.boff, a.P, a.G); break;
    default: k_descriptor<TPA, 20><<<grid, T, 0, st>>>(a.kp, a.box, a.n, a.cap, a.x, a.elem, a.nbr, a.boff, a.P, a.G); break;
  }
}

void launch_descriptor(const DescArgs &a, cudaStream_t st, long &launches) {
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

}  // namespace tmd
