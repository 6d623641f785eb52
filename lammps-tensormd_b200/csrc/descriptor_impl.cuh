// descriptor_impl.cuh -- tensor-moment descriptor P and rotation invariants G.
//
// For atom i and element block b (tensormd.cpp:165-176):
//   P[b,k,d] = sum_{j in b} H_k(r_ij) M_d(u_ij)       (kernel.cu:1105, cuBLAS
//                                                        strided GEMM there)
//   G[b,k,m] = sum_d T[m,d] P[b,k,d]^2, G[b,k,0] = sign(P0) sqrt(.)
//                                                      (kernel.cu:1028-1096)
// The reference materialises R, M and H per (atom, block, padded slot) and
// runs a batched GEMM; here a group of TPA = K/4 lanes owns one atom and each
// lane accumulates 4 filters x D monomials in registers with packed FP32x2
// FMAs (sm_100 FFMA2).  Each lane computes the FP64 geometry of one pair of a
// chunk of TPA neighbors and publishes it in shared memory; the group then
// reads each pair with vector loads (broadcast).  Neighbor entries are fetched
// two chunks ahead and neighbor positions one chunk ahead, so the gather
// latency overlaps the arithmetic.  Nothing per pair goes to global memory.
//
// Output layout: P[n][B][K][D] (kept for the force kernel), G[n][B*K*M] (the
// MLP input rows, m fastest, as TensorMD::get_G).
#pragma once

#include "pair_math.cuh"
#include "tmd_kernels.h"

namespace tmd {

constexpr int kPairThreads = 128;  // block size of the pair kernels

// Geometry slot in shared memory: three 16-byte vectors per lane.
struct GeoSlot {
  float4 a;  // r, rlo, ux, uy
  float4 b;  // uz, fc, dfc, tq
  float4 c;  // ti (bits), unused
};

__device__ inline void geo_store(GeoSlot *s, const PairGeo &g) {
  s->a = make_float4(g.r, g.rlo, g.ux, g.uy);
  s->b = make_float4(g.uz, g.fc, g.dfc, g.tq);
  s->c = make_float4(__int_as_float(g.ti), 0.f, 0.f, 0.f);
}

__device__ inline PairGeo geo_load(const GeoSlot *s) {
  PairGeo g;
  float4 a = s->a, b = s->b;
  g.r = a.x; g.rlo = a.y; g.ux = a.z; g.uy = a.w;
  g.uz = b.x; g.fc = b.y; g.dfc = b.z; g.tq = b.w;
  g.ti = __float_as_int(s->c.x);
  return g;
}

// Monomials as FP32 pairs (D2 = ceil(D/2), the last pair padded with 0).
template <int D, int D2>
__device__ inline void moments2(float x, float y, float z, float2 M2[D2]) {
  float M[2 * D2];
  moments<D>(x, y, z, M);
  if (D & 1) M[D] = 0.f;
#pragma unroll
  for (int p = 0; p < D2; p++) M2[p] = make_float2(M[2 * p], M[2 * p + 1]);
}

template <int TPA, int D, int RK>
__global__ void __launch_bounds__(kPairThreads, 4)
k_descriptor(KParams kp, BoxP box, int n, int cap, const double *__restrict__ x,
             const int *__restrict__ elem, const uint32_t *__restrict__ nbr,
             const int *__restrict__ boff, float *__restrict__ P,
             float *__restrict__ G) {
  constexpr int D2 = (D + 1) / 2;
  __shared__ GeoSlot geo[kPairThreads];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt / TPA;
  const int sub = gt % TPA;
  if (a >= n) return;
  const int lane = threadIdx.x & 31;
  const unsigned gmask =
      TPA == 32 ? 0xffffffffu : (((1u << TPA) - 1u) << (lane & ~(TPA - 1)));
  GeoSlot *gslot = geo + (threadIdx.x - sub);  // slots of this atom's group
  const int B = kp.B, K = kp.K, M = kp.M;
  const int k0 = 4 * sub;
  const Radial4<RK> R = load_radial4<RK>(kp, k0);
  const double xi = x[3 * a], yi = x[3 * a + 1], zi = x[3 * a + 2];
  const uint32_t *row = nbr + (size_t)a * cap;
  const int *bo = boff + (size_t)a * (B + 1);
  for (int b = 0; b < B; b++) {
    float2 acc[4][D2];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int p = 0; p < D2; p++) acc[q][p] = make_float2(0.f, 0.f);
    const int s0 = bo[b], s1 = bo[b + 1];
    NbPos pnext = load_nb(x, s0 + sub < s1 ? row[s0 + sub] : 0u, s0 + sub < s1);
    uint32_t enext = (s0 + TPA + sub < s1) ? row[s0 + TPA + sub] : 0u;
    for (int t0 = s0; t0 < s1; t0 += TPA) {
      const NbPos pc = pnext;
      pnext = load_nb(x, enext, t0 + TPA + sub < s1);
      enext = (t0 + 2 * TPA + sub < s1) ? row[t0 + 2 * TPA + sub] : 0u;
      PairGeo mine;
      pair_geometry(kp, box, xi, yi, zi, pc, mine);
      __syncwarp(gmask);
      geo_store(gslot + sub, mine);
      __syncwarp(gmask);
      const int cnt = min(TPA, s1 - t0);
      for (int c = 0; c < cnt; c++) {
        const PairGeo g = geo_load(gslot + c);
        if (g.ti < 0) continue;
        float H[4], dH[4];
        radial4<RK, false>(kp, R, g, H, dH);
        float2 M2[D2];
        moments2<D, D2>(g.ux, g.uy, g.uz, M2);
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const float2 h2 = make_float2(H[q], H[q]);
#pragma unroll
          for (int p = 0; p < D2; p++) acc[q][p] = __ffma2_rn(h2, M2[p], acc[q][p]);
        }
      }
    }
    // P rows of this lane: 4 filters x D values, contiguous
    float *Pp = P + (((size_t)a * B + b) * K + k0) * D;
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int d = 0; d < D; d++) Pp[q * D + d] = (d & 1) ? acc[q][d >> 1].y : acc[q][d >> 1].x;
    // G = T P^2 for the 4 filters
    float *Gp = G + (size_t)a * kp.nin + ((size_t)b * K + k0) * M;
#pragma unroll
    for (int q = 0; q < 4; q++) {
      for (int m = 0; m < M; m++) {
        float s = 0.f;
#pragma unroll
        for (int d = 0; d < D; d++) {
          float pv = (d & 1) ? acc[q][d >> 1].y : acc[q][d >> 1].x;
          s = fmaf(kp.T[m * D + d], pv * pv, s);
        }
        if (m == 0) s = copysignf(1.f, acc[q][0].x) * sqrtf(s);
        Gp[q * M + m] = s;
      }
    }
  }
}

template <int TPA, int RK>
void launch_descriptor_tpa(const DescArgs &a, cudaStream_t st) {
  const int T = kPairThreads;
  long threads = (long)a.n * TPA;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
#define TMD_DESC_ARGS a.kp, a.box, a.n, a.cap, a.x, a.elem, a.nbr, a.boff, a.P, a.G
  switch (a.kp.D) {
    case 1: k_descriptor<TPA, 1, RK><<<grid, T, 0, st>>>(TMD_DESC_ARGS); break;
    case 4: k_descriptor<TPA, 4, RK><<<grid, T, 0, st>>>(TMD_DESC_ARGS); break;
    case 10: k_descriptor<TPA, 10, RK><<<grid, T, 0, st>>>(TMD_DESC_ARGS); break;
    default: k_descriptor<TPA, 20, RK><<<grid, T, 0, st>>>(TMD_DESC_ARGS); break;
  }
#undef TMD_DESC_ARGS
}

template <int RK>
void launch_descriptor_rk(const DescArgs &a, cudaStream_t st) {
  switch (a.kp.K / 4) {
    case 1: launch_descriptor_tpa<1, RK>(a, st); break;
    case 2: launch_descriptor_tpa<2, RK>(a, st); break;
    case 4: launch_descriptor_tpa<4, RK>(a, st); break;
    case 8: launch_descriptor_tpa<8, RK>(a, st); break;
    case 16: launch_descriptor_tpa<16, RK>(a, st); break;
    default: launch_descriptor_tpa<32, RK>(a, st); break;
  }
}

}  // namespace tmd
