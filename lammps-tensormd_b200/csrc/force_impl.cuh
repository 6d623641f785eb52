// force_impl.cuh -- dE_i/dx_j for every neighbor pair, without atomics.
//
// Reverse mode through the descriptor (tensormd.cpp:563-602):
//   dEdG'[b,k,0] = 0.5 dEdG[b,k,0] / G[b,k,0]   (0 if |G0| < 1e-8)
//   S[b,k,d] = dE/dP = 2 P[b,k,d] sum_m T[m,d] dEdG'[b,k,m]
//                                         (kernel.cu:775-817, tensor_ops.cpp:633-674)
//   U_k = sum_d S[k,d] M_d, V_d = sum_k S[k,d] H_k
//   df = (sum_k U_k dH_k) u + sum_d V_d dM_d/dx_j     (F1 + F2, kernel.cu:541-631,
//                                                       tensor_ops.cpp:126-190,470-535)
// S of an (atom, block) is formed when the kernel reaches the block (dedp_row).
// The reference writes U, V, F1 and F2 per padded slot and scatters df with
// FP64 atomics (kernel.cu:1639-1758).  Here S stays in registers (4 filters x D
// per lane as FP32 pairs, TPA = K/4 lanes per atom), U and V are packed FP32x2
// FMAs, sum_d V_d dM_d/dx_j is the gradient of the polynomial
// Q(u) = sum_d V_d M_d(u), and df (times the pair_coeff scale) goes to its
// slot pdf[i*cap + t] (zero for entries beyond rc).  Active pairs are queued
// in shared memory as in the descriptor kernel (PairRing).  The reaction -df
// on j is summed later by k_gather through the partner slot, in a fixed order.
//
// wv[i] = sum over i's pairs of -r_ij (x) df (xx, yy, zz, xy, xz, yz): the
// per-pair virial of sum_forces_device (kernel.cu:1714-1758), accumulated in
// FP64 by the lane that owns the pair in its chunk; its sum over atoms is the
// global virial.
#pragma once

#include "descriptor_impl.cuh"

namespace tmd {

// dE/dG' of one (atom, block, filter) row (kernel2_GPU, kernel.cu:730-848;
// tensor_ops.cpp:633-674): dE/dG'_m = dE/dG_m for m > 0 and
// dE/dG'_0 = 0.5 dE/dG_0 / G_0 (0 when |G_0| < 1e-8); then
// S[k][d] = 2 P[k][d] sum_m T[m][d] dE/dG'_m, m ascending.
__device__ inline void dedp_row_g(const float *__restrict__ G, const float *__restrict__ dEdG,
                                  size_t row, int M, float gp[4]) {
#pragma unroll
  for (int m = 0; m < 4; m++) gp[m] = m < M ? __ldg(dEdG + row * M + m) : 0.f;
  const float g0 = __ldg(G + row * M);
  gp[0] = fabsf(g0) < 1e-8f ? 0.f : gp[0] / g0 * 0.5f;
}
__device__ inline float dedp_elem(const float gp[4], const float *T, int D, int M, int d,
                                  float p) {
  float t = 0.f;
#pragma unroll
  for (int m = 0; m < 4; m++)
    if (m < M) t = fmaf(gp[m], T[m * D + d], t);
  return 2.f * t * p;
}

template <int TPA, int D, int RK, bool MULTI>
__global__ void __launch_bounds__(kPairThreads, 3)
k_force(KParams kp, BoxP box, int n, int cap, float scale,
        const double *__restrict__ x, const int *__restrict__ elem,
        const uint32_t *__restrict__ nbr, const int *__restrict__ boff,
        const float *__restrict__ P, const float *__restrict__ G,
        const float *__restrict__ dEdG, float4 *__restrict__ pdf,
        double *__restrict__ wv, const BoxP *__restrict__ cbox,
        const int *__restrict__ acell) {
  constexpr int D2 = (D + 1) / 2;
  __shared__ GeoSlot geo[2 * kPairThreads];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt / TPA;
  const int sub = gt % TPA;
  if (a >= n) return;
  const unsigned live = live_lanes(gt, (long)n * TPA);
  const int lane = threadIdx.x & 31;
  PairRing<TPA> pr;
  pr.sub = sub;
  pr.gshift = lane & ~(TPA - 1);
  pr.gmask = PairRing<TPA>::kBits << pr.gshift;
  pr.ring = geo + 2 * (threadIdx.x - sub);
  const unsigned gmask = pr.gmask;
  const int B = kp.B, K = kp.K;
  const int k0 = 4 * sub;
  const Radial4<RK> R = load_radial4<RK>(kp, k0);
  const BoxP &bx = box_of<MULTI>(box, cbox, acell, a);
  const double xi = x[3 * a], yi = x[3 * a + 1], zi = x[3 * a + 2];
  const uint32_t *row = nbr + (size_t)a * cap;
  const int *bo = boff + (size_t)a * (B + 1);
  double w6[6] = {0, 0, 0, 0, 0, 0};
  for (int b = 0; b < B; b++) {
    // the warp's groups wait for each other at the end of every element
    // block, so no group runs ahead into the next block while others still
    // work on this one (that would split the warp across two copies of the
    // pair loop)
    if (b > 0) __syncwarp(live);
    const int s0 = bo[b], s1 = bo[b + 1];
    if (s0 == s1) continue;
    // S = dE/dP of this lane's 4 filters as FP32 pairs over d, formed here
    // (a rolled loop: the pair loop below must stay in the instruction cache)
    float2 S2[4][D2];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int p = 0; p < D2; p++) S2[q][p] = make_float2(0.f, 0.f);
    {
      const size_t row0 = ((size_t)a * B + b) * K + k0;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        float gp[4];
        dedp_row_g(G, dEdG, row0 + q, kp.M, gp);
        const float *Pp = P + (row0 + q) * D;
#pragma unroll
        for (int p = 0; p < D2; p++) {
          const float s0 = dedp_elem(gp, kp.T, D, kp.M, 2 * p, __ldg(Pp + 2 * p));
          const float s1 = 2 * p + 1 < D
                               ? dedp_elem(gp, kp.T, D, kp.M, 2 * p + 1, __ldg(Pp + 2 * p + 1))
                               : 0.f;
          S2[q][p] = make_float2(s0, s1);
        }
      }
    }
    float4 *pdf_row = pdf + (size_t)a * cap;
    pr.begin(x, row, s0, s1);
    for (;;) {
      // inactive entries get their zero pdf inside feed()
      const int cnt = pr.feed(kp, bx, xi, yi, zi, x, row, pdf_row);
      if (cnt == 0) break;
      float3 mydf = make_float3(0.f, 0.f, 0.f);
      for (int c = 0; c < cnt; c++) {
        const PairGeo g = geo_load(pr.slot(c));
        float H[4], dH[4];
        radial4<RK, true>(kp, R, g, H, dH);
        float2 M2[D2];
        moments2<D, D2>(g.ux, g.uy, g.uz, M2);
        // V_d = sum_k S[k,d] H_k and W_d = sum_k S[k,d] dH_k: 2 x D2
        // independent FFMA2 chains of length 4; then the F1 scalar
        // sum_k U_k dH_k = sum_d M_d W_d as two interleaved partial dots
        float2 V2[D2], W2[D2];
#pragma unroll
        for (int p = 0; p < D2; p++) {
          V2[p] = make_float2(0.f, 0.f);
          W2[p] = make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
          const float2 h2 = make_float2(H[q], H[q]);
          const float2 d2 = make_float2(dH[q], dH[q]);
#pragma unroll
          for (int p = 0; p < D2; p++) {
            V2[p] = __ffma2_rn(S2[q][p], h2, V2[p]);
            W2[p] = __ffma2_rn(S2[q][p], d2, W2[p]);
          }
        }
        float2 fa = make_float2(0.f, 0.f), fb = make_float2(0.f, 0.f);
#pragma unroll
        for (int p = 0; p < D2; p += 2) {
          fa = __ffma2_rn(M2[p], W2[p], fa);
          if (p + 1 < D2) fb = __ffma2_rn(M2[p + 1], W2[p + 1], fb);
        }
        const float f1 = (fa.x + fb.x) + (fa.y + fb.y);
        float V[2 * D2];
#pragma unroll
        for (int p = 0; p < D2; p++) { V[2 * p] = V2[p].x; V[2 * p + 1] = V2[p].y; }
        float gq[3], nvm;
        poly_grad<D>(V, g.ux, g.uy, g.uz, gq, nvm);
        const float rinv = g.rinv;
        float fx = f1 * g.ux + (gq[0] - g.ux * nvm) * rinv;
        float fy = f1 * g.uy + (gq[1] - g.uy * nvm) * rinv;
        float fz = f1 * g.uz + (gq[2] - g.uz * nvm) * rinv;
#pragma unroll
        for (int o = TPA >> 1; o > 0; o >>= 1) {
          fx += __shfl_xor_sync(gmask, fx, o, TPA);
          fy += __shfl_xor_sync(gmask, fy, o, TPA);
          fz += __shfl_xor_sync(gmask, fz, o, TPA);
        }
        if (c == sub) mydf = make_float3(fx * scale, fy * scale, fz * scale);
      }
      // lane c owns pair c of the chunk: store its pdf slot and add its
      // virial, with the separation as r (hi + lo) times u
      if (sub < cnt) {
        const GeoSlot *s = pr.slot(sub);
        const float4 ga = s->a, gb = s->b;
        const int t = __float_as_int(s->c.y);
        pdf_row[t] = make_float4(mydf.x, mydf.y, mydf.z, 0.f);
        double rr = (double)ga.x + (double)ga.y;
        double rx = (double)gb.x * rr, ry = (double)gb.y * rr, rz = (double)gb.z * rr;
        w6[0] -= rx * mydf.x;
        w6[1] -= ry * mydf.y;
        w6[2] -= rz * mydf.z;
        w6[3] -= rx * mydf.y;
        w6[4] -= rx * mydf.z;
        w6[5] -= ry * mydf.z;
      }
      pr.pop(cnt);
    }
  }
#pragma unroll
  for (int c = 0; c < 6; c++) {
#pragma unroll
    for (int o = TPA >> 1; o > 0; o >>= 1) w6[c] += __shfl_xor_sync(gmask, w6[c], o, TPA);
  }
  if (sub == 0) {
#pragma unroll
    for (int c = 0; c < 6; c++) wv[(size_t)a * 6 + c] = w6[c];
  }
}

template <int TPA, int RK, bool MULTI>
void launch_force_tpa(const ForceArgs &a, cudaStream_t st) {
  const int T = kPairThreads;
  long threads = (long)a.n * TPA;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
#define TMD_FORCE_ARGS a.kp, a.box, a.n, a.cap, a.scale, a.x, a.elem, a.nbr, a.boff, a.P, a.G, a.dEdG, a.pdf, a.wv, a.cbox, a.acell
  switch (a.kp.D) {
    case 1: k_force<TPA, 1, RK, MULTI><<<grid, T, 0, st>>>(TMD_FORCE_ARGS); break;
    case 4: k_force<TPA, 4, RK, MULTI><<<grid, T, 0, st>>>(TMD_FORCE_ARGS); break;
    case 10: k_force<TPA, 10, RK, MULTI><<<grid, T, 0, st>>>(TMD_FORCE_ARGS); break;
    default: k_force<TPA, 20, RK, MULTI><<<grid, T, 0, st>>>(TMD_FORCE_ARGS); break;
  }
#undef TMD_FORCE_ARGS
}

}  // namespace tmd

#include "force_pl.cuh"

namespace tmd {

// One radial kind and box mode per translation unit (parallel compilation).
template <int RK, bool MULTI>
void launch_force_rk(const ForceArgs &a, cudaStream_t st) {
  if (a.variant != kForceFilterLane) {
    launch_force_pl<RK, MULTI>(a, st);
    return;
  }
  switch (a.kp.K / 4) {
    case 1: launch_force_tpa<1, RK, MULTI>(a, st); break;
    case 2: launch_force_tpa<2, RK, MULTI>(a, st); break;
    case 4: launch_force_tpa<4, RK, MULTI>(a, st); break;
    case 8: launch_force_tpa<8, RK, MULTI>(a, st); break;
    case 16: launch_force_tpa<16, RK, MULTI>(a, st); break;
    default: launch_force_tpa<32, RK, MULTI>(a, st); break;
  }
}

}  // namespace tmd
