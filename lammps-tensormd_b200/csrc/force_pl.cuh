// force_pl.cuh -- pair-per-lane form of the pair-force kernel.
//
// Same mathematics and outputs as k_force (force_impl.cuh): S = dE/dP of each
// (atom, element block) formed from P, G and dE/dG when the group reaches the
// block (dedp_row_g / dedp_elem), then for every active
// pair of atom i, V_d = sum_k S[k,d] H_k, W_d = sum_k S[k,d] dH_k,
// df = (sum_d M_d W_d) u + grad Q(V) / r, scaled, into pdf[i*cap + t]; FP64
// per-atom virial into wv[i].
//
// k_force gives each lane 4 filters of an atom and sums the lanes' partial
// forces, so every lane of the atom's group evaluates the monomials, the
// gradient of Q and the force expression of every pair.  Here W lanes share
// one atom and each lane takes whole pairs: S of the current element block
// (K x D floats) is staged once in shared memory and read by all lanes of the
// group as broadcast vectors, and the monomials, grad Q and the force of a
// pair are computed once.  The pairs are the compact list of active pairs
// that the descriptor step wrote (pgeo, pcnt: geometry computed once per
// step, skin-shell entries already given a zero pair force); lane c of the
// group takes pair c of each chunk of W, so only the last chunk of a block
// leaves lanes idle.
#pragma once

#include <algorithm>

#include "descriptor_impl.cuh"

namespace tmd {

// Shared-memory layout of k_force_pl (floats): radial parameters [4][K] (none
// for the table kind) and T [4][D4], then per atom group an S block [K][D4]
// + 4 (the extra 4 floats put consecutive groups' blocks in different banks)
// and the dE/dG' rows [K][4].
template <int D>
struct PlLayout {
  static constexpr int D4 = (D + 3) / 4 * 4;
  static __host__ __device__ inline int params(int K, int rk) {
    return (rk == kRadTable ? 0 : 4 * K) + 4 * D4;
  }
  static __host__ __device__ inline int group(int K) { return K * D4 + 4 + 4 * K; }
  static __host__ inline size_t bytes(int K, int rk, int groups) {
    return sizeof(float) * ((size_t)params(K, rk) + (size_t)groups * group(K));
  }
};

// KC: the filter count when fixed at compile time (0: kp.K at run time); with
// it the filter loop unrolls fully and the radial basis of the next filters
// can be scheduled beside the contraction of the current ones.
template <int W, int D, int RK, bool MULTI, int KC = 0>
__global__ void __launch_bounds__(kPairThreads, 4)
k_force_pl(KParams kp, BoxP box, int n, int cap, float scale,
           const double *__restrict__ x, const int *__restrict__ elem,
           const uint32_t *__restrict__ nbr, const int *__restrict__ boff,
           const float *__restrict__ P, const float *__restrict__ G,
           const float *__restrict__ dEdG, float4 *__restrict__ pdf,
           double *__restrict__ wv, const BoxP *__restrict__ cbox,
           const int *__restrict__ acell, const float4 *__restrict__ pgeo,
           const int *__restrict__ pcnt) {
  using L = PlLayout<D>;
  constexpr int D4 = L::D4;
  constexpr int P2 = D4 / 2;  // FP32 pairs per S row (pad columns hold 0)
  extern __shared__ float4 pl_dyn[];
  const int K = KC > 0 ? KC : kp.K, B = kp.B, M = kp.M;
  float *rp = reinterpret_cast<float *>(pl_dyn);
  float *Ts = rp + (RK == kRadTable ? 0 : 4 * K);  // T[m][d], rows of D4
  for (int i = threadIdx.x; i < 4 * D4; i += blockDim.x) {
    const int m = i / D4, d = i - m * D4;
    Ts[i] = (m < M && d < D) ? kp.T[m * D + d] : 0.f;
  }
  if (RK != kRadTable) {
    for (int i = threadIdx.x; i < K; i += blockDim.x) {
      rp[i] = RK == kRadGauss ? kp.p1[i] : kp.p0[i];
      rp[K + i] = RK == kRadGauss ? kp.p1lo[i] : kp.p1[i];
      rp[2 * K + i] = RK == kRadGauss ? -2.f * kp.gc[i] : kp.p2[i];
      rp[3 * K + i] = RK == kRadGauss ? -kp.gcl[i] : 0.f;
    }
  }
  __syncthreads();
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt / W;
  const int sub = gt % W;
  if (a >= n) return;
  const unsigned live = live_lanes(gt, (long)n * W);
  const int lane = threadIdx.x & 31;
  const unsigned gmask = PairRing<W>::kBits << (lane & ~(W - 1));
  float *Sg = rp + L::params(K, RK) + (threadIdx.x / W) * L::group(K);
  float *gpg = Sg + K * D4 + 4;  // dE/dG' rows [K][4]
  const float4 *pg_row = pgeo + (size_t)a * cap * 2;
  float4 *pdf_row = pdf + (size_t)a * cap;
  float w6[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int pos = 0;  // first active pair of the block in the compact list
  for (int b = 0; b < B; b++) {
    if (b > 0) __syncwarp(live);  // keep the warp's groups on the same block
    const int np = pcnt[(size_t)a * B + b];
    if (np == 0) continue;
    // S = dE/dP of (atom, block) as [K][D4] rows: dE/dG' rows first, then
    // one element per lane step (same arithmetic and order as dedp_elem)
    __syncwarp(gmask);
    const size_t row0 = ((size_t)a * B + b) * K;
    for (int k = sub; k < K; k += W) {
      float gp[4];
      dedp_row_g(G, dEdG, row0 + k, M, gp);
      *reinterpret_cast<float4 *>(gpg + 4 * k) = make_float4(gp[0], gp[1], gp[2], gp[3]);
    }
    __syncwarp(gmask);
    {
      // 4-column units of the [K][D4] block, kBatch P loads in flight per lane
      constexpr int kBatch = 4;
      const int nv = K * D4 / 4;
      for (int v0 = sub; v0 < nv; v0 += W * kBatch) {
        float4 pv[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
          const int v = v0 + u * W;
          pv[u] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (v < nv) {
            const int k = (4 * v) / D4, d0 = 4 * v - k * D4;
            const float *Pr = P + (row0 + k) * D;
            if constexpr (D == D4) {
              pv[u] = __ldg(reinterpret_cast<const float4 *>(Pr + d0));
            } else {
              pv[u].x = d0 < D ? __ldg(Pr + d0) : 0.f;
              pv[u].y = d0 + 1 < D ? __ldg(Pr + d0 + 1) : 0.f;
              pv[u].z = d0 + 2 < D ? __ldg(Pr + d0 + 2) : 0.f;
              pv[u].w = d0 + 3 < D ? __ldg(Pr + d0 + 3) : 0.f;
            }
          }
        }
#pragma unroll
        for (int u = 0; u < kBatch; u++) {
          const int v = v0 + u * W;
          if (v < nv) {
            const int k = (4 * v) / D4, d0 = 4 * v - k * D4;
            const float4 g4 = *reinterpret_cast<const float4 *>(gpg + 4 * k);
            const float gp[4] = {g4.x, g4.y, g4.z, g4.w};
            const float p[4] = {pv[u].x, pv[u].y, pv[u].z, pv[u].w};
            float s[4];
#pragma unroll
            for (int j = 0; j < 4; j++)
              s[j] = d0 + j < D ? dedp_elem(gp, Ts, D4, M, d0 + j, p[j]) : 0.f;
            *reinterpret_cast<float4 *>(Sg + 4 * v) = make_float4(s[0], s[1], s[2], s[3]);
          }
        }
      }
    }
    __syncwarp(gmask);
    // the lane's next pair's geometry is loaded while the current one runs
    float4 nga = make_float4(0.f, 0.f, 0.f, 0.f), ngb = nga;
    if (sub < np) {
      nga = __ldg(pg_row + 2 * (pos + sub));
      ngb = __ldg(pg_row + 2 * (pos + sub) + 1);
    }
    for (int c0 = 0; c0 < np; c0 += W) {
      const int c = c0 + sub;
      const float4 cga = nga, cgb = ngb;
      if (c + W < np) {
        nga = __ldg(pg_row + 2 * (pos + c + W));
        ngb = __ldg(pg_row + 2 * (pos + c + W) + 1);
      }
      if (c < np) {
        int t;
        const PairGeo g = decode_pair_geo<RK>(cga, cgb, t);
        float2 V2[P2], W2[P2];
#pragma unroll
        for (int p = 0; p < P2; p++) {
          V2[p] = make_float2(0.f, 0.f);
          W2[p] = make_float2(0.f, 0.f);
        }
        const bool on = RK != kRadTable || (g.ti > 0 && g.ti < kp.tab_n - 2);
#pragma unroll
        for (int k0 = 0; k0 < (KC > 0 ? KC : K); k0 += 4) {
          if (!on) break;
          Radial4<RK> R;
          R.k0 = k0;
          if (RK != kRadTable) {
            const float4 pa = *reinterpret_cast<const float4 *>(rp + k0);
            const float4 pb = *reinterpret_cast<const float4 *>(rp + K + k0);
            const float4 pc = *reinterpret_cast<const float4 *>(rp + 2 * K + k0);
            const float4 pd = RK == kRadGauss ? *reinterpret_cast<const float4 *>(rp + 3 * K + k0)
                                              : make_float4(0.f, 0.f, 0.f, 0.f);
            const float va[4] = {pa.x, pa.y, pa.z, pa.w}, vb[4] = {pb.x, pb.y, pb.z, pb.w},
                        vc[4] = {pc.x, pc.y, pc.z, pc.w}, vd[4] = {pd.x, pd.y, pd.z, pd.w};
#pragma unroll
            for (int q = 0; q < 4; q++) {
              if (RK == kRadGauss) {
                R.b[q] = va[q]; R.blo[q] = vb[q]; R.gc[q] = vc[q]; R.gl[q] = vd[q];
              }
              if (RK == kRadGeneric) { R.a[q] = va[q]; R.b[q] = vb[q]; R.c[q] = vc[q]; }
            }
          }
          float H[4], dH[4];
          radial4<RK, true>(kp, R, g, H, dH);
#pragma unroll
          for (int q = 0; q < 4; q++) {
            const float2 h2 = make_float2(H[q], H[q]);
            const float2 d2 = make_float2(dH[q], dH[q]);
            const float4 *Sk = reinterpret_cast<const float4 *>(Sg + (k0 + q) * D4);
#pragma unroll
            for (int v = 0; v < D4 / 4; v++) {
              const float4 s = Sk[v];
              const float2 lo = make_float2(s.x, s.y), hi = make_float2(s.z, s.w);
              V2[2 * v] = __ffma2_rn(lo, h2, V2[2 * v]);
              W2[2 * v] = __ffma2_rn(lo, d2, W2[2 * v]);
              V2[2 * v + 1] = __ffma2_rn(hi, h2, V2[2 * v + 1]);
              W2[2 * v + 1] = __ffma2_rn(hi, d2, W2[2 * v + 1]);
            }
          }
        }
        float M[D4];
        moments<D>(g.ux, g.uy, g.uz, M);
#pragma unroll
        for (int d = D; d < D4; d++) M[d] = 0.f;
        float2 fa = make_float2(0.f, 0.f), fb = make_float2(0.f, 0.f);
#pragma unroll
        for (int p = 0; p < P2; p += 2) {
          fa = __ffma2_rn(make_float2(M[2 * p], M[2 * p + 1]), W2[p], fa);
          if (p + 1 < P2)
            fb = __ffma2_rn(make_float2(M[2 * p + 2], M[2 * p + 3]), W2[p + 1], fb);
        }
        const float f1 = (fa.x + fb.x) + (fa.y + fb.y);
        float V[D4];
#pragma unroll
        for (int p = 0; p < P2; p++) { V[2 * p] = V2[p].x; V[2 * p + 1] = V2[p].y; }
        float gq[3], nvm;
        poly_grad<D>(V, g.ux, g.uy, g.uz, gq, nvm);
        const float rinv = g.rinv;
        const float fx = (f1 * g.ux + (gq[0] - g.ux * nvm) * rinv) * scale;
        const float fy = (f1 * g.uy + (gq[1] - g.uy * nvm) * rinv) * scale;
        const float fz = (f1 * g.uz + (gq[2] - g.uz * nvm) * rinv) * scale;
        pdf_row[t] = make_float4(fx, fy, fz, 0.f);
        // per-pair virial in FP32 (df itself is FP32), summed in FP32 over
        // the lane's few pairs of the atom, then in FP64 over lanes and atoms
        const float rx = g.ux * g.r, ry = g.uy * g.r, rz = g.uz * g.r;
        w6[0] -= rx * fx;
        w6[1] -= ry * fy;
        w6[2] -= rz * fz;
        w6[3] -= rx * fy;
        w6[4] -= rx * fz;
        w6[5] -= ry * fz;
      }
    }
    pos += np;
  }
  double w6d[6];
#pragma unroll
  for (int c = 0; c < 6; c++) {
    w6d[c] = (double)w6[c];
#pragma unroll
    for (int o = W >> 1; o > 0; o >>= 1) w6d[c] += __shfl_xor_sync(gmask, w6d[c], o, W);
  }
  if (sub == 0) {
#pragma unroll
    for (int c = 0; c < 6; c++) wv[(size_t)a * 6 + c] = w6d[c];
  }
}

// Atom groups per block: as many as fit 128 threads and 48 KB of shared
// memory (the dynamic parameters and S blocks).
template <int D>
inline int force_pl_groups(int W, int K, int rk) {
  const size_t per = sizeof(float) * (size_t)PlLayout<D>::group(K);
  const size_t base = sizeof(float) * (size_t)PlLayout<D>::params(K, rk);
  int g = kPairThreads / W;
  while (g > 1 && base + g * per > 48 * 1024) g--;
  return g;
}

template <int W, int RK, bool MULTI>
void launch_force_pl_w(const ForceArgs &a, cudaStream_t st) {
#define TMD_FORCE_ARGS a.kp, a.box, a.n, a.cap, a.scale, a.x, a.elem, a.nbr, a.boff, a.P, a.G, a.dEdG, a.pdf, a.wv, a.cbox, a.acell, a.pgeo, a.pcnt
#define TMD_PL_CASE(DV)                                                                     \
  case DV: {                                                                                \
    const int g = force_pl_groups<DV>(W, a.kp.K, RK);                         \
    const int T = g * W;                                                                    \
    const long threads = (long)a.n * W;                                                     \
    const int grid = (int)std::max(1L, (threads + T - 1) / T);                              \
    k_force_pl<W, DV, RK, MULTI><<<grid, T, PlLayout<DV>::bytes(a.kp.K, RK, g), st>>>(      \
        TMD_FORCE_ARGS);                                                                    \
    break;                                                                                  \
  }
  switch (a.kp.D) {
    TMD_PL_CASE(1)
    TMD_PL_CASE(4)
    TMD_PL_CASE(10)
    default: {
      const int g = force_pl_groups<20>(W, a.kp.K, RK);
      const int T = g * W;
      const long threads = (long)a.n * W;
      const int grid = (int)std::max(1L, (threads + T - 1) / T);
      const size_t sm = PlLayout<20>::bytes(a.kp.K, RK, g);
      if (a.kp.K == 16)
        k_force_pl<W, 20, RK, MULTI, 16><<<grid, T, sm, st>>>(TMD_FORCE_ARGS);
      else if (a.kp.K == 32)
        k_force_pl<W, 20, RK, MULTI, 32><<<grid, T, sm, st>>>(TMD_FORCE_ARGS);
      else
        k_force_pl<W, 20, RK, MULTI><<<grid, T, sm, st>>>(TMD_FORCE_ARGS);
      break;
    }
  }
#undef TMD_PL_CASE
#undef TMD_FORCE_ARGS
}

template <int RK, bool MULTI>
void launch_force_pl(const ForceArgs &a, cudaStream_t st) {
  switch (a.variant) {
    case kForcePairLane8: launch_force_pl_w<8, RK, MULTI>(a, st); break;
    case kForcePairLane32: launch_force_pl_w<32, RK, MULTI>(a, st); break;
    default: launch_force_pl_w<16, RK, MULTI>(a, st); break;
  }
}

}  // namespace tmd
