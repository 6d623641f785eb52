// tdnp.cu -- the temperature-dependent model (tdnp = 1 potentials) on the
// device: the per-element nets H, U and S of tdnp.cpp in place of the MLP.
//
// Per atom (TDNP::forward / backward, tdnp.cpp:167-226, nnp.cu:295-318):
//   y = H(G) with y[ydim-1] = T (the electron temperature, eV)
//   u = U(y), s = S(y) (s *= T in the Sommerfeld form); E_atom = u,
//   A_atom = u - T s
//   dE/dG = H^T-backward of (dU/dy - c dS/dy), c = T (T^2 Sommerfeld), the
//   temperature column's gradient set to zero
// so the forces are those of the free energy A.  One warp per atom: lanes
// over a layer's outputs for the forward products (W read row by row,
// coalesced) and over its inputs for the backward ones (W^T); activations,
// act' and gradients of the warp's atom in shared memory; FP32 arithmetic,
// the outputs of U and S (sums over their last layer) in FP64, as the MLP's
// output layer.
#include "tc_util.cuh"
#include "tmd_kernels.h"

namespace tmd {

namespace {

constexpr int kTdnpWarps = 4;

// One layer of the warp's net: out = act(in W + b) (hidden) or in W + b
// (last, linear); dz = act'.  Lanes over the N outputs.
__device__ inline void tdnp_fwd_layer(const TdnpLayer &L, bool hidden, bool res, int actfn,
                                      const float *in, float *out, float *dz, int lane) {
  for (int n = lane; n < L.N; n += 32) {
    float z = L.b ? __ldg(L.b + n) : 0.f;
    for (int k = 0; k < L.K; k++) z = fmaf(in[k], __ldg(L.W + (size_t)k * L.N + n), z);
    if (hidden) {
      float d;
      float y = tc::act_fwd(actfn, z, d);
      if (res) y += in[n];
      out[n] = y;
      dz[n] = d;
    } else {
      out[n] = z;
    }
  }
  __syncwarp();
}

// gin[k] = sum_n g[n] (dz[n] if dz) W[k][n] (+ gres[k]); lanes over the K
// inputs, W^T rows contiguous.
__device__ inline void tdnp_bwd_layer(const TdnpLayer &L, const float *g, const float *dz,
                                      const float *gres, float *gin, int lane) {
  for (int k = lane; k < L.K; k += 32) {
    float s = 0.f;
    for (int n = 0; n < L.N; n++) {
      const float gz = dz ? g[n] * dz[n] : g[n];
      s = fmaf(gz, __ldg(L.WT + (size_t)n * L.K + k), s);
    }
    if (gres) s += gres[k];
    gin[k] = s;
  }
  __syncwarp();
}

// Forward of a scalar net (U or S) from y: hidden layers, then the summed
// last layer in FP64.  act holds (nl) activation rows, dz (nl - 1) rows.
__device__ inline double tdnp_scalar_fwd(const TdnpArgs &a, int net, int e, const float *y,
                                         float *act, float *dz, int lane) {
  const int nl = a.nl[net];
  const TdnpLayer *Ls = a.layers + ((size_t)net * a.nelt + e) * kMaxLayers;
  const float *in = y;
  for (int l = 0; l < nl - 1; l++) {
    float *out = act + (size_t)(l + 1) * a.maxw;
    const bool res = a.resnet[net] && l > 0 && Ls[l].K == Ls[l].N;
    tdnp_fwd_layer(Ls[l], true, res, a.actfn[net], in, out, dz + (size_t)l * a.maxw, lane);
    in = out;
  }
  const TdnpLayer &Lo = Ls[nl - 1];
  double s = 0.0;
  for (int k = lane; k < Lo.K; k += 32) s = fma((double)in[k], __ldg(Lo.Wd + k), s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s + Lo.bd;
}

// Gradient of a scalar net's output with respect to its input y (width
// ydim) into g, from the activations of tdnp_scalar_fwd.
__device__ inline void tdnp_scalar_bwd(const TdnpArgs &a, int net, int e, const float *dz,
                                       float *ga, float *gb, float *g, int lane) {
  const int nl = a.nl[net];
  const TdnpLayer *Ls = a.layers + ((size_t)net * a.nelt + e) * kMaxLayers;
  const TdnpLayer &Lo = Ls[nl - 1];
  float *gcur = nl >= 2 ? ga : g;
  for (int k = lane; k < Lo.K; k += 32) gcur[k] = __ldg(Lo.Wf + k);
  __syncwarp();
  for (int l = nl - 2; l >= 0; l--) {
    const bool res = a.resnet[net] && l > 0 && Ls[l].K == Ls[l].N;
    float *gnext = l == 0 ? g : (gcur == ga ? gb : ga);
    tdnp_bwd_layer(Ls[l], gcur, dz + (size_t)l * a.maxw, res ? gcur : nullptr, gnext, lane);
    gcur = gnext;
  }
}

__global__ void __launch_bounds__(32 * kTdnpWarps)
k_mlp_tdnp(TdnpArgs a) {
  extern __shared__ float4 tdnp_sm4[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  float *ws = reinterpret_cast<float *>(tdnp_sm4) + (size_t)wib * a.warp_floats;
  // per warp: H activations (nlH + 1 rows) and act' (nlH rows), U and S
  // activations (nl rows) and act' (nl - 1 rows), three gradient rows
  const int W = a.maxw, nlH = a.nl[0];
  float *actH = ws, *dzH = actH + (size_t)(nlH + 1) * W;
  float *actU = dzH + (size_t)nlH * W, *dzU = actU + (size_t)a.nl[1] * W;
  float *actS = dzU + (size_t)a.nl[1] * W, *dzS = actS + (size_t)a.nl[2] * W;
  float *g0 = dzS + (size_t)a.nl[2] * W, *g1 = g0 + W, *g2 = g1 + W, *gu = g2 + W;
  const int nwarp = gridDim.x * kTdnpWarps;
  for (int at = blockIdx.x * kTdnpWarps + wib; at < a.n; at += nwarp) {
    const int e = a.elem[at];
    for (int k = lane; k < a.nin; k += 32) actH[k] = __ldg(a.G + (size_t)at * a.nin + k);
    __syncwarp();
    // H: G -> y
    const TdnpLayer *LH = a.layers + (size_t)e * kMaxLayers;
    for (int l = 0; l < nlH; l++) {
      const bool hidden = l < nlH - 1;
      const bool res = a.resnet[0] && l > 0 && LH[l].K == LH[l].N;
      tdnp_fwd_layer(LH[l], hidden, res, a.actfn[0], actH + (size_t)l * W,
                     actH + (size_t)(l + 1) * W, dzH + (size_t)l * W, lane);
    }
    float *y = actH + (size_t)nlH * W;
    if (lane == 0) y[a.ydim - 1] = a.T;
    __syncwarp();
    const double u = tdnp_scalar_fwd(a, 1, e, y, actU, dzU, lane);
    double s = tdnp_scalar_fwd(a, 2, e, y, actS, dzS, lane);
    if (a.sommerfeld) s *= (double)a.T;
    // gradient of A = u - T s with respect to y, the temperature held fixed
    tdnp_scalar_bwd(a, 1, e, dzU, g0, g1, gu, lane);   // dU/dy into gu
    tdnp_scalar_bwd(a, 2, e, dzS, g0, g1, g2, lane);   // dS/dy into g2
    for (int k = lane; k < a.ydim; k += 32) gu[k] = k == a.ydim - 1 ? 0.f : gu[k] - a.c * g2[k];
    __syncwarp();
    // H backward: the last layer is linear, then the hidden ones
    float *gcur = gu;
    for (int l = nlH - 1; l >= 0; l--) {
      const bool res = a.resnet[0] && l > 0 && LH[l].K == LH[l].N;
      float *gnext = gcur == g0 ? g1 : g0;
      const float *dzl = l == nlH - 1 ? nullptr : dzH + (size_t)l * W;
      if (l == 0) {
        // dE/dG straight to global memory
        for (int k = lane; k < LH[0].K; k += 32) {
          float sacc = 0.f;
          for (int n = 0; n < LH[0].N; n++) {
            const float gz = dzl ? gcur[n] * dzl[n] : gcur[n];
            sacc = fmaf(gz, __ldg(LH[0].WT + (size_t)n * LH[0].K + k), sacc);
          }
          a.dEdG[(size_t)at * a.nin + k] = sacc;
        }
      } else {
        tdnp_bwd_layer(LH[l], gcur, dzl, res ? gcur : nullptr, gnext, lane);
        gcur = gnext;
      }
    }
    if (lane == 0) {
      a.E[at] = u;
      a.Sa[at] = s;
      a.Aa[at] = u - (double)a.T * s;
    }
    __syncwarp();
  }
}

}  // namespace

size_t tdnp_warp_floats(const int nl[3], int maxw) {
  // H: nl+1 activation rows + nl act' rows; U, S: nl activation rows +
  // nl act' rows (one spare); four gradient rows
  return (size_t)maxw * ((2 * nl[0] + 1) + 2 * nl[1] + 2 * nl[2] + 4);
}

int launch_mlp_tdnp(const TdnpArgs &a, cudaStream_t st, long &launches) {
  if (a.n <= 0) return 0;
  const size_t smem = a.warp_floats * sizeof(float) * kTdnpWarps;
  if (smem > 227 * 1024) return -1;
  static size_t prepared = 0;
  if (smem > 48 * 1024 && smem > prepared) {
    cudaFuncSetAttribute(k_mlp_tdnp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    prepared = smem;
  }
  int grid = (a.n + kTdnpWarps - 1) / kTdnpWarps;
  if (grid > 148 * 16) grid = 148 * 16;
  k_mlp_tdnp<<<grid, 32 * kTdnpWarps, smem, st>>>(a);
  launches += 1;
  return 0;
}

}  // namespace tmd
