// mlp.cu -- per-element atomic MLP E_i = NN_e(G_i) and dE/dG, FP32 plain form.
//
// Semantics (src/ML-TENSORMD/gpu/cuda/nnp.cu:9-57,149-281, nnp.cpp:246-365):
//   hidden layer l:  z = x W_l + b_l,  y = act(z) (+ x if use_resnet_dt,
//                    l > 0 and the layer keeps its width)
//   output layer:    E = x W_L (+ b_L if apply_output_bias)
//   backward:        g_{L-1} = W_L (sum over outputs), g_{l-1} = (g_l * act'(z_l))
//                    W_l^T (+ g_l on residual layers); dE/dG = g_{-1}
// Activations: 0 ReLU, 1 softplus, 2 tanh, 3 squareplus.
//
// One CTA (256 threads) owns TR atoms of one element.  The G rows, every
// hidden activation and act'(z) stay in shared memory (k-major, stride
// TR + 4), so forward and backward run in one launch; weights stream through a
// 32 x 64 shared-memory chunk.  Each thread computes an (TR/16) x 4 register
// tile per 64-column pass.
#include <float.h>

#include "tmd_kernels.h"

namespace tmd {

namespace {

constexpr int kThreads = 256;
constexpr int KC = 32;   // reduction chunk
constexpr int CB = 64;   // output column block
constexpr int WCP = 68;  // padded chunk row (floats)

__device__ inline float act_fwd(int actfn, float z, float &d) {
  switch (actfn) {
    case 0:
      d = z > 0.f ? 1.f : 0.f;
      return z > 0.f ? z : 0.f;
    case 1: {
      float ex = expf(z);
      const float thr = -13.942385152878742f;  // log(FLT_EPSILON) + 2
      d = 1.f / (1.f + 1.f / ex);
      return z < -thr ? log1pf(ex) : z;
    }
    case 2: {
      float y = tanhf(z);
      d = 1.f - y * y;
      return y;
    }
    default: {
      // squareplus 0.5 (z + sqrt(z^2 + 4)); for z < 0 the same value is
      // 2 / (sqrt(z^2 + 4) - z), which avoids the cancellation that costs
      // FP32 most of its digits when z << 0
      float q = sqrtf(z * z + 4.f);
      float y = z >= 0.f ? 0.5f * (z + q) : 2.f / (q - z);
      d = y / q;
      return y;
    }
  }
}

// out(r, c) = sum_k inT[k][r] * W(k, c); W(k, c) = trans ? Wg[c*Kd + k]
// : Wg[k*N + c].  epi(r, c, value) for c < N.
template <int TR, class Epi>
__device__ inline void tile_gemm(const float *inT, int ldt, int Kd,
                                 const float *__restrict__ Wg, int N, bool trans,
                                 float *Wc, Epi epi) {
  constexpr int RT = TR / 16;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  for (int c0 = 0; c0 < N; c0 += CB) {
    float acc[RT][4];
#pragma unroll
    for (int i = 0; i < RT; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    for (int kc = 0; kc < Kd; kc += KC) {
      __syncthreads();
      if (!trans) {
        for (int idx = tid; idx < KC * CB; idx += kThreads) {
          int k = idx / CB, c = idx % CB;
          int gk = kc + k, gc = c0 + c;
          Wc[k * WCP + c] = (gk < Kd && gc < N) ? __ldg(Wg + (size_t)gk * N + gc) : 0.f;
        }
      } else {
        for (int idx = tid; idx < KC * CB; idx += kThreads) {
          int c = idx / KC, k = idx % KC;
          int gk = kc + k, gc = c0 + c;
          Wc[k * WCP + c] = (gk < Kd && gc < N) ? __ldg(Wg + (size_t)gc * Kd + gk) : 0.f;
        }
      }
      __syncthreads();
      const int kmax = min(KC, Kd - kc);
      for (int k = 0; k < kmax; k++) {
        float4 w = *reinterpret_cast<const float4 *>(Wc + k * WCP + 4 * tx);
        const float *xr = inT + (size_t)(kc + k) * ldt + ty * RT;
        float xv[RT];
        if (RT == 4) {
          float4 t = *reinterpret_cast<const float4 *>(xr);
          xv[0] = t.x; xv[1] = t.y; xv[2 % RT] = t.z; xv[3 % RT] = t.w;
        } else {
          float2 t = *reinterpret_cast<const float2 *>(xr);
          xv[0] = t.x; xv[1 % RT] = t.y;
        }
#pragma unroll
        for (int i = 0; i < RT; i++) {
          acc[i][0] = fmaf(xv[i], w.x, acc[i][0]);
          acc[i][1] = fmaf(xv[i], w.y, acc[i][1]);
          acc[i][2] = fmaf(xv[i], w.z, acc[i][2]);
          acc[i][3] = fmaf(xv[i], w.w, acc[i][3]);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < RT; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) {
        int c = c0 + 4 * tx + j;
        if (c < N) epi(ty * RT + i, c, acc[i][j]);
      }
  }
  __syncthreads();
}

template <int TR>
__global__ void __launch_bounds__(kThreads)
k_mlp_fp32(MlpArgs a) {
  extern __shared__ float sm[];
  constexpr int LDT = TR + 4;
  const int tile = blockIdx.x;
  const int elt = a.tiles[3 * tile], start = a.tiles[3 * tile + 1],
            count = a.tiles[3 * tile + 2];
  const MlpLayer *Ls = a.layers + (size_t)elt * a.nl;
  const int L = a.nl;
  const int maxh = a.maxh;
  float *act0 = sm;                                 // [max(nin, maxh)][LDT]
  float *act1 = act0 + (size_t)max(a.nin, maxh) * LDT;  // [maxh][LDT]
  float *dzb = act1 + (size_t)maxh * LDT;           // sum_l N_l x LDT
  int dz_off[kMaxLayers];
  {
    int o = 0;
    for (int l = 0; l < L - 1; l++) { dz_off[l] = o; o += Ls[l].N * LDT; }
    dz_off[L - 1] = o;
  }
  float *Wc = dzb + dz_off[L - 1];                  // [KC][WCP]
  __shared__ int rows[TR];
  const int tid = threadIdx.x;
  if (tid < TR) rows[tid] = tid < count ? a.perm[start + tid] : -1;
  __syncthreads();
  // G tile, transposed
  const int nin = a.nin;
  for (int idx = tid; idx < TR * nin; idx += kThreads) {
    int r = idx / nin, k = idx % nin;
    int at = rows[r];
    act0[(size_t)k * LDT + r] = at >= 0 ? __ldg(a.G + (size_t)at * nin + k) : 0.f;
  }
  __syncthreads();
  // forward hidden layers
  float *in = act0, *out = act1;
  for (int l = 0; l < L - 1; l++) {
    const MlpLayer ly = Ls[l];
    float *dz = dzb + dz_off[l];
    const bool res = a.resnet && l > 0 && ly.K == ly.N;
    const float *bias = ly.b;
    const int actfn = a.actfn;
    float *o = out, *ip = in;
    tile_gemm<TR>(in, LDT, ly.K, ly.W, ly.N, false, Wc,
                  [&](int r, int c, float v) {
                    float z = v + (bias ? __ldg(bias + c) : 0.f);
                    float d;
                    float y = act_fwd(actfn, z, d);
                    if (res) y += ip[(size_t)c * LDT + r];
                    o[(size_t)c * LDT + r] = y;
                    dz[(size_t)c * LDT + r] = d;
                  });
    float *t = in; in = out; out = t;
  }
  // output layer in FP64 (one output per atom; the reference sums outputs)
  {
    const MlpLayer ly = Ls[L - 1];
    const int per = kThreads / TR;  // threads per row
    const int r = tid / per, part = tid % per;
    double s = 0.0;
    for (int k = part; k < ly.K; k += per) {
      double wsum = 0.0;
      for (int o2 = 0; o2 < ly.N; o2++) wsum += __ldg(ly.Wd + (size_t)k * ly.N + o2);
      s = fma((double)in[(size_t)k * LDT + r], wsum, s);
    }
    for (int o2 = per >> 1; o2 > 0; o2 >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o2);
    if (part == 0 && rows[r] >= 0) {
      double e = s;
      if (ly.bd)
        for (int o2 = 0; o2 < ly.N; o2++) e += __ldg(ly.bd + o2);
      a.E[rows[r]] = e;
    }
  }
  __syncthreads();
  // backward: g of the last hidden output = row sums of W_L, times act'
  {
    const MlpLayer ly = Ls[L - 1];
    float *dz = dzb + dz_off[L - 2 >= 0 ? L - 2 : 0];
    float *g = out;  // free buffer: holds g_{L-2}
    for (int idx = tid; idx < ly.K * TR; idx += kThreads) {
      int k = idx / TR, r = idx % TR;
      float wsum = 0.f;
      for (int o2 = 0; o2 < ly.N; o2++) wsum += __ldg(ly.W + (size_t)k * ly.N + o2);
      g[(size_t)k * LDT + r] = wsum;
      if (L >= 2) dz[(size_t)k * LDT + r] *= wsum;  // gz = g * act'
    }
    __syncthreads();
    // now `out` holds g_{L-2}, dz_{L-2} holds gz_{L-2}
    float *gcur = out, *gnext = in;
    for (int l = L - 2; l >= 0; l--) {
      const MlpLayer lw = Ls[l];
      float *gz = dzb + dz_off[l];
      if (l == 0) {
        const int *rw = rows;
        float *dE = a.dEdG;
        tile_gemm<TR>(gz, LDT, lw.N, lw.W, lw.K, true, Wc,
                      [&](int r, int c, float v) {
                        int at = rw[r];
                        if (at >= 0) dE[(size_t)at * nin + c] = v;
                      });
      } else {
        const bool res = a.resnet && lw.K == lw.N;
        float *dzn = dzb + dz_off[l - 1];
        float *gc = gcur, *gn = gnext;
        tile_gemm<TR>(gz, LDT, lw.N, lw.W, lw.K, true, Wc,
                      [&](int r, int c, float v) {
                        float gv = v + (res ? gc[(size_t)c * LDT + r] : 0.f);
                        gn[(size_t)c * LDT + r] = gv;
                        dzn[(size_t)c * LDT + r] *= gv;
                      });
        float *t = gcur; gcur = gnext; gnext = t;
      }
    }
  }
}

}  // namespace

size_t mlp_fp32_smem(int nl, const int *sizes, int tr) {
  // sizes[0..nl]: n_in, layer widths
  int maxh = 1;
  for (int l = 1; l < nl; l++) maxh = maxh > sizes[l] ? maxh : sizes[l];
  int w0 = sizes[0] > maxh ? sizes[0] : maxh;
  size_t ldt = tr + 4;
  size_t f = ((size_t)w0 + maxh) * ldt;
  for (int l = 0; l < nl - 1; l++) f += (size_t)sizes[l + 1] * ldt;
  f += (size_t)KC * WCP;
  return f * sizeof(float);
}

void launch_mlp_fp32(const MlpArgs &a, cudaStream_t st, long &launches) {
  if (a.ntiles <= 0) return;
  launches += 1;
  if (a.tr == 64) {
    k_mlp_fp32<64><<<a.ntiles, kThreads, a.smem, st>>>(a);
  } else {
    k_mlp_fp32<32><<<a.ntiles, kThreads, a.smem, st>>>(a);
  }
}

void mlp_fp32_prepare(int tr, size_t smem) {
  if (tr == 64)
    cudaFuncSetAttribute(k_mlp_fp32<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  else
    cudaFuncSetAttribute(k_mlp_fp32<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace tmd
