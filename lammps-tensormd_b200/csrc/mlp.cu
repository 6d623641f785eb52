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

#include <vector>

#include "tc_util.cuh"
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
      // tanh' = sech^2 z = 4 e / (1 + e)^2 with e = exp(-2|z|): the same
      // value as 1 - tanh^2, without its cancellation (at |z| = 3 one ulp
      // of tanh is 1e-5 of 1 - tanh^2, an error that does not cancel in the
      // virial)
      const float e = expf(-2.f * fabsf(z));
      const float u = 1.f + e;
      d = 4.f * e / (u * u);
      return tanhf(z);
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

// ---------------------------------------------------------------------------
// Resident-weight form.  The hidden layers' W of the current element stay in
// shared memory (row-major, row stride ldw = 32*ceil(N/32) + 4 floats, zero
// padding) for the whole life of a persistent CTA, which walks the tiles
// (sorted by element) with a grid stride and reloads the weights only when the
// element changes.  The forward GEMM reads W rows as float4 over 4 output
// columns (as tile_gemm); the backward GEMM contracts over the output width,
// so a thread owns outputs k = k0 + tx + 16 j and reads the rows W[k][c..c+3]
// as float4 (row stride = 4 mod 32 words: the 8 threads of a phase hit
// distinct banks).  Same FP32 arithmetic in the same order as k_mlp_fp32.
// ---------------------------------------------------------------------------
// Tiles of 128 atoms on 16 warps, or of 64 atoms on 8 warps when an input
// width as large as 4 elements x 16 filters x 4 moments needs the smaller
// activation buffers: a 4 x 4 register tile per thread either way.

struct ResLayout {
  int woff[kMaxLayers], ldw[kMaxLayers], boff[kMaxLayers], dzoff[kMaxLayers];
  int wsf, wsd, act0, act1, total;  // floats
};

__host__ __device__ inline int round_up(int v, int m) { return (v + m - 1) / m * m; }

// sizes[0..nl]: n_in, layer widths.
__host__ __device__ inline ResLayout res_layout(int nl, const int *sizes, int tr) {
  ResLayout r{};
  const int ldt = tr + 4;
  int maxh = 1;
  for (int l = 1; l < nl; l++) maxh = maxh > sizes[l] ? maxh : sizes[l];
  int o = 0;
  for (int l = 0; l < nl - 1; l++) {
    r.ldw[l] = round_up(sizes[l + 1], 32) + 4;
    r.woff[l] = o;
    o += sizes[l] * r.ldw[l];
  }
  for (int l = 0; l < nl - 1; l++) { r.boff[l] = o; o += round_up(sizes[l + 1], 4); }
  r.wsf = o; o += round_up(sizes[nl - 1], 4);
  o = round_up(o, 2);
  r.wsd = o; o += 2 * round_up(sizes[nl - 1], 2);  // doubles
  const int w0 = sizes[0] > maxh ? sizes[0] : maxh;
  r.act0 = o; o += round_up(w0, 4) * ldt;
  r.act1 = o; o += round_up(maxh, 4) * ldt;
  for (int l = 0; l < nl - 1; l++) { r.dzoff[l] = o; o += round_up(sizes[l + 1], 4) * ldt; }
  r.total = round_up(o, 4);
  return r;
}

// RT consecutive floats of one k-row of a transposed tile (16-byte aligned
// for RT >= 4).
template <int RT>
__device__ inline void load_rows(const float *src, float v[RT]) {
  if constexpr (RT % 4 == 0) {
#pragma unroll
    for (int q = 0; q < RT / 4; q++) {
      const float4 t = reinterpret_cast<const float4 *>(src)[q];
      v[4 * q] = t.x; v[4 * q + 1] = t.y; v[4 * q + 2] = t.z; v[4 * q + 3] = t.w;
    }
  } else {
    const float2 t = *reinterpret_cast<const float2 *>(src);
    v[0] = t.x; v[1 % RT] = t.y;
  }
}

// Forward: out(r, c) = sum_k inT[k][r] W[k][c] for c < N, r < TR.
template <int TR, int NT, class Epi>
__device__ inline void res_gemm_fwd(const float *inT, int Kd, const float *W, int ldw, int N,
                                    Epi epi) {
  constexpr int LDT = TR + 4, RT = TR / (NT / 16);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int N4 = round_up(N, 4);
  for (int c0 = 0; c0 < N4; c0 += 64) {
    const int cc = c0 + 4 * tx;
    if (cc >= N4) continue;
    float acc[RT][4];
#pragma unroll
    for (int i = 0; i < RT; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    const float *wp = W + cc;
    const float *xp = inT + ty * RT;
#pragma unroll 4
    for (int k = 0; k < Kd; k++) {
      const float4 w = *reinterpret_cast<const float4 *>(wp + k * ldw);
      float xv[RT];
      load_rows<RT>(xp + k * LDT, xv);
#pragma unroll
      for (int i = 0; i < RT; i++) {
        acc[i][0] = fmaf(xv[i], w.x, acc[i][0]);
        acc[i][1] = fmaf(xv[i], w.y, acc[i][1]);
        acc[i][2] = fmaf(xv[i], w.z, acc[i][2]);
        acc[i][3] = fmaf(xv[i], w.w, acc[i][3]);
      }
    }
#pragma unroll
    for (int i = 0; i < RT; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (cc + j < N) epi(ty * RT + i, cc + j, acc[i][j]);
  }
}

// Backward: out(r, k) = sum_c gzT[c][r] W[k][c] for k < Kout, r < TR; gzT
// has round_up(Nc, 4) rows (padding rows finite), W zero beyond column Nc.
template <int TR, int NT, class Epi>
__device__ inline void res_gemm_bwd(const float *gzT, int Nc, const float *W, int ldw, int Kout,
                                    Epi epi) {
  constexpr int LDT = TR + 4, RT = TR / (NT / 16);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int Nc4 = round_up(Nc, 4);
  for (int k0 = 0; k0 < Kout; k0 += 64) {
    float acc[RT][4];
#pragma unroll
    for (int i = 0; i < RT; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    bool kv[4];
    const float *wr[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int k = k0 + tx + 16 * j;
      kv[j] = k < Kout;
      wr[j] = W + (size_t)(kv[j] ? k : 0) * ldw;
    }
    const float *gp = gzT + ty * RT;
#pragma unroll 2
    for (int c = 0; c < Nc4; c += 4) {
      float4 wj[4];
#pragma unroll
      for (int j = 0; j < 4; j++)
        wj[j] = *reinterpret_cast<const float4 *>(wr[j] + c);  // row 0 where !kv[j]: not stored
      float g[4][RT];
#pragma unroll
      for (int q = 0; q < 4; q++) load_rows<RT>(gp + (c + q) * LDT, g[q]);
#pragma unroll
      for (int i = 0; i < RT; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          acc[i][j] = fmaf(g[0][i], wj[j].x, acc[i][j]);
          acc[i][j] = fmaf(g[1][i], wj[j].y, acc[i][j]);
          acc[i][j] = fmaf(g[2][i], wj[j].z, acc[i][j]);
          acc[i][j] = fmaf(g[3][i], wj[j].w, acc[i][j]);
        }
    }
#pragma unroll
    for (int i = 0; i < RT; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (kv[j]) epi(ty * RT + i, k0 + tx + 16 * j, acc[i][j]);
  }
}

template <int TR, int NT>
__global__ void __launch_bounds__(NT, 1)
k_mlp_fp32r(MlpArgs a) {
  extern __shared__ float4 smr4[];
  float *sm = reinterpret_cast<float *>(smr4);
  constexpr int LDT = TR + 4;
  const int L = a.nl, nin = a.nin;
  int sizes[kMaxLayers + 1];
  sizes[0] = nin;
  const MlpLayer *L0 = a.layers;
  for (int l = 0; l < L; l++) sizes[l + 1] = L0[l].N;
  const ResLayout lay = res_layout(L, sizes, TR);
  float *act0 = sm + lay.act0, *act1 = sm + lay.act1;
  float *wsf = sm + lay.wsf;
  double *wsd = reinterpret_cast<double *>(sm + lay.wsd);
  __shared__ int rows[TR];
  const int tid = threadIdx.x;
  const int Klast = sizes[L - 1];
  // padding rows of the activation-gradient buffers are read by the backward
  // GEMM (times zero weights): keep them finite
  for (int l = 0; l < L - 1; l++) {
    const int N = sizes[l + 1], N4 = round_up(N, 4);
    for (int idx = tid; idx < (N4 - N) * LDT; idx += NT) sm[lay.dzoff[l] + N * LDT + idx] = 0.f;
  }
  int cur_elt = -1;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int elt = a.tiles[3 * tile], start = a.tiles[3 * tile + 1],
              count = a.tiles[3 * tile + 2];
    __syncthreads();  // the previous tile is done with every buffer
    if (elt != cur_elt) {
      cur_elt = elt;
      const MlpLayer *Ls = a.layers + (size_t)elt * L;
      for (int l = 0; l < L - 1; l++) {
        const int K = Ls[l].K, N = Ls[l].N, ldw = lay.ldw[l];
        float *Wd = sm + lay.woff[l];
        for (int idx = tid; idx < K * ldw; idx += NT) {
          const int k = idx / ldw, c = idx - k * ldw;
          Wd[idx] = c < N ? __ldg(Ls[l].W + (size_t)k * N + c) : 0.f;
        }
        float *bd = sm + lay.boff[l];
        for (int c = tid; c < N; c += NT) bd[c] = Ls[l].b ? __ldg(Ls[l].b + c) : 0.f;
      }
      const MlpLayer lo = Ls[L - 1];
      for (int k = tid; k < lo.K; k += NT) {
        double sd = 0.0;
        float sf = 0.f;
        for (int o2 = 0; o2 < lo.N; o2++) {
          sd += __ldg(lo.Wd + (size_t)k * lo.N + o2);
          sf += __ldg(lo.W + (size_t)k * lo.N + o2);
        }
        wsd[k] = sd;
        wsf[k] = sf;
      }
    }
    if (tid < TR) rows[tid] = tid < count ? a.perm[start + tid] : -1;
    __syncthreads();
    // G tile, transposed.  The whole CTA waits on these loads, so with rows
    // a multiple of 4 wide they go as float4, four per thread in flight, a
    // warp covering 32 rows of one column quad (conflict-free stores)
    if ((nin & 3) == 0) {
      const int nq = nin >> 2, total = TR * nq;
      for (int base = tid; base < total; base += 4 * NT) {
        float4 gv[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int idx = base + u * NT;
          gv[u] = make_float4(0.f, 0.f, 0.f, 0.f);
          if (idx < total) {
            const int q = idx / TR, r = idx - q * TR;
            const int at = rows[r];
            if (at >= 0) gv[u] = __ldg(reinterpret_cast<const float4 *>(a.G + (size_t)at * nin) + q);
          }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int idx = base + u * NT;
          if (idx < total) {
            const int q = idx / TR, r = idx - q * TR;
            float *dst = act0 + (size_t)(4 * q) * LDT + r;
            dst[0] = gv[u].x;
            dst[LDT] = gv[u].y;
            dst[2 * LDT] = gv[u].z;
            dst[3 * LDT] = gv[u].w;
          }
        }
      }
    } else {
      for (int idx = tid; idx < TR * nin; idx += NT) {
        const int r = idx / nin, k = idx - r * nin;
        const int at = rows[r];
        act0[(size_t)k * LDT + r] = at >= 0 ? __ldg(a.G + (size_t)at * nin + k) : 0.f;
      }
    }
    __syncthreads();
    float *in = act0, *out = act1;
    for (int l = 0; l < L - 1; l++) {
      const int K = sizes[l], N = sizes[l + 1];
      float *dz = sm + lay.dzoff[l];
      const float *bias = sm + lay.boff[l];
      const bool res = a.resnet && l > 0 && K == N;
      const int actfn = a.actfn;
      float *o = out;
      const float *ip = in;
      res_gemm_fwd<TR, NT>(in, K, sm + lay.woff[l], lay.ldw[l], N, [&](int r, int c, float v) {
        const float z = v + bias[c];
        float d;
        float y = act_fwd(actfn, z, d);
        if (res) y += ip[(size_t)c * LDT + r];
        o[(size_t)c * LDT + r] = y;
        dz[(size_t)c * LDT + r] = d;
      });
      __syncthreads();
      float *t = in; in = out; out = t;
    }
    // output layer in FP64
    {
      const MlpLayer lo = a.layers[(size_t)elt * L + L - 1];
      const int per = NT / TR;
      const int r = tid / per, part = tid % per;
      double s = 0.0;
      for (int k = part; k < Klast; k += per) s = fma((double)in[(size_t)k * LDT + r], wsd[k], s);
      for (int o2 = per >> 1; o2 > 0; o2 >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o2);
      if (part == 0 && rows[r] >= 0) {
        double e = s;
        if (lo.bd)
          for (int o2 = 0; o2 < lo.N; o2++) e += __ldg(lo.bd + o2);
        a.E[rows[r]] = e;
      }
    }
    // backward seed: g of the last hidden output = row sums of W_L, times act'
    {
      float *dz = sm + lay.dzoff[L - 2 >= 0 ? L - 2 : 0];
      float *g = out;
      for (int idx = tid; idx < Klast * TR; idx += NT) {
        const int k = idx / TR, r = idx - k * TR;
        g[(size_t)k * LDT + r] = wsf[k];
        if (L >= 2) dz[(size_t)k * LDT + r] *= wsf[k];
      }
    }
    __syncthreads();
    float *gcur = out, *gnext = in;
    for (int l = L - 2; l >= 0; l--) {
      const int K = sizes[l], N = sizes[l + 1];
      const float *gz = sm + lay.dzoff[l];
      const float *Wl = sm + lay.woff[l];
      if (l == 0) {
        const int *rw = rows;
        float *dE = a.dEdG;
        res_gemm_bwd<TR, NT>(gz, N, Wl, lay.ldw[l], K, [&](int r, int k, float v) {
          const int at = rw[r];
          if (at >= 0) dE[(size_t)at * nin + k] = v;
        });
      } else {
        const bool res = a.resnet && K == N;
        float *dzn = sm + lay.dzoff[l - 1];
        const float *gc = gcur;
        float *gn = gnext;
        res_gemm_bwd<TR, NT>(gz, N, Wl, lay.ldw[l], K, [&](int r, int k, float v) {
          const float gv = v + (res ? gc[(size_t)k * LDT + r] : 0.f);
          gn[(size_t)k * LDT + r] = gv;
          dzn[(size_t)k * LDT + r] *= gv;
        });
        __syncthreads();
        float *t = gcur; gcur = gnext; gnext = t;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Warp-tile form (k_mlp_fp32w) for MLPs with 64-wide hidden layers and no
// residual layers (the 64-64 nets of the benchmark, batch and serving
// configs).  In the resident form a thread's 4 x 4 register tile takes two
// 16-byte shared-memory loads per 16 FMAs, so the GEMMs wait on shared memory
// about as long as on the FMA pipe, and 16 warps meet at a block barrier
// after every layer.  Here each warp owns a tile of 16 atoms from start to
// end (no block barrier except when the element changes): lane (ty, tx) =
// (lane / 8, lane % 8) owns rows ty + 4 i (i < 4) and 8 columns of each
// 64-column GEMM, a 4 x 8 register tile fed by three 16-byte loads per k step
// for 32 FMAs.  Forward columns are 4 tx + j and 32 + 4 tx + j (j < 4: one
// 128-byte row segment per warp load); backward outputs k = k0 + tx + 8 j (W
// rows of the 8 tx lanes 4 banks apart).  The G rows of a tile are copied to
// the warp's area with cp.async (zero-filled past the last atom; the next
// tile's rows prefetched to L2 one tile ahead); every hidden output is formed
// in registers before it overwrites the GEMM's input in place, and the
// activation runs as a short loop over the lane's own four-column groups.
// Each output is summed over the reduction index in ascending order with the
// FMAs of the resident form (same dE/dG bits); the output layer in FP64,
// summed over a lane's four columns and across the 8 lanes of a row, the two
// column halves in order.
// ---------------------------------------------------------------------------
constexpr int kWtRI = 4;                 // rows per lane
constexpr int kWtRows = 4 * kWtRI;       // atoms per warp tile
constexpr int kWtThreads = 512;          // 16 warps per CTA
constexpr int kWtWidth = 64;             // hidden width this form supports

struct WtLayout {
  int woff[kMaxLayers], ldw[kMaxLayers], boff[kMaxLayers];
  int wsf, wsd, ef;  // FP32 / FP64 row sums of W_out; floats of the element block
  int ldg, ldh, wf;  // G and hidden row strides; floats per warp area
};

__host__ __device__ inline WtLayout wt_layout(int nl, const int *sizes) {
  WtLayout r{};
  int o = 0;
  for (int l = 0; l < nl - 1; l++) {
    r.ldw[l] = sizes[l + 1] + 4;
    r.woff[l] = o;
    o += sizes[l] * r.ldw[l];
  }
  for (int l = 0; l < nl - 1; l++) { r.boff[l] = o; o += round_up(sizes[l + 1], 4); }
  r.wsf = o; o += round_up(sizes[nl - 1], 4);
  r.wsd = o; o += 2 * round_up(sizes[nl - 1], 2);
  r.ef = round_up(o, 4);
  r.ldg = round_up(sizes[0], 4) + 4;
  r.ldh = kWtWidth + 4;
  // G staging and the hidden buffers (output / gradient, then act' of every
  // hidden layer but the last) share the warp area
  const int gfl = kWtRows * r.ldg, hfl = (nl - 1) * kWtRows * r.ldh;
  r.wf = round_up(gfl > hfl ? gfl : hfl, 4) + 2 * kWtRows;  // + FP64 row energies
  return r;
}

// out(r_i, c0 + col_j) = sum_k A[r_i][k] W[k][c0 + col_j], k ascending.
__device__ __forceinline__ void wt_gemm_fwd(const float *A, int lda, int K, const float *W,
                                            int ldw, int ty, int tx, float (&acc)[kWtRI][8]) {
  const float *ap = A + ty * lda;
  const float *wp = W + 4 * tx;
#pragma unroll 2
  for (int k = 0; k < K; k += 4) {
    float4 av[kWtRI], b0[4], b1[4];
#pragma unroll
    for (int i = 0; i < kWtRI; i++) av[i] = *reinterpret_cast<const float4 *>(ap + 4 * i * lda + k);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      b0[q] = *reinterpret_cast<const float4 *>(wp + (k + q) * ldw);
      b1[q] = *reinterpret_cast<const float4 *>(wp + (k + q) * ldw + 32);
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const float bq[8] = {b0[q].x, b0[q].y, b0[q].z, b0[q].w, b1[q].x, b1[q].y, b1[q].z, b1[q].w};
#pragma unroll
      for (int i = 0; i < kWtRI; i++) {
        const float x = q == 0 ? av[i].x : (q == 1 ? av[i].y : (q == 2 ? av[i].z : av[i].w));
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = fmaf(x, bq[j], acc[i][j]);
      }
    }
  }
}

// out(r_i, k_j) = sum_c A[r_i][c] W[k_j][c], c ascending, k_j = k0 + tx + 8 j.
// Columns k_j >= Kout read row 0 (a valid row) with no per-load select;
// their sums are never stored (the callers store k < Kout only).  Dropping
// the select took the MLP from 0.2095 to 0.1836 ms at 128,000 atoms.
__device__ __forceinline__ void wt_gemm_bwd(const float *A, int lda, int N, const float *W,
                                            int ldw, int k0, int Kout, int ty, int tx,
                                            float (&acc)[kWtRI][8]) {
  const float *ap = A + ty * lda;
  const float *wr[8];
#pragma unroll
  for (int j = 0; j < 8; j++) {
    const int k = k0 + tx + 8 * j;
    wr[j] = W + (k < Kout ? k : 0) * ldw;
  }
#pragma unroll 2
  for (int c = 0; c < N; c += 4) {
    float4 av[kWtRI], wv[8];
#pragma unroll
    for (int i = 0; i < kWtRI; i++) av[i] = *reinterpret_cast<const float4 *>(ap + 4 * i * lda + c);
#pragma unroll
    for (int j = 0; j < 8; j++)
      wv[j] = *reinterpret_cast<const float4 *>(wr[j] + c);
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int i = 0; i < kWtRI; i++) {
        const float x = q == 0 ? av[i].x : (q == 1 ? av[i].y : (q == 2 ? av[i].z : av[i].w));
#pragma unroll
        for (int j = 0; j < 8; j++) {
          const float wq = q == 0 ? wv[j].x : (q == 1 ? wv[j].y : (q == 2 ? wv[j].z : wv[j].w));
          acc[i][j] = fmaf(x, wq, acc[i][j]);
        }
      }
  }
}

template <int ACT>
__global__ void __launch_bounds__(kWtThreads, 1)
k_mlp_fp32w(MlpArgs a) {
  extern __shared__ float4 smw4[];
  float *sm = reinterpret_cast<float *>(smw4);
  const int L = a.nl, nin = a.nin;
  int sizes[kMaxLayers + 1];
  sizes[0] = nin;
  for (int l = 0; l < L; l++) sizes[l + 1] = a.layers[l].N;
  const WtLayout lay = wt_layout(L, sizes);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ty = lane >> 3, tx = lane & 7;
  const int ldh = lay.ldh, ldg = lay.ldg;
  float *wa = sm + lay.ef + w * lay.wf;  // this warp's area
  float *x1 = wa;                        // hidden output / gradient [32][ldh]
  float *dzb = wa + kWtRows * ldh;       // act' of hidden layer l at dzb + l * 32 * ldh
  double *erow = reinterpret_cast<double *>(wa + lay.wf - 2 * kWtRows);  // row energies
  const float *wsf = sm + lay.wsf;
  const double *wsd = reinterpret_cast<const double *>(sm + lay.wsd);
  int cur_elt = -1;
  for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
    const int elt = a.tiles[3 * tile], start = a.tiles[3 * tile + 1],
              count = a.tiles[3 * tile + 2];
    if (elt != cur_elt) {  // the same for every warp of the block
      __syncthreads();     // every warp is done with the previous element's weights
      cur_elt = elt;
      const MlpLayer *Ls = a.layers + (size_t)elt * L;
      for (int l = 0; l < L - 1; l++) {
        const int K = Ls[l].K, N = Ls[l].N, ldw = lay.ldw[l];
        float *Wd = sm + lay.woff[l];
        if ((reinterpret_cast<uintptr_t>(Ls[l].W) & 15) == 0) {
          // rows of N = 64 floats as 16-byte vectors (the 4 pad columns unused)
          const int n4 = N >> 2;
          for (int idx = threadIdx.x; idx < K * n4; idx += blockDim.x) {
            const int k = idx / n4, c4 = idx - k * n4;
            *reinterpret_cast<float4 *>(Wd + k * ldw + 4 * c4) =
                __ldg(reinterpret_cast<const float4 *>(Ls[l].W + (size_t)k * N) + c4);
          }
        } else {
          for (int idx = threadIdx.x; idx < K * ldw; idx += blockDim.x) {
            const int k = idx / ldw, c = idx - k * ldw;
            Wd[idx] = c < N ? __ldg(Ls[l].W + (size_t)k * N + c) : 0.f;
          }
        }
        float *bd = sm + lay.boff[l];
        for (int c = threadIdx.x; c < N; c += blockDim.x) bd[c] = Ls[l].b ? __ldg(Ls[l].b + c) : 0.f;
      }
      const MlpLayer lo = Ls[L - 1];
      double *wsdw = reinterpret_cast<double *>(sm + lay.wsd);
      for (int k = threadIdx.x; k < lo.K; k += blockDim.x) {
        double sd = 0.0;
        float sf = 0.f;
        for (int o2 = 0; o2 < lo.N; o2++) {
          sd += __ldg(lo.Wd + (size_t)k * lo.N + o2);
          sf += __ldg(lo.W + (size_t)k * lo.N + o2);
        }
        wsdw[k] = sd;
        sm[lay.wsf + k] = sf;
      }
      __syncthreads();
    }
    const int r0 = kWtRows * w;  // the warp's first row of the tile
    {
      // the next tile's G rows of this warp into L2 while this one runs
      const int nt = tile + gridDim.x;
      if (nt < a.ntiles) {
        const int ns = a.tiles[3 * nt + 1], nc = a.tiles[3 * nt + 2];
        if (lane < kWtRows && r0 + lane < nc) {
          const char *p = reinterpret_cast<const char *>(a.G + (size_t)a.perm[ns + r0 + lane] * nin);
          for (int off = 0; off < nin * 4; off += 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(p + off));
        }
      }
    }
    if (r0 >= count) continue;
    // lane r < kWtRows holds the atom of row r (-1 past the last atom)
    const int prow = lane < kWtRows && r0 + lane < count ? a.perm[start + r0 + lane] : -1;
    int at[kWtRI];
#pragma unroll
    for (int i = 0; i < kWtRI; i++) at[i] = __shfl_sync(0xffffffffu, prow, ty + 4 * i);
    // G rows of the tile into the warp area (row stride ldg), zero past the
    // last atom
    {
      const int nq = nin >> 2, total = kWtRows * nq;
      for (int base = 0; base < total; base += 32) {  // the same trip count in every lane
        const int idx = base + lane;
        const int r = idx < total ? idx / nq : 0, q = idx - r * nq;
        const int atr = __shfl_sync(0xffffffffu, prow, r);
        if (idx < total) {
          const float *src = a.G + (size_t)(atr >= 0 ? atr : 0) * nin + 4 * q;
          const uint32_t dst = tc::smem_u32(wa + r * ldg + 4 * q);
          asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
                       "r"(atr >= 0 ? 16 : 0));
        }
      }
      asm volatile("cp.async.commit_group;");
      asm volatile("cp.async.wait_group 0;" ::: "memory");
      __syncwarp();
    }
    // ---------------- forward ----------------
    for (int l = 0; l < L - 1; l++) {
      float acc[kWtRI][8];
#pragma unroll
      for (int i = 0; i < kWtRI; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
      wt_gemm_fwd(wa, l == 0 ? ldg : ldh, sizes[l], sm + lay.woff[l], lay.ldw[l], ty, tx, acc);
      __syncwarp();  // the input is read in full before the outputs overwrite it
      const float *bias = sm + lay.boff[l];
      // z = acc + b into the hidden buffer; the activation then runs as a
      // short loop over the lane's own four-column groups (the unrolled
      // register form would inline the activation 4 kWtRI times)
#pragma unroll
      for (int i = 0; i < kWtRI; i++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int r = ty + 4 * i, c = 32 * h + 4 * tx;
          *reinterpret_cast<float4 *>(x1 + r * ldh + c) =
              make_float4(acc[i][4 * h] + bias[c], acc[i][4 * h + 1] + bias[c + 1],
                          acc[i][4 * h + 2] + bias[c + 2], acc[i][4 * h + 3] + bias[c + 3]);
        }
      const bool last = l == L - 2;
      float *dz = dzb + (size_t)l * kWtRows * ldh;
#pragma unroll 1
      for (int ih = 0; ih < 2 * kWtRI; ih++) {
        const int r = ty + 4 * (ih >> 1), c = 32 * (ih & 1) + 4 * tx;
        const float4 z4 = *reinterpret_cast<const float4 *>(x1 + r * ldh + c);
        float y[4], d[4];
        y[0] = act_fwd(ACT, z4.x, d[0]);
        y[1] = act_fwd(ACT, z4.y, d[1]);
        y[2] = act_fwd(ACT, z4.z, d[2]);
        y[3] = act_fwd(ACT, z4.w, d[3]);
        if (!last) {
          *reinterpret_cast<float4 *>(x1 + r * ldh + c) = make_float4(y[0], y[1], y[2], y[3]);
          *reinterpret_cast<float4 *>(dz + r * ldh + c) = make_float4(d[0], d[1], d[2], d[3]);
        } else {
          // output layer in FP64 (the row's two column halves, each summed
          // over the 8 lanes of the row); gradient seed = row sums of W_out
          // times act'
          double p = 0.0;
#pragma unroll
          for (int u = 0; u < 4; u++) p = fma((double)y[u], wsd[c + u], p);
          p += __shfl_xor_sync(0xffffffffu, p, 1);
          p += __shfl_xor_sync(0xffffffffu, p, 2);
          p += __shfl_xor_sync(0xffffffffu, p, 4);
          if (tx == 0) erow[r] = (ih & 1) ? erow[r] + p : p;
          *reinterpret_cast<float4 *>(x1 + r * ldh + c) =
              make_float4(d[0] * wsf[c], d[1] * wsf[c + 1], d[2] * wsf[c + 2], d[3] * wsf[c + 3]);
        }
      }
      __syncwarp();
    }
    {
      const MlpLayer lo = a.layers[(size_t)elt * L + L - 1];
      double eb = 0.0;
      if (lo.bd)
        for (int o2 = 0; o2 < lo.N; o2++) eb += __ldg(lo.bd + o2);
      if (prow >= 0) a.E[prow] = erow[lane] + eb;  // prow >= 0 only for lanes < kWtRows
    }
    // ---------------- backward ----------------
    for (int l = L - 2; l >= 0; l--) {
      const int K = sizes[l];
      for (int k0 = 0; k0 < K; k0 += 64) {
        float acc[kWtRI][8];
#pragma unroll
        for (int i = 0; i < kWtRI; i++)
#pragma unroll
          for (int j = 0; j < 8; j++) acc[i][j] = 0.f;
        wt_gemm_bwd(x1, ldh, sizes[l + 1], sm + lay.woff[l], lay.ldw[l], k0, K, ty, tx, acc);
        if (l == 0) {
#pragma unroll
          for (int i = 0; i < kWtRI; i++) {
            if (at[i] < 0) continue;
            float *dst = a.dEdG + (size_t)at[i] * nin;
#pragma unroll
            for (int j = 0; j < 8; j++) {
              const int k = k0 + tx + 8 * j;
              if (k < K) dst[k] = acc[i][j];
            }
          }
        } else {
          __syncwarp();  // the gradient is read in full before it is overwritten
          const float *dz = dzb + (size_t)(l - 1) * kWtRows * ldh;
#pragma unroll
          for (int i = 0; i < kWtRI; i++) {
            const int r = ty + 4 * i;
#pragma unroll
            for (int j = 0; j < 8; j++) {
              const int k = tx + 8 * j;
              x1[r * ldh + k] = dz[r * ldh + k] * acc[i][j];
            }
          }
          __syncwarp();
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Streamed-weight form (k_mlp_fp32s) for MLPs whose weights do not fit in
// shared memory (e.g. 512-128-128-128 per element: 393 KB of FP32 W per
// direction).  Persistent CTAs of 256 threads walk 64-atom tiles.  Every GEMM
// of a tile is a sequence of chunks: 32 reduction rows x a 128-column output
// block of a weight array packed on the host as [block][rows][128] (forward:
// W, blocks over N; backward: W^T, blocks over K), so a chunk is one
// contiguous 16 KB that thread 0 copies with cp.async.bulk into a ring of S
// shared-memory stages, S - 1 chunks ahead (across layers and tiles), each
// completing on its stage's mbarrier.  Layer 0 reads G in 32-column chunks,
// gathered and transposed by all threads into the chunk's stage (the next
// chunk's G rows are loaded while the current chunk is multiplied).  Hidden
// activations, gradients and act' stay in shared memory (k-major, stride
// 64 + 4), as in the resident form.  Thread (ty, tx) of the 16 x 16 grid owns
// rows 4ty..4ty+3 and columns 4tx..4tx+3, 64+4tx..64+4tx+3 of a block: per
// reduction row one float4 of A, two of W and 16 FFMA2.  Products and sums
// per output in the same order as the other FP32 forms (reduction index
// ascending); the output layer in FP64.
// ---------------------------------------------------------------------------
constexpr int kFsTR = 64;
constexpr int kFsThreads = 256;
constexpr int kFsKC = 32;
constexpr int kFsCB = 128;
constexpr int kFsLDT = kFsTR + 4;
constexpr int kFsMaxStages = 6;
constexpr int kFsMaxChunks = 256;

struct FsChunk {
  short l, dir, blk, r0;
};

struct FsLayout {  // offsets in floats
  int stage;       // floats per stage: W chunk [32][128], then G chunk [32][68]
  int h0, h1, g, bias, wout, total;  // g: output gradients of residual MLPs
  int dzoff[kMaxLayers], boff[kMaxLayers];
};

__host__ __device__ inline FsLayout fs_layout(int nl, const int *sizes, int S, int resnet) {
  FsLayout f{};
  int maxh = 1;
  for (int l = 1; l < nl; l++) maxh = maxh > sizes[l] ? maxh : sizes[l];
  f.stage = kFsKC * kFsCB + kFsKC * kFsLDT;
  int o = S * f.stage;
  f.h0 = o; o += maxh * kFsLDT;
  f.h1 = o; o += maxh * kFsLDT;
  f.g = o;
  if (resnet) o += maxh * kFsLDT;
  for (int l = 0; l + 2 < nl; l++) { f.dzoff[l] = o; o += sizes[l + 1] * kFsLDT; }
  f.bias = o;
  int ob = 0;
  for (int l = 0; l + 1 < nl; l++) { f.boff[l] = ob; ob += sizes[l + 1]; }
  o += round_up(ob, 4);
  f.wout = round_up(o, 4);  // doubles from here
  o = f.wout + 2 * round_up(sizes[nl - 1], 2);
  f.total = round_up(o, 4);
  return f;
}

__global__ void __launch_bounds__(kFsThreads, 1)
k_mlp_fp32s(MlpArgs a) {
  extern __shared__ float4 fs4[];
  float *sm = reinterpret_cast<float *>(fs4);
  __shared__ __align__(8) uint64_t fullb[kFsMaxStages];
  __shared__ int rows_s[kFsTR];
  __shared__ FsChunk sched[kFsMaxChunks];
  __shared__ int nq_s, sz_s[kMaxLayers + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int L = a.nl, nin = a.nin, S = a.stages;
  if (tid == 0) {
    sz_s[0] = nin;
    for (int l = 0; l < L; l++) sz_s[l + 1] = a.layers[l].N;
    int k = 0;
    for (int l = 0; l < L - 1; l++)
      for (int nb = 0; nb * kFsCB < sz_s[l + 1]; nb++)
        for (int r0 = 0; r0 < sz_s[l]; r0 += kFsKC) sched[k++] = FsChunk{(short)l, 0, (short)nb, (short)r0};
    for (int l = L - 2; l >= 0; l--)
      for (int kb = 0; kb * kFsCB < sz_s[l]; kb++)
        for (int r0 = 0; r0 < sz_s[l + 1]; r0 += kFsKC) sched[k++] = FsChunk{(short)l, 1, (short)kb, (short)r0};
    nq_s = k;
    for (int s = 0; s < S; s++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc::smem_u32(&fullb[s])));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  __syncthreads();
  const int *sizes = sz_s;
  const int nq = nq_s;
  const FsLayout lay = fs_layout(L, sizes, S, a.resnet);
  float *bias_s = sm + lay.bias;
  // residual MLPs: g = dE/dy of the current hidden layer's output, [c][r]
  float *gres = sm + lay.g;
  double *wout_s = reinterpret_cast<double *>(sm + lay.wout);
  const int ntile_cta =
      blockIdx.x < a.ntiles ? (a.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  const int q_end = ntile_cta * nq;
  int q_issue = 0;  // thread 0: next chunk to copy
  bool ok = true;

  auto issue_to = [&](int qlim) {  // thread 0
    while (q_issue < qlim && q_issue < q_end) {
      const int t = blockIdx.x + (q_issue / nq) * gridDim.x;
      const FsChunk ch = sched[q_issue % nq];
      const MlpLayer &ly = a.layers[(size_t)a.tiles[3 * t] * L + ch.l];
      const int rows = ch.dir ? ly.N : ly.K;
      const float *src = (ch.dir ? ly.Wtp : ly.Wp) + ((size_t)ch.blk * rows + ch.r0) * kFsCB;
      const uint32_t bar = tc::smem_u32(&fullb[q_issue % S]);
      const uint32_t bytes = kFsKC * kFsCB * 4;
      tc::mbar_expect_tx(bar, bytes);
      tc::bulk_g2s(tc::smem_u32(sm + (size_t)(q_issue % S) * lay.stage), src, bytes, bar);
      q_issue++;
    }
  };
  if (tid == 0) issue_to(S - 1);

  int q = 0, cur_elt = -1;
  float4 gr[2];
  // G rows of reduction columns k0..k0+31 of this tile, into registers
  auto load_g = [&](int k0) {
#pragma unroll
    for (int u = 0; u < 2; u++) {
      const int idx = tid + u * kFsThreads, r = idx >> 3, q4 = idx & 7;
      const int at = rows_s[r];
      gr[u] = at >= 0 ? __ldg(reinterpret_cast<const float4 *>(a.G + (size_t)at * nin + k0 + 4 * q4))
                      : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  // wait for chunk q, free the previous stage for chunk q + S - 1
  auto next_chunk = [&]() -> float * {
    bool okc = true;
    if (tid == 0) okc = tc::mbar_wait(&fullb[q % S], (uint32_t)(q / S) & 1u);
    ok = __syncthreads_and(okc && ok) != 0;
    if (tid == 0 && ok) issue_to(q + S);
    return sm + (size_t)(q % S) * lay.stage;
  };
  auto fma_chunk = [&](const float *A, const float *Bw, float2 (&acc)[4][4]) {
    // fully unrolled: constant shared-memory offsets, loads scheduled ahead
    // (432,000-atom alloy MLP 6.27 -> 5.86 ms against an unroll of 4)
#pragma unroll
    for (int k = 0; k < kFsKC; k++) {
      const float4 av = *reinterpret_cast<const float4 *>(A + k * kFsLDT + 4 * ty);
      const float4 b0 = *reinterpret_cast<const float4 *>(Bw + k * kFsCB + 4 * tx);
      const float4 b1 = *reinterpret_cast<const float4 *>(Bw + k * kFsCB + 64 + 4 * tx);
      const float2 bb[4] = {make_float2(b0.x, b0.y), make_float2(b0.z, b0.w),
                            make_float2(b1.x, b1.y), make_float2(b1.z, b1.w)};
      const float ar[4] = {av.x, av.y, av.z, av.w};
#pragma unroll
      for (int i = 0; i < 4; i++) {
        const float2 a2 = make_float2(ar[i], ar[i]);
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = __ffma2_rn(a2, bb[j], acc[i][j]);
      }
    }
  };
  auto col_of = [&](int blk, int j) { return blk * kFsCB + (j < 4 ? 4 * tx + j : 64 + 4 * tx + j - 4); };
  auto acc_at = [&](const float2 (&acc)[4][4], int i, int j) {
    const float2 v = acc[i][j >> 1];
    return (j & 1) ? v.y : v.x;
  };

  for (int tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x) {
    const int elt = a.tiles[3 * tile], start = a.tiles[3 * tile + 1],
              count = a.tiles[3 * tile + 2];
    const MlpLayer *Ls = a.layers + (size_t)elt * L;
    if (tid < kFsTR) rows_s[tid] = tid < count ? a.perm[start + tid] : -1;
    if (elt != cur_elt) {
      cur_elt = elt;
      for (int l = 0; l < L - 1; l++)
        for (int c = tid; c < sizes[l + 1]; c += kFsThreads)
          bias_s[lay.boff[l] + c] = Ls[l].b ? __ldg(Ls[l].b + c) : 0.f;
      for (int c = tid; c < sizes[L - 1]; c += kFsThreads) wout_s[c] = __ldg(Ls[L - 1].Wd + c);
    }
    __syncthreads();
    float *hin = sm + lay.h0, *hout = sm + lay.h1;
    double ep[4] = {0.0, 0.0, 0.0, 0.0};
    load_g(0);

    // ---------------- forward ----------------
    for (int l = 0; l < L - 1 && ok; l++) {
      const int K = sizes[l], N = sizes[l + 1];
      const bool last = (l == L - 2);
      const bool res = a.resnet && l > 0 && K == N;  // y = act(z) + x (nnp.cpp:176-181)
      const float *bl = bias_s + lay.boff[l];
      float *dz = last ? nullptr : sm + lay.dzoff[l];
      for (int nb = 0; nb * kFsCB < N && ok; nb++) {
        float2 acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = make_float2(0.f, 0.f);
        for (int k0 = 0; k0 < K; k0 += kFsKC) {
          float *stW = sm + (size_t)(q % S) * lay.stage, *stG = stW + kFsKC * kFsCB;
          if (l == 0) {
#pragma unroll
            for (int u = 0; u < 2; u++) {
              const int idx = tid + u * kFsThreads, r = idx >> 3, q4 = idx & 7;
              const float v[4] = {gr[u].x, gr[u].y, gr[u].z, gr[u].w};
#pragma unroll
              for (int j = 0; j < 4; j++) stG[(4 * q4 + j) * kFsLDT + r] = v[j];
            }
          }
          next_chunk();
          if (!ok) break;
          if (l == 0) {  // the next chunk's G rows
            if (k0 + kFsKC < K) load_g(k0 + kFsKC);
            else if ((nb + 1) * kFsCB < N) load_g(0);
          }
          fma_chunk(l == 0 ? stG : hin + (size_t)k0 * kFsLDT, stW, acc);
          q++;
        }
        if (!ok) break;
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int r = 4 * ty + i;
#pragma unroll
          for (int j = 0; j < 8; j++) {
            const int c = col_of(nb, j);
            if (c < N) {
              float d;
              float y = act_fwd(a.actfn, acc_at(acc, i, j) + bl[c], d);
              if (res) y += hin[(size_t)c * kFsLDT + r];
              if (!last) {
                hout[(size_t)c * kFsLDT + r] = y;
                dz[(size_t)c * kFsLDT + r] = d;
              } else {
                // output layer in FP64; gradient seed g = w_out, gz = g * act'
                const double w = wout_s[c];
                ep[i] = fma((double)y, w, ep[i]);
                hout[(size_t)c * kFsLDT + r] = (float)w * d;
                if (a.resnet) gres[(size_t)c * kFsLDT + r] = (float)w;
              }
            }
          }
        }
      }
      __syncthreads();
      float *t = hin; hin = hout; hout = t;
    }
    if (!ok) break;
    {
      const MlpLayer lo = Ls[L - 1];
#pragma unroll
      for (int i = 0; i < 4; i++) {
        double e = ep[i];
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o, 16);
        const int at = rows_s[4 * ty + i];
        if (tx == 0 && at >= 0) {
          if (lo.bd)
            for (int o2 = 0; o2 < lo.N; o2++) e += __ldg(lo.bd + o2);
          a.E[at] = e;
        }
      }
    }

    // ---------------- backward ----------------
    for (int l = L - 2; l >= 0 && ok; l--) {
      const int K = sizes[l], N = sizes[l + 1];
      const float *dzp = l > 0 ? sm + lay.dzoff[l - 1] : nullptr;
      // g_{l-1} = (g_l act'_l) W_l^T, plus g_l through a residual layer
      const bool res = a.resnet && l > 0 && K == N;
      for (int kb = 0; kb * kFsCB < K && ok; kb++) {
        float2 acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
          for (int j = 0; j < 4; j++) acc[i][j] = make_float2(0.f, 0.f);
        for (int n0 = 0; n0 < N; n0 += kFsKC) {
          const float *stW = next_chunk();
          if (!ok) break;
          fma_chunk(hin + (size_t)n0 * kFsLDT, stW, acc);
          q++;
        }
        if (!ok) break;
#pragma unroll
        for (int i = 0; i < 4; i++) {
          const int r = 4 * ty + i;
          if (l > 0) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
              const int c = col_of(kb, j);
              if (c < K) {
                float g = acc_at(acc, i, j);
                if (res) g += gres[(size_t)c * kFsLDT + r];
                if (a.resnet) gres[(size_t)c * kFsLDT + r] = g;  // same element: in place
                hout[(size_t)c * kFsLDT + r] = g * dzp[(size_t)c * kFsLDT + r];
              }
            }
          } else {
            const int at = rows_s[r];
            if (at >= 0) {
              float *dst = a.dEdG + (size_t)at * nin;
              const int c0 = kb * kFsCB + 4 * tx, c1 = c0 + 64;
              if (c0 < K) *reinterpret_cast<float4 *>(dst + c0) =
                  make_float4(acc[i][0].x, acc[i][0].y, acc[i][1].x, acc[i][1].y);
              if (c1 < K) *reinterpret_cast<float4 *>(dst + c1) =
                  make_float4(acc[i][2].x, acc[i][2].y, acc[i][3].x, acc[i][3].y);
            }
          }
        }
      }
      __syncthreads();
      float *t = hin; hin = hout; hout = t;
    }
  }
  // copies still in flight (an error path leaves some): wait (bounded)
  if (tid == 0) {
    bool fine = ok;
    for (int qq = q; qq < q_issue; qq++)
      if (!tc::mbar_wait(&fullb[qq % S], (uint32_t)(qq / S) & 1u)) fine = false;
    if (!fine && a.status) atomicOr(a.status, kStatusTimeout);
  }
}

}  // namespace

size_t mlp_fp32r_smem(int nl, const int *sizes, int tr) {
  return sizeof(float) * (size_t)res_layout(nl, sizes, tr).total;
}

int mlp_fp32w_rows() { return kWtRows; }

size_t mlp_fp32w_smem(int nl, const int *sizes, int resnet, int warps) {
  if (resnet || nl < 2 || nl - 1 > kMaxLayers || warps < 1 || 32 * warps > kWtThreads) return 0;
  if (sizes[0] % 4 != 0 || sizes[0] < 4) return 0;
  for (int l = 1; l < nl; l++)
    if (sizes[l] != kWtWidth) return 0;
  const WtLayout w = wt_layout(nl, sizes);
  return sizeof(float) * ((size_t)w.ef + (size_t)warps * w.wf);
}

void mlp_fp32w_prepare(size_t smem) {
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaFuncSetAttribute(k_mlp_fp32w<0>, at, (int)smem);
  cudaFuncSetAttribute(k_mlp_fp32w<1>, at, (int)smem);
  cudaFuncSetAttribute(k_mlp_fp32w<2>, at, (int)smem);
  cudaFuncSetAttribute(k_mlp_fp32w<3>, at, (int)smem);
}

size_t mlp_fp32s_smem(int nl, const int *sizes, int resnet, int *stages) {
  *stages = 0;
  if (nl < 2 || nl - 1 > kMaxLayers) return 0;
  for (int l = 0; l < nl; l++)
    if (sizes[l] % kFsKC != 0 || sizes[l] > 32767) return 0;
  int nq = 0;
  for (int l = 0; l < nl - 1; l++) {
    const int K = sizes[l], N = sizes[l + 1];
    nq += ((N + kFsCB - 1) / kFsCB) * (K / kFsKC) + ((K + kFsCB - 1) / kFsCB) * (N / kFsKC);
  }
  if (nq > kFsMaxChunks) return 0;
  // 227 KB per block, less the kernel's static shared memory (the chunk
  // schedule and barriers)
  cudaFuncAttributes fa{};
  if (cudaFuncGetAttributes(&fa, k_mlp_fp32s) != cudaSuccess) return 0;
  const size_t limit = 227 * 1024 - fa.sharedSizeBytes;
  int S = kFsMaxStages;
  while (S >= 2 && sizeof(float) * (size_t)fs_layout(nl, sizes, S, resnet).total > limit) S--;
  if (S < 2) return 0;
  *stages = S;
  return sizeof(float) * (size_t)fs_layout(nl, sizes, S, resnet).total;
}

void mlp_fp32s_pack(const float *W, int K, int N, std::vector<float> &fwd, std::vector<float> &bwd) {
  // forward [N blocks][K][128]: block nb row k = W[k][128 nb ..]; backward
  // [K blocks][N][128]: block kb row n = W[128 kb ..][n]; zero beyond N / K
  const int nbF = (N + kFsCB - 1) / kFsCB, kbB = (K + kFsCB - 1) / kFsCB;
  fwd.assign((size_t)nbF * K * kFsCB, 0.f);
  bwd.assign((size_t)kbB * N * kFsCB, 0.f);
  for (int k = 0; k < K; k++)
    for (int n = 0; n < N; n++) {
      const float w = W[(size_t)k * N + n];
      fwd[((size_t)(n / kFsCB) * K + k) * kFsCB + n % kFsCB] = w;
      bwd[((size_t)(k / kFsCB) * N + n) * kFsCB + k % kFsCB] = w;
    }
}

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
  if (a.streamed > 0) {
    const int grid = a.ntiles < a.streamed ? a.ntiles : a.streamed;
    k_mlp_fp32s<<<grid, kFsThreads, a.smem, st>>>(a);
    return;
  }
  if (a.warped > 0) {
    const int grid = a.ntiles < a.resident ? a.ntiles : a.resident;
    const int T = 32 * a.warped;
    switch (a.actfn) {
      case 0: k_mlp_fp32w<0><<<grid, T, a.smem, st>>>(a); break;
      case 1: k_mlp_fp32w<1><<<grid, T, a.smem, st>>>(a); break;
      case 2: k_mlp_fp32w<2><<<grid, T, a.smem, st>>>(a); break;
      default: k_mlp_fp32w<3><<<grid, T, a.smem, st>>>(a); break;
    }
    return;
  }
  if (a.resident > 0) {
    const int grid = a.ntiles < a.resident ? a.ntiles : a.resident;
    if (a.tr == 128)
      k_mlp_fp32r<128, 512><<<grid, 512, a.smem, st>>>(a);
    else
      k_mlp_fp32r<64, 256><<<grid, 256, a.smem, st>>>(a);
    return;
  }
  if (a.tr == 64) {
    k_mlp_fp32<64><<<a.ntiles, kThreads, a.smem, st>>>(a);
  } else {
    k_mlp_fp32<32><<<a.ntiles, kThreads, a.smem, st>>>(a);
  }
}

void mlp_fp32s_prepare(size_t smem) {
  cudaFuncSetAttribute(k_mlp_fp32s, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

void mlp_fp32_prepare(int tr, size_t smem, bool resident) {
  if (resident && tr == 128)
    cudaFuncSetAttribute(k_mlp_fp32r<128, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  else if (resident)
    cudaFuncSetAttribute(k_mlp_fp32r<64, 256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)smem);
  else if (tr == 64)
    cudaFuncSetAttribute(k_mlp_fp32<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  else
    cudaFuncSetAttribute(k_mlp_fp32<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace tmd
