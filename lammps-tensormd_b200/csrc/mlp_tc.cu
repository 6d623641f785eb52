// mlp_tc.cu -- per-element MLP forward + backward on the 5th-generation tensor
// cores (tcgen05, sm_100a): BF16 operands, FP32 accumulation in tensor memory.
//
// Same semantics as the FP32 kernel (nnp.cu:9-57,149-281, nnp.cpp:246-365);
// only the GEMM operand precision changes.  One CTA of 128 threads owns 128
// atoms of one element (the MMA M dimension); thread t owns atom row t, which
// is TMEM lane t, so each thread reads its row of every accumulator with
// tcgen05.ld and runs the epilogue (bias, activation, act', residual, the
// FP64 output layer and the gradient seed) on its own row.
//
//   forward  layer l:  D[128 x N_l] = X_l[128 x K_l] . W_l           (TMEM)
//   backward layer l:  D[128 x K_l] = (g_l * act'_l)[128 x N_l] . W_l^T
//
// Operands live in shared memory in the canonical K-major no-swizzle layout
// of tcgen05 (8-row x 16-byte core matrices): A = activations / gradients
// written by the epilogue, or the G tile staged from global memory; B =
// weights pre-packed on the host in 64-column chunks that are copied to
// shared memory as contiguous blocks.  One thread issues the MMAs and a
// tcgen05.commit arrives on an mbarrier; every wait is bounded, and a timeout
// sets an error bit, releases the tensor memory and leaves the kernel.
#include <cuda_bf16.h>

#include <cstring>

#include "tc_util.cuh"
#include "tmd_kernels.h"

namespace tmd {

namespace {

using tc::TM;
using tc::KCH;
using tc::TMEM_COLS;
using tc::smem_u32;
using tc::sdesc;
using tc::commit;
using tc::mbar_wait;
using tc::tmem_ld32;
using tc::act_fwd;
using tc::bulk_g2s;
using tc::mbar_expect_tx;
constexpr int EPC = 8;       // BF16 elements per 16-byte core-matrix row
constexpr int KSTEP = 16;    // MMA K of kind::f16

// Instruction descriptor of kind::f16: D = FP32, A = B = BF16, K-major both,
// N >> 3 at [17,23), M >> 4 at [24,29).
__device__ inline uint32_t idesc_bf16(int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(TM >> 4) << 24);
}

__device__ inline void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t id,
                                uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(id), "r"(acc));
}

__device__ inline int core_off(int r, int k, int kfull) { return tc::core_off<EPC>(r, k, kfull); }

template <typename DZ>
__device__ inline DZ dz_store(float v);
template <>
__device__ inline float dz_store<float>(float v) { return v; }
template <>
__device__ inline __nv_bfloat16 dz_store<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

}  // namespace

// Store v as a BF16 operand: with NP = 3 also the residual v - hi in the
// second buffer (lo), so a product of two split operands is
// hi*hi' + hi*lo' + lo*hi' (FP32-class accuracy on BF16 tensor cores).
template <int NP>
__device__ inline void put_op(__nv_bfloat16 *buf, size_t lo_stride, int off, float v) {
  __nv_bfloat16 h = __float2bfloat16_rn(v);
  buf[off] = h;
  if (NP == 3) buf[lo_stride + off] = __float2bfloat16_rn(v - __bfloat162float(h));
}

// DZ: storage type of act'(z) per hidden layer (FP32 when it fits in shared
// memory, BF16 otherwise).  NP: 1 = BF16 products, 3 = split BF16 (hi/lo).
template <typename DZ, int NP>
__global__ void __launch_bounds__(TM)
k_mlp_tc(MlpTcArgs a) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base_s;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tile = blockIdx.x;
  const int elt = a.tiles[3 * tile], start = a.tiles[3 * tile + 1], count = a.tiles[3 * tile + 2];
  const int row_atom = tid < count ? a.perm[start + tid] : -1;
  const MlpTcLayer *Ls = a.layers + (size_t)elt * a.nl;
  const int L = a.nl;
  const int maxh = a.maxh;  // multiple of 64
  const int nin = a.nin;    // multiple of 64
  typedef __nv_bfloat16 T;
  // operand buffers; with NP = 3 each holds hi, then lo at +lo stride
  constexpr int NB = NP == 3 ? 2 : 1;
  T *opA = reinterpret_cast<T *>(smraw);                 // [NB][TM][KCH] staged G chunk
  T *opB = opA + NB * TM * KCH;                          // [NB][128][KCH] weight chunk
  T *actb = opB + NB * 128 * KCH;                        // [NB][TM][maxh] activations / gz
  const size_t act_lo = (size_t)TM * maxh;
  DZ *dzb = reinterpret_cast<DZ *>(actb + NB * TM * maxh);  // act' per hidden layer
  float *gres = reinterpret_cast<float *>(dzb + (size_t)(L - 1) * TM * maxh);  // resnet only

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base_s;
  const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  if (a.probe_wait > 0) {
    // failure-detection hook: a bounded wait on a barrier nothing arrives on
    // yet, before any MMA or copy is issued
    const bool done = mbar_wait(&mbar, 0u, a.probe_wait);
    ok = __syncthreads_and(done ? 1 : 0) != 0;
  }

  // D[TM x nout] (TMEM columns 0..nout-1) = A[TM x kred] . B^T with B rows
  // n0..n0+nout-1 of a packed weight block of brows rows.
  // a_src: 0 = stage the G tile from global memory, 1 = actb (whole buffer).
  // bsize: elements of one packed weight block (the lo block follows it)
  auto gemm = [&](int a_src, int kred, const T *Bpk, int brows, int n0, int nout) {
    const size_t bsize = (size_t)brows * kred;
    const int nch = kred / KCH;
    for (int c = 0; c < nch && ok; c++) {
      if (a_src == 0) {
        for (int idx = tid; idx < TM * KCH; idx += TM) {
          int r = idx / KCH, k = idx % KCH;
          int at = r < count ? a.perm[start + r] : -1;
          float v = at >= 0 ? __ldg(a.G + (size_t)at * nin + c * KCH + k) : 0.f;
          put_op<NP>(opA, (size_t)TM * KCH, core_off(r, k, KCH), v);
        }
      }
      for (int h = 0; h < NB; h++) {
        // packed weights: hi block, then (NP = 3) lo block of the same shape
        const T *blk = Bpk + (size_t)h * bsize;
        const uint4 *src = reinterpret_cast<const uint4 *>(blk + ((size_t)c * brows + n0) * KCH);
        uint4 *dst = reinterpret_cast<uint4 *>(opB + (size_t)h * 128 * KCH);
        const int nvec = nout * KCH * (int)sizeof(T) / 16;
        for (int i = tid; i < nvec; i += TM) dst[i] = __ldg(src + i);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t id = idesc_bf16(nout);
#pragma unroll
        for (int s = 0; s < KCH / KSTEP; s++) {
          uint64_t da;
          if (a_src == 0)
            da = sdesc(smem_u32(opA) + (uint32_t)(s * KSTEP / EPC) * 128u, 128u,
                       (uint32_t)(KCH / EPC) * 128u);
          else
            da = sdesc(smem_u32(actb) + (uint32_t)((c * KCH + s * KSTEP) / EPC) * 128u, 128u,
                       (uint32_t)(maxh / EPC) * 128u);
          uint64_t db = sdesc(smem_u32(opB) + (uint32_t)(s * KSTEP / EPC) * 128u, 128u,
                              (uint32_t)(KCH / EPC) * 128u);
          mma_bf16(tmem, da, db, id, (c > 0 || s > 0) ? 1u : 0u);
          if (NP == 3) {
            // start-address offsets of the lo halves (descriptor units of 16 B)
            const uint64_t a_lo = (uint64_t)(((a_src == 0 ? (size_t)TM * KCH : act_lo) * 2) >> 4);
            const uint64_t b_lo = (uint64_t)(((size_t)128 * KCH * 2) >> 4);
            mma_bf16(tmem, da, db + b_lo, id, 1u);  // hi * lo'
            mma_bf16(tmem, da + a_lo, db, id, 1u);  // lo * hi'
          }
        }
        commit(&mbar);
      }
      // every thread waits (bounded); the outcome is made block-uniform so all
      // threads take the same path through the remaining barriers
      const bool done = mbar_wait(&mbar, phase);
      ok = __syncthreads_and(done ? 1 : 0) != 0;
      phase ^= 1u;
      asm volatile("tcgen05.fence::after_thread_sync;");
    }
  };

  // ---------------- forward ----------------
  double E = 0.0;
  for (int l = 0; l < L - 1 && ok; l++) {
    const MlpTcLayer ly = Ls[l];
    gemm(l == 0 ? 0 : 1, ly.K, reinterpret_cast<const T *>(ly.Wf), ly.N, 0, ly.N);
    if (!ok) break;
    const bool res = a.resnet && l > 0 && ly.K == ly.N;
    const bool last = (l == L - 2);
    const double *wout = Ls[L - 1].wd;
    DZ *dz = dzb + (size_t)l * TM * maxh;
    for (int c0 = 0; c0 < ly.N; c0 += 32) {
      float v[32];
      tmem_ld32(trow + c0, v);
#pragma unroll 4
      for (int j = 0; j < 32; j++) {
        const int c = c0 + j;
        float z = v[j] + __ldg(ly.b + c);
        float d;
        float y = act_fwd(a.actfn, z, d);
        if (res) y += gres[(size_t)tid * maxh + c];  // layer input, FP32
        if (!last) {
          dz[(size_t)tid * maxh + c] = dz_store<DZ>(d);
          put_op<NP>(actb, act_lo, core_off(tid, c, maxh), y);
          if (a.resnet) gres[(size_t)tid * maxh + c] = y;
        } else {
          // output layer in FP64; gradient seed g = w_out, gz = g * act'
          const double w = __ldg(wout + c);
          E = fma((double)y, w, E);
          put_op<NP>(actb, act_lo, core_off(tid, c, maxh), (float)w * d);
          if (a.resnet) gres[(size_t)tid * maxh + c] = (float)w;
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
  }
  if (ok && row_atom >= 0) a.E[row_atom] = E + (Ls[L - 1].bd ? *Ls[L - 1].bd : 0.0);

  // ---------------- backward ----------------
  for (int l = L - 2; l >= 0 && ok; l--) {
    const MlpTcLayer ly = Ls[l];
    if (l == 0) {
      for (int n0 = 0; n0 < ly.K && ok; n0 += 128) {
        const int nout = min(128, ly.K - n0);
        gemm(1, ly.N, reinterpret_cast<const T *>(ly.Wb), ly.K, n0, nout);
        if (!ok) break;
        for (int c0 = 0; c0 < nout; c0 += 32) {
          float v[32];
          tmem_ld32(trow + c0, v);
          if (row_atom >= 0) {
            float4 *dst = reinterpret_cast<float4 *>(a.dEdG + (size_t)row_atom * nin + n0 + c0);
#pragma unroll
            for (int j = 0; j < 8; j++)
              dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
      }
    } else {
      gemm(1, ly.N, reinterpret_cast<const T *>(ly.Wb), ly.K, 0, ly.K);
      if (!ok) break;
      const bool res = a.resnet && ly.K == ly.N;
      const DZ *dzn = dzb + (size_t)(l - 1) * TM * maxh;
      for (int c0 = 0; c0 < ly.K; c0 += 32) {
        float v[32];
        tmem_ld32(trow + c0, v);
#pragma unroll 4
        for (int j = 0; j < 32; j++) {
          const int c = c0 + j;
          float g = v[j] + (res ? gres[(size_t)tid * maxh + c] : 0.f);
          if (a.resnet) gres[(size_t)tid * maxh + c] = g;
          put_op<NP>(actb, act_lo, core_off(tid, c, maxh),
                     g * (float)dzn[(size_t)tid * maxh + c]);
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();
    }
  }
  if (!ok && tid == 0) atomicOr(a.status, kStatusTimeout);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
}

// ---------------------------------------------------------------------------
// Persistent form for MLPs whose packed hidden weights fit in shared memory
// next to one tile's operand and act' buffers (no residual layers).  One CTA
// of 256 threads per SM walks the tiles (sorted by element) with a grid
// stride; the element's packed W^T and W blocks (hi, and lo for the split
// form) stay in shared memory until the element changes, so the GEMMs read
// only shared memory.  Thread t owns tile row 32 (w % 4) + lane (its TMEM
// lane) and, with warp w / 4, one half of every 64-column group of the
// accumulator: two threads share a row's epilogue.  Operands are written as
// whole 16-byte core rows, act' column-major ([layer][column][row]) so a
// warp's stores are contiguous.  MMAs, commit and the bounded waits are as in
// k_mlp_tc.
// ---------------------------------------------------------------------------
namespace {
constexpr int kTcpThreads = 256;

// Two values as a BF16 pair (bits), and their lo residuals for the split form.
__device__ inline uint32_t bf16x2_bits(float a, float b, uint32_t &lo_bits) {
  const __nv_bfloat162 hb = __floats2bfloat162_rn(a, b);
  const __nv_bfloat162 lb = __floats2bfloat162_rn(a - __low2float(hb), b - __high2float(hb));
  lo_bits = *reinterpret_cast<const uint32_t *>(&lb);
  return *reinterpret_cast<const uint32_t *>(&hb);
}

// 8 consecutive values as one 16-byte core row of BF16 (and the lo residuals).
// The values come as scalars so that the caller's arrays stay in registers.
template <int NP>
__device__ inline void put_core_row(__nv_bfloat16 *buf, size_t lo_stride, int off, float v0,
                                    float v1, float v2, float v3, float v4, float v5, float v6,
                                    float v7) {
  uint32_t l0, l1, l2, l3;
  const uint4 hi = make_uint4(bf16x2_bits(v0, v1, l0), bf16x2_bits(v2, v3, l1),
                              bf16x2_bits(v4, v5, l2), bf16x2_bits(v6, v7, l3));
  *reinterpret_cast<uint4 *>(buf + off) = hi;
  if (NP == 3) *reinterpret_cast<uint4 *>(buf + lo_stride + off) = make_uint4(l0, l1, l2, l3);
}
#define TMD_PUT_ROW(NP, buf, lo, off, v, b)                                                \
  put_core_row<NP>(buf, lo, off, v[b], v[b + 1], v[b + 2], v[b + 3], v[b + 4], v[b + 5], \
                   v[b + 6], v[b + 7])

// Elements of the resident weight blocks of one element's hidden layers.
__host__ __device__ inline size_t tcp_weight_elems(int nl, const int *sizes, int nb) {
  size_t w = 0;
  for (int l = 0; l < nl - 1; l++) w += 2 * (size_t)nb * sizes[l] * sizes[l + 1];
  return w;
}
}  // namespace

template <int NP, typename DZ>
__global__ void __launch_bounds__(kTcpThreads, 1)
k_mlp_tcp(MlpTcArgs a) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base_s;
  __shared__ int rows_s[TM];
  __shared__ double epart[2][TM];
  typedef __nv_bfloat16 T;
  constexpr int NB = NP == 3 ? 2 : 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quad = warp & 3, half = warp >> 2;
  const int row = quad * 32 + lane;
  const int L = a.nl, nin = a.nin, maxh = a.maxh;
  const int maxw = nin > maxh ? nin : maxh;
  int sizes[kMaxLayers + 1];
  sizes[0] = nin;
  for (int l = 0; l < L; l++) sizes[l + 1] = a.layers[l].N;
  T *wsm = reinterpret_cast<T *>(smraw);
  T *actb = wsm + tcp_weight_elems(L, sizes, NB);
  const size_t act_lo = (size_t)TM * maxw;
  DZ *dzb = reinterpret_cast<DZ *>(actb + NB * act_lo);  // act' [layer][column][row]
  // act' of every hidden layer but the last (whose act' is folded into the
  // gradient seed in its forward epilogue)
  size_t dzoff[kMaxLayers] = {};
  {
    size_t o = 0;
    for (int l = 0; l < L - 2; l++) { dzoff[l] = o; o += (size_t)sizes[l + 1] * TM; }
  }

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base_s;
  const uint32_t trow = tmem + ((uint32_t)(quad * 32) << 16);
  uint32_t phase = 0;
  bool ok = true;
  if (a.probe_wait > 0) {
    // failure-detection hook: a bounded wait on a barrier nothing arrives on
    // yet, before any MMA or copy is issued
    const bool done = mbar_wait(&mbar, 0u, a.probe_wait);
    ok = __syncthreads_and(done ? 1 : 0) != 0;
  }

  // D[TM x nout] = A[TM x kred] . B^T; A = actb laid out with kfull columns,
  // B rows n0..n0+nout-1 of a resident packed block of brows rows (hi, then
  // lo bsize elements later).
  auto gemm = [&](int kfull, int kred, const T *B, int brows, int n0, int nout) {
    const size_t bsize = (size_t)brows * kred;
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t id = idesc_bf16(nout);
      const uint64_t a_lo = (uint64_t)((act_lo * 2) >> 4);
      const uint64_t b_lo = (uint64_t)((bsize * 2) >> 4);
      for (int c = 0; c < kred / KCH; c++) {
#pragma unroll
        for (int s = 0; s < KCH / KSTEP; s++) {
          const uint64_t da = sdesc(smem_u32(actb) + (uint32_t)((c * KCH + s * KSTEP) / EPC) * 128u,
                                    128u, (uint32_t)(kfull / EPC) * 128u);
          const uint64_t db = sdesc(smem_u32(B + ((size_t)c * brows + n0) * KCH) +
                                        (uint32_t)(s * KSTEP / EPC) * 128u,
                                    128u, (uint32_t)(KCH / EPC) * 128u);
          mma_bf16(tmem, da, db, id, (c > 0 || s > 0) ? 1u : 0u);
          if (NP == 3) {
            mma_bf16(tmem, da, db + b_lo, id, 1u);  // hi * lo'
            mma_bf16(tmem, da + a_lo, db, id, 1u);  // lo * hi'
          }
        }
      }
      commit(&mbar);
    }
    const bool done = mbar_wait(&mbar, phase);
    ok = __syncthreads_and(done ? 1 : 0) != 0;
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;");
  };
  // operand writes visible to the tensor core, TMEM reads done, then barrier
  auto publish = [&]() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
  };

  int cur_elt = -1;
  for (int tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x) {
    const int elt = a.tiles[3 * tile], start = a.tiles[3 * tile + 1],
              count = a.tiles[3 * tile + 2];
    const MlpTcLayer *Ls = a.layers + (size_t)elt * L;
    __syncthreads();  // the previous tile is done with every buffer
    if (elt != cur_elt) {
      cur_elt = elt;
      T *w = wsm;
      for (int l = 0; l < L - 1; l++) {
        const size_t nblk = (size_t)NB * sizes[l] * sizes[l + 1];  // elements per direction
        for (int dir = 0; dir < 2; dir++) {
          const uint4 *src = reinterpret_cast<const uint4 *>(dir == 0 ? Ls[l].Wf : Ls[l].Wb);
          uint4 *dst = reinterpret_cast<uint4 *>(w);
          const int nvec = (int)(nblk * sizeof(T) / 16);
          for (int i = tid; i < nvec; i += kTcpThreads) dst[i] = __ldg(src + i);
          w += nblk;
        }
      }
    }
    if (tid < TM) rows_s[tid] = tid < count ? a.perm[start + tid] : -1;
    __syncthreads();
    // G tile as BF16 operand (kfull = nin), one 16-byte core row per step
    {
      const int nq = nin / 8;
      for (int idx = tid; idx < TM * nq; idx += kTcpThreads) {
        const int r = idx / nq, k8 = idx - r * nq;
        const int at = rows_s[r];
        float v[8];
        if (at >= 0) {
          const float4 *g = reinterpret_cast<const float4 *>(a.G + (size_t)at * nin + 8 * k8);
          const float4 p = __ldg(g), q = __ldg(g + 1);
          v[0] = p.x; v[1] = p.y; v[2] = p.z; v[3] = p.w;
          v[4] = q.x; v[5] = q.y; v[6] = q.z; v[7] = q.w;
        } else {
#pragma unroll
          for (int j = 0; j < 8; j++) v[j] = 0.f;
        }
        TMD_PUT_ROW(NP, actb, act_lo, core_off(r, 8 * k8, nin), v, 0);
      }
    }
    publish();
    const int row_atom = rows_s[row];

    // ---------------- forward ----------------
    double E = 0.0;
    const T *wl = wsm;
    for (int l = 0; l < L - 1 && ok; l++) {
      const MlpTcLayer ly = Ls[l];
      const int K = sizes[l], N = sizes[l + 1];
      gemm(l == 0 ? nin : maxh, K, wl, N, 0, N);
      wl += 2 * (size_t)NB * K * N;
      if (!ok) break;
      const bool last = (l == L - 2);
      const double *wout = Ls[L - 1].wd;
      DZ *dz = dzb + dzoff[l];
      for (int c0 = 32 * half; c0 < N; c0 += 64) {
        float v[32];
        tmem_ld32(trow + c0, v);
#pragma unroll
        for (int j = 0; j < 32; j++) {
          const int c = c0 + j;
          const float z = v[j] + __ldg(ly.b + c);
          float d;
          const float y = act_fwd(a.actfn, z, d);
          if (!last) {
            dz[(size_t)c * TM + row] = dz_store<DZ>(d);
            v[j] = y;
          } else {
            // output layer in FP64; gradient seed g = w_out, gz = g * act'
            const double w = __ldg(wout + c);
            E = fma((double)y, w, E);
            v[j] = (float)w * d;
          }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) TMD_PUT_ROW(NP, actb, act_lo, core_off(row, c0 + 8 * q, maxh), v, 8 * q);
      }
      publish();
    }
    if (!ok) break;
    epart[half][row] = E;
    __syncthreads();
    if (half == 0 && row_atom >= 0)
      a.E[row_atom] = (epart[0][row] + epart[1][row]) + (Ls[L - 1].bd ? *Ls[L - 1].bd : 0.0);

    // ---------------- backward ----------------
    for (int l = L - 2; l >= 0 && ok; l--) {
      size_t woff = 0;
      for (int q = 0; q < l; q++) woff += 2 * (size_t)NB * sizes[q] * sizes[q + 1];
      const int K = sizes[l], N = sizes[l + 1];
      const T *wb = wsm + woff + (size_t)NB * K * N;  // W block after the W^T block
      if (l == 0) {
        for (int n0 = 0; n0 < K && ok; n0 += 128) {
          const int nout = min(128, K - n0);
          gemm(maxh, N, wb, K, n0, nout);
          if (!ok) break;
          for (int c0 = 32 * half; c0 < nout; c0 += 64) {
            float v[32];
            tmem_ld32(trow + c0, v);
            if (row_atom >= 0) {
              float4 *dst = reinterpret_cast<float4 *>(a.dEdG + (size_t)row_atom * nin + n0 + c0);
#pragma unroll
              for (int j = 0; j < 8; j++)
                dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
            }
          }
          asm volatile("tcgen05.fence::before_thread_sync;");
          __syncthreads();
        }
      } else {
        gemm(maxh, N, wb, K, 0, K);
        if (!ok) break;
        const DZ *dzn = dzb + dzoff[l - 1];
        for (int c0 = 32 * half; c0 < K; c0 += 64) {
          float v[32];
          tmem_ld32(trow + c0, v);
#pragma unroll
          for (int j = 0; j < 32; j++) v[j] *= (float)dzn[(size_t)(c0 + j) * TM + row];
#pragma unroll
          for (int q = 0; q < 4; q++) TMD_PUT_ROW(NP, actb, act_lo, core_off(row, c0 + 8 * q, maxh), v, 8 * q);
        }
        publish();
      }
    }
  }
  if (!ok && tid == 0) atomicOr(a.status, kStatusTimeout);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
}

// ---------------------------------------------------------------------------
// Streamed-weight persistent form for MLPs whose weights do not fit in shared
// memory (e.g. 512-128-128-128 per element with four elements: 393 KB of
// BF16 W^T and W blocks per element).  One CTA of 512 threads per SM walks
// the tiles with a grid stride.  The weight chunks every tile needs (64
// reduction columns x the GEMM's rows, contiguous in the packed blocks) are a
// fixed schedule; thread 0 streams them from global memory (L2-resident)
// into a ring of S shared-memory stages with cp.async.bulk copies that
// complete on a per-stage mbarrier, up to S - 1 chunks ahead of the MMAs and
// across layer and tile boundaries, and issues every MMA; a tcgen05.commit
// per chunk frees its stage.  The G tile is converted to BF16 in 64-column
// chunks by all threads into two slots (written while the previous chunk's
// MMAs run), which alias the activation buffer of the hidden layers.  act'
// of the hidden layers stays in tensor memory (tcgen05.st) next to the
// accumulator: TMEM columns [0, accw) accumulate, then one block of act'
// columns per hidden layer; the final dE/dG GEMM (nin output columns) runs in
// 128-column blocks, up to four at a time, over all 512 columns once every
// act' has been used.  The epilogue thread mapping, operand writes, bounded
// waits and error path are those of k_mlp_tcp; on an error thread 0 also
// waits (bounded) for the copies still in flight before TMEM is released.
// CPS = 2 (BF16 form, where it fits): two CTAs of 256 threads per SM, each
// with half of TMEM (256 columns, act' stored as packed BF16 pairs) and half
// of shared memory, so one CTA's epilogues and block-wide waits run while the
// other's MMAs issue (432,000-atom 4-element alloy, 512-128-128-128
// softplus: 1.71 -> 1.44 ms per BF16 MLP; force error against FP64
// 6.7e-4 -> 7.4e-4 eV/A from the BF16 act').
// ---------------------------------------------------------------------------
namespace {
constexpr int kTcsThreads = 512;              // CTA size with one CTA per SM
constexpr int kTcsParts = kTcsThreads / 128;  // column parts per tile row (most)
constexpr int kTcsMaxChunks = 192;
constexpr int kTcsMaxBias = 512;
constexpr int kTcsMaxStages = 8;
constexpr int kTcsTmemCols = 512;

struct TcsChunk {  // one weight chunk of the per-tile schedule
  short l, dir, c, n0, nrows;
};

// Operand formats of the streamed form.  Both keep 128-byte chunk rows (KC
// reduction columns), so a weight chunk of R rows is R x 128 bytes either way.
//   OpBf16: kind::f16 with BF16 A and B, 8 elements per 16-byte core row,
//           MMA K = 16; activations from fast intrinsics (operands are BF16).
//   OpTf32: kind::tf32, 4 elements per core row, MMA K = 8; the values are
//           FP32 words rounded to TF32 (cvt.rna), split as hi + lo with
//           NP = 3 (hi*hi' + hi*lo' + lo*hi': the 3xTF32 scheme, ~21
//           significant bits per product, FP32 accumulation); activations
//           and act' from the accurate functions of the FP32 forms.
struct OpBf16 {
  typedef __nv_bfloat16 T;
  static constexpr int EPC = 8, KSTEP = 16, KC = 64;
  static constexpr bool kFastAct = true;
  static constexpr bool kSplitAcc = false;
  __device__ static uint32_t idesc(int N) { return idesc_bf16(N); }
  __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    mma_bf16(d, a, b, id, acc);
  }
  // 8 consecutive columns [c, c + 8) of row r (kfull columns): one core row
  template <int NP>
  __device__ static void put8(T *buf, size_t lo, int r, int c, int kfull, const float *v) {
    put_core_row<NP>(buf, lo, tc::core_off<EPC>(r, c, kfull), v[0], v[1], v[2], v[3], v[4],
                     v[5], v[6], v[7]);
  }
};

__device__ inline uint32_t tf32_rna(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return r;
}

struct OpTf32 {
  typedef float T;
  static constexpr int EPC = 4, KSTEP = 8, KC = 32;
  static constexpr bool kFastAct = false;
  static constexpr bool kSplitAcc = true;
  // D = FP32 [4,6) = 1, A = B = TF32 [7,10) = [10,13) = 2, K-major both
  __device__ static uint32_t idesc(int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(TM >> 4) << 24);
  }
  __device__ static void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(id), "r"(acc));
  }
  template <int NP>
  __device__ static void put4(T *buf, size_t lo, int off, float v0, float v1, float v2,
                              float v3) {
    const uint32_t h0 = tf32_rna(v0), h1 = tf32_rna(v1), h2 = tf32_rna(v2), h3 = tf32_rna(v3);
    *reinterpret_cast<uint4 *>(buf + off) = make_uint4(h0, h1, h2, h3);
    if (NP == 3)
      *reinterpret_cast<uint4 *>(buf + lo + off) =
          make_uint4(tf32_rna(v0 - __uint_as_float(h0)), tf32_rna(v1 - __uint_as_float(h1)),
                     tf32_rna(v2 - __uint_as_float(h2)), tf32_rna(v3 - __uint_as_float(h3)));
  }
  // 8 consecutive columns: two core rows in neighbouring core matrices
  template <int NP>
  __device__ static void put8(T *buf, size_t lo, int r, int c, int kfull, const float *v) {
    put4<NP>(buf, lo, tc::core_off<EPC>(r, c, kfull), v[0], v[1], v[2], v[3]);
    put4<NP>(buf, lo, tc::core_off<EPC>(r, c + 4, kfull), v[4], v[5], v[6], v[7]);
  }
};

// 32 act' values of one row as 16 packed BF16 pairs (column pair j in
// 32-bit column j), and back
__device__ inline void tmem_st16_pk(uint32_t taddr, const float v[32]) {
  uint32_t r[16];
#pragma unroll
  for (int j = 0; j < 16; j++) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
    r[j] = *reinterpret_cast<const uint32_t *>(&h);
  }
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
      "%13,%14,%15,%16};" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]),
      "r"(r[15])
      : "memory");
}
__device__ inline void tmem_ld16_pk(uint32_t taddr, float v[32]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; j++) {
    v[2 * j] = __uint_as_float(r[j] << 16);
    v[2 * j + 1] = __uint_as_float(r[j] & 0xffff0000u);
  }
}

__device__ inline void tmem_st32(uint32_t taddr, const float v[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
      "%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(
          taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
      "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
      "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
      "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
      "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
      "r"(__float_as_uint(v[15])), "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])),
      "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])), "r"(__float_as_uint(v[20])),
      "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
      "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])),
      "r"(__float_as_uint(v[27])), "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])),
      "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
      : "memory");
}

// Shared-memory plan of the streamed form: elements of one stage and of the
// operand region (per hi/lo part), TMEM accumulator width; kc = reduction
// columns per chunk (the format's KC).
struct TcsPlan {
  int maxrows, stage_elems, a_elems, accw;
};
__host__ __device__ inline TcsPlan tcs_plan(int nin, int maxh, int nb, int kc) {
  TcsPlan p;
  p.maxrows = maxh > 128 ? maxh : 128;
  p.stage_elems = nb * p.maxrows * kc;
  const int g2 = 2 * TM * kc, h = TM * maxh;
  p.a_elems = g2 > h ? g2 : h;
  p.accw = p.maxrows;
  (void)nin;
  return p;
}
}  // namespace

template <int NP, class OP, int CPS>
__global__ void __launch_bounds__(kTcsThreads / CPS, CPS)
k_mlp_tcs(MlpTcArgs a) {
  constexpr int NT = kTcsThreads / CPS, PARTS = NT / 128, TCOLS = kTcsTmemCols / CPS;
  constexpr bool PK = CPS == 2;  // act' as packed BF16 pairs
  static_assert(!PK || NP == 1, "packed act' only in the BF16 form");
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) uint64_t full_b[kTcsMaxStages], empty_b[kTcsMaxStages], gbar[2],
      accb[4], drainb;
  __shared__ uint32_t tmem_base_s;
  __shared__ int rows_s[TM];
  __shared__ double epart[kTcsParts][TM];
  __shared__ TcsChunk sched[kTcsMaxChunks];
  __shared__ int nq_s, sz_s[kMaxLayers + 1], act_s[kMaxLayers], bo_s[kMaxLayers];
  __shared__ float bias_s[kTcsMaxBias];   // hidden biases of the current element
  __shared__ double wout_s[256];          // its output-layer weights
  typedef typename OP::T T;
  constexpr int NB = NP == 3 ? 2 : 1;
  constexpr int EPC = OP::EPC, KSTEP = OP::KSTEP, KC = OP::KC;
  // split accumulators (3xTF32): hi*hi' into D_hi, hi*lo' + lo*hi' into D_lo,
  // summed in the epilogue, so that only one MMA per K step adds to a
  // full-magnitude accumulator
  constexpr bool kSplit = OP::kSplitAcc && NP == 3;
  // split, where TMEM has room: the hi*hi' products of odd K steps into a
  // second accumulator D_hi2 (half the full-magnitude accumulations each)
  const bool hi2 = kSplit && a.hi2;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int quad = warp & 3, part = warp >> 2;
  const int row = quad * 32 + lane;
  const int L = a.nl, nin = a.nin, maxh = a.maxh, S = a.stages;
  const TcsPlan pl = tcs_plan(nin, maxh, NB, KC);
  T *stage0 = reinterpret_cast<T *>(smraw);
  T *abuf = stage0 + (size_t)S * pl.stage_elems;
  const uint64_t a_lo_u = (uint64_t)(((size_t)pl.a_elems * sizeof(T)) >> 4);  // lo part, 16-B units
  const uint64_t b_lo_u = (uint64_t)(((size_t)pl.maxrows * KC * sizeof(T)) >> 4);

  if (tid == 0) {
    // layer widths, act' TMEM columns and bias offsets per hidden layer
    sz_s[0] = nin;
    for (int l = 0; l < L; l++) sz_s[l + 1] = a.layers[l].N;
    // act' of the last hidden layer is never stored (its gradient seed is
    // formed in its forward epilogue)
    int o = (kSplit ? (a.hi2 ? 3 : 2) : 1) * pl.accw, ob = 0;
    for (int l = 0; l < L - 1; l++) {
      act_s[l] = o;
      bo_s[l] = ob;
      if (l < L - 2) o += PK ? sz_s[l + 1] / 2 : sz_s[l + 1];
      ob += sz_s[l + 1];
    }
    const int *sizes = sz_s;
    int k = 0;
    for (int l = 0; l < L - 1; l++)
      for (int c = 0; c < sizes[l] / KC; c++)
        sched[k++] = TcsChunk{(short)l, 0, (short)c, 0, (short)sizes[l + 1]};
    for (int l = L - 2; l >= 1; l--)
      for (int c = 0; c < sizes[l + 1] / KC; c++)
        sched[k++] = TcsChunk{(short)l, 1, (short)c, 0, (short)sizes[l]};
    for (int n0 = 0; n0 < sizes[0]; n0 += 128)
      for (int c = 0; c < sizes[1] / KC; c++)
        sched[k++] = TcsChunk{0, 1, (short)c, (short)n0, (short)min(128, sizes[0] - n0)};
    nq_s = k;
    for (int s = 0; s < S; s++) {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&full_b[s])));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&empty_b[s])));
    }
    for (int j = 0; j < 2; j++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&gbar[j])));
    for (int j = 0; j < 4; j++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&accb[j])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&drainb)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&tmem_base_s)),
                 "r"(TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base_s;
  const uint32_t trow = tmem + ((uint32_t)(quad * 32) << 16);
  const int nq = nq_s;
  const int *sizes = sz_s;
  const int ntile_cta =
      blockIdx.x < a.ntiles ? (a.ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  const int q_end = ntile_cta * nq;
  int q_issue = 0, q_mma = 0;  // thread 0: next chunk to copy / to multiply
  bool ok0 = true;             // thread 0: its own waits
  bool ok = true;
  if (a.probe_wait > 0) {
    // failure-detection hook: a bounded wait on a barrier nothing arrives on
    // yet, before any MMA or copy is issued
    const bool done = mbar_wait(&drainb, 0u, a.probe_wait);
    ok = __syncthreads_and(done ? 1 : 0) != 0;
  }
  if (!ok) ok0 = false;
  uint32_t gk[2] = {0, 0}, ak[4] = {0, 0, 0, 0};  // completions consumed per barrier

  // thread 0: copy chunks up to (not including) qlim into their stages
  auto issue_to = [&](int qlim) {
    while (ok0 && q_issue < qlim && q_issue < q_end) {
      const int s = q_issue % S;
      if (q_issue >= S && !mbar_wait(&empty_b[s], (uint32_t)((q_issue / S) - 1) & 1u)) {
        ok0 = false;
        break;
      }
      const int t = blockIdx.x + (q_issue / nq) * gridDim.x;
      const TcsChunk ch = sched[q_issue % nq];
      const MlpTcLayer &ly = a.layers[(size_t)a.tiles[3 * t] * L + ch.l];
      const int K = sizes[ch.l], N = sizes[ch.l + 1];
      const int brows = ch.dir ? K : N;
      const T *src = reinterpret_cast<const T *>(ch.dir ? ly.Wb : ly.Wf) +
                     ((size_t)ch.c * brows + ch.n0) * KC;
      const uint32_t bytes = (uint32_t)(ch.nrows * KC * sizeof(T));
      const uint32_t bar = smem_u32(&full_b[s]);
      T *dst = stage0 + (size_t)s * pl.stage_elems;
      mbar_expect_tx(bar, bytes * NB);
      bulk_g2s(smem_u32(dst), src, bytes, bar);
      if (NP == 3) bulk_g2s(smem_u32(dst + (size_t)pl.maxrows * KC), src + (size_t)K * N, bytes, bar);
      q_issue++;
    }
  };
  // thread 0: the MMAs of the next chunk into TMEM column tcol (and, split,
  // the lo products into column tlo, the odd K steps' hi products into thi2
  // with hi2); A at a_addr (hi part) with 8-row group stride a_sbo bytes.
  // kst counts the K steps of the current GEMM.
  int kst = 0;
  auto mma_next = [&](uint32_t a_addr, uint32_t a_sbo, uint32_t tcol, uint32_t tlo, uint32_t thi2,
                      bool first) {
    if (!ok0) return;
    if (first) kst = 0;
    const int q = q_mma;
    const int s = q % S;
    if (!mbar_wait(&full_b[s], (uint32_t)(q / S) & 1u)) {
      ok0 = false;
      return;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    const TcsChunk ch = sched[q % nq];
    const uint32_t id = OP::idesc(ch.nrows);
    const uint32_t bbase = smem_u32(stage0 + (size_t)s * pl.stage_elems);
#pragma unroll
    for (int ks = 0; ks < KC / KSTEP; ks++) {
      const uint64_t da = sdesc(a_addr + (uint32_t)(ks * KSTEP / EPC) * 128u, 128u, a_sbo);
      const uint64_t db = sdesc(bbase + (uint32_t)(ks * KSTEP / EPC) * 128u, 128u,
                                (uint32_t)(KC / EPC) * 128u);
      const int g = kst++;
      const uint32_t acc = g >= 1 ? 1u : 0u;
      if (hi2) OP::mma(tmem + ((g & 1) ? thi2 : tcol), da, db, id, g >= 2 ? 1u : 0u);
      else OP::mma(tmem + tcol, da, db, id, acc);
      if (kSplit) {
        OP::mma(tmem + tlo, da, db + b_lo_u, id, acc);  // hi * lo'
        OP::mma(tmem + tlo, da + a_lo_u, db, id, 1u);   // lo * hi'
      } else if (NP == 3) {
        OP::mma(tmem + tcol, da, db + b_lo_u, id, 1u);  // hi * lo'
        OP::mma(tmem + tcol, da + a_lo_u, db, id, 1u);  // lo * hi'
      }
    }
    commit(&empty_b[s]);
    q_mma++;
    issue_to(q_mma + S - 1);
  };
  // every thread: wait for completion number k of barrier b (bounded)
  auto wait_all = [&](uint64_t *b, uint32_t &k) {
    const bool done = mbar_wait(b, k & 1u);
    k++;
    ok = __syncthreads_and((done && ok && (tid != 0 || ok0)) ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;");
  };
  auto publish = [&]() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    ok = __syncthreads_and((ok && (tid != 0 || ok0)) ? 1 : 0) != 0;
  };
  const uint32_t a_sbo_h = (uint32_t)(maxh / EPC) * 128u;   // activation buffer
  const uint32_t a_sbo_g = (uint32_t)(KC / EPC) * 128u;     // G chunk slot
  const uint32_t abase = smem_u32(abuf);
  const uint32_t lo_col = (uint32_t)pl.accw;                // D_lo of the layer GEMMs (split)
  const uint32_t hi2_col = 2u * (uint32_t)pl.accw;          // D_hi2 (hi2)
  // z = D_hi (+ D_hi2) + D_lo of 32 columns at c0 into v; d is scratch
  auto acc_ld = [&](int c0, float (&v)[32], float (&d)[32]) {
    tmem_ld32(trow + c0, v);
    if (hi2) {
      tmem_ld32(trow + hi2_col + c0, d);
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] += d[j];
    }
    if (kSplit) {
      tmem_ld32(trow + lo_col + c0, d);
#pragma unroll
      for (int j = 0; j < 32; j++) v[j] += d[j];
    }
  };

  int cur_elt = -1;
  if (tid == 0) issue_to(S - 1);
  for (int tile = blockIdx.x; tile < a.ntiles && ok; tile += gridDim.x) {
    const int elt = a.tiles[3 * tile], start = a.tiles[3 * tile + 1],
              count = a.tiles[3 * tile + 2];
    const MlpTcLayer *Ls = a.layers + (size_t)elt * L;
    if (tid < TM) rows_s[tid] = tid < count ? a.perm[start + tid] : -1;
    if (elt != cur_elt) {  // the element's biases and output weights
      cur_elt = elt;
      for (int l = 0; l < L - 1; l++)
        for (int c = tid; c < sizes[l + 1]; c += NT)
          bias_s[bo_s[l] + c] = __ldg(Ls[l].b + c);
      for (int c = tid; c < sizes[L - 1]; c += NT) wout_s[c] = __ldg(Ls[L - 1].wd + c);
    }
    __syncthreads();
    const int row_atom = rows_s[row];

    // ---------------- layer 0: G chunks through two slots ----------------
    // each thread converts kGRows core rows (8 columns of one atom row) per
    // chunk; the rows of chunk c + 1 are loaded while chunk c is published
    // and multiplied
    constexpr int kGRows = TM * (KC / 8) / NT;
    static_assert(kGRows * NT == TM * (KC / 8), "G chunk split");
    float4 gv[kGRows][2];
    auto load_g = [&](int c) {
#pragma unroll
      for (int u = 0; u < kGRows; u++) {
        const int idx = tid + u * NT;
        const int r = idx / (KC / 8), k8 = idx - r * (KC / 8);
        const int at = rows_s[r];
        if (at >= 0) {
          const float4 *g = reinterpret_cast<const float4 *>(a.G + (size_t)at * nin + c * KC + 8 * k8);
          gv[u][0] = __ldg(g);
          gv[u][1] = __ldg(g + 1);
        } else {
          gv[u][0] = gv[u][1] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
      }
    };
    load_g(0);
    for (int c = 0; c < nin / KC && ok; c++) {
      const int slot = c & 1;
      T *gs = abuf + (size_t)slot * TM * KC;
      if (c >= 2) wait_all(&gbar[slot], gk[slot]);  // the MMAs of chunk c - 2 are done
      if (!ok) break;
#pragma unroll
      for (int u = 0; u < kGRows; u++) {
        const int idx = tid + u * NT;
        const int r = idx / (KC / 8), k8 = idx - r * (KC / 8);
        const float v[8] = {gv[u][0].x, gv[u][0].y, gv[u][0].z, gv[u][0].w,
                            gv[u][1].x, gv[u][1].y, gv[u][1].z, gv[u][1].w};
        OP::template put8<NP>(gs, pl.a_elems, r, 8 * k8, KC, v);
      }
      if (c + 1 < nin / KC) load_g(c + 1);
      publish();
      if (!ok) break;
      if (tid == 0) {
        mma_next(smem_u32(gs), a_sbo_g, 0, lo_col, hi2_col, c == 0);
        commit(&gbar[slot]);
      }
    }
    if (!ok) break;
    if (tid == 0) commit(&accb[0]);
    wait_all(&accb[0], ak[0]);
    if (!ok) break;
    // each slot used this tile has one completion not yet consumed (its last
    // chunk, done by now): consume it so the parities stay in step
    for (int slot = 0; slot < 2; slot++)
      if ((nin / KC - slot + 1) / 2 > 0) wait_all(&gbar[slot], gk[slot]);
    if (!ok) break;

    // ---------------- forward epilogues and hidden layers ----------------
    double E = 0.0;
    for (int l = 0; l < L - 1 && ok; l++) {
      const int K = sizes[l], N = sizes[l + 1];
      const float *bl = bias_s + bo_s[l];
      const int actl = act_s[l];
      if (l > 0) {
        if (tid == 0) {
          for (int c = 0; c < K / KC; c++)
            mma_next(abase + (uint32_t)(c * KC / EPC) * 128u, a_sbo_h, 0, lo_col, hi2_col, c == 0);
          commit(&accb[0]);
        }
        wait_all(&accb[0], ak[0]);
        if (!ok) break;
      }
      const bool last = (l == L - 2);
      for (int c0 = 32 * part; c0 < N; c0 += 32 * PARTS) {
        float v[32], d[32];
        acc_ld(c0, v, d);
#pragma unroll
        for (int j = 0; j < 32; j++) {
          const int cc = c0 + j;
          const float z = v[j] + bl[cc];
          const float y = OP::kFastAct ? tc::act_fwd_fast(a.actfn, z, d[j])
                                       : tc::act_fwd(a.actfn, z, d[j]);
          if (!last) {
            v[j] = y;
          } else {
            // output layer in FP64; gradient seed g = w_out, gz = g * act'
            const double w = wout_s[cc];
            E = fma((double)y, w, E);
            v[j] = (float)w * d[j];
          }
        }
        if (!last) {
          if (PK) tmem_st16_pk(trow + actl + c0 / 2, d);
          else tmem_st32(trow + actl + c0, d);
        }
#pragma unroll
        for (int q = 0; q < 4; q++) OP::template put8<NP>(abuf, pl.a_elems, row, c0 + 8 * q, maxh, v + 8 * q);
      }
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      publish();
    }
    if (!ok) break;
    epart[part][row] = E;
    __syncthreads();
    if (part == 0 && row_atom >= 0)
      a.E[row_atom] = (PARTS == 4 ? (epart[0][row] + epart[1][row]) + (epart[2][row] + epart[3][row])
                                  : epart[0][row] + epart[1][row]) +
                      (Ls[L - 1].bd ? *Ls[L - 1].bd : 0.0);

    // ---------------- backward through the hidden layers ----------------
    for (int l = L - 2; l >= 1 && ok; l--) {
      const int K = sizes[l], N = sizes[l + 1];
      if (tid == 0) {
        for (int c = 0; c < N / KC; c++)
          mma_next(abase + (uint32_t)(c * KC / EPC) * 128u, a_sbo_h, 0, lo_col, hi2_col, c == 0);
        commit(&accb[0]);
      }
      wait_all(&accb[0], ak[0]);
      if (!ok) break;
      const int actp = act_s[l - 1];
      for (int c0 = 32 * part; c0 < K; c0 += 32 * PARTS) {
        float v[32], d[32];
        acc_ld(c0, v, d);
        if (PK) tmem_ld16_pk(trow + actp + c0 / 2, d);
        else tmem_ld32(trow + actp + c0, d);
#pragma unroll
        for (int j = 0; j < 32; j++) v[j] *= d[j];
#pragma unroll
        for (int q = 0; q < 4; q++) OP::template put8<NP>(abuf, pl.a_elems, row, c0 + 8 * q, maxh, v + 8 * q);
      }
      publish();
    }
    if (!ok) break;

    // ---------------- dE/dG = gz . W_0^T in 128-column blocks ----------------
    {
      // 128-column blocks over all TCOLS columns, each block np_ groups of
      // 128 columns (hi, then lo and hi2 when split): up to TCOLS / 128
      // blocks at a time
      const int N0 = sizes[1];
      const int nblk = (nin + 127) / 128;
      const int np_ = kSplit ? (hi2 ? 3 : 2) : 1, conc = (TCOLS / 128) / np_;
      for (int b0 = 0; b0 < nblk && ok; b0 += conc) {
        const int b1 = min(nblk, b0 + conc);
        if (tid == 0) {
          for (int b = b0; b < b1; b++) {
            const uint32_t cb = (uint32_t)(128 * np_ * (b - b0));
            for (int c = 0; c < N0 / KC; c++)
              mma_next(abase + (uint32_t)(c * KC / EPC) * 128u, a_sbo_h, cb, cb + 128u,
                       cb + 256u, c == 0);
            commit(&accb[b - b0]);
          }
        }
        for (int b = b0; b < b1 && ok; b++) {
          wait_all(&accb[b - b0], ak[b - b0]);
          if (!ok) break;
          const int n0 = 128 * b, nout = min(128, nin - n0);
          for (int c0 = 32 * part; c0 < nout; c0 += 32 * PARTS) {
            float v[32];
            const uint32_t cb = (uint32_t)(128 * np_ * (b - b0));
            tmem_ld32(trow + cb + c0, v);
            for (int pp = 1; pp < np_; pp++) {
              float w[32];
              tmem_ld32(trow + cb + 128u * pp + c0, w);
#pragma unroll
              for (int j = 0; j < 32; j++) v[j] += w[j];
            }
            if (row_atom >= 0) {
              float4 *dst = reinterpret_cast<float4 *>(a.dEdG + (size_t)row_atom * nin + n0 + c0);
#pragma unroll
              for (int j = 0; j < 8; j++)
                dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
            }
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        ok = __syncthreads_and(ok ? 1 : 0) != 0;
      }
    }
  }
  // drain: copies still in flight (error path) and every MMA, then free TMEM
  if (tid == 0) {
    bool fine = ok && ok0;
    for (int q = q_mma; q < q_issue; q++)
      if (!mbar_wait(&full_b[q % S], (uint32_t)(q / S) & 1u)) fine = false;
    commit(&drainb);
    if (!mbar_wait(&drainb, 0)) fine = false;
    if (!fine) atomicOr(a.status, kStatusTimeout);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TCOLS));
}

size_t mlp_tcs_smem(int nl, const int *sizes, int resnet, int np, int tf32, int cps,
                    int *stages) {
  *stages = 0;
  if (resnet || nl < 2 || nl - 1 > kMaxLayers) return 0;
  if (cps != 1 && (cps != 2 || np != 1 || tf32)) return 0;
  const int kc = tf32 ? OpTf32::KC : OpBf16::KC;
  const size_t esz = tf32 ? 4 : 2;
  const int nin = sizes[0];
  int maxh = 1, acts = 0;  // act' columns: every hidden layer but the last
  for (int l = 1; l < nl; l++) {
    if (sizes[l] % kc != 0 || sizes[l] > 256) return 0;
    maxh = maxh > sizes[l] ? maxh : sizes[l];
    if (l < nl - 1) acts += sizes[l];
  }
  if (nin % kc != 0) return 0;
  const int nb = np == 3 ? 2 : 1;
  const TcsPlan pl = tcs_plan(nin, maxh, nb, kc);
  const bool split = tf32 && np == 3;  // D_hi and D_lo accumulators
  if ((split ? 2 : 1) * pl.accw + (cps == 2 ? acts / 2 : acts) > kTcsTmemCols / cps) return 0;
  // chunk schedule length
  int nq = 0;
  for (int l = 0; l < nl - 1; l++) nq += sizes[l] / kc;
  for (int l = nl - 2; l >= 1; l--) nq += sizes[l + 1] / kc;
  nq += ((nin + 127) / 128) * (sizes[1] / kc);
  if (nq > kTcsMaxChunks) return 0;
  // as many stages as fit next to the operand region and ~12 KB of static
  // data; with two CTAs per SM each gets half of the SM's 228 KB less the
  // 1 KB the runtime reserves per CTA and the kernel's own static data
  size_t limit = 227 * 1024 - 12 * 1024;
  if (cps == 2) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, k_mlp_tcs<1, OpBf16, 2>) != cudaSuccess) return 0;
    limit = 228 * 1024 / 2 - 1024 - fa.sharedSizeBytes;
  }
  const size_t abytes = (size_t)nb * pl.a_elems * esz, sbytes = (size_t)pl.stage_elems * esz;
  if (abytes + 2 * sbytes > limit) return 0;
  int S = (int)((limit - abytes) / sbytes);
  if (S > kTcsMaxStages) S = kTcsMaxStages;
  *stages = S;
  return abytes + (size_t)S * sbytes;
}

int mlp_tcs_hi2(int nl, const int *sizes, int np, int tf32) {
  // room in TMEM for a second hi accumulator next to D_hi, D_lo and act'
  if (!(tf32 && np == 3)) return 0;
  int maxh = 1, acts = 0;
  for (int l = 1; l < nl; l++) {
    maxh = maxh > sizes[l] ? maxh : sizes[l];
    if (l < nl - 1) acts += sizes[l];
  }
  const TcsPlan pl = tcs_plan(sizes[0], maxh, 2, OpTf32::KC);
  return 3 * pl.accw + acts <= kTcsTmemCols ? 1 : 0;
}

void mlp_tcs_prepare(size_t smem, int np, int tf32, int cps) {
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (tf32) cudaFuncSetAttribute(k_mlp_tcs<3, OpTf32, 1>, at, (int)smem);
  else if (np == 3) cudaFuncSetAttribute(k_mlp_tcs<3, OpBf16, 1>, at, (int)smem);
  else if (cps == 2) cudaFuncSetAttribute(k_mlp_tcs<1, OpBf16, 2>, at, (int)smem);
  else cudaFuncSetAttribute(k_mlp_tcs<1, OpBf16, 1>, at, (int)smem);
}

size_t mlp_tcp_smem(int nl, const int *sizes, int resnet, int np, bool dz_bf16) {
  if (resnet || nl < 2) return 0;
  const size_t nb = np == 3 ? 2 : 1;
  int maxh = 1;
  for (int l = 1; l < nl; l++) maxh = maxh > sizes[l] ? maxh : sizes[l];
  const int maxw = sizes[0] > maxh ? sizes[0] : maxh;
  size_t b = tcp_weight_elems(nl, sizes, (int)nb) * 2;  // resident W^T and W blocks
  b += nb * (size_t)TM * maxw * 2;                      // operand buffer
  for (int l = 1; l < nl - 1; l++) b += (size_t)sizes[l] * TM * (dz_bf16 ? 2 : 4);  // act'
  return b;
}

void pack_core_chunks(const float *src, int rows, int cols, long ld_r, long ld_k,
                      uint16_t *dst) {
  // chunk c holds columns [64c, 64c + 64) of every row; inside a chunk the
  // element (r, k) sits at ((r/8) * 8 + k/8) * 64 + (r%8) * 8 + k%8
  const int nch = (cols + KCH - 1) / KCH;
  for (int c = 0; c < nch; c++)
    for (int r = 0; r < rows; r++)
      for (int kk = 0; kk < KCH; kk++) {
        int k = c * KCH + kk;
        float v = k < cols ? src[(long)r * ld_r + (long)k * ld_k] : 0.f;
        __nv_bfloat16 h = __float2bfloat16_rn(v);
        uint16_t bits;
        memcpy(&bits, &h, 2);
        size_t off = (size_t)c * rows * KCH +
                     (size_t)(((r >> 3) * (KCH / EPC) + kk / EPC) * (8 * EPC) + (r & 7) * EPC + kk % EPC);
        dst[off] = bits;
      }
}

float tf32_round_host(float v) {
  // round to the 10-bit TF32 mantissa, ties away from zero (as cvt.rna)
  uint32_t b;
  memcpy(&b, &v, 4);
  if ((b & 0x7f800000u) != 0x7f800000u) b = (b + 0x1000u) & 0xffffe000u;
  float r;
  memcpy(&r, &b, 4);
  return r;
}

void pack_core_chunks_tf32(const float *src, int rows, int cols, long ld_r, long ld_k, int part,
                           float *dst) {
  // chunks of 32 columns; inside a chunk the element (r, k) sits at
  // ((r/8) * 8 + k/4) * 32 + (r%8) * 4 + k%4; part 0 = hi = tf32(v),
  // part 1 = lo = tf32(v - hi)
  constexpr int kc = OpTf32::KC, epc = OpTf32::EPC;
  const int nch = (cols + kc - 1) / kc;
  for (int c = 0; c < nch; c++)
    for (int r = 0; r < rows; r++)
      for (int kk = 0; kk < kc; kk++) {
        const int k = c * kc + kk;
        const float v = k < cols ? src[(long)r * ld_r + (long)k * ld_k] : 0.f;
        const float hi = tf32_round_host(v);
        const size_t off = (size_t)c * rows * kc +
                           (size_t)(((r >> 3) * (kc / epc) + kk / epc) * (8 * epc) + (r & 7) * epc + kk % epc);
        dst[off] = part == 0 ? hi : tf32_round_host(v - hi);
      }
}

size_t mlp_tc_smem(int nl, int maxh, int resnet, bool dz_bf16, int np) {
  const size_t nb = np == 3 ? 2 : 1;
  size_t b = nb * ((size_t)TM * KCH * 2 + (size_t)128 * KCH * 2);  // opA + opB
  b += nb * (size_t)TM * maxh * 2;                                 // actb
  b += (size_t)(nl - 1) * TM * maxh * (dz_bf16 ? 2 : 4);           // act'
  if (resnet) b += (size_t)TM * maxh * 4;                          // residual rows
  return b;
}

void mlp_tc_prepare(size_t smem, bool dz_bf16, int np) {
  const int s = (int)smem;
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (np == 3) {
    if (dz_bf16) cudaFuncSetAttribute(k_mlp_tc<__nv_bfloat16, 3>, at, s);
    else cudaFuncSetAttribute(k_mlp_tc<float, 3>, at, s);
  } else {
    if (dz_bf16) cudaFuncSetAttribute(k_mlp_tc<__nv_bfloat16, 1>, at, s);
    else cudaFuncSetAttribute(k_mlp_tc<float, 1>, at, s);
  }
}

void mlp_tcp_prepare(size_t smem, int np, bool dz_bf16) {
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (np == 3) cudaFuncSetAttribute(k_mlp_tcp<3, float>, at, (int)smem);
  else if (dz_bf16) cudaFuncSetAttribute(k_mlp_tcp<1, __nv_bfloat16>, at, (int)smem);
  else cudaFuncSetAttribute(k_mlp_tcp<1, float>, at, (int)smem);
}

void launch_mlp_tc(const MlpTcArgs &a, cudaStream_t st, long &launches) {
  if (a.ntiles <= 0) return;
  if (a.streamed > 0) {
    const int grid = a.ntiles < a.streamed ? a.ntiles : a.streamed;
    if (a.tf32) k_mlp_tcs<3, OpTf32, 1><<<grid, kTcsThreads, a.smem_s, st>>>(a);
    else if (a.np == 3) k_mlp_tcs<3, OpBf16, 1><<<grid, kTcsThreads, a.smem_s, st>>>(a);
    else if (a.cps_s == 2) k_mlp_tcs<1, OpBf16, 2><<<grid, kTcsThreads / 2, a.smem_s, st>>>(a);
    else k_mlp_tcs<1, OpBf16, 1><<<grid, kTcsThreads, a.smem_s, st>>>(a);
    launches += 1;
    return;
  }
  if (a.persistent > 0) {
    const int grid = a.ntiles < a.persistent ? a.ntiles : a.persistent;
    if (a.np == 3) k_mlp_tcp<3, float><<<grid, kTcpThreads, a.smem_p, st>>>(a);
    else if (a.dz_bf16_p) k_mlp_tcp<1, __nv_bfloat16><<<grid, kTcpThreads, a.smem_p, st>>>(a);
    else k_mlp_tcp<1, float><<<grid, kTcpThreads, a.smem_p, st>>>(a);
    launches += 1;
    return;
  }
  if (a.np == 3) {
    if (a.dz_bf16) k_mlp_tc<__nv_bfloat16, 3><<<a.ntiles, TM, a.smem, st>>>(a);
    else k_mlp_tc<float, 3><<<a.ntiles, TM, a.smem, st>>>(a);
  } else {
    if (a.dz_bf16) k_mlp_tc<__nv_bfloat16, 1><<<a.ntiles, TM, a.smem, st>>>(a);
    else k_mlp_tc<float, 1><<<a.ntiles, TM, a.smem, st>>>(a);
  }
  launches += 1;
}

}  // namespace tmd
