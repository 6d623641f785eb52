// mlp_fp8.cu -- per-element MLP forward + backward on the tcgen05 tensor cores
// with FP8 (e4m3) operands and FP32 accumulation in tensor memory.
//
// Same structure and semantics as the BF16 kernel (mlp_tc.cu; nnp.cu:9-57,
// 149-281, nnp.cpp:246-365) with tcgen05.mma kind::f8f6f4 (K = 32 per
// instruction) on the same 8-row x 16-byte core-matrix layout.  Scaling:
//   weights      one scale per layer, s_w = 448 / max|W_l| (host, at load)
//   A operands   one scale per atom row, s_a = 448 / max|row| (the G row, the
//                activations or the gradients of that atom); a row scale
//                factors out of the K sum, so the epilogue divides the
//                accumulator row by s_a * s_w exactly
// The epilogue makes two passes over the accumulator row: the first finds
// the row maximum of the values it will store, the second recomputes them and
// stores them quantised.  The FP64 output layer, the residual rows and
// act'(z) stay as in the BF16 kernel (FP32 / FP64).
#include <cuda_fp8.h>

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
constexpr int EPC8 = 16;     // e4m3 elements per 16-byte core-matrix row
constexpr int KSTEP8 = 32;   // MMA K of kind::f8f6f4 for 8-bit operands
constexpr float kE4M3Max = 448.f;

// Instruction descriptor of kind::f8f6f4: D = FP32 [4,6) = 1, A = B = E4M3
// ([7,10) = [10,13) = 0), K-major both, N >> 3 at [17,23), M >> 4 at [24,29).
__device__ inline uint32_t idesc_fp8(int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);
}

__device__ inline void mma_fp8(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t id,
                               uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(id), "r"(acc));
}

__device__ inline uint8_t q8(float v) {
  return (uint8_t)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
}

__device__ inline float row_scale(float amax) { return amax > 0.f ? kE4M3Max / amax : 1.f; }

__device__ inline int off8(int r, int k, int kfull) { return tc::core_off<EPC8>(r, k, kfull); }

template <typename DZ>
__device__ inline DZ dz_put(float v);
template <>
__device__ inline float dz_put<float>(float v) { return v; }
template <>
__device__ inline __nv_bfloat16 dz_put<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

}  // namespace

template <typename DZ>
__global__ void __launch_bounds__(TM)
k_mlp_fp8(MlpTcArgs a) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_base_s;
  __shared__ float rsc[TM];  // row scales of the staged G tile
  const int tid = threadIdx.x, warp = tid >> 5;
  const int tile = blockIdx.x;
  const int elt = a.tiles[3 * tile], start = a.tiles[3 * tile + 1], count = a.tiles[3 * tile + 2];
  const int row_atom = tid < count ? a.perm[start + tid] : -1;
  const MlpTcLayer *Ls = a.layers + (size_t)elt * a.nl;
  const int L = a.nl;
  const int maxh = a.maxh;  // multiple of 64
  const int nin = a.nin;    // multiple of 64
  uint8_t *opA = smraw;                                    // [TM][KCH] staged G chunk
  uint8_t *opB = opA + TM * KCH;                           // [128][KCH] weight chunk
  uint8_t *actb = opB + 128 * KCH;                         // [TM][maxh] activations / gz
  DZ *dzb = reinterpret_cast<DZ *>(actb + (size_t)TM * maxh);  // act' per hidden layer
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
  // row scale of this atom's G row
  {
    float amax = 0.f;
    if (row_atom >= 0)
      for (int k = 0; k < nin; k++) amax = fmaxf(amax, fabsf(__ldg(a.G + (size_t)row_atom * nin + k)));
    rsc[tid] = row_scale(amax);
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
  float sa = rsc[tid];  // scale of this thread's row of the current A operand

  // D[TM x nout] = A[TM x kred] . B^T, B rows n0..n0+nout-1 of a packed block
  // of brows rows.  a_src 0: stage the G tile (scaled by its row scales);
  // 1: actb.
  auto gemm = [&](int a_src, int kred, const uint8_t *Bpk, int brows, int n0, int nout) {
    const int nch = kred / KCH;
    for (int c = 0; c < nch && ok; c++) {
      if (a_src == 0) {
        for (int idx = tid; idx < TM * KCH; idx += TM) {
          int r = idx / KCH, k = idx % KCH;
          int at = r < count ? a.perm[start + r] : -1;
          float v = at >= 0 ? __ldg(a.G + (size_t)at * nin + c * KCH + k) : 0.f;
          opA[off8(r, k, KCH)] = q8(v * rsc[r]);
        }
      }
      const uint4 *src = reinterpret_cast<const uint4 *>(Bpk + ((size_t)c * brows + n0) * KCH);
      uint4 *dst = reinterpret_cast<uint4 *>(opB);
      const int nvec = nout * KCH / 16;
      for (int i = tid; i < nvec; i += TM) dst[i] = __ldg(src + i);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t id = idesc_fp8(nout);
#pragma unroll
        for (int s = 0; s < KCH / KSTEP8; s++) {
          uint64_t da;
          if (a_src == 0)
            da = sdesc(smem_u32(opA) + (uint32_t)(s * KSTEP8 / EPC8) * 128u, 128u,
                       (uint32_t)(KCH / EPC8) * 128u);
          else
            da = sdesc(smem_u32(actb) + (uint32_t)((c * KCH + s * KSTEP8) / EPC8) * 128u, 128u,
                       (uint32_t)(maxh / EPC8) * 128u);
          uint64_t db = sdesc(smem_u32(opB) + (uint32_t)(s * KSTEP8 / EPC8) * 128u, 128u,
                              (uint32_t)(KCH / EPC8) * 128u);
          mma_fp8(tmem, da, db, id, (c > 0 || s > 0) ? 1u : 0u);
        }
        commit(&mbar);
      }
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
    gemm(l == 0 ? 0 : 1, ly.K, reinterpret_cast<const uint8_t *>(ly.Wf), ly.N, 0, ly.N);
    if (!ok) break;
    const float inv = 1.f / (sa * ly.wscale);
    const bool res = a.resnet && l > 0 && ly.K == ly.N;
    const bool last = (l == L - 2);
    const double *wout = Ls[L - 1].wd;
    DZ *dz = dzb + (size_t)l * TM * maxh;
    // pass 1: the row maximum of what the epilogue stores as the next A
    float amax = 0.f;
    for (int c0 = 0; c0 < ly.N; c0 += 32) {
      float v[32];
      tmem_ld32(trow + c0, v);
      for (int j = 0; j < 32; j++) {
        const int c = c0 + j;
        float d;
        float y = act_fwd(a.actfn, v[j] * inv + __ldg(ly.b + c), d);
        if (res) y += gres[(size_t)tid * maxh + c];
        amax = fmaxf(amax, fabsf(last ? (float)__ldg(wout + c) * d : y));
      }
    }
    const float sn = row_scale(amax);
    // pass 2: recompute, store act', the quantised next operand, the energy
    for (int c0 = 0; c0 < ly.N; c0 += 32) {
      float v[32];
      tmem_ld32(trow + c0, v);
      for (int j = 0; j < 32; j++) {
        const int c = c0 + j;
        float d;
        float y = act_fwd(a.actfn, v[j] * inv + __ldg(ly.b + c), d);
        if (res) y += gres[(size_t)tid * maxh + c];
        if (!last) {
          dz[(size_t)tid * maxh + c] = dz_put<DZ>(d);
          actb[off8(tid, c, maxh)] = q8(y * sn);
          if (a.resnet) gres[(size_t)tid * maxh + c] = y;
        } else {
          const double w = __ldg(wout + c);
          E = fma((double)y, w, E);
          actb[off8(tid, c, maxh)] = q8((float)w * d * sn);
          if (a.resnet) gres[(size_t)tid * maxh + c] = (float)w;
        }
      }
    }
    sa = sn;
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
  }
  if (ok && row_atom >= 0) a.E[row_atom] = E + (Ls[L - 1].bd ? *Ls[L - 1].bd : 0.0);

  // ---------------- backward ----------------
  for (int l = L - 2; l >= 0 && ok; l--) {
    const MlpTcLayer ly = Ls[l];
    const float inv = 1.f / (sa * ly.wscale);
    if (l == 0) {
      for (int n0 = 0; n0 < ly.K && ok; n0 += 128) {
        const int nout = min(128, ly.K - n0);
        gemm(1, ly.N, reinterpret_cast<const uint8_t *>(ly.Wb), ly.K, n0, nout);
        if (!ok) break;
        for (int c0 = 0; c0 < nout; c0 += 32) {
          float v[32];
          tmem_ld32(trow + c0, v);
          if (row_atom >= 0) {
            float4 *dst = reinterpret_cast<float4 *>(a.dEdG + (size_t)row_atom * nin + n0 + c0);
#pragma unroll
            for (int j = 0; j < 8; j++)
              dst[j] = make_float4(v[4 * j] * inv, v[4 * j + 1] * inv, v[4 * j + 2] * inv,
                                   v[4 * j + 3] * inv);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
      }
    } else {
      gemm(1, ly.N, reinterpret_cast<const uint8_t *>(ly.Wb), ly.K, 0, ly.K);
      if (!ok) break;
      const bool res = a.resnet && ly.K == ly.N;
      const DZ *dzn = dzb + (size_t)(l - 1) * TM * maxh;
      float amax = 0.f;
      for (int c0 = 0; c0 < ly.K; c0 += 32) {
        float v[32];
        tmem_ld32(trow + c0, v);
        for (int j = 0; j < 32; j++) {
          const int c = c0 + j;
          const float g = v[j] * inv + (res ? gres[(size_t)tid * maxh + c] : 0.f);
          amax = fmaxf(amax, fabsf(g * (float)dzn[(size_t)tid * maxh + c]));
        }
      }
      const float sn = row_scale(amax);
      for (int c0 = 0; c0 < ly.K; c0 += 32) {
        float v[32];
        tmem_ld32(trow + c0, v);
        for (int j = 0; j < 32; j++) {
          const int c = c0 + j;
          const float g = v[j] * inv + (res ? gres[(size_t)tid * maxh + c] : 0.f);
          if (a.resnet) gres[(size_t)tid * maxh + c] = g;
          actb[off8(tid, c, maxh)] = q8(g * (float)dzn[(size_t)tid * maxh + c] * sn);
        }
      }
      sa = sn;
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

void pack_core_chunks_fp8(const float *src, int rows, int cols, long ld_r, long ld_k,
                          float scale, uint8_t *dst) {
  // chunk c holds columns [64c, 64c + 64) of every row; inside a chunk the
  // element (r, k) sits at ((r/8) * 4 + k/16) * 128 + (r%8) * 16 + k%16
  const int nch = (cols + KCH - 1) / KCH;
  for (int c = 0; c < nch; c++)
    for (int r = 0; r < rows; r++)
      for (int kk = 0; kk < KCH; kk++) {
        int k = c * KCH + kk;
        float v = k < cols ? src[(long)r * ld_r + (long)k * ld_k] * scale : 0.f;
        dst[(size_t)c * rows * KCH + tc::core_off<EPC8>(r, kk, KCH)] =
            (uint8_t)__nv_cvt_float_to_fp8(v, __NV_SATFINITE, __NV_E4M3);
      }
}

size_t mlp_fp8_smem(int nl, int maxh, int resnet, bool dz_bf16) {
  size_t b = (size_t)TM * KCH + (size_t)128 * KCH;        // opA + opB
  b += (size_t)TM * maxh;                                  // actb
  b += (size_t)(nl - 1) * TM * maxh * (dz_bf16 ? 2 : 4);   // act'
  if (resnet) b += (size_t)TM * maxh * 4;                  // residual rows
  return b;
}

void mlp_fp8_prepare(size_t smem, bool dz_bf16) {
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  if (dz_bf16) cudaFuncSetAttribute(k_mlp_fp8<__nv_bfloat16>, at, (int)smem);
  else cudaFuncSetAttribute(k_mlp_fp8<float>, at, (int)smem);
}

void launch_mlp_fp8(const MlpTcArgs &a, cudaStream_t st, long &launches) {
  if (a.ntiles <= 0) return;
  if (a.dz_bf16) k_mlp_fp8<__nv_bfloat16><<<a.ntiles, TM, a.smem, st>>>(a);
  else k_mlp_fp8<float><<<a.ntiles, TM, a.smem, st>>>(a);
  launches += 1;
}

}  // namespace tmd
