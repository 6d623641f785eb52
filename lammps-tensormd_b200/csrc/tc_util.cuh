// tc_util.cuh -- tcgen05 (sm_100a) helpers shared by the tensor-core MLP
// kernels: shared-memory matrix descriptors, MMA commit, bounded mbarrier
// wait, TMEM loads, and the activations of nnp.cu:9-57.
#pragma once

#include <cstdint>

namespace tmd {
namespace tc {

constexpr int TM = 128;      // atoms per tile (MMA M)
constexpr int KCH = 64;      // reduction chunk (columns) staged at a time
constexpr int TMEM_COLS = 128;
constexpr long long kWaitCycles = 4000000000LL;  // about 2 s

__device__ inline uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// K-major, no-swizzle shared-memory matrix descriptor (sm_100 format:
// start >> 4 [0,14), LBO >> 4 [16,30), SBO >> 4 [32,46), version 1 [46,48),
// layout SWIZZLE_NONE [61,64) = 0).  Core matrices are 8 rows x 16 bytes;
// LBO = distance between the two core columns of one MMA K step, SBO =
// distance between 8-row groups.
__device__ inline uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

__device__ inline void commit(uint64_t *mbar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(mbar)));
}

// Bounded wait for the mbarrier phase; false on timeout (after `limit`
// clock cycles).
__device__ inline bool mbar_wait(uint64_t *mbar, uint32_t phase, long long limit = kWaitCycles) {
  const uint32_t a = smem_u32(mbar);
  const long long t0 = clock64();
  while (true) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(a), "r"(phase)
        : "memory");
    if (ok) return true;
    if (clock64() - t0 > limit) return false;
  }
}

// Global -> shared bulk copy (no multicast) completing on mbarrier `bar`;
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ inline void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
      "[%3];" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Arrive on `bar` and add `bytes` to the transaction count of its phase.
__device__ inline void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ inline void tmem_ld32(uint32_t taddr, float v[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// Activation and its derivative (nnp.cu:9-57; squareplus without the FP32
// cancellation for z < 0).
__device__ inline float act_fwd(int actfn, float z, float &d) {
  switch (actfn) {
    case 0:
      d = z > 0.f ? 1.f : 0.f;
      return z > 0.f ? z : 0.f;
    case 1: {
      float ex = expf(z);
      d = 1.f / (1.f + 1.f / ex);
      return z < 13.942385152878742f ? log1pf(ex) : z;
    }
    case 2: {
      // sech^2 z = 4 e / (1 + e)^2, e = exp(-2|z|): no 1 - tanh^2 cancellation
      const float e = expf(-2.f * fabsf(z));
      const float u = 1.f + e;
      d = 4.f * e / (u * u);
      return tanhf(z);
    }
    default: {
      float q = sqrtf(z * z + 4.f);
      float y = z >= 0.f ? 0.5f * (z + q) : 2.f / (q - z);
      d = y / q;
      return y;
    }
  }
}

// The same activations from fast intrinsics (__expf, __logf, __frcp_rn),
// for the tensor-core forms whose operands are BF16: absolute errors of a
// few 1e-7, far below the operand rounding.  Where a closed form loses
// relative accuracy the Taylor series takes over: log(1 + e) = e - e^2/2 +
// e^3/3 for e < 1e-3 (softplus of z < -6.9), tanh a = a - a^3/3 for a <
// 4e-3.  Same thresholds as act_fwd for the large-argument branches.
__device__ inline float act_fwd_fast(int actfn, float z, float &d) {
  switch (actfn) {
    case 0:
      d = z > 0.f ? 1.f : 0.f;
      return z > 0.f ? z : 0.f;
    case 1: {
      const float ex = __expf(fminf(z, 80.f));
      d = ex * __frcp_rn(1.f + ex);
      const float lg = ex < 1e-3f ? ex * (1.f - ex * (0.5f - ex * (1.f / 3.f)))
                                  : __logf(1.f + ex);
      return z < 13.942385152878742f ? lg : z;
    }
    case 2: {
      const float a = fabsf(z);
      const float t = __expf(-2.f * fminf(a, 40.f));
      const float y0 = a < 4e-3f ? a - a * a * a * (1.f / 3.f) : (1.f - t) * __frcp_rn(1.f + t);
      const float y = copysignf(y0, z);
      const float u = 1.f + t;
      d = 4.f * t * __frcp_rn(u * u);  // sech^2 z without 1 - tanh^2 cancellation
      return y;
    }
    default: {
      const float q = sqrtf(z * z + 4.f);
      const float y = z >= 0.f ? 0.5f * (z + q) : 2.f * __frcp_rn(q - z);
      d = y * __frcp_rn(q);
      return y;
    }
  }
}

// element offset of (r, k) in a K-major core-matrix operand with kfull
// columns and epc elements per 16-byte core row
template <int EPC>
__device__ __host__ inline int core_off(int r, int k, int kfull) {
  return ((r >> 3) * (kfull / EPC) + k / EPC) * (8 * EPC) + (r & 7) * EPC + (k % EPC);
}

}  // namespace tc
}  // namespace tmd
