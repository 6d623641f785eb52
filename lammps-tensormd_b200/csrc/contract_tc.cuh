// contract_tc.cuh -- pieces of the warp-per-atom descriptor and force kernels
// that run the per-atom contractions on the tensor cores (mma.sync m16n8k8,
// TF32 operands split into hi + lo, three products: FP32-class accuracy).
//
// A warp owns one atom.  Its lanes compute the FP64 geometry of 32 list
// entries at a time and queue the active pairs (r < rc) in a shared-memory
// ring; every radial value and monomial of a pair is then computed once, by
// the lane whose MMA fragment holds it, and the contractions
//   P[k][d] = sum_pairs H_k M_d                 (descriptor)
//   V[pair][d] = sum_k H_k S[k][d], W[pair][d] = sum_k dH_k S[k][d]   (force)
// run as MMAs over chunks of pairs.  Fragment layout of m16n8k8 (TF32): with
// g = lane / 4 and q = lane % 4, A holds (g, q), (g+8, q), (g, q+4),
// (g+8, q+4); B holds (q, g), (q+4, g); C holds (g, 2q), (g, 2q+1),
// (g+8, 2q), (g+8, 2q+1).
#pragma once

#include "descriptor_impl.cuh"

namespace tmd {
namespace ctc {

// Radial parameters of one filter k (k >= K: a padding filter, H = 0).
template <int RK>
struct RadialF {
  float a, b, c, blo, gc;
  int k;
};

template <int RK>
__device__ inline RadialF<RK> load_radial1(const KParams &kp, int k) {
  RadialF<RK> R{0.f, 0.f, 0.f, 0.f, 0.f, k};
  if (k >= kp.K) return R;
  if (RK == kRadGeneric) { R.a = kp.p0[k]; R.c = kp.p2[k]; }
  if (RK != kRadTable) R.b = kp.p1[k];
  if (RK == kRadGauss) { R.blo = kp.p1lo[k]; R.gc = kp.gc[k]; }
  return R;
}

// H_k(r) and dH_k/dr of one filter: the per-filter form of radial4.
template <int RK, bool DERIV>
__device__ inline void radial1(const KParams &kp, const RadialF<RK> &R, const PairGeo &g,
                               float &H, float &dH) {
  H = 0.f;
  if (DERIV) dH = 0.f;
  if (R.k >= kp.K || g.ti < 0) return;
  if (RK == kRadTable) {
    if (g.ti <= 0 || g.ti >= kp.tab_n - 2) return;
    const int K = kp.K;
    const float *row = kp.table + (size_t)g.ti * 4 * K;
    const float y = __ldg(row + R.k), s = __ldg(row + K + R.k);
    const float c1 = __ldg(row + 2 * K + R.k), c2 = __ldg(row + 3 * K + R.k);
    const float q = g.tq, dx = kp.tab_dx, rr = dx - q;
    float c3 = fabsf(c2 * rr);
    float c4 = c3 + fabsf(c1 * q);
    if (c4 > 0.f) c3 /= c4;
    c4 = c2 + c3 * (c1 - c2);
    H = y + q * (s - rr * c4);
    if (DERIV) dH = s + (q - rr) * c4 + dx * (c4 - c2) * (1.f - c3);
    return;
  }
  const float r = g.r;
  float f, df;
  if (RK == kRadGauss) {
    const float d = (r - R.b) + (g.rlo - R.blo);
    f = expf(-R.gc * d * d);
    df = -2.f * R.gc * d * f;
  } else {
    if (kp.method == 0) {
      const float xr = r / R.a;
      f = expf(-powf(xr, R.b));
      df = -f * R.b * powf(xr, R.b - 1.f) / R.a;
    } else if (kp.method == 1) {
      const float gdr = R.b * (r - R.c);
      const float e1 = expf(-gdr), e2 = expf(-2.f * gdr);
      f = R.a * (e2 - 2.f * e1);
      df = -R.a * R.b * 2.f * (e2 - e1);
    } else {
      f = R.a * expf(-R.b * ((r - R.c) / R.c));
      df = -f * R.b / R.c;
    }
  }
  H = g.fc * f;
  if (DERIV) dH = g.dfc * f + g.fc * df;
}

// Exponents (a, b, c) of monomial d = x^a y^b z^c in the order of
// kernel.cu:1197-1232 (1, x, y, z, xx, xy, xz, yy, yz, zz, xxx, xxy, xxz,
// xyy, xyz, xzz, yyy, yyz, yzz, zzz), packed a | b << 2 | c << 4; d >= D
// gives -1 (a padding column).
__device__ inline int mono_exp(int d, int D) {
  if (d >= D) return -1;
  constexpr unsigned char e[20] = {0x00, 0x01, 0x04, 0x10, 0x02, 0x05, 0x11, 0x08, 0x14, 0x20,
                                   0x03, 0x06, 0x12, 0x09, 0x15, 0x21, 0x0C, 0x18, 0x24, 0x30};
  int v = 0;
#pragma unroll
  for (int i = 0; i < 20; i++) v = (i == d) ? e[i] : v;
  return v;
}

__device__ inline float ipow(float x, int n) {
  return n == 0 ? 1.f : (n == 1 ? x : (n == 2 ? x * x : x * x * x));
}

// M_d(u) for packed exponents e (0 for a padding column).
__device__ inline float mono(int e, float x, float y, float z) {
  if (e < 0) return 0.f;
  return ipow(x, e & 3) * ipow(y, (e >> 2) & 3) * ipow(z, e >> 4);
}

// grad_u M_d and rank n_d of monomial e (zeros for a padding column).
__device__ inline void mono_grad(int e, float x, float y, float z, float &gx, float &gy,
                                 float &gz, float &rank) {
  gx = gy = gz = rank = 0.f;
  if (e < 0) return;
  const int a = e & 3, b = (e >> 2) & 3, c = e >> 4;
  const float px = ipow(x, a), py = ipow(y, b), pz = ipow(z, c);
  if (a) gx = a * ipow(x, a - 1) * py * pz;
  if (b) gy = b * px * ipow(y, b - 1) * pz;
  if (c) gz = c * px * py * ipow(z, c - 1);
  rank = (float)(a + b + c);
}

__device__ inline void split_tf32(float v, uint32_t &hi, uint32_t &lo) {
  uint32_t h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(v));
  const float r = v - __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(r));
  hi = h;
  lo = l;
}

__device__ inline void mma_tf32(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// C += A . B with A and B split: lo*hi + hi*lo + hi*hi (small terms first).
__device__ inline void mma3(float c[4], const uint32_t ah[4], const uint32_t al[4],
                            uint32_t bh0, uint32_t bh1, uint32_t bl0, uint32_t bl1) {
  mma_tf32(c, al[0], al[1], al[2], al[3], bh0, bh1);
  mma_tf32(c, ah[0], ah[1], ah[2], ah[3], bl0, bl1);
  mma_tf32(c, ah[0], ah[1], ah[2], ah[3], bh0, bh1);
}

// Ring of active pairs of the current atom and element block, per warp.
constexpr int kRing = 64;

struct WarpRing {
  GeoSlot *ring;
  int lane, head, qn, t, s1;

  __device__ inline GeoSlot *slot(int c) const { return ring + ((head + c) & (kRing - 1)); }

  // Queue entries until >= want pairs are waiting or the block's row ends;
  // inactive entries get a zero pdf slot when pdf_row is given.
  __device__ inline int feed(const KParams &kp, const BoxP &box, double xi, double yi, double zi,
                             const double *__restrict__ x, const uint32_t *__restrict__ row,
                             float4 *__restrict__ pdf_row, int want) {
    while (qn < want && t < s1) {
      const bool valid = t + lane < s1;
      const NbPos p = load_nb(x, valid ? row[t + lane] : 0u, valid);
      PairGeo g;
      pair_geometry(kp, box, xi, yi, zi, p, g);
      const bool act = g.ti >= 0;
      const unsigned bal = __ballot_sync(0xffffffffu, act);
      if (act) geo_store(slot(qn + __popc(bal & ((1u << lane) - 1u))), g, t + lane);
      else if (pdf_row != nullptr && valid) pdf_row[t + lane] = make_float4(0.f, 0.f, 0.f, 0.f);
      qn += __popc(bal);
      t += 32;
    }
    __syncwarp();
    return min(qn, want);
  }
  __device__ inline void pop(int cnt) {
    __syncwarp();
    head = (head + cnt) & (kRing - 1);
    qn -= cnt;
  }
};

__device__ inline PairGeo geo_or_zero(const WarpRing &w, int c, int cnt) {
  if (c < cnt) return geo_load(w.slot(c));
  PairGeo g;
  g.r = 1.f; g.rlo = g.ux = g.uy = g.uz = g.fc = g.dfc = g.tq = 0.f;
  g.ti = -1;
  return g;
}

}  // namespace ctc
}  // namespace tmd
