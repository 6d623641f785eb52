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
// FMAs (sm_100 FFMA2).  Each lane computes the FP64 geometry of one entry of
// a chunk of TPA neighbors; the active pairs (r < rc) are queued in shared
// memory (PairRing) and the group reads each pair with vector loads
// (broadcast).  Neighbor entries are fetched two chunks ahead and neighbor
// positions one chunk ahead, so the gather latency overlaps the arithmetic.
// Nothing per pair goes to global memory.
//
// Output layout: P[n][B][K][D] (kept for the force kernel), then
// k_invariants forms G[n][B*K*M] (the MLP input rows, m fastest, as
// TensorMD::get_G) from P.
#pragma once

#include "pair_math.cuh"
#include "tmd_kernels.h"

namespace tmd {

constexpr int kPairThreads = 128;  // block size of the pair kernels

// Geometry slot in shared memory: three 16-byte vectors per lane; the inputs
// of the radial basis (r, r_lo, f_c, table offset) share the first, so the
// per-pair radial of the descriptor reads one vector.
struct GeoSlot {
  float4 a;  // r, rlo, fc, tq
  float4 b;  // ux, uy, uz, dfc
  float4 c;  // ti (bits), neighbor slot t (bits), 1/r, unused
};

__device__ inline void geo_store(GeoSlot *s, const PairGeo &g, int t) {
  s->a = make_float4(g.r, g.rlo, g.fc, g.tq);
  s->b = make_float4(g.ux, g.uy, g.uz, g.dfc);
  s->c = make_float4(__int_as_float(g.ti), __int_as_float(t), g.rinv, 0.f);
}

__device__ inline PairGeo geo_load(const GeoSlot *s) {
  PairGeo g;
  float4 a = s->a, b = s->b;
  g.r = a.x; g.rlo = a.y; g.fc = a.z; g.tq = a.w;
  g.ux = b.x; g.uy = b.y; g.uz = b.z; g.dfc = b.w;
  const float4 c = s->c;
  g.ti = __float_as_int(c.x);
  g.rinv = c.z;
  return g;
}

// The fields of a slot that the radial basis reads (r, r_lo, f_c for the
// analytic kinds; interval and offset for the table).
template <int RK>
__device__ inline PairGeo geo_load_radial(const GeoSlot *s) {
  PairGeo g;
  g.ux = g.uy = g.uz = g.dfc = g.rinv = 0.f;
  if (RK == kRadTable) {
    g.r = g.rlo = g.fc = 0.f;
    g.tq = s->a.w;
    g.ti = __float_as_int(s->c.x);
  } else {
    const float4 a = s->a;
    g.r = a.x; g.rlo = a.y;
    g.fc = a.z;
    g.tq = 0.f;
    g.ti = 0;
  }
  return g;
}

// Lanes of thread gt's warp whose global thread index is below nthreads
// (threads past the last atom return at kernel entry).
__device__ inline unsigned live_lanes(int gt, long nthreads) {
  const long rem = nthreads - (long)(gt & ~31);
  return rem >= 32 ? 0xffffffffu : ((1u << rem) - 1u);
}

// Box of atom a: the system's box, or in multi-cell mode the box of a's cell.
template <bool MULTI>
__device__ inline const BoxP &box_of(const BoxP &box, const BoxP *__restrict__ cbox,
                                     const int *__restrict__ acell, int a) {
  if constexpr (MULTI) return cbox[acell[a]];
  else return box;
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

// The active pairs of one atom's row, TPA at a time.  About 40% of a row
// lies in the skin shell (rc < r < rc + skin) and rows are sorted by image
// and index, not by distance, so active pairs are scattered along the row.
// Each group therefore keeps a ring of 2*TPA geometry slots in shared memory:
// feed() computes the geometry of the next TPA entries (one per lane) and
// appends the active ones in row order (ballot + prefix count) until the ring
// holds TPA pairs or the row ends.  The group then runs its per-pair work on
// exactly TPA pairs, and a warp's groups stay converged on full chunks
// instead of idling on other groups' inactive entries.
template <int TPA>
struct PairRing {
  static constexpr int kSlots = 2 * TPA;
  static constexpr unsigned kBits = TPA == 32 ? 0xffffffffu : ((1u << TPA) - 1u);
  GeoSlot *ring;        // this group's 2*TPA slots
  unsigned gmask;       // this group's lanes in the warp
  int gshift, sub;      // first lane of the group, lane within the group
  int head, qn;         // ring head and number of queued pairs
  int t, s1;            // next row entry to fetch, end of the block's entries
  NbPos pnext;          // positions of entries t..t+TPA-1 (one per lane)
  uint32_t enext;       // packed entries t+TPA..t+2TPA-1

  __device__ inline void begin(const double *__restrict__ x,
                               const uint32_t *__restrict__ row, int s0, int s1_) {
    head = 0; qn = 0; t = s0; s1 = s1_;
    pnext = load_nb(x, s0 + sub < s1 ? row[s0 + sub] : 0u, s0 + sub < s1);
    enext = (s0 + TPA + sub < s1) ? row[s0 + TPA + sub] : 0u;
  }
  __device__ inline GeoSlot *slot(int c) const { return ring + ((head + c) & (kSlots - 1)); }

  // Fill the ring to >= TPA pairs (or the end of the row); returns the number
  // of pairs in the next chunk.  When pdf_row is given, each inactive entry's
  // pdf slot is written as zero here.
  __device__ inline int feed(const KParams &kp, const BoxP &box, double xi, double yi,
                             double zi, const double *__restrict__ x,
                             const uint32_t *__restrict__ row, float4 *__restrict__ pdf_row) {
    return feed_with(kp, box, xi, yi, zi, x, row, pdf_row, [](int, const PairGeo &) {});
  }
  // As feed; extra(slot index, geometry) runs for every queued pair, on the
  // lane that computed it (per-pair data kept beside the ring).
  template <class Extra>
  __device__ inline int feed_with(const KParams &kp, const BoxP &box, double xi, double yi,
                                  double zi, const double *__restrict__ x,
                                  const uint32_t *__restrict__ row,
                                  float4 *__restrict__ pdf_row, Extra extra) {
    while (qn < TPA && t < s1) {
      const NbPos pc = pnext;
      pnext = load_nb(x, enext, t + TPA + sub < s1);
      enext = (t + 2 * TPA + sub < s1) ? row[t + 2 * TPA + sub] : 0u;
      PairGeo g;
      pair_geometry(kp, box, xi, yi, zi, pc, g);
      const bool act = g.ti >= 0;
      const unsigned bal = (__ballot_sync(gmask, act) >> gshift) & kBits;
      if (act) {
        const int c = qn + __popc(bal & ((1u << sub) - 1u));
        geo_store(slot(c), g, t + sub);
        extra((head + c) & (kSlots - 1), g);
      } else if (pdf_row != nullptr && t + sub < s1)
        pdf_row[t + sub] = make_float4(0.f, 0.f, 0.f, 0.f);
      qn += __popc(bal);
      t += TPA;
    }
    __syncwarp(gmask);
    return min(qn, TPA);
  }
  // Drop the chunk just processed (after every lane has read its slots).
  __device__ inline void pop(int cnt) {
    __syncwarp(gmask);
    head = (head + cnt) & (kSlots - 1);
    qn -= cnt;
  }
};

// Compact geometry of an active pair, written by the descriptor kernels for
// the pair-lane force kernel (two float4: r, rlo, ux, uy | uz, fc, dfc, t for
// analytic radial kinds; uz, tq, ti, t for the table), so that the force
// kernel reads the active pairs instead of testing every list entry again.
template <int RK>
__device__ inline void store_pair_geo(const GeoSlot *s, float4 *__restrict__ dst) {
  const float4 a = s->a, b = s->b, c = s->c;
  dst[0] = make_float4(a.x, a.y, b.x, b.y);
  dst[1] = RK == kRadTable ? make_float4(b.z, a.w, c.x, c.y) : make_float4(b.z, a.z, b.w, c.y);
}

template <int RK>
__device__ inline PairGeo decode_pair_geo(const float4 a, const float4 b, int &t) {
  PairGeo g;
  g.r = a.x; g.rlo = a.y; g.ux = a.z; g.uy = a.w; g.uz = b.x;
  if (RK == kRadTable) {
    g.tq = b.y; g.ti = __float_as_int(b.z); g.fc = g.dfc = 0.f;
  } else {
    g.fc = b.y; g.dfc = b.z; g.ti = 0; g.tq = 0.f;
  }
  t = __float_as_int(b.w);
  g.rinv = __frcp_rn(g.r);  // 1/r rounded to nearest, as pair_geometry
  return g;
}

template <int RK>
__device__ inline PairGeo load_pair_geo(const float4 *__restrict__ src, int &t) {
  return decode_pair_geo<RK>(__ldg(src), __ldg(src + 1), t);
}

template <int TPA, int D, int RK, bool MULTI>
__global__ void __launch_bounds__(kPairThreads, 4)
k_descriptor(KParams kp, BoxP box, int n, int cap, const double *__restrict__ x,
             const int *__restrict__ elem, const uint32_t *__restrict__ nbr,
             const int *__restrict__ boff, float *__restrict__ P,
             float *__restrict__ G, const BoxP *__restrict__ cbox,
             const int *__restrict__ acell, float4 *__restrict__ pdf,
             float4 *__restrict__ pgeo, int *__restrict__ pcnt) {
  constexpr int D2 = (D + 1) / 2;
  __shared__ GeoSlot geo[2 * kPairThreads + kPairThreads];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt / TPA;
  const int sub = gt % TPA;
  if (a >= n) return;
  const int lane = threadIdx.x & 31;
  PairRing<TPA> pr;
  pr.sub = sub;
  pr.gshift = lane & ~(TPA - 1);
  pr.gmask = PairRing<TPA>::kBits << pr.gshift;
  // the ring of this atom's group; one spare slot per group puts the groups
  // of a warp in different banks (their reads of slot c do not conflict)
  pr.ring = geo + 2 * (threadIdx.x - sub) + threadIdx.x / TPA;
  const int B = kp.B, K = kp.K;
  const int k0 = 4 * sub;
  const Radial4<RK> R = load_radial4<RK>(kp, k0);
  const BoxP &bx = box_of<MULTI>(box, cbox, acell, a);
  const double xi = x[3 * a], yi = x[3 * a + 1], zi = x[3 * a + 2];
  const uint32_t *row = nbr + (size_t)a * cap;
  const int *bo = boff + (size_t)a * (B + 1);
  const unsigned live = live_lanes(gt, (long)n * TPA);
  float4 *pdf_row = pdf + (size_t)a * cap;
  float4 *pg_row = pgeo + (size_t)a * cap * 2;
  int nact = 0;
  for (int b = 0; b < B; b++) {
    // keep the warp's groups on the same element block (see k_force)
    if (b > 0) __syncwarp(live);
    const int nact0 = nact;
    float2 acc[4][D2];
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
      for (int p = 0; p < D2; p++) acc[q][p] = make_float2(0.f, 0.f);
    pr.begin(x, row, bo[b], bo[b + 1]);
    for (;;) {
      const int cnt = pr.feed(kp, bx, xi, yi, zi, x, row, pdf_row);
      if (cnt == 0) break;
      if (sub < cnt) store_pair_geo<RK>(pr.slot(sub), pg_row + 2 * (nact + sub));
      nact += cnt;
      for (int c = 0; c < cnt; c++) {
        const PairGeo g = geo_load(pr.slot(c));
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
      pr.pop(cnt);
    }
    if (sub == 0) pcnt[(size_t)a * B + b] = nact - nact0;
    // P rows of this lane: 4 filters x D values, contiguous (G = T P^2 is
    // formed by k_invariants)
    float *Pp = P + (((size_t)a * B + b) * K + k0) * D;
    if constexpr (D % 2 == 0) {
      float2 *P2 = reinterpret_cast<float2 *>(Pp);
#pragma unroll
      for (int q = 0; q < 4; q++)
#pragma unroll
        for (int p = 0; p < D2; p++) P2[q * D2 + p] = acc[q][p];
    } else {
#pragma unroll
      for (int q = 0; q < 4; q++)
#pragma unroll
        for (int d = 0; d < D; d++) Pp[q * D + d] = (d & 1) ? acc[q][d >> 1].y : acc[q][d >> 1].x;
    }
  }
}

// Wide-group form: W = min(K, 32) lanes per atom, FPL = K / W filters per
// lane.  With K = 16 the 4-filter form packs 8 atoms into a warp whose groups
// fetch, test and queue their rows at different rates, so much of the warp
// idles; here a warp holds one or two atoms.  The lane that computes a pair's
// geometry also computes its D monomials once and keeps them beside the ring
// slot; every lane then reads them as broadcast vectors and accumulates
// P[k][d] for its own filters in the same order (pairs in row order, FP32
// pairs over d) as k_descriptor, then forms its filters' G rows from the P
// rows it holds (no k_invariants pass).
template <int W, int FPL, int D, int RK, bool MULTI>
__global__ void __launch_bounds__(kPairThreads, 6)
k_descriptor_w(KParams kp, BoxP box, int n, int cap, const double *__restrict__ x,
               const uint32_t *__restrict__ nbr, const int *__restrict__ boff,
               float *__restrict__ P, float *__restrict__ G,
               const BoxP *__restrict__ cbox,
               const int *__restrict__ acell, float4 *__restrict__ pdf,
               float4 *__restrict__ pgeo, int *__restrict__ pcnt) {
  constexpr int D4 = (D + 3) / 4 * 4;
  constexpr int M = D == 1 ? 1 : (D == 4 ? 2 : (D == 10 ? 3 : 4));
  constexpr int P2 = D4 / 2;
  __shared__ GeoSlot geo[2 * kPairThreads + kPairThreads / 4];
  __shared__ __align__(16) float mono[2 * kPairThreads * D4 + kPairThreads];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt / W;
  const int sub = gt % W;
  if (a >= n) return;
  const int lane = threadIdx.x & 31;
  PairRing<W> pr;
  pr.sub = sub;
  pr.gshift = lane & ~(W - 1);
  pr.gmask = PairRing<W>::kBits << pr.gshift;
  // the group's ring and monomial slots, each group offset by one spare slot
  // (12 words) and 4 words so that the groups of a warp read different banks
  pr.ring = geo + 2 * (threadIdx.x - sub) + threadIdx.x / W;
  float *mr = mono + 2 * (threadIdx.x - sub) * D4 + 4 * (threadIdx.x / W);
  const int B = kp.B, K = kp.K;
  const int kf = sub * FPL;
  Radial1<RK> R[FPL];
#pragma unroll
  for (int f = 0; f < FPL; f++) R[f] = load_radial1<RK>(kp, kf + f);
  const BoxP &bx = box_of<MULTI>(box, cbox, acell, a);
  const double xi = x[3 * a], yi = x[3 * a + 1], zi = x[3 * a + 2];
  const uint32_t *row = nbr + (size_t)a * cap;
  const int *bo = boff + (size_t)a * (B + 1);
  const unsigned live = live_lanes(gt, (long)n * W);
  auto keep_monomials = [&](int idx, const PairGeo &g) {
    float M[D4];
    moments<D>(g.ux, g.uy, g.uz, M);
#pragma unroll
    for (int d = D; d < D4; d++) M[d] = 0.f;
    float4 *dst = reinterpret_cast<float4 *>(mr + idx * D4);
#pragma unroll
    for (int v = 0; v < D4 / 4; v++)
      dst[v] = make_float4(M[4 * v], M[4 * v + 1], M[4 * v + 2], M[4 * v + 3]);
  };
  float4 *pdf_row = pdf + (size_t)a * cap;
  float4 *pg_row = pgeo + (size_t)a * cap * 2;
  int nact = 0;
  for (int b = 0; b < B; b++) {
    if (b > 0) __syncwarp(live);
    const int nact0 = nact;
    float2 acc[FPL][P2];
#pragma unroll
    for (int f = 0; f < FPL; f++)
#pragma unroll
      for (int p = 0; p < P2; p++) acc[f][p] = make_float2(0.f, 0.f);
    pr.begin(x, row, bo[b], bo[b + 1]);
    for (;;) {
      const int cnt = pr.feed_with(kp, bx, xi, yi, zi, x, row, pdf_row, keep_monomials);
      if (cnt == 0) break;
      if (sub < cnt) store_pair_geo<RK>(pr.slot(sub), pg_row + 2 * (nact + sub));
      nact += cnt;
#pragma unroll 2
      for (int c = 0; c < cnt; c++) {
        const PairGeo g = geo_load_radial<RK>(pr.slot(c));
        const float4 *ms = reinterpret_cast<const float4 *>(
            mr + ((pr.head + c) & (PairRing<W>::kSlots - 1)) * D4);
        float2 h2[FPL];
#pragma unroll
        for (int f = 0; f < FPL; f++) {
          const float h = radial1<RK>(kp, R[f], g);
          h2[f] = make_float2(h, h);
        }
#pragma unroll
        for (int v = 0; v < D4 / 4; v++) {
          const float4 m4 = ms[v];
          const float2 lo = make_float2(m4.x, m4.y), hi = make_float2(m4.z, m4.w);
#pragma unroll
          for (int f = 0; f < FPL; f++) {
            acc[f][2 * v] = __ffma2_rn(h2[f], lo, acc[f][2 * v]);
            acc[f][2 * v + 1] = __ffma2_rn(h2[f], hi, acc[f][2 * v + 1]);
          }
        }
      }
      pr.pop(cnt);
    }
    if (sub == 0) pcnt[(size_t)a * B + b] = nact - nact0;
    float *Pp = P + (((size_t)a * B + b) * K + kf) * D;
    float *Gp = G + (((size_t)a * B + b) * K + kf) * M;
#pragma unroll
    for (int f = 0; f < FPL; f++) {
      if constexpr (D % 2 == 0) {
        float2 *P2p = reinterpret_cast<float2 *>(Pp + f * D);
#pragma unroll
        for (int p = 0; p < D / 2; p++) P2p[p] = acc[f][p];
      } else {
#pragma unroll
        for (int d = 0; d < D; d++) Pp[f * D + d] = (d & 1) ? acc[f][d >> 1].y : acc[f][d >> 1].x;
      }
      // G row of the filter, in the order of k_invariants
#pragma unroll
      for (int m = 0; m < M; m++) {
        float s = 0.f;
#pragma unroll
        for (int d = 0; d < D; d++) {
          const float pv = (d & 1) ? acc[f][d >> 1].y : acc[f][d >> 1].x;
          s = fmaf(kp.T[m * D + d], pv * pv, s);
        }
        if (m == 0) s = copysignf(1.f, acc[f][0].x) * sqrtf(s);
        Gp[f * M + m] = s;
      }
    }
  }
}

// Two-stream wide form: W lanes per atom as two pair streams of FL = W/2
// lanes, FPL = K/FL filters per lane.  The geometry ring is k_descriptor_w's;
// of each chunk of queued pairs, stream 0 takes the even and stream 1 the odd
// ones, so every monomial vector read from shared memory feeds 2 * FPL packed
// FMAs instead of 2 (the read and the radial of a pair are shared by more
// filters per lane) while a warp still holds W = min(K, 32) lanes per atom.
// The streams' partial P are added (stream 0 + stream 1) by a shuffle at the
// end of each element block; each stream then forms and writes half of the
// lane's filters' P and G rows.
template <int W, int FPL, int D, int RK, bool MULTI>
__global__ void __launch_bounds__(kPairThreads, 4)
k_descriptor_w2(KParams kp, BoxP box, int n, int cap, const double *__restrict__ x,
                const uint32_t *__restrict__ nbr, const int *__restrict__ boff,
                float *__restrict__ P, float *__restrict__ G,
                const BoxP *__restrict__ cbox,
                const int *__restrict__ acell, float4 *__restrict__ pdf,
                float4 *__restrict__ pgeo, int *__restrict__ pcnt) {
  constexpr int FL = W / 2;
  constexpr int D4 = (D + 3) / 4 * 4;
  constexpr int M = D == 1 ? 1 : (D == 4 ? 2 : (D == 10 ? 3 : 4));
  constexpr int P2 = D4 / 2;
  __shared__ GeoSlot geo[2 * kPairThreads + kPairThreads / 4];
  __shared__ __align__(16) float mono[2 * kPairThreads * D4 + kPairThreads];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt / W;
  const int sub = gt % W;
  if (a >= n) return;
  const int lane = threadIdx.x & 31;
  const int stream = sub / FL, fl = sub % FL;
  PairRing<W> pr;
  pr.sub = sub;
  pr.gshift = lane & ~(W - 1);
  pr.gmask = PairRing<W>::kBits << pr.gshift;
  // the group's ring and monomial slots, each group offset by one spare slot
  // (12 words) and 4 words so that the groups of a warp read different banks
  pr.ring = geo + 2 * (threadIdx.x - sub) + threadIdx.x / W;
  float *mr = mono + 2 * (threadIdx.x - sub) * D4 + 4 * (threadIdx.x / W);
  const int B = kp.B, K = kp.K;
  const int kf = fl * FPL;
  Radial1<RK> R[FPL];
#pragma unroll
  for (int f = 0; f < FPL; f++) R[f] = load_radial1<RK>(kp, kf + f);
  const BoxP &bx = box_of<MULTI>(box, cbox, acell, a);
  const double xi = x[3 * a], yi = x[3 * a + 1], zi = x[3 * a + 2];
  const uint32_t *row = nbr + (size_t)a * cap;
  const int *bo = boff + (size_t)a * (B + 1);
  const unsigned live = live_lanes(gt, (long)n * W);
  auto keep_monomials = [&](int idx, const PairGeo &g) {
    float Mv[D4];
    moments<D>(g.ux, g.uy, g.uz, Mv);
#pragma unroll
    for (int d = D; d < D4; d++) Mv[d] = 0.f;
    float4 *dst = reinterpret_cast<float4 *>(mr + idx * D4);
#pragma unroll
    for (int v = 0; v < D4 / 4; v++)
      dst[v] = make_float4(Mv[4 * v], Mv[4 * v + 1], Mv[4 * v + 2], Mv[4 * v + 3]);
  };
  float4 *pdf_row = pdf + (size_t)a * cap;
  float4 *pg_row = pgeo + (size_t)a * cap * 2;
  int nact = 0;
  for (int b = 0; b < B; b++) {
    if (b > 0) __syncwarp(live);
    const int nact0 = nact;
    float2 acc[FPL][P2];
#pragma unroll
    for (int f = 0; f < FPL; f++)
#pragma unroll
      for (int p = 0; p < P2; p++) acc[f][p] = make_float2(0.f, 0.f);
    pr.begin(x, row, bo[b], bo[b + 1]);
    for (;;) {
      const int cnt = pr.feed_with(kp, bx, xi, yi, zi, x, row, pdf_row, keep_monomials);
      if (cnt == 0) break;
      if (sub < cnt) store_pair_geo<RK>(pr.slot(sub), pg_row + 2 * (nact + sub));
      nact += cnt;
      for (int c = stream; c < cnt; c += 2) {
        const PairGeo g = geo_load_radial<RK>(pr.slot(c));
        const float4 *ms = reinterpret_cast<const float4 *>(
            mr + ((pr.head + c) & (PairRing<W>::kSlots - 1)) * D4);
        float2 h2[FPL];
#pragma unroll
        for (int f = 0; f < FPL; f++) {
          const float h = radial1<RK>(kp, R[f], g);
          h2[f] = make_float2(h, h);
        }
#pragma unroll
        for (int v = 0; v < D4 / 4; v++) {
          const float4 m4 = ms[v];
          const float2 lo = make_float2(m4.x, m4.y), hi = make_float2(m4.z, m4.w);
#pragma unroll
          for (int f = 0; f < FPL; f++) {
            acc[f][2 * v] = __ffma2_rn(h2[f], lo, acc[f][2 * v]);
            acc[f][2 * v + 1] = __ffma2_rn(h2[f], hi, acc[f][2 * v + 1]);
          }
        }
      }
      pr.pop(cnt);
    }
    if (sub == 0) pcnt[(size_t)a * B + b] = nact - nact0;
    // P = stream 0 + stream 1 (both streams hold the sum afterwards)
#pragma unroll
    for (int f = 0; f < FPL; f++)
#pragma unroll
      for (int p = 0; p < P2; p++) {
        const float ox = __shfl_xor_sync(pr.gmask, acc[f][p].x, FL, W);
        const float oy = __shfl_xor_sync(pr.gmask, acc[f][p].y, FL, W);
        acc[f][p] = stream == 0 ? make_float2(acc[f][p].x + ox, acc[f][p].y + oy)
                                : make_float2(ox + acc[f][p].x, oy + acc[f][p].y);
      }
    float *Pp = P + (((size_t)a * B + b) * K + kf) * D;
    float *Gp = G + (((size_t)a * B + b) * K + kf) * M;
#pragma unroll
    for (int f = 0; f < FPL; f++) {
      if ((f & 1) != stream) continue;  // each stream writes half the filters
      if constexpr (D % 2 == 0) {
        float2 *P2p = reinterpret_cast<float2 *>(Pp + f * D);
#pragma unroll
        for (int p = 0; p < D / 2; p++) P2p[p] = acc[f][p];
      } else {
#pragma unroll
        for (int d = 0; d < D; d++) Pp[f * D + d] = (d & 1) ? acc[f][d >> 1].y : acc[f][d >> 1].x;
      }
#pragma unroll
      for (int m = 0; m < M; m++) {
        float sacc = 0.f;
#pragma unroll
        for (int d = 0; d < D; d++) {
          const float pv = (d & 1) ? acc[f][d >> 1].y : acc[f][d >> 1].x;
          sacc = fmaf(kp.T[m * D + d], pv * pv, sacc);
        }
        if (m == 0) sacc = copysignf(1.f, acc[f][0].x) * sqrtf(sacc);
        Gp[f * M + m] = sacc;
      }
    }
  }
}

template <int W, int FPL, int RK, bool MULTI>
void launch_descriptor_w2(const DescArgs &a, cudaStream_t st) {
  const int T = kPairThreads;
  const long threads = (long)a.n * W;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
#define TMD_DESCW_ARGS a.kp, a.box, a.n, a.cap, a.x, a.nbr, a.boff, a.P, a.G, a.cbox, a.acell, a.pdf, a.pgeo, a.pcnt
  switch (a.kp.D) {
    case 1: k_descriptor_w2<W, FPL, 1, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESCW_ARGS); break;
    case 4: k_descriptor_w2<W, FPL, 4, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESCW_ARGS); break;
    case 10: k_descriptor_w2<W, FPL, 10, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESCW_ARGS); break;
    default: k_descriptor_w2<W, FPL, 20, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESCW_ARGS); break;
  }
#undef TMD_DESCW_ARGS
}

// ---------------------------------------------------------------------------
// Split form: the pair geometry in a kernel of its own, the contraction in
// another.  In the fused forms each lane computes the FP64 geometry of one
// list entry at a time (a dependent chain: image, difference, squared
// distance, square root, cutoff) and the atom's group waits on it before the
// contraction can use the pair; at the registers the contraction needs, 16-24
// warps per SM cannot hide that latency.  Here k_pair_geo runs with a warp
// per atom and few registers (many warps per SM), tests every entry, and
// writes the compact geometry of the active pairs block by block (the same
// pgeo/pcnt the force kernel reads) and zero pair forces for the rest; the
// contraction kernel then streams the compact pairs.

// Warp per atom: entries of each element block in rounds of 32, active ones
// compacted in row order (ballot + prefix count).
template <int RK, bool MULTI>
__global__ void __launch_bounds__(256, 6)
k_pair_geo(KParams kp, BoxP box, int n, int cap, const double *__restrict__ x,
           const uint32_t *__restrict__ nbr, const int *__restrict__ boff,
           const BoxP *__restrict__ cbox, const int *__restrict__ acell,
           float4 *__restrict__ pdf, float4 *__restrict__ pgeo, int *__restrict__ pcnt) {
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int B = kp.B;
  for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < n; a += nw) {
    const BoxP &bx = box_of<MULTI>(box, cbox, acell, a);
    const double xi = x[3 * a], yi = x[3 * a + 1], zi = x[3 * a + 2];
    const uint32_t *row = nbr + (size_t)a * cap;
    const int *bo = boff + (size_t)a * (B + 1);
    float4 *pdf_row = pdf + (size_t)a * cap;
    float4 *pg_row = pgeo + (size_t)a * cap * 2;
    int nact = 0;
    for (int b = 0; b < B; b++) {
      const int s0 = bo[b], s1 = bo[b + 1];
      int cnt = 0;
      // entries are loaded two rounds ahead and their positions one round
      // ahead, so the dependent gather (entry, then position) overlaps work
      NbPos pn = load_nb(x, s0 + lane < s1 ? row[s0 + lane] : 0u, s0 + lane < s1);
      uint32_t en = s0 + 32 + lane < s1 ? row[s0 + 32 + lane] : 0u;
      for (int t0 = s0; t0 < s1; t0 += 32) {
        const NbPos pc = pn;
        const int tn = t0 + 32 + lane;
        pn = load_nb(x, en, tn < s1);
        en = tn + 32 < s1 ? row[tn + 32] : 0u;
        PairGeo g;
        pair_geometry(kp, bx, xi, yi, zi, pc, g);
        const bool act = g.ti >= 0;
        const unsigned bal = __ballot_sync(0xffffffffu, act);
        const int t = t0 + lane;
        if (act) {
          const int c = nact + cnt + __popc(bal & ((1u << lane) - 1u));
          float4 *dst = pg_row + 2 * c;
          dst[0] = make_float4(g.r, g.rlo, g.ux, g.uy);
          dst[1] = RK == kRadTable
                       ? make_float4(g.uz, g.tq, __int_as_float(g.ti), __int_as_float(t))
                       : make_float4(g.uz, g.fc, g.dfc, __int_as_float(t));
        } else if (t < s1) {
          pdf_row[t] = make_float4(0.f, 0.f, 0.f, 0.f);
        }
        cnt += __popc(bal);
      }
      if (lane == 0) pcnt[(size_t)a * B + b] = cnt;
      nact += cnt;
    }
  }
}

// Contraction over the compact pairs: W = min(K, 32) lanes per atom, FPL =
// K / W filters per lane.  Pairs come in chunks of W; lane c of the group
// loads pair c's geometry (one chunk ahead), forms its D monomials and puts
// them and the radial inputs in the group's shared-memory slots (two chunk
// buffers, so one warp sync per chunk); every lane then accumulates its
// filters over the chunk's pairs in row order, as k_descriptor_w.
template <int W, int FPL, int D, int RK>
__global__ void __launch_bounds__(kPairThreads, 8)
k_descriptor_c(KParams kp, int n, int cap, float *__restrict__ P, float *__restrict__ G,
               const float4 *__restrict__ pgeo, const int *__restrict__ pcnt) {
  constexpr int D4 = (D + 3) / 4 * 4;
  constexpr int M = D == 1 ? 1 : (D == 4 ? 2 : (D == 10 ? 3 : 4));
  constexpr int P2 = D4 / 2;
  constexpr int SL = D4 + 4;  // floats per slot: monomials, then (r, rlo, fc | tq, ti)
  __shared__ __align__(16) float slots[2 * kPairThreads * SL + kPairThreads];
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int a = gt / W;
  const int sub = gt % W;
  if (a >= n) return;
  const int lane = threadIdx.x & 31;
  const unsigned gmask = PairRing<W>::kBits << (lane & ~(W - 1));
  const unsigned live = live_lanes(gt, (long)n * W);
  // the group's 2 x W slots, groups offset by 4 words: the groups of a warp
  // read slot c from different banks
  float *sg = slots + 2 * (threadIdx.x - sub) * SL + 4 * (threadIdx.x / W);
  const int B = kp.B, K = kp.K;
  const int kf = sub * FPL;
  Radial1<RK> R[FPL];
#pragma unroll
  for (int f = 0; f < FPL; f++) R[f] = load_radial1<RK>(kp, kf + f);
  const float4 *pg_row = pgeo + (size_t)a * cap * 2;
  int pos = 0, buf = 0;
  for (int b = 0; b < B; b++) {
    if (b > 0) __syncwarp(live);
    const int np = pcnt[(size_t)a * B + b];
    float2 acc[FPL][P2];
#pragma unroll
    for (int f = 0; f < FPL; f++)
#pragma unroll
      for (int p = 0; p < P2; p++) acc[f][p] = make_float2(0.f, 0.f);
    float4 ga = make_float4(0.f, 0.f, 0.f, 0.f), gb = ga;
    if (sub < np) {
      ga = __ldg(pg_row + 2 * (pos + sub));
      gb = __ldg(pg_row + 2 * (pos + sub) + 1);
    }
    for (int c0 = 0; c0 < np; c0 += W) {
      const int cnt = min(W, np - c0);
      float *slot = sg + (buf * W + sub) * SL;
      if (sub < cnt) {
        float Mv[D4];
        moments<D>(ga.z, ga.w, gb.x, Mv);
#pragma unroll
        for (int d = D; d < D4; d++) Mv[d] = 0.f;
#pragma unroll
        for (int v = 0; v < D4 / 4; v++)
          reinterpret_cast<float4 *>(slot)[v] =
              make_float4(Mv[4 * v], Mv[4 * v + 1], Mv[4 * v + 2], Mv[4 * v + 3]);
        // radial inputs: r, rlo, fc (analytic) or tq, interval (table)
        reinterpret_cast<float4 *>(slot)[D4 / 4] =
            RK == kRadTable ? make_float4(0.f, 0.f, gb.y, gb.z) : make_float4(ga.x, ga.y, gb.y, 0.f);
      }
      // next chunk's geometry in flight while this one is multiplied
      const int cn = c0 + W + sub;
      if (cn < np) {
        ga = __ldg(pg_row + 2 * (pos + cn));
        gb = __ldg(pg_row + 2 * (pos + cn) + 1);
      }
      __syncwarp(gmask);
      const float *cs = sg + buf * W * SL;
#pragma unroll 2
      for (int c = 0; c < cnt; c++) {
        const float4 *ms = reinterpret_cast<const float4 *>(cs + c * SL);
        const float4 rr = ms[D4 / 4];
        PairGeo g;
        g.ux = g.uy = g.uz = g.dfc = g.rinv = 0.f;
        if (RK == kRadTable) {
          g.r = g.rlo = g.fc = 0.f;
          g.tq = rr.z;
          g.ti = __float_as_int(rr.w);
        } else {
          g.r = rr.x; g.rlo = rr.y; g.fc = rr.z; g.tq = 0.f; g.ti = 0;
        }
        float2 h2[FPL];
#pragma unroll
        for (int f = 0; f < FPL; f++) {
          const float h = radial1<RK>(kp, R[f], g);
          h2[f] = make_float2(h, h);
        }
#pragma unroll
        for (int v = 0; v < D4 / 4; v++) {
          const float4 m4 = ms[v];
          const float2 lo = make_float2(m4.x, m4.y), hi = make_float2(m4.z, m4.w);
#pragma unroll
          for (int f = 0; f < FPL; f++) {
            acc[f][2 * v] = __ffma2_rn(h2[f], lo, acc[f][2 * v]);
            acc[f][2 * v + 1] = __ffma2_rn(h2[f], hi, acc[f][2 * v + 1]);
          }
        }
      }
      buf ^= 1;
    }
    pos += np;
    float *Pp = P + (((size_t)a * B + b) * K + kf) * D;
    float *Gp = G + (((size_t)a * B + b) * K + kf) * M;
#pragma unroll
    for (int f = 0; f < FPL; f++) {
      if constexpr (D % 2 == 0) {
        float2 *P2p = reinterpret_cast<float2 *>(Pp + f * D);
#pragma unroll
        for (int p = 0; p < D / 2; p++) P2p[p] = acc[f][p];
      } else {
#pragma unroll
        for (int d = 0; d < D; d++) Pp[f * D + d] = (d & 1) ? acc[f][d >> 1].y : acc[f][d >> 1].x;
      }
#pragma unroll
      for (int m = 0; m < M; m++) {
        float sacc = 0.f;
#pragma unroll
        for (int d = 0; d < D; d++) {
          const float pv = (d & 1) ? acc[f][d >> 1].y : acc[f][d >> 1].x;
          sacc = fmaf(kp.T[m * D + d], pv * pv, sacc);
        }
        if (m == 0) sacc = copysignf(1.f, acc[f][0].x) * sqrtf(sacc);
        Gp[f * M + m] = sacc;
      }
    }
  }
}

template <int W, int FPL, int RK, bool MULTI>
void launch_descriptor_split(const DescArgs &a, cudaStream_t st) {
  {
    const int T = 256;
    long g = ((long)a.n * 32 + T - 1) / T;
    if (g > 148 * 16) g = 148 * 16;
    if (g < 1) g = 1;
    k_pair_geo<RK, MULTI><<<(int)g, T, 0, st>>>(a.kp, a.box, a.n, a.cap, a.x, a.nbr, a.boff,
                                               a.cbox, a.acell, a.pdf, a.pgeo, a.pcnt);
  }
  const int T = kPairThreads;
  const long threads = (long)a.n * W;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
#define TMD_DESCC_ARGS a.kp, a.n, a.cap, a.P, a.G, a.pgeo, a.pcnt
  switch (a.kp.D) {
    case 1: k_descriptor_c<W, FPL, 1, RK><<<grid, T, 0, st>>>(TMD_DESCC_ARGS); break;
    case 4: k_descriptor_c<W, FPL, 4, RK><<<grid, T, 0, st>>>(TMD_DESCC_ARGS); break;
    case 10: k_descriptor_c<W, FPL, 10, RK><<<grid, T, 0, st>>>(TMD_DESCC_ARGS); break;
    default: k_descriptor_c<W, FPL, 20, RK><<<grid, T, 0, st>>>(TMD_DESCC_ARGS); break;
  }
#undef TMD_DESCC_ARGS
}

template <int W, int FPL, int RK, bool MULTI>
void launch_descriptor_w(const DescArgs &a, cudaStream_t st) {
  const int T = kPairThreads;
  const long threads = (long)a.n * W;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
#define TMD_DESCW_ARGS a.kp, a.box, a.n, a.cap, a.x, a.nbr, a.boff, a.P, a.G, a.cbox, a.acell, a.pdf, a.pgeo, a.pcnt
  switch (a.kp.D) {
    case 1: k_descriptor_w<W, FPL, 1, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESCW_ARGS); break;
    case 4: k_descriptor_w<W, FPL, 4, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESCW_ARGS); break;
    case 10: k_descriptor_w<W, FPL, 10, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESCW_ARGS); break;
    default: k_descriptor_w<W, FPL, 20, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESCW_ARGS); break;
  }
#undef TMD_DESCW_ARGS
}

// G[b,k,m] = sum_d T[m,d] P[b,k,d]^2, G[b,k,0] = sign(P0) sqrt(.)
// (kernel_1_fused_device, kernel.cu:1028-1061): one thread per output, the D
// values of the row from L1, coalesced writes in the MLP row layout.
template <int D, int M>
__global__ void k_invariants(long nout, KParams kp, const float *__restrict__ P,
                             float *__restrict__ G) {
  __shared__ float sT[M * D];  // lanes read different m: no per-lane param index
  for (int i = threadIdx.x; i < M * D; i += blockDim.x) sT[i] = kp.T[i];
  __syncthreads();
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nout) return;
  const long row = e / M;
  const int m = (int)(e - row * M);
  const float *p = P + row * D;
  float s = 0.f;
#pragma unroll
  for (int d = 0; d < D; d++) {
    const float pv = __ldg(p + d);
    s = fmaf(sT[m * D + d], pv * pv, s);
  }
  if (m == 0) s = copysignf(1.f, __ldg(p)) * sqrtf(s);
  G[e] = s;
}

inline void launch_invariants(const DescArgs &a, cudaStream_t st) {
  const long nout = (long)a.n * a.kp.B * a.kp.K * a.kp.M;
  if (nout == 0) return;
  const int T = 256;
  const unsigned grid = (unsigned)((nout + T - 1) / T);
  switch (a.kp.D) {
    case 1: k_invariants<1, 1><<<grid, T, 0, st>>>(nout, a.kp, a.P, a.G); break;
    case 4: k_invariants<4, 2><<<grid, T, 0, st>>>(nout, a.kp, a.P, a.G); break;
    case 10: k_invariants<10, 3><<<grid, T, 0, st>>>(nout, a.kp, a.P, a.G); break;
    default: k_invariants<20, 4><<<grid, T, 0, st>>>(nout, a.kp, a.P, a.G); break;
  }
}

template <int TPA, int RK, bool MULTI>
void launch_descriptor_tpa(const DescArgs &a, cudaStream_t st) {
  const int T = kPairThreads;
  long threads = (long)a.n * TPA;
  int grid = (int)((threads + T - 1) / T);
  if (grid < 1) grid = 1;
#define TMD_DESC_ARGS a.kp, a.box, a.n, a.cap, a.x, a.elem, a.nbr, a.boff, a.P, a.G, a.cbox, a.acell, a.pdf, a.pgeo, a.pcnt
  switch (a.kp.D) {
    case 1: k_descriptor<TPA, 1, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESC_ARGS); break;
    case 4: k_descriptor<TPA, 4, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESC_ARGS); break;
    case 10: k_descriptor<TPA, 10, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESC_ARGS); break;
    default: k_descriptor<TPA, 20, RK, MULTI><<<grid, T, 0, st>>>(TMD_DESC_ARGS); break;
  }
#undef TMD_DESC_ARGS
}

// One radial kind and box mode; each (kind, mode) pair is instantiated in its
// own translation unit so the variants compile in parallel.
template <int RK, bool MULTI>
void launch_descriptor_rk(const DescArgs &a, cudaStream_t st) {
  if (a.variant == kDescSplit) {
    switch (a.kp.K) {
      case 4: launch_descriptor_split<4, 1, RK, MULTI>(a, st); break;
      case 8: launch_descriptor_split<8, 1, RK, MULTI>(a, st); break;
      case 16: launch_descriptor_split<16, 1, RK, MULTI>(a, st); break;
      case 32: launch_descriptor_split<32, 1, RK, MULTI>(a, st); break;
      case 64: launch_descriptor_split<32, 2, RK, MULTI>(a, st); break;
      default: launch_descriptor_split<32, 4, RK, MULTI>(a, st); break;
    }
    return;
  }
  if (a.variant == kDescWide2 && a.kp.K >= 4 && a.kp.K <= 64) {
    switch (a.kp.K) {
      case 4: launch_descriptor_w2<4, 2, RK, MULTI>(a, st); return;
      case 8: launch_descriptor_w2<8, 2, RK, MULTI>(a, st); return;
      case 16: launch_descriptor_w2<16, 2, RK, MULTI>(a, st); return;
      case 32: launch_descriptor_w2<32, 2, RK, MULTI>(a, st); return;
      case 64: launch_descriptor_w2<32, 4, RK, MULTI>(a, st); return;
      default: break;  // other filter counts: the one-stream wide form
    }
  }
  if (a.variant == kDescWide || a.variant == kDescWide2) {
    switch (a.kp.K) {
      case 4: launch_descriptor_w<4, 1, RK, MULTI>(a, st); break;
      case 8: launch_descriptor_w<8, 1, RK, MULTI>(a, st); break;
      case 16: launch_descriptor_w<16, 1, RK, MULTI>(a, st); break;
      case 32: launch_descriptor_w<32, 1, RK, MULTI>(a, st); break;
      case 64: launch_descriptor_w<32, 2, RK, MULTI>(a, st); break;
      default: launch_descriptor_w<32, 4, RK, MULTI>(a, st); break;
    }
    return;
  }

  switch (a.kp.K / 4) {
    case 1: launch_descriptor_tpa<1, RK, MULTI>(a, st); break;
    case 2: launch_descriptor_tpa<2, RK, MULTI>(a, st); break;
    case 4: launch_descriptor_tpa<4, RK, MULTI>(a, st); break;
    case 8: launch_descriptor_tpa<8, RK, MULTI>(a, st); break;
    case 16: launch_descriptor_tpa<16, RK, MULTI>(a, st); break;
    default: launch_descriptor_tpa<32, RK, MULTI>(a, st); break;
  }
}

}  // namespace tmd
