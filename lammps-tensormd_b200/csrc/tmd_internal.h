// tmd_internal.h -- shared device-side types of the tensormd B200 path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tmd {

constexpr int kMaxElt = 8;      // potential elements (reference MAX_ELETYPES 5)
constexpr int kMaxK = 128;      // radial filters
constexpr int kMaxD = 20;       // monomials of rank <= 3
constexpr int kMaxLayers = 12;  // MLP layers
constexpr int kShiftR = 3;      // periodic image shift range [-3, 3] per axis
constexpr int kShiftBits = 9;   // 7^3 = 343 codes
constexpr int kAtomBits = 23;   // atom index bits of a neighbor entry
constexpr uint32_t kAtomMask = (1u << kAtomBits) - 1u;
constexpr int kMaxAtoms = (1 << kAtomBits) - 1;

// Model constants passed to kernels by value.
struct KParams {
  int K, D, M, B, nin;  // filters, monomials, moments, element blocks, b*k*m
  int radial;           // 0 analytic function, 1 rational table
  int method;           // analytic: 0 pexp, 1 morse, 2 density, 3 Gaussian SF
  int fctype;           // 0 cosine, else polynomial (gamma = 5)
  float rc, inv_rc, inv_rc2;
  double rcsq;          // FP64 force cutoff test rij2 < rcsq
  float T[4 * kMaxD];   // multiplicity tensor T[m][d]
  float p0[kMaxK], p1[kMaxK], p2[kMaxK];
  // Gaussian SF: exp(-gc (r - omega)^2) with gc = eta / rc^2 rounded once
  // from FP64, omega = p1 + p1lo (FP32 hi/lo pair)
  float gc[kMaxK], p1lo[kMaxK];
  float gcl[kMaxK];     // gc * log2(e): exp(-gc d^2) evaluated as exp2(-gcl d^2)
  int eltij[kMaxElt * kMaxElt];  // element block of (elt_i, elt_j)
  const float *table;   // [tab_n][4][K] : y, s, c1, c2
  int tab_n;
  float tab_dx;
  double tab_dxd, tab_xdxd;
};

// Periodic cell.
struct BoxP {
  double lo[3];
  double xprd, yprd, zprd, xy, xz, yz;
  double hinv[6];       // inverse of the upper-triangular cell matrix
  int pbc[3];
  int triclinic;
};

// Cell-list geometry used by the neighbor build.
struct BinP {
  int nb[3];  // bins per axis (fractional coordinates)
  int ns[3];  // stencil half-extent per axis
  int ncell;
};

__host__ __device__ inline int shift_code(int sx, int sy, int sz) {
  return (sx + kShiftR) + 7 * (sy + kShiftR) + 49 * (sz + kShiftR);
}
__host__ __device__ inline void shift_decode(int code, int &sx, int &sy, int &sz) {
  sx = code % 7 - kShiftR;
  sy = (code / 7) % 7 - kShiftR;
  sz = code / 49 - kShiftR;
}
__host__ __device__ inline uint32_t nb_pack(int j, int code) {
  return (uint32_t(code) << kAtomBits) | uint32_t(j);
}
__host__ __device__ inline int neg_code(int code) {
  int sx, sy, sz;
  shift_decode(code, sx, sy, sz);
  return shift_code(-sx, -sy, -sz);
}

// Image of position p shifted by (sx, sy, sz) cell vectors, one hop at a time
// in x, then y, then z (AtomVec::pack_border: x + pbc*prd per swap).
__host__ __device__ inline void image_of(const BoxP &b, double px, double py,
                                         double pz, int sx, int sy, int sz,
                                         double &ox, double &oy, double &oz) {
  double st = sx > 0 ? 1.0 : -1.0;
  for (int t = 0; t < (sx > 0 ? sx : -sx); t++) px = px + st * b.xprd;
  st = sy > 0 ? 1.0 : -1.0;
  for (int t = 0; t < (sy > 0 ? sy : -sy); t++) {
    px = px + st * b.xy;
    py = py + st * b.yprd;
  }
  st = sz > 0 ? 1.0 : -1.0;
  for (int t = 0; t < (sz > 0 ? sz : -sz); t++) {
    px = px + st * b.xz;
    py = py + st * b.yz;
    pz = pz + st * b.zprd;
  }
  ox = px; oy = py; oz = pz;
}

}  // namespace tmd
