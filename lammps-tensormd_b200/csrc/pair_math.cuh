// pair_math.cuh -- per-pair geometry, radial basis and angular moments.
//
// Radial functions H_k(r) = f_c(r) g_k(r) follow descriptor.cpp:51-138 and
// cutoff.cpp:20-37; the rational table follows ration.cu:27-69 (endpoint
// intervals forced to zero, ration.hpp:29).  Monomials are ordered as
// kernel.cu:1197-1232: 1, x, y, z, xx, xy, xz, yy, yz, zz, xxx, xxy, xxz,
// xyy, xyz, xzz, yyy, yyz, yzz, zzz.
#pragma once

#include "tmd_internal.h"

namespace tmd {

// Pair geometry computed by one lane and broadcast to the atom's group.
struct PairGeo {
  float r, rlo;         // distance as an FP32 hi/lo pair (r = hi + lo)
  float ux, uy, uz;     // unit vector (x_j - x_i) / r
  float fc, dfc;        // analytic cutoff and derivative
  float tq;             // table: offset inside the interval
  float rinv;           // 1 / r (FP32)
  int ti;               // table interval (0 for analytic), -1 when inactive
};

__device__ inline double rsq_plain(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)),
                   __dmul_rn(dz, dz));
}

// Position of neighbor entry e, loaded early so the gather latency overlaps
// the previous chunk's arithmetic.
struct NbPos {
  double x, y, z;
  int code;  // shift code, -1 when the slot is empty
};

__device__ inline NbPos load_nb(const double *__restrict__ x, uint32_t e, bool valid) {
  NbPos p;
  if (valid) {
    int j = e & kAtomMask;
    p.x = __ldg(x + 3 * j);
    p.y = __ldg(x + 3 * j + 1);
    p.z = __ldg(x + 3 * j + 2);
    p.code = int(e >> kAtomBits);
  } else {
    p.x = p.y = p.z = 0.0;
    p.code = -1;
  }
  return p;
}

// Geometry of one pair (FP64 difference and cutoff test rij2 < rc^2 &&
// rij2 > 1e-10 as kernel.cu:1163).  g.ti = -1 if inactive.
__device__ inline void pair_geometry(const KParams &kp, const BoxP &box, double xi,
                                     double yi, double zi, const NbPos &p,
                                     PairGeo &g) {
  g.ti = -1;
  g.r = g.rlo = g.ux = g.uy = g.uz = g.fc = g.dfc = g.tq = g.rinv = 0.f;
  if (p.code < 0) return;
  int sx, sy, sz;
  shift_decode(p.code, sx, sy, sz);
  double gx, gy, gz;
  image_of(box, p.x, p.y, p.z, sx, sy, sz, gx, gy, gz);
  double dx = gx - xi, dy = gy - yi, dz = gz - zi;
  double r2 = rsq_plain(dx, dy, dz);
  if (!(r2 < kp.rcsq && r2 > 1e-10)) return;
  double r = sqrt(r2);
  float rf = float(r);
  float rinv = 1.0f / rf;
  g.r = rf;
  g.rinv = rinv;
  g.rlo = float(r - double(rf));
  g.ux = float(dx) * rinv;
  g.uy = float(dy) * rinv;
  g.uz = float(dz) * rinv;
  if (kp.radial == 1) {
    int ti = int(r * kp.tab_xdxd);
    if (ti > kp.tab_n - 2) ti = kp.tab_n - 2;
    g.ti = ti;
    g.tq = float(r - ti * kp.tab_dxd);
  } else {
    g.ti = 0;
    float z = rf * kp.inv_rc;
    if (kp.fctype == 0) {
      z = z > 1.f ? 1.f : z;
      float s, c;
      sincospif(z, &s, &c);
      g.fc = 0.5f + 0.5f * c;
      g.dfc = -0.5f * 3.14159265358979f * s * kp.inv_rc;
    } else {
      const float gm = 5.f;
      z = z > 3.14159265358979f ? 3.14159265358979f : z;
      float z4 = z * z * z * z, z5 = z4 * z;
      g.fc = 1.f + gm * z5 * z - (gm + 1.f) * z5;
      g.dfc = (gm + 1.f) * gm * kp.inv_rc * (z5 - z4);
    }
  }
}

__device__ inline PairGeo shfl_geo(unsigned mask, const PairGeo &g, int src,
                                   int width) {
  PairGeo o;
  o.r = __shfl_sync(mask, g.r, src, width);
  o.rlo = __shfl_sync(mask, g.rlo, src, width);
  o.ux = __shfl_sync(mask, g.ux, src, width);
  o.uy = __shfl_sync(mask, g.uy, src, width);
  o.uz = __shfl_sync(mask, g.uz, src, width);
  o.fc = __shfl_sync(mask, g.fc, src, width);
  o.dfc = __shfl_sync(mask, g.dfc, src, width);
  o.tq = __shfl_sync(mask, g.tq, src, width);
  o.rinv = __shfl_sync(mask, g.rinv, src, width);
  o.ti = __shfl_sync(mask, g.ti, src, width);
  return o;
}

// 2^x for x <= 0 by the ex2.approx.ftz instruction (one MUFU operation).  On
// the B200 it returns exp2f's value bit for bit for every FP32 x in
// [-126, 0] (all 1.1e9 inputs compared); below -126, where exp2f returns a
// subnormal, it returns 0.  The Gaussian radial basis takes it in place of
// exp2f's extra range handling.
__device__ __forceinline__ float exp2_nonpos(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Radial kinds the kernels are specialised on.
constexpr int kRadTable = 0;    // rational-interpolation table (FNN or tabulated)
constexpr int kRadGauss = 1;    // analytic Gaussian SF (descriptor::method 3)
constexpr int kRadGeneric = 2;  // analytic power-exponential / Morse / density

inline int radial_kind(const KParams &kp) {
  if (kp.radial == 1) return kRadTable;
  return kp.method == 3 ? kRadGauss : kRadGeneric;
}

// Radial parameters of a lane's 4 filters, loaded once per kernel.  For the
// Gaussian kind gc holds -2 gc and gl holds -gcl (signs and the factor 2
// applied once at load, exactly).
template <int RK>
struct Radial4 {
  float a[RK == kRadGeneric ? 4 : 1], b[RK == kRadTable ? 1 : 4],
      c[RK == kRadGeneric ? 4 : 1], blo[RK == kRadGauss ? 4 : 1],
      gc[RK == kRadGauss ? 4 : 1], gl[RK == kRadGauss ? 4 : 1];
  int k0;
};

template <int RK>
__device__ inline Radial4<RK> load_radial4(const KParams &kp, int k0) {
  Radial4<RK> R;
  R.k0 = k0;
#pragma unroll
  for (int t = 0; t < 4; t++) {
    if (RK == kRadGeneric) {
      R.a[t] = kp.p0[k0 + t];
      R.c[t] = kp.p2[k0 + t];
    }
    if (RK != kRadTable) R.b[t] = kp.p1[k0 + t];
    if (RK == kRadGauss) {
      R.blo[t] = kp.p1lo[k0 + t];
      R.gc[t] = -2.f * kp.gc[k0 + t];
      R.gl[t] = -kp.gcl[k0 + t];
    }
  }
  return R;
}

// H_k and (optionally) dH_k/dr for the lane's filters k0..k0+3.
template <int RK, bool DERIV>
__device__ inline void radial4(const KParams &kp, const Radial4<RK> &R, const PairGeo &g,
                               float H[4], float dH[4]) {
  if (RK == kRadTable) {
    if (g.ti <= 0 || g.ti >= kp.tab_n - 2) {
#pragma unroll
      for (int q = 0; q < 4; q++) { H[q] = 0.f; if (DERIV) dH[q] = 0.f; }
      return;
    }
    const int K = kp.K, k0 = R.k0;
    const float4 *row = reinterpret_cast<const float4 *>(kp.table + (size_t)g.ti * 4 * K);
    float4 y4 = __ldg(row + (k0 >> 2));
    float4 s4 = __ldg(row + ((K + k0) >> 2));
    float4 a4 = __ldg(row + ((2 * K + k0) >> 2));
    float4 b4 = __ldg(row + ((3 * K + k0) >> 2));
    const float ys[4] = {y4.x, y4.y, y4.z, y4.w};
    const float ss[4] = {s4.x, s4.y, s4.z, s4.w};
    const float c1s[4] = {a4.x, a4.y, a4.z, a4.w};
    const float c2s[4] = {b4.x, b4.y, b4.z, b4.w};
    const float q = g.tq, dx = kp.tab_dx, rr = dx - q;
#pragma unroll
    for (int t = 0; t < 4; t++) {
      float c1 = c1s[t], c2 = c2s[t], s = ss[t];
      float c3 = fabsf(c2 * rr);
      float c4 = c3 + fabsf(c1 * q);
      if (c4 > 0.f) c3 = __fdividef(c3, c4);  // weight in [0, 1]: 2-ulp quotient
      c4 = c2 + c3 * (c1 - c2);
      H[t] = ys[t] + q * (s - rr * c4);
      if (DERIV) dH[t] = s + (q - rr) * c4 + dx * (c4 - c2) * (1.f - c3);
    }
    return;
  }
  const float r = g.r;
#pragma unroll
  for (int t = 0; t < 4; t++) {
    float f, df;
    if (RK == kRadGauss) {
      // (r - omega) from the hi/lo pairs of both: no systematic rounding of
      // the Gaussian centre
      float d = (r - R.b[t]) + (g.rlo - R.blo[t]);
      f = exp2_nonpos(R.gl[t] * d * d);
      if (DERIV) {
        // dH = dfc f + fc (gc d f) = f (dfc + fc gc d): one FFMA and two FMULs
        H[t] = g.fc * f;
        dH[t] = f * fmaf(g.fc * R.gc[t], d, g.dfc);
        continue;
      }
      df = 0.f;
    } else {
      const float a = R.a[t], b = R.b[t], c = R.c[t];
      if (kp.method == 0) {
        float xr = r / a;
        float pw = powf(xr, b);
        f = expf(-pw);
        df = -f * b * powf(xr, b - 1.f) / a;
      } else if (kp.method == 1) {
        float gdr = b * (r - c);
        float e1 = expf(-gdr), e2 = expf(-2.f * gdr);
        f = a * (e2 - 2.f * e1);
        df = -a * b * 2.f * (e2 - e1);
      } else {
        float z = -b * ((r - c) / c);
        f = a * expf(z);
        df = -f * b / c;
      }
    }
    H[t] = g.fc * f;
    if (DERIV) dH[t] = g.dfc * f + g.fc * df;
  }
}

// Radial parameters of one filter k, loaded once per kernel by the lane that
// owns the filter (the wide-group descriptor form).
template <int RK>
struct Radial1 {
  float a, b, c, blo, gc, gl;
  int k;
};

template <int RK>
__device__ inline Radial1<RK> load_radial1(const KParams &kp, int k) {
  Radial1<RK> R{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, k};
  if (RK == kRadGeneric) { R.a = kp.p0[k]; R.c = kp.p2[k]; }
  if (RK != kRadTable) R.b = kp.p1[k];
  if (RK == kRadGauss) { R.blo = kp.p1lo[k]; R.gc = kp.gc[k]; R.gl = kp.gcl[k]; }
  return R;
}

// H_k of one filter: the expressions of radial4 for a single k.
template <int RK>
__device__ inline float radial1(const KParams &kp, const Radial1<RK> &R, const PairGeo &g) {
  if (RK == kRadTable) {
    if (g.ti <= 0 || g.ti >= kp.tab_n - 2) return 0.f;
    const int K = kp.K;
    const float *row = kp.table + (size_t)g.ti * 4 * K + R.k;
    const float y = __ldg(row), s = __ldg(row + K), c1 = __ldg(row + 2 * K),
                c2 = __ldg(row + 3 * K);
    const float q = g.tq, dx = kp.tab_dx, rr = dx - q;
    float c3 = fabsf(c2 * rr);
    float c4 = c3 + fabsf(c1 * q);
    if (c4 > 0.f) c3 = __fdividef(c3, c4);
    c4 = c2 + c3 * (c1 - c2);
    return y + q * (s - rr * c4);
  }
  float f;
  if (RK == kRadGauss) {
    float d = (g.r - R.b) + (g.rlo - R.blo);
    f = exp2_nonpos(-R.gl * d * d);
  } else {
    const float r = g.r, a = R.a, b = R.b, c = R.c;
    if (kp.method == 0) {
      float xr = r / a;
      float pw = powf(xr, b);
      f = expf(-pw);
    } else if (kp.method == 1) {
      float gdr = b * (r - c);
      float e1 = expf(-gdr), e2 = expf(-2.f * gdr);
      f = a * (e2 - 2.f * e1);
    } else {
      float z = -b * ((r - c) / c);
      f = a * expf(z);
    }
  }
  return g.fc * f;
}

template <int D>
__device__ inline void moments(float x, float y, float z, float M[D]) {
  M[0] = 1.f;
  if (D > 1) { M[1] = x; M[2] = y; M[3] = z; }
  if (D > 4) {
    float xx = x * x, xy = x * y, xz = x * z, yy = y * y, yz = z * y, zz = z * z;
    M[4] = xx; M[5] = xy; M[6] = xz; M[7] = yy; M[8] = yz; M[9] = zz;
    if (D > 10) {
      M[10] = xx * x; M[11] = xx * y; M[12] = xx * z; M[13] = xy * y;
      M[14] = xy * z; M[15] = xz * z; M[16] = yy * y; M[17] = yy * z;
      M[18] = yz * z; M[19] = zz * z;
    }
  }
}

// Gradient of Q(u) = sum_d V_d M_d(u) with respect to u, and sum_d n_d V_d M_d
// (n_d = rank of monomial d).  Then dQ/dx_j = (gradQ - u * nVM) / r, which
// is sum_d V_d dM_d/dx_j (tensor_ops.cpp calculate_dM_{p,d,f}).  Each M_d is
// homogeneous of degree n_d, so u . grad M_d = n_d M_d (Euler) and nVM is
// formed as u . gradQ.
template <int D>
__device__ inline void poly_grad(const float V[D], float x, float y, float z,
                                 float gq[3], float &nvm) {
  // Horner form: grad_a Q = V_a + x P_a + y Q_a + z R_a, with P, Q, R the
  // coefficients of x, y, z once the linear terms are taken out (three short
  // independent chains instead of one long sum per component)
  float gx = 0.f, gy = 0.f, gz = 0.f;
  if (D > 1) {
    float Px = 0.f, Qx = 0.f, Rx = 0.f, Py = 0.f, Qy = 0.f, Ry = 0.f, Pz = 0.f, Qz = 0.f,
          Rz = 0.f;
    if (D > 4) {
      // xx, xy, xz, yy, yz, zz
      Px = 2.f * V[4]; Qx = V[5]; Rx = V[6];
      Py = V[5]; Qy = 2.f * V[7]; Ry = V[8];
      Pz = V[6]; Qz = V[8]; Rz = 2.f * V[9];
      if (D > 10) {
        // xxx xxy xxz xyy xyz xzz yyy yyz yzz zzz
        Px = fmaf(3.f * V[10], x, fmaf(2.f * V[11], y, fmaf(2.f * V[12], z, Px)));
        Qx = fmaf(V[13], y, fmaf(V[14], z, Qx));
        Rx = fmaf(V[15], z, Rx);
        Py = fmaf(V[11], x, fmaf(2.f * V[13], y, fmaf(V[14], z, Py)));
        Qy = fmaf(3.f * V[16], y, fmaf(2.f * V[17], z, Qy));
        Ry = fmaf(V[18], z, Ry);
        Pz = fmaf(V[12], x, fmaf(V[14], y, fmaf(2.f * V[15], z, Pz)));
        Qz = fmaf(V[17], y, fmaf(2.f * V[18], z, Qz));
        Rz = fmaf(3.f * V[19], z, Rz);
      }
    }
    gx = fmaf(x, Px, fmaf(y, Qx, fmaf(z, Rx, V[1])));
    gy = fmaf(x, Py, fmaf(y, Qy, fmaf(z, Ry, V[2])));
    gz = fmaf(x, Pz, fmaf(y, Qz, fmaf(z, Rz, V[3])));
  }
  gq[0] = gx; gq[1] = gy; gq[2] = gz;
  nvm = x * gx + y * gy + z * gz;
}

}  // namespace tmd
