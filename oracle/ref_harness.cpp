// ref_harness.cpp -- drives the reference's own CPU contraction kernels
// (src/ML-TENSORMD/tensor_ops.cpp, compiled from the reference tree by
// oracle/build_ref.py into oracle/_ref/) on per-pair inputs prepared by a
// test, so the oracle's restatement of P, dE/dP, U, V, F1 and F2 can be
// checked against the reference's implementation of the same steps.
// Test infrastructure (a checker), not part of the product.
//
// Sequence of TensorMD::run on its CPU path (tensormd.cpp:563-602):
//   P = kernel_P(M, H)                    P_dkba = sum_c M_dcba H_kcba
//   dEdG' = kernel_dEdG(G, dEdG)          dEdG'0 = 0.5 dEdG0 / G0
//   S = kernel_dEdS(T, dEdG', P)          S_dkba = 2 sum_m T_md dEdG'_mkba P_dkba
//   U = kernel_U(S, M), V = kernel_V(S, H)
//   F = kernel_F1(U, dH, u, mask) + kernel_fused_F2(V, R, u, mask)
// Arrays are C-ordered [a][b][c][...] (atom, element block, padded neighbor
// slot, innermost index), which is the column-major Eigen layout the kernels
// use with the innermost index first.
#include <vector>

#include "tensor_ops.h"

using Eigen::Tensor;
using Eigen::TensorMap;

extern "C" int tmdr_pair_forces(int na, int nb, int nc, int nk, int nd, int nm,
                                int max_moment, const double *M, const double *H,
                                const double *dH, const double *u, const double *R,
                                const int *mask, const double *T, const double *G,
                                double *dEdG, double *P, double *S, double *F) {
  using T4 = TensorMap<Tensor<double, 4>>;
  T4 Mm(const_cast<double *>(M), nd, nc, nb, na);
  T4 Hm(const_cast<double *>(H), nk, nc, nb, na);
  T4 dHm(const_cast<double *>(dH), nk, nc, nb, na);
  T4 um(const_cast<double *>(u), 3, nc, nb, na);
  TensorMap<Tensor<double, 3>> Rm(const_cast<double *>(R), nc, nb, na);
  TensorMap<Tensor<int, 3>> maskm(const_cast<int *>(mask), nc, nb, na);
  T4 Pm(P, nd, nk, nb, na);
  kernel_P<double>(Mm, Hm, &Pm);
  T4 Gm(const_cast<double *>(G), nm, nk, nb, na);
  T4 dEdGm(dEdG, nm, nk, nb, na);
  kernel_dEdG<double>(Gm, &dEdGm);
  Tensor<double, 2> Tt(nm, nd);
  for (int m = 0; m < nm; m++)
    for (int d = 0; d < nd; d++) Tt(m, d) = T[m * nd + d];
  T4 Sm(S, nd, nk, nb, na);
  kernel_dEdS<double>(Tt, dEdGm, Pm, &Sm);
  Tensor<double, 4> U(nk, nc, nb, na);
  T4 Um(U.data(), nk, nc, nb, na);
  kernel_U<double>(Sm, Mm, &Um);
  std::vector<double> Vbuf((size_t)nd * nc * nb * na);
  T4 Vm(Vbuf.data(), nd, nc, nb, na);
  kernel_V<double>(Sm, Hm, &Vm);
  T4 F1(F, 3, nc, nb, na);
  kernel_F1<double>(U, dHm, um, maskm, &F1);
  Tensor<double, 4> F2(3, nc, nb, na);
  F2.setZero();
  kernel_fused_F2<double>(max_moment, Vm, Rm, um, maskm, &F2);
  const size_t nf = (size_t)3 * nc * nb * na;
  for (size_t i = 0; i < nf; i++) F[i] += F2.data()[i];
  return 0;
}
