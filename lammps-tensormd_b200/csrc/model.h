// model.h -- host description of a loaded tensormd potential.
#pragma once

#include <algorithm>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "npz.h"
#include "tmd_internal.h"

namespace tmd {

struct ModelError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

struct HostModel {
  std::string path;
  std::vector<std::string> type_elements;  // pair_coeff element per type
  std::vector<int> typemap;                // [ntypes+1], index 0 unused
  std::vector<double> typemass;
  double interp_dx = -1.0;
  int precision = 0;                       // TMD_PREC_*
  int file_precision = 64;
  double rmax = 0, rcsq = 0;
  int nelt = 0, mm = 0, K = 0, D = 0, M = 0, nin = 0;
  int fctype = 0, use_fnn = 0, method = 0, tsym = 0;
  std::vector<double> masses;
  std::vector<std::string> symbols;
  std::vector<double> p0, p1, p2;
  // rational table [tab_n][4][K]
  int tab_n = 0;
  double tab_dx = 0, tab_xdx = 0;
  std::vector<float> table;
  // MLP
  int nl = 0, actfn = 0, outbias = 0, resnet = 0;
  std::vector<int> sizes;                              // [nl+1]
  std::vector<std::vector<std::vector<float>>> W, Bs;  // [e][l]
  std::vector<std::vector<double>> Wout, Bout;         // [e] output layer, FP64
  // temperature-dependent model (tdnp = 1, tdnp.cpp): nets H, U, S replace
  // the MLP; etemp from pair_coeff (eV)
  struct Net {
    int nl = 0, actfn = 0, outbias = 0, resnet = 0;
    std::vector<int> sizes;                         // [nl+1]
    std::vector<std::vector<std::vector<double>>> W, B;  // [e][l], FP64 as read
  };
  int tdnp = 0, sommerfeld = 0, ydim = 0;
  double etemp = 0.0;
  Net tH, tU, tS;
};

// Parse "file.npz El1 El2 ... [interp dx] [cmax ...] [precision ...]" and the
// file.  Throws ModelError / std::runtime_error.
HostModel parse_model(const std::string &coeff_args);
// The MLP of the file (tdnp = 0) or its TDNP nets (tdnp = 1), into h.
void parse_nnp(const Npz &z, HostModel &h);
void parse_tdnp(const Npz &z, HostModel &h);

void fill_kparams(const HostModel &h, KParams &kp);

}  // namespace tmd
