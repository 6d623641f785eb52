// model.cpp -- potential file -> device model.
//
// Restates, on the host and once per pair_coeff:
//   PairTensorMD::coeff / setup_eltmap / read_potential_file
//                                  (pair_tensormd.cpp:214-317,349-399)
//   TensorMD::read_npz / setup_global (tensormd.cpp:109-280): T tensor,
//                                  element blocks eltij_pos
//   NeuralNetworkPotential::setup_global (nnp.cpp:110-205): residual rule
//   Descriptor (descriptor.h:45-85) and FeaturePotential::setup_ration
//   (fnn.cpp:77-105): FNN evaluated on the grid x_i = i*dx (bias + activation
//   only for softplus/squareplus as forward_fnn_GPU, nnp.cu:59-116), times
//   the cutoff, then BatchRation1d::setup (ration.hpp:166-225) coefficients.
#include "model.h"

#include <cmath>
#include <cstring>
#include <sstream>
#include <stdexcept>

namespace tmd {

namespace {

[[noreturn]] void bad(const std::string &m) { throw ModelError(m); }

const NpyArray &need(const Npz &z, const std::string &k) {
  auto it = z.find(k);
  if (it == z.end()) bad("potential file has no key '" + k + "'");
  return it->second;
}

bool has(const Npz &z, const std::string &k) { return z.find(k) != z.end(); }

template <typename S>
S act_host(int actfn, S z) {
  if (actfn == 1) {
    const S thr = std::log(std::numeric_limits<S>::epsilon()) + S(2);
    S ex = std::exp(z);
    return z < -thr ? std::log1p(ex) : z;
  }
  S q = std::sqrt(z * z + S(4));
  return S(0.5) * (z + q);
}

template <typename S>
S cutoff_host(int fctype, S rc, S r) {
  if (fctype == 0) {
    S z = std::min(r / rc, S(1)) * S(M_PI);
    return S(0.5) + S(0.5) * std::cos(z);
  }
  S g = 5;
  S z = std::min(r / rc, S(M_PI));
  S z4 = z * z * z * z, z5 = z4 * z;
  return S(1) + g * z5 * z - (g + S(1)) * z5;
}

// y[n][K] on the grid, already multiplied by the cutoff.
template <typename S>
std::vector<S> grid_values(const Npz &z, const HostModel &h, int n, S delta, int K) {
  std::vector<S> y((size_t)n * K);
  S rc = S(h.rmax);
  if (h.use_fnn) {
    int nl = need(z, "fnn::nlayers").iscalar();
    const auto &ls = need(z, "fnn::layer_sizes");
    std::vector<int> sizes{1};
    for (size_t i = 0; i < ls.size(); i++) sizes.push_back(int(ls.d[i]));
    if ((int)sizes.size() != nl + 1) bad("fnn::layer_sizes does not match fnn::nlayers");
    int act = need(z, "fnn::actfn").iscalar();
    int outb = need(z, "fnn::apply_output_bias").iscalar();
    int res_raw = need(z, "fnn::use_resnet_dt").iscalar();
    int n_res = 0;
    for (int i = 0; i < nl; i++)
      if (i > 0 && sizes[i] == sizes[i + 1]) n_res++;
    bool res = res_raw && n_res > 0;
    if (sizes[nl] != K) bad("fnn output width differs from fnn::num_filters");
    std::vector<std::vector<S>> W(nl), Bv(nl);
    for (int l = 0; l < nl; l++) {
      const auto &w = need(z, "fnn::weights_0_" + std::to_string(l));
      if ((int)w.size() != sizes[l] * sizes[l + 1]) bad("fnn weight shape mismatch");
      W[l].assign(w.d.begin(), w.d.end());
      if (l < nl - 1 || outb) {
        const auto &b = need(z, "fnn::biases_0_" + std::to_string(l));
        Bv[l].assign(b.d.begin(), b.d.end());
      }
    }
    int maxw = *std::max_element(sizes.begin(), sizes.end());
    std::vector<S> a(maxw), o(maxw);
    for (int i = 0; i < n; i++) {
      S xi = S(i) * delta;
      a[0] = xi;
      for (int l = 0; l < nl; l++) {
        int Kl = sizes[l], Nl = sizes[l + 1];
        for (int c = 0; c < Nl; c++) {
          S s = 0;
          for (int k = 0; k < Kl; k++) s += a[k] * W[l][(size_t)k * Nl + c];
          if (l < nl - 1) {
            if (act == 1 || act == 3) {
              s += Bv[l][c];
              s = act_host<S>(act, s);
              if (l > 0 && res && Kl == Nl) s += a[c];
            }
          } else if (outb) {
            s += Bv[l][c];
          }
          o[c] = s;
        }
        std::swap(a, o);
      }
      S fc = cutoff_host<S>(h.fctype, rc, xi);
      for (int k = 0; k < K; k++) y[(size_t)i * K + k] = a[k] * fc;
    }
  } else {
    for (int i = 0; i < n; i++) {
      S r = S(i) * delta;
      S fc = cutoff_host<S>(h.fctype, rc, r);
      for (int k = 0; k < K; k++) {
        S a = S(h.p0[k]), b = S(h.p1[k]), c = S(h.p2[k]), f;
        switch (h.method) {
          case 0: f = std::exp(-std::pow(r / a, b)); break;
          case 1: {
            S gdr = b * (r - c);
            f = a * (std::exp(-2 * gdr) - 2 * std::exp(-gdr));
            break;
          }
          case 2: f = a * std::exp(-b * ((r - c) / c)); break;
          default: f = std::exp(-a * (r - b) * (r - b) / (rc * rc)); break;
        }
        y[(size_t)i * K + k] = f * fc;
      }
    }
  }
  return y;
}

template <typename S>
void build_table_t(const Npz &z, HostModel &h, double dx_in) {
  S delta = S(dx_in);
  S rmax = S(h.rmax);
  int n = int(rmax / delta) + 1;
  if (n < 4) bad("interp dx is too large for the cutoff");
  const int K = h.K;
  std::vector<S> y = grid_values<S>(z, h, n, delta, K);
  S xdx = S(1) / delta;
  std::vector<S> s((size_t)n * K, S(0)), c1((size_t)n * K, S(0)), c2((size_t)n * K, S(0));
  for (int i = 0; i < n - 1; i++)
    for (int k = 0; k < K; k++)
      s[(size_t)i * K + k] = (y[(size_t)(i + 1) * K + k] - y[(size_t)i * K + k]) * xdx;
  for (int i = 0; i < n - 1; i++) {
    for (int k = 0; k < K; k++) {
      S si = s[(size_t)i * K + k];
      if (i == 0) {
        S sp = s[(size_t)(i + 1) * K + k];
        c1[(size_t)i * K + k] = 0;
        c2[(size_t)i * K + k] =
            (si * (si - (sp - si) / 2) <= 0) ? si * xdx : (sp - si) * xdx / 2;
      } else if (i == n - 2) {
        S sm = s[(size_t)(i - 1) * K + k];
        c1[(size_t)i * K + k] = (si - sm) * xdx / 2;
        c2[(size_t)i * K + k] = 0;
      } else {
        S sm = s[(size_t)(i - 1) * K + k], sp = s[(size_t)(i + 1) * K + k];
        if (i == 1 && sm * (sm - (si - sm) / 2) <= 0)
          c1[(size_t)i * K + k] = (si - 2 * sm) * xdx;
        else
          c1[(size_t)i * K + k] = (si - sm) * xdx / 2;
        c2[(size_t)i * K + k] = (sp - si) * xdx / 2;
      }
    }
  }
  h.tab_n = n;
  h.tab_dx = double(delta);
  h.tab_xdx = 1.0 / double(delta);
  h.table.assign((size_t)n * 4 * K, 0.f);
  for (int i = 0; i < n; i++)
    for (int k = 0; k < K; k++) {
      size_t b = (size_t)i * 4 * K;
      h.table[b + k] = float(y[(size_t)i * K + k]);
      h.table[b + K + k] = float(s[(size_t)i * K + k]);
      h.table[b + 2 * K + k] = float(c1[(size_t)i * K + k]);
      h.table[b + 3 * K + k] = float(c2[(size_t)i * K + k]);
    }
}

std::vector<std::string> split_ws(const std::string &s) {
  std::istringstream is(s);
  std::vector<std::string> v;
  std::string t;
  while (is >> t) v.push_back(t);
  return v;
}

}  // namespace

HostModel parse_model(const std::string &coeff_args) {
  HostModel h;
  auto tok = split_ws(coeff_args);
  if (tok.empty()) bad("pair_coeff needs a potential file");
  // PairTensorMD::coeff accepts "* *" in front; tolerate it here.
  size_t i0 = 0;
  if (tok.size() >= 2 && tok[0] == "*" && tok[1] == "*") i0 = 2;
  if (i0 >= tok.size()) bad("pair_coeff needs a potential file");
  h.path = tok[i0];
  bool read_elt = true;
  for (size_t i = i0 + 1; i < tok.size();) {
    const std::string &v = tok[i];
    auto value = [&](const char *kw) -> std::string {
      if (i + 1 >= tok.size()) bad(std::string("pair_coeff keyword ") + kw + " needs a value");
      return tok[i + 1];
    };
    if (v == "interp") {
      h.interp_dx = std::strtod(value("interp").c_str(), nullptr);
      if (!(h.interp_dx > 0)) bad("interp dx must be > 0");
      read_elt = false;
      i += 2;
    } else if (v == "etemp") {
      // electron temperature in K, kept in eV (pair_tensormd.cpp:33,245-246)
      h.etemp = std::strtod(value("etemp").c_str(), nullptr) / 11604.522060401008;
      if (!(h.etemp >= 0)) bad("etemp must be >= 0");
      read_elt = false;
      i += 2;
    } else if (v == "cmax") {
      std::string c = value("cmax");
      if (c != "exact" && c != "default") bad("Unknown option for cmax");
      read_elt = false;
      i += 2;
    } else if (v == "precision") {
      std::string c = value("precision");
      if (c == "fp32") h.precision = 0;
      else if (c == "bf16") h.precision = 1;
      else if (c == "fp8") h.precision = 2;
      else if (c == "bf16x3") h.precision = 3;
      else if (c == "tf32x3") h.precision = 4;
      else bad("precision must be fp32, tf32x3, bf16, bf16x3 or fp8");
      read_elt = false;
      i += 2;
    } else if (read_elt) {
      h.type_elements.push_back(v);
      i++;
    } else {
      bad("unexpected pair_coeff argument '" + v + "'");
    }
  }
  if (h.type_elements.empty()) bad("Incorrect args for pair coefficients");

  Npz z = load_npz(h.path);
  h.file_precision = has(z, "precision") ? need(z, "precision").iscalar() : 64;
  h.tdnp = has(z, "tdnp") && need(z, "tdnp").iscalar() == 1;
  if (h.tdnp && h.precision != 0)
    bad("TDNP potentials run the plain FP32 form (no precision keyword)");
  h.rmax = need(z, "rmax").scalar();
  h.nelt = need(z, "nelt").iscalar();
  h.mm = need(z, "max_moment").iscalar();
  if (h.nelt < 1 || h.nelt > kMaxElt) bad("nelt out of range");
  if (h.mm < 0 || h.mm > 3) bad("max_moment > 3 is not supported");
  const auto &ms = need(z, "masses");
  h.masses.assign(ms.d.begin(), ms.d.end());
  if ((int)h.masses.size() < h.nelt) bad("masses has fewer entries than nelt");
  const auto &num = need(z, "numbers");
  for (int e = 0; e < h.nelt; e++) {
    std::string s;
    size_t i = 2 * e;
    if (i < num.size()) s.push_back(char(int(num.d[i])));
    if (i + 1 < num.size() && num.d[i + 1] > 0) s.push_back(char(int(num.d[i + 1])));
    h.symbols.push_back(s);
  }
  // PairTensorMD::setup_eltmap: LAMMPS type t -> potential element
  h.typemap.assign(h.type_elements.size() + 1, -1);
  h.typemass.assign(h.type_elements.size() + 1, 0.0);
  for (size_t t = 0; t < h.type_elements.size(); t++) {
    if (h.type_elements[t] == "NULL") continue;
    for (int e = 0; e < h.nelt; e++)
      if (h.type_elements[t] == h.symbols[e]) {
        h.typemap[t + 1] = e;
        h.typemass[t + 1] = h.masses[e];
      }
    if (h.typemap[t + 1] < 0)
      bad("element " + h.type_elements[t] + " is not in the potential file");
  }
  h.fctype = need(z, "fctype").iscalar();
  h.use_fnn = need(z, "use_fnn").iscalar();
  h.tsym = has(z, "is_T_symmetric") && need(z, "is_T_symmetric").iscalar() == 1;
  if (h.use_fnn) {
    h.K = need(z, "fnn::num_filters").iscalar();
    if (!(h.interp_dx > 0))
      bad("an FNN radial basis needs 'interp dx' (the reference only evaluates it "
          "through the interpolation table)");
  } else {
    h.method = has(z, "descriptor::method") ? need(z, "descriptor::method").iscalar() : 0;
    const char *names[4][3] = {{"descriptor::rl", "descriptor::pl", nullptr},
                               {"descriptor::D", "descriptor::gamma", "descriptor::r0"},
                               {"descriptor::A", "descriptor::beta", "descriptor::re"},
                               {"descriptor::eta", "descriptor::omega", nullptr}};
    if (h.method < 0 || h.method > 3) bad("descriptor::method out of range");
    const auto &a0 = need(z, names[h.method][0]);
    h.K = (int)a0.size();
    h.p0.assign(a0.d.begin(), a0.d.end());
    const auto &a1 = need(z, names[h.method][1]);
    h.p1.assign(a1.d.begin(), a1.d.end());
    if (names[h.method][2]) {
      const auto &a2 = need(z, names[h.method][2]);
      h.p2.assign(a2.d.begin(), a2.d.end());
    } else {
      h.p2.assign(h.K, 0.0);
    }
  }
  if (h.K < 4 || h.K > kMaxK || (h.K & 3) || ((h.K / 4) & (h.K / 4 - 1)))
    bad("num_filters must be 4 * 2^j with 4 <= k <= 128 (got " + std::to_string(h.K) + ")");
  static const int nv[4] = {1, 4, 10, 20};
  h.D = nv[h.mm];
  h.M = h.mm + 1;
  if (h.tdnp) {
    parse_tdnp(z, h);
  } else {
    parse_nnp(z, h);
  }
  if (h.interp_dx > 0) {
    if (h.file_precision == 32)
      build_table_t<float>(z, h, h.interp_dx);
    else
      build_table_t<double>(z, h, h.interp_dx);
  }
  // cutforcesq is a Scalar in TensorMD<Scalar> (tensormd.h:80)
  if (h.file_precision == 32) {
    float r = float(h.rmax);
    h.rcsq = double(r * r);
  } else {
    h.rcsq = h.rmax * h.rmax;
  }
  return h;
}

namespace {
// The NNP of a tdnp = 0 file (nnp.cpp:110-145).
void parse_nnp_impl(const Npz &z, HostModel &h) {
  h.nl = need(z, "nlayers").iscalar();
  h.actfn = need(z, "actfn").iscalar();
  h.outbias = need(z, "apply_output_bias").iscalar();
  int res_raw = need(z, "use_resnet_dt").iscalar();
  const auto &ls = need(z, "layer_sizes");
  if ((int)ls.size() != h.nl || h.nl < 2 || h.nl > kMaxLayers)
    bad("layer_sizes / nlayers unsupported (need 2..12 layers)");
  const auto &w00 = need(z, "weights_0_0");
  h.nin = w00.shape.empty() ? 1 : (int)w00.shape[0];
  if (h.nin != h.nelt * h.K * h.M)
    bad("weights_0_0 rows (" + std::to_string(h.nin) + ") != nelt*k*m");
  h.sizes.assign(1, h.nin);
  for (size_t i = 0; i < ls.size(); i++) h.sizes.push_back(int(ls.d[i]));
  if (h.sizes[h.nl] != 1) bad("only one MLP output (atomic energy) is supported");
  for (int l = 1; l < h.nl; l++)
    if (h.sizes[l] > 512) bad("hidden layers wider than 512 are not supported");
  if (h.nin > 1024) bad("descriptor width above 1024 is not supported");
  int n_res = 0;
  for (int l = 0; l < h.nl; l++)
    if (l > 0 && h.sizes[l] == h.sizes[l + 1]) n_res++;
  h.resnet = (res_raw && n_res > 0) ? 1 : 0;
  h.W.assign(h.nelt, std::vector<std::vector<float>>(h.nl));
  h.Bs.assign(h.nelt, std::vector<std::vector<float>>(h.nl));
  h.Wout.assign(h.nelt, {});
  h.Bout.assign(h.nelt, {});
  for (int e = 0; e < h.nelt; e++)
    for (int l = 0; l < h.nl; l++) {
      const auto &w = need(z, "weights_" + std::to_string(e) + "_" + std::to_string(l));
      if ((int)w.size() != h.sizes[l] * h.sizes[l + 1])
        bad("weights_" + std::to_string(e) + "_" + std::to_string(l) + " has a wrong shape");
      h.W[e][l].assign(w.d.begin(), w.d.end());
      if (l == h.nl - 1) h.Wout[e] = w.d;
      if (l < h.nl - 1 || h.outbias) {
        const auto &b = need(z, "biases_" + std::to_string(e) + "_" + std::to_string(l));
        if ((int)b.size() != h.sizes[l + 1]) bad("bias shape mismatch");
        h.Bs[e][l].assign(b.d.begin(), b.d.end());
        if (l == h.nl - 1) h.Bout[e] = b.d;
      }
    }
}

// The H, U, S nets of a tdnp = 1 file (tdnp.cpp:46-139): H maps the
// descriptor to ydim - 1 values, to which the reference appends the
// electron temperature (a zero weight column, tdnp.cpp:80-97); U and S map
// the ydim values to an atom's internal energy and entropy.
void parse_net(const Npz &z, const HostModel &h, const std::string &sc, int n_in,
               HostModel::Net &t) {
  t.nl = need(z, sc + "::nlayers").iscalar();
  t.actfn = need(z, sc + "::actfn").iscalar();
  t.outbias = need(z, sc + "::apply_output_bias").iscalar();
  const int res_raw = need(z, sc + "::use_resnet_dt").iscalar();
  const auto &ls = need(z, sc + "::layer_sizes");
  if ((int)ls.size() != t.nl || t.nl < 1 || t.nl > kMaxLayers)
    bad(sc + "::layer_sizes / nlayers unsupported");
  t.sizes.assign(1, n_in);
  for (size_t i = 0; i < ls.size(); i++) t.sizes.push_back(int(ls.d[i]));
  for (int l = 0; l <= t.nl; l++)
    if (t.sizes[l] < 1 || t.sizes[l] > 1024) bad(sc + " layer widths must be 1..1024");
  int n_res = 0;
  for (int l = 1; l < t.nl; l++)
    if (t.sizes[l] == t.sizes[l + 1]) n_res++;
  t.resnet = (res_raw && n_res > 0) ? 1 : 0;
  t.W.assign(h.nelt, std::vector<std::vector<double>>(t.nl));
  t.B.assign(h.nelt, std::vector<std::vector<double>>(t.nl));
  for (int e = 0; e < h.nelt; e++)
    for (int l = 0; l < t.nl; l++) {
      const std::string key = "_" + std::to_string(e) + "_" + std::to_string(l);
      const auto &w = need(z, sc + "::weights" + key);
      if ((int)w.size() != t.sizes[l] * t.sizes[l + 1]) bad(sc + "::weights" + key + " has a wrong shape");
      t.W[e][l] = w.d;
      if (l < t.nl - 1 || t.outbias) {
        const auto &b = need(z, sc + "::biases" + key);
        if ((int)b.size() != t.sizes[l + 1]) bad(sc + "::biases" + key + " has a wrong shape");
        t.B[e][l] = b.d;
      }
    }
}

void parse_tdnp_impl(const Npz &z, HostModel &h) {
  h.sommerfeld = has(z, "tdnp::Sommerfeld") && need(z, "tdnp::Sommerfeld").iscalar() == 1;
  const auto &w00 = need(z, "H::weights_0_0");
  h.nin = w00.shape.empty() ? 1 : (int)w00.shape[0];
  if (h.nin != h.nelt * h.K * h.M) bad("H::weights_0_0 rows != nelt*k*m");
  parse_net(z, h, "H", h.nin, h.tH);
  h.ydim = h.tH.sizes[h.tH.nl] + 1;
  // the temperature column: zero weights and bias
  const int L = h.tH.nl, K = h.tH.sizes[L - 1], N = h.ydim - 1;
  for (int e = 0; e < h.nelt; e++) {
    std::vector<double> w((size_t)K * (N + 1), 0.0);
    for (int k = 0; k < K; k++)
      for (int n = 0; n < N; n++) w[(size_t)k * (N + 1) + n] = h.tH.W[e][L - 1][(size_t)k * N + n];
    h.tH.W[e][L - 1] = w;
    if (!h.tH.B[e][L - 1].empty()) h.tH.B[e][L - 1].push_back(0.0);
  }
  h.tH.sizes[L] = h.ydim;
  parse_net(z, h, "U", h.ydim, h.tU);
  parse_net(z, h, "S", h.ydim, h.tS);
  if ((int)need(z, "U::weights_0_0").shape[0] != h.ydim ||
      (int)need(z, "S::weights_0_0").shape[0] != h.ydim)
    bad("U and S must take the ydim outputs of H (with the temperature column)");
}
}  // namespace

void parse_nnp(const Npz &z, HostModel &h) { parse_nnp_impl(z, h); }
void parse_tdnp(const Npz &z, HostModel &h) { parse_tdnp_impl(z, h); }


void fill_kparams(const HostModel &h, KParams &kp) {
  std::memset(&kp, 0, sizeof(kp));
  kp.K = h.K;
  kp.D = h.D;
  kp.M = h.M;
  kp.B = h.nelt;
  kp.nin = h.nin;
  kp.radial = h.interp_dx > 0 ? 1 : 0;
  kp.method = h.method;
  kp.fctype = h.fctype;
  kp.rc = float(h.rmax);
  kp.inv_rc = float(1.0 / h.rmax);
  kp.inv_rc2 = float(1.0 / (h.rmax * h.rmax));
  kp.rcsq = h.rcsq;
  // T tensor (tensormd.cpp:202-233), stored T[m*D + d]
  const int D = h.D;
  auto T = [&](int m, int d) -> float & { return kp.T[m * D + d]; };
  T(0, 0) = 1;
  if (h.mm > 0) { T(1, 1) = 1; T(1, 2) = 1; T(1, 3) = 1; }
  if (h.mm > 1) {
    const float t2[6] = {1, 2, 2, 1, 2, 1};
    for (int i = 0; i < 6; i++) T(2, 4 + i) = t2[i];
    if (h.tsym) T(2, 0) = float(-1.0 / 3.0);
  }
  if (h.mm > 2) {
    const float t3[10] = {1, 3, 3, 3, 6, 3, 1, 3, 3, 1};
    for (int i = 0; i < 10; i++) T(3, 10 + i) = t3[i];
    if (h.tsym) { T(3, 1) = T(3, 2) = T(3, 3) = float(-3.0 / 5.0); }
  }
  for (int k = 0; k < h.K; k++) {
    if (!h.p0.empty()) kp.p0[k] = float(h.p0[k]);
    if (!h.p1.empty()) {
      kp.p1[k] = float(h.p1[k]);
      kp.p1lo[k] = float(h.p1[k] - double(kp.p1[k]));
    }
    if (!h.p2.empty()) kp.p2[k] = float(h.p2[k]);
    if (!h.p0.empty()) {
      kp.gc[k] = float(h.p0[k] / (h.rmax * h.rmax));
      kp.gcl[k] = float(h.p0[k] / (h.rmax * h.rmax) * 1.4426950408889634);  // log2(e)
    }
  }
  // element blocks: tensormd.cpp:165-176
  for (int i = 0; i < h.nelt; i++) {
    int k = 1;
    for (int j = 0; j < h.nelt; j++) kp.eltij[i * kMaxElt + j] = (i == j) ? 0 : k++;
  }
  kp.tab_n = h.tab_n;
  kp.tab_dx = float(h.tab_dx);
  kp.tab_dxd = h.tab_dx;
  kp.tab_xdxd = h.tab_xdx;
}

}  // namespace tmd
