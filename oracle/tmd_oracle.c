/* tmd_oracle.c -- FP64 CPU restatement of the pair_style tensormd force path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * product path in lammps-tensormd_b200/.  Only tests/, __graft_entry__.smoke()
 * and the cpu_baseline leg of bench.py may load it.  The product never links
 * or calls it.
 *
 * What it restates (reference paths relative to the lammps-tensormd tree):
 *   neighbor list      src/npair_full_bin_atomonly.cpp:32-92 (full list,
 *                      rsq <= cutneighsq, i != j), ghosts as periodic images
 *                      whose coordinates follow AtomVec::pack_border's
 *                      x + pbc*prd per communication hop (x, then y, then z)
 *   pair geometry      src/ML-TENSORMD/gpu/cuda/kernel.cu:1149-1176
 *                      (rij2 < rc^2 && rij2 > 1e-10, dij = x_j - x_i)
 *   monomials M_d      kernel.cu:1197-1232 (order 1,x,y,z,xx,xy,xz,yy,...)
 *   element blocks     src/ML-TENSORMD/tensormd.cpp:165-176
 *   T tensor           tensormd.cpp:202-276
 *   radial functions   src/ML-TENSORMD/descriptor.cpp:51-138,
 *                      cutoff.cpp:20-37
 *   rational table     src/ML-TENSORMD/gpu/cuda/ration.cu:12-71
 *                      (table built by oracle/pack.py from ration.hpp:166-225)
 *   P, G               tensor_ops.cpp:601-627, kernel.cu:1028-1061
 *   MLP fwd/bwd        src/ML-TENSORMD/gpu/cuda/nnp.cu:9-57,149-281,
 *                      nnp.cpp:246-365, activation.hpp:114-261
 *   dE/dG -> dE/dP     tensor_ops.cpp:633-674, kernel.cu:775-817
 *   F1, F2 (dE_i/dx_j) tensor_ops.cpp:126-190,262-535
 *   force/virial sign  kernel.cu:1714-1758 (f_i += df, f_j -= df,
 *                      vatom += 0.5 * (-r_ij (x) df) on i and j)
 *   fix nve            src/fix_nve.cpp:64-141, metal units update.cpp:187-206
 *
 * dM is written in closed form: for a monomial M of degree n in the unit
 * vector u = d/r, dM/dx_j[b] = (dM/du_b - n * u_b * M) / r, which reproduces
 * the tables of tensor_ops.cpp calculate_dM_{p,d,f} term by term.
 *
 * ReLU: the reference's CPU ReLU derivative is evaluated on the clamped
 * output and is therefore always 1 (activation.hpp:158-177); this oracle
 * uses the mathematical derivative (1 for z > 0, else 0).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OM_MAXL 16
#define OM_MAXE 8
#define OM_MAXD 20

/* One MLP of a TDNP model (tdnp.cpp setup_one): weights W[e][l] (K x N,
 * row-major), biases b[e][l] (NULL for a last layer without output bias). */
typedef struct {
  int nl, actfn, resnet, outbias;
  int sizes[OM_MAXL + 1];
  const double *W[OM_MAXE][OM_MAXL], *b[OM_MAXE][OM_MAXL];
} om_net;

typedef struct {
  int nelt, max_moment, K, D, M, fctype, radial, desc_method, tsym;
  int nl, actfn, resnet, outbias, n_in, tab_n;
  int sizes[OM_MAXL + 1];
  double rmax, tab_dx;
  double T[4 * OM_MAXD];
  const double *dp0, *dp1, *dp2, *tab;
  const double *W[OM_MAXE][OM_MAXL], *b[OM_MAXE][OM_MAXL];
  double *store;
  /* temperature-dependent model (tdnp.cpp): H maps G to y (ydim values, the
   * last one the electron temperature), U and S map y to the atom's internal
   * energy and entropy; the forces are those of A = U - T S */
  int tdnp, sommerfeld, ydim;
  double etemp;                  /* eV */
  om_net H, U, S;
  double *tstore;
  double tdnp_S, tdnp_A;         /* totals of the last compute */
} om_model;

/* exponents (ax, ay, az) of monomial d, order of kernel.cu:1197-1232 */
static const int om_exp[OM_MAXD][3] = {
    {0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {1, 1, 0}, {1, 0, 1},
    {0, 2, 0}, {0, 1, 1}, {0, 0, 2}, {3, 0, 0}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0},
    {1, 1, 1}, {1, 0, 2}, {0, 3, 0}, {0, 2, 1}, {0, 1, 2}, {0, 0, 3}};

static void om_set_T(om_model *m)
{
  /* tensormd.cpp:202-233 */
  memset(m->T, 0, sizeof(m->T));
  double *T = m->T;
  int D = m->D;
  T[0 * D + 0] = 1;
  if (m->max_moment > 0) {
    T[1 * D + 1] = T[1 * D + 2] = T[1 * D + 3] = 1;
  }
  if (m->max_moment > 1) {
    const double t2[6] = {1, 2, 2, 1, 2, 1};
    for (int i = 0; i < 6; i++) T[2 * D + 4 + i] = t2[i];
    if (m->tsym) T[2 * D + 0] = -1.0 / 3.0;
  }
  if (m->max_moment > 2) {
    const double t3[10] = {1, 3, 3, 3, 6, 3, 1, 3, 3, 1};
    for (int i = 0; i < 10; i++) T[3 * D + 10 + i] = t3[i];
    if (m->tsym) T[3 * D + 1] = T[3 * D + 2] = T[3 * D + 3] = -3.0 / 5.0;
  }
}

/* Blob layout: see oracle/pack.py (pack_model). */
void *tmdo_model_new(const int *ib, int ni, const double *db, int nd)
{
  (void)ni;
  om_model *m = (om_model *)calloc(1, sizeof(om_model));
  if (!m) return NULL;
  m->nelt = ib[1];
  m->max_moment = ib[2];
  m->K = ib[3];
  m->fctype = ib[4];
  m->radial = ib[5];
  m->desc_method = ib[6];
  m->tsym = ib[7];
  m->nl = ib[8];
  m->actfn = ib[9];
  int resnet_raw = ib[10];
  m->outbias = ib[11];
  m->n_in = ib[12];
  m->tab_n = ib[13];
  if (m->max_moment < 0 || m->max_moment > 3 || m->nelt > OM_MAXE ||
      m->nl > OM_MAXL) {
    free(m);
    return NULL;
  }
  m->sizes[0] = m->n_in;
  for (int l = 0; l < m->nl; l++) m->sizes[l + 1] = ib[14 + l];
  /* nnp.cpp:176-181: residual only when some hidden layer keeps its width */
  int n_res = 0;
  for (int l = 0; l < m->nl; l++)
    if (l > 0 && m->sizes[l] == m->sizes[l + 1]) n_res++;
  m->resnet = (resnet_raw && n_res > 0) ? 1 : 0;
  static const int nv[4] = {1, 4, 10, 20};
  m->D = nv[m->max_moment];
  m->M = m->max_moment + 1;
  om_set_T(m);

  m->store = (double *)malloc(sizeof(double) * (size_t)nd);
  memcpy(m->store, db, sizeof(double) * (size_t)nd);
  const double *p = m->store;
  m->rmax = *p++;
  m->tab_dx = *p++;
  m->dp0 = p; p += m->K;
  m->dp1 = p; p += m->K;
  m->dp2 = p; p += m->K;
  m->tab = p; p += (size_t)m->tab_n * 4 * m->K;
  for (int e = 0; e < m->nelt; e++)
    for (int l = 0; l < m->nl; l++) {
      m->W[e][l] = p;
      p += (size_t)m->sizes[l] * m->sizes[l + 1];
      if (l < m->nl - 1 || m->outbias) {
        m->b[e][l] = p;
        p += m->sizes[l + 1];
      } else {
        m->b[e][l] = NULL;
      }
    }
  return m;
}

void tmdo_model_free(void *h)
{
  om_model *m = (om_model *)h;
  if (!m) return;
  free(m->store);
  free(m->tstore);
  free(m);
}

/* TDNP nets (blob of oracle/pack.py pack_tdnp): ints = [sommerfeld, ydim,
 * then per net H, U, S: nl, actfn, resnet_raw, outbias, sizes[0..nl]];
 * doubles = per net, element, layer: W (sizes[l] x sizes[l+1]) and, for
 * hidden layers or with the output bias, b.  H's last layer has ydim
 * outputs, the last column zero (tdnp.cpp:80-97). */
int tmdo_model_set_tdnp(void *h, const int *ib, int ni, const double *db, int nd)
{
  (void)ni;
  om_model *m = (om_model *)h;
  m->tdnp = 1;
  m->sommerfeld = ib[0];
  m->ydim = ib[1];
  m->tstore = (double *)malloc(sizeof(double) * (size_t)(nd > 0 ? nd : 1));
  memcpy(m->tstore, db, sizeof(double) * (size_t)nd);
  const int *q = ib + 2;
  const double *p = m->tstore;
  om_net *nets[3] = {&m->H, &m->U, &m->S};
  for (int k = 0; k < 3; k++) {
    om_net *t = nets[k];
    t->nl = *q++;
    t->actfn = *q++;
    int res_raw = *q++;
    t->outbias = *q++;
    if (t->nl < 1 || t->nl > OM_MAXL) return -1;
    for (int l = 0; l <= t->nl; l++) t->sizes[l] = *q++;
    int n_res = 0;
    for (int l = 1; l < t->nl; l++)
      if (t->sizes[l] == t->sizes[l + 1]) n_res++;
    t->resnet = (res_raw && n_res > 0) ? 1 : 0;
    for (int e = 0; e < m->nelt; e++)
      for (int l = 0; l < t->nl; l++) {
        t->W[e][l] = p;
        p += (size_t)t->sizes[l] * t->sizes[l + 1];
        if (l < t->nl - 1 || t->outbias) {
          t->b[e][l] = p;
          p += t->sizes[l + 1];
        } else {
          t->b[e][l] = NULL;
        }
      }
  }
  return 0;
}

void tmdo_set_etemp(void *h, double etemp_ev) { ((om_model *)h)->etemp = etemp_ev; }

void tmdo_tdnp_totals(void *h, double *out)
{
  om_model *m = (om_model *)h;
  out[0] = m->tdnp_S;
  out[1] = m->tdnp_A;
}

int tmdo_model_dims(void *h, int *out)
{
  om_model *m = (om_model *)h;
  out[0] = m->K;
  out[1] = m->D;
  out[2] = m->M;
  out[3] = m->nelt;
  out[4] = m->n_in;
  out[5] = m->resnet;
  return 0;
}

/* ------------------------------------------------------------------ */
/* radial basis H_k(r), dH_k/dr                                        */
/* ------------------------------------------------------------------ */

static void om_cutoff(const om_model *m, double r, double *s, double *ds)
{
  double rc = m->rmax;
  if (m->fctype == 0) { /* cutoff.cpp:28-37 */
    double z = r / rc;
    if (z > 1.0) z = 1.0;
    z *= M_PI;
    *s = 0.5 + 0.5 * cos(z);
    *ds = -0.5 * M_PI * sin(z) / rc;
  } else { /* polynomial, gamma = 5 (tensormd.cpp:161) */
    double g = 5.0;
    double z = r / rc;
    if (z > M_PI) z = M_PI;
    double z4 = z * z * z * z, z5 = z4 * z;
    *s = 1 + g * z5 * z - (g + 1) * z5;
    *ds = (g + 1) * g / rc * (z5 - z4);
  }
}

static void om_radial(const om_model *m, double r, double *H, double *dH)
{
  int K = m->K;
  if (m->radial == 1) {
    /* rational-interpolation table, ration.cu:27-69 with
     * endpoints_force_zero = true (ration.hpp:29) */
    double dx = m->tab_dx, xdx = 1.0 / dx;
    int i = (int)(r * xdx);
    if (i > m->tab_n - 2) i = m->tab_n - 2;
    double q = r - i * dx;
    double rr = dx - q;
    if (i == 0 || i == m->tab_n - 2) {
      for (int k = 0; k < K; k++) H[k] = dH[k] = 0.0;
      return;
    }
    const double *py = m->tab + ((size_t)i * 4 + 0) * K;
    const double *ps = m->tab + ((size_t)i * 4 + 1) * K;
    const double *pc1 = m->tab + ((size_t)i * 4 + 2) * K;
    const double *pc2 = m->tab + ((size_t)i * 4 + 3) * K;
    for (int k = 0; k < K; k++) {
      double s = ps[k], c1 = pc1[k], c2 = pc2[k];
      double c3 = fabs(c2 * rr);
      double c4 = c3 + fabs(c1 * q);
      if (c4 > 0.0) c3 /= c4;
      c4 = c2 + c3 * (c1 - c2);
      H[k] = py[k] + q * (s - rr * c4);
      dH[k] = s + (q - rr) * c4 + dx * (c4 - c2) * (1 - c3);
    }
    return;
  }
  double s, ds;
  om_cutoff(m, r, &s, &ds);
  double rc2 = m->rmax * m->rmax;
  for (int k = 0; k < K; k++) {
    double f, df;
    double a = m->dp0[k], b = m->dp1[k], c = m->dp2[k];
    switch (m->desc_method) {
      case 0: { /* power-exponential, descriptor.cpp:57-68 */
        double x = r / a;
        f = exp(-pow(x, b));
        df = -f * b * pow(x, b - 1.0) / a;
        break;
      }
      case 1: { /* Morse, descriptor.cpp:78-92 */
        double gdr = b * (r - c);
        double e1 = exp(-gdr), e2 = exp(-2 * gdr);
        f = a * (e2 - 2 * e1);
        df = -a * b * 2 * (e2 - e1);
        break;
      }
      case 2: { /* density, descriptor.cpp:102-115 */
        double z = -b * ((r - c) / c);
        f = a * exp(z);
        df = -f * b / c;
        break;
      }
      default: { /* SF Gaussian, descriptor.cpp:125-137 */
        double dxr = r - b;
        f = exp(-a * dxr * dxr / rc2);
        df = -2.0 * a / rc2 * dxr * f;
        break;
      }
    }
    H[k] = s * f;
    dH[k] = ds * f + s * df;
  }
}

/* monomials M_d(u) and dM_d/dx_j (layout dM[x * D + d]) */
static void om_moments(int D, double ux, double uy, double uz, double rinv,
                       double *Mv, double *dM)
{
  double u[3] = {ux, uy, uz};
  for (int d = 0; d < D; d++) {
    const int *e = om_exp[d];
    double v = 1.0;
    for (int c = 0; c < 3; c++)
      for (int t = 0; t < e[c]; t++) v *= u[c];
    Mv[d] = v;
    if (!dM) continue;
    int n = e[0] + e[1] + e[2];
    for (int bdir = 0; bdir < 3; bdir++) {
      double g = 0.0;
      if (e[bdir] > 0) {
        g = (double)e[bdir];
        for (int c = 0; c < 3; c++) {
          int pw = e[c] - (c == bdir ? 1 : 0);
          for (int t = 0; t < pw; t++) g *= u[c];
        }
      }
      dM[bdir * D + d] = (g - n * u[bdir] * v) * rinv;
    }
  }
}

/* ------------------------------------------------------------------ */
/* MLP                                                                */
/* ------------------------------------------------------------------ */

static double om_act(int actfn, double z, double *dz)
{
  switch (actfn) {
    case 0: /* ReLU */
      *dz = z > 0 ? 1.0 : 0.0;
      return z > 0 ? z : 0.0;
    case 1: { /* softplus, nnp.cu:23-35 */
      double ex = exp(z);
      double thr = log(2.220446049250313e-16) + 2.0;
      double y = z;
      if (z < -thr) y = log1p(ex);
      *dz = 1.0 / (1.0 + 1.0 / ex);
      return y;
    }
    case 2: { /* tanh, activation.hpp:225-238 */
      double y = tanh(z);
      *dz = 1.0 - y * y;
      return y;
    }
    default: { /* squareplus, nnp.cu:9-21 */
      double q = sqrt(z * z + 4.0);
      double y = 0.5 * (z + q);
      *dz = y / q;
      return y;
    }
  }
}

/* E = MLP_e(g); grad = dE/dg.  work holds (nl+1) * maxw * 2 doubles. */
static double om_mlp(const om_model *m, int e, const double *g, double *grad,
                     double *work, int maxw)
{
  int L = m->nl;
  double *act = work;                            /* act[l] : input of layer l */
  double *dz = work + (size_t)(L + 1) * maxw;    /* act'(z) of layer l */
  memcpy(act, g, sizeof(double) * m->n_in);
  double E = 0.0;
  for (int l = 0; l < L; l++) {
    int Kl = m->sizes[l], Nl = m->sizes[l + 1];
    const double *W = m->W[e][l], *b = m->b[e][l];
    double *x = act + (size_t)l * maxw, *y = act + (size_t)(l + 1) * maxw;
    double *d = dz + (size_t)l * maxw;
    for (int n = 0; n < Nl; n++) {
      double z = 0.0;
      for (int k = 0; k < Kl; k++) z += x[k] * W[(size_t)k * Nl + n];
      if (b) z += b[n];
      if (l < L - 1) {
        double yy = om_act(m->actfn, z, &d[n]);
        if (l > 0 && m->resnet && Kl == Nl) yy += x[n];
        y[n] = yy;
      } else {
        y[n] = z;
      }
    }
  }
  for (int n = 0; n < m->sizes[L]; n++) E += act[(size_t)L * maxw + n];
  /* backward: nnp.cu:149-198 */
  double *gcur = grad; /* reuse grad as a scratch of width maxw first */
  double tmpA[1024], tmpB[1024];
  double *gy = tmpA, *gx = tmpB;
  {
    int Kl = m->sizes[L - 1], Nl = m->sizes[L];
    const double *W = m->W[e][L - 1];
    for (int k = 0; k < Kl; k++) {
      double s = 0.0;
      for (int n = 0; n < Nl; n++) s += W[(size_t)k * Nl + n];
      gy[k] = s;
    }
  }
  for (int l = L - 2; l >= 0; l--) {
    int Kl = m->sizes[l], Nl = m->sizes[l + 1];
    const double *W = m->W[e][l];
    const double *d = dz + (size_t)l * maxw;
    for (int k = 0; k < Kl; k++) {
      double s = 0.0;
      for (int n = 0; n < Nl; n++) s += gy[n] * d[n] * W[(size_t)k * Nl + n];
      if (l > 0 && m->resnet && Kl == Nl) s += gy[k];
      gx[k] = s;
    }
    double *t = gy; gy = gx; gx = t;
  }
  memcpy(gcur, gy, sizeof(double) * m->n_in);
  return E;
}

/* Forward of one TDNP net for element e: act[l] (width sizes[l], stride
 * maxw) holds the input of layer l, dz[l] the act' of hidden layer l; the
 * last layer is linear (nnp.cu:200-281).  Returns the sum of the outputs. */
static double om_net_fwd(const om_net *t, int e, int actfn_ovr, double *act, double *dz,
                         int maxw)
{
  (void)actfn_ovr;
  int L = t->nl;
  for (int l = 0; l < L; l++) {
    int Kl = t->sizes[l], Nl = t->sizes[l + 1];
    const double *W = t->W[e][l], *b = t->b[e][l];
    double *x = act + (size_t)l * maxw, *y = act + (size_t)(l + 1) * maxw;
    double *d = dz + (size_t)l * maxw;
    for (int n = 0; n < Nl; n++) {
      double z = 0.0;
      for (int k = 0; k < Kl; k++) z += x[k] * W[(size_t)k * Nl + n];
      if (b) z += b[n];
      if (l < L - 1) {
        double yy = om_act(t->actfn, z, &d[n]);
        if (l > 0 && t->resnet && Kl == Nl) yy += x[n];
        y[n] = yy;
      } else {
        y[n] = z;
      }
    }
  }
  double s = 0.0;
  for (int n = 0; n < t->sizes[L]; n++) s += act[(size_t)L * maxw + n];
  return s;
}

/* Backward of one net from the gradient gout of its outputs (NULL: 1 for
 * every output, the gradient of their sum) to gin (width sizes[0]), with the
 * activations of om_net_fwd (nnp.cu:149-198). */
static void om_net_bwd(const om_net *t, int e, const double *gout, const double *dz, int maxw,
                       double *gin)
{
  int L = t->nl;
  double ga[1024], gb[1024];
  double *gy = ga, *gx = gb;
  {
    int Kl = t->sizes[L - 1], Nl = t->sizes[L];
    const double *W = t->W[e][L - 1];
    for (int k = 0; k < Kl; k++) {
      double s = 0.0;
      for (int n = 0; n < Nl; n++) s += (gout ? gout[n] : 1.0) * W[(size_t)k * Nl + n];
      gy[k] = s;
    }
  }
  for (int l = L - 2; l >= 0; l--) {
    int Kl = t->sizes[l], Nl = t->sizes[l + 1];
    const double *W = t->W[e][l];
    const double *d = dz + (size_t)l * maxw;
    for (int k = 0; k < Kl; k++) {
      double s = 0.0;
      for (int n = 0; n < Nl; n++) s += gy[n] * d[n] * W[(size_t)k * Nl + n];
      if (l > 0 && t->resnet && Kl == Nl) s += gy[k];
      gx[k] = s;
    }
    double *tt = gy; gy = gx; gx = tt;
  }
  memcpy(gin, gy, sizeof(double) * t->sizes[0]);
}

/* TDNP atom (tdnp.cpp:167-226, nnp.cu:295-318): y = H(G), y[ydim-1] = T;
 * u = U(y), s = S(y) (times T with the Sommerfeld form); the gradient of
 * A = u - T s (T^2 s_net with Sommerfeld) back through H, the temperature
 * column held fixed.  Returns u; *s_out, *a_out. */
#define OM_TW 1024 /* widest TDNP layer */
#define OM_TWORK (6 * (OM_MAXL + 1) * OM_TW + 3 * OM_TW)

static double om_tdnp(const om_model *m, int e, const double *g, double *grad,
                      double *s_out, double *a_out, double *work)
{
  enum { W = OM_TW };
  double *actH = work, *dzH = actH + (OM_MAXL + 1) * W;
  double *actU = dzH + (OM_MAXL + 1) * W, *dzU = actU + (OM_MAXL + 1) * W;
  double *actS = dzU + (OM_MAXL + 1) * W, *dzS = actS + (OM_MAXL + 1) * W;
  double *gu = dzS + (OM_MAXL + 1) * W, *gs = gu + W, *gyv = gs + W;
  double T = m->etemp;
  memcpy(actH, g, sizeof(double) * m->n_in);
  om_net_fwd(&m->H, e, 0, actH, dzH, W);
  double *y = actH + (size_t)m->H.nl * W;
  y[m->ydim - 1] = T;
  memcpy(actU, y, sizeof(double) * m->ydim);
  memcpy(actS, y, sizeof(double) * m->ydim);
  double u = om_net_fwd(&m->U, e, 0, actU, dzU, W);
  double s = om_net_fwd(&m->S, e, 0, actS, dzS, W);
  if (m->sommerfeld) s *= T;
  om_net_bwd(&m->U, e, NULL, dzU, W, gu);
  om_net_bwd(&m->S, e, NULL, dzS, W, gs);
  double scale = m->sommerfeld ? T * T : T;
  for (int k = 0; k < m->ydim; k++) gyv[k] = gu[k] - scale * gs[k];
  gyv[m->ydim - 1] = 0.0;
  om_net_bwd(&m->H, e, gyv, dzH, W, grad);
  *s_out = s;
  *a_out = u - T * s;
  return u;
}

/* ------------------------------------------------------------------ */
/* neighbor list                                                       */
/* ------------------------------------------------------------------ */

typedef struct {
  double lo[3], xprd, yprd, zprd, xy, xz, yz;
  int pbc[3];
} om_box;

static void om_box_from(const double *bx, const int *pbc, om_box *b)
{
  b->lo[0] = bx[0]; b->lo[1] = bx[1]; b->lo[2] = bx[2];
  b->xprd = bx[3]; b->yprd = bx[4]; b->zprd = bx[5];
  b->xy = bx[6]; b->xz = bx[7]; b->yz = bx[8];
  b->pbc[0] = pbc[0]; b->pbc[1] = pbc[1]; b->pbc[2] = pbc[2];
}

/* image of atom position p shifted by (sx, sy, sz) box vectors, applied
 * one hop at a time in x, then y, then z order (AtomVec::pack_border). */
static void om_image(const om_box *b, const double *p, int sx, int sy, int sz,
                     double *o)
{
  double x = p[0], y = p[1], z = p[2];
  int st = sx > 0 ? 1 : -1;
  for (int t = 0; t < abs(sx); t++) x += st * b->xprd;
  st = sy > 0 ? 1 : -1;
  for (int t = 0; t < abs(sy); t++) { x += st * b->xy; y += st * b->yprd; }
  st = sz > 0 ? 1 : -1;
  for (int t = 0; t < abs(sz); t++) {
    x += st * b->xz; y += st * b->yz; z += st * b->zprd;
  }
  o[0] = x; o[1] = y; o[2] = z;
}

static void om_frac(const om_box *b, const double *p, double *f)
{
  double dx = p[0] - b->lo[0], dy = p[1] - b->lo[1], dz = p[2] - b->lo[2];
  double fz = dz / b->zprd;
  double fy = (dy - fz * b->yz) / b->yprd;
  double fx = (dx - fy * b->xy - fz * b->xz) / b->xprd;
  f[0] = fx; f[1] = fy; f[2] = fz;
}

/* Full neighbor list with cutoff `cut` (rsq <= cut^2, no FMA contraction:
 * this file is compiled with -ffp-contract=off).  Entries are (j, sx, sy,
 * sz) packed as 4 ints.  Pass out=NULL to count only.  Returns total count
 * or -1 if cap exceeded.  counts[i] receives per-atom counts. */
long tmdo_neighbors(int n, const double *x, const double *boxv, const int *pbc,
                    double cut, int *counts, int *out, long cap)
{
  om_box b;
  om_box_from(boxv, pbc, &b);
  double cutsq = cut * cut;
  /* perpendicular widths of the cell */
  double V = b.xprd * b.yprd * b.zprd;
  double ax[3] = {b.xprd, 0, 0}, bv[3] = {b.xy, b.yprd, 0},
         cv[3] = {b.xz, b.yz, b.zprd};
  double bxc[3] = {bv[1] * cv[2] - bv[2] * cv[1], bv[2] * cv[0] - bv[0] * cv[2],
                   bv[0] * cv[1] - bv[1] * cv[0]};
  double cxa[3] = {cv[1] * ax[2] - cv[2] * ax[1], cv[2] * ax[0] - cv[0] * ax[2],
                   cv[0] * ax[1] - cv[1] * ax[0]};
  double axb[3] = {ax[1] * bv[2] - ax[2] * bv[1], ax[2] * bv[0] - ax[0] * bv[2],
                   ax[0] * bv[1] - ax[1] * bv[0]};
  double w[3] = {V / sqrt(bxc[0] * bxc[0] + bxc[1] * bxc[1] + bxc[2] * bxc[2]),
                 V / sqrt(cxa[0] * cxa[0] + cxa[1] * cxa[1] + cxa[2] * cxa[2]),
                 V / sqrt(axb[0] * axb[0] + axb[1] * axb[1] + axb[2] * axb[2])};
  int nb[3], ns[3];
  for (int a = 0; a < 3; a++) {
    nb[a] = (int)floor(w[a] / (cut * (1.0 + 1e-6)));
    if (nb[a] < 1) nb[a] = 1;
    if (nb[a] > 256) nb[a] = 256;
    ns[a] = (int)ceil(cut * (1.0 + 1e-9) / (w[a] / nb[a]));
    if (!b.pbc[a]) { /* non-periodic: no images, cells only */
      if (ns[a] > nb[a]) ns[a] = nb[a];
    }
  }
  int ncell = nb[0] * nb[1] * nb[2];
  int *head = (int *)malloc(sizeof(int) * ncell);
  int *next = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  int *cell = (int *)malloc(sizeof(int) * 3 * (n > 0 ? n : 1));
  for (int c = 0; c < ncell; c++) head[c] = -1;
  for (int i = n - 1; i >= 0; i--) {
    double f[3];
    om_frac(&b, x + 3 * i, f);
    int ci[3];
    for (int a = 0; a < 3; a++) {
      int q = (int)floor(f[a] * nb[a]);
      if (q < 0) q = 0;
      if (q >= nb[a]) q = nb[a] - 1;
      ci[a] = q;
    }
    cell[3 * i] = ci[0]; cell[3 * i + 1] = ci[1]; cell[3 * i + 2] = ci[2];
    int c = (ci[2] * nb[1] + ci[1]) * nb[0] + ci[0];
    next[i] = head[c];
    head[c] = i;
  }
  long total = 0;
  int overflow = 0;
  for (int i = 0; i < n; i++) {
    const double *xi = x + 3 * i;
    int cnt = 0;
    for (int oz = -ns[2]; oz <= ns[2]; oz++)
      for (int oy = -ns[1]; oy <= ns[1]; oy++)
        for (int ox = -ns[0]; ox <= ns[0]; ox++) {
          int cc[3] = {cell[3 * i] + ox, cell[3 * i + 1] + oy,
                       cell[3 * i + 2] + oz};
          int sh[3], wc[3], skip = 0;
          for (int a = 0; a < 3; a++) {
            int q = cc[a];
            int s = (int)floor((double)q / nb[a]);
            int wq = q - s * nb[a];
            if (!b.pbc[a] && s != 0) skip = 1;
            sh[a] = s;
            wc[a] = wq;
          }
          if (skip) continue;
          int c = (wc[2] * nb[1] + wc[1]) * nb[0] + wc[0];
          for (int j = head[c]; j >= 0; j = next[j]) {
            if (j == i && sh[0] == 0 && sh[1] == 0 && sh[2] == 0) continue;
            double xj[3];
            om_image(&b, x + 3 * j, sh[0], sh[1], sh[2], xj);
            double dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
            double rsq = dx * dx + dy * dy + dz * dz;
            if (rsq <= cutsq) {
              if (out) {
                if (total < cap) {
                  int *o = out + 4 * total;
                  o[0] = j; o[1] = sh[0]; o[2] = sh[1]; o[3] = sh[2];
                } else {
                  overflow = 1;
                }
              }
              total++;
              cnt++;
            }
          }
        }
    if (counts) counts[i] = cnt;
  }
  free(head);
  free(next);
  free(cell);
  return overflow ? -1 : total;
}

/* ------------------------------------------------------------------ */
/* force evaluation                                                    */
/* ------------------------------------------------------------------ */

/* Evaluate energy, forces and virial for n atoms.
 *   x[n*3], elem[n] (0-based element of the potential), box[9] =
 *   (xlo, ylo, zlo, xprd, yprd, zprd, xy, xz, yz), pbc[3]
 *   nbr: per-atom offsets (n+1) into ent (4 ints per entry: j,sx,sy,sz)
 *   outputs (nullable): eatom[n], f[n*3], virial[6], vatom[n*6],
 *   G[n*n_in], dEdG[n*n_in]
 * Returns total energy (scaled). */
double tmdo_compute(void *h, int n, const double *x, const int *elem,
                    const double *boxv, const int *pbc, const long *off,
                    const int *ent, double scale, double *eatom, double *f,
                    double *virial, double *vatom, double *Gout,
                    double *dEdGout)
{
  om_model *m = (om_model *)h;
  om_box b;
  om_box_from(boxv, pbc, &b);
  int K = m->K, D = m->D, Mm = m->M, B = m->nelt;
  int nin = m->n_in;
  double rc2 = m->rmax * m->rmax;
  int maxw = nin;
  for (int l = 0; l <= m->nl; l++)
    if (m->sizes[l] > maxw) maxw = m->sizes[l];
  long npair = off[n];
  double *dfbuf = (double *)calloc((size_t)(npair > 0 ? npair : 1) * 3,
                                   sizeof(double));
  double *Ebuf = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
  double *Sbuf = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  double *Abuf = (double *)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  int eltij[OM_MAXE][OM_MAXE];
  for (int i = 0; i < B; i++) {
    int k = 1;
    for (int j = 0; j < B; j++) eltij[i][j] = (i == j) ? 0 : k++;
  }

#pragma omp parallel
  {
    double *P = (double *)malloc(sizeof(double) * B * K * D);
    double *S = (double *)malloc(sizeof(double) * B * K * D);
    double *G = (double *)malloc(sizeof(double) * nin);
    double *dG = (double *)malloc(sizeof(double) * (nin > 1024 ? nin : 1024));
    double *work = (double *)malloc(sizeof(double) * (size_t)(m->nl + 1) * maxw * 2);
    double *twork = m->tdnp ? (double *)malloc(sizeof(double) * OM_TWORK) : NULL;
    double H[256], dH[256], Mv[OM_MAXD], dM[3 * OM_MAXD];
#pragma omp for schedule(dynamic, 16)
    for (int i = 0; i < n; i++) {
      const double *xi = x + 3 * i;
      int ei = elem[i];
      memset(P, 0, sizeof(double) * B * K * D);
      for (long s = off[i]; s < off[i + 1]; s++) {
        const int *en = ent + 4 * s;
        int j = en[0];
        double xj[3];
        om_image(&b, x + 3 * j, en[1], en[2], en[3], xj);
        double dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
        double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < rc2 && r2 > 1e-10)) continue;
        double r = sqrt(r2), rinv = 1.0 / r;
        om_radial(m, r, H, dH);
        om_moments(D, dx * rinv, dy * rinv, dz * rinv, rinv, Mv, NULL);
        double *Pb = P + (size_t)eltij[ei][elem[j]] * K * D;
        for (int k = 0; k < K; k++)
          for (int d = 0; d < D; d++) Pb[k * D + d] += H[k] * Mv[d];
      }
      /* G = T (P^2), G0 = sign(P0) sqrt(.) */
      for (int bb = 0; bb < B; bb++)
        for (int k = 0; k < K; k++) {
          const double *Pk = P + ((size_t)bb * K + k) * D;
          for (int mm = 0; mm < Mm; mm++) {
            double t = 0.0;
            for (int d = 0; d < D; d++) t += Pk[d] * Pk[d] * m->T[mm * D + d];
            G[((size_t)bb * K + k) * Mm + mm] = t;
          }
          double *g0 = &G[((size_t)bb * K + k) * Mm];
          g0[0] = sqrt(g0[0]) * (Pk[0] < 0 ? -1.0 : 1.0);
        }
      if (Gout) memcpy(Gout + (size_t)i * nin, G, sizeof(double) * nin);
      double E;
      if (m->tdnp) {
        E = om_tdnp(m, ei, G, dG, &Sbuf[i], &Abuf[i], twork);
      } else {
        E = om_mlp(m, ei, G, dG, work, maxw);
      }
      Ebuf[i] = E;
      if (dEdGout) memcpy(dEdGout + (size_t)i * nin, dG, sizeof(double) * nin);
      /* dE/dG0 -> 0.5 dEdG0 / G0, then dE/dP */
      for (int bb = 0; bb < B; bb++)
        for (int k = 0; k < K; k++) {
          double *dg = &dG[((size_t)bb * K + k) * Mm];
          double g0 = G[((size_t)bb * K + k) * Mm];
          if (fabs(g0) < 1e-8) dg[0] = 0.0;
          else dg[0] = dg[0] / g0 * 0.5;
          const double *Pk = P + ((size_t)bb * K + k) * D;
          double *Sk = S + ((size_t)bb * K + k) * D;
          for (int d = 0; d < D; d++) {
            double t = 0.0;
            for (int mm = 0; mm < Mm; mm++) t += dg[mm] * m->T[mm * D + d];
            Sk[d] = 2.0 * t * Pk[d];
          }
        }
      /* per-pair dE_i/dx_j */
      for (long s = off[i]; s < off[i + 1]; s++) {
        const int *en = ent + 4 * s;
        int j = en[0];
        double xj[3];
        om_image(&b, x + 3 * j, en[1], en[2], en[3], xj);
        double dx = xj[0] - xi[0], dy = xj[1] - xi[1], dz = xj[2] - xi[2];
        double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < rc2 && r2 > 1e-10)) continue;
        double r = sqrt(r2), rinv = 1.0 / r;
        double u[3] = {dx * rinv, dy * rinv, dz * rinv};
        om_radial(m, r, H, dH);
        om_moments(D, u[0], u[1], u[2], rinv, Mv, dM);
        const double *Sb = S + (size_t)eltij[ei][elem[j]] * K * D;
        double f1 = 0.0, f2[3] = {0, 0, 0};
        for (int k = 0; k < K; k++) {
          double U = 0.0;
          for (int d = 0; d < D; d++) U += Sb[k * D + d] * Mv[d];
          f1 += U * dH[k];
        }
        for (int d = 0; d < D; d++) {
          double V = 0.0;
          for (int k = 0; k < K; k++) V += Sb[k * D + d] * H[k];
          f2[0] += V * dM[0 * D + d];
          f2[1] += V * dM[1 * D + d];
          f2[2] += V * dM[2 * D + d];
        }
        for (int a = 0; a < 3; a++)
          dfbuf[3 * s + a] = (f1 * u[a] + f2[a]) * scale;
      }
    }
    free(P); free(S); free(G); free(dG); free(work); free(twork);
  }

  /* deterministic serial accumulation */
  double etot = 0.0;
  if (f) memset(f, 0, sizeof(double) * 3 * n);
  if (vatom) memset(vatom, 0, sizeof(double) * 6 * n);
  double vir[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < n; i++) {
    etot += Ebuf[i] * scale;
    if (eatom) eatom[i] = Ebuf[i] * scale;
    const double *xi = x + 3 * i;
    for (long s = off[i]; s < off[i + 1]; s++) {
      const int *en = ent + 4 * s;
      int j = en[0];
      const double *df = dfbuf + 3 * s;
      if (df[0] == 0.0 && df[1] == 0.0 && df[2] == 0.0) continue;
      if (f) {
        for (int a = 0; a < 3; a++) {
          f[3 * i + a] += df[a];
          f[3 * j + a] -= df[a];
        }
      }
      double xj[3];
      om_image(&b, x + 3 * j, en[1], en[2], en[3], xj);
      double d[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
      double v6[6] = {-d[0] * df[0], -d[1] * df[1], -d[2] * df[2],
                      -d[0] * df[1], -d[0] * df[2], -d[1] * df[2]};
      for (int c = 0; c < 6; c++) {
        vir[c] += v6[c];
        if (vatom) {
          vatom[6 * i + c] += 0.5 * v6[c];
          vatom[6 * j + c] += 0.5 * v6[c];
        }
      }
    }
  }
  if (virial)
    for (int c = 0; c < 6; c++) virial[c] = vir[c];
  double st = 0.0, at = 0.0;
  for (int i = 0; i < n; i++) {
    st += Sbuf[i] * scale;
    at += Abuf[i] * scale;
  }
  m->tdnp_S = st;
  m->tdnp_A = at;
  free(dfbuf);
  free(Ebuf);
  free(Sbuf);
  free(Abuf);
  return etot;
}

/* ------------------------------------------------------------------ */
/* fix nve (metal units) with neighbor rebuild every step              */
/* ------------------------------------------------------------------ */

#define OM_FTM2V (1.0 / 1.0364269e-4)
#define OM_MVV2E 1.0364269e-4

static void om_remap(const om_box *b, int n, double *x)
{
  /* Domain::pbc() for orthogonal boxes: x += prd if below lo, x -= prd
   * (clamped to lo) if at or above hi; triclinic boxes remap through the
   * fractional coordinates. */
  int tri = (b->xy != 0.0 || b->xz != 0.0 || b->yz != 0.0);
  for (int i = 0; i < n; i++) {
    double *p = x + 3 * i;
    if (!tri) {
      double prd[3] = {b->xprd, b->yprd, b->zprd};
      for (int a = 0; a < 3; a++) {
        if (!b->pbc[a]) continue;
        double hi = b->lo[a] + prd[a];
        if (p[a] < b->lo[a]) p[a] += prd[a];
        if (p[a] >= hi) {
          p[a] -= prd[a];
          if (p[a] < b->lo[a]) p[a] = b->lo[a];
        }
      }
    } else {
      double fr[3];
      om_frac(b, p, fr);
      int s[3] = {0, 0, 0};
      for (int a = 0; a < 3; a++)
        if (b->pbc[a]) s[a] = (int)floor(fr[a]);
      if (s[0] || s[1] || s[2]) {
        double q[3];
        om_image(b, p, -s[0], -s[1], -s[2], q);
        p[0] = q[0]; p[1] = q[1]; p[2] = q[2];
      }
    }
  }
}

/* Run nsteps of velocity Verlet.  mass_e[nelt] per element.  Neighbor
 * lists are rebuilt every step with cutoff rmax + skin.  thermo (nullable)
 * receives per step (nsteps+1 rows): pe, ke. Returns 0 on success. */
int tmdo_nve(void *h, int n, double *x, double *v, const int *elem,
             const double *mass_e, const double *boxv, const int *pbc,
             double dt, int nsteps, double skin, double *f, double *thermo)
{
  om_model *m = (om_model *)h;
  om_box b;
  om_box_from(boxv, pbc, &b);
  double cut = m->rmax + skin;
  double dtf = 0.5 * dt * OM_FTM2V;
  long *off = (long *)malloc(sizeof(long) * (n + 1));
  int *cnt = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  int *ent = NULL;
  long cap = 0;
  int rc = 0;
  for (int step = 0; step <= nsteps; step++) {
    if (step > 0) {
      for (int i = 0; i < n; i++) {
        double dtfm = dtf / mass_e[elem[i]];
        for (int a = 0; a < 3; a++) {
          v[3 * i + a] += dtfm * f[3 * i + a];
          x[3 * i + a] += dt * v[3 * i + a];
        }
      }
      om_remap(&b, n, x);
    }
    long tot = tmdo_neighbors(n, x, boxv, pbc, cut, cnt, NULL, 0);
    if (tot > cap) {
      free(ent);
      cap = tot + tot / 4 + 16;
      ent = (int *)malloc(sizeof(int) * 4 * cap);
    }
    tmdo_neighbors(n, x, boxv, pbc, cut, cnt, ent, cap);
    off[0] = 0;
    for (int i = 0; i < n; i++) off[i + 1] = off[i] + cnt[i];
    double pe = tmdo_compute(h, n, x, elem, boxv, pbc, off, ent, 1.0, NULL, f,
                             NULL, NULL, NULL, NULL);
    if (step > 0) {
      for (int i = 0; i < n; i++) {
        double dtfm = dtf / mass_e[elem[i]];
        for (int a = 0; a < 3; a++) v[3 * i + a] += dtfm * f[3 * i + a];
      }
    }
    if (thermo) {
      double ke = 0.0;
      for (int i = 0; i < n; i++)
        ke += mass_e[elem[i]] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] +
                                 v[3 * i + 2] * v[3 * i + 2]);
      thermo[2 * step] = pe;
      thermo[2 * step + 1] = 0.5 * OM_MVV2E * ke;
    }
  }
  free(off);
  free(cnt);
  free(ent);
  return rc;
}

/* ------------------------------------------------------------------ */
/* fix nvt: Nose-Hoover chain thermostat (FixNH, fix_nh.cpp)            */
/* ------------------------------------------------------------------ */

#define OM_BOLTZ 8.617343e-5
#define OM_NHC 3 /* mtchain default (fix_nh.cpp:81) */

typedef struct {
  double eta[OM_NHC], eta_dot[OM_NHC + 1], eta_dotdot[OM_NHC], eta_mass[OM_NHC];
  double t_current, t_target, ke_target, tdof, t_freq;
} om_nhc;

/* temperature of compute temp: mvv2e sum m v^2 / (dof boltz), dof = 3N - 3 */
static double om_temp(int n, const double *v, const int *elem, const double *mass_e,
                      double tdof)
{
  double s = 0.0;
  for (int i = 0; i < n; i++)
    s += mass_e[elem[i]] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] +
                            v[3 * i + 2] * v[3 * i + 2]);
  return s * OM_MVV2E / (tdof * OM_BOLTZ);
}

/* FixNH::nhc_temp_integrate (fix_nh.cpp:1758-1822) with nc_tchain = 1 and
 * drag = 0 (the defaults, fix_nh.cpp:78-86); returns factor_eta. */
static double om_nhc_integrate(om_nhc *c, double dt)
{
  const double dthalf = 0.5 * dt, dt4 = 0.25 * dt, dt8 = 0.125 * dt;
  double kecurrent = c->tdof * OM_BOLTZ * c->t_current;
  c->eta_mass[0] = c->tdof * OM_BOLTZ * c->t_target / (c->t_freq * c->t_freq);
  for (int k = 1; k < OM_NHC; k++)
    c->eta_mass[k] = OM_BOLTZ * c->t_target / (c->t_freq * c->t_freq);
  c->eta_dotdot[0] = c->eta_mass[0] > 0.0 ? (kecurrent - c->ke_target) / c->eta_mass[0] : 0.0;
  double expfac;
  for (int k = OM_NHC - 1; k > 0; k--) {
    expfac = exp(-dt8 * c->eta_dot[k + 1]);
    c->eta_dot[k] *= expfac;
    c->eta_dot[k] += c->eta_dotdot[k] * dt4;
    c->eta_dot[k] *= expfac;
  }
  expfac = exp(-dt8 * c->eta_dot[1]);
  c->eta_dot[0] *= expfac;
  c->eta_dot[0] += c->eta_dotdot[0] * dt4;
  c->eta_dot[0] *= expfac;
  const double factor = exp(-dthalf * c->eta_dot[0]);
  c->t_current *= factor * factor;
  kecurrent = c->tdof * OM_BOLTZ * c->t_current;
  c->eta_dotdot[0] = c->eta_mass[0] > 0.0 ? (kecurrent - c->ke_target) / c->eta_mass[0] : 0.0;
  for (int k = 0; k < OM_NHC; k++) c->eta[k] += dthalf * c->eta_dot[k];
  c->eta_dot[0] *= expfac;
  c->eta_dot[0] += c->eta_dotdot[0] * dt4;
  c->eta_dot[0] *= expfac;
  for (int k = 1; k < OM_NHC; k++) {
    expfac = exp(-dt8 * c->eta_dot[k + 1]);
    c->eta_dot[k] *= expfac;
    c->eta_dotdot[k] = (c->eta_mass[k - 1] * c->eta_dot[k - 1] * c->eta_dot[k - 1] -
                        OM_BOLTZ * c->t_target) / c->eta_mass[k];
    c->eta_dot[k] += c->eta_dotdot[k] * dt4;
    c->eta_dot[k] *= expfac;
  }
  return factor;
}

/* Energy of the chain, FixNH::compute_scalar (fix_nh.cpp:1447-1473). */
static double om_nhc_energy(const om_nhc *c)
{
  double kt = OM_BOLTZ * c->t_target;
  double e = c->ke_target * c->eta[0] + 0.5 * c->eta_mass[0] * c->eta_dot[0] * c->eta_dot[0];
  for (int k = 1; k < OM_NHC; k++)
    e += kt * c->eta[k] + 0.5 * c->eta_mass[k] * c->eta_dot[k] * c->eta_dot[k];
  return e;
}

/* nsteps of fix nvt temp t_start t_stop t_damp (Verlet + FixNH::setup /
 * initial_integrate / final_integrate, fix_nh.cpp:741-930) from a fresh
 * thermostat; thermo[(nsteps+1)*3] = (pe, ke, chain energy) after every
 * step. */
int tmdo_nvt(void *h, int n, double *x, double *v, const int *elem,
             const double *mass_e, const double *boxv, const int *pbc, double dt,
             int nsteps, double skin, double t_start, double t_stop, double t_damp,
             double *f, double *thermo)
{
  om_model *m = (om_model *)h;
  om_box b;
  om_box_from(boxv, pbc, &b);
  double cut = m->rmax + skin;
  double dtf = 0.5 * dt * OM_FTM2V;
  long *off = (long *)malloc(sizeof(long) * (n + 1));
  int *cnt = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  int *ent = NULL;
  long cap = 0;
  om_nhc c;
  memset(&c, 0, sizeof c);
  c.tdof = 3.0 * n - 3.0;
  c.t_freq = 1.0 / t_damp;
  for (int step = 0; step <= nsteps; step++) {
    if (step == 0) {
      /* FixNH::setup */
      c.t_current = om_temp(n, v, elem, mass_e, c.tdof);
      c.t_target = t_start;
      c.ke_target = c.tdof * OM_BOLTZ * c.t_target;
      c.eta_mass[0] = c.tdof * OM_BOLTZ * c.t_target / (c.t_freq * c.t_freq);
      for (int k = 1; k < OM_NHC; k++)
        c.eta_mass[k] = OM_BOLTZ * c.t_target / (c.t_freq * c.t_freq);
      for (int k = 1; k < OM_NHC; k++)
        c.eta_dotdot[k] = (c.eta_mass[k - 1] * c.eta_dot[k - 1] * c.eta_dot[k - 1] -
                           OM_BOLTZ * c.t_target) / c.eta_mass[k];
    } else {
      /* initial_integrate: compute_temp_target, nhc, nve_v, nve_x */
      double delta = (double)step / (double)nsteps;
      c.t_target = t_start + delta * (t_stop - t_start);
      c.ke_target = c.tdof * OM_BOLTZ * c.t_target;
      double fe = om_nhc_integrate(&c, dt);
      for (int i = 0; i < 3 * n; i++) v[i] *= fe;
      for (int i = 0; i < n; i++) {
        double dtfm = dtf / mass_e[elem[i]];
        for (int a = 0; a < 3; a++) {
          v[3 * i + a] += dtfm * f[3 * i + a];
          x[3 * i + a] += dt * v[3 * i + a];
        }
      }
      om_remap(&b, n, x);
    }
    long tot = tmdo_neighbors(n, x, boxv, pbc, cut, cnt, NULL, 0);
    if (tot > cap) {
      free(ent);
      cap = tot + tot / 4 + 16;
      ent = (int *)malloc(sizeof(int) * 4 * cap);
    }
    tmdo_neighbors(n, x, boxv, pbc, cut, cnt, ent, cap);
    off[0] = 0;
    for (int i = 0; i < n; i++) off[i + 1] = off[i] + cnt[i];
    double pe = tmdo_compute(h, n, x, elem, boxv, pbc, off, ent, 1.0, NULL, f,
                             NULL, NULL, NULL, NULL);
    if (step > 0) {
      /* final_integrate: nve_v, t_current, nhc */
      for (int i = 0; i < n; i++) {
        double dtfm = dtf / mass_e[elem[i]];
        for (int a = 0; a < 3; a++) v[3 * i + a] += dtfm * f[3 * i + a];
      }
      c.t_current = om_temp(n, v, elem, mass_e, c.tdof);
      double fe = om_nhc_integrate(&c, dt);
      for (int i = 0; i < 3 * n; i++) v[i] *= fe;
    }
    if (thermo) {
      double ke = 0.0;
      for (int i = 0; i < n; i++)
        ke += mass_e[elem[i]] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] +
                                 v[3 * i + 2] * v[3 * i + 2]);
      thermo[3 * step] = pe;
      thermo[3 * step + 1] = 0.5 * OM_MVV2E * ke;
      thermo[3 * step + 2] = om_nhc_energy(&c);
    }
  }
  free(off);
  free(cnt);
  free(ent);
  return 0;
}

/* ------------------------------------------------------------------ */
/* min_style fire (FIRE 2.0 as LAMMPS runs it by default)              */
/* ------------------------------------------------------------------ */

/* Forces and energy at x: neighbor list at rmax + skin, then the force
 * evaluation (a fresh list every call, as LAMMPS reneighbours). */
static double om_eval(void *h, int n, const double *x, const int *elem, const double *boxv,
                      const int *pbc, double skin, double *f)
{
  om_model *m = (om_model *)h;
  double cut = m->rmax + skin;
  int *cnt = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  long *off = (long *)malloc(sizeof(long) * (n + 1));
  long tot = tmdo_neighbors(n, x, boxv, pbc, cut, cnt, NULL, 0);
  int *ent = (int *)malloc(sizeof(int) * 4 * (tot > 0 ? tot : 1));
  tmdo_neighbors(n, x, boxv, pbc, cut, cnt, ent, tot);
  off[0] = 0;
  for (int i = 0; i < n; i++) off[i + 1] = off[i] + cnt[i];
  double pe = tmdo_compute(h, n, x, elem, boxv, pbc, off, ent, 1.0, NULL, f, NULL, NULL,
                           NULL, NULL);
  free(cnt);
  free(off);
  free(ent);
  return pe;
}

/* Energy minimisation with min_style fire at LAMMPS's defaults (min.cpp:63-72:
 * dmax 0.1 A, delaystep 20, dtgrow 1.1, dtshrink 0.5, alpha0 0.25,
 * alphashrink 0.99, tmax 10, tmin 0.02, integrator eulerimplicit,
 * halfstepback yes, abcfire no), one iteration as MinFire::run_iterate
 * (min_fire.cpp:149-619): P = v.f over the atoms; P > 0 mixes
 * v <- (1 - a) v + a sqrt(v.v / f.f) f after the Euler kick and, more than
 * delaystep iterations after the last P <= 0, grows dt (capped at tmax dt0)
 * and shrinks a; P <= 0 (past the first delaystep iterations) resets a and
 * halves dt (not below tmin dt0), steps x back by dt v / 2, zeroes v and
 * re-evaluates the forces; then dt is limited so that no atom moves more than
 * dmax along an axis, v += dt f / m (metal units), x += dt v, and the forces
 * are evaluated.  Velocities start at zero (MinFire::setup_style).  The run
 * stops after an iteration whose largest per-atom |F|^2 is below ftol^2
 * (min_modify norm max) or after maxiter iterations.  x is
 * remapped into the periodic box after each move.  Returns the iterations
 * run; f receives the forces at the final x and *pe the energy. */
int tmdo_fire(void *h, int n, double *x, const int *elem, const double *mass_e,
              const double *boxv, const int *pbc, double dt0, double ftol, int maxiter,
              double skin, double *f, double *pe)
{
  const double dmax = 0.1, dtgrow = 1.1, dtshrink = 0.5, alpha0 = 0.25, alphashrink = 0.99;
  const int delaystep = 20;
  const double dtmax = 10.0 * dt0, dtmin = 0.02 * dt0;
  om_box b;
  om_box_from(boxv, pbc, &b);
  double *v = (double *)calloc(3 * (size_t)(n > 0 ? n : 1), sizeof(double));
  double dt = dt0, alpha = alpha0;
  int last_negative = 0, flagv0 = 1, iter = 0;
  double e = om_eval(h, n, x, elem, boxv, pbc, skin, f);
  for (iter = 1; iter <= maxiter; iter++) {
    double vdotf = 0.0, scale1 = 0.0, scale2 = 0.0;
    for (int i = 0; i < 3 * n; i++) vdotf += v[i] * f[i];
    if (vdotf > 0.0) {
      double vdotv = 0.0, fdotf = 0.0;
      for (int i = 0; i < 3 * n; i++) {
        vdotv += v[i] * v[i];
        fdotf += f[i] * f[i];
      }
      scale1 = 1.0 - alpha;
      scale2 = fdotf <= 1e-20 ? 0.0 : alpha * sqrt(vdotv / fdotf);
      if (iter - last_negative > delaystep) {
        dt = fmin(dt * dtgrow, dtmax);
        alpha *= alphashrink;
      }
    } else {
      last_negative = iter;
      if (!(iter < delaystep)) {
        alpha = alpha0;
        if (dt * dtshrink >= dtmin) dt *= dtshrink;
      }
      for (int i = 0; i < 3 * n; i++) x[i] -= 0.5 * dt * v[i];
      om_remap(&b, n, x);
      for (int i = 0; i < 3 * n; i++) v[i] = 0.0;
      flagv0 = 1;
    }
    if (flagv0) {
      e = om_eval(h, n, x, elem, boxv, pbc, skin, f);
      double dtf = dt * OM_FTM2V;
      for (int i = 0; i < n; i++) {
        double dtfm = dtf / mass_e[elem[i]];
        for (int a = 0; a < 3; a++) v[3 * i + a] = dtfm * f[3 * i + a];
      }
    }
    double dtv = dt;
    for (int i = 0; i < n; i++) {
      double vmax = fmax(fabs(v[3 * i]), fabs(v[3 * i + 1]));
      vmax = fmax(vmax, fabs(v[3 * i + 2]));
      if (dtv * vmax > dmax) dtv = dmax / vmax;
    }
    if (flagv0)
      for (int i = 0; i < 3 * n; i++) v[i] = 0.0;
    double dtf = dtv * OM_FTM2V;
    for (int i = 0; i < n; i++) {
      double dtfm = dtf / mass_e[elem[i]];
      for (int a = 0; a < 3; a++) {
        v[3 * i + a] += dtfm * f[3 * i + a];
        if (vdotf > 0.0) v[3 * i + a] = scale1 * v[3 * i + a] + scale2 * f[3 * i + a];
        x[3 * i + a] += dtv * v[3 * i + a];
      }
    }
    om_remap(&b, n, x);
    e = om_eval(h, n, x, elem, boxv, pbc, skin, f);
    flagv0 = 0;
    double fmax2 = 0.0;
    for (int i = 0; i < n; i++) {
      double s = f[3 * i] * f[3 * i] + f[3 * i + 1] * f[3 * i + 1] + f[3 * i + 2] * f[3 * i + 2];
      if (s > fmax2) fmax2 = s;
    }
    if (fmax2 < ftol * ftol) break;
  }
  if (pe) *pe = e;
  free(v);
  return iter > maxiter ? maxiter : iter;
}
