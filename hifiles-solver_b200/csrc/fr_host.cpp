// fr_host.cpp -- host set-up of the FR path (bases, operators, mesh wiring,
// metrics).  FP64, run once per solver.
#include "fr_host.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <unordered_map>

namespace frb {

// The reference reads its 1-D solution points from tables printed to 15
// decimals (data/loc_1d_gauss_pts.dat and data/loc_1d_gauss_lobatto_pts.dat,
// included at src/eles_hexas.cpp:196-218); a few entries are truncated rather
// than rounded and the tables are not exactly symmetric.  Operators that agree
// with the reference to round-off need exactly these constants.
static const double kGauss[11][11] = {
    {0.0},
    {-0.577350269189626, 0.577350269189626},
    {-0.774596669241483, -0.0, 0.774596669241483},
    {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053},
    {-0.906179845938664, -0.538469310105683, -0.0, 0.538469310105683, 0.906179845938664},
    {-0.932469514203152, -0.661209386466264, -0.238619186083197, 0.238619186083197, 0.661209386466265,
     0.932469514203152},
    {-0.949107912342758, -0.741531185599395, -0.405845151377397, 0.0, 0.405845151377397, 0.741531185599394,
     0.949107912342758},
    {-0.960289856497536, -0.796666477413627, -0.525532409916329, -0.18343464249565, 0.18343464249565,
     0.525532409916329, 0.796666477413627, 0.960289856497536},
    {-0.968160239507626, -0.836031107326636, -0.613371432700591, -0.324253423403809, 0.0, 0.324253423403809,
     0.613371432700591, 0.836031107326636, 0.968160239507626},
    {-0.973906528517172, -0.865063366688985, -0.679409568299024, -0.433395394129247, -0.148874338981631,
     0.148874338981632, 0.433395394129247, 0.679409568299024, 0.865063366688984, 0.973906528517171},
    {-0.978228658146057, -0.887062599768095, -0.730152005574049, -0.519096129206812, -0.269543155952345, -0.0,
     0.269543155952345, 0.519096129206812, 0.730152005574049, 0.887062599768095, 0.978228658146057},
};
static const double kLobatto[11][11] = {
    {0.0},
    {-1.0, 1.0},
    {-1.0, -0.0, 1.0},
    {-1.0, -0.447213595499958, 0.447213595499958, 1.0},
    {-1.0, -0.654653670707977, -0.0, 0.654653670707977, 1.0},
    {-1.0, -0.765055323929465, -0.285231516480645, 0.285231516480645, 0.765055323929465, 1.0},
    {-1.0, -0.830223896278567, -0.468848793470714, 0.0, 0.468848793470714, 0.830223896278567, 1.0},
    {-1.0, -0.871740148509607, -0.591700181433142, -0.209299217902479, 0.209299217902479, 0.591700181433142,
     0.871740148509607, 1.0},
    {-1.0, -0.89975799541146, -0.677186279510738, -0.363117463826178, -0.0, 0.363117463826178, 0.677186279510738,
     0.89975799541146, 1.0},
    {-1.0, -0.919533908166459, -0.738773865105505, -0.477924949810445, -0.165278957666387, 0.165278957666387,
     0.477924949810444, 0.738773865105505, 0.919533908166459, 1.0},
    {-1.0, -0.934001430408059, -0.784483473663144, -0.565235326996205, -0.295758135586939, 0.0,
     0.295758135586939, 0.565235326996205, 0.784483473663144, 0.934001430408059, 1.0},
};

bool points_1d(int P, int type, double* out)
{
  if (P < 0 || P > kMaxP) return false;
  if (type == 0) { for (int i = 0; i <= P; i++) out[i] = kGauss[P][i]; return true; }
  if (type == 1 && P >= 1) { for (int i = 0; i <= P; i++) out[i] = kLobatto[P][i]; return true; }
  return false;
}

// Lagrange basis through pts, product form (src/funcs.cpp:57-74).
double lagrange(double r, int mode, const double* pts, int n)
{
  double v = 1.0;
  for (int i = 0; i < n; i++)
    if (i != mode) v = v * ((r - pts[i]) / (pts[mode] - pts[i]));
  return v;
}

// Derivative of the Lagrange basis as a sum of partial products (src/funcs.cpp:78-108).
double dlagrange(double r, int mode, const double* pts, int n)
{
  double acc = 0.0;
  for (int i = 0; i < n; i++) {
    if (i == mode) continue;
    double num = 1.0, den = 1.0;
    for (int j = 0; j < n; j++) {
      if (j != mode && j != i) num = num * (r - pts[j]);
      if (j != mode) den = den * (pts[mode] - pts[j]);
    }
    acc = acc + (num / den);
  }
  return acc;
}

// Legendre polynomial by the three-term recursion (src/funcs.cpp:161-181).
double legendre(double r, int n)
{
  if (n == 0) return 1.0;
  if (n == 1) return r;
  return ((2 * n - 1) * r * legendre(r, n - 1) - (n - 1) * legendre(r, n - 2)) / n;
}

// Derivative of the Legendre polynomial (src/funcs.cpp:185-212).
double dlegendre(double r, int n)
{
  if (n == 0) return 0.0;
  if (r > -1.0 && r < 1.0) return (n * ((r * legendre(r, n)) - legendre(r, n - 1))) / ((r * r) - 1.0);
  if (r == -1.0) return std::pow(-1.0, n - 1.0) * 0.5 * n * (n + 1.0);
  return 0.5 * n * (n + 1.0);
}

// Derivative of the 1-D VCJH correction functions (src/funcs.cpp:216-250).
double dvcjh(double r, int side, int P, double eta)
{
  if (side == 0) {
    if (P == 0) return 0.5 * std::pow(-1.0, P) * (dlegendre(r, P) - (dlegendre(r, P + 1) / (1.0 + eta)));
    return 0.5 * std::pow(-1.0, P) *
           (dlegendre(r, P) - (((eta * dlegendre(r, P - 1)) + dlegendre(r, P + 1)) / (1.0 + eta)));
  }
  if (P == 0) return 0.5 * (dlegendre(r, P) + (dlegendre(r, P + 1) / (1.0 + eta)));
  return 0.5 * (dlegendre(r, P) + (((eta * dlegendre(r, P - 1)) + dlegendre(r, P + 1)) / (1.0 + eta)));
}

static double factorial(int n) { double f = 1; for (int i = 2; i <= n; i++) f *= i; return f; }

// eta of the named VCJH members (src/funcs.cpp:1503-1546).
double vcjh_eta(int scheme, int P, double user_eta)
{
  switch (scheme) {
    case 0: return user_eta;
    case 1: return 0.0;
    case 2: return (1.0 * P) / (1.0 * (P + 1));
    case 3: return P == 0 ? NAN : (1.0 * (P + 1)) / (1.0 * P);
    case 4: {
      double c;
      if (P == 2) c = 0.206; else if (P == 3) c = 3.80e-3; else if (P == 4) c = 4.67e-5;
      else if (P == 5) c = 4.28e-7; else return NAN;
      double ap = 1. / std::pow(2.0, P) * factorial(2 * P) / (factorial(P) * factorial(P));
      return c * (2 * P + 1) / 2 * (factorial(P) * ap) * (factorial(P) * ap);
    }
    default: return NAN;
  }
}

bool make_line(int P, int upts_type, int vcjh_scheme, double eta, Line1D& L, std::string& err)
{
  if (!points_1d(P, upts_type, L.loc)) { err = "unsupported order / point type"; return false; }
  L.P = P; L.n1 = P + 1;
  L.eta = vcjh_eta(vcjh_scheme, P, eta);
  if (std::isnan(L.eta)) { err = "VCJH scheme not defined for this order"; return false; }
  int n = L.n1;
  for (int m = 0; m < n; m++) {
    L.Lm[m] = lagrange(-1.0, m, L.loc, n);
    L.Lp[m] = lagrange(1.0, m, L.loc, n);
  }
  for (int k = 0; k < n; k++) {
    for (int m = 0; m < n; m++) L.D[k][m] = dlagrange(L.loc[k], m, L.loc, n);
    L.gL[k] = dvcjh(L.loc[k], 0, P, L.eta);
    L.gR[k] = dvcjh(L.loc[k], 1, P, L.eta);
  }
  // quadrature weights of the point set: integrals of the Lagrange basis,
  // exact by Gauss-Legendre quadrature on n1+1 points computed here.
  {
    int q = n + 1;
    double x[kMaxP + 3], w[kMaxP + 3];
    for (int i = 0; i < q; i++) {
      double t = -std::cos(M_PI * (i + 0.75) / (q + 0.5));
      for (int it = 0; it < 100; it++) {
        double p0 = 1.0, p1 = t;
        for (int k = 2; k <= q; k++) { double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
        double dp = q * (t * p1 - p0) / (t * t - 1.0);
        double dt = p1 / dp; t -= dt;
        if (std::fabs(dt) < 1e-16) break;
      }
      double p0 = 1.0, p1 = t;
      for (int k = 2; k <= q; k++) { double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
      double dp = q * (t * p1 - p0) / (t * t - 1.0);
      x[i] = t; w[i] = 2.0 / ((1.0 - t * t) * dp * dp);
    }
    for (int m = 0; m < n; m++) {
      double s = 0;
      for (int i = 0; i < q; i++) s += w[i] * lagrange(x[i], m, L.loc, n);
      L.w[m] = s;
    }
  }
  return true;
}

// Point sets of the reference's quadrilateral / hexahedron (solution points
// x-fastest; flux points face by face with the per-face orientation of
// src/eles_quads.cpp:259-300 and src/eles_hexas.cpp:262-324).
void element_points(int dims, const Line1D& L, std::vector<double>& lu, std::vector<double>& tf, std::vector<double>& tn)
{
  int n1 = L.n1, P = L.P;
  const double* X = L.loc;
  if (dims == 2) {
    lu.assign(2 * n1 * n1, 0.0); tf.assign(2 * 4 * n1, 0.0); tn.assign(2 * 4 * n1, 0.0);
    for (int b = 0; b < n1; b++)
      for (int a = 0; a < n1; a++) { int u = a + n1 * b; lu[2 * u] = X[a]; lu[2 * u + 1] = X[b]; }
    for (int f = 0; f < 4; f++)
      for (int j = 0; j < n1; j++) {
        int q = j + n1 * f;
        double* t = &tf[2 * q]; double* nn = &tn[2 * q];
        switch (f) {
          case 0: t[0] = X[j]; t[1] = -1.0; nn[1] = -1.0; break;
          case 1: t[0] = 1.0; t[1] = X[j]; nn[0] = 1.0; break;
          case 2: t[0] = X[P - j]; t[1] = 1.0; nn[1] = 1.0; break;
          default: t[0] = -1.0; t[1] = X[P - j]; nn[0] = -1.0; break;
        }
      }
    return;
  }
  int n2 = n1 * n1;
  lu.assign(3 * n2 * n1, 0.0); tf.assign(3 * 6 * n2, 0.0); tn.assign(3 * 6 * n2, 0.0);
  for (int c = 0; c < n1; c++)
    for (int b = 0; b < n1; b++)
      for (int a = 0; a < n1; a++) {
        int u = a + n1 * b + n2 * c;
        lu[3 * u] = X[a]; lu[3 * u + 1] = X[b]; lu[3 * u + 2] = X[c];
      }
  for (int f = 0; f < 6; f++)
    for (int j = 0; j < n1; j++)
      for (int k = 0; k < n1; k++) {
        int q = k + n1 * j + n2 * f;
        double* t = &tf[3 * q]; double* nn = &tn[3 * q];
        switch (f) {
          case 0: t[0] = X[P - k]; t[1] = X[j]; t[2] = -1.0; nn[2] = -1.0; break;
          case 1: t[0] = X[k]; t[1] = -1.0; t[2] = X[j]; nn[1] = -1.0; break;
          case 2: t[0] = 1.0; t[1] = X[k]; t[2] = X[j]; nn[0] = 1.0; break;
          case 3: t[0] = X[P - k]; t[1] = 1.0; t[2] = X[j]; nn[1] = 1.0; break;
          case 4: t[0] = -1.0; t[1] = X[P - k]; t[2] = X[j]; nn[0] = -1.0; break;
          default: t[0] = X[k]; t[1] = X[j]; t[2] = 1.0; nn[2] = 1.0; break;
        }
      }
}

// Bi/tri-linear shape functions on the 2^dims corner nodes and their
// derivatives, written as products of 2-point Lagrange factors exactly as the
// reference evaluates its shape basis (src/eles_hexas.cpp:985-1060).
static void shape(int dims, const double* r, double* N, double* dN)
{
  static const double c2[2] = {-1.0, 1.0};
  int ns = 1 << dims;
  for (int s = 0; s < ns; s++) {
    int a = s & 1, b = (s >> 1) & 1, c = (s >> 2) & 1;
    double la = lagrange(r[0], a, c2, 2), lb = lagrange(r[1], b, c2, 2);
    double da = dlagrange(r[0], a, c2, 2), db = dlagrange(r[1], b, c2, 2);
    if (dims == 2) {
      N[s] = la * lb; dN[s] = da * lb; dN[s + ns] = la * db;
    } else {
      double lc = lagrange(r[2], c, c2, 2), dc = dlagrange(r[2], c, c2, 2);
      N[s] = la * lb * lc; dN[s] = da * lb * lc; dN[s + ns] = la * db * lc; dN[s + 2 * ns] = la * lb * dc;
    }
  }
}

// Position and Jacobian dx_i/dr_j of the isoparametric map (src/eles.cpp:5744-5855).
static void map_point(const Mesh& m, long long e, const double* r, double* pos, double* J)
{
  int D = m.dims, ns = 1 << D;
  double N[8], dN[24];
  shape(D, r, N, dN);
  const int* cv = &m.c2v[(size_t)ns * e];
  for (int i = 0; i < D; i++) {
    double s = 0.0;
    for (int j = 0; j < ns; j++) s += N[j] * m.xv[(size_t)D * cv[j] + i];
    pos[i] = s;
  }
  for (int j = 0; j < D; j++)
    for (int k = 0; k < D; k++) {
      double s = 0.0;
      for (int i = 0; i < ns; i++) s += dN[i + ns * k] * m.xv[(size_t)D * cv[i] + j];
      J[j + D * k] = s;
    }
}

// n-point Gauss-Legendre rule on [-1, 1]: Newton's iteration on the Legendre
// three-term recurrence from the Chebyshev-like first guesses
// cos(pi (i + 3/4) / (n + 1/2)), weights 2 / ((1 - x^2) P_n'(x)^2).
static void gauss_legendre(int n, double* x, double* w)
{
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; i++) {
    double z = std::cos(pi * (i + 0.75) / (n + 0.5)), dp = 0.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; k++) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (n == 1) { p1 = z; p0 = 1.0; }
      dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[n - 1 - i] = z;
    w[n - 1 - i] = 2.0 / ((1.0 - z * z) * dp * dp);
  }
}

int volume_cubature(int dims, int rule, std::vector<double>& loc, std::vector<double>& w)
{
  if (rule < 1 || rule > 12 || (dims != 2 && dims != 3)) return 0;
  double x[12], wx[12];
  if (rule == 1) { x[0] = 0.0; wx[0] = 2.0; }
  else gauss_legendre(rule, x, wx);
  const int n = dims == 2 ? rule * rule : rule * rule * rule;
  loc.assign((size_t)dims * n, 0.0);
  w.assign((size_t)n, 0.0);
  for (int q = 0; q < n; q++) {
    int i0, i1, i2 = 0;
    if (dims == 2) {               // quads: first coordinate fastest
      i0 = q % rule; i1 = q / rule;
      loc[2 * q] = x[i0]; loc[2 * q + 1] = x[i1];
      w[q] = wx[i0] * wx[i1];
    } else {                       // hexes: first coordinate slowest
      i0 = q / (rule * rule); i1 = (q / rule) % rule; i2 = q % rule;
      loc[3 * q] = x[i0]; loc[3 * q + 1] = x[i1]; loc[3 * q + 2] = x[i2];
      w[q] = wx[i0] * wx[i1] * wx[i2];
    }
  }
  return n;
}

void volume_cubature_setup(const Mesh& m, const Line1D& L, int nc, const double* loc, std::vector<double>& opp,
                           std::vector<double>& detj)
{
  const int D = m.dims, n1 = m.n1, nu = m.nu;
  const size_t E = m.ne;
  opp.assign((size_t)nc * nu, 0.0);
  for (int j = 0; j < nc; j++)
    for (int k = 0; k < nu; k++) {
      const int a = k % n1, b = (k / n1) % n1, c = D == 3 ? k / (n1 * n1) : 0;
      double v = lagrange(loc[D * j], a, L.loc, n1) * lagrange(loc[D * j + 1], b, L.loc, n1);
      if (D == 3) v = v * lagrange(loc[D * j + 2], c, L.loc, n1);
      opp[j + (size_t)nc * k] = v;
    }
  detj.assign((size_t)nc * E, 0.0);
  for (size_t e = 0; e < E; e++)
    for (int j = 0; j < nc; j++) {
      double p[3], J[9];
      map_point(m, (long long)e, &loc[D * j], p, J);
      double det;
      if (D == 2) {
        det = J[0] * J[3] - J[2] * J[1];
      } else {
        det = J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
              J[6] * (J[1] * J[5] - J[4] * J[2]);
      }
      detj[j + (size_t)nc * e] = det;
    }
}

static bool compute_metrics(Mesh& m, const Line1D& L, std::string& err)
{
  std::vector<double> lu, tf, tn;
  element_points(m.dims, L, lu, tf, tn);
  int D = m.dims, nu = m.nu, nf = m.nf;
  size_t E = m.ne;
  m.pos_upts.assign((size_t)nu * E * D, 0); m.pos_fpts.assign((size_t)nf * E * D, 0);
  m.detjac.assign((size_t)nu * E, 0); m.JG.assign((size_t)D * D * nu * E, 0);
  m.tdA.assign((size_t)nf * E, 0); m.nrm.assign((size_t)nf * E * D, 0);
  for (size_t e = 0; e < E; e++) {
    double p[3], J[9];
    for (int u = 0; u < nu; u++) {
      map_point(m, e, &lu[D * u], p, J);
      for (int k = 0; k < D; k++) m.pos_upts[u + nu * (e + E * k)] = p[k];
      double* G = &m.JG[(size_t)D * D * (u + nu * e)];
      double det;
      // adjugate of the Jacobian and its determinant (src/eles.cpp:4615-4680)
      if (D == 2) {
        double xr = J[0], xs = J[2], yr = J[1], ys = J[3];
        det = xr * ys - xs * yr;
        G[0] = ys; G[2] = -xs; G[1] = -yr; G[3] = xr;
      } else {
        double xr = J[0], xs = J[3], xt = J[6], yr = J[1], ys = J[4], yt = J[7], zr = J[2], zs = J[5], zt = J[8];
        det = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
        G[0] = ys * zt - yt * zs; G[3] = xt * zs - xs * zt; G[6] = xs * yt - xt * ys;
        G[1] = yt * zr - yr * zt; G[4] = xr * zt - xt * zr; G[7] = xt * yr - xr * yt;
        G[2] = yr * zs - ys * zr; G[5] = xs * zr - xr * zs; G[8] = xr * ys - xs * yr;
      }
      if (!(det > 0)) { err = "non-positive Jacobian at a solution point"; return false; }
      m.detjac[u + nu * e] = det;
    }
    // transformed normal adj(J)^T n_ref, its length tdA and the unit normal
    // (src/eles.cpp:4720-4800)
    for (int f = 0; f < nf; f++) {
      map_point(m, e, &tf[D * f], p, J);
      for (int k = 0; k < D; k++) m.pos_fpts[f + nf * (e + E * k)] = p[k];
      const double* t = &tn[D * f];
      double v[3];
#define JJ(a, b) J[(a) + D * (b)]
      if (D == 2) {
        v[0] = (t[0] * JJ(1, 1)) - (t[1] * JJ(1, 0));
        v[1] = -(t[0] * JJ(0, 1)) + (t[1] * JJ(0, 0));
        double a = std::sqrt(v[0] * v[0] + v[1] * v[1]);
        m.tdA[f + nf * e] = a;
        for (int k = 0; k < 2; k++) m.nrm[f + nf * (e + E * k)] = v[k] / a;
      } else {
        v[0] = ((t[0] * (JJ(1, 1) * JJ(2, 2) - JJ(1, 2) * JJ(2, 1))) + (t[1] * (JJ(1, 2) * JJ(2, 0) - JJ(1, 0) * JJ(2, 2))) +
                (t[2] * (JJ(1, 0) * JJ(2, 1) - JJ(1, 1) * JJ(2, 0))));
        v[1] = ((t[0] * (JJ(0, 2) * JJ(2, 1) - JJ(0, 1) * JJ(2, 2))) + (t[1] * (JJ(0, 0) * JJ(2, 2) - JJ(0, 2) * JJ(2, 0))) +
                (t[2] * (JJ(0, 1) * JJ(2, 0) - JJ(0, 0) * JJ(2, 1))));
        v[2] = ((t[0] * (JJ(0, 1) * JJ(1, 2) - JJ(0, 2) * JJ(1, 1))) + (t[1] * (JJ(0, 2) * JJ(1, 0) - JJ(0, 0) * JJ(1, 2))) +
                (t[2] * (JJ(0, 0) * JJ(1, 1) - JJ(0, 1) * JJ(1, 0))));
        double a = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        m.tdA[f + nf * e] = a;
        for (int k = 0; k < 3; k++) m.nrm[f + nf * (e + E * k)] = v[k] / a;
      }
#undef JJ
    }
  }
  return true;
}

namespace {
struct Key {
  long long c[3];
  bool operator==(const Key& o) const { return c[0] == o.c[0] && c[1] == o.c[1] && c[2] == o.c[2]; }
};
struct KeyHash {
  size_t operator()(const Key& k) const {
    return (size_t)(k.c[0] * 73856093LL) ^ (size_t)(k.c[1] * 19349663LL) ^ (size_t)(k.c[2] * 83492791LL);
  }
};
double wrap_coord(double c, double L, double lo)
{
  if (L <= 0) return c;
  double t = (c - lo) / L;
  t -= std::floor(t + 1e-9);
  if (t > 1.0 - 1e-9) t -= 1.0;
  return lo + t * L;
}
}  // namespace

constexpr int kUnwired = -2147483647 - 1;

void finish_wiring(Mesh& m)
{
  size_t E = m.ne;
  int D = m.dims, nf = m.nf;
  m.mate.assign((size_t)nf * E, kUnwired);
  m.is_left.assign((size_t)nf * E, 0);
  m.nL.assign((size_t)nf * E * D, 0.0);
  for (size_t j = 0; j < m.bf.size(); j++) {   // boundary points: own side is the left one
    long long a = m.bf[j];
    m.mate[a] = -1 - (int)j;
    m.is_left[a] = 1;
    size_t ea = a / nf, fa = a % nf;
    for (int d = 0; d < D; d++) m.nL[fa + nf * (ea + E * d)] = m.nrm[fa + nf * (ea + E * d)];
  }
  for (size_t i = 0; i < m.il.size(); i++) {
    long long a = m.il[i], b = m.ir[i];
    m.mate[a] = (int)b; m.mate[b] = (int)a;
    m.is_left[a] = 1; m.is_left[b] = 0;
    size_t ea = a / nf, fa = a % nf, eb = b / nf, fb = b % nf;
    for (int d = 0; d < D; d++) {
      double n = m.nrm[fa + nf * (ea + E * d)];
      m.nL[fa + nf * (ea + E * d)] = n;
      m.nL[fb + nf * (eb + E * d)] = n;
    }
  }
}

// Face matching for conforming meshes with periodic translations: faces are
// paired by their centroid (after wrapping periodic coordinates), flux points
// of paired faces by physical position.  The element with the lower index is
// the left side.  This takes the place of CompConnectivity, the cyclic-face
// search and the rotation look-up table of the reference
// (src/geometry.cpp:2412-2720, 3489-3666; src/inters.cpp:187-296).
static bool wire(Mesh& m, const double* shift, const int* bctype, std::string& err)
{
  int D = m.dims, nf = m.nf, nface = m.nface, nfpf = m.nfpf;
  size_t E = m.ne;
  double lo[3] = {1e300, 1e300, 1e300}, h = 1e300;
  size_t nv = m.xv.size() / D;
  for (size_t v = 0; v < nv; v++)
    for (int d = 0; d < D; d++) lo[d] = std::min(lo[d], m.xv[D * v + d]);
  int ns = 1 << D;
  for (size_t e = 0; e < E; e++) {
    double s = 0;
    for (int d = 0; d < D; d++) {
      double t = m.xv[D * m.c2v[ns * e + 1] + d] - m.xv[D * m.c2v[ns * e] + d];
      s += t * t;
    }
    h = std::min(h, std::sqrt(s));
  }
  double tol = 1e-6 * h;
  auto coord = [&](size_t fl, size_t e, int d) {
    return wrap_coord(m.pos_fpts[fl + nf * (e + E * d)], shift[d], lo[d]);
  };
  std::unordered_map<Key, long long, KeyHash> open;
  open.reserve(E * nface);
  m.il.clear(); m.ir.clear(); m.bf.clear(); m.bt.clear();
  m.il.reserve(E * nf / 2); m.ir.reserve(E * nf / 2);
  for (size_t e = 0; e < E; e++)
    for (int fc = 0; fc < nface; fc++) {
      const int bc = bctype ? bctype[e * nface + fc] : 0;
      if (bc != 0) {
        if (!((bc >= 1 && bc <= 7) || (bc >= 11 && bc <= 16))) { err = "unknown boundary type"; return false; }
        for (int q = 0; q < nfpf; q++) {
          m.bf.push_back((int)(fc * nfpf + q + nf * e));
          m.bt.push_back((unsigned char)bc);
        }
        continue;
      }
      Key k{{0, 0, 0}};
      for (int d = 0; d < D; d++) {
        double s = 0;
        for (int q = 0; q < nfpf; q++) s += m.pos_fpts[(fc * nfpf + q) + nf * (e + E * d)];
        k.c[d] = (long long)std::llround(wrap_coord(s / nfpf, shift[d], lo[d]) / tol);
      }
      auto it = open.find(k);
      if (it == open.end()) { open.emplace(k, (long long)(e * nface + fc)); continue; }
      size_t ea = it->second / nface; int fa = it->second % nface;
      open.erase(it);
      for (int q = 0; q < nfpf; q++) {
        size_t pa = fa * nfpf + q;
        int best = -1; double bd = 1e300;
        for (int r = 0; r < nfpf; r++) {
          size_t pb = fc * nfpf + r;
          double dd = 0;
          for (int d = 0; d < D; d++) {
            double t = coord(pa, ea, d) - coord(pb, e, d);
            if (shift[d] > 0) { if (t > 0.5 * shift[d]) t -= shift[d]; if (t < -0.5 * shift[d]) t += shift[d]; }
            dd += t * t;
          }
          if (dd < bd) { bd = dd; best = (int)pb; }
        }
        if (bd > tol * tol * 1e6) { err = "flux points of a face pair do not coincide"; return false; }
        m.il.push_back((int)(pa + nf * ea));
        m.ir.push_back((int)(best + nf * e));
      }
    }
  if (!open.empty()) { err = "unmatched faces without a boundary type"; return false; }
  finish_wiring(m);
  for (size_t i = 0; i < m.mate.size(); i++)
    if (m.mate[i] == kUnwired) { err = "flux points of a face pair do not map one to one"; return false; }
  return true;
}

bool build_mesh(int dims, const Line1D& L, long long nv, const double* xv, long long ne, const int* c2v,
                const double* shift, const int* bctype, Mesh& m, std::string& err)
{
  if (dims != 2 && dims != 3) { err = "dims must be 2 or 3"; return false; }
  if (ne <= 0 || nv <= 0 || !xv || !c2v) { err = "empty mesh"; return false; }
  m.dims = dims; m.P = L.P; m.n1 = L.n1;
  m.nu = dims == 2 ? L.n1 * L.n1 : L.n1 * L.n1 * L.n1;
  m.nfpf = dims == 2 ? L.n1 : L.n1 * L.n1;
  m.nface = 2 * dims; m.nf = m.nface * m.nfpf; m.nfields = dims + 2;
  m.ne = ne;
  if ((double)m.nf * (double)ne >= 2147483647.0) { err = "mesh too large for 32-bit flux-point indices"; return false; }
  int ns = 1 << dims;
  m.xv.assign(xv, xv + (size_t)nv * dims);
  m.c2v.assign(c2v, c2v + (size_t)ne * ns);
  for (size_t i = 0; i < m.c2v.size(); i++)
    if (m.c2v[i] < 0 || m.c2v[i] >= nv) { err = "vertex index out of range"; return false; }
  if (!compute_metrics(m, L, err)) return false;
  return wire(m, shift, bctype, err);
}

}  // namespace frb
