// fr_mixed.cpp -- host set-up of tetrahedra, prisms and hexahedra for the
// per-operator path: point sets, nodal bases, the dense operators opp_0 ..
// opp_6 with the VCJH correction, and for a mesh of those elements the
// metrics and the interface and boundary tables that the fr_op_* entry points
// take.  It replaces what the reference's eles_tets / eles_pris / eles_hexas
// set-up (setup_ele_type_specific, set_opp_*, set_transforms) and its
// int_inters / bdy_inters wiring compute before the time loop.  Everything is
// FP64 on the host, once per mesh.
//
// The modal bases are the orthonormal Dubiner polynomials of the reference
// triangle and tetrahedron (Hesthaven & Warburton, Nodal Discontinuous
// Galerkin Methods, 2008: Simplex2DP, Simplex3DP and their gradients), the
// nodal bases their combinations through the inverse Vandermonde matrix of
// the solution points.  The point sets are the published ones the reference
// tabulates (fr_simplex_points.inc).  Face integrals use collapsed
// Gauss-Legendre rules computed here, exact for the polynomial degrees
// involved, in place of the reference's tabulated cubature rules.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "fr_b200.h"
#include "fr_host.hpp"

namespace frb {
extern thread_local std::string g_err;
namespace mixed {

#include "fr_simplex_points.inc"

static fr_status fail(fr_status s, const std::string& m)
{
  g_err = m;
  return s;
}

// ---------------------------------------------------------------- dense algebra
using Mat = std::vector<double>;   // row-major n x m

// Inverse by Gauss-Jordan elimination with partial pivoting; false if singular.
static bool invert(int n, const Mat& a, Mat& inv)
{
  Mat w(a);
  inv.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) inv[(size_t)i * n + i] = 1.0;
  for (int c = 0; c < n; c++) {
    int p = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(w[(size_t)r * n + c]) > std::fabs(w[(size_t)p * n + c])) p = r;
    if (w[(size_t)p * n + c] == 0.0) return false;
    if (p != c)
      for (int k = 0; k < n; k++) {
        std::swap(w[(size_t)p * n + k], w[(size_t)c * n + k]);
        std::swap(inv[(size_t)p * n + k], inv[(size_t)c * n + k]);
      }
    double d = w[(size_t)c * n + c];
    for (int k = 0; k < n; k++) { w[(size_t)c * n + k] /= d; inv[(size_t)c * n + k] /= d; }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      double f = w[(size_t)r * n + c];
      if (f == 0.0) continue;
      for (int k = 0; k < n; k++) {
        w[(size_t)r * n + k] -= f * w[(size_t)c * n + k];
        inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
      }
    }
  }
  return true;
}

static Mat matmul(int n, int k, int m, const Mat& a, const Mat& b)
{
  Mat c((size_t)n * m, 0.0);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < m; j++) {
      double s = 0.0;
      for (int l = 0; l < k; l++) s += a[(size_t)i * k + l] * b[(size_t)l * m + j];
      c[(size_t)i * m + j] = s;
    }
  return c;
}

// ------------------------------------------------------------ modal bases
// Orthonormal Jacobi polynomial P_n^(a,b) on [-1, 1] by the three-term
// recurrence (Hesthaven & Warburton, JacobiP).
static double jacobi(double x, int ia, int ib, int n)
{
  double a = ia, b = ib;
  double g0 = std::pow(2.0, a + b + 1) / (a + b + 1) * std::tgamma(a + 1) * std::tgamma(b + 1) / std::tgamma(a + b + 1);
  double p0 = 1.0 / std::sqrt(g0);
  if (n == 0) return p0;
  double g1 = (a + 1) * (b + 1) / (a + b + 3) * g0;
  double p1 = ((a + b + 2) * x / 2 + (a - b) / 2) / std::sqrt(g1);
  double aold = 2 / (2 + a + b) * std::sqrt((a + 1) * (b + 1) / (a + b + 3));
  for (int i = 1; i < n; i++) {
    double h1 = 2 * i + a + b;
    double anew = 2 / (h1 + 2) * std::sqrt((i + 1) * (i + 1 + a + b) * (i + 1 + a) * (i + 1 + b) / (h1 + 1) / (h1 + 3));
    double bnew = -(a * a - b * b) / h1 / (h1 + 2);
    double p2 = (-aold * p0 + (x - bnew) * p1) / anew;
    p0 = p1; p1 = p2; aold = anew;
  }
  return p1;
}

static double djacobi(double x, int a, int b, int n)
{
  return n == 0 ? 0.0 : std::sqrt(n * (n + a + b + 1.0)) * jacobi(x, a + 1, b + 1, n - 1);
}

// Mode (i, j) of the triangle basis of order N, in order of total degree.
static void tri_modes(int N, std::vector<std::array<int, 2>>& m)
{
  m.clear();
  for (int k = 0; k <= N; k++)
    for (int j = 0; j <= k; j++) m.push_back({k - j, j});
}

static void tet_modes(int N, std::vector<std::array<int, 3>>& m)
{
  m.clear();
  for (int t = 0; t <= N; t++)
    for (int n = 0; n <= t; n++)
      for (int k = 0; k <= n; k++) { int j = n - k; m.push_back({t - j - k, j, k}); }
}

static void rs_to_ab(double r, double s, double& a, double& b)
{
  a = (s == 1.0) ? -1.0 : 2.0 * (1.0 + r) / (1.0 - s) - 1.0;
  b = s;
}

static double dub2(double r, double s, int i, int j)
{
  double a, b;
  rs_to_ab(r, s, a, b);
  return std::sqrt(2.0) * jacobi(a, 0, 0, i) * jacobi(b, 2 * i + 1, 0, j) * std::pow(1.0 - b, i);
}

static void grad_dub2(double r, double s, int i, int j, double& dr, double& ds)
{
  double a, b;
  rs_to_ab(r, s, a, b);
  double fa = jacobi(a, 0, 0, i), dfa = djacobi(a, 0, 0, i);
  double gb = jacobi(b, 2 * i + 1, 0, j), dgb = djacobi(b, 2 * i + 1, 0, j);
  double q = 0.5 * (1.0 - b);
  double x = dfa * gb, y = dfa * (gb * (0.5 * (1.0 + a)));
  if (i > 0) { x *= std::pow(q, i - 1); y *= std::pow(q, i - 1); }
  double t = dgb * std::pow(q, i);
  if (i > 0) t -= 0.5 * i * gb * std::pow(q, i - 1);
  y += fa * t;
  double sc = std::pow(2.0, i + 0.5);
  dr = x * sc; ds = y * sc;
}

static void rst_to_abc(double r, double s, double t, double& a, double& b, double& c)
{
  a = (s + t == 0.0) ? -1.0 : -2.0 * (1.0 + r) / (s + t) - 1.0;
  b = (t == 1.0) ? -1.0 : 2.0 * (1.0 + s) / (1.0 - t) - 1.0;
  c = t;
}

static double dub3(const double* x, const std::array<int, 3>& m)
{
  double a, b, c;
  rst_to_abc(x[0], x[1], x[2], a, b, c);
  int i = m[0], j = m[1], k = m[2];
  return 2.0 * std::sqrt(2.0) * jacobi(a, 0, 0, i) * jacobi(b, 2 * i + 1, 0, j) * jacobi(c, 2 * i + 2 * j + 2, 0, k) *
         std::pow(1.0 - b, i) * std::pow(1.0 - c, i + j);
}

static void grad_dub3(const double* x, const std::array<int, 3>& m, double* g)
{
  double a, b, c;
  rst_to_abc(x[0], x[1], x[2], a, b, c);
  int i = m[0], j = m[1], k = m[2];
  double fa = jacobi(a, 0, 0, i), dfa = djacobi(a, 0, 0, i);
  double gb = jacobi(b, 2 * i + 1, 0, j), dgb = djacobi(b, 2 * i + 1, 0, j);
  double hc = jacobi(c, 2 * (i + j) + 2, 0, k), dhc = djacobi(c, 2 * (i + j) + 2, 0, k);
  double qb = 0.5 * (1.0 - b), qc = 0.5 * (1.0 - c);
  double vr = dfa * (gb * hc);
  if (i > 0) vr *= std::pow(qb, i - 1);
  if (i + j > 0) vr *= std::pow(qc, i + j - 1);
  double vs = 0.5 * (1.0 + a) * vr;
  double t = dgb * std::pow(qb, i);
  if (i > 0) t += -0.5 * i * (gb * std::pow(qb, i - 1));
  if (i + j > 0) t *= std::pow(qc, i + j - 1);
  t = fa * (t * hc);
  vs += t;
  double vt = 0.5 * (1.0 + a) * vr + 0.5 * (1.0 + b) * t;
  double u = dhc * std::pow(qc, i + j);
  if (i + j > 0) u -= 0.5 * (i + j) * (hc * std::pow(qc, i + j - 1));
  u = fa * (gb * u);
  u *= std::pow(qb, i);
  vt += u;
  double sc = std::pow(2.0, 2 * i + j + 1.5);
  g[0] = vr * sc; g[1] = vs * sc; g[2] = vt * sc;
}

// n-point Gauss-Legendre rule on [-1, 1] (Newton on the Legendre recurrence).
static void gauss(int n, std::vector<double>& x, std::vector<double>& w)
{
  x.resize(n); w.resize(n);
  for (int i = 0; i < n; i++) {
    double t = -std::cos(M_PI * (i + 0.75) / (n + 0.5)), dp = 1.0;
    for (int it = 0; it < 100; it++) {
      double p0 = 1.0, p1 = t;
      for (int k = 2; k <= n; k++) { double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
      dp = n * (t * p1 - p0) / (t * t - 1.0);
      double dt = p1 / dp;
      t -= dt;
      if (std::fabs(dt) < 1e-16) break;
    }
    double p0 = 1.0, p1 = t;
    for (int k = 2; k <= n; k++) { double p2 = ((2 * k - 1) * t * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
    dp = n * (t * p1 - p0) / (t * t - 1.0);
    x[i] = t; w[i] = 2.0 / ((1.0 - t * t) * dp * dp);
  }
}

// Collapsed Gauss rule on the reference triangle (-1,-1), (1,-1), (-1,1):
// exact for polynomials of degree <= 2 n - 2 (weights sum to its area 2).
static void tri_rule(int n, std::vector<double>& r, std::vector<double>& s, std::vector<double>& w)
{
  std::vector<double> xa, wa, xb, wb;
  gauss(n, xa, wa);
  gauss(n + 1, xb, wb);
  r.clear(); s.clear(); w.clear();
  for (size_t q = 0; q < xb.size(); q++)
    for (size_t p = 0; p < xa.size(); p++) {
      r.push_back(0.5 * (1.0 + xa[p]) * (1.0 - xb[q]) - 1.0);
      s.push_back(xb[q]);
      w.push_back(wa[p] * wb[q] * 0.5 * (1.0 - xb[q]));
    }
}

// -------------------------------------------------------- VCJH constants
static double factorial(int n) { double f = 1; for (int i = 2; i <= n; i++) f *= i; return f; }
static double binom(int n, int k) { return std::round(factorial(n) / (factorial(k) * factorial(n - k))); }

// c of the VCJH families on triangles (dims 2) and tetrahedra (dims 3): the
// user's c (scheme 0), DG (1), SD-like (2), HU-like (3) and c+ (4).  The
// SD- and HU-like members scale the 1-D c_SD / c_HU by the ratio of the
// simplex to the 1-D c+ (published values: Castonguay, Vincent & Jameson 2012
// for triangles, Williams & Jameson 2014 for tetrahedra; the reference's
// src/funcs.cpp:586-635 and src/eles_tets.cpp:1165-1215 use the same numbers).
static bool vcjh_c(int dims, int scheme, int P, double user_c, double& c)
{
  double ap = 1. / std::pow(2.0, P) * factorial(2 * P) / (factorial(P) * factorial(P));
  double c_sd = (2.0 * P) / ((2 * P + 1) * (P + 1) * (factorial(P) * ap) * (factorial(P) * ap));
  double c_hu = (2.0 * (P + 1)) / ((2 * P + 1) * P * (factorial(P) * ap) * (factorial(P) * ap));
  if (scheme == 0) { c = user_c; return true; }
  if (scheme == 1) { c = 0.0; return true; }
  static const double cp1[6] = {0, 0, 0.206, 3.80e-3, 4.67e-5, 4.28e-7};
  static const double cp2[6] = {0, 0, 3.13e-2, 4.67e-4, 6.55e-6, 0};
  static const double cp3[6] = {0, 0, 3.07e-2, 5.44e-4, 9.92e-6, 1.10e-7};
  if (P < 2 || P > 5) return false;
  double cplus = dims == 2 ? cp2[P] : cp3[P];
  if (cplus == 0.0) return false;
  if (scheme == 2) { c = (c_sd / cp1[P]) * cplus; return true; }
  if (scheme == 3) { c = (c_hu / cp1[P]) * cplus; return true; }
  if (scheme == 4) { c = cplus; return true; }
  return false;
}

// Filter of the simplex VCJH schemes: F = (I + M^-1 K)^-1 with M^-1 = V V^T
// and K = c sum_w coeff_w (D^w)^T D^w over the mixed derivatives D^w of
// order P (triangles: Dr^(P-k) Ds^k with binomial weights; tetrahedra:
// Dr^a Ds^b Dt^g with trinomial weights), all divided by the point count.
static Mat vcjh_filter(int dims, int P, double c, const Mat& V, const std::vector<Mat>& Dn)
{
  int n = (int)std::lround(std::sqrt((double)V.size()));
  Mat I((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) I[(size_t)i * n + i] = 1.0;
  Mat K((size_t)n * n, 0.0);
  auto add = [&](const Mat& Dw, double coeff) {
    Mat DT((size_t)n * n);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) DT[(size_t)j * n + i] = Dw[(size_t)i * n + j];
    Mat DTD = matmul(n, n, n, DT, Dw);
    for (size_t q = 0; q < K.size(); q++) K[q] += c * coeff * DTD[q];
  };
  auto power = [&](Mat M, int d, int e) {
    for (int q = 0; q < e; q++) M = matmul(n, n, n, M, Dn[d]);
    return M;
  };
  if (dims == 2) {
    for (int k = 0; k <= P; k++) add(power(power(I, 1, k), 0, P - k), (1.0 / n) * binom(P, k));
  } else {
    for (int v = 1; v <= P + 1; v++)
      for (int w = 1; w <= v; w++)
        add(power(power(power(I, 0, P - v + 1), 1, v - w), 2, w - 1),
            (1.0 / n) * binom(P, v - 1) * binom(v - 1, w - 1));
  }
  Mat VT((size_t)n * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) VT[(size_t)j * n + i] = V[(size_t)i * n + j];
  Mat A = matmul(n, n, n, matmul(n, n, n, V, VT), K);
  for (int i = 0; i < n; i++) A[(size_t)i * n + i] += 1.0;
  Mat F;
  invert(n, A, F);
  return F;
}

// ------------------------------------------------------------ element types
struct Element {
  int type = 0, D = 3, P = 0, nu = 0, nf = 0, nface = 0;
  int nfpf[6] = {};
  int face0[7] = {};                    // first flux point of each face
  std::vector<double> lu, tf, tn;       // (n, 3) point-major (z = 0 in 2-D)
  // tets and triangles: inverse Vandermonde of the solution points; prisms:
  // of the triangle points, plus the 1-D points
  std::vector<std::array<int, 3>> m3;
  std::vector<std::array<int, 2>> m2;
  Mat Vinv;
  int ntri = 0;
  std::vector<double> x1d;
  Line1D line;                          // quads, hexes and the prisms' 1-D direction
  Mat opp3;                             // (nu, nf) row-major
};

static int tri_count(int P) { return (P + 1) * (P + 2) / 2; }

// Nodal basis of every solution point at x (l[nu]).
static void basis(const Element& E, const double* x, double* l)
{
  if (E.type == FR_ELE_TRI) {
    std::vector<double> phi(E.nu);
    for (int i = 0; i < E.nu; i++) phi[i] = dub2(x[0], x[1], E.m2[i][0], E.m2[i][1]);
    for (int j = 0; j < E.nu; j++) {
      double s = 0.0;
      for (int i = 0; i < E.nu; i++) s += E.Vinv[(size_t)i * E.nu + j] * phi[i];
      l[j] = s;
    }
  } else if (E.type == FR_ELE_QUAD) {
    int n1 = E.P + 1;
    for (int b = 0; b < n1; b++)
      for (int a = 0; a < n1; a++) l[a + n1 * b] = lagrange(x[0], a, E.line.loc, n1) * lagrange(x[1], b, E.line.loc, n1);
  } else if (E.type == FR_ELE_TET) {
    std::vector<double> phi(E.nu);
    for (int i = 0; i < E.nu; i++) phi[i] = dub3(x, E.m3[i]);
    for (int j = 0; j < E.nu; j++) {
      double s = 0.0;
      for (int i = 0; i < E.nu; i++) s += E.Vinv[(size_t)i * E.nu + j] * phi[i];
      l[j] = s;
    }
  } else if (E.type == FR_ELE_PRISM) {
    int nt = E.ntri, n1 = E.P + 1;
    std::vector<double> phi(nt), lt(nt);
    for (int i = 0; i < nt; i++) phi[i] = dub2(x[0], x[1], E.m2[i][0], E.m2[i][1]);
    for (int j = 0; j < nt; j++) {
      double s = 0.0;
      for (int i = 0; i < nt; i++) s += E.Vinv[(size_t)i * nt + j] * phi[i];
      lt[j] = s;
    }
    for (int c = 0; c < n1; c++) {
      double lz = lagrange(x[2], c, E.x1d.data(), n1);
      for (int j = 0; j < nt; j++) l[nt * c + j] = lt[j] * lz;
    }
  } else {
    int n1 = E.P + 1;
    for (int c = 0; c < n1; c++)
      for (int b = 0; b < n1; b++)
        for (int a = 0; a < n1; a++)
          l[a + n1 * (b + n1 * c)] = lagrange(x[0], a, E.line.loc, n1) * lagrange(x[1], b, E.line.loc, n1) *
                                     lagrange(x[2], c, E.line.loc, n1);
  }
}

// Derivative along reference coordinate d of every nodal basis function at x.
static void dbasis(const Element& E, const double* x, int d, double* l)
{
  if (E.type == FR_ELE_TRI) {
    std::vector<double> dphi(E.nu);
    for (int i = 0; i < E.nu; i++) {
      double gr, gs;
      grad_dub2(x[0], x[1], E.m2[i][0], E.m2[i][1], gr, gs);
      dphi[i] = d == 0 ? gr : gs;
    }
    for (int j = 0; j < E.nu; j++) {
      double s = 0.0;
      for (int i = 0; i < E.nu; i++) s += E.Vinv[(size_t)i * E.nu + j] * dphi[i];
      l[j] = s;
    }
  } else if (E.type == FR_ELE_QUAD) {
    int n1 = E.P + 1;
    const double* X = E.line.loc;
    for (int b = 0; b < n1; b++)
      for (int a = 0; a < n1; a++) {
        double fa = d == 0 ? dlagrange(x[0], a, X, n1) : lagrange(x[0], a, X, n1);
        double fb = d == 1 ? dlagrange(x[1], b, X, n1) : lagrange(x[1], b, X, n1);
        l[a + n1 * b] = fa * fb;
      }
  } else if (E.type == FR_ELE_TET) {
    std::vector<double> dphi(E.nu);
    for (int i = 0; i < E.nu; i++) { double g[3]; grad_dub3(x, E.m3[i], g); dphi[i] = g[d]; }
    for (int j = 0; j < E.nu; j++) {
      double s = 0.0;
      for (int i = 0; i < E.nu; i++) s += E.Vinv[(size_t)i * E.nu + j] * dphi[i];
      l[j] = s;
    }
  } else if (E.type == FR_ELE_PRISM) {
    int nt = E.ntri, n1 = E.P + 1;
    std::vector<double> phi(nt), lt(nt);
    for (int i = 0; i < nt; i++) {
      if (d == 2) { phi[i] = dub2(x[0], x[1], E.m2[i][0], E.m2[i][1]); continue; }
      double gr, gs;
      grad_dub2(x[0], x[1], E.m2[i][0], E.m2[i][1], gr, gs);
      phi[i] = d == 0 ? gr : gs;
    }
    for (int j = 0; j < nt; j++) {
      double s = 0.0;
      for (int i = 0; i < nt; i++) s += E.Vinv[(size_t)i * nt + j] * phi[i];
      lt[j] = s;
    }
    for (int c = 0; c < n1; c++) {
      double lz = d == 2 ? dlagrange(x[2], c, E.x1d.data(), n1) : lagrange(x[2], c, E.x1d.data(), n1);
      for (int j = 0; j < nt; j++) l[nt * c + j] = lt[j] * lz;
    }
  } else {
    int n1 = E.P + 1;
    const double* X = E.line.loc;
    for (int c = 0; c < n1; c++)
      for (int b = 0; b < n1; b++)
        for (int a = 0; a < n1; a++) {
          double fa = d == 0 ? dlagrange(x[0], a, X, n1) : lagrange(x[0], a, X, n1);
          double fb = d == 1 ? dlagrange(x[1], b, X, n1) : lagrange(x[1], b, X, n1);
          double fc = d == 2 ? dlagrange(x[2], c, X, n1) : lagrange(x[2], c, X, n1);
          l[a + n1 * (b + n1 * c)] = fa * fb * fc;
        }
  }
}

static void set_faces(Element& E)
{
  E.face0[0] = 0;
  for (int f = 0; f < E.nface; f++) E.face0[f + 1] = E.face0[f] + E.nfpf[f];
  E.nf = E.face0[E.nface];
}

// Nodal derivative matrices D_d (row-major nu x nu, D_d[k][j] = dl_j/dr_d at
// solution point k) of a modal basis given its Vandermonde V.
static std::vector<Mat> nodal_derivatives(const Element& E)
{
  std::vector<Mat> D(E.D, Mat((size_t)E.nu * E.nu));
  std::vector<double> l(E.nu);
  for (int d = 0; d < E.D; d++)
    for (int k = 0; k < E.nu; k++) {
      dbasis(E, &E.lu[3 * k], d, l.data());
      for (int j = 0; j < E.nu; j++) D[d][(size_t)k * E.nu + j] = l[j];
    }
  return D;
}

// Tetrahedra (src/eles_tets.cpp:68-140 set-up, 233-331 points, 589-623
// normals, 972-1131 correction).
static bool setup_tet(Element& E, const fr_element_opts& o, std::string& err)
{
  int P = E.P, nt = tri_count(P);
  if (P < 1 || P > 5) { err = "tetrahedra: order 1-5"; return false; }
  E.nu = (P + 1) * (P + 2) * (P + 3) / 6;
  E.nface = 4;
  for (int f = 0; f < 4; f++) E.nfpf[f] = nt;
  set_faces(E);
  const double* up = o.upts_type_tet == 0 ? kTetInter[P] : o.upts_type_tet == 1 ? kTetAlpha[P] : nullptr;
  const double* fp = o.fpts_type_tet == 0 ? kTriInter[P] : o.fpts_type_tet == 1 ? kTriAlpha[P] : nullptr;
  if (!up || !fp) { err = "tetrahedra: point type 0 (interior) or 1 (alpha-optimised)"; return false; }
  E.lu.assign(up, up + 3 * E.nu);
  // flux points: the triangle set mapped onto each face, row by row
  E.tf.assign(3 * E.nf, 0.0);
  E.tn.assign(3 * E.nf, 0.0);
  for (int j = 0; j <= P; j++)
    for (int i = 0; i <= P - j; i++) {
      int q = j * (P + 1) - (j - 1) * j / 2 + i;
      int qr = j * (P + 1) - (j - 1) * j / 2 + (P - j - i);
      double a = fp[2 * q], b = fp[2 * q + 1];
      double* t0 = &E.tf[3 * q];
      t0[0] = fp[2 * qr]; t0[1] = a; t0[2] = b;
      double* t1 = &E.tf[3 * (nt + q)];
      t1[0] = -1.0; t1[1] = b; t1[2] = a;
      double* t2 = &E.tf[3 * (2 * nt + q)];
      t2[0] = a; t2[1] = -1.0; t2[2] = b;
      double* t3 = &E.tf[3 * (3 * nt + q)];
      t3[0] = b; t3[1] = a; t3[2] = -1.0;
    }
  for (int f = 0; f < 4; f++)
    for (int q = 0; q < nt; q++) {
      double* n = &E.tn[3 * (f * nt + q)];
      if (f == 0) n[0] = n[1] = n[2] = 1. / std::sqrt(3.);
      else n[f - 1] = -1.0;
    }
  tet_modes(P, E.m3);
  Mat V((size_t)E.nu * E.nu);
  for (int i = 0; i < E.nu; i++)
    for (int j = 0; j < E.nu; j++) V[(size_t)i * E.nu + j] = dub3(&E.lu[3 * i], E.m3[j]);
  if (!invert(E.nu, V, E.Vinv)) { err = "tetrahedra: singular Vandermonde matrix"; return false; }

  // DG lifting of each flux point's unit jump: sum_i phi_i(x) int_face phi_i l_q dA
  std::vector<std::array<int, 2>> m2;
  tri_modes(P, m2);
  std::vector<double> qr, qs, qw;
  tri_rule(P + 2, qr, qs, qw);
  Mat dg((size_t)E.nu * E.nf, 0.0);
  std::vector<double> phiu((size_t)E.nu * E.nu);
  for (int j = 0; j < E.nu; j++)
    for (int i = 0; i < E.nu; i++) phiu[(size_t)j * E.nu + i] = dub3(&E.lu[3 * j], E.m3[i]);
  for (int f = 0; f < 4; f++) {
    // face coordinates (rho, sigma) and the map back to (r, s, t)
    auto param = [f](const double* x, double& rho, double& sig) {
      if (f == 0) { rho = x[0]; sig = x[2]; }
      else if (f == 1) { rho = x[2]; sig = x[1]; }
      else if (f == 2) { rho = x[0]; sig = x[2]; }
      else { rho = x[1]; sig = x[0]; }
    };
    auto point = [f](double rho, double sig, double* x) {
      if (f == 0) { x[0] = rho; x[2] = sig; x[1] = -1. - sig - rho; }
      else if (f == 1) { x[0] = -1.0; x[1] = sig; x[2] = rho; }
      else if (f == 2) { x[0] = rho; x[1] = -1.0; x[2] = sig; }
      else { x[0] = sig; x[1] = rho; x[2] = -1.0; }
    };
    double jac = f == 0 ? std::sqrt(3.) : 1.0;
    Mat M((size_t)nt * nt), Minv;
    for (int m = 0; m < nt; m++) {
      double rho, sig;
      param(&E.tf[3 * (f * nt + m)], rho, sig);
      for (int q = 0; q < nt; q++) M[(size_t)m * nt + q] = dub2(rho, sig, m2[q][0], m2[q][1]);
    }
    if (!invert(nt, M, Minv)) { err = "tetrahedra: singular face Vandermonde matrix"; return false; }
    for (int m = 0; m < nt; m++) {
      std::vector<double> coeff(E.nu, 0.0);
      for (size_t p = 0; p < qw.size(); p++) {
        double g = 0.0;
        for (int q = 0; q < nt; q++) g += Minv[(size_t)q * nt + m] * dub2(qr[p], qs[p], m2[q][0], m2[q][1]);
        double x[3];
        point(qr[p], qs[p], x);
        for (int i = 0; i < E.nu; i++) coeff[i] += qw[p] * dub3(x, E.m3[i]) * g;
      }
      for (int j = 0; j < E.nu; j++) {
        double s = 0.0;
        for (int i = 0; i < E.nu; i++) s += coeff[i] * jac * phiu[(size_t)j * E.nu + i];
        dg[(size_t)j * E.nf + f * nt + m] = s;
      }
    }
  }
  double c;
  if (!vcjh_c(3, o.vcjh_scheme_tet, P, o.c_tet, c)) { err = "tetrahedra: VCJH scheme not defined for this order"; return false; }
  std::vector<Mat> Dn = nodal_derivatives(E);
  Mat F = vcjh_filter(3, P, c, V, Dn);
  E.opp3 = matmul(E.nu, E.nu, E.nf, F, dg);
  return true;
}

// Triangle VCJH correction at the triangle points for unit jumps at the edge
// points (3 edges x (P+1) points), edge by edge: edge 0 s = -1, edge 1 the
// hypotenuse from (1,-1) to (-1,1), edge 2 r = -1 (src/funcs.cpp:371-405,
// 806-893); (ntri, 3 (P+1)) row-major.
static bool tri_correction(int P, const double* tri, const double* x1d, int scheme, double user_c, Mat& out,
                           std::string& err)
{
  int nt = tri_count(P), ne = 3 * (P + 1);
  std::vector<std::array<int, 2>> m2;
  tri_modes(P, m2);
  Mat V((size_t)nt * nt), Vinv;
  for (int i = 0; i < nt; i++)
    for (int j = 0; j < nt; j++) V[(size_t)i * nt + j] = dub2(tri[2 * i], tri[2 * i + 1], m2[j][0], m2[j][1]);
  if (!invert(nt, V, Vinv)) { err = "prisms: singular triangle Vandermonde matrix"; return false; }
  // The edge integrals use the reference's fixed 5-point Gauss rule
  // (cubature_1d(10) in eval_div_dg_tri, src/funcs.cpp:819, takes (10 + 1) / 2
  // points, src/cubature_1d.cpp:61): exact for the degree-2P integrands up to
  // P = 4; at P = 5 the reference's lift is that rule's, and so is this one.
  std::vector<double> gx, gw;
  gauss(5, gx, gw);
  Mat dg((size_t)nt * ne, 0.0);
  for (int e = 0; e < 3; e++) {
    double half = e == 1 ? std::sqrt(2.) : 1.0;
    for (int m = 0; m <= P; m++) {
      std::vector<double> coeff(nt, 0.0);
      for (size_t p = 0; p < gx.size(); p++) {
        double x = gx[p], r, s;
        if (e == 0) { r = x; s = -1.0; }
        else if (e == 1) { r = -x; s = x; }
        else { r = -1.0; s = -x; }
        double g = lagrange(x, m, x1d, P + 1);
        for (int i = 0; i < nt; i++) coeff[i] += gw[p] * dub2(r, s, m2[i][0], m2[i][1]) * g;
      }
      for (int j = 0; j < nt; j++) {
        double s = 0.0;
        for (int i = 0; i < nt; i++) s += coeff[i] * half * dub2(tri[2 * j], tri[2 * j + 1], m2[i][0], m2[i][1]);
        dg[(size_t)j * ne + e * (P + 1) + m] = s;
      }
    }
  }
  double c;
  if (!vcjh_c(2, scheme, P, user_c, c)) { err = "prisms: triangle VCJH scheme not defined for this order"; return false; }
  std::vector<Mat> Dn(2, Mat((size_t)nt * nt));
  for (int d = 0; d < 2; d++) {
    Mat Vd((size_t)nt * nt);
    for (int i = 0; i < nt; i++)
      for (int j = 0; j < nt; j++) {
        double gr, gs;
        grad_dub2(tri[2 * i], tri[2 * i + 1], m2[j][0], m2[j][1], gr, gs);
        Vd[(size_t)i * nt + j] = d == 0 ? gr : gs;
      }
    // D = Vd V^-1 acting on nodal values
    Dn[d] = matmul(nt, nt, nt, Vd, Vinv);
  }
  Mat F = vcjh_filter(2, P, c, V, Dn);
  out = matmul(nt, nt, ne, F, dg);
  return true;
}

// Prisms: triangle x 1-D line (src/eles_pris.cpp:51-130 set-up, 198-352
// points, 582-623 normals, 995-1194 correction).
static bool setup_prism(Element& E, const fr_element_opts& o, std::string& err)
{
  int P = E.P, nt = tri_count(P), n1 = P + 1;
  if (P < 1 || P > 5) { err = "prisms: order 1-5"; return false; }
  E.ntri = nt;
  E.nu = nt * n1;
  E.nface = 5;
  E.nfpf[0] = E.nfpf[1] = nt;
  E.nfpf[2] = E.nfpf[3] = E.nfpf[4] = n1 * n1;
  set_faces(E);
  const double* tri = o.upts_type_pri_tri == 0 ? kTriInter[P] : o.upts_type_pri_tri == 1 ? kTriAlpha[P] : nullptr;
  if (!tri) { err = "prisms: triangle point type 0 (interior) or 1 (alpha-optimised)"; return false; }
  E.x1d.assign(n1, 0.0);
  if (!points_1d(P, o.upts_type_pri_1d, E.x1d.data())) { err = "prisms: 1-D point type 0 (Gauss) or 1 (Lobatto)"; return false; }
  const double* X = E.x1d.data();
  E.lu.assign(3 * E.nu, 0.0);
  for (int c = 0; c < n1; c++)
    for (int j = 0; j < nt; j++) {
      double* p = &E.lu[3 * (nt * c + j)];
      p[0] = tri[2 * j]; p[1] = tri[2 * j + 1]; p[2] = X[c];
    }
  E.tf.assign(3 * E.nf, 0.0);
  E.tn.assign(3 * E.nf, 0.0);
  for (int q = 0; q < nt; q++) {
    double* a = &E.tf[3 * q];
    a[0] = tri[2 * q + 1]; a[1] = tri[2 * q]; a[2] = -1.0;
    double* b = &E.tf[3 * (nt + q)];
    b[0] = tri[2 * q]; b[1] = tri[2 * q + 1]; b[2] = 1.0;
    E.tn[3 * q + 2] = -1.0;
    E.tn[3 * (nt + q) + 2] = 1.0;
  }
  for (int f = 0; f < 3; f++)
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n1; j++) {
        int q = E.face0[2 + f] + i * n1 + j;
        double* t = &E.tf[3 * q];
        double* n = &E.tn[3 * q];
        if (f == 0) { t[0] = X[j]; t[1] = -1.0; n[1] = -1.0; }
        else if (f == 1) { t[0] = X[P - j]; t[1] = X[j]; n[0] = n[1] = 1. / std::sqrt(2.); }
        else { t[0] = -1.0; t[1] = X[P - j]; n[0] = -1.0; }
        t[2] = X[i];
      }
  tri_modes(P, E.m2);
  Mat V((size_t)nt * nt);
  for (int i = 0; i < nt; i++)
    for (int j = 0; j < nt; j++) V[(size_t)i * nt + j] = dub2(tri[2 * i], tri[2 * i + 1], E.m2[j][0], E.m2[j][1]);
  if (!invert(nt, V, E.Vinv)) { err = "prisms: singular triangle Vandermonde matrix"; return false; }
  Mat ct;
  if (!tri_correction(P, tri, X, o.vcjh_scheme_tri, o.c_tri, ct, err)) return false;
  double eta = vcjh_eta(o.vcjh_scheme_pri_1d, P, o.eta_pri);
  if (std::isnan(eta)) { err = "prisms: 1-D VCJH scheme not defined for this order"; return false; }
  // face-0 flux point q sits over the triangle point with its row and
  // column indices exchanged (the face's (r, s) are swapped)
  std::vector<int> swap_rc(nt);
  for (int j = 0; j <= P; j++)
    for (int i = 0; i <= P - j; i++) swap_rc[j * (P + 1) - (j - 1) * j / 2 + i] = i * (P + 1) - (i - 1) * i / 2 + j;
  E.opp3.assign((size_t)E.nu * E.nf, 0.0);
  for (int u = 0; u < E.nu; u++) {
    int u1 = u / nt, ut = u % nt;
    double z = E.lu[3 * u + 2];
    for (int q = 0; q < E.nf; q++) {
      double v = 0.0;
      if (q < nt) {
        if (swap_rc[q] == ut) v = -dvcjh(z, 0, P, eta);
      } else if (q < 2 * nt) {
        if (q - nt == ut) v = dvcjh(z, 1, P, eta);
      } else {
        int f = (q - 2 * nt) / (n1 * n1), r = (q - 2 * nt) % (n1 * n1);
        if (r / n1 == u1) v = ct[(size_t)ut * (3 * n1) + f * n1 + r % n1];
      }
      E.opp3[(size_t)u * E.nf + q] = v;
    }
  }
  return true;
}

// Triangles (src/eles_tris.cpp:66-137 set-up, 185-272 points, 450-478
// normals, 644-648 correction): flux points on the edges at the 1-D points
// of fpts_type_tri.
static bool setup_tri(Element& E, const fr_element_opts& o, std::string& err)
{
  int P = E.P, n1 = P + 1;
  if (P < 1 || P > 5) { err = "triangles: order 1-5"; return false; }
  E.D = 2;
  E.nu = tri_count(P);
  E.nface = 3;
  for (int f = 0; f < 3; f++) E.nfpf[f] = n1;
  set_faces(E);
  const double* tri = o.upts_type_tri == 0 ? kTriInter[P] : o.upts_type_tri == 1 ? kTriAlpha[P] : nullptr;
  if (!tri) { err = "triangles: point type 0 (interior) or 1 (alpha-optimised)"; return false; }
  E.x1d.assign(n1, 0.0);
  if (!points_1d(P, o.fpts_type_tri, E.x1d.data())) { err = "triangles: flux point type 0 (Gauss) or 1 (Lobatto)"; return false; }
  const double* X = E.x1d.data();
  E.lu.assign(3 * E.nu, 0.0);
  for (int j = 0; j < E.nu; j++) { E.lu[3 * j] = tri[2 * j]; E.lu[3 * j + 1] = tri[2 * j + 1]; }
  E.tf.assign(3 * E.nf, 0.0);
  E.tn.assign(3 * E.nf, 0.0);
  for (int f = 0; f < 3; f++)
    for (int j = 0; j < n1; j++) {
      double* t = &E.tf[3 * (n1 * f + j)];
      double* n = &E.tn[3 * (n1 * f + j)];
      if (f == 0) { t[0] = X[j]; t[1] = -1.0; n[1] = -1.0; }
      else if (f == 1) { t[0] = X[P - j]; t[1] = X[j]; n[0] = n[1] = 1. / std::sqrt(2.); }
      else { t[0] = -1.0; t[1] = X[P - j]; n[0] = -1.0; }
    }
  tri_modes(P, E.m2);
  Mat V((size_t)E.nu * E.nu);
  for (int i = 0; i < E.nu; i++)
    for (int j = 0; j < E.nu; j++) V[(size_t)i * E.nu + j] = dub2(tri[2 * i], tri[2 * i + 1], E.m2[j][0], E.m2[j][1]);
  if (!invert(E.nu, V, E.Vinv)) { err = "triangles: singular Vandermonde matrix"; return false; }
  return tri_correction(P, tri, X, o.vcjh_scheme_tri, o.c_tri, E.opp3, err);
}

// Quadrilaterals in the reference's point orders (src/eles_quads.cpp:237-300),
// corrected like the hexahedra.
static bool setup_quad(Element& E, const fr_element_opts& o, std::string& err)
{
  if (!make_line(E.P, o.upts_type_quad, o.vcjh_scheme_quad, o.eta_quad, E.line, err)) return false;
  int n1 = E.P + 1;
  E.D = 2;
  E.nu = n1 * n1;
  E.nface = 4;
  for (int f = 0; f < 4; f++) E.nfpf[f] = n1;
  set_faces(E);
  std::vector<double> lu, tf, tn;
  element_points(2, E.line, lu, tf, tn);
  E.lu.assign(3 * E.nu, 0.0); E.tf.assign(3 * E.nf, 0.0); E.tn.assign(3 * E.nf, 0.0);
  for (int k = 0; k < E.nu; k++) for (int d = 0; d < 2; d++) E.lu[3 * k + d] = lu[2 * k + d];
  for (int q = 0; q < E.nf; q++)
    for (int d = 0; d < 2; d++) { E.tf[3 * q + d] = tf[2 * q + d]; E.tn[3 * q + d] = tn[2 * q + d]; }
  E.opp3.assign((size_t)E.nu * E.nf, 0.0);
  for (int q = 0; q < E.nf; q++) {
    const double* t = &E.tf[3 * q];
    const double* n = &E.tn[3 * q];
    int ax = n[0] != 0 ? 0 : 1;
    bool plus = n[ax] > 0;
    for (int u = 0; u < E.nu; u++) {
      int c[2] = {u % n1, u / n1};
      if (E.line.loc[c[1 - ax]] == t[1 - ax]) E.opp3[(size_t)u * E.nf + q] = plus ? E.line.gR[c[ax]] : -E.line.gL[c[ax]];
    }
  }
  return true;
}

// Hexahedra in the reference's point orders (src/eles_hexas.cpp:240-324),
// correction g'_L / g'_R along the face normal on the line of solution points
// through each flux point.
static bool setup_hex(Element& E, const fr_element_opts& o, std::string& err)
{
  if (!make_line(E.P, o.upts_type_hexa, o.vcjh_scheme_hexa, o.eta_hexa, E.line, err)) return false;
  int n1 = E.P + 1;
  E.nu = n1 * n1 * n1;
  E.nface = 6;
  for (int f = 0; f < 6; f++) E.nfpf[f] = n1 * n1;
  set_faces(E);
  element_points(3, E.line, E.lu, E.tf, E.tn);
  E.opp3.assign((size_t)E.nu * E.nf, 0.0);
  for (int q = 0; q < E.nf; q++) {
    const double* t = &E.tf[3 * q];
    const double* n = &E.tn[3 * q];
    int ax = n[0] != 0 ? 0 : n[1] != 0 ? 1 : 2;
    bool plus = n[ax] > 0;
    for (int u = 0; u < E.nu; u++) {
      int c[3] = {u % n1, (u / n1) % n1, u / (n1 * n1)};
      bool on = true;
      for (int d = 0; d < 3; d++)
        if (d != ax && E.line.loc[c[d]] != t[d]) on = false;
      if (on) E.opp3[(size_t)u * E.nf + q] = plus ? E.line.gR[c[ax]] : -E.line.gL[c[ax]];
    }
  }
  return true;
}

static bool make_element(int type, int P, const fr_element_opts& o, Element& E, std::string& err)
{
  E = Element();
  E.type = type; E.P = P;
  if (type == FR_ELE_TRI) return setup_tri(E, o, err);
  if (type == FR_ELE_QUAD) return setup_quad(E, o, err);
  if (type == FR_ELE_TET) return setup_tet(E, o, err);
  if (type == FR_ELE_PRISM) return setup_prism(E, o, err);
  if (type == FR_ELE_HEX) return setup_hex(E, o, err);
  err = "element type: 0 (triangle), 1 (quadrilateral), 2 (tetrahedron), 3 (prism) or 4 (hexahedron)";
  return false;
}

// ------------------------------------------------------------- geometry
static int shape_nodes(int type)
{
  return type == FR_ELE_TRI ? 3 : type == FR_ELE_QUAD ? 4 : type == FR_ELE_TET ? 4 : type == FR_ELE_PRISM ? 6 : 8;
}
static int type_dims(int type) { return type == FR_ELE_TRI || type == FR_ELE_QUAD ? 2 : 3; }

// Linear shape functions of the reference's vertex orders
// (src/eles_tets.cpp:862-950, src/eles_pris.cpp:852-990,
// src/eles_hexas.cpp:985-1060) and their derivatives dN[node + ns * d].
static void shape(int type, const double* r, double* N, double* dN)
{
  if (type == FR_ELE_TRI) {
    N[0] = -0.5 * (r[0] + r[1]); N[1] = 0.5 * (r[0] + 1.); N[2] = 0.5 * (r[1] + 1.);
    dN[0] = -0.5; dN[1] = 0.5; dN[2] = 0.0;
    dN[3] = -0.5; dN[4] = 0.0; dN[5] = 0.5;
  } else if (type == FR_ELE_QUAD) {
    static const double c2[2] = {-1.0, 1.0};
    for (int s = 0; s < 4; s++) {
      int a = s & 1, b = (s >> 1) & 1;
      double la = lagrange(r[0], a, c2, 2), lb = lagrange(r[1], b, c2, 2);
      N[s] = la * lb; dN[s] = dlagrange(r[0], a, c2, 2) * lb; dN[s + 4] = la * dlagrange(r[1], b, c2, 2);
    }
  } else if (type == FR_ELE_TET) {
    N[0] = -0.5 * (r[0] + r[1] + r[2] + 1.); N[1] = 0.5 * (r[0] + 1.); N[2] = 0.5 * (r[1] + 1.); N[3] = 0.5 * (r[2] + 1.);
    for (int d = 0; d < 3; d++)
      for (int k = 0; k < 4; k++) dN[k + 4 * d] = k == 0 ? -0.5 : (k == d + 1 ? 0.5 : 0.0);
  } else if (type == FR_ELE_PRISM) {
    double x = r[0], y = r[1], z = r[2];
    N[0] = 1. / 4. * (x + y) * (z - 1.); N[1] = -1. / 4. * (x + 1.) * (z - 1.); N[2] = -1. / 4. * (y + 1.) * (z - 1.);
    N[3] = -1. / 4. * (x + y) * (z + 1.); N[4] = 1. / 4. * (x + 1.) * (z + 1.); N[5] = 1. / 4. * (y + 1.) * (z + 1.);
    double* a = dN;
    a[0] = 1. / 4. * (z - 1.); a[1] = -1. / 4. * (z - 1.); a[2] = 0; a[3] = -1. / 4. * (z + 1.); a[4] = 1. / 4. * (z + 1.); a[5] = 0;
    double* b = dN + 6;
    b[0] = 1. / 4. * (z - 1.); b[1] = 0; b[2] = -1. / 4. * (z - 1.); b[3] = -1. / 4. * (z + 1.); b[4] = 0; b[5] = 1. / 4. * (z + 1.);
    double* c = dN + 12;
    c[0] = 1. / 4. * (x + y); c[1] = -1. / 4. * (x + 1.); c[2] = -1. / 4. * (y + 1.);
    c[3] = -1. / 4. * (x + y); c[4] = 1. / 4. * (x + 1.); c[5] = 1. / 4. * (y + 1.);
  } else {
    static const double c2[2] = {-1.0, 1.0};
    for (int s = 0; s < 8; s++) {
      int a = s & 1, b = (s >> 1) & 1, c = (s >> 2) & 1;
      double la = lagrange(r[0], a, c2, 2), lb = lagrange(r[1], b, c2, 2), lc = lagrange(r[2], c, c2, 2);
      double da = dlagrange(r[0], a, c2, 2), db = dlagrange(r[1], b, c2, 2), dc = dlagrange(r[2], c, c2, 2);
      N[s] = la * lb * lc; dN[s] = da * lb * lc; dN[s + 8] = la * db * lc; dN[s + 16] = la * lb * dc;
    }
  }
}

// Position and Jacobian J[j + D k] = dx_j / dr_k of one element at r
// (vertices xv with stride 3).
static void map_point(int type, const double* xv, const int* cv, const double* r, double* pos, double* J)
{
  int ns = shape_nodes(type), D = type_dims(type);
  double N[8], dN[24];
  shape(type, r, N, dN);
  for (int i = 0; i < D; i++) {
    double s = 0.0;
    for (int j = 0; j < ns; j++) s += N[j] * xv[3 * (size_t)cv[j] + i];
    pos[i] = s;
  }
  for (int j = 0; j < D; j++)
    for (int k = 0; k < D; k++) {
      double s = 0.0;
      for (int i = 0; i < ns; i++) s += dN[i + ns * k] * xv[3 * (size_t)cv[i] + j];
      J[j + D * k] = s;
    }
}

// 2-D: adj(J), det(J) and the transformed normal (src/eles.cpp:4615-4800).
static double adjugate2(const double* J, double* G)
{
  double xr = J[0], xs = J[2], yr = J[1], ys = J[3];
  G[0] = ys; G[2] = -xs; G[1] = -yr; G[3] = xr;
  return xr * ys - xs * yr;
}

static void face_normal2(const double* J, const double* t, double* v)
{
  v[0] = (t[0] * J[3]) - (t[1] * J[1]);
  v[1] = -(t[0] * J[2]) + (t[1] * J[0]);
}

// adj(J) in JGinv's layout (G[a + 3 b] = JGinv(a, b)) and det(J)
// (src/eles.cpp:4615-4680).
static double adjugate(const double* J, double* G)
{
  double xr = J[0], xs = J[3], xt = J[6], yr = J[1], ys = J[4], yt = J[7], zr = J[2], zs = J[5], zt = J[8];
  double det = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
  G[0] = ys * zt - yt * zs; G[3] = xt * zs - xs * zt; G[6] = xs * yt - xt * ys;
  G[1] = yt * zr - yr * zt; G[4] = xr * zt - xt * zr; G[7] = xt * yr - xr * yt;
  G[2] = yr * zs - ys * zr; G[5] = xs * zr - xr * zs; G[8] = xr * ys - xs * yr;
  return det;
}

// Transformed normal adj(J)^T n_ref (src/eles.cpp:4720-4800).
static void face_normal(const double* J, const double* t, double* v)
{
#define JJ(a, b) J[(a) + 3 * (b)]
  v[0] = ((t[0] * (JJ(1, 1) * JJ(2, 2) - JJ(1, 2) * JJ(2, 1))) + (t[1] * (JJ(1, 2) * JJ(2, 0) - JJ(1, 0) * JJ(2, 2))) +
          (t[2] * (JJ(1, 0) * JJ(2, 1) - JJ(1, 1) * JJ(2, 0))));
  v[1] = ((t[0] * (JJ(0, 2) * JJ(2, 1) - JJ(0, 1) * JJ(2, 2))) + (t[1] * (JJ(0, 0) * JJ(2, 2) - JJ(0, 2) * JJ(2, 0))) +
          (t[2] * (JJ(0, 1) * JJ(2, 0) - JJ(0, 0) * JJ(2, 1))));
  v[2] = ((t[0] * (JJ(0, 1) * JJ(1, 2) - JJ(0, 2) * JJ(1, 1))) + (t[1] * (JJ(0, 2) * JJ(1, 0) - JJ(0, 0) * JJ(1, 2))) +
          (t[2] * (JJ(0, 0) * JJ(1, 1) - JJ(0, 1) * JJ(1, 0))));
#undef JJ
}

}  // namespace mixed

// Row-major (nu_to, nu_from) matrix whose row j holds every nodal basis
// function of the points `from` (one element of `type` and `order`,
// point-major with D = 2 or 3 coordinates each) at to[j]: the reference's
// opp_r (eles::set_opp_r, src/eles.cpp:4135-4153) with the bases of
// eval_nodal_basis_restart (src/eles_tris.cpp:585-600, src/eles_tets.cpp,
// src/eles_pris.cpp).  Quads and hexes take their 1-D points from the x of
// the first order + 1 points, prisms their triangle points from the first
// (order+1)(order+2)/2 points and their 1-D points from z every that many.
bool nodal_interp(int type, int order, const double* from, int nu_from, const double* to, int nu_to,
                  std::vector<double>& R, std::string& err)
{
  using namespace mixed;
  if (order < 0 || order > kMaxP) { err = "restart order 0-" + std::to_string(kMaxP); return false; }
  const int D = type_dims(type), n1 = order + 1, nt = tri_count(order);
  int nu = 0;
  switch (type) {
    case FR_ELE_TRI: nu = nt; break;
    case FR_ELE_QUAD: nu = n1 * n1; break;
    case FR_ELE_TET: nu = nt * (order + 3) / 3; break;
    case FR_ELE_PRISM: nu = nt * n1; break;
    case FR_ELE_HEX: nu = n1 * n1 * n1; break;
    default: err = "element type 0-4"; return false;
  }
  if (nu_from != nu) { err = "point count does not match the order"; return false; }
  Element E;
  E.type = type; E.P = order; E.D = D; E.nu = nu;
  Mat V;
  int nv = 0;
  if (type == FR_ELE_TRI || type == FR_ELE_PRISM) {
    nv = nt;
    tri_modes(order, E.m2);
    V.resize((size_t)nt * nt);
    for (int i = 0; i < nt; i++)
      for (int j = 0; j < nt; j++) V[(size_t)i * nt + j] = dub2(from[D * i], from[D * i + 1], E.m2[j][0], E.m2[j][1]);
    if (type == FR_ELE_PRISM) {
      E.ntri = nt;
      E.x1d.resize(n1);
      for (int c = 0; c < n1; c++) E.x1d[c] = from[D * (nt * c) + 2];
    }
  } else if (type == FR_ELE_TET) {
    nv = nu;
    tet_modes(order, E.m3);
    V.resize((size_t)nu * nu);
    for (int i = 0; i < nu; i++)
      for (int j = 0; j < nu; j++) V[(size_t)i * nu + j] = dub3(&from[3 * i], E.m3[j]);
  } else {
    E.line.P = order; E.line.n1 = n1;
    for (int a = 0; a < n1; a++) E.line.loc[a] = from[D * a];
  }
  if (nv && !invert(nv, V, E.Vinv)) { err = "restart points give a singular Vandermonde matrix"; return false; }
  R.assign((size_t)nu_to * nu, 0.0);
  for (int j = 0; j < nu_to; j++) {
    double x[3] = {to[D * j], to[D * j + 1], D == 3 ? to[D * j + 2] : 0.0};
    basis(E, x, &R[(size_t)j * nu]);
  }
  return true;
}

}  // namespace frb

using namespace frb;
using namespace frb::mixed;

struct fr_mixed {
  int dims = 3, order = 0;
  int n_types = 0;
  int types[3] = {};                        // ele_type of each slot
  Element el[3];
  std::vector<int> c2v[3];                  // (ns, ne) per slot
  std::vector<long long> cell_of[3];        // global cell of each element
  std::vector<double> JG[3], dj[3], tdA[3], nrm[3], pu[3], pf[3];
  // interface groups: triangular faces (3-D) or edges (2-D), then
  // quadrilateral faces
  int n_igroups = 0, igroup_nfpi[2] = {};
  std::vector<int> itab[2];                 // (6, nfpi, ni) with ni = size / (6 nfpi)
  int n_bgroups = 0, bgroup_nfpi[2] = {};
  std::vector<int> btab[2];                 // (4, nfpi, ni)
};

namespace {
struct FKey {
  long long c[3];
  int kind;
  bool operator==(const FKey& o) const {
    return kind == o.kind && c[0] == o.c[0] && c[1] == o.c[1] && c[2] == o.c[2];
  }
};
struct FKeyHash {
  size_t operator()(const FKey& k) const {
    return (size_t)(k.c[0] * 73856093LL) ^ (size_t)(k.c[1] * 19349663LL) ^ (size_t)(k.c[2] * 83492791LL) ^
           (size_t)k.kind;
  }
};
double wrap(double c, double L, double lo)
{
  if (L <= 0) return c;
  double t = (c - lo) / L;
  t -= std::floor(t + 1e-9);
  if (t > 1.0 - 1e-9) t -= 1.0;
  return lo + t * L;
}
}  // namespace

static const fr_element_opts kDefaultOpts = {0, 0, 0, 0.0, 0, 0, 0, 0.0, 0, 0.0, 0, 1, 0.0, 0, 0, 0, 1, 0.0};

static bool element_sizes(int ele_type, int P, int& nu, int& nfc, int* per)
{
  int nt = (P + 1) * (P + 2) / 2, nq = (P + 1) * (P + 1);
  switch (ele_type) {
    case FR_ELE_TRI: nu = nt; nfc = 3; for (int f = 0; f < 3; f++) per[f] = P + 1; return true;
    case FR_ELE_QUAD: nu = nq; nfc = 4; for (int f = 0; f < 4; f++) per[f] = P + 1; return true;
    case FR_ELE_TET: nu = nt * (P + 3) / 3; nfc = 4; for (int f = 0; f < 4; f++) per[f] = nt; return true;
    case FR_ELE_PRISM: nu = nt * (P + 1); nfc = 5; per[0] = per[1] = nt; per[2] = per[3] = per[4] = nq; return true;
    case FR_ELE_HEX: nu = nq * (P + 1); nfc = 6; for (int f = 0; f < 6; f++) per[f] = nq; return true;
  }
  return false;
}

extern "C" {

fr_status fr_element_sizes(int ele_type, int order, int* n_upts, int* n_fpts, int* n_faces, int* n_fpts_per_face)
{
  g_err.clear();
  if (order < 1 || order > 5) return fail(FR_ERR_UNSUPPORTED, "order 1-5");
  int nu = 0, nfc = 0, per[6] = {};
  if (!element_sizes(ele_type, order, nu, nfc, per))
    return fail(FR_ERR_ARG, "element type: 0 (triangle), 1 (quadrilateral), 2 (tetrahedron), 3 (prism), 4 (hexahedron)");
  int nf = 0;
  for (int f = 0; f < nfc; f++) nf += per[f];
  if (n_upts) *n_upts = nu;
  if (n_fpts) *n_fpts = nf;
  if (n_faces) *n_faces = nfc;
  if (n_fpts_per_face)
    for (int f = 0; f < nfc; f++) n_fpts_per_face[f] = per[f];
  return FR_OK;
}

fr_status fr_element_operators(int ele_type, int order, const fr_element_opts* opts, double* loc_upts,
                               double* tloc_fpts, double* tnorm_fpts, double* opp_0, double* opp_1, double* opp_2,
                               double* opp_3, double* opp_5)
{
  g_err.clear();
  const fr_element_opts& o = opts ? *opts : kDefaultOpts;
  Element E;
  std::string err;
  if (!make_element(ele_type, order, o, E, err)) return fail(FR_ERR_UNSUPPORTED, err);
  int nu = E.nu, nf = E.nf, D = E.D;
  for (int k = 0; k < nu; k++)
    for (int d = 0; d < D; d++)
      if (loc_upts) loc_upts[d + D * k] = E.lu[3 * k + d];
  for (int q = 0; q < nf; q++)
    for (int d = 0; d < D; d++) {
      if (tloc_fpts) tloc_fpts[d + D * q] = E.tf[3 * q + d];
      if (tnorm_fpts) tnorm_fpts[d + D * q] = E.tn[3 * q + d];
    }
  std::vector<double> l(nu);
  for (int q = 0; q < nf; q++) {
    basis(E, &E.tf[3 * q], l.data());
    for (int u = 0; u < nu; u++) {
      if (opp_0) opp_0[q + (size_t)nf * u] = l[u];
      for (int d = 0; d < D; d++)
        if (opp_1) opp_1[q + (size_t)nf * (u + (size_t)nu * d)] = l[u] * E.tn[3 * q + d];
    }
  }
  if (opp_2)
    for (int d = 0; d < D; d++)
      for (int k = 0; k < nu; k++) {
        dbasis(E, &E.lu[3 * k], d, l.data());
        for (int u = 0; u < nu; u++) opp_2[k + (size_t)nu * (u + (size_t)nu * d)] = l[u];
      }
  for (int u = 0; u < nu; u++)
    for (int q = 0; q < nf; q++) {
      double v = E.opp3[(size_t)u * nf + q];
      if (opp_3) opp_3[u + (size_t)nu * q] = v;
      for (int d = 0; d < D; d++)
        if (opp_5) opp_5[u + (size_t)nu * (q + (size_t)nf * d)] = v * E.tn[3 * q + d];
    }
  return FR_OK;
}

fr_status fr_mixed_create(int dims, int order, const fr_element_opts* opts, long long n_verts, const double* xv_in,
                          long long n_cells, const int* cell_type, const int* cell_verts, const double* period,
                          long long n_bfaces, const long long* bface_cell, const int* bface_face,
                          const int* bface_type, fr_mixed** out)
{
  g_err.clear();
  if (!out || !xv_in || !cell_type || !cell_verts || n_verts <= 0 || n_cells <= 0)
    return fail(FR_ERR_ARG, "null or empty mesh");
  if (dims != 2 && dims != 3) return fail(FR_ERR_ARG, "dims must be 2 or 3");
  if (n_bfaces > 0 && (!bface_cell || !bface_face || !bface_type)) return fail(FR_ERR_ARG, "null boundary list");
  *out = nullptr;
  const int D = dims;
  const fr_element_opts& o = opts ? *opts : kDefaultOpts;
  std::unique_ptr<fr_mixed> m(new fr_mixed());
  m->dims = D;
  m->order = order;
  std::vector<double> xv((size_t)3 * n_verts, 0.0);     // stride 3, z = 0 in 2-D
  for (long long v = 0; v < n_verts; v++)
    for (int d = 0; d < D; d++) xv[3 * v + d] = xv_in[D * v + d];
  // element slots in the order tris, quads, tets, prisms, hexes; per cell its slot/index
  std::vector<int> slot_of(n_cells);
  std::vector<long long> ele_of(n_cells);
  int slot_for[5] = {-1, -1, -1, -1, -1};
  for (int t : {FR_ELE_TRI, FR_ELE_QUAD, FR_ELE_TET, FR_ELE_PRISM, FR_ELE_HEX})
    for (long long c = 0; c < n_cells; c++)
      if (cell_type[c] == t) {
        if (type_dims(t) != D) return fail(FR_ERR_ARG, "cell type does not match dims");
        if (slot_for[t] < 0) {
          if (m->n_types == 3) return fail(FR_ERR_ARG, "at most three element types");
          slot_for[t] = m->n_types;
          m->types[m->n_types] = t;
          std::string err;
          if (!make_element(t, order, o, m->el[m->n_types], err)) return fail(FR_ERR_UNSUPPORTED, err);
          m->n_types++;
        }
        break;
      }
  for (long long c = 0; c < n_cells; c++) {
    int t = cell_type[c];
    if (t < 0 || t > 4 || slot_for[t] < 0) return fail(FR_ERR_ARG, "cell type: 0 (tri), 1 (quad), 2 (tet), 3 (prism) or 4 (hex)");
    int s = slot_for[t];
    slot_of[c] = s;
    ele_of[c] = (long long)m->cell_of[s].size();
    m->cell_of[s].push_back(c);
    for (int k = 0; k < shape_nodes(t); k++) {
      int v = cell_verts[8 * c + k];
      if (v < 0 || v >= n_verts) return fail(FR_ERR_ARG, "vertex index out of range");
      m->c2v[s].push_back(v);
    }
  }
  // metrics (reference layouts: JGinv (D,D,nu,E), detjac (nu,E), tdA (nf,E), norm (nf,E,D))
  for (int s = 0; s < m->n_types; s++) {
    const Element& E = m->el[s];
    int ns = shape_nodes(E.type);
    size_t ne = m->cell_of[s].size(), nu = E.nu, nf = E.nf;
    m->JG[s].assign((size_t)D * D * nu * ne, 0.0); m->dj[s].assign(nu * ne, 0.0);
    m->tdA[s].assign(nf * ne, 0.0); m->nrm[s].assign(D * nf * ne, 0.0);
    m->pu[s].assign(D * nu * ne, 0.0); m->pf[s].assign(D * nf * ne, 0.0);
    for (size_t e = 0; e < ne; e++) {
      const int* cv = &m->c2v[s][ns * e];
      double p[3], J[9], G[9];
      for (size_t u = 0; u < nu; u++) {
        map_point(E.type, xv.data(), cv, &E.lu[3 * u], p, J);
        double det = D == 2 ? adjugate2(J, G) : adjugate(J, G);
        if (!(det > 0)) return fail(FR_ERR_MESH, "non-positive Jacobian at a solution point");
        m->dj[s][u + nu * e] = det;
        for (int a = 0; a < D * D; a++) m->JG[s][a + D * D * (u + nu * e)] = G[a];
        for (int d = 0; d < D; d++) m->pu[s][u + nu * (e + ne * d)] = p[d];
      }
      for (size_t q = 0; q < nf; q++) {
        map_point(E.type, xv.data(), cv, &E.tf[3 * q], p, J);
        double v[3] = {0, 0, 0};
        if (D == 2) face_normal2(J, &E.tn[3 * q], v); else face_normal(J, &E.tn[3 * q], v);
        double a = std::sqrt(D == 2 ? v[0] * v[0] + v[1] * v[1] : v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        m->tdA[s][q + nf * e] = a;
        for (int d = 0; d < D; d++) {
          m->nrm[s][q + nf * (e + ne * d)] = v[d] / a;
          m->pf[s][q + nf * (e + ne * d)] = p[d];
        }
      }
    }
  }
  // boundary faces by (cell, local face)
  std::unordered_map<long long, int> bmap;
  for (long long b = 0; b < n_bfaces; b++) {
    long long c = bface_cell[b];
    if (c < 0 || c >= n_cells) return fail(FR_ERR_ARG, "boundary face cell out of range");
    int bt = bface_type[b];
    if (!((bt >= 1 && bt <= 7) || (bt >= 11 && bt <= 16))) return fail(FR_ERR_ARG, "unknown boundary type");
    if (bface_face[b] < 0 || bface_face[b] >= m->el[slot_of[c]].nface) return fail(FR_ERR_ARG, "boundary face index");
    bmap[c * 8 + bface_face[b]] = bt;
  }
  // pair faces by their flux-point centroid (periodic coordinates wrapped),
  // flux points of paired faces by physical position; the lower cell is the
  // left side (the reference's CompConnectivity / cyclic search / rotation
  // tables, src/geometry.cpp:2412-2720, 3489-3666, src/inters.cpp:187-296)
  double per[3] = {0, 0, 0}, lo[3] = {0, 0, 0}, h = 1e300;
  if (period)
    for (int d = 0; d < D; d++) per[d] = period[d];
  for (int d = 0; d < D; d++) lo[d] = 1e300;
  for (long long v = 0; v < n_verts; v++)
    for (int d = 0; d < D; d++) lo[d] = std::min(lo[d], xv[3 * v + d]);
  for (long long c = 0; c < n_cells; c++) {
    const int* cv = &cell_verts[8 * c];
    double s2 = 0;
    for (int d = 0; d < D; d++) { double t = xv[3 * (size_t)cv[1] + d] - xv[3 * (size_t)cv[0] + d]; s2 += t * t; }
    h = std::min(h, std::sqrt(s2));
  }
  double tol = 1e-6 * h;
  auto fpos = [&](int s, size_t e, int q, int d) {
    size_t ne = m->cell_of[s].size(), nf = m->el[s].nf;
    return m->pf[s][q + nf * (e + ne * d)];
  };
  std::unordered_map<FKey, long long, FKeyHash> open;
  int nt = (order + 1) * (order + 2) / 2;
  // per group: left/right triples, gathered as rows then transposed
  std::vector<std::array<int, 6>> rows[2];
  std::vector<std::array<int, 4>> brows[2];
  for (long long c = 0; c < n_cells; c++) {
    int s = slot_of[c];
    const Element& E = m->el[s];
    size_t e = (size_t)ele_of[c];
    for (int fc = 0; fc < E.nface; fc++) {
      int np = E.nfpf[fc], kind = (D == 2 || np == nt) ? 0 : 1, q0 = E.face0[fc];
      auto bi = bmap.find(c * 8 + fc);
      if (bi != bmap.end()) {
        for (int q = 0; q < np; q++) brows[kind].push_back({E.type, (int)e, q0 + q, bi->second});
        continue;
      }
      FKey k{{0, 0, 0}, kind};
      for (int d = 0; d < D; d++) {
        double sm = 0;
        for (int q = 0; q < np; q++) sm += fpos(s, e, q0 + q, d);
        k.c[d] = (long long)std::llround(wrap(sm / np, per[d], lo[d]) / tol);
      }
      auto it = open.find(k);
      if (it == open.end()) { open.emplace(k, c * 8 + fc); continue; }
      long long ca = it->second / 8;
      int fa = (int)(it->second % 8);
      open.erase(it);
      int sa = slot_of[ca];
      size_t ea = (size_t)ele_of[ca];
      const Element& EA = m->el[sa];
      int qa0 = EA.face0[fa];
      std::vector<char> used(np, 0);
      for (int q = 0; q < np; q++) {
        int best = -1;
        double bd = 1e300;
        for (int r = 0; r < np; r++) {
          double dd = 0;
          for (int d = 0; d < D; d++) {
            double t = wrap(fpos(sa, ea, qa0 + q, d), per[d], lo[d]) - wrap(fpos(s, e, q0 + r, d), per[d], lo[d]);
            if (per[d] > 0) { if (t > 0.5 * per[d]) t -= per[d]; if (t < -0.5 * per[d]) t += per[d]; }
            dd += t * t;
          }
          if (dd < bd) { bd = dd; best = r; }
        }
        if (bd > tol * tol * 1e6 || used[best]) return fail(FR_ERR_MESH, "flux points of a face pair do not coincide");
        used[best] = 1;
        rows[kind].push_back({EA.type, (int)ea, qa0 + q, E.type, (int)e, q0 + best});
      }
    }
  }
  if (!open.empty()) return fail(FR_ERR_MESH, "unmatched faces without a boundary type");
  for (int kind = 0; kind < 2; kind++) {
    if (!rows[kind].empty()) {
      int g = m->n_igroups++;
      int np = kind == 0 ? (D == 2 ? order + 1 : nt) : (order + 1) * (order + 1);
      size_t ni = rows[kind].size() / np;
      m->igroup_nfpi[g] = np;
      m->itab[g].assign(6 * rows[kind].size(), 0);
      for (size_t i = 0; i < ni; i++)
        for (int q = 0; q < np; q++)
          for (int w = 0; w < 6; w++) m->itab[g][w + 6 * (q + np * i)] = rows[kind][i * np + q][w];
    }
    if (!brows[kind].empty()) {
      int g = m->n_bgroups++;
      int np = kind == 0 ? (D == 2 ? order + 1 : nt) : (order + 1) * (order + 1);
      size_t ni = brows[kind].size() / np;
      m->bgroup_nfpi[g] = np;
      m->btab[g].assign(4 * brows[kind].size(), 0);
      for (size_t i = 0; i < ni; i++)
        for (int q = 0; q < np; q++)
          for (int w = 0; w < 4; w++) m->btab[g][w + 4 * (q + np * i)] = brows[kind][i * np + q][w];
    }
  }
  *out = m.release();
  return FR_OK;
}

fr_status fr_mixed_destroy(fr_mixed* m)
{
  delete m;
  return FR_OK;
}

fr_status fr_mixed_info(const fr_mixed* m, int* n_types, int* ele_types, long long* n_eles, int* n_inter_groups,
                        int* n_bdy_groups)
{
  g_err.clear();
  if (!m) return fail(FR_ERR_ARG, "null mesh");
  if (n_types) *n_types = m->n_types;
  for (int s = 0; s < m->n_types; s++) {
    if (ele_types) ele_types[s] = m->types[s];
    if (n_eles) n_eles[s] = (long long)m->cell_of[s].size();
  }
  if (n_inter_groups) *n_inter_groups = m->n_igroups;
  if (n_bdy_groups) *n_bdy_groups = m->n_bgroups;
  return FR_OK;
}

fr_status fr_mixed_metrics(const fr_mixed* m, int slot, double* JGinv_upts, double* detjac_upts, double* tdA_fpts,
                           double* norm_fpts, double* pos_upts, long long* cell_of_ele)
{
  g_err.clear();
  if (!m || slot < 0 || slot >= m->n_types) return fail(FR_ERR_ARG, "element slot");
  auto cp = [](const std::vector<double>& v, double* o) { if (o) std::memcpy(o, v.data(), v.size() * sizeof(double)); };
  cp(m->JG[slot], JGinv_upts); cp(m->dj[slot], detjac_upts); cp(m->tdA[slot], tdA_fpts);
  cp(m->nrm[slot], norm_fpts); cp(m->pu[slot], pos_upts);
  if (cell_of_ele)
    for (size_t e = 0; e < m->cell_of[slot].size(); e++) cell_of_ele[e] = m->cell_of[slot][e];
  return FR_OK;
}

fr_status fr_mixed_inters(const fr_mixed* m, int group, int* n_fpts_per_inter, long long* n_inters, int* table)
{
  g_err.clear();
  if (!m || group < 0 || group >= m->n_igroups) return fail(FR_ERR_ARG, "interface group");
  int np = m->igroup_nfpi[group];
  if (n_fpts_per_inter) *n_fpts_per_inter = np;
  if (n_inters) *n_inters = (long long)(m->itab[group].size() / (6 * (size_t)np));
  if (table) std::memcpy(table, m->itab[group].data(), m->itab[group].size() * sizeof(int));
  return FR_OK;
}

fr_status fr_mixed_bdy_inters(const fr_mixed* m, int group, int* n_fpts_per_inter, long long* n_inters, int* table)
{
  g_err.clear();
  if (!m || group < 0 || group >= m->n_bgroups) return fail(FR_ERR_ARG, "boundary group");
  int np = m->bgroup_nfpi[group];
  if (n_fpts_per_inter) *n_fpts_per_inter = np;
  if (n_inters) *n_inters = (long long)(m->btab[group].size() / (4 * (size_t)np));
  if (table) std::memcpy(table, m->btab[group].data(), m->btab[group].size() * sizeof(int));
  return FR_OK;
}

}  // extern "C"
