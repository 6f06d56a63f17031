/* fr_oracle.c -- CPU restatement of the HiFiLES FR residual and RK45 stage
 * (quadrilaterals and hexahedra, Euler / Navier-Stokes, Rusanov + LDG).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Never linked into
 * or called by the product.  Parity is pinned against the reference itself
 * (oracle/_ref built from the reference sources) and against the reference's
 * own regression known-answer values; see tests/golden/.
 *
 * The arithmetic deliberately repeats the reference's operation order:
 * operators are the reference's dense matrices (set_opp_0..6,
 * src/eles.cpp:3620-4052) applied over their exact non-zeros in increasing
 * column order, which is what the reference's column loop in dgemm
 * (src/global.cpp:38-102) does once exact zeros are skipped.  Build with
 * -ffp-contract=off semantics (gcc's default on x86-64) so no FMA is formed.
 */
#include "fr_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXP 11

typedef struct {           /* CSR view of a dense column-major operator */
  int rows, cols;
  double* dense;           /* (rows, cols) column-major */
  int* rp; int* ci; double* v;
} op_t;

struct or_mesh {
  int dims, order, n1, nu, nf, nface, nfpf, nfields;
  int ne, nv;
  double loc1[MAXP + 1];
  double w1[MAXP + 1];
  double eta;
  int vcjh;
  double *loc_upts, *tloc_fpts, *tnorm_fpts;   /* (D, n) */
  op_t opp0, opp1[3], opp2[3], opp3, opp5[3];
  double *xv; int* c2v;                         /* shape nodes */
  double *pos_upts, *pos_fpts;                  /* (n, E, D) */
  double *detjac, *JG, *tdA, *nrm;
  int nint; int *il, *ir;                       /* interface fpts */
  int nb; int* bf; unsigned char* bt;           /* boundary fpts: flat index, boundary type */
  int* bct;                                     /* (E, nface) boundary type per face, 0 = matched */
  /* work arrays */
  double *ufp, *gup, *gfp, *tf, *ntd, *ntc, *ddu, *sgu, *sgf;
};

/* ---------------------------------------------------------------- 1-D basis */

/* eval_lagrange, src/funcs.cpp:57-74 */
static double lag(double r, int mode, const double* pts, int n)
{
  double t = 1.0;
  for (int i = 0; i < n; i++)
    if (i != mode) t = t * ((r - pts[i]) / (pts[mode] - pts[i]));
  return t;
}

/* eval_d_lagrange, src/funcs.cpp:78-108 */
static double dlag(double r, int mode, const double* pts, int n)
{
  double s = 0.0;
  for (int i = 0; i < n; i++) {
    if (i == mode) continue;
    double a = 1.0, b = 1.0;
    for (int j = 0; j < n; j++) {
      if (j != mode && j != i) a = a * (r - pts[j]);
      if (j != mode) b = b * (pts[mode] - pts[j]);
    }
    s = s + (a / b);
  }
  return s;
}

/* eval_legendre, src/funcs.cpp:161-181 */
static double leg(double r, int n)
{
  if (n == 0) return 1.0;
  if (n == 1) return r;
  return ((2 * n - 1) * r * leg(r, n - 1) - (n - 1) * leg(r, n - 2)) / n;
}

/* eval_d_legendre, src/funcs.cpp:185-212 */
static double dleg(double r, int n)
{
  if (n == 0) return 0.0;
  if (r > -1.0 && r < 1.0) return (n * ((r * leg(r, n)) - leg(r, n - 1))) / ((r * r) - 1.0);
  if (r == -1.0) return pow(-1.0, n - 1.0) * 0.5 * n * (n + 1.0);
  return 0.5 * n * (n + 1.0);
}

/* eval_d_vcjh_1d, src/funcs.cpp:216-250 (side 0: left, 1: right) */
static double dvcjh(double r, int side, int P, double eta)
{
  if (side == 0) {
    if (P == 0) return 0.5 * pow(-1.0, P) * (dleg(r, P) - (dleg(r, P + 1) / (1.0 + eta)));
    return 0.5 * pow(-1.0, P) * (dleg(r, P) - (((eta * dleg(r, P - 1)) + dleg(r, P + 1)) / (1.0 + eta)));
  }
  if (P == 0) return 0.5 * (dleg(r, P) + (dleg(r, P + 1) / (1.0 + eta)));
  return 0.5 * (dleg(r, P) + (((eta * dleg(r, P - 1)) + dleg(r, P + 1)) / (1.0 + eta)));
}

static double fact(int n) { double f = 1; for (int i = 2; i <= n; i++) f *= i; return f; }

/* compute_eta, src/funcs.cpp:1503-1546 */
static double vcjh_eta(int scheme, int P, double user_eta)
{
  if (scheme == 0) return user_eta;
  if (scheme == 1) return 0.0;
  if (scheme == 2) return (1.0 * P) / (1.0 * (P + 1));
  if (scheme == 3) return (1.0 * (P + 1)) / (1.0 * P);
  if (scheme == 4) {
    double c;
    if (P == 2) c = 0.206; else if (P == 3) c = 3.80e-3; else if (P == 4) c = 4.67e-5;
    else if (P == 5) c = 4.28e-7; else { fprintf(stderr, "c_+ not defined for P=%d\n", P); return NAN; }
    double ap = 1. / pow(2.0, P) * fact(2 * P) / (fact(P) * fact(P));
    return c * (2 * P + 1) / 2 * (fact(P) * ap) * (fact(P) * ap);
  }
  return NAN;
}

/* The reference's tabulated 1-D solution points (data/loc_1d_gauss_pts.dat and
 * data/loc_1d_gauss_lobatto_pts.dat, 15 decimals, not always correctly rounded).
 * Operator parity at round-off level needs these exact constants. */
static const double GAUSS_TAB[11][11] = {
  {0.0},
  {-0.577350269189626, 0.577350269189626},
  {-0.774596669241483, -0.0, 0.774596669241483},
  {-0.861136311594053, -0.339981043584856, 0.339981043584856, 0.861136311594053},
  {-0.906179845938664, -0.538469310105683, -0.0, 0.538469310105683, 0.906179845938664},
  {-0.932469514203152, -0.661209386466264, -0.238619186083197, 0.238619186083197, 0.661209386466265, 0.932469514203152},
  {-0.949107912342758, -0.741531185599395, -0.405845151377397, 0.0, 0.405845151377397, 0.741531185599394, 0.949107912342758},
  {-0.960289856497536, -0.796666477413627, -0.525532409916329, -0.18343464249565, 0.18343464249565, 0.525532409916329, 0.796666477413627, 0.960289856497536},
  {-0.968160239507626, -0.836031107326636, -0.613371432700591, -0.324253423403809, 0.0, 0.324253423403809, 0.613371432700591, 0.836031107326636, 0.968160239507626},
  {-0.973906528517172, -0.865063366688985, -0.679409568299024, -0.433395394129247, -0.148874338981631, 0.148874338981632, 0.433395394129247, 0.679409568299024, 0.865063366688984, 0.973906528517171},
  {-0.978228658146057, -0.887062599768095, -0.730152005574049, -0.519096129206812, -0.269543155952345, -0.0, 0.269543155952345, 0.519096129206812, 0.730152005574049, 0.887062599768095, 0.978228658146057},
};
static const double LOBATTO_TAB[11][11] = {
  {0}, /* P=0: not tabulated */
  {-1.0, 1.0},
  {-1.0, -0.0, 1.0},
  {-1.0, -0.447213595499958, 0.447213595499958, 1.0},
  {-1.0, -0.654653670707977, -0.0, 0.654653670707977, 1.0},
  {-1.0, -0.765055323929465, -0.285231516480645, 0.285231516480645, 0.765055323929465, 1.0},
  {-1.0, -0.830223896278567, -0.468848793470714, 0.0, 0.468848793470714, 0.830223896278567, 1.0},
  {-1.0, -0.871740148509607, -0.591700181433142, -0.209299217902479, 0.209299217902479, 0.591700181433142, 0.871740148509607, 1.0},
  {-1.0, -0.89975799541146, -0.677186279510738, -0.363117463826178, -0.0, 0.363117463826178, 0.677186279510738, 0.89975799541146, 1.0},
  {-1.0, -0.919533908166459, -0.738773865105505, -0.477924949810445, -0.165278957666387, 0.165278957666387, 0.477924949810444, 0.738773865105505, 0.919533908166459, 1.0},
  {-1.0, -0.934001430408059, -0.784483473663144, -0.565235326996205, -0.295758135586939, 0.0, 0.295758135586939, 0.565235326996205, 0.784483473663144, 0.934001430408059, 1.0},
};

/* Gauss-Legendre (type 0) or Gauss-Lobatto (type 1) points on [-1,1]: the
 * reference's table for P <= 10 (read at src/eles_hexas.cpp:196-218), else
 * Newton iterates rounded to 15 decimals. */
void or_points_1d(int P, int type, double* out)
{
  int n = P + 1;
  if (P <= 10 && (type == 0 || P >= 1)) {
    for (int i = 0; i < n; i++) out[i] = type == 0 ? GAUSS_TAB[P][i] : LOBATTO_TAB[P][i];
    return;
  }
  const double pi = 3.14159265358979323846;
  for (int i = 0; i < n; i++) {
    double x;
    if (n == 1) { x = 0.0; }
    else if (type == 0) {
      x = -cos(pi * (i + 0.75) / (n + 0.5));
      for (int it = 0; it < 100; it++) {
        double p0 = 1.0, p1 = x;
        for (int k = 2; k <= n; k++) { double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
        double dp = n * (x * p1 - p0) / (x * x - 1.0);
        double dx = p1 / dp; x -= dx;
        if (fabs(dx) < 1e-17) break;
      }
    } else {
      if (i == 0) x = -1.0; else if (i == n - 1) x = 1.0;
      else {
        int N = n - 1;  /* interior roots of P'_N */
        x = -cos(pi * i / N);
        for (int it = 0; it < 100; it++) {
          double p0 = 1.0, p1 = x;
          for (int k = 2; k <= N; k++) { double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
          /* q = (1-x^2) P'_N = N (P_{N-1} - x P_N);  q' = -N(N+1) P_N */
          double q = N * (p0 - x * p1), dq = -N * (N + 1.0) * p1;
          double dx = q / dq; x -= dx;
          if (fabs(dx) < 1e-17) break;
        }
      }
    }
    char buf[64];
    snprintf(buf, sizeof buf, "%.15f", x);
    out[i] = strtod(buf, NULL);
  }
}

/* ------------------------------------------------------------ element data */

/* Hex point sets: set_loc_upts / set_tloc_fpts / set_tnorm_fpts,
 * src/eles_hexas.cpp:240-324, 572-628.  Quad: src/eles_quads.cpp:237-300, 443-480. */
static void build_points(or_mesh* m)
{
  int n1 = m->n1, P = m->order, D = m->dims;
  const double* L = m->loc1;
  m->loc_upts = calloc((size_t)D * m->nu, sizeof(double));
  m->tloc_fpts = calloc((size_t)D * m->nf, sizeof(double));
  m->tnorm_fpts = calloc((size_t)D * m->nf, sizeof(double));
  if (D == 2) {
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n1; j++) {
        int u = j + n1 * i;
        m->loc_upts[0 + 2 * u] = L[j]; m->loc_upts[1 + 2 * u] = L[i];
      }
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < n1; j++) {
        int f = j + n1 * i; double* t = m->tloc_fpts + 2 * f; double* nn = m->tnorm_fpts + 2 * f;
        if (i == 0) { t[0] = L[j]; t[1] = -1.0; nn[0] = 0.0; nn[1] = -1.0; }
        else if (i == 1) { t[0] = 1.0; t[1] = L[j]; nn[0] = 1.0; nn[1] = 0.0; }
        else if (i == 2) { t[0] = L[P - j]; t[1] = 1.0; nn[0] = 0.0; nn[1] = 1.0; }
        else { t[0] = -1.0; t[1] = L[P - j]; nn[0] = -1.0; nn[1] = 0.0; }
      }
  } else {
    for (int i = 0; i < n1; i++)
      for (int j = 0; j < n1; j++)
        for (int k = 0; k < n1; k++) {
          int u = k + n1 * j + n1 * n1 * i;
          m->loc_upts[3 * u] = L[k]; m->loc_upts[3 * u + 1] = L[j]; m->loc_upts[3 * u + 2] = L[i];
        }
    for (int i = 0; i < 6; i++)
      for (int j = 0; j < n1; j++)
        for (int k = 0; k < n1; k++) {
          int f = k + n1 * j + n1 * n1 * i; double* t = m->tloc_fpts + 3 * f; double* nn = m->tnorm_fpts + 3 * f;
          nn[0] = nn[1] = nn[2] = 0.0;
          if (i == 0) { t[0] = L[P - k]; t[1] = L[j]; t[2] = -1.0; nn[2] = -1.0; }
          else if (i == 1) { t[0] = L[k]; t[1] = -1.0; t[2] = L[j]; nn[1] = -1.0; }
          else if (i == 2) { t[0] = 1.0; t[1] = L[k]; t[2] = L[j]; nn[0] = 1.0; }
          else if (i == 3) { t[0] = L[P - k]; t[1] = 1.0; t[2] = L[j]; nn[1] = 1.0; }
          else if (i == 4) { t[0] = -1.0; t[1] = L[P - k]; t[2] = L[j]; nn[0] = -1.0; }
          else { t[0] = L[k]; t[1] = L[j]; t[2] = 1.0; nn[2] = 1.0; }
        }
  }
}

/* tensor index of a solution point (eles_hexas::eval_nodal_basis, src/eles_hexas.cpp:917-933) */
static void upt_idx(const or_mesh* m, int u, int* ix)
{
  int n1 = m->n1;
  if (m->dims == 2) { ix[1] = u / n1; ix[0] = u - n1 * ix[1]; ix[2] = 0; }
  else { ix[2] = u / (n1 * n1); ix[1] = (u - n1 * n1 * ix[2]) / n1; ix[0] = u - n1 * ix[1] - n1 * n1 * ix[2]; }
}

static double nodal(const or_mesh* m, int u, const double* loc)
{
  int ix[3]; upt_idx(m, u, ix);
  if (m->dims == 2) return lag(loc[0], ix[0], m->loc1, m->n1) * lag(loc[1], ix[1], m->loc1, m->n1);
  return lag(loc[0], ix[0], m->loc1, m->n1) * lag(loc[1], ix[1], m->loc1, m->n1) * lag(loc[2], ix[2], m->loc1, m->n1);
}

/* eval_d_nodal_basis, src/eles_hexas.cpp:953-981 */
static double dnodal(const or_mesh* m, int u, int c, const double* loc)
{
  int ix[3]; upt_idx(m, u, ix);
  const double* L = m->loc1; int n = m->n1;
  if (m->dims == 2) {
    if (c == 0) return dlag(loc[0], ix[0], L, n) * lag(loc[1], ix[1], L, n);
    return lag(loc[0], ix[0], L, n) * dlag(loc[1], ix[1], L, n);
  }
  if (c == 0) return dlag(loc[0], ix[0], L, n) * lag(loc[1], ix[1], L, n) * lag(loc[2], ix[2], L, n);
  if (c == 1) return lag(loc[0], ix[0], L, n) * dlag(loc[1], ix[1], L, n) * lag(loc[2], ix[2], L, n);
  return lag(loc[0], ix[0], L, n) * lag(loc[1], ix[1], L, n) * dlag(loc[2], ix[2], L, n);
}

/* eval_div_vcjh_basis: hex src/eles_hexas.cpp:1167-1192, quad src/eles_quads.cpp:1107-1130 */
static double div_vcjh(const or_mesh* m, int f, const double* loc)
{
  int P = m->order, n = m->n1; const double* L = m->loc1; double eta = m->eta;
  if (m->dims == 2) {
    int i = f / n, j = f - n * i;
    if (i == 0) return -lag(loc[0], j, L, n) * dvcjh(loc[1], 0, P, eta);
    if (i == 1) return lag(loc[1], j, L, n) * dvcjh(loc[0], 1, P, eta);
    if (i == 2) return lag(loc[0], P - j, L, n) * dvcjh(loc[1], 1, P, eta);
    return -lag(loc[1], P - j, L, n) * dvcjh(loc[0], 0, P, eta);
  }
  int nn = n * n, i = f / nn, j = (f - nn * i) / n, k = f - nn * i - n * j;
  if (i == 0) return -lag(loc[0], P - k, L, n) * lag(loc[1], j, L, n) * dvcjh(loc[2], 0, P, eta);
  if (i == 1) return -lag(loc[0], k, L, n) * lag(loc[2], j, L, n) * dvcjh(loc[1], 0, P, eta);
  if (i == 2) return lag(loc[1], k, L, n) * lag(loc[2], j, L, n) * dvcjh(loc[0], 1, P, eta);
  if (i == 3) return lag(loc[0], P - k, L, n) * lag(loc[2], j, L, n) * dvcjh(loc[1], 1, P, eta);
  if (i == 4) return -lag(loc[1], P - k, L, n) * lag(loc[2], j, L, n) * dvcjh(loc[0], 0, P, eta);
  return lag(loc[0], k, L, n) * lag(loc[1], j, L, n) * dvcjh(loc[2], 1, P, eta);
}

static void op_finish(op_t* o)
{
  int nnz = 0;
  for (int c = 0; c < o->cols; c++)
    for (int r = 0; r < o->rows; r++) if (o->dense[r + (size_t)o->rows * c] != 0.0) nnz++;
  o->rp = calloc(o->rows + 1, sizeof(int)); o->ci = malloc((nnz + 1) * sizeof(int)); o->v = malloc((nnz + 1) * sizeof(double));
  int k = 0;
  for (int r = 0; r < o->rows; r++) {
    o->rp[r] = k;
    for (int c = 0; c < o->cols; c++) {
      double a = o->dense[r + (size_t)o->rows * c];
      if (a != 0.0) { o->ci[k] = c; o->v[k] = a; k++; }
    }
  }
  o->rp[o->rows] = k;
}

static void op_alloc(op_t* o, int rows, int cols) { o->rows = rows; o->cols = cols; o->dense = calloc((size_t)rows * cols, sizeof(double)); }

static void build_operators(or_mesh* m)
{
  int D = m->dims, nu = m->nu, nf = m->nf;
  op_alloc(&m->opp0, nf, nu);            /* set_opp_0, src/eles.cpp:3624-3644 */
  for (int u = 0; u < nu; u++) for (int f = 0; f < nf; f++)
    m->opp0.dense[f + nf * u] = nodal(m, u, m->tloc_fpts + D * f);
  op_finish(&m->opp0);
  for (int d = 0; d < D; d++) {          /* set_opp_1, src/eles.cpp:3680-3705 */
    op_alloc(&m->opp1[d], nf, nu);
    for (int u = 0; u < nu; u++) for (int f = 0; f < nf; f++)
      m->opp1[d].dense[f + nf * u] = nodal(m, u, m->tloc_fpts + D * f) * m->tnorm_fpts[d + D * f];
    op_finish(&m->opp1[d]);
    op_alloc(&m->opp2[d], nu, nu);       /* set_opp_2 / set_opp_4, src/eles.cpp:3749-3770, 3867-3890 */
    for (int u = 0; u < nu; u++) for (int k = 0; k < nu; k++)
      m->opp2[d].dense[k + nu * u] = dnodal(m, u, d, m->loc_upts + D * k);
    op_finish(&m->opp2[d]);
  }
  op_alloc(&m->opp3, nu, nf);            /* set_opp_3 / fill_opp_3, src/eles_hexas.cpp:1148-1163 */
  for (int f = 0; f < nf; f++) for (int u = 0; u < nu; u++)
    m->opp3.dense[u + nu * f] = div_vcjh(m, f, m->loc_upts + D * u);
  op_finish(&m->opp3);
  for (int d = 0; d < D; d++) {          /* set_opp_5, src/eles.cpp:3932-3950 */
    op_alloc(&m->opp5[d], nu, nf);
    for (int f = 0; f < nf; f++) for (int u = 0; u < nu; u++)
      m->opp5[d].dense[u + nu * f] = m->opp3.dense[u + nu * f] * m->tnorm_fpts[d + D * f];
    op_finish(&m->opp5[d]);
  }
}

/* C(:, col) = beta*C + A * B(:, col) for every column (dgemm, src/global.cpp:38-102;
 * beta is 0 or 1 as in every call on the path). */
static void op_apply(const op_t* o, const double* B, double* C, long ncols, int accumulate)
{
  for (long j = 0; j < ncols; j++) {
    const double* b = B + (size_t)o->cols * j;
    double* c = C + (size_t)o->rows * j;
    for (int r = 0; r < o->rows; r++) {
      double s = accumulate ? c[r] : 0.0;
      for (int k = o->rp[r]; k < o->rp[r + 1]; k++) s += b[o->ci[k]] * o->v[k];
      c[r] = s;
    }
  }
}

/* ------------------------------------------------------------------ metrics */

/* 2-node Lagrange shape functions (eles_hexas::eval_nodal_s_basis / eval_d_nodal_s_basis
 * for a perfect-cube node count, src/eles_hexas.cpp:985-1060) */
static void shape_d(const or_mesh* m, const double* loc, double* dN /* (nsp, D) */, double* N)
{
  static const double L2[2] = {-1.0, 1.0};
  int D = m->dims, nsp = 1 << D;
  for (int s = 0; s < nsp; s++) {
    int a = s & 1, b = (s >> 1) & 1, c = (s >> 2) & 1;
    if (D == 2) {
      N[s] = lag(loc[0], a, L2, 2) * lag(loc[1], b, L2, 2);
      dN[s + nsp * 0] = dlag(loc[0], a, L2, 2) * lag(loc[1], b, L2, 2);
      dN[s + nsp * 1] = lag(loc[0], a, L2, 2) * dlag(loc[1], b, L2, 2);
    } else {
      N[s] = lag(loc[0], a, L2, 2) * lag(loc[1], b, L2, 2) * lag(loc[2], c, L2, 2);
      dN[s + nsp * 0] = dlag(loc[0], a, L2, 2) * lag(loc[1], b, L2, 2) * lag(loc[2], c, L2, 2);
      dN[s + nsp * 1] = lag(loc[0], a, L2, 2) * dlag(loc[1], b, L2, 2) * lag(loc[2], c, L2, 2);
      dN[s + nsp * 2] = lag(loc[0], a, L2, 2) * lag(loc[1], b, L2, 2) * dlag(loc[2], c, L2, 2);
    }
  }
}

/* calc_pos / calc_d_pos, src/eles.cpp:5744-5757, 5841-5855 */
static void map_point(const or_mesh* m, int e, const double* loc, double* pos, double* dpos /* (D,D) [i + D*j] = dx_i/dr_j */)
{
  int D = m->dims, nsp = 1 << D;
  double dN[24], N[8];
  shape_d(m, loc, dN, N);
  const int* cv = m->c2v + (size_t)nsp * e;
  for (int i = 0; i < D; i++) {
    double s = 0.0;
    for (int j = 0; j < nsp; j++) s += N[j] * m->xv[(size_t)D * cv[j] + i];
    pos[i] = s;
  }
  for (int j = 0; j < D; j++)
    for (int k = 0; k < D; k++) {
      double s = 0.0;
      for (int i = 0; i < nsp; i++) s += dN[i + nsp * k] * m->xv[(size_t)D * cv[i] + j];
      dpos[j + D * k] = s;
    }
}

/* set_transforms, src/eles.cpp:4557-4847 (static mesh) */
static int build_metrics(or_mesh* m)
{
  int D = m->dims, E = m->ne, nu = m->nu, nf = m->nf;
  m->pos_upts = malloc((size_t)nu * E * D * sizeof(double));
  m->pos_fpts = malloc((size_t)nf * E * D * sizeof(double));
  m->detjac = malloc((size_t)nu * E * sizeof(double));
  m->JG = malloc((size_t)D * D * nu * E * sizeof(double));
  m->tdA = malloc((size_t)nf * E * sizeof(double));
  m->nrm = malloc((size_t)nf * E * D * sizeof(double));
  double pos[3], dp[9];
  for (int e = 0; e < E; e++) {
    for (int u = 0; u < nu; u++) {
      map_point(m, e, m->loc_upts + D * u, pos, dp);
      for (int k = 0; k < D; k++) m->pos_upts[u + (size_t)nu * (e + (size_t)E * k)] = pos[k];
      double* J = m->JG + (size_t)D * D * (u + (size_t)nu * e);
      if (D == 2) {
        double xr = dp[0], xs = dp[2], yr = dp[1], ys = dp[3];
        m->detjac[u + (size_t)nu * e] = xr * ys - xs * yr;
        J[0 + 2 * 0] = ys; J[0 + 2 * 1] = -xs; J[1 + 2 * 0] = -yr; J[1 + 2 * 1] = xr;
      } else {
        double xr = dp[0 + 3 * 0], xs = dp[0 + 3 * 1], xt = dp[0 + 3 * 2];
        double yr = dp[1 + 3 * 0], ys = dp[1 + 3 * 1], yt = dp[1 + 3 * 2];
        double zr = dp[2 + 3 * 0], zs = dp[2 + 3 * 1], zt = dp[2 + 3 * 2];
        m->detjac[u + (size_t)nu * e] = xr * (ys * zt - yt * zs) - xs * (yr * zt - yt * zr) + xt * (yr * zs - ys * zr);
        J[0 + 3 * 0] = ys * zt - yt * zs; J[0 + 3 * 1] = xt * zs - xs * zt; J[0 + 3 * 2] = xs * yt - xt * ys;
        J[1 + 3 * 0] = yt * zr - yr * zt; J[1 + 3 * 1] = xr * zt - xt * zr; J[1 + 3 * 2] = xt * yr - xr * yt;
        J[2 + 3 * 0] = yr * zs - ys * zr; J[2 + 3 * 1] = xs * zr - xr * zs; J[2 + 3 * 2] = xr * ys - xs * yr;
      }
      if (m->detjac[u + (size_t)nu * e] < 0) { fprintf(stderr, "oracle: negative Jacobian\n"); return -1; }
    }
    for (int f = 0; f < nf; f++) {
      map_point(m, e, m->tloc_fpts + D * f, pos, dp);
      for (int k = 0; k < D; k++) m->pos_fpts[f + (size_t)nf * (e + (size_t)E * k)] = pos[k];
      const double* tn = m->tnorm_fpts + D * f;
      double t[3];
#define DP(a, b) dp[(a) + D * (b)]
      if (D == 2) {
        t[0] = (tn[0] * DP(1, 1)) - (tn[1] * DP(1, 0));
        t[1] = -(tn[0] * DP(0, 1)) + (tn[1] * DP(0, 0));
        double a = sqrt(t[0] * t[0] + t[1] * t[1]);
        m->tdA[f + (size_t)nf * e] = a;
        m->nrm[f + (size_t)nf * (e + (size_t)E * 0)] = t[0] / a;
        m->nrm[f + (size_t)nf * (e + (size_t)E * 1)] = t[1] / a;
      } else {
        t[0] = ((tn[0] * (DP(1, 1) * DP(2, 2) - DP(1, 2) * DP(2, 1))) + (tn[1] * (DP(1, 2) * DP(2, 0) - DP(1, 0) * DP(2, 2))) + (tn[2] * (DP(1, 0) * DP(2, 1) - DP(1, 1) * DP(2, 0))));
        t[1] = ((tn[0] * (DP(0, 2) * DP(2, 1) - DP(0, 1) * DP(2, 2))) + (tn[1] * (DP(0, 0) * DP(2, 2) - DP(0, 2) * DP(2, 0))) + (tn[2] * (DP(0, 1) * DP(2, 0) - DP(0, 0) * DP(2, 1))));
        t[2] = ((tn[0] * (DP(0, 1) * DP(1, 2) - DP(0, 2) * DP(1, 1))) + (tn[1] * (DP(0, 2) * DP(1, 0) - DP(0, 0) * DP(1, 2))) + (tn[2] * (DP(0, 0) * DP(1, 1) - DP(0, 1) * DP(1, 0))));
        double a = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
        m->tdA[f + (size_t)nf * e] = a;
        for (int k = 0; k < 3; k++) m->nrm[f + (size_t)nf * (e + (size_t)E * k)] = t[k] / a;
      }
#undef DP
    }
  }
  return 0;
}

/* ----------------------------------------------------- interface matching */

typedef struct { double key[3]; int e, face; } facerec;
static int g_dims;
static int cmp_face(const void* a, const void* b)
{
  const facerec *x = a, *y = b;
  for (int d = 0; d < g_dims; d++) {
    if (x->key[d] < y->key[d]) return -1;
    if (x->key[d] > y->key[d]) return 1;
  }
  return 0;
}

static double wrap(double c, double L, double lo)
{
  if (L <= 0) return c;
  double t = (c - lo) / L;
  t -= floor(t + 1e-9);
  if (t > 1.0 - 1e-9) t -= 1.0;
  return lo + t * L;
}

/* Pairs faces whose centroids coincide modulo the periodic shifts, then pairs
 * the flux points of matched faces by physical position.  This plays the role
 * of CompConnectivity + cyclic matching + get_lut (src/geometry.cpp:2412-2720,
 * 3489-3666; src/inters.cpp:187-296) for conforming meshes: the lower element
 * index becomes the left side. */
static int build_interfaces(or_mesh* m, const double* shift)
{
  int D = m->dims, E = m->ne, nface = m->nface, nfpf = m->nfpf, nf = m->nf;
  double lo[3] = {1e300, 1e300, 1e300}, h = 1e300;
  for (int v = 0; v < m->nv; v++) for (int d = 0; d < D; d++) if (m->xv[D * v + d] < lo[d]) lo[d] = m->xv[D * v + d];
  for (int e = 0; e < E; e++) {
    double d0 = 0; for (int d = 0; d < D; d++) { double t = m->xv[D * m->c2v[(1 << D) * e + 1] + d] - m->xv[D * m->c2v[(1 << D) * e] + d]; d0 += t * t; }
    if (sqrt(d0) < h) h = sqrt(d0);
  }
  double tol = 1e-6 * h;
  facerec* fr = malloc((size_t)E * nface * sizeof(facerec));
  int nrec = 0, nbf = 0;
  for (int e = 0; e < E; e++)
    for (int fc = 0; fc < nface; fc++)
      if (m->bct && m->bct[(size_t)e * nface + fc] > 0) nbf++;
  m->nb = nbf * nfpf;
  m->bf = malloc(sizeof(int) * (m->nb + 1)); m->bt = malloc(m->nb + 1);
  nbf = 0;
  for (int e = 0; e < E; e++)
    for (int fc = 0; fc < nface; fc++) {
      if (m->bct && m->bct[(size_t)e * nface + fc] > 0) {   /* boundary face: its points in face order */
        for (int q = 0; q < nfpf; q++) {
          m->bf[nbf] = fc * nfpf + q + nf * e;
          m->bt[nbf++] = (unsigned char)m->bct[(size_t)e * nface + fc];
        }
        continue;
      }
      facerec* r = fr + nrec++;
      r->e = e; r->face = fc;
      for (int d = 0; d < D; d++) {
        double s = 0;
        for (int q = 0; q < nfpf; q++) s += m->pos_fpts[(fc * nfpf + q) + (size_t)nf * (e + (size_t)E * d)];
        double c = wrap(s / nfpf, shift[d], lo[d]);
        r->key[d] = floor(c / tol + 0.5) * tol;
      }
    }
  g_dims = D;
  qsort(fr, (size_t)nrec, sizeof(facerec), cmp_face);
  int nint = nrec / 2;
  m->nint = nint * nfpf;
  m->il = malloc(sizeof(int) * (m->nint + 1)); m->ir = malloc(sizeof(int) * (m->nint + 1));
  int k = 0;
  for (int i = 0; i < nrec; i += 2) {
    if (i + 1 >= nrec || cmp_face(fr + i, fr + i + 1) != 0) { fprintf(stderr, "oracle: unmatched face\n"); free(fr); return -1; }
    facerec *a = fr + i, *b = fr + i + 1;
    if (b->e < a->e || (b->e == a->e && b->face < a->face)) { facerec* t = a; a = b; b = t; }
    for (int q = 0; q < nfpf; q++) {
      int fa = a->face * nfpf + q, best = -1; double bd = 1e300;
      for (int r = 0; r < nfpf; r++) {
        int fb = b->face * nfpf + r; double dd = 0;
        for (int d = 0; d < D; d++) {
          double x = wrap(m->pos_fpts[fa + (size_t)nf * (a->e + (size_t)E * d)], shift[d], lo[d]);
          double y = wrap(m->pos_fpts[fb + (size_t)nf * (b->e + (size_t)E * d)], shift[d], lo[d]);
          double t = x - y;
          if (shift[d] > 0) { if (t > 0.5 * shift[d]) t -= shift[d]; if (t < -0.5 * shift[d]) t += shift[d]; }
          dd += t * t;
        }
        if (dd < bd) { bd = dd; best = fb; }
      }
      m->il[k] = fa + nf * a->e; m->ir[k] = best + nf * b->e; k++;
    }
  }
  free(fr);
  return 0;
}

/* ----------------------------------------------------------------- set-up */

static or_mesh* mesh_core(int dims, int order, int upts_type, int vcjh_scheme, double eta)
{
  if ((dims != 2 && dims != 3) || order < 0 || order > MAXP - 1) return NULL;
  or_mesh* m = calloc(1, sizeof(or_mesh));
  m->dims = dims; m->order = order; m->n1 = order + 1;
  m->nu = dims == 2 ? m->n1 * m->n1 : m->n1 * m->n1 * m->n1;
  m->nface = 2 * dims; m->nfpf = dims == 2 ? m->n1 : m->n1 * m->n1;
  m->nf = m->nface * m->nfpf; m->nfields = dims + 2;
  or_points_1d(order, upts_type, m->loc1);
  m->vcjh = vcjh_scheme;
  m->eta = vcjh_eta(vcjh_scheme, order, eta);
  /* Gauss quadrature weights of the solution points (for the kinetic energy only). */
  for (int i = 0; i < m->n1; i++) {
    double x = m->loc1[i], p0 = 1.0, p1 = x;
    for (int k = 2; k <= m->n1; k++) { double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k; p0 = p1; p1 = p2; }
    double dp = m->n1 * (x * p1 - p0) / (x * x - 1.0);
    m->w1[i] = m->n1 == 1 ? 2.0 : 2.0 / ((1.0 - x * x) * dp * dp);
  }
  build_points(m);
  build_operators(m);
  return m;
}

static void alloc_work(or_mesh* m)
{
  size_t E = m->ne, F = m->nfields, D = m->dims;
  m->ufp = calloc(m->nf * E * F, sizeof(double));
  m->gup = calloc(m->nu * E * F * D, sizeof(double));
  m->gfp = calloc(m->nf * E * F * D, sizeof(double));
  m->tf = calloc(m->nu * E * F * D, sizeof(double));
  m->ntd = calloc(m->nf * E * F, sizeof(double));
  m->ntc = calloc(m->nf * E * F, sizeof(double));
  m->ddu = calloc(m->nf * E * F, sizeof(double));
  m->sgu = calloc(m->nu * E * F * D, sizeof(double));
  m->sgf = calloc(m->nf * E * F * D, sizeof(double));
}

or_mesh* or_mesh_new(int dims, int order, int n_verts, const double* xv, int n_eles, const int* c2v,
                     const double* shift, int upts_type, int vcjh_scheme, double eta)
{
  return or_mesh_new_bc(dims, order, n_verts, xv, n_eles, c2v, shift, NULL, upts_type, vcjh_scheme, eta);
}

or_mesh* or_mesh_new_bc(int dims, int order, int n_verts, const double* xv, int n_eles, const int* c2v,
                        const double* shift, const int* bctype, int upts_type, int vcjh_scheme, double eta)
{
  or_mesh* m = mesh_core(dims, order, upts_type, vcjh_scheme, eta);
  if (!m) return NULL;
  int nsp = 1 << dims;
  m->nv = n_verts; m->ne = n_eles;
  m->xv = malloc(sizeof(double) * dims * n_verts); memcpy(m->xv, xv, sizeof(double) * dims * n_verts);
  m->c2v = malloc(sizeof(int) * nsp * n_eles); memcpy(m->c2v, c2v, sizeof(int) * nsp * n_eles);
  if (bctype) {
    m->bct = malloc(sizeof(int) * 2 * dims * n_eles);
    memcpy(m->bct, bctype, sizeof(int) * 2 * dims * n_eles);
  }
  if (build_metrics(m) || build_interfaces(m, shift)) { or_mesh_free(m); return NULL; }
  alloc_work(m);
  return m;
}

or_mesh* or_box_new(int dims, int order, const int* n, const double* lo, const double* hi,
                    double jitter, unsigned long long seed, int upts_type, int vcjh_scheme, double eta)
{
  return or_box_new_bc(dims, order, n, lo, hi, jitter, seed, NULL, upts_type, vcjh_scheme, eta);
}

or_mesh* or_box_new_bc(int dims, int order, const int* n, const double* lo, const double* hi, double jitter,
                       unsigned long long seed, const int* side_bc, int upts_type, int vcjh_scheme, double eta)
{
  int nx = n[0], ny = n[1], nz = dims == 3 ? n[2] : 1;
  int vx = nx + 1, vy = ny + 1, vz = dims == 3 ? nz + 1 : 1;
  int nv = vx * vy * vz, ne = nx * ny * nz, nsp = 1 << dims;
  double* xv = malloc(sizeof(double) * dims * nv);
  int* c2v = malloc(sizeof(int) * nsp * ne);
  unsigned long long s = seed * 6364136223846793005ULL + 1442695040888963407ULL;
  for (int k = 0; k < vz; k++)
    for (int j = 0; j < vy; j++)
      for (int i = 0; i < vx; i++) {
        int v = i + vx * (j + vy * k);
        int ijk[3] = {i, j, k}, nn[3] = {nx, ny, nz};
        int interior = 1;
        for (int d = 0; d < dims; d++) if (ijk[d] == 0 || ijk[d] == nn[d]) interior = 0;
        for (int d = 0; d < dims; d++) {
          double h = (hi[d] - lo[d]) / nn[d];
          double x = lo[d] + (hi[d] - lo[d]) * ijk[d] / nn[d];
          s = s * 6364136223846793005ULL + 1442695040888963407ULL;
          double r = ((s >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
          if (interior && jitter > 0) x += jitter * h * r;
          xv[dims * v + d] = x;
        }
      }
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++) {
        int e = i + nx * (j + ny * k);
        for (int c = 0; c < (dims == 3 ? 2 : 1); c++)
          for (int b = 0; b < 2; b++)
            for (int a = 0; a < 2; a++)
              c2v[nsp * e + a + 2 * b + 4 * c] = (i + a) + vx * ((j + b) + vy * (k + c));
      }
  double shift[3] = {0, 0, 0};
  for (int d = 0; d < dims; d++) shift[d] = hi[d] - lo[d];
  int* bct = NULL;
  if (side_bc) {
    /* local face of each box side: quads y- 0, x+ 1, y+ 2, x- 3; hexes z- 0,
     * y- 1, x+ 2, y+ 3, x- 4, z+ 5 (the reference's face numbering) */
    static const int q_face[4] = {3, 1, 0, 2}, h_face[6] = {4, 2, 1, 3, 0, 5};
    int nface = 2 * dims;
    bct = calloc((size_t)ne * nface, sizeof(int));
    for (int d = 0; d < dims; d++)
      if (side_bc[2 * d] > 0 || side_bc[2 * d + 1] > 0) shift[d] = 0.0;
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
          int e = i + nx * (j + ny * k), ijk[3] = {i, j, k}, nn[3] = {nx, ny, nz};
          for (int d = 0; d < dims; d++)
            for (int sd = 0; sd < 2; sd++) {
              int bc = side_bc[2 * d + sd];
              if (bc <= 0) continue;
              if ((sd == 0 && ijk[d] == 0) || (sd == 1 && ijk[d] == nn[d] - 1)) {
                int fc = dims == 2 ? q_face[2 * d + sd] : h_face[2 * d + sd];
                bct[(size_t)e * nface + fc] = bc;
              }
            }
        }
  }
  or_mesh* m = or_mesh_new_bc(dims, order, nv, xv, ne, c2v, shift, bct, upts_type, vcjh_scheme, eta);
  free(xv); free(c2v); free(bct);
  return m;
}

static void op_free(op_t* o) { free(o->dense); free(o->rp); free(o->ci); free(o->v); }

void or_mesh_free(or_mesh* m)
{
  if (!m) return;
  op_free(&m->opp0); op_free(&m->opp3);
  for (int d = 0; d < 3; d++) { op_free(&m->opp1[d]); op_free(&m->opp2[d]); op_free(&m->opp5[d]); }
  free(m->loc_upts); free(m->tloc_fpts); free(m->tnorm_fpts); free(m->xv); free(m->c2v);
  free(m->pos_upts); free(m->pos_fpts); free(m->detjac); free(m->JG); free(m->tdA); free(m->nrm);
  free(m->il); free(m->ir); free(m->bf); free(m->bt); free(m->bct);
  free(m->ufp); free(m->gup); free(m->gfp); free(m->tf); free(m->ntd); free(m->ntc); free(m->ddu);
  free(m->sgu); free(m->sgf);
  free(m);
}

int or_n_boundary(const or_mesh* m) { return m->nb; }

void or_get_boundary(const or_mesh* m, int* fpt_idx, int* type)
{
  for (int i = 0; i < m->nb; i++) { fpt_idx[i] = m->bf[i]; type[i] = m->bt[i]; }
}

void or_sizes(const or_mesh* m, int* o)
{
  o[0] = m->ne; o[1] = m->nu; o[2] = m->nf; o[3] = m->nfields; o[4] = m->dims; o[5] = m->nint;
}

void or_get_geometry(const or_mesh* m, double* pos_upts, double* detjac, double* JG, double* tdA, double* nrm, double* pos_fpts)
{
  size_t E = m->ne, D = m->dims;
  if (pos_upts) memcpy(pos_upts, m->pos_upts, sizeof(double) * m->nu * E * D);
  if (detjac) memcpy(detjac, m->detjac, sizeof(double) * m->nu * E);
  if (JG) memcpy(JG, m->JG, sizeof(double) * D * D * m->nu * E);
  if (tdA) memcpy(tdA, m->tdA, sizeof(double) * m->nf * E);
  if (nrm) memcpy(nrm, m->nrm, sizeof(double) * m->nf * E * D);
  if (pos_fpts) memcpy(pos_fpts, m->pos_fpts, sizeof(double) * m->nf * E * D);
}

void or_get_interfaces(const or_mesh* m, int* l, int* r)
{
  memcpy(l, m->il, sizeof(int) * m->nint);
  memcpy(r, m->ir, sizeof(int) * m->nint);
}

void or_set_geometry(or_mesh* m, const double* detjac, const double* JG, const double* tdA, const double* nrm)
{
  size_t E = m->ne, D = m->dims;
  memcpy(m->detjac, detjac, sizeof(double) * m->nu * E);
  memcpy(m->JG, JG, sizeof(double) * D * D * m->nu * E);
  memcpy(m->tdA, tdA, sizeof(double) * m->nf * E);
  memcpy(m->nrm, nrm, sizeof(double) * m->nf * E * D);
}

void or_set_interfaces(or_mesh* m, int n, const int* l, const int* r)
{
  free(m->il); free(m->ir); free(m->bf); free(m->bt); free(m->bct);
  m->nint = n;
  m->il = malloc(sizeof(int) * n); m->ir = malloc(sizeof(int) * n);
  memcpy(m->il, l, sizeof(int) * n); memcpy(m->ir, r, sizeof(int) * n);
}

int or_get_operator(const or_mesh* m, int which, int dim, double* out, int* shape)
{
  const op_t* o;
  switch (which) {
    case 0: case 6: o = &m->opp0; break;
    case 1: o = &m->opp1[dim]; break;
    case 2: case 4: o = &m->opp2[dim]; break;
    case 3: o = &m->opp3; break;
    case 5: o = &m->opp5[dim]; break;
    default: return -1;
  }
  shape[0] = o->rows; shape[1] = o->cols;
  if (out) memcpy(out, o->dense, sizeof(double) * o->rows * o->cols);
  return 0;
}

/* ---------------------------------------------------------------- physics */

/* calc_invf_2d / calc_invf_3d, src/flux.cpp:36-128 (Euler/NS, no SA) */
static void invf(int D, double g, const double* u, double* f /* (F, D) [k + F*l] */)
{
  if (D == 2) {
    double vx = u[1] / u[0], vy = u[2] / u[0];
    double p = (g - 1.0) * (u[3] - (0.5 * u[0] * ((vx * vx) + (vy * vy))));
    f[0 + 4 * 0] = u[1]; f[1 + 4 * 0] = p + (u[1] * vx); f[2 + 4 * 0] = u[2] * vx; f[3 + 4 * 0] = vx * (u[3] + p);
    f[0 + 4 * 1] = u[2]; f[1 + 4 * 1] = u[1] * vy; f[2 + 4 * 1] = p + (u[2] * vy); f[3 + 4 * 1] = vy * (u[3] + p);
  } else {
    double vx = u[1] / u[0], vy = u[2] / u[0], vz = u[3] / u[0];
    double p = (g - 1.0) * (u[4] - (0.5 * u[0] * ((vx * vx) + (vy * vy) + (vz * vz))));
    f[0 + 5 * 0] = u[1]; f[1 + 5 * 0] = p + (u[1] * vx); f[2 + 5 * 0] = u[2] * vx; f[3 + 5 * 0] = u[3] * vx; f[4 + 5 * 0] = vx * (u[4] + p);
    f[0 + 5 * 1] = u[2]; f[1 + 5 * 1] = u[1] * vy; f[2 + 5 * 1] = p + (u[2] * vy); f[3 + 5 * 1] = u[3] * vy; f[4 + 5 * 1] = vy * (u[4] + p);
    f[0 + 5 * 2] = u[3]; f[1 + 5 * 2] = u[1] * vz; f[2 + 5 * 2] = u[2] * vz; f[3 + 5 * 2] = p + (u[3] * vz); f[4 + 5 * 2] = vz * (u[4] + p);
  }
}

/* calc_visf_2d / calc_visf_3d, src/flux.cpp:132-431 (no SA: mu_t = 0) */
static void visf(int D, const or_physics* ph, const double* u, const double* gu /* (F,D) [k+F*l] */, double* f)
{
  double g = ph->gamma;
  if (D == 2) {
    double rho = u[0], mx = u[1], my = u[2], ene = u[3];
    double rx = gu[0], mxx = gu[1], myx = gu[2], ex = gu[3];
    double ry = gu[4], mxy = gu[5], myy = gu[6], ey = gu[7];
    double uu = mx / rho, vv = my / rho;
    double inte = ene / rho - 0.5 * (uu * uu + vv * vv);
    double rt = (g - 1.0) * inte / (ph->rt_inf);
    double mu = (ph->mu_inf) * pow(rt, 1.5) * (1. + (ph->c_sth)) / (rt + (ph->c_sth));
    mu = mu + ph->fix_vis * (ph->mu_inf - mu);
    double mut = 0.0;
    double dux = (mxx - rx * uu) / rho, duy = (mxy - ry * uu) / rho;
    double dvx = (myx - rx * vv) / rho, dvy = (myy - ry * vv) / rho;
    double dkex = 0.5 * (uu * uu + vv * vv) * rx + rho * (uu * dux + vv * dvx);
    double dkey = 0.5 * (uu * uu + vv * vv) * ry + rho * (uu * duy + vv * dvy);
    double dex = (ex - dkex - rx * inte) / rho, dey = (ey - dkey - ry * inte) / rho;
    double diag = (dux + dvy) / 3.0;
    double txx = 2.0 * (mu + mut) * (dux - diag), txy = (mu + mut) * (duy + dvx), tyy = 2.0 * (mu + mut) * (dvy - diag);
    double kt = (mu / ph->prandtl + 0.0) * g;   /* mu_t/prandtl_t = 0 without a turbulence model */
    f[0] = 0.0; f[1] = -txx; f[2] = -txy; f[3] = -(uu * txx + vv * txy + kt * dex);
    f[4] = 0.0; f[5] = -txy; f[6] = -tyy; f[7] = -(uu * txy + vv * tyy + kt * dey);
  } else {
    double rho = u[0], mx = u[1], my = u[2], mz = u[3], ene = u[4];
    double rx = gu[0 + 5 * 0], mxx = gu[1 + 5 * 0], myx = gu[2 + 5 * 0], mzx = gu[3 + 5 * 0], ex = gu[4 + 5 * 0];
    double ry = gu[0 + 5 * 1], mxy = gu[1 + 5 * 1], myy = gu[2 + 5 * 1], mzy = gu[3 + 5 * 1], ey = gu[4 + 5 * 1];
    double rz = gu[0 + 5 * 2], mxz = gu[1 + 5 * 2], myz = gu[2 + 5 * 2], mzz = gu[3 + 5 * 2], ez = gu[4 + 5 * 2];
    double uu = mx / rho, vv = my / rho, ww = mz / rho;
    double inte = ene / rho - 0.5 * (uu * uu + vv * vv + ww * ww);
    double rt = (g - 1.0) * inte / (ph->rt_inf);
    double mu = (ph->mu_inf) * pow(rt, 1.5) * (1 + (ph->c_sth)) / (rt + (ph->c_sth));
    mu = mu + ph->fix_vis * (ph->mu_inf - mu);
    double mut = 0.0;
    double dux = (mxx - rx * uu) / rho, duy = (mxy - ry * uu) / rho, duz = (mxz - rz * uu) / rho;
    double dvx = (myx - rx * vv) / rho, dvy = (myy - ry * vv) / rho, dvz = (myz - rz * vv) / rho;
    double dwx = (mzx - rx * ww) / rho, dwy = (mzy - ry * ww) / rho, dwz = (mzz - rz * ww) / rho;
    double ke2 = 0.5 * (uu * uu + vv * vv + ww * ww);
    double dkex = ke2 * rx + rho * (uu * dux + vv * dvx + ww * dwx);
    double dkey = ke2 * ry + rho * (uu * duy + vv * dvy + ww * dwy);
    double dkez = ke2 * rz + rho * (uu * duz + vv * dvz + ww * dwz);
    double dex = (ex - dkex - rx * inte) / rho, dey = (ey - dkey - ry * inte) / rho, dez = (ez - dkez - rz * inte) / rho;
    double diag = (dux + dvy + dwz) / 3.0;
    double txx = 2.0 * (mu + mut) * (dux - diag), tyy = 2.0 * (mu + mut) * (dvy - diag), tzz = 2.0 * (mu + mut) * (dwz - diag);
    double txy = (mu + mut) * (duy + dvx), txz = (mu + mut) * (duz + dwx), tyz = (mu + mut) * (dvz + dwy);
    double kt = (mu / ph->prandtl + 0.0) * g;
    f[0 + 5 * 0] = 0.0; f[1 + 5 * 0] = -txx; f[2 + 5 * 0] = -txy; f[3 + 5 * 0] = -txz; f[4 + 5 * 0] = -(uu * txx + vv * txy + ww * txz + kt * dex);
    f[0 + 5 * 1] = 0.0; f[1 + 5 * 1] = -txy; f[2 + 5 * 1] = -tyy; f[3 + 5 * 1] = -tyz; f[4 + 5 * 1] = -(uu * txy + vv * tyy + ww * tyz + kt * dey);
    f[0 + 5 * 2] = 0.0; f[1 + 5 * 2] = -txz; f[2 + 5 * 2] = -tyz; f[3 + 5 * 2] = -tzz; f[4 + 5 * 2] = -(uu * txz + vv * tyz + ww * tzz + kt * dez);
  }
}

/* inters::rusanov_flux, src/inters.cpp:311-365 (static mesh: v_g = 0) */
static void rusanov(int D, int F, double g, const double* ul, const double* ur, const double* n, double* fn)
{
  double fl[15], fr[15], fnl[5], fnr[5];
  invf(D, g, ul, fl); invf(D, g, ur, fr);
  for (int k = 0; k < F; k++) {
    fnl[k] = 0.; fnr[k] = 0.;
    for (int l = 0; l < D; l++) { fnl[k] += fl[k + F * l] * n[l]; fnr[k] += fr[k + F * l] * n[l]; }
  }
  double vxl = ul[1] / ul[0], vxr = ur[1] / ur[0], vyl = ul[2] / ul[0], vyr = ur[2] / ur[0];
  double vnl, vnr, vng, pl, pr;
  if (D == 2) {
    vnl = vxl * n[0] + vyl * n[1]; vnr = vxr * n[0] + vyr * n[1]; vng = 0.0 * n[0] + 0.0 * n[1];
    pl = (g - 1.0) * (ul[3] - (0.5 * ul[0] * ((vxl * vxl) + (vyl * vyl))));
    pr = (g - 1.0) * (ur[3] - (0.5 * ur[0] * ((vxr * vxr) + (vyr * vyr))));
  } else {
    double vzl = ul[3] / ul[0], vzr = ur[3] / ur[0];
    vnl = vxl * n[0] + vyl * n[1] + vzl * n[2]; vnr = vxr * n[0] + vyr * n[1] + vzr * n[2];
    vng = 0.0 * n[0] + 0.0 * n[1] + 0.0 * n[2];
    pl = (g - 1.0) * (ul[4] - (0.5 * ul[0] * ((vxl * vxl) + (vyl * vyl) + (vzl * vzl))));
    pr = (g - 1.0) * (ur[4] - (0.5 * ur[0] * ((vxr * vxr) + (vyr * vyr) + (vzr * vzr))));
  }
  double vav = sqrt(0.25 * (vnl + vnr) * (vnl + vnr));
  double cav = sqrt((g * (pl + pr)) / (ul[0] + ur[0]));
  double eig = fabs(vav - vng + cav);
  for (int k = 0; k < F; k++) fn[k] = 0.5 * ((fnl[k] + fnr[k]) - eig * (ur[k] - ul[k]));
}

/* inters::roe_flux, src/inters.cpp:390-508, in 2-D (the reference stops with
 * "Roe not implemented in 3D"); static mesh, v_g = 0 */
static void roe(double g, const double* ul, const double* ur, const double* n, double* fn)
{
  double vl[2] = {ul[1] / ul[0], ul[2] / ul[0]}, vr[2] = {ur[1] / ur[0], ur[2] / ur[0]};
  double pl = (g - 1.0) * (ul[3] - (0.5 * ul[0] * ((vl[0] * vl[0]) + (vl[1] * vl[1]))));
  double pr = (g - 1.0) * (ur[3] - (0.5 * ur[0] * ((vr[0] * vr[0]) + (vr[1] * vr[1]))));
  double hl = (ul[3] + pl) / ul[0], hr = (ur[3] + pr) / ur[0];
  double sq = sqrt(ur[0] / ul[0]);
  double rr = 1. / (sq + 1.);
  double um[2], usq = 0., unm = 0., vgn = 0., rl = 0., rrn = 0., du[4];
  for (int i = 0; i < 2; i++) um[i] = rr * (vl[i] + sq * vr[i]);
  double hm = rr * (hl + sq * hr);
  for (int i = 0; i < 2; i++) usq += 0.5 * um[i] * um[i];
  double am2 = (g - 1.) * (hm - usq);
  double am = sqrt(am2);
  for (int i = 0; i < 2; i++) { unm += um[i] * n[i]; vgn += 0.0 * n[i]; }
  for (int i = 0; i < 2; i++) { rl += ul[i + 1] * n[i]; rrn += ur[i + 1] * n[i]; }
  fn[0] = rl + rrn;
  fn[1] = rl * vl[0] + rrn * vr[0] + (pl + pr) * n[0];
  fn[2] = rl * vl[1] + rrn * vr[1] + (pl + pr) * n[1];
  fn[3] = rl * hl + rrn * hr;
  for (int i = 0; i < 4; i++) du[i] = ur[i] - ul[i];
  double l0 = fabs(unm - vgn), lP = fabs(unm - vgn + am), lM = fabs(unm - vgn - am);
  double eps = 0.5 * (fabs(rl / ul[0] - rrn / ur[0]) + fabs(sqrt(g * pl / ul[0]) - sqrt(g * pr / ur[0])));
  if (l0 < 2. * eps) l0 = 0.25 * l0 * l0 / eps + eps;
  if (lP < 2. * eps) lP = 0.25 * lP * lP / eps + eps;
  if (lM < 2. * eps) lM = 0.25 * lM * lM / eps + eps;
  double a2 = 0.5 * (lP + lM) - l0;
  double a3 = 0.5 * (lP - lM) / am;
  double a1 = a2 * (g - 1.) / am2;
  double a4 = a3 * (g - 1.);
  double a5 = usq * du[0] - um[0] * du[1] - um[1] * du[2] + du[3];
  double a6 = unm * du[0] - n[0] * du[1] - n[1] * du[2];
  double aL1 = a1 * a5 - a3 * a6, bL1 = a4 * a5 - a2 * a6;
  fn[0] = fn[0] - (l0 * du[0] + aL1);
  fn[1] = fn[1] - (l0 * du[1] + aL1 * um[0] + bL1 * n[0]);
  fn[2] = fn[2] - (l0 * du[2] + aL1 * um[1] + bL1 * n[1]);
  fn[3] = fn[3] - (l0 * du[3] + aL1 * hm + bL1 * unm);
  for (int i = 0; i < 4; i++) fn[i] = 0.5 * fn[i] - 0.5 * vgn * (ur[i] + ul[i]);
}

/* Ghost state of a boundary flux point: bdy_inters::set_inv_boundary_conditions
 * for the Navier-Stokes/Euler types, src/bdy_inters.cpp:391-860, static mesh
 * (grid velocity v_g = 0), no turbulence model. */
static void bc_ghost(int D, int type, const double* ul, const double* n, const or_physics* ph, double* ur)
{
  const double g = ph->gamma, R_ref = ph->R_ref;
  const double* P = ph->bdy;
  const double rho_bound = P[0], *v_bound = P + 1, p_bound = P[4], *v_wall = P + 5, T_wall = P[8];
  const double vg[3] = {0.0, 0.0, 0.0};
  double rho_l = ul[0], v_l[3], e_l = ul[D + 1], v_sq = 0., p_l, rho_r = 0, v_r[3] = {0, 0, 0}, e_r = 0, p_r, T_r, vn_l;
  for (int i = 0; i < D; i++) v_l[i] = ul[i + 1] / ul[0];
  for (int i = 0; i < D; i++) v_sq += (v_l[i] * v_l[i]);
  p_l = (g - 1.0) * (e_l - 0.5 * rho_l * v_sq);
  if (type == 1) {                           /* sub_in_simp */
    rho_r = rho_bound;
    for (int i = 0; i < D; i++) v_r[i] = v_bound[i];
    p_r = p_l;
    v_sq = 0.; for (int i = 0; i < D; i++) v_sq += (v_r[i] * v_r[i]);
    e_r = (p_r / (g - 1.0)) + 0.5 * rho_r * v_sq;
  } else if (type == 2) {                    /* sub_out_simp */
    rho_r = rho_l;
    for (int i = 0; i < D; i++) v_r[i] = v_l[i];
    p_r = p_bound;
    v_sq = 0.; for (int i = 0; i < D; i++) v_sq += (v_r[i] * v_r[i]);
    e_r = (p_r / (g - 1.0)) + 0.5 * rho_r * v_sq;
  } else if (type == 3) {                    /* sub_in_char */
    double p_total_bound = P[9], T_total_bound = P[10];
    const double* nfs = P + 11;
    vn_l = 0.; for (int i = 0; i < D; i++) vn_l += v_l[i] * n[i];
    double c_l = sqrt(g * p_l / rho_l);
    double R_plus = vn_l + 2.0 * c_l / (g - 1.0);
    double h_total = g * R_ref / (g - 1.0) * T_total_bound;
    v_sq = 0.; for (int i = 0; i < D; i++) v_sq += v_l[i] * v_l[i];
    double c_total_sq = (g - 1.0) * (h_total - (e_l / rho_l + p_l / rho_l) + 0.5 * v_sq) + c_l * c_l;
    double alpha = 0.; for (int i = 0; i < D; i++) alpha += n[i] * nfs[i];
    double aa = 1.0 + 0.5 * (g - 1.0) * alpha * alpha;
    double bb = -(g - 1.0) * alpha * R_plus;
    double cc = 0.5 * (g - 1.0) * R_plus * R_plus - 2.0 * c_total_sq / (g - 1.0);
    double dd = bb * bb - 4.0 * aa * cc;
    dd = sqrt(fmax(dd, 0.0));
    double V_r = (-bb + dd) / (2.0 * aa);
    V_r = fmax(V_r, 0.0);
    v_sq = V_r * V_r;
    double c_r_sq = c_total_sq - 0.5 * (g - 1.0) * v_sq;
    double Mach_sq = v_sq / (c_r_sq);
    Mach_sq = fmin(Mach_sq, 1.0);
    v_sq = Mach_sq * c_r_sq;
    V_r = sqrt(v_sq);
    c_r_sq = c_total_sq - 0.5 * (g - 1.0) * v_sq;
    for (int i = 0; i < D; i++) v_r[i] = V_r * nfs[i];
    T_r = c_r_sq / (g * R_ref);
    p_r = p_total_bound * pow(T_r / T_total_bound, g / (g - 1.0));
    rho_r = p_r / (R_ref * T_r);
    e_r = (p_r / (g - 1.0)) + 0.5 * rho_r * v_sq;
  } else if (type == 4) {                    /* sub_out_char */
    vn_l = 0.; for (int i = 0; i < D; i++) vn_l += v_l[i] * n[i];
    double c_l = sqrt(g * p_l / rho_l);
    double R_plus = vn_l + 2.0 * c_l / (g - 1.0);
    double s = p_l / pow(rho_l, g);
    p_r = p_bound;
    rho_r = pow(p_r / s, 1.0 / g);
    double c_r = sqrt(g * p_r / rho_r);
    double vn_r = R_plus - 2.0 * c_r / (g - 1.0);
    v_sq = 0.;
    for (int i = 0; i < D; i++) { v_r[i] = v_l[i] + (vn_r - vn_l) * n[i]; v_sq += (v_r[i] * v_r[i]); }
    e_r = (p_r / (g - 1.0)) + 0.5 * rho_r * v_sq;
  } else if (type == 5) {                    /* sup_in */
    rho_r = rho_bound;
    for (int i = 0; i < D; i++) v_r[i] = v_bound[i];
    p_r = p_bound;
    v_sq = 0.; for (int i = 0; i < D; i++) v_sq += (v_r[i] * v_r[i]);
    e_r = (p_r / (g - 1.0)) + 0.5 * rho_r * v_sq;
  } else if (type == 6) {                    /* sup_out */
    rho_r = rho_l;
    for (int i = 0; i < D; i++) v_r[i] = v_l[i];
    e_r = e_l;
  } else if (type == 7) {                    /* slip_wall */
    rho_r = rho_l;
    vn_l = 0.; for (int i = 0; i < D; i++) vn_l += (v_l[i] - vg[i]) * n[i];
    for (int i = 0; i < D; i++) v_r[i] = v_l[i] - 2.0 * vn_l * n[i];
    e_r = e_l;
  } else if (type == 11 || type == 13) {     /* isotherm_fix, isotherm_move */
    p_r = p_l;
    T_r = T_wall;
    rho_r = p_r / (R_ref * T_r);
    for (int i = 0; i < D; i++) v_r[i] = type == 11 ? vg[i] : v_wall[i] + vg[i];
    v_sq = 0.; for (int i = 0; i < D; i++) v_sq += (v_r[i] * v_r[i]);
    e_r = (p_r / (g - 1.0)) + 0.5 * rho_r * v_sq;
  } else if (type == 12 || type == 14) {     /* adiabat_fix, adiabat_move */
    rho_r = rho_l;
    p_r = p_l;
    for (int i = 0; i < D; i++) v_r[i] = type == 12 ? vg[i] : v_wall[i] + vg[i];
    v_sq = 0.; for (int i = 0; i < D; i++) v_sq += (v_r[i] * v_r[i]);
    e_r = (p_r / (g - 1.0)) + 0.5 * rho_r * v_sq;
  } else if (type == 15) {                   /* char */
    vn_l = 0.; for (int i = 0; i < D; i++) vn_l += v_l[i] * n[i];
    double vn_bound = 0; for (int i = 0; i < D; i++) vn_bound += v_bound[i] * n[i];
    double r_plus = vn_l + 2. / (g - 1.) * sqrt(g * p_l / rho_l);
    double r_minus = vn_bound - 2. / (g - 1.) * sqrt(g * p_bound / rho_bound);
    double c_star = 0.25 * (g - 1.) * (r_plus - r_minus);
    double vn_star = 0.5 * (r_plus + r_minus);
    if (vn_l < 0) {
      double one_over_s = pow(rho_bound, g) / p_bound;
      v_sq = 0.; for (int i = 0; i < D; i++) v_sq += v_bound[i] * v_bound[i];
      double h_free_stream = g / (g - 1.) * p_bound / rho_bound + 0.5 * v_sq;
      rho_r = pow(1. / g * (one_over_s * c_star * c_star), 1. / (g - 1.));
      for (int i = 0; i < D; i++) v_r[i] = vn_star * n[i] + (v_bound[i] - vn_bound * n[i]);
      p_r = rho_r / g * c_star * c_star;
      e_r = rho_r * h_free_stream - p_r;
    } else {
      double one_over_s = pow(rho_l, g) / p_l;
      rho_r = pow(1. / g * (one_over_s * c_star * c_star), 1. / (g - 1.));
      for (int i = 0; i < D; i++) v_r[i] = vn_star * n[i] + (v_l[i] - vn_l * n[i]);
      p_r = rho_r / g * c_star * c_star;
      v_sq = 0.; for (int i = 0; i < D; i++) v_sq += (v_r[i] * v_r[i]);
      e_r = (p_r / (g - 1.0)) + 0.5 * rho_r * v_sq;
    }
  } else if (type == 16) {                   /* slip_wall_dual */
    rho_r = rho_l;
    vn_l = 0.; for (int i = 0; i < D; i++) vn_l += v_l[i] * n[i];
    for (int i = 0; i < D; i++) v_r[i] = v_l[i] - vn_l * n[i];
    e_r = e_l;
  }
  ur[0] = rho_r;
  for (int i = 0; i < D; i++) ur[i + 1] = rho_r * v_r[i];
  ur[D + 1] = e_r;
}

/* bdy_inters::set_vis_boundary_conditions for the adiabatic walls (12, 14):
 * the energy gradient of the ghost side is replaced so that the wall has no
 * temperature gradient, src/bdy_inters.cpp:1062-1113.  g: (F, D), [k + F*d]. */
static void bc_vis_gradient(int D, const or_physics* ph, const double* ul, const double* ur, double* g)
{
  int F = D + 2;
  double v_sq = 0., gv[9];
  for (int i = 0; i < D; i++) v_sq += (ul[i + 1] * ul[i + 1]);
  double p_l = (ph->gamma - 1.0) * (ul[D + 1] - 0.5 * v_sq / ul[0]);
  double p_r = p_l;
  double inte = p_r / ((ph->gamma - 1.0) * ur[0]);
  for (int j = 0; j < D; j++)
    for (int i = 0; i < D; i++)
      gv[j * D + i] = (g[(j + 1) + F * i] - g[0 + F * i] * ur[j + 1] / ur[0]) / ur[0];
  for (int i = 0; i < D; i++) {
    if (D == 2)
      g[3 + F * i] = inte * g[0 + F * i] + 0.5 * ((ur[1] * ur[1] + ur[2] * ur[2]) / (ur[0] * ur[0])) * g[0 + F * i] +
                     ur[0] * ((ur[1] / ur[0]) * gv[0 * D + i] + (ur[2] / ur[0]) * gv[1 * D + i]);
    else
      g[4 + F * i] = inte * g[0 + F * i] +
                     0.5 * ((ur[1] * ur[1] + ur[2] * ur[2] + ur[3] * ur[3]) / (ur[0] * ur[0])) * g[0 + F * i] +
                     ur[0] * ((ur[1] / ur[0]) * gv[0 * D + i] + (ur[2] / ur[0]) * gv[1 * D + i] +
                              (ur[3] / ur[0]) * gv[2 * D + i]);
  }
}

/* inters::ldg_flux with flux_spec 1 (Dirichlet: own flux) or 2 (von Neumann:
 * ghost flux), src/inters.cpp:589-622, then the normal component. */
static void ldg_flux_bdy(int D, int F, int spec, const double* ul, const double* ur, const double* fl,
                         const double* fr, const double* n, double tau, double* fn)
{
  double fc[15];
  const double* f = spec == 1 ? fl : fr;
  for (int k = 0; k < F; k++)
    for (int d = 0; d < D; d++) fc[k + F * d] = f[k + F * d] + tau * n[d] * (ul[k] - ur[k]);
  for (int k = 0; k < F; k++) {
    fn[k] = fc[k + F * 0] * n[0];
    for (int l = 1; l < D; l++) fn[k] += fc[k + F * l] * n[l];
  }
}

/* sign switch shared by ldg_flux and ldg_solution, src/inters.cpp:555-564, 651-660 */
static double ldg_beta(int D, double pen, const double* n)
{
  if (D == 2) { if ((n[0] + n[1]) < 0.) pen = -pen; }
  else { if ((n[0] + n[1] + sqrt(2.) * n[2]) < 0.) pen = -pen; }
  return pen;
}

/* inters::ldg_flux (interior), src/inters.cpp:550-641 */
static void ldg_flux(int D, int F, const double* ul, const double* ur, const double* fl, const double* fr,
                     const double* n, double tau, double pen, double* fn)
{
  pen = ldg_beta(D, pen, n);
  double fc[15];
  for (int k = 0; k < F; k++) {
    if (D == 2) {
      double jump = n[0] * (fl[k] - fr[k]) + n[1] * (fl[k + F] - fr[k + F]);
      fc[k] = 0.5 * (fl[k] + fr[k]) + pen * n[0] * (jump) + tau * n[0] * (ul[k] - ur[k]);
      fc[k + F] = 0.5 * (fl[k + F] + fr[k + F]) + pen * n[1] * (jump) + tau * n[1] * (ul[k] - ur[k]);
    } else {
      double jump = n[0] * (fl[k] - fr[k]) + n[1] * (fl[k + F] - fr[k + F]) + n[2] * (fl[k + 2 * F] - fr[k + 2 * F]);
      for (int l = 0; l < 3; l++)
        fc[k + F * l] = 0.5 * (fl[k + F * l] + fr[k + F * l]) + pen * n[l] * (jump) + tau * n[l] * (ul[k] - ur[k]);
    }
  }
  for (int k = 0; k < F; k++) {
    fn[k] = fc[k] * n[0];
    for (int l = 1; l < D; l++) fn[k] += fc[k + F * l] * n[l];
  }
}

/* Learned closure (sgs_model 5; no reference counterpart): a 6-64-64-1
 * perceptron, tanh/tanh/softplus, in float, gives c >= 0 of
 * mu_t = rho Delta^2 |S| c from the invariants of the resolved velocity
 * gradient (A_ij = d u_i / d x_j, S its deviatoric symmetric part, W its
 * antisymmetric part, a2 = sum A_ij^2):
 *   x = (tr S^2/a2, tr W^2/a2, tr S^3/a2^1.5, tr S W^2/a2^1.5, tr S^2 W^2/a2^2, log Delta).
 * Parameter layout: W1[64][6] b1[64] W2[64][64] b2[64] w3[64] b3 xmean[6] xscale[6]. */
enum { MLP_IN = 6, MLP_H = 64, MLP_W1 = 0, MLP_B1 = 384, MLP_W2 = 448, MLP_B2 = 4544, MLP_W3 = 4608,
       MLP_B3 = 4672, MLP_XM = 4673, MLP_XS = 4679 };

static float mlp_eval_c(const float* w, const float* xr)
{
  float x[MLP_IN], h1[MLP_H];
  for (int k = 0; k < MLP_IN; k++) x[k] = (xr[k] - w[MLP_XM + k]) * w[MLP_XS + k];
  for (int i = 0; i < MLP_H; i++) {
    float a = w[MLP_B1 + i];
    for (int k = 0; k < MLP_IN; k++) a = fmaf(w[MLP_W1 + i * MLP_IN + k], x[k], a);
    h1[i] = tanhf(a);
  }
  float o = w[MLP_B3];
  for (int j = 0; j < MLP_H; j++) {
    float a = w[MLP_B2 + j];
    for (int i = 0; i < MLP_H; i++) a = fmaf(w[MLP_W2 + j * MLP_H + i], h1[i], a);
    o = fmaf(w[MLP_W3 + j], tanhf(a), o);
  }
  return o > 20.f ? o : log1pf(expf(o));
}

static void sgsf_learned(int D, const or_physics* ph, const double* q, const double* g, double detjac, int order,
                         double* f)
{
  int F = D + 2;
  double rho = q[0], u[3], ke = 0.0, A[3][3], S[3][3], W[3][3], de[3], tr = 0.0, a2 = 0.0;
  for (int i = 0; i < D; i++) { u[i] = q[i + 1] / rho; ke = ke + 0.5 * u[i] * u[i]; }
  double inte = q[F - 1] / rho - ke;
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) A[i][j] = (g[(i + 1) + F * j] - u[i] * g[0 + F * j]) / rho;
  for (int j = 0; j < D; j++) {
    double ud = 0.0;
    for (int i = 0; i < D; i++) ud = ud + u[i] * A[i][j];
    de[j] = (g[(F - 1) + F * j] - ke * g[0 + F * j] - rho * ud - g[0 + F * j] * inte) / rho;
  }
  for (int i = 0; i < D; i++) tr = tr + A[i][i];
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) {
      S[i][j] = 0.5 * (A[i][j] + A[j][i]) - (i == j ? tr / 3.0 : 0.0);
      W[i][j] = 0.5 * (A[i][j] - A[j][i]);
      a2 = a2 + A[i][j] * A[i][j];
    }
  a2 = a2 + 1e-30;
  double S2[3][3], W2[3][3], trS2 = 0, trW2 = 0, trS3 = 0, trSW2 = 0, trS2W2 = 0;
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) {
      double s = 0, w = 0;
      for (int k = 0; k < D; k++) { s = s + S[i][k] * S[k][j]; w = w + W[i][k] * W[k][j]; }
      S2[i][j] = s; W2[i][j] = w;
    }
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) {
      trS2 = trS2 + S[i][j] * S[j][i];
      trW2 = trW2 + W[i][j] * W[j][i];
      trS3 = trS3 + S2[i][j] * S[j][i];
      trSW2 = trSW2 + S[i][j] * W2[j][i];
      trS2W2 = trS2W2 + S2[i][j] * W2[j][i];
    }
  double ra = 1.0 / a2, ra15 = ra / sqrt(a2);
  double vol = detjac * (D == 3 ? 8. : 4.);
  double delta = ph->filter_ratio * (D == 3 ? cbrt(vol) : sqrt(vol)) / (order + 1.);
  float x[MLP_IN] = {(float)(trS2 * ra), (float)(trW2 * ra), (float)(trS3 * ra15), (float)(trSW2 * ra15),
                     (float)(trS2W2 * ra * ra), (float)log(delta)};
  double c = (double)mlp_eval_c(ph->mlp, x);
  double mu_t = rho * delta * delta * sqrt(2.0 * trS2) * c;
  for (int j = 0; j < D; j++) {
    f[0 + F * j] = 0.0;
    f[(F - 1) + F * j] = -ph->gamma * mu_t / 0.5 * de[j];
    for (int i = 1; i < F - 1; i++) f[i + F * j] = -2.0 * mu_t * S[i - 1][j];
  }
}

/* Eddy-viscosity SGS flux at a solution point: eles::calc_sgsf_upts for
 * sgs_model 0 (Smagorinsky) and 1 (WALE) without a wall model,
 * src/eles.cpp:2456-2778.  Kept as the reference computes it, including two
 * index choices of its own: the "velocity" vector is u(i) = q(i)/rho for
 * i < D, so its first entry is rho/rho (src/eles.cpp:2483), and du(i,j)
 * subtracts u(j)*drho(j) (src/eles.cpp:2656).  Both enter the kinetic-energy
 * gradient of the energy flux; the strain rate sees only the second. */
static void sgsf(int D, const or_physics* ph, const double* u, const double* gu /* (F,D) [k+F*l] */, double detjac,
                 int order, double* f /* (F,D) */)
{
  if (ph->sgs_model == 5) {
    sgsf_learned(D, ph, u, gu, detjac, order, f);
    return;
  }
  int F = D + 2;
  double uu[3], drho[3], dene[3], dke[3], de[3], dmom[3][3], du[3][3], S[3][3];
  double ke = 0.0, diag = 0.0, Smod = 0.0, Pr = 0.5, mu_t = 0.0;
  double rho = u[0];
  for (int i = 0; i < D; i++) { uu[i] = u[i] / rho; ke += 0.5 * pow(uu[i], 2); }
  double inte = u[F - 1] / rho - ke;
  for (int k = 0; k < F * D; k++) f[k] = 0.0;
  double vol = detjac * (D == 3 ? 8. : 4.);                     /* calc_ele_vol */
  double delta = ph->filter_ratio * pow(vol, 1. / D) / (order + 1.);
  for (int i = 0; i < D; i++) {
    drho[i] = gu[0 + F * i];
    dene[i] = gu[(F - 1) + F * i];
    for (int j = 1; j < F - 1; j++) dmom[i][j - 1] = gu[j + F * i];
  }
  for (int i = 0; i < D; i++) {
    dke[i] = ke * drho[i];
    for (int j = 0; j < D; j++) {
      du[i][j] = (dmom[i][j] - uu[j] * drho[j]) / rho;
      dke[i] += rho * uu[j] * du[i][j];
    }
    de[i] = (dene[i] - dke[i] - drho[i] * inte) / rho;
  }
  for (int i = 0; i < D; i++) {
    for (int j = 0; j < D; j++) S[i][j] = (du[i][j] + du[j][i]) / 2.0;
    diag += S[i][i] / 3.0;
  }
  for (int i = 0; i < D; i++) S[i][i] -= diag;
  for (int i = 0; i < D; i++)
    for (int j = 0; j < D; j++) Smod += 2.0 * S[i][j] * S[i][j];
  Smod = sqrt(Smod);
  if (ph->sgs_model == 0) {
    double Cs = 0.1;
    mu_t = rho * Cs * Cs * delta * delta * Smod;
  } else {
    double Cs = 0.5, num = 0.0, denom = 0.0, eps = 1.e-12, Sq[3][3];
    diag = 0.0;
    for (int i = 0; i < D; i++)
      for (int j = 0; j < D; j++) {
        Sq[i][j] = 0.0;
        for (int k = 0; k < D; ++k) Sq[i][j] += (du[i][k] * du[k][j] + du[j][k] * du[k][i]) / 2.0;
        diag += du[i][j] * du[j][i] / 3.0;
      }
    for (int i = 0; i < D; i++) Sq[i][i] -= diag;
    for (int i = 0; i < D; i++)
      for (int j = 0; j < D; j++) { num += Sq[i][j] * Sq[i][j]; denom += S[i][j] * S[i][j]; }
    denom = pow(denom, 2.5) + pow(num, 1.25);
    num = pow(num, 1.5);
    mu_t = rho * Cs * Cs * delta * delta * num / (denom + eps);
  }
  for (int j = 0; j < D; j++) {
    f[0 + F * j] = 0.0;
    f[(F - 1) + F * j] = -1.0 * ph->gamma * mu_t / Pr * de[j];
    for (int i = 1; i < F - 1; i++) f[i + F * j] = -2.0 * mu_t * S[i - 1][j];
  }
}

/* --------------------------------------------------------------- residual */

void or_stage_offsets(const or_mesh* m, long long* off)
{
  long long E = m->ne, F = m->nfields, D = m->dims, nu = m->nu, nf = m->nf;
  long long sz[9] = {nf * E * F, nu * E * F * D, nf * E * F * D, nu * E * F * D, nf * E * F, nf * E * F, nf * E * F,
                     nu * E * F * D, nf * E * F * D};
  off[0] = 0;
  for (int i = 0; i < 9; i++) off[i + 1] = off[i] + sz[i];
}

void or_residual(or_mesh* m, const or_physics* ph, const double* u, double* div, double* stages)
{
  int D = m->dims, F = m->nfields, nu = m->nu, nf = m->nf;
  long E = m->ne, EF = E * F;
  double g = ph->gamma;

  /* extrapolate_solution, src/eles.cpp:1256-1327 */
  op_apply(&m->opp0, u, m->ufp, EF, 0);
  /* calculate_gradient, src/eles.cpp:1667-1766 */
  if (ph->viscous)
    for (int d = 0; d < D; d++) op_apply(&m->opp2[d], u, m->gup + (size_t)nu * EF * d, EF, 0);
  /* evaluate_invFlux, src/eles.cpp:1331-1418 */
  for (long e = 0; e < E; e++)
    for (int j = 0; j < nu; j++) {
      double q[5], f[15];
      for (int k = 0; k < F; k++) q[k] = u[j + nu * (e + E * k)];
      invf(D, g, q, f);
      const double* J = m->JG + (size_t)D * D * (j + nu * e);
      for (int k = 0; k < F; k++)
        for (int l = 0; l < D; l++) {
          double s = 0.;
          for (int mm = 0; mm < D; mm++) s += J[l + D * mm] * f[k + F * mm];
          m->tf[j + nu * (e + E * (k + (size_t)F * l))] = s;
        }
    }
  /* int_inters::calculate_common_invFlux, src/int_inters.cpp:225-354 */
  for (int i = 0; i < m->nint; i++) {
    long a = m->il[i], b = m->ir[i];
    long ea = a / nf, eb = b / nf;
    double ul[5], ur[5], n[3], fn[5];
    for (int k = 0; k < F; k++) { ul[k] = m->ufp[a + (size_t)nf * E * k]; ur[k] = m->ufp[b + (size_t)nf * E * k]; }
    for (int d = 0; d < D; d++) n[d] = m->nrm[a + (size_t)nf * E * d];
    if (ph->riemann == 2 && D == 2) roe(g, ul, ur, n, fn);
    else rusanov(D, F, g, ul, ur, n, fn);
    double tl = m->tdA[a], tr = m->tdA[b];
    for (int k = 0; k < F; k++) {
      m->ntc[a + (size_t)nf * E * k] = fn[k] * tl;
      m->ntc[b + (size_t)nf * E * k] = -fn[k] * tr;
    }
    if (ph->viscous) {
      double pen = ldg_beta(D, ph->pen_fact, n);   /* ldg_solution, src/inters.cpp:645-678 */
      for (int k = 0; k < F; k++) {
        double uc = 0.5 * (ul[k] + ur[k]) - pen * (ul[k] - ur[k]);
        m->ddu[a + (size_t)nf * E * k] = (uc - ul[k]);
        m->ddu[b + (size_t)nf * E * k] = (uc - ur[k]);
      }
    }
    (void)ea; (void)eb;
  }
  /* bdy_inters::evaluate_boundaryConditions_invFlux, src/bdy_inters.cpp:245-389 */
  for (int i = 0; i < m->nb; i++) {
    long a = m->bf[i];
    int type = m->bt[i];
    double ul[5], ur[5], n[3], fn[5], fl[15], fr[15];
    for (int k = 0; k < F; k++) ul[k] = m->ufp[a + (size_t)nf * E * k];
    for (int d = 0; d < D; d++) n[d] = m->nrm[a + (size_t)nf * E * d];
    bc_ghost(D, type, ul, n, ph, ur);
    invf(D, g, ul, fl); invf(D, g, ur, fr);
    if (type == 16) {                        /* right_flux of the own flux, src/inters.cpp:299-308 */
      for (int k = 0; k < F; k++) { fn[k] = 0.; for (int l = 0; l < D; l++) fn[k] += fl[k + F * l] * n[l]; }
    } else if (ph->riemann == 2 && D == 2) {
      roe(g, ul, ur, n, fn);
    } else {                                 /* convective_flux_boundary, src/inters.cpp:368-387 */
      for (int k = 0; k < F; k++) {
        double a1 = 0., b1 = 0.;
        for (int l = 0; l < D; l++) { a1 += fl[k + F * l] * n[l]; b1 += fr[k + F * l] * n[l]; }
        fn[k] = 0.5 * (a1 + b1);
      }
    }
    for (int k = 0; k < F; k++) m->ntc[a + (size_t)nf * E * k] = fn[k] * m->tdA[a];
    if (ph->viscous)                         /* ldg_solution, flux_spec 1 or 2: u_c = (u_r + u_l)/2 */
      for (int k = 0; k < F; k++) {
        double uc = 0.5 * (ur[k] + ul[k]);
        m->ddu[a + (size_t)nf * E * k] = (uc - ul[k]);
      }
  }
  if (ph->viscous) {
    /* correct_gradient, src/eles.cpp:1770-1968 */
    for (int d = 0; d < D; d++) op_apply(&m->opp5[d], m->ddu, m->gup + (size_t)nu * EF * d, EF, 1);
    for (long e = 0; e < E; e++)
      for (int j = 0; j < nu; j++) {
        double dj = m->detjac[j + nu * e], inv = 1.0 / dj;
        const double* J = m->JG + (size_t)D * D * (j + nu * e);
        for (int k = 0; k < F; k++) {
          size_t b0 = j + nu * (e + E * k), st = (size_t)nu * EF;
          if (D == 2) {
            double rx = J[0] * inv, ry = J[0 + 2 * 1] * inv, sx = J[1] * inv, sy = J[1 + 2 * 1] * inv;
            double ur_ = m->gup[b0], us = m->gup[b0 + st];
            m->gup[b0] = ur_ * rx + us * sx;
            m->gup[b0 + st] = ur_ * ry + us * sy;
          } else {
            double rx = J[0 + 3 * 0] * inv, ry = J[0 + 3 * 1] * inv, rz = J[0 + 3 * 2] * inv;
            double sx = J[1 + 3 * 0] * inv, sy = J[1 + 3 * 1] * inv, sz = J[1 + 3 * 2] * inv;
            double tx = J[2 + 3 * 0] * inv, ty = J[2 + 3 * 1] * inv, tz = J[2 + 3 * 2] * inv;
            double ur_ = m->gup[b0], us = m->gup[b0 + st], ut = m->gup[b0 + 2 * st];
            m->gup[b0] = ur_ * rx + us * sx + ut * tx;
            m->gup[b0 + st] = ur_ * ry + us * sy + ut * ty;
            m->gup[b0 + 2 * st] = ur_ * rz + us * sz + ut * tz;
          }
        }
      }
    /* extrapolate_corrected_gradient, src/eles.cpp:1973-2052 */
    for (int d = 0; d < D; d++) op_apply(&m->opp0, m->gup + (size_t)nu * EF * d, m->gfp + (size_t)nf * EF * d, EF, 0);
    /* evaluate_viscFlux, src/eles.cpp:2321-2453 (no LES, no motion) */
    for (long e = 0; e < E; e++)
      for (int j = 0; j < nu; j++) {
        double q[5], gq[15], f[15];
        for (int k = 0; k < F; k++) {
          q[k] = u[j + nu * (e + E * k)];
          for (int d = 0; d < D; d++) gq[k + F * d] = m->gup[j + nu * (e + E * (k + (size_t)F * d))];
        }
        visf(D, ph, q, gq, f);
        const double* J = m->JG + (size_t)D * D * (j + nu * e);
        if (ph->les) {
          /* evaluate_viscFlux with LES, src/eles.cpp:2369-2409 */
          double sf[15];
          sgsf(D, ph, q, gq, m->detjac[j + nu * e], m->order, sf);
          for (int k = 0; k < F; k++)
            for (int l = 0; l < D; l++) f[k + F * l] += sf[k + F * l];
          for (int k = 0; k < F; k++)
            for (int l = 0; l < D; l++) {
              double s = 0.0;
              for (int mm = 0; mm < D; mm++) s += J[l + D * mm] * sf[k + F * mm];
              m->sgu[j + nu * (e + E * (k + (size_t)F * l))] = s;
            }
        }
        for (int k = 0; k < F; k++)
          for (int l = 0; l < D; l++)
            for (int mm = 0; mm < D; mm++)
              m->tf[j + nu * (e + E * (k + (size_t)F * l))] += J[l + D * mm] * f[k + F * mm];
      }
    /* evaluate_sgsFlux, src/eles.cpp:3294-3368 */
    if (ph->les)
      for (int d = 0; d < D; d++) op_apply(&m->opp0, m->sgu + (size_t)nu * EF * d, m->sgf + (size_t)nf * EF * d, EF, 0);
  }
  /* extrapolate_totalFlux, src/eles.cpp:1423-1512 */
  for (int d = 0; d < D; d++) op_apply(&m->opp1[d], m->tf + (size_t)nu * EF * d, m->ntd, EF, d > 0);
  /* calculate_divergence, src/eles.cpp:1517-1589 */
  for (int d = 0; d < D; d++) op_apply(&m->opp2[d], m->tf + (size_t)nu * EF * d, div, EF, d > 0);
  if (ph->viscous) {
    /* int_inters::calculate_common_viscFlux, src/int_inters.cpp:359-470 */
    for (int i = 0; i < m->nint; i++) {
      long a = m->il[i], b = m->ir[i];
      double ul[5], ur[5], gl[15], gr[15], fl[15], fr[15], n[3], fn[5];
      for (int k = 0; k < F; k++) {
        ul[k] = m->ufp[a + (size_t)nf * E * k]; ur[k] = m->ufp[b + (size_t)nf * E * k];
        for (int d = 0; d < D; d++) {
          gl[k + F * d] = m->gfp[a + (size_t)nf * E * (k + (size_t)F * d)];
          gr[k + F * d] = m->gfp[b + (size_t)nf * E * (k + (size_t)F * d)];
        }
      }
      visf(D, ph, ul, gl, fl); visf(D, ph, ur, gr, fr);
      if (ph->les)      /* src/int_inters.cpp:411-423: the extrapolated SGS flux joins the viscous flux */
        for (int d = 0; d < D; d++)
          for (int k = 0; k < F; k++) {
            fl[k + F * d] += m->sgf[a + (size_t)nf * E * (k + (size_t)F * d)];
            fr[k + F * d] += m->sgf[b + (size_t)nf * E * (k + (size_t)F * d)];
          }
      for (int d = 0; d < D; d++) n[d] = m->nrm[a + (size_t)nf * E * d];
      ldg_flux(D, F, ul, ur, fl, fr, n, ph->tau, ph->pen_fact, fn);
      for (int k = 0; k < F; k++) {
        m->ntc[a + (size_t)nf * E * k] += fn[k] * m->tdA[a];
        m->ntc[b + (size_t)nf * E * k] += -fn[k] * m->tdA[b];
      }
    }
    /* bdy_inters::evaluate_boundaryConditions_viscFlux, src/bdy_inters.cpp:905-1057 */
    for (int i = 0; i < m->nb; i++) {
      long a = m->bf[i];
      int type = m->bt[i], spec = (type == 12 || type == 14) ? 2 : 1;
      double ul[5], ur[5], gl[15], gr[15], fl[15] = {0}, fr[15] = {0}, n[3], fn[5];
      for (int k = 0; k < F; k++) {
        ul[k] = m->ufp[a + (size_t)nf * E * k];
        for (int d = 0; d < D; d++) gl[k + F * d] = m->gfp[a + (size_t)nf * E * (k + (size_t)F * d)];
      }
      for (int d = 0; d < D; d++) n[d] = m->nrm[a + (size_t)nf * E * d];
      bc_ghost(D, type, ul, n, ph, ur);
      if (spec == 2) {
        for (int q = 0; q < F * D; q++) gr[q] = gl[q];
        bc_vis_gradient(D, ph, ul, ur, gr);
        visf(D, ph, ur, gr, fr);
      } else {
        visf(D, ph, ul, gl, fl);
      }
      if (ph->les)
        for (int d = 0; d < D; d++)
          for (int k = 0; k < F; k++) fl[k + F * d] += m->sgf[a + (size_t)nf * E * (k + (size_t)F * d)];
      ldg_flux_bdy(D, F, spec, ul, ur, fl, fr, n, ph->tau, fn);
      for (int k = 0; k < F; k++) m->ntc[a + (size_t)nf * E * k] += fn[k] * m->tdA[a];
    }
  }
  if (stages) {
    long long off[10]; or_stage_offsets(m, off);
    memcpy(stages + off[0], m->ufp, sizeof(double) * nf * EF);
    if (ph->viscous) {
      memcpy(stages + off[1], m->gup, sizeof(double) * nu * EF * D);
      memcpy(stages + off[2], m->gfp, sizeof(double) * nf * EF * D);
      memcpy(stages + off[6], m->ddu, sizeof(double) * nf * EF);
    }
    memcpy(stages + off[3], m->tf, sizeof(double) * nu * EF * D);
    memcpy(stages + off[4], m->ntd, sizeof(double) * nf * EF);
    memcpy(stages + off[5], m->ntc, sizeof(double) * nf * EF);
    if (ph->les) {
      memcpy(stages + off[7], m->sgu, sizeof(double) * nu * EF * D);
      memcpy(stages + off[8], m->sgf, sizeof(double) * nf * EF * D);
    }
  }
  /* calculate_corrected_divergence, src/eles.cpp:1594-1661 */
  for (size_t i = 0; i < (size_t)nf * EF; i++) m->ntc[i] += -1.0 * m->ntd[i];
  op_apply(&m->opp3, m->ntc, div, EF, 1);
}

/* RK45 coefficients of eles::AdvanceSolution, src/eles.cpp:1093-1113 */
static const double RK4A[5] = {0.0, -0.417890474499852, -1.192151694642677, -1.697784692471528, -1.514183444257156};
static const double RK4B[5] = {0.149659021999229, 0.379210312999627, 0.822955029386982, 0.699450455949122, 0.153057247968152};

void or_rk45(or_mesh* m, const or_physics* ph, double* u, double* reg, double dt, int n_steps, double* norms)
{
  int F = m->nfields, nu = m->nu;
  long E = m->ne;
  double* div = malloc(sizeof(double) * nu * E * F);
  for (int s = 0; s < n_steps; s++) {
    for (int st = 0; st < 5; st++) {
      or_residual(m, ph, u, div, NULL);
      for (long e = 0; e < E; e++)          /* src/eles.cpp:1155-1178, const_src = src = 0 */
        for (int k = 0; k < F; k++)
          for (int j = 0; j < nu; j++) {
            size_t i = j + nu * (e + E * k);
            double rhs = -div[i] / m->detjac[j + nu * e] + 0.0 + 0.0;
            double res = reg[i];
            res = RK4A[st] * res + dt * rhs;
            reg[i] = res;
            u[i] += RK4B[st] * res;
          }
    }
    if (norms) {                             /* compute_res_upts + CalcNormResidual, L1 */
      for (int k = 0; k < F; k++) {
        double sum = 0.;
        for (long e = 0; e < E; e++) {
          double cs = 0;
          for (int j = 0; j < nu; j++) cs += fabs(div[j + nu * (e + E * k)] / m->detjac[j + nu * e] - 0.0 - 0.0);
          sum += cs;
        }
        norms[k + F * s] = sum / (double)(nu * E);
      }
    }
  }
  free(div);
}

double or_kinetic_energy(const or_mesh* m, const double* u)
{
  int D = m->dims, nu = m->nu, n1 = m->n1;
  long E = m->ne;
  double ke = 0.0;
  for (long e = 0; e < E; e++)
    for (int j = 0; j < nu; j++) {
      int ix[3]; upt_idx(m, j, ix);
      double w = m->w1[ix[0]] * m->w1[ix[1]] * (D == 3 ? m->w1[ix[2]] : 1.0);
      double rho = u[j + nu * e], k2 = 0;
      for (int d = 0; d < D; d++) { double mm = u[j + nu * (e + E * (1 + d))]; k2 += mm * mm; }
      ke += w * m->detjac[j + nu * e] * 0.5 * k2 / rho;
    }
  return ke;
}
