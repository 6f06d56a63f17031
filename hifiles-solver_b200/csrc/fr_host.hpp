// fr_host.hpp -- host-side set-up of the FR path: 1-D bases and correction
// functions, tensor-product element operators, mesh wiring and metrics.
//
// Everything here runs once per solver on the host in FP64; the results are
// uploaded and then only read by the kernels.
#pragma once

#include <string>
#include <vector>

namespace frb {

constexpr int kMaxP = 10;

// 1-D solution points on [-1, 1] (upts_type 0 Gauss, 1 Gauss-Lobatto).
// Returns false if (P, type) is not available.
bool points_1d(int P, int type, double* out);

double lagrange(double r, int mode, const double* pts, int n);
double dlagrange(double r, int mode, const double* pts, int n);
double legendre(double r, int n);
double dlegendre(double r, int n);
double dvcjh(double r, int side, int P, double eta);   // side 0: left, 1: right
double vcjh_eta(int scheme, int P, double user_eta);   // NaN if undefined

// The 1-D pieces every tensor-product operator of the reference factors into.
// For Gauss-type solution points all the reference's dense operators
// (opp_0 .. opp_6) have exactly one non-zero factor per line, equal to one
// of these numbers (the other factors are Lagrange polynomials evaluated at
// their own nodes, i.e. exactly 1 or 0).
struct Line1D {
  int P = 0, n1 = 0;
  double loc[kMaxP + 1] = {};
  double Lm[kMaxP + 1] = {};              // l_m(-1)
  double Lp[kMaxP + 1] = {};              // l_m(+1)
  double D[kMaxP + 1][kMaxP + 1] = {};    // D[k][m] = l'_m(xi_k)
  double gL[kMaxP + 1] = {};              // g_L'(xi_k)  (left correction function)
  double gR[kMaxP + 1] = {};              // g_R'(xi_k)
  double w[kMaxP + 1] = {};               // quadrature weights of the points
  double eta = 0.0;
};

bool make_line(int P, int upts_type, int vcjh_scheme, double eta, Line1D& out, std::string& err);

// Row-major (nu_to, nu_from) matrix carrying values at the solution points
// `from` of one element (type 0-4, the given order; D coordinates per point)
// to the points `to` through that element's nodal basis (fr_mixed.cpp).
bool nodal_interp(int type, int order, const double* from, int nu_from, const double* to, int nu_to,
                  std::vector<double>& R, std::string& err);

// Conforming mesh of one tensor element type with periodic wiring.
struct Mesh {
  int dims = 0, P = 0, n1 = 0, nu = 0, nf = 0, nface = 0, nfpf = 0, nfields = 0;
  long long ne = 0;
  std::vector<double> xv;      // (nv, dims)
  std::vector<int> c2v;        // (ne, 2^dims)
  // metrics in the reference layouts
  std::vector<double> pos_upts, pos_fpts;   // (n, ne, dims)
  std::vector<double> detjac;               // (nu, ne)
  std::vector<double> JG;                   // (dims, dims, nu, ne)
  std::vector<double> tdA;                  // (nf, ne)
  std::vector<double> nrm;                  // (nf, ne, dims)
  // interface wiring: flat flux-point indices fpt + nf*ele
  std::vector<int> il, ir;
  // per element flux point: index of the matching point on the other side,
  // whether this side is the left one, and the left side's unit normal
  std::vector<int> mate;                    // (nf, ne)
  std::vector<unsigned char> is_left;       // (nf, ne)
  std::vector<double> nL;                   // (nf, ne, dims)
  // boundary flux points (faces given a boundary type): flat index, type;
  // their mate is -1 - (position in this list)
  std::vector<int> bf;
  std::vector<unsigned char> bt;
};

// Default volume cubature of the integral diagnostics: the tensor
// Gauss-Legendre rule of `rule` points per direction in the reference's point
// order (quads: first coordinate fastest; hexes: first coordinate slowest),
// in full double precision (the reference's data/cubature_{quad,hexa}.dat
// print the same rules to 12-15 significant digits).  Returns the point count
// (0 for an unsupported rule); loc is (dims, n) with the point index slowest.
int volume_cubature(int dims, int rule, std::vector<double>& loc, std::vector<double>& w);
// The reference's interpolation to the cubature points, opp(j, k) = the
// nodal basis of solution point k at cubature point j (nc, nu), first index
// fastest (eles::set_opp_volume_cubpts, src/eles.cpp:4111-4130), and the
// Jacobian determinant at every cubature point (nc, ne) (src/eles.cpp:5320-5352).
void volume_cubature_setup(const Mesh& m, const Line1D& L, int nc, const double* loc, std::vector<double>& opp,
                           std::vector<double>& detj);

// Local point sets (reference orderings) of the element type.
void element_points(int dims, const Line1D& L, std::vector<double>& loc_upts, std::vector<double>& tloc_fpts,
                    std::vector<double>& tnorm_fpts);

// bctype (ne, 2*dims) or null: reference boundary type of each local face
// (0 = matched with another face).
bool build_mesh(int dims, const Line1D& L, long long nv, const double* xv, long long ne, const int* c2v,
                const double* shift, const int* bctype, Mesh& m, std::string& err);

// Recompute the per-fpt interface data (mate, is_left, nL) after the metrics
// were replaced.
void finish_wiring(Mesh& m);

}  // namespace frb
