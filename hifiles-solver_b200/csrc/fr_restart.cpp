// fr_restart.cpp -- restart files in the reference's text format, host side.
//
// Layout written by write_restart (src/output.cpp:1057-1107) with each
// type's write_restart_info (src/eles_tris.cpp:546-563,
// src/eles_quads.cpp:725-741, src/eles_tets.cpp:782-800,
// src/eles_pris.cpp:700-726, src/eles_hexas.cpp:882-900) and
// eles::write_restart_data (src/eles.cpp:697-722), element types in the
// order triangles, quads, tets, prisms, hexes, every number printed like an
// ostream of precision 15 (%.15g):
//
//   <time>
//   per element type present:
//     TRIS | QUADS | TETS | PRIS | HEXAS
//     Order
//     <order>
//     Number of solution points per ... element
//     <n_upts>
//     the solution points:
//       quads, hexes: "Location of solution points in 1D", one line
//       triangles, tets: "Location of solution points in triangular |
//         tetrahedral elements", one line of coordinates per point
//       prisms: "Number of solution points in triangle", <n_tri>, the 1-D
//         line as above, "Location of solution points in triangle", one
//         line of (x, y) per triangle point
//     n_eles
//     <n_eles>
//     ele2global_ele array
//     <g_0> <g_1> ...
//     data
//     per element: <global id> then n_upts lines of <u_0> ... <u_{F-1}>
//     (blank line)
//
// Reading follows read_restart / each type's read_restart_info /
// eles::read_restart_data (src/solver.cpp:390-445, src/eles_tris.cpp:511-543,
// src/eles_tets.cpp:749-780, src/eles_pris.cpp:655-698,
// src/eles_hexas.cpp:851-879, src/eles.cpp:623-694): the file's solution
// points may be of another order or family; its values are carried to this
// solver's points through the nodal basis on the file's points, the
// reference's opp_r (eles::set_opp_r, src/eles.cpp:4135-4153).  Points that
// agree with the file's to 1e-13 (the file holds 15 digits) are taken as the
// same points and the values are copied, so a file read back at its own
// points gives exactly the numbers it holds.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "fr_b200.h"
#include "fr_host.hpp"

namespace frb {
extern thread_local std::string g_err;
}
using namespace frb;

namespace {

fr_status rs_fail(fr_status s, const std::string& m)
{
  g_err = m;
  return s;
}

const char* type_name(int t)
{
  static const char* const n[5] = {"TRIS", "QUADS", "TETS", "PRIS", "HEXAS"};
  return t >= 0 && t < 5 ? n[t] : nullptr;
}
int type_dims(int t) { return t == 0 || t == 1 ? 2 : 3; }
int upts_count(int t, int P)
{
  const int n1 = P + 1, nt = (P + 1) * (P + 2) / 2;
  switch (t) {
    case 0: return nt;
    case 1: return n1 * n1;
    case 2: return nt * (P + 3) / 3;
    case 3: return nt * n1;
    case 4: return n1 * n1 * n1;
  }
  return -1;
}

std::string g15(double v)
{
  char b[40];
  std::snprintf(b, sizeof b, "%.15g", v);
  return b;
}

bool next_line(std::istream& in, std::string& s)
{
  if (!std::getline(in, s)) return false;
  if (!s.empty() && s.back() == '\r') s.pop_back();
  return true;
}

// The numbers of one line; false if a token is not a number.
bool parse_numbers(const std::string& s, std::vector<double>& out)
{
  out.clear();
  const char* p = s.c_str();
  for (;;) {
    while (*p == ' ' || *p == '\t') p++;
    if (!*p) return true;
    char* end = nullptr;
    const double x = std::strtod(p, &end);
    if (end == p) return false;
    out.push_back(x);
    p = end;
  }
}

// The header of one block as write_restart_info prints it.
fr_status block_header(const fr_restart_block& B, std::string& out)
{
  const int t = B.ele_type, P = B.order, n1 = P + 1, nt = (P + 1) * (P + 2) / 2, nu = B.n_upts;
  const std::string order = "\nOrder\n" + std::to_string(P) + "\n";
  const double* x = B.loc_pts;
  switch (t) {
    case 1:
    case 4:
      if (!B.loc_1d) return rs_fail(FR_ERR_ARG, "quads and hexes need loc_1d");
      out += std::string(type_name(t)) + order + "Number of solution points per " +
             (t == 1 ? "quadrilateral" : "hexahedral") + " element\n" + std::to_string(nu) +
             "\nLocation of solution points in 1D\n";
      for (int i = 0; i < n1; i++) out += g15(B.loc_1d[i]) + " ";
      out += "\n";
      return FR_OK;
    case 0:
    case 2: {
      if (!x) return rs_fail(FR_ERR_ARG, "triangles and tets need loc_pts");
      const int D = type_dims(t);
      out += std::string(type_name(t)) + order +
             (t == 0 ? "Number of solution points per triangular element\n" : "Number of solution points per element\n") +
             std::to_string(nu) + "\nLocation of solution points in " + (t == 0 ? "triangular" : "tetrahedral") +
             " elements\n";
      for (int k = 0; k < nu; k++) {
        for (int d = 0; d < D; d++) out += g15(x[D * k + d]) + " ";
        out += "\n";
      }
      return FR_OK;
    }
    case 3:
      if (!x) return rs_fail(FR_ERR_ARG, "prisms need loc_pts");
      out += std::string("PRIS") + order + "Number of solution points per prismatic element\n" + std::to_string(nu) +
             "\nNumber of solution points in triangle\n" + std::to_string(nt) + "\nLocation of solution points in 1D\n";
      for (int c = 0; c < n1; c++) out += g15(x[3 * (nt * c) + 2]) + " ";
      out += "\nLocation of solution points in triangle\n";
      for (int k = 0; k < nt; k++) out += g15(x[3 * k]) + " " + g15(x[3 * k + 1]) + " \n";
      return FR_OK;
  }
  return rs_fail(FR_ERR_UNSUPPORTED, "restart blocks exist for element types 0-4");
}

// Reads one block's header after its name line, as read_restart_info does:
// the file's order and its solution points (point-major, D per point).
fr_status read_header(std::istream& f, int t, int& order_r, std::vector<double>& pts)
{
  std::string s;
  const int D = type_dims(t);
  int nu_r = -1, nt_r = -1;
  next_line(f, s);                                    // "Order"
  f >> order_r;
  next_line(f, s);
  next_line(f, s);                                    // "Number of solution points ..."
  f >> nu_r;
  next_line(f, s);
  if (t == 3) {
    next_line(f, s);                                  // "Number of solution points in triangle"
    f >> nt_r;
    next_line(f, s);
  }
  next_line(f, s);                                    // "Location of solution points ..."
  if (!f || order_r < 0 || order_r > kMaxP || nu_r != upts_count(t, order_r) ||
      (t == 3 && nt_r != (order_r + 1) * (order_r + 2) / 2))
    return rs_fail(FR_ERR_ARG, "restart file: inconsistent order and point count");
  const int n1 = order_r + 1;
  pts.assign((size_t)nu_r * D, 0.0);
  if (t == 1 || t == 4) {
    std::vector<double> l(n1);
    for (int i = 0; i < n1; i++)
      if (!(f >> l[i])) return rs_fail(FR_ERR_ARG, "restart file: bad point locations");
    for (int j = 0; j < nu_r; j++) {
      pts[D * j] = l[j % n1];
      pts[D * j + 1] = l[(j / n1) % n1];
      if (D == 3) pts[D * j + 2] = l[j / (n1 * n1)];
    }
  } else if (t == 3) {
    std::vector<double> l(n1), tri(2 * (size_t)nt_r);
    for (int i = 0; i < n1; i++)
      if (!(f >> l[i])) return rs_fail(FR_ERR_ARG, "restart file: bad point locations");
    next_line(f, s);
    next_line(f, s);                                  // "Location of solution points in triangle"
    for (int i = 0; i < 2 * nt_r; i++)
      if (!(f >> tri[i])) return rs_fail(FR_ERR_ARG, "restart file: bad point locations");
    for (int c = 0; c < n1; c++)
      for (int j = 0; j < nt_r; j++) {
        double* p = &pts[3 * (nt_r * c + j)];
        p[0] = tri[2 * j]; p[1] = tri[2 * j + 1]; p[2] = l[c];
      }
  } else {
    for (size_t i = 0; i < pts.size(); i++)
      if (!(f >> pts[i])) return rs_fail(FR_ERR_ARG, "restart file: bad point locations");
  }
  return FR_OK;
}

// The block of type t of a restart file carried to the points `mine`
// (nu of them, point-major) of n_eles elements, matched by global id.
fr_status read_block(const char* path, int t, const double* mine, int nu, int n_eles, int n_fields,
                     const int* ele2global, double* disu_upts, double* time_out)
{
  const char* nm = type_name(t);
  if (!nm) return rs_fail(FR_ERR_UNSUPPORTED, "restart blocks exist for element types 0-4");
  const int D = type_dims(t);
  std::ifstream f(path);
  if (!f) return rs_fail(FR_ERR_ARG, std::string("cannot open ") + path);
  double time;
  if (!(f >> time)) return rs_fail(FR_ERR_ARG, "restart file: no time on the first line");
  if (time_out) *time_out = time;
  std::string s;
  next_line(f, s);
  bool found = false;
  while (next_line(f, s))
    if (s == nm) { found = true; break; }
  if (!found) return rs_fail(FR_ERR_ARG, std::string("restart file has no ") + nm + " block");
  int order_r = -1;
  std::vector<double> pts;
  if (fr_status r = read_header(f, t, order_r, pts)) return r;
  const int nu_r = (int)(pts.size() / D);
  bool same = nu_r == nu;
  for (int i = 0; same && i < nu * D; i++) same = std::fabs(pts[i] - mine[i]) <= 1e-13;
  std::vector<double> R;
  std::string err;
  if (!same && !nodal_interp(t, order_r, pts.data(), nu_r, mine, nu, R, err)) return rs_fail(FR_ERR_ARG, err);
  while (next_line(f, s))
    if (s == "n_eles") break;
  long long ne_r = -1;
  if (!(f >> ne_r) || ne_r < 0) return rs_fail(FR_ERR_ARG, "restart file: bad n_eles");
  next_line(f, s);
  next_line(f, s);                                    // "ele2global_ele array"
  next_line(f, s);                                    // the array
  next_line(f, s);                                    // "data"
  std::unordered_map<long long, int> where;
  for (int e = 0; e < n_eles; e++) where[ele2global ? ele2global[e] : e] = e;
  const size_t NE = (size_t)n_eles;
  std::vector<char> seen(n_eles, 0);
  std::vector<double> v((size_t)nu_r * n_fields), row;
  for (long long i = 0; i < ne_r; i++) {
    // one line with the element's global id, then one line of n_fields values per point
    if (!next_line(f, s) || !parse_numbers(s, row) || row.size() != 1)
      return rs_fail(FR_ERR_ARG, "restart file: truncated element data");
    const long long g = (long long)row[0];
    for (int j = 0; j < nu_r; j++) {
      if (!next_line(f, s) || !parse_numbers(s, row))
        return rs_fail(FR_ERR_ARG, "restart file: truncated element data");
      if ((int)row.size() != n_fields)
        return rs_fail(FR_ERR_ARG, "restart file holds " + std::to_string(row.size()) + " fields per point, not " +
                                       std::to_string(n_fields));
      for (int k = 0; k < n_fields; k++) v[j + (size_t)nu_r * k] = row[k];
    }
    auto it = where.find(g);
    if (it == where.end()) continue;                  // another rank's element
    const int e = it->second;
    seen[e] = 1;
    for (int k = 0; k < n_fields; k++)
      for (int j = 0; j < nu; j++) {
        double acc;
        if (same) {
          acc = v[j + (size_t)nu_r * k];
        } else {
          acc = 0.0;
          for (int jr = 0; jr < nu_r; jr++) acc += R[(size_t)j * nu_r + jr] * v[jr + (size_t)nu_r * k];
        }
        disu_upts[j + (size_t)nu * (e + NE * k)] = acc;
      }
  }
  for (int e = 0; e < n_eles; e++)
    if (!seen[e]) return rs_fail(FR_ERR_ARG, "restart file lacks element " + std::to_string(ele2global ? ele2global[e] : e));
  return FR_OK;
}

}  // namespace

fr_status fr_restart_write(const char* path, double time, const fr_restart_block* blocks, int n_blocks)
{
  g_err.clear();
  if (!path || !blocks || n_blocks < 1) return rs_fail(FR_ERR_ARG, "null argument");
  std::vector<int> ord;
  for (int b = 0; b < n_blocks; b++) {
    const fr_restart_block& B = blocks[b];
    if (!type_name(B.ele_type)) return rs_fail(FR_ERR_UNSUPPORTED, "restart blocks exist for element types 0-4");
    if (B.order < 0 || B.order > kMaxP || B.n_eles < 0 || B.n_fields < 1 || (B.n_eles > 0 && !B.disu_upts))
      return rs_fail(FR_ERR_ARG, "bad restart block");
    if (B.n_upts != upts_count(B.ele_type, B.order)) return rs_fail(FR_ERR_ARG, "n_upts does not match the order");
    for (int o : ord)
      if (blocks[o].ele_type == B.ele_type) return rs_fail(FR_ERR_ARG, "two restart blocks of one element type");
    ord.push_back(b);
  }
  // the reference writes its element types in the order of their codes
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return blocks[a].ele_type < blocks[b].ele_type; });
  std::string out = g15(time) + "\n";
  for (int b : ord) {
    const fr_restart_block& B = blocks[b];
    if (B.n_eles == 0) continue;                      // the reference writes only types present
    if (fr_status r = block_header(B, out)) return r;
    const int nu = B.n_upts;
    out += "n_eles\n" + std::to_string(B.n_eles) + "\nele2global_ele array\n";
    for (int e = 0; e < B.n_eles; e++) out += std::to_string(B.ele2global ? B.ele2global[e] : e) + " ";
    out += "\ndata\n";
    const size_t NE = (size_t)B.n_eles;
    for (int e = 0; e < B.n_eles; e++) {
      out += std::to_string(B.ele2global ? B.ele2global[e] : e) + "\n";
      for (int j = 0; j < nu; j++) {
        for (int k = 0; k < B.n_fields; k++) out += g15(B.disu_upts[j + (size_t)nu * (e + NE * k)]) + " ";
        out += "\n";
      }
    }
    out += "\n";
  }
  std::ofstream f(path, std::ios::binary);
  if (!f) return rs_fail(FR_ERR_ARG, std::string("cannot open ") + path + " for writing");
  f << out;
  if (!f) return rs_fail(FR_ERR_ARG, std::string("write to ") + path + " failed");
  return FR_OK;
}

fr_status fr_restart_read(const char* path, int ele_type, int order, int upts_type, int n_eles, int n_fields,
                          const int* ele2global, double* disu_upts, double* time_out)
{
  g_err.clear();
  if (!path || !disu_upts || n_eles < 0 || n_fields < 1) return rs_fail(FR_ERR_ARG, "null argument");
  if (ele_type != 1 && ele_type != 4)
    return rs_fail(FR_ERR_UNSUPPORTED, "fr_restart_read takes quads (1) and hexes (4); fr_restart_read_points any type");
  Line1D mine;
  std::string err;
  if (!make_line(order, upts_type, 1, 0.0, mine, err)) return rs_fail(FR_ERR_ARG, err);
  const int D = type_dims(ele_type), n1 = order + 1, nu = upts_count(ele_type, order);
  std::vector<double> pts((size_t)nu * D);
  for (int j = 0; j < nu; j++) {
    pts[D * j] = mine.loc[j % n1];
    pts[D * j + 1] = mine.loc[(j / n1) % n1];
    if (D == 3) pts[D * j + 2] = mine.loc[j / (n1 * n1)];
  }
  return read_block(path, ele_type, pts.data(), nu, n_eles, n_fields, ele2global, disu_upts, time_out);
}

fr_status fr_restart_read_points(const char* path, int ele_type, int n_upts, const double* loc_pts, int n_eles,
                                 int n_fields, const int* ele2global, double* disu_upts, double* time_out)
{
  g_err.clear();
  if (!path || !disu_upts || !loc_pts || n_upts < 1 || n_eles < 0 || n_fields < 1)
    return rs_fail(FR_ERR_ARG, "null argument");
  return read_block(path, ele_type, loc_pts, n_upts, n_eles, n_fields, ele2global, disu_upts, time_out);
}
