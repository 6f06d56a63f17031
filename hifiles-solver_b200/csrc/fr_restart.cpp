// fr_restart.cpp -- restart files in the reference's text format, host side.
//
// Layout written by write_restart (src/output.cpp:1057-1107) with
// eles::write_restart_info (src/eles_quads.cpp:725-741,
// src/eles_hexas.cpp:882-900) and eles::write_restart_data
// (src/eles.cpp:697-722), every number printed like an ostream of
// precision 15 (%.15g):
//
//   <time>
//   per element type present:
//     QUADS | HEXAS
//     Order
//     <order>
//     Number of solution points per quadrilateral | hexahedral element
//     <n_upts>
//     Location of solution points in 1D
//     <x_0> <x_1> ... <x_P>
//     n_eles
//     <n_eles>
//     ele2global_ele array
//     <g_0> <g_1> ...
//     data
//     per element: <global id> then n_upts lines of <u_0> ... <u_{F-1}>
//     (blank line)
//
// Reading follows read_restart / eles::read_restart_info / read_restart_data
// (src/solver.cpp:390-445, src/eles_hexas.cpp:851-879,
// src/eles.cpp:623-694): the file's solution points may be of another order;
// its values are carried to this solver's points by the tensor Lagrange
// interpolation of eles::set_opp_r (src/eles.cpp:4135-4153).
#include <cmath>
#include <cstdio>
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

const char* type_name(int t) { return t == 1 ? "QUADS" : (t == 4 ? "HEXAS" : nullptr); }
const char* type_phrase(int t)
{
  return t == 1 ? "Number of solution points per quadrilateral element"
                : "Number of solution points per hexahedral element";
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

}  // namespace

fr_status fr_restart_write(const char* path, double time, const fr_restart_block* blocks, int n_blocks)
{
  g_err.clear();
  if (!path || !blocks || n_blocks < 1) return rs_fail(FR_ERR_ARG, "null argument");
  std::string out = g15(time) + "\n";
  for (int b = 0; b < n_blocks; b++) {
    const fr_restart_block& B = blocks[b];
    const char* nm = type_name(B.ele_type);
    const int dims = B.ele_type == 1 ? 2 : 3;
    if (!nm) return rs_fail(FR_ERR_UNSUPPORTED, "restart blocks exist for quads (1) and hexes (4)");
    if (B.order < 0 || B.n_eles < 0 || B.n_fields < 1 || !B.loc_1d || (B.n_eles > 0 && !B.disu_upts))
      return rs_fail(FR_ERR_ARG, "bad restart block");
    const int n1 = B.order + 1, nu = dims == 2 ? n1 * n1 : n1 * n1 * n1;
    if (B.n_upts != nu) return rs_fail(FR_ERR_ARG, "n_upts does not match the order");
    if (B.n_eles == 0) continue;                      // the reference writes only types present
    out += std::string(nm) + "\nOrder\n" + std::to_string(B.order) + "\n" + type_phrase(B.ele_type) + "\n" +
           std::to_string(nu) + "\nLocation of solution points in 1D\n";
    for (int i = 0; i < n1; i++) out += g15(B.loc_1d[i]) + " ";
    out += "\nn_eles\n" + std::to_string(B.n_eles) + "\nele2global_ele array\n";
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
  const char* nm = type_name(ele_type);
  if (!nm) return rs_fail(FR_ERR_UNSUPPORTED, "restart blocks exist for quads (1) and hexes (4)");
  const int dims = ele_type == 1 ? 2 : 3;
  Line1D mine;
  std::string err;
  if (!make_line(order, upts_type, 1, 0.0, mine, err)) return rs_fail(FR_ERR_ARG, err);
  std::ifstream f(path);
  if (!f) return rs_fail(FR_ERR_ARG, std::string("cannot open ") + path);
  double t;
  if (!(f >> t)) return rs_fail(FR_ERR_ARG, "restart file: no time on the first line");
  if (time_out) *time_out = t;
  std::string s;
  next_line(f, s);
  bool found = false;
  while (next_line(f, s))
    if (s == nm) { found = true; break; }
  if (!found) return rs_fail(FR_ERR_ARG, std::string("restart file has no ") + nm + " block");
  int order_r = -1, nu_r = -1;
  next_line(f, s);                                    // "Order"
  f >> order_r;
  next_line(f, s);
  next_line(f, s);                                    // "Number of solution points ..."
  f >> nu_r;
  next_line(f, s);
  next_line(f, s);                                    // "Location of solution points in 1D"
  const int n1r = order_r + 1;
  if (order_r < 0 || order_r > 20 || nu_r != (dims == 2 ? n1r * n1r : n1r * n1r * n1r))
    return rs_fail(FR_ERR_ARG, "restart file: inconsistent order and point count");
  std::vector<double> loc_r(n1r);
  for (int i = 0; i < n1r; i++)
    if (!(f >> loc_r[i])) return rs_fail(FR_ERR_ARG, "restart file: bad point locations");
  // 1-D interpolation matrix from the file's points to ours: R[a][m] = l_m(x_a)
  const int n1 = order + 1;
  std::vector<double> R((size_t)n1 * n1r);
  for (int a = 0; a < n1; a++)
    for (int m = 0; m < n1r; m++) R[(size_t)a * n1r + m] = lagrange(mine.loc[a], m, loc_r.data(), n1r);
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
  const int nu = dims == 2 ? n1 * n1 : n1 * n1 * n1;
  const size_t NE = (size_t)n_eles;
  std::vector<char> seen(n_eles, 0);
  std::vector<double> v((size_t)nu_r * n_fields);
  for (long long i = 0; i < ne_r; i++) {
    long long g;
    if (!(f >> g)) return rs_fail(FR_ERR_ARG, "restart file: truncated element data");
    for (int j = 0; j < nu_r; j++)
      for (int k = 0; k < n_fields; k++)
        if (!(f >> v[j + (size_t)nu_r * k])) return rs_fail(FR_ERR_ARG, "restart file: truncated element data");
    auto it = where.find(g);
    if (it == where.end()) continue;                  // another rank's element
    const int e = it->second;
    seen[e] = 1;
    for (int k = 0; k < n_fields; k++)
      for (int j = 0; j < nu; j++) {
        const int a = j % n1, b = (j / n1) % n1, c = dims == 3 ? j / (n1 * n1) : 0;
        double acc = 0.0;
        for (int jr = 0; jr < nu_r; jr++) {
          const int ar = jr % n1r, br = (jr / n1r) % n1r, cr = dims == 3 ? jr / (n1r * n1r) : 0;
          double w = R[(size_t)a * n1r + ar] * R[(size_t)b * n1r + br];
          if (dims == 3) w *= R[(size_t)c * n1r + cr];
          acc += w * v[jr + (size_t)nu_r * k];
        }
        disu_upts[j + (size_t)nu * (e + NE * k)] = acc;
      }
  }
  for (int e = 0; e < n_eles; e++)
    if (!seen[e]) return rs_fail(FR_ERR_ARG, "restart file lacks element " + std::to_string(ele2global ? ele2global[e] : e));
  return FR_OK;
}
