// fr_vtu.cpp -- VTK unstructured-grid output (.vtu, XML with inline base64
// binary arrays) of a flow solution, the role of the reference's Paraview
// writer (write_vtu, src/output.cpp:580-1055).  Quads and hexes: the points
// are the solution points themselves, and each element is cut into the P^D
// sub-cells (quads / hexahedra) that join neighbouring solution points.
// Triangles, tets and prisms (fr_vtu_write_mixed): like the reference, the
// solution is interpolated through the element's nodal basis to plot points,
// here the equispaced lattice of order P, which is cut into P^D sub-cells
// (triangles; tetrahedra, four from each inner octahedron; wedges).  Point
// data: density, velocity, pressure, energy.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "fr_b200.h"
#include "fr_host.hpp"

namespace frb {
extern thread_local std::string g_err;
}
using namespace frb;

namespace {

fr_status vtu_fail(fr_status s, const std::string& m)
{
  g_err = m;
  return s;
}

std::string b64(const unsigned char* p, size_t n)
{
  static const char* T = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
  std::string o;
  o.reserve((n + 2) / 3 * 4);
  for (size_t i = 0; i < n; i += 3) {
    uint32_t v = (uint32_t)p[i] << 16;
    if (i + 1 < n) v |= (uint32_t)p[i + 1] << 8;
    if (i + 2 < n) v |= p[i + 2];
    o += T[(v >> 18) & 63];
    o += T[(v >> 12) & 63];
    o += i + 1 < n ? T[(v >> 6) & 63] : '=';
    o += i + 2 < n ? T[v & 63] : '=';
  }
  return o;
}

// VTK's binary inline encoding: a UInt32 byte count, then the bytes, encoded together.
template <typename T>
std::string encode(const std::vector<T>& a)
{
  std::vector<unsigned char> buf(4 + a.size() * sizeof(T));
  uint32_t nb = (uint32_t)(a.size() * sizeof(T));
  std::memcpy(buf.data(), &nb, 4);
  if (!a.empty()) std::memcpy(buf.data() + 4, a.data(), nb);
  return b64(buf.data(), buf.size());
}

// Everything a file holds, at its points: positions, the four point arrays
// from the conserved state, and the cells.
struct Grid {
  std::vector<float> xyz, vel, rho, p, ene;
  std::vector<int32_t> conn, offs;
  std::vector<uint8_t> types;
  void point(const double* x, int dims, const double* u, double gamma)
  {
    const double r = u[0], e = u[dims + 1];
    double ke = 0.0;
    float v3[3] = {0.f, 0.f, 0.f}, x3[3] = {0.f, 0.f, 0.f};
    for (int d = 0; d < dims; d++) {
      const double v = u[d + 1] / r;
      v3[d] = (float)v;
      x3[d] = (float)x[d];
      ke += 0.5 * r * v * v;
    }
    xyz.insert(xyz.end(), x3, x3 + 3);
    vel.insert(vel.end(), v3, v3 + 3);
    rho.push_back((float)r);
    ene.push_back((float)e);
    p.push_back((float)((gamma - 1.0) * (e - ke)));
  }
  void cell(const int32_t* v, int n, uint8_t type)
  {
    conn.insert(conn.end(), v, v + n);
    offs.push_back((int32_t)conn.size());
    types.push_back(type);
  }
};

fr_status write_grid(const char* path, const Grid& g)
{
  std::ofstream f(path, std::ios::binary);
  if (!f) return vtu_fail(FR_ERR_ARG, std::string("cannot open ") + path);
  f << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" "
       "header_type=\"UInt32\">\n<UnstructuredGrid>\n<Piece NumberOfPoints=\""
    << g.rho.size() << "\" NumberOfCells=\"" << g.types.size()
    << "\">\n<PointData Scalars=\"Density\" Vectors=\"Velocity\">\n";
  f << "<DataArray type=\"Float32\" Name=\"Density\" format=\"binary\">" << encode(g.rho) << "</DataArray>\n";
  f << "<DataArray type=\"Float32\" Name=\"Velocity\" NumberOfComponents=\"3\" format=\"binary\">" << encode(g.vel)
    << "</DataArray>\n";
  f << "<DataArray type=\"Float32\" Name=\"Pressure\" format=\"binary\">" << encode(g.p) << "</DataArray>\n";
  f << "<DataArray type=\"Float32\" Name=\"Energy\" format=\"binary\">" << encode(g.ene) << "</DataArray>\n";
  f << "</PointData>\n<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">"
    << encode(g.xyz) << "</DataArray>\n</Points>\n<Cells>\n";
  f << "<DataArray type=\"Int32\" Name=\"connectivity\" format=\"binary\">" << encode(g.conn) << "</DataArray>\n";
  f << "<DataArray type=\"Int32\" Name=\"offsets\" format=\"binary\">" << encode(g.offs) << "</DataArray>\n";
  f << "<DataArray type=\"UInt8\" Name=\"types\" format=\"binary\">" << encode(g.types) << "</DataArray>\n";
  f << "</Cells>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
  if (!f) return vtu_fail(FR_ERR_ARG, std::string("write to ") + path + " failed");
  return FR_OK;
}

// Sub-cells of one element of order P (local point indices, VTK cell type):
// quads and hexes over the tensor solution points (x fastest), the others
// over the equispaced lattice of plot_points.
struct SubCells {
  std::vector<int32_t> v;
  int nv = 0;
  uint8_t type = 0;
};

// index of lattice point (i, j) of a triangle of order m (rows of constant j)
inline int tri_idx(int m, int i, int j) { return j * (m + 1) - j * (j - 1) / 2 + i; }

// The triangle lattice's P^2 sub-triangles, counter-clockwise in (r, s).
std::vector<std::array<int, 3>> tri_cells(int P)
{
  std::vector<std::array<int, 3>> c;
  for (int j = 0; j < P; j++)
    for (int i = 0; i + j < P; i++) {
      c.push_back({tri_idx(P, i, j), tri_idx(P, i + 1, j), tri_idx(P, i, j + 1)});
      if (i + j < P - 1) c.push_back({tri_idx(P, i + 1, j), tri_idx(P, i + 1, j + 1), tri_idx(P, i, j + 1)});
    }
  return c;
}

SubCells sub_cells(int type, int P)
{
  SubCells S;
  const int n1 = P + 1;
  if (type == FR_ELE_QUAD || type == FR_ELE_HEX) {
    const bool hex = type == FR_ELE_HEX;
    auto id = [&](int a, int b, int c) { return a + n1 * (b + n1 * c); };
    S.nv = hex ? 8 : 4;
    S.type = hex ? 12 : 9;   // VTK_HEXAHEDRON, VTK_QUAD
    for (int c = 0; c < (hex ? P : 1); c++)
      for (int b = 0; b < P; b++)
        for (int a = 0; a < P; a++) {
          const int32_t q[8] = {id(a, b, c),     id(a + 1, b, c),     id(a + 1, b + 1, c),     id(a, b + 1, c),
                                id(a, b, c + 1), id(a + 1, b, c + 1), id(a + 1, b + 1, c + 1), id(a, b + 1, c + 1)};
          S.v.insert(S.v.end(), q, q + S.nv);
        }
  } else if (type == FR_ELE_TRI) {
    S.nv = 3;
    S.type = 5;              // VTK_TRIANGLE
    for (auto& t : tri_cells(P)) S.v.insert(S.v.end(), t.begin(), t.end());
  } else if (type == FR_ELE_PRISM) {
    // wedges: VTK wants the base triangle's normal pointing away from the top
    const int nt = n1 * (n1 + 1) / 2;
    S.nv = 6;
    S.type = 13;             // VTK_WEDGE
    for (int c = 0; c < P; c++)
      for (auto& t : tri_cells(P)) {
        const int32_t w[6] = {t[0] + nt * c, t[2] + nt * c, t[1] + nt * c,
                              t[0] + nt * (c + 1), t[2] + nt * (c + 1), t[1] + nt * (c + 1)};
        S.v.insert(S.v.end(), w, w + 6);
      }
  } else {
    // tets: at every lattice point (i, j, k) a corner tet; in every inner
    // octahedron four tets around its (i+1, j, k) - (i, j+1, k+1) diagonal;
    // in every inverted corner one more: P^3 in all, each turned to positive volume
    std::vector<int> off(n1 + 1, 0);
    for (int k = 0; k < n1; k++) off[k + 1] = off[k] + (P - k + 1) * (P - k + 2) / 2;
    auto id = [&](int i, int j, int k) { return off[k] + tri_idx(P - k, i, j); };
    auto add = [&](std::array<int, 3> a, std::array<int, 3> b, std::array<int, 3> c, std::array<int, 3> d) {
      long long vol = 0;
      const int u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, w[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]},
                x[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
      vol = (long long)u[0] * (w[1] * x[2] - w[2] * x[1]) - (long long)u[1] * (w[0] * x[2] - w[2] * x[0]) +
            (long long)u[2] * (w[0] * x[1] - w[1] * x[0]);
      if (vol < 0) std::swap(b, c);
      const int32_t t[4] = {id(a[0], a[1], a[2]), id(b[0], b[1], b[2]), id(c[0], c[1], c[2]), id(d[0], d[1], d[2])};
      S.v.insert(S.v.end(), t, t + 4);
    };
    S.nv = 4;
    S.type = 10;             // VTK_TETRA
    for (int k = 0; k < P; k++)
      for (int j = 0; j + k < P; j++)
        for (int i = 0; i + j + k < P; i++) {
          add({i, j, k}, {i + 1, j, k}, {i, j + 1, k}, {i, j, k + 1});
          if (i + j + k < P - 1) {
            const std::array<int, 3> A{i + 1, j, k}, B{i, j + 1, k + 1}, ring[4] = {
                {i, j + 1, k}, {i + 1, j + 1, k}, {i + 1, j, k + 1}, {i, j, k + 1}};
            for (int r = 0; r < 4; r++) add(A, B, ring[r], ring[(r + 1) % 4]);
          }
          if (i + j + k < P - 2) add({i + 1, j + 1, k}, {i + 1, j, k + 1}, {i, j + 1, k + 1}, {i + 1, j + 1, k + 1});
        }
  }
  return S;
}

// The equispaced plot lattice of order P of a triangle, tet or prism
// ((n, D) point-major on the reference element [-1, 1]).
std::vector<double> plot_points(int type, int P)
{
  std::vector<double> x;
  const double h = 2.0 / P;
  if (type == FR_ELE_TRI || type == FR_ELE_PRISM) {
    for (int c = 0; c < (type == FR_ELE_PRISM ? P + 1 : 1); c++)
      for (int j = 0; j <= P; j++)
        for (int i = 0; i + j <= P; i++) {
          x.push_back(-1.0 + h * i);
          x.push_back(-1.0 + h * j);
          if (type == FR_ELE_PRISM) x.push_back(-1.0 + h * c);
        }
  } else {
    for (int k = 0; k <= P; k++)
      for (int j = 0; j + k <= P; j++)
        for (int i = 0; i + j + k <= P; i++) {
          x.push_back(-1.0 + h * i);
          x.push_back(-1.0 + h * j);
          x.push_back(-1.0 + h * k);
        }
  }
  return x;
}

}  // namespace

extern "C" fr_status fr_vtu_write(const char* path, int dims, int order, int n_eles, const double* pos_upts,
                                  const double* disu_upts, double gamma)
{
  g_err.clear();
  if (!path || !pos_upts || !disu_upts || n_eles < 1 || order < 1) return vtu_fail(FR_ERR_ARG, "bad argument");
  if (dims != 2 && dims != 3) return vtu_fail(FR_ERR_ARG, "dims must be 2 or 3");
  fr_vtu_block b{dims == 2 ? FR_ELE_QUAD : FR_ELE_HEX, n_eles, nullptr, pos_upts, disu_upts};
  return fr_vtu_write_mixed(path, order, &b, 1, gamma);
}

extern "C" fr_status fr_vtu_write_mixed(const char* path, int order, const fr_vtu_block* blocks, int n_blocks,
                                        double gamma)
{
  g_err.clear();
  if (!path || !blocks || n_blocks < 1 || order < 1 || order > kMaxP) return vtu_fail(FR_ERR_ARG, "bad argument");
  const int dims = blocks[0].ele_type == FR_ELE_TRI || blocks[0].ele_type == FR_ELE_QUAD ? 2 : 3;
  const int F = dims + 2, n1 = order + 1, nt = n1 * (n1 + 1) / 2;
  size_t total = 0;
  for (int b = 0; b < n_blocks; b++) {
    const fr_vtu_block& B = blocks[b];
    const int t = B.ele_type;
    if (t < 0 || t > 4) return vtu_fail(FR_ERR_ARG, "element type 0-4");
    if ((t == FR_ELE_TRI || t == FR_ELE_QUAD ? 2 : 3) != dims) return vtu_fail(FR_ERR_ARG, "blocks of one dimension");
    if (B.n_eles < 0 || (B.n_eles > 0 && (!B.pos_upts || !B.disu_upts)))
      return vtu_fail(FR_ERR_ARG, "bad block");
    if (B.n_eles > 0 && t != FR_ELE_QUAD && t != FR_ELE_HEX && !B.loc_pts)
      return vtu_fail(FR_ERR_ARG, "triangles, tets and prisms need loc_pts");
    const int nl = t == FR_ELE_TRI ? nt : t == FR_ELE_QUAD ? n1 * n1 : t == FR_ELE_TET ? nt * (order + 3) / 3
                 : t == FR_ELE_PRISM ? nt * n1 : n1 * n1 * n1;
    total += (size_t)nl * B.n_eles;
  }
  if (total > 0x7fffffffULL) return vtu_fail(FR_ERR_ARG, "too many points for one file");
  Grid g;
  for (int b = 0; b < n_blocks; b++) {
    const fr_vtu_block& B = blocks[b];
    if (B.n_eles == 0) continue;
    const int t = B.ele_type;
    const bool tensor = t == FR_ELE_QUAD || t == FR_ELE_HEX;
    const int nu = t == FR_ELE_TRI ? nt : t == FR_ELE_QUAD ? n1 * n1 : t == FR_ELE_TET ? nt * (order + 3) / 3
                 : t == FR_ELE_PRISM ? nt * n1 : n1 * n1 * n1;
    // the nodal basis of the solution points at the plot points (identity for quads and hexes)
    std::vector<double> R;
    int nl = nu;
    if (!tensor) {
      const std::vector<double> L = plot_points(t, order);
      nl = (int)(L.size() / dims);
      std::string err;
      if (!nodal_interp(t, order, B.loc_pts, nu, L.data(), nl, R, err)) return vtu_fail(FR_ERR_ARG, err);
    }
    const SubCells S = sub_cells(t, order);
    const size_t E = (size_t)B.n_eles, NE = (size_t)nu * E;
    std::vector<double> x(dims), u(F);
    for (size_t e = 0; e < E; e++) {
      const int32_t base = (int32_t)g.rho.size();
      for (int j = 0; j < nl; j++) {
        if (tensor) {
          const size_t ix = j + (size_t)nu * e;
          for (int d = 0; d < dims; d++) x[d] = B.pos_upts[ix + NE * d];
          for (int k = 0; k < F; k++) u[k] = B.disu_upts[ix + NE * k];
        } else {
          for (int d = 0; d < dims; d++) x[d] = 0.0;
          for (int k = 0; k < F; k++) u[k] = 0.0;
          for (int i = 0; i < nu; i++) {
            const double w = R[(size_t)j * nu + i];
            const size_t ix = i + (size_t)nu * e;
            for (int d = 0; d < dims; d++) x[d] += w * B.pos_upts[ix + NE * d];
            for (int k = 0; k < F; k++) u[k] += w * B.disu_upts[ix + NE * k];
          }
        }
        g.point(x.data(), dims, u.data(), gamma);
      }
      for (size_t c = 0; c < S.v.size(); c += S.nv) {
        int32_t v[8];
        for (int q = 0; q < S.nv; q++) v[q] = base + S.v[c + q];
        g.cell(v, S.nv, S.type);
      }
    }
  }
  return write_grid(path, g);
}
