// fr_vtu.cpp -- VTK unstructured-grid output (.vtu, XML with inline base64
// binary arrays) of a flow solution, the role of the reference's Paraview
// writer (write_vtu, src/output.cpp:580-1055).  The reference interpolates to
// separate plot points; here the points are the solution points themselves,
// and each element is cut into the P^D sub-cells (quads / hexahedra) that join
// neighbouring solution points.  Point data: density, velocity, pressure,
// energy.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "fr_b200.h"

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

}  // namespace

extern "C" fr_status fr_vtu_write(const char* path, int dims, int order, int n_eles, const double* pos_upts,
                                  const double* disu_upts, double gamma)
{
  g_err.clear();
  if (!path || !pos_upts || !disu_upts || n_eles < 1 || order < 1) return vtu_fail(FR_ERR_ARG, "bad argument");
  if (dims != 2 && dims != 3) return vtu_fail(FR_ERR_ARG, "dims must be 2 or 3");
  const int n1 = order + 1, nu = dims == 2 ? n1 * n1 : n1 * n1 * n1, F = dims + 2;
  const size_t E = (size_t)n_eles, npts = (size_t)nu * E;
  if (npts > 0x7fffffffULL) return vtu_fail(FR_ERR_ARG, "too many points for one file");
  std::vector<float> xyz(npts * 3, 0.f), vel(npts * 3, 0.f), rho(npts), p(npts), ene(npts);
  for (size_t i = 0; i < npts; i++) {
    for (int d = 0; d < dims; d++) xyz[3 * i + d] = (float)pos_upts[i + npts * d];
    const double r = disu_upts[i], e = disu_upts[i + npts * (F - 1)];
    double ke = 0.0;
    for (int d = 0; d < dims; d++) {
      const double v = disu_upts[i + npts * (d + 1)] / r;
      vel[3 * i + d] = (float)v;
      ke += 0.5 * r * v * v;
    }
    rho[i] = (float)r;
    ene[i] = (float)e;
    p[i] = (float)((gamma - 1.0) * (e - ke));
  }
  const int sub = dims == 2 ? order * order : order * order * order;
  const int nv = dims == 2 ? 4 : 8;
  std::vector<int32_t> conn, offs;
  std::vector<uint8_t> types;
  conn.reserve(E * sub * nv);
  for (size_t e = 0; e < E; e++) {
    const int32_t base = (int32_t)(e * nu);
    for (int c = 0; c < (dims == 3 ? order : 1); c++)
      for (int b = 0; b < order; b++)
        for (int a = 0; a < order; a++) {
          auto id = [&](int ia, int ib, int ic) { return base + ia + n1 * (ib + n1 * ic); };
          if (dims == 2) {
            const int32_t q[4] = {id(a, b, 0), id(a + 1, b, 0), id(a + 1, b + 1, 0), id(a, b + 1, 0)};
            conn.insert(conn.end(), q, q + 4);
            types.push_back(9);     // VTK_QUAD
          } else {
            const int32_t h[8] = {id(a, b, c),     id(a + 1, b, c),     id(a + 1, b + 1, c),     id(a, b + 1, c),
                                  id(a, b, c + 1), id(a + 1, b, c + 1), id(a + 1, b + 1, c + 1), id(a, b + 1, c + 1)};
            conn.insert(conn.end(), h, h + 8);
            types.push_back(12);    // VTK_HEXAHEDRON
          }
          offs.push_back((int32_t)conn.size());
        }
  }
  std::ofstream f(path, std::ios::binary);
  if (!f) return vtu_fail(FR_ERR_ARG, std::string("cannot open ") + path);
  f << "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\" "
       "header_type=\"UInt32\">\n<UnstructuredGrid>\n<Piece NumberOfPoints=\""
    << npts << "\" NumberOfCells=\"" << types.size() << "\">\n<PointData Scalars=\"Density\" Vectors=\"Velocity\">\n";
  f << "<DataArray type=\"Float32\" Name=\"Density\" format=\"binary\">" << encode(rho) << "</DataArray>\n";
  f << "<DataArray type=\"Float32\" Name=\"Velocity\" NumberOfComponents=\"3\" format=\"binary\">" << encode(vel)
    << "</DataArray>\n";
  f << "<DataArray type=\"Float32\" Name=\"Pressure\" format=\"binary\">" << encode(p) << "</DataArray>\n";
  f << "<DataArray type=\"Float32\" Name=\"Energy\" format=\"binary\">" << encode(ene) << "</DataArray>\n";
  f << "</PointData>\n<Points>\n<DataArray type=\"Float32\" NumberOfComponents=\"3\" format=\"binary\">"
    << encode(xyz) << "</DataArray>\n</Points>\n<Cells>\n";
  f << "<DataArray type=\"Int32\" Name=\"connectivity\" format=\"binary\">" << encode(conn) << "</DataArray>\n";
  f << "<DataArray type=\"Int32\" Name=\"offsets\" format=\"binary\">" << encode(offs) << "</DataArray>\n";
  f << "<DataArray type=\"UInt8\" Name=\"types\" format=\"binary\">" << encode(types) << "</DataArray>\n";
  f << "</Cells>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n";
  if (!f) return vtu_fail(FR_ERR_ARG, std::string("write to ") + path + " failed");
  return FR_OK;
}
