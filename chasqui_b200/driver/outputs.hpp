// chasqui_b200 driver — the reference's output formats.
//
//   legacy VTK, big-endian floats, PLUTO-compatible layout (src/output.hpp:32-85):
//     rho prs vx1 vx2 vx3 Bx1 Bx2 Bx3 as cell data over the active cells, i fastest
//   history file columns (src/main.cpp:218-235): time dt mass mom1 mom2 mom3 etot ekin emag
//     eint divB_max divB_L1, 12 significant digits
//   restart: a 40-byte header {magic "CHSQ", nx1, nx2, nx3, ng, cycle, time, real_size} as
//     laid out by g++ on x86-64, then u0, b1f0, b2f0, b3f0 in the packed reference layout
//     including ghosts (src/restart.hpp:11-56)
#pragma once
#include <cstdint>
#include <cstring>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>
#include "problems.hpp"

namespace chqd {

inline void put_be_floats(std::ofstream &f, const std::vector<float> &v) {
  std::vector<unsigned char> b(v.size() * 4);
  for (size_t n = 0; n < v.size(); ++n) {
    uint32_t x;
    std::memcpy(&x, &v[n], 4);
    for (int q = 0; q < 4; ++q) b[4 * n + q] = (unsigned char)(x >> (24 - 8 * q));
  }
  f.write(reinterpret_cast<const char *>(b.data()), (std::streamsize)b.size());
}

inline void put_be_int(std::ofstream &f, int32_t v) {
  unsigned char b[4];
  for (int q = 0; q < 4; ++q) b[q] = (unsigned char)((uint32_t)v >> (24 - 8 * q));
  f.write(reinterpret_cast<const char *>(b), 4);
}

// w: (6, nk, nj, ni) primitives, bcc: (3, nk, nj, ni) cell-centred field, both downloaded
// Legacy VTK dump in the reference's layout (src/output.hpp:32-84). `cells` holds the eight
// big-endian float32 scalar planes (rho, prs, vx1, vx2, vx3, Bx1, Bx2, Bx3 over the active
// cells, i fastest) exactly as the file stores them; the device builds them (the "vtk"
// snapshot field), so the host writes them without touching the values.
inline void write_vtk(const Grid &g, const char *cells, const std::string &path, double time, int cycle) {
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot write " + path);
  f << "# vtk DataFile Version 2.0\nChasqui MHD VTK Data\nBINARY\nDATASET RECTILINEAR_GRID\n";
  f << "FIELD FieldData 2\nTIME 1 1 float\n";
  put_be_floats(f, {(float)time});
  f << "\nCYCLE 1 1 int\n";
  put_be_int(f, cycle);
  f << "\n";
  const int n2 = g.two_d ? g.nx2 + 1 : 1, n3 = g.three_d ? g.nx3 + 1 : 1;
  f << "DIMENSIONS " << g.nx1 + 1 << " " << n2 << " " << n3 << "\n";
  std::vector<float> x(g.nx1 + 1), y(n2), z(n3);
  for (int i = 0; i <= g.nx1; ++i) x[i] = (float)g.x1f(g.is + i);
  for (int j = 0; j < n2; ++j) y[j] = (float)(g.two_d ? g.x2f(g.js + j) : g.x2min);
  for (int k = 0; k < n3; ++k) z[k] = (float)(g.three_d ? g.x3f(g.ks + k) : g.x3min);
  f << "X_COORDINATES " << g.nx1 + 1 << " float\n";
  put_be_floats(f, x);
  f << "\nY_COORDINATES " << n2 << " float\n";
  put_be_floats(f, y);
  f << "\nZ_COORDINATES " << n3 << " float\n";
  put_be_floats(f, z);
  f << "\n";
  const size_t ncell = (size_t)g.nx1 * g.nx2 * g.nx3;
  f << "CELL_DATA " << ncell << "\n";
  const char *names[8] = {"rho", "prs", "vx1", "vx2", "vx3", "Bx1", "Bx2", "Bx3"};
  for (int q = 0; q < 8; ++q) {
    f << "SCALARS " << names[q] << " float\nLOOKUP_TABLE default\n";
    f.write(cells + (size_t)q * ncell * 4, (std::streamsize)(ncell * 4));
    f << "\n";
  }
}

struct RestartHeader {
  int magic = 0x43485351;
  int nx1, nx2, nx3, ng;
  int cycle;
  double time;
  int real_size;
};
static_assert(sizeof(RestartHeader) == 40, "restart header layout");

inline void write_restart(const Grid &g, const std::string &path, double time, int cycle, const std::vector<double> &u,
                          const std::vector<double> &b1, const std::vector<double> &b2, const std::vector<double> &b3) {
  RestartHeader h;
  h.nx1 = g.nx1; h.nx2 = g.nx2; h.nx3 = g.nx3; h.ng = g.ng;
  h.cycle = cycle;
  h.time = time;
  h.real_size = (int)sizeof(double);
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot write " + path);
  f.write(reinterpret_cast<const char *>(&h), sizeof(h));
  for (const std::vector<double> *a : {&u, &b1, &b2, &b3})
    f.write(reinterpret_cast<const char *>(a->data()), (std::streamsize)(a->size() * sizeof(double)));
}

inline void read_restart(const Grid &g, const std::string &path, double &time, int &cycle, std::vector<double> &u,
                         std::vector<double> &b1, std::vector<double> &b2, std::vector<double> &b3) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot open restart file " + path);
  RestartHeader h;
  f.read(reinterpret_cast<char *>(&h), sizeof(h));
  if (!f || h.magic != 0x43485351) throw std::runtime_error("not a Chasqui restart file: " + path);
  if (h.nx1 != g.nx1 || h.nx2 != g.nx2 || h.nx3 != g.nx3 || h.ng != g.ng || h.real_size != (int)sizeof(double))
    throw std::runtime_error("restart file does not match the mesh (nx, nghost or precision differ)");
  for (std::vector<double> *a : {&u, &b1, &b2, &b3})
    f.read(reinterpret_cast<char *>(a->data()), (std::streamsize)(a->size() * sizeof(double)));
  if (!f) throw std::runtime_error("restart file is truncated: " + path);
  time = h.time;
  cycle = h.cycle;
}

}  // namespace chqd
