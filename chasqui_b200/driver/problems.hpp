// chasqui_b200 driver — the reference's problem generators on the host (src/pgen.hpp).
//
// Each generator fills primitives and face fields in the reference's packed layout; the
// conversion to conserved variables follows src/pgen.hpp:286-303 (entropy s = p / rho^gamma
// with the host's pow, as in the reference). Field expressions keep the reference's operation
// order so that a run started here begins from the reference's bit pattern. Magnetic fields
// come either directly on faces or from a vector potential on edges (div B = 0 to round-off).
#pragma once
#include <cmath>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>
#include "params.hpp"

namespace chqd {

constexpr double kPi = 3.14159265358979323846;

// geometry of the reference's Mesh (src/mesh.hpp:36-74)
struct Grid {
  int nx1, nx2, nx3, ng, ni, nj, nk, is, ie, js, je, ks, ke;
  bool two_d, three_d;
  double x1min, x1max, x2min, x2max, x3min, x3max, dx1, dx2, dx3;
  void setup() {
    ni = nx1 + 2 * ng;
    nj = (nx2 > 1) ? nx2 + 2 * ng : 1;
    nk = (nx3 > 1) ? nx3 + 2 * ng : 1;
    is = ng; ie = ng + nx1 - 1;
    js = (nx2 > 1) ? ng : 0; je = (nx2 > 1) ? ng + nx2 - 1 : 0;
    ks = (nx3 > 1) ? ng : 0; ke = (nx3 > 1) ? ng + nx3 - 1 : 0;
    two_d = nx2 > 1;
    three_d = nx3 > 1;
    dx1 = (x1max - x1min) / nx1;
    dx2 = (x2max - x2min) / nx2;
    dx3 = (x3max - x3min) / nx3;
  }
  double x1v(int i) const { return x1min + (i - is + 0.5) * dx1; }
  double x2v(int j) const { return x2min + (j - js + 0.5) * dx2; }
  double x3v(int k) const { return x3min + (k - ks + 0.5) * dx3; }
  double x1f(int i) const { return x1min + (i - is) * dx1; }
  double x2f(int j) const { return x2min + (j - js) * dx2; }
  double x3f(int k) const { return x3min + (k - ks) * dx3; }
  size_t cells() const { return (size_t)nk * nj * ni; }
  size_t faces() const { return (size_t)(nk + 1) * (nj + 1) * (ni + 1); }
  size_t c(int k, int j, int i) const { return ((size_t)k * nj + j) * ni + i; }
  size_t f(int k, int j, int i) const { return ((size_t)k * (nj + 1) + j) * (ni + 1) + i; }
};

enum { QD = 0, QVX = 1, QVY = 2, QVZ = 3, QP = 4, QS = 5 };

// host state in the reference layout: w/u (6, nk, nj, ni), face fields (nk+1, nj+1, ni+1)
struct HostState {
  std::vector<double> w, u, b1, b2, b3;
  explicit HostState(const Grid &g)
      : w(6 * g.cells(), 0.0), u(6 * g.cells(), 0.0), b1(g.faces(), 0.0), b2(g.faces(), 0.0), b3(g.faces(), 0.0) {}
  double &W(const Grid &g, int n, int k, int j, int i) { return w[n * g.cells() + g.c(k, j, i)]; }
};

// face fields as the curl of A(component, x, y, z) sampled at edge centres (src/pgen.hpp:29-50)
template <class F> void curl_potential(const Grid &g, HostState &h, F A) {
  const double idx = 1.0 / g.dx1, idy = 1.0 / g.dx2, idz = 1.0 / g.dx3;
  for (int k = 0; k < g.nk + 1; ++k)
    for (int j = 0; j < g.nj + 1; ++j)
      for (int i = 0; i < g.ni + 1; ++i) {
        const double xf = g.x1f(i), yf = g.x2f(j), zf = g.x3f(k);
        const double xv = g.x1v(i), yv = g.x2v(j), zv = g.x3v(k);
        double b1 = 0.0;
        if (g.two_d) b1 += (A(2, xf, g.x2f(j + 1), zv) - A(2, xf, yf, zv)) * idy;
        if (g.three_d) b1 -= (A(1, xf, yv, g.x3f(k + 1)) - A(1, xf, yv, zf)) * idz;
        double b2 = -(A(2, g.x1f(i + 1), yf, zv) - A(2, xf, yf, zv)) * idx;
        if (g.three_d) b2 += (A(0, xv, yf, g.x3f(k + 1)) - A(0, xv, yf, zf)) * idz;
        double b3 = (A(1, g.x1f(i + 1), yv, zf) - A(1, xf, yv, zf)) * idx;
        if (g.two_d) b3 -= (A(0, xv, g.x2f(j + 1), zf) - A(0, xv, yf, zf)) * idy;
        const size_t l = g.f(k, j, i);
        h.b1[l] = b1;
        h.b2[l] = b2;
        h.b3[l] = b3;
      }
}

template <class F> void each_cell(const Grid &g, F fn) {
  for (int k = 0; k < g.nk; ++k)
    for (int j = 0; j < g.nj; ++j)
      for (int i = 0; i < g.ni; ++i) fn(k, j, i);
}
template <class F> void each_face(const Grid &g, F fn) {
  for (int k = 0; k < g.nk + 1; ++k)
    for (int j = 0; j < g.nj + 1; ++j)
      for (int i = 0; i < g.ni + 1; ++i) fn(k, j, i);
}

inline void set_prim(const Grid &g, HostState &h, int k, int j, int i, double d, double vx, double vy, double vz,
                     double p) {
  h.W(g, QD, k, j, i) = d;
  h.W(g, QVX, k, j, i) = vx;
  h.W(g, QVY, k, j, i) = vy;
  h.W(g, QVZ, k, j, i) = vz;
  h.W(g, QP, k, j, i) = p;
}

// circularly polarised Alfven wave along x' = x cos(th) + y sin(th) (src/pgen.hpp:54-92)
inline void pgen_cpaw(Params &pin, const Grid &g, HostState &h) {
  const double dens = pin.real("problem", "dens", 1.0);
  const double pres = pin.real("problem", "pres", 0.1);
  const double b0 = pin.real("problem", "b_par", 1.0);
  const double amp = pin.real("problem", "amp", 0.1);
  const double lambda = pin.real("problem", "lambda", 1.0);
  const double th = pin.real("problem", "angle", 0.0) * kPi / 180.0;
  const double vflow = pin.real("problem", "vflow", 0.0);
  const double dir = pin.real("problem", "dir", 1.0);
  const double kw = 2.0 * kPi / lambda;
  const double cth = std::cos(th), sth = std::sin(th);
  const double fac = -dir * amp / std::sqrt(dens);
  curl_potential(g, h, [=](int c, double x, double y, double) -> double {
    const double xp = x * cth + y * sth, yp = -x * sth + y * cth;
    const double ayp = (amp / kw) * std::sin(kw * xp);
    if (c == 0) return -ayp * sth;
    if (c == 1) return ayp * cth;
    return b0 * yp + (amp / kw) * std::cos(kw * xp);
  });
  if (!g.two_d) each_face(g, [&](int k, int j, int i) { h.b1[g.f(k, j, i)] += b0 * cth; });
  each_cell(g, [&](int k, int j, int i) {
    const double xp = g.x1v(i) * cth + g.x2v(j) * sth;
    const double vyp = fac * std::sin(kw * xp), vz = fac * std::cos(kw * xp);
    set_prim(g, h, k, j, i, dens, vflow * cth - vyp * sth, vflow * sth + vyp * cth, vz, pres);
  });
}

// Orszag-Tang vortex (src/pgen.hpp:94-111)
inline void pgen_orszag_tang(Params &, const Grid &g, HostState &h) {
  const double b0 = 1.0 / std::sqrt(4.0 * kPi);
  curl_potential(g, h, [=](int c, double x, double y, double) -> double {
    if (c != 2) return 0.0;
    return b0 / (2.0 * kPi) * std::cos(2.0 * kPi * y) + b0 / (4.0 * kPi) * std::cos(4.0 * kPi * x);
  });
  each_cell(g, [&](int k, int j, int i) {
    set_prim(g, h, k, j, i, 25.0 / (36.0 * kPi), -std::sin(2.0 * kPi * g.x2v(j)), std::sin(2.0 * kPi * g.x1v(i)), 0.0,
             5.0 / (12.0 * kPi));
  });
}

// over-pressured sphere in a uniform oblique field (src/pgen.hpp:114-135)
inline void pgen_blast(Params &pin, const Grid &g, HostState &h) {
  const double pout = pin.real("problem", "pres_out", 0.1);
  const double pinn = pin.real("problem", "pres_in", 10.0);
  const double rad = pin.real("problem", "radius", 0.1);
  const double b0 = pin.real("problem", "b0", 1.0);
  const double ang = pin.real("problem", "angle", 45.0) * kPi / 180.0;
  double bx = b0 * std::cos(ang), by = b0 * std::sin(ang);
  if (std::fabs(bx) < 1e-14 * b0) bx = 0.0;   // exact zero for axis-aligned fields
  if (std::fabs(by) < 1e-14 * b0) by = 0.0;
  each_face(g, [&](int k, int j, int i) {
    const size_t l = g.f(k, j, i);
    h.b1[l] = bx;
    h.b2[l] = by;
    h.b3[l] = 0.0;
  });
  each_cell(g, [&](int k, int j, int i) {
    const double x = g.x1v(i), y = g.two_d ? g.x2v(j) : 0.0, z = g.three_d ? g.x3v(k) : 0.0;
    const double r = std::sqrt(x * x + y * y + z * z);
    set_prim(g, h, k, j, i, 1.0, 0.0, 0.0, 0.0, (r < rad) ? pinn : pout);
  });
}

// advected field loop, A_z = max(A0 (R - r), 0) (src/pgen.hpp:138-155)
inline void pgen_field_loop(Params &pin, const Grid &g, HostState &h) {
  const double a0 = pin.real("problem", "amp", 1.0e-3);
  const double rad = pin.real("problem", "radius", 0.3);
  const double vx = pin.real("problem", "vx", 1.0);
  const double vy = pin.real("problem", "vy", 0.5);
  const double vz = pin.real("problem", "vz", 0.0);
  curl_potential(g, h, [=](int c, double x, double y, double) -> double {
    if (c != 2) return 0.0;
    const double r = std::sqrt(x * x + y * y);
    return std::fmax(a0 * (rad - r), 0.0);
  });
  each_cell(g, [&](int k, int j, int i) { set_prim(g, h, k, j, i, 1.0, vx, vy, vz, 1.0); });
}

// Riemann problem along x, Brio & Wu by default, optional seeded density noise
// (src/pgen.hpp:158-185; std::mt19937 seeded 42, U(-1, 1) drawn in cell order)
inline void pgen_shock_tube(Params &pin, const Grid &g, HostState &h) {
  const double dl = pin.real("problem", "dl", 1.0), pl = pin.real("problem", "pl", 1.0);
  const double dr = pin.real("problem", "dr", 0.125), pr = pin.real("problem", "pr", 0.1);
  const double byl = pin.real("problem", "byl", 1.0), byr = pin.real("problem", "byr", -1.0);
  const double bx = pin.real("problem", "bx", 0.75);
  const double x0 = pin.real("problem", "x0", 0.0);
  const double ul = pin.real("problem", "ul", 0.0), ur = pin.real("problem", "ur", 0.0);
  const double perturb = pin.real("problem", "perturb", 0.0);
  std::mt19937 rng(42);
  std::uniform_real_distribution<double> noise(-1.0, 1.0);
  each_face(g, [&](int k, int j, int i) {
    const size_t l = g.f(k, j, i);
    h.b1[l] = bx;
    h.b2[l] = (g.x1v(i) < x0) ? byl : byr;
    h.b3[l] = 0.0;
  });
  each_cell(g, [&](int k, int j, int i) {
    const bool left = g.x1v(i) < x0;
    set_prim(g, h, k, j, i, (left ? dl : dr) * (1.0 + perturb * noise(rng)), left ? ul : ur, 0.0, 0.0, left ? pl : pr);
  });
}

// Gresho vortex at Mach `mach` (src/pgen.hpp:192-218)
inline void pgen_gresho(Params &pin, const Grid &g, HostState &h) {
  const double mach = pin.real("problem", "mach", 0.1);
  const double gamma = pin.real("mhd", "gamma", 5.0 / 3.0);
  const double p0 = 1.0 / (gamma * mach * mach);
  each_cell(g, [&](int k, int j, int i) {
    const double x = g.x1v(i), y = g.two_d ? g.x2v(j) : 0.0;
    const double r = std::sqrt(x * x + y * y);
    double vphi, p;
    if (r < 0.2) {
      vphi = 5.0 * r;
      p = p0 + 12.5 * r * r;
    } else if (r < 0.4) {
      vphi = 2.0 - 5.0 * r;
      p = p0 + 12.5 * r * r - 20.0 * r + 4.0 * std::log(r / 0.2) + 4.0;
    } else {
      vphi = 0.0;
      p = p0 - 2.0 + 4.0 * std::log(2.0);
    }
    const double ir = (r > 1e-14) ? 1.0 / r : 0.0;
    set_prim(g, h, k, j, i, 1.0, -vphi * y * ir, vphi * x * ir, 0.0, p);
  });
}

// uniform state (src/pgen.hpp:221-232)
inline void pgen_uniform(Params &pin, const Grid &g, HostState &h) {
  const double d = pin.real("problem", "dens", 1.0), p = pin.real("problem", "pres", 1.0);
  const double vx = pin.real("problem", "vx", 0.0), vy = pin.real("problem", "vy", 0.0), vz = pin.real("problem", "vz", 0.0);
  const double bx = pin.real("problem", "bx", 0.0), by = pin.real("problem", "by", 0.0), bz = pin.real("problem", "bz", 0.0);
  each_face(g, [&](int k, int j, int i) {
    const size_t l = g.f(k, j, i);
    h.b1[l] = bx;
    h.b2[l] = by;
    h.b3[l] = bz;
  });
  each_cell(g, [&](int k, int j, int i) { set_prim(g, h, k, j, i, d, vx, vy, vz, p); });
}

// sinusoidal decay under one diffusive process (src/pgen.hpp:235-266)
inline void pgen_diffusion_test(Params &pin, const Grid &g, HostState &h) {
  const std::string var = pin.str("problem", "var", "b");
  const int axis = pin.integer("problem", "axis", 1);
  const double amp = pin.real("problem", "amp", 1.0e-3);
  const double d0 = pin.real("problem", "dens", 1.0), p0 = pin.real("problem", "pres", 1.0);
  const double L = (axis == 1) ? (g.x1max - g.x1min) : (axis == 2) ? (g.x2max - g.x2min) : (g.x3max - g.x3min);
  const double kw = 2.0 * kPi / L;
  const int comp = axis % 3;
  auto coord = [&](int k, int j, int i) { return (axis == 1) ? g.x1v(i) : (axis == 2) ? g.x2v(j) : g.x3v(k); };
  if (var == "b")
    each_face(g, [&](int k, int j, int i) {
      const double val = amp * std::sin(kw * coord(k, j, i));
      const size_t l = g.f(k, j, i);
      (comp == 0 ? h.b1 : comp == 1 ? h.b2 : h.b3)[l] = val;
    });
  each_cell(g, [&](int k, int j, int i) {
    const double x = coord(k, j, i);
    double d = d0, p = p0, v[3] = {0.0, 0.0, 0.0};
    if (var == "v") v[comp] = amp * std::sin(kw * x);
    if (var == "temp") {
      const double T = p0 / d0 + amp * std::sin(kw * x);
      d = p0 / T;
    }
    if (var == "b") {
      const double s = amp * std::sin(kw * x);
      p = p0 - 0.5 * (s * s);
    }
    set_prim(g, h, k, j, i, d, v[0], v[1], v[2], p);
  });
}

// generator by name, then conserved variables from primitives and face fields
inline void initialize(const std::string &name, Params &pin, const Grid &g, double gamma, HostState &h) {
  if (name == "cpaw") pgen_cpaw(pin, g, h);
  else if (name == "orszag_tang") pgen_orszag_tang(pin, g, h);
  else if (name == "blast") pgen_blast(pin, g, h);
  else if (name == "field_loop") pgen_field_loop(pin, g, h);
  else if (name == "shock_tube") pgen_shock_tube(pin, g, h);
  else if (name == "uniform") pgen_uniform(pin, g, h);
  else if (name == "gresho") pgen_gresho(pin, g, h);
  else if (name == "diffusion_test") pgen_diffusion_test(pin, g, h);
  else throw std::runtime_error("unknown problem: " + name);
  const double gm1 = gamma - 1.0;
  const size_t nc = g.cells();
  each_cell(g, [&](int k, int j, int i) {
    const size_t l = g.c(k, j, i), f = g.f(k, j, i);
    const double bx = 0.5 * (h.b1[f] + h.b1[g.f(k, j, i + 1)]);
    const double by = g.two_d ? 0.5 * (h.b2[f] + h.b2[g.f(k, j + 1, i)]) : h.b2[f];
    const double bz = g.three_d ? 0.5 * (h.b3[f] + h.b3[g.f(k + 1, j, i)]) : h.b3[f];
    const double d = h.w[QD * nc + l], vx = h.w[QVX * nc + l], vy = h.w[QVY * nc + l], vz = h.w[QVZ * nc + l];
    const double p = h.w[QP * nc + l];
    h.u[0 * nc + l] = d;
    h.u[1 * nc + l] = d * vx;
    h.u[2 * nc + l] = d * vy;
    h.u[3 * nc + l] = d * vz;
    h.u[4 * nc + l] = p / gm1 + 0.5 * d * (vx * vx + vy * vy + vz * vz) + 0.5 * (bx * bx + by * by + bz * bz);
    h.w[QS * nc + l] = p / std::pow(d, gamma);
    h.u[5 * nc + l] = d * h.w[QS * nc + l];
  });
}

}  // namespace chqd
