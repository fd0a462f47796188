// chasqui_b200 — problem generators on the device.
//
// Initial conditions of the workloads this path is measured on, written directly into a
// mesh's u0 / b?f0 (all cells and faces, ghosts included, as the reference's host generators
// do before their first boundary fill). Primitive -> conserved follows src/pgen.hpp:286-300
// (face-averaged centred B, E = p/(gamma-1) + rho v^2/2 + B^2/2, entropy rho p / rho^gamma).
// Face fields from a vector potential use the discrete curl of src/pgen.hpp:30-50, so
// div B = 0 to round-off.
//   orszag_tang : src/pgen.hpp:94-111, optional pressure rescale to plasma beta
//   cpaw        : circularly polarised Alfven wave along 2 pi (m1/L1, m2/L2, m3/L3) (the
//                 reference's CPAW, src/pgen.hpp:54-91, rotates only in x-y)
//   blast       : src/pgen.hpp:114-135 plus seeded uniform relative density noise from a
//                 counter-based splitmix64 stream over the active cells in C order
#pragma once
#include "chq_common.cuh"

namespace chq {

enum : int { PG_ORSZAG_TANG = 0, PG_CPAW = 1, PG_BLAST = 2 };

struct PgenArgs {
  Geom g;
  int problem;
  double gamma;
  double prm[12];
  // cpaw basis (e1 along k, e2, e3 transverse) and wavenumber
  double e1[3], e2[3], e3[3], kmag;
  // blast: uniform field (b0 cos(angle), b0 sin(angle)), tiny components flushed to zero
  double bxy[2];
  double *u, *b1, *b2, *b3;
};

CHQ_HD double pg_x1v(const Geom &g, int i) { return g.x1min + (i - g.is + 0.5) * g.dx1; }
CHQ_HD double pg_x2v(const Geom &g, int j) { return g.x2min + (j - g.js + 0.5) * g.dx2; }
CHQ_HD double pg_x3v(const Geom &g, int k) { return g.x3min + (k - g.ks + g.koff + 0.5) * g.dx3; }
CHQ_HD double pg_x1f(const Geom &g, int i) { return g.x1min + (i - g.is) * g.dx1; }
CHQ_HD double pg_x2f(const Geom &g, int j) { return g.x2min + (j - g.js) * g.dx2; }
CHQ_HD double pg_x3f(const Geom &g, int k) { return g.x3min + (k - g.ks + g.koff) * g.dx3; }

// splitmix64 of (seed, index): uniform double in [0, 1) from the top 53 bits
CHQ_HD double pg_uniform(unsigned long long seed, unsigned long long idx) {
  unsigned long long z = seed + (idx + 1ULL) * 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// vector potential component c at (x, y, z)
CHQ_D double pg_A(const PgenArgs &a, int c, double x, double y, double z) {
  if (a.problem == PG_ORSZAG_TANG) {
    if (c != 2) return 0.0;
    const double b0 = 1.0 / sqrt(4.0 * M_PI);
    return b0 / (2.0 * M_PI) * cos(2.0 * M_PI * y) + b0 / (4.0 * M_PI) * cos(4.0 * M_PI * x);
  }
  // cpaw: A = (amp/k) (sin(k s) e2 + cos(k s) e3), s = e1 . x
  const double amp = a.prm[6];
  const double s = x * a.e1[0] + y * a.e1[1] + z * a.e1[2];
  const double ks = a.kmag * s;
  return (amp / a.kmag) * (sin(ks) * a.e2[c] + cos(ks) * a.e3[c]);
}

__global__ void __launch_bounds__(256) pgen_faces_kernel(const PgenArgs a) {
  const Geom &g = a.g;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nfx = (long)(g.ni + 1), nfy = (long)(g.nj + 1);
  const int i = (int)(t % nfx);
  const int j = (int)((t / nfx) % nfy);
  const int k = (int)(t / (nfx * nfy));
  if (k > g.nk) return;
  const long l = g.idx(k, j, i);
  double b1 = 0.0, b2 = 0.0, b3 = 0.0;
  if (a.problem == PG_BLAST) {
    // uniform field components, evaluated on the host (chq_init_problem) with the host's
    // cos/sin so that they carry the same bits as the host generator's
    b1 = a.bxy[0];
    b2 = a.bxy[1];
  } else {
    const double xf = pg_x1f(g, i), yf = pg_x2f(g, j), zf = pg_x3f(g, k);
    const double xv = pg_x1v(g, i), yv = pg_x2v(g, j), zv = pg_x3v(g, k);
    const double xf1 = pg_x1f(g, i + 1), yf1 = pg_x2f(g, j + 1), zf1 = pg_x3f(g, k + 1);
    const double idx = 1.0 / g.dx1, idy = 1.0 / g.dx2, idz = 1.0 / g.dx3;
    if (g.two_d) b1 += (pg_A(a, 2, xf, yf1, zv) - pg_A(a, 2, xf, yf, zv)) * idy;
    if (g.three_d) b1 -= (pg_A(a, 1, xf, yv, zf1) - pg_A(a, 1, xf, yv, zf)) * idz;
    b2 = -(pg_A(a, 2, xf1, yf, zv) - pg_A(a, 2, xf, yf, zv)) * idx;
    if (g.three_d) b2 += (pg_A(a, 0, xv, yf, zf1) - pg_A(a, 0, xv, yf, zf)) * idz;
    b3 = (pg_A(a, 1, xf1, yv, zf) - pg_A(a, 1, xf, yv, zf)) * idx;
    if (g.two_d) b3 -= (pg_A(a, 0, xv, yf1, zf) - pg_A(a, 0, xv, yf, zf)) * idy;
    if (a.problem == PG_CPAW) {
      // the uniform parallel field (not representable by a periodic potential)
      const double bpar = a.prm[5];
      b1 += bpar * a.e1[0];
      b2 += bpar * a.e1[1];
      b3 += bpar * a.e1[2];
    }
  }
  a.b1[l] = b1;
  a.b2[l] = b2;
  a.b3[l] = b3;
}

__global__ void __launch_bounds__(256) pgen_cells_kernel(const PgenArgs a) {
  const Geom &g = a.g;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int i = (int)(t % g.ni);
  const int j = (int)((t / g.ni) % g.nj);
  const int k = (int)(t / ((long)g.ni * g.nj));
  if (k >= g.nk) return;
  const long l = g.idx(k, j, i);
  const long vs = g.vstride;
  double d, vx = 0.0, vy = 0.0, vz = 0.0, p;
  const double x = pg_x1v(g, i), y = pg_x2v(g, j), z = pg_x3v(g, k);
  if (a.problem == PG_ORSZAG_TANG) {
    const double b0 = 1.0 / sqrt(4.0 * M_PI);
    d = 25.0 / (36.0 * M_PI);
    vx = -sin(2.0 * M_PI * y);
    vy = sin(2.0 * M_PI * x);
    p = (a.prm[0] > 0.0) ? a.prm[0] * b0 * b0 / 2.0 : 5.0 / (12.0 * M_PI);
  } else if (a.problem == PG_CPAW) {
    d = a.prm[3];
    p = a.prm[4];
    const double s = x * a.e1[0] + y * a.e1[1] + z * a.e1[2];
    const double fac = -a.prm[6] / sqrt(d);
    const double vt2 = fac * sin(a.kmag * s), vt3 = fac * cos(a.kmag * s);
    vx = vt2 * a.e2[0] + vt3 * a.e3[0];
    vy = vt2 * a.e2[1] + vt3 * a.e3[1];
    vz = vt2 * a.e2[2] + vt3 * a.e3[2];
  } else {
    const double xb = x, yb = g.two_d ? y : 0.0, zb = g.three_d ? z : 0.0;
    const double r = sqrt(xb * xb + yb * yb + zb * zb);
    p = (r < a.prm[2]) ? a.prm[0] : a.prm[1];
    d = 1.0;
    const double amp = a.prm[5];
    const bool active = (i >= g.is && i <= g.ie && j >= g.js && j <= g.je && k >= g.ks && k <= g.ke);
    if (amp != 0.0 && active) {
      const unsigned long long idx =
          ((unsigned long long)(k - g.ks + g.koff) * g.nx2 + (unsigned long long)(j - g.js)) * g.nx1 + (unsigned long long)(i - g.is);
      const unsigned long long seed = (unsigned long long)a.prm[6];
      d = 1.0 + amp * (2.0 * pg_uniform(seed, idx) - 1.0);
    }
  }
  const double bx = 0.5 * (a.b1[l] + a.b1[l + 1]);
  const double by = g.two_d ? 0.5 * (a.b2[l] + a.b2[l + g.sj]) : a.b2[l];
  const double bz = g.three_d ? 0.5 * (a.b3[l] + a.b3[l + g.sk]) : a.b3[l];
  const double gm1 = a.gamma - 1.0;
  a.u[IDN * vs + l] = d;
  a.u[IM1 * vs + l] = d * vx;
  a.u[IM2 * vs + l] = d * vy;
  a.u[IM3 * vs + l] = d * vz;
  a.u[IEN * vs + l] = p / gm1 + 0.5 * d * (vx * vx + vy * vy + vz * vz) + 0.5 * (bx * bx + by * by + bz * bz);
  const double s = p / pow(d, a.gamma);
  a.u[IENT * vs + l] = d * s;
}

}  // namespace chq
