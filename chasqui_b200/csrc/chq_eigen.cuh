// chasqui_b200 — eigenvectors of the 1-D adiabatic ideal-MHD system in primitive variables
// W = (rho, u, v, w, p, by, bz) with bx held fixed (Roe & Balsara 1996; Stone et al. 2008,
// App. A), for reconstruction in characteristic variables. Right eigenvectors are the
// columns of Rm, left eigenvectors the rows of Lm; wave order u-cf, u-ca, u-cs, u, u+cs,
// u+ca, u+cf. Degenerate limits (B_perp = 0, bx = 0, cf = cs) follow
// src/eigen_mhd.hpp:14-82. All 49 entries of L and R are written (the structural zeros
// explicitly), so the projections can run over full 7 x 7 matrices.
#pragma once
#include "chq_common.cuh"

namespace chq {

template <class T> struct Eigen7 {
  T L[7][7];
  T R[7][7];
};

template <class T> CHQ_HD void eigensystem(T d, T p, T by, T bz, T bx, T gamma, Eigen7<T> &E) {
  const T sqrtd = sqrt_(d);
  const T isqrtd = T(1) / sqrtd;
  const T asq = gamma * p / d;
  const T a = sqrt_(asq);
  const T casq = divz(bx * bx, d);
  const T bperpsq = by * by + bz * bz;
  const T ctsq = divz(bperpsq, d);
  const T tsum = asq + casq + ctsq;
  const T tdif = asq + ctsq - casq;
  const T disc = sqrt_(fmax_(tdif * tdif + T(4) * ctsq * casq, T(0)));
  const T cfsq = T(0.5) * (tsum + disc);
  const T cssq = fmax_(T(0.5) * (tsum - disc), T(0));
  const T cf = sqrt_(cfsq), cs = sqrt_(cssq);
  T alf, als;
  if (cfsq - cssq <= T(1e-12) * cfsq) {
    alf = T(1); als = T(0);
  } else if (ctsq <= T(1e-12) * (asq + casq)) {
    if (asq >= casq) { alf = T(1); als = T(0); } else { alf = T(0); als = T(1); }
  } else if (asq - cssq <= T(0)) {
    alf = T(0); als = T(1);
  } else if (cfsq - asq <= T(0)) {
    alf = T(1); als = T(0);
  } else {
    alf = sqrt_((asq - cssq) / (cfsq - cssq));
    als = sqrt_((cfsq - asq) / (cfsq - cssq));
  }
  T bety, betz;
  if (bperpsq > T(0)) {
    const T ib = T(1) / sqrt_(bperpsq);
    bety = by * ib;
    betz = bz * ib;
  } else {
    bety = T(1) / sqrt_(T(2));
    betz = bety;
  }
  const T s = (bx >= T(0)) ? T(1) : T(-1);
  const T cff = cf * alf, css = cs * als;
  const T qf = cff * s, qs = css * s;
  const T af = a * alf * sqrtd, as = a * als * sqrtd;
#pragma unroll
  for (int i = 0; i < 7; ++i)
#pragma unroll
    for (int j = 0; j < 7; ++j) { E.L[i][j] = T(0); E.R[i][j] = T(0); }
  auto &Rm = E.R;
  Rm[0][0] = d * alf; Rm[0][2] = d * als; Rm[0][3] = T(1); Rm[0][4] = d * als; Rm[0][6] = d * alf;
  Rm[1][0] = -cff; Rm[1][2] = -css; Rm[1][4] = css; Rm[1][6] = cff;
  Rm[2][0] = qs * bety; Rm[2][1] = -betz; Rm[2][2] = -qf * bety; Rm[2][4] = qf * bety; Rm[2][5] = betz; Rm[2][6] = -qs * bety;
  Rm[3][0] = qs * betz; Rm[3][1] = bety; Rm[3][2] = -qf * betz; Rm[3][4] = qf * betz; Rm[3][5] = -bety; Rm[3][6] = -qs * betz;
  Rm[4][0] = d * alf * asq; Rm[4][2] = d * als * asq; Rm[4][4] = d * als * asq; Rm[4][6] = d * alf * asq;
  Rm[5][0] = as * bety; Rm[5][1] = -betz * s * sqrtd; Rm[5][2] = -af * bety; Rm[5][4] = -af * bety; Rm[5][5] = -betz * s * sqrtd; Rm[5][6] = as * bety;
  Rm[6][0] = as * betz; Rm[6][1] = bety * s * sqrtd; Rm[6][2] = -af * betz; Rm[6][4] = -af * betz; Rm[6][5] = bety * s * sqrtd; Rm[6][6] = as * betz;
  auto &Lm = E.L;
  const T norm = T(0.5) / asq;
  const T ncff = norm * cff, ncss = norm * css, nqf = norm * qf, nqs = norm * qs;
  const T naf = divz(norm * af, d), nas = divz(norm * as, d);
  Lm[0][1] = -ncff; Lm[0][2] = nqs * bety; Lm[0][3] = nqs * betz; Lm[0][4] = divz(norm * alf, d); Lm[0][5] = nas * bety; Lm[0][6] = nas * betz;
  Lm[1][2] = -T(0.5) * betz; Lm[1][3] = T(0.5) * bety; Lm[1][5] = -T(0.5) * betz * s * isqrtd; Lm[1][6] = T(0.5) * bety * s * isqrtd;
  Lm[2][1] = -ncss; Lm[2][2] = -nqf * bety; Lm[2][3] = -nqf * betz; Lm[2][4] = divz(norm * als, d); Lm[2][5] = -naf * bety; Lm[2][6] = -naf * betz;
  Lm[3][0] = T(1); Lm[3][4] = -T(1) / asq;
  Lm[4][1] = ncss; Lm[4][2] = nqf * bety; Lm[4][3] = nqf * betz; Lm[4][4] = divz(norm * als, d); Lm[4][5] = -naf * bety; Lm[4][6] = -naf * betz;
  Lm[5][2] = T(0.5) * betz; Lm[5][3] = -T(0.5) * bety; Lm[5][5] = -T(0.5) * betz * s * isqrtd; Lm[5][6] = T(0.5) * bety * s * isqrtd;
  Lm[6][1] = ncff; Lm[6][2] = -nqs * bety; Lm[6][3] = -nqs * betz; Lm[6][4] = divz(norm * alf, d); Lm[6][5] = nas * bety; Lm[6][6] = nas * betz;
}

}  // namespace chq
