// chasqui_b200 — reconstruction in per-cell form.
//
// The reference reconstructs per FACE from a 6-cell stencil (src/recon.hpp:1-7), so every
// cell's limited parabola is evaluated twice (once for each of its faces). Here each cell c
// produces its own pair (aL, aR) = (value at its left face, value at its right face) from the
// 5 cells q5[0..4] = q_{c-2..c+2}; face i then takes ql = aR_{i-1}, qr = aL_i. Every
// expression is evaluated with the same operands in the same order as the reference's
// per-face form, so both give bitwise-identical face states (this is checked against the
// reference library in the tests). The mirror-symmetric grouping of sums is part of the
// parity contract and is kept as published (Fleischmann, Adami & Adams 2019).
#pragma once
#include "chq_common.cuh"

namespace chq {

// van Leer harmonic slope (src/recon.hpp:14-18)
template <class T> CHQ_HD T vl_slope(T qm, T q0, T qp) {
  const T dl = q0 - qm, dr = qp - q0;
  const T d2 = dl * dr;
  return (d2 > T(0)) ? T(2) * d2 / (dl + dr) : T(0);
}

// monotonised central slope, CW84 eq. 1.8 (src/recon.hpp:21-27)
template <class T> CHQ_HD T mc_slope(T qm, T q0, T qp) {
  const T dl = q0 - qm, dr = qp - q0;
  if (dl * dr <= T(0)) return T(0);
  const T dc = T(0.5) * (qp - qm);
  const T lim = T(2) * fmin_(fabs_(dl), fabs_(dr));
  return sgn(dc) * fmin_(fabs_(dc), lim);
}

// CW84 interface value between cells a and b (src/recon.hpp:42-44)
template <class T> CHQ_HD T ppm_face(T qa, T qb, T dqa, T dqb) {
  return T(0.5) * (qa + qb) + div6(dqa - dqb);
}

// CW84 parabola monotonisation of one cell (src/recon.hpp:47-57)
template <class T> CHQ_HD void ppm_limit(T q, T &qL, T &qR) {
  if ((qR - q) * (q - qL) <= T(0)) {
    qL = q;
    qR = q;
    return;
  }
  const T d = qR - qL;
  const T c = q - T(0.5) * (qL + qR);
  const T d2over6 = div6(d * d);
  if (d * c > d2over6) qL = T(3) * q - T(2) * qR;
  else if (d * c < -d2over6) qR = T(3) * q - T(2) * qL;
}

// extremum-preserving 4th-order interface between q0 and qp1 (src/recon.hpp:85-100)
template <class T> CHQ_HD T ppmx_face(T qm1, T q0, T qp1, T qp2) {
  const T C = T(1.25);
  T qf = (T(7) / T(12)) * (q0 + qp1) - (T(1) / T(12)) * (qm1 + qp2);
  if ((qf - q0) * (qp1 - qf) < T(0)) {
    const T d2 = T(3) * ((q0 + qp1) - T(2) * qf);
    const T d2l = (qm1 + qp1) - T(2) * q0;
    const T d2r = (q0 + qp2) - T(2) * qp1;
    T d2lim = T(0);
    if (d2 * d2l > T(0) && d2 * d2r > T(0)) d2lim = sgn(d2) * fmin_(fmin_(C * fabs_(d2l), C * fabs_(d2r)), fabs_(d2));
    qf = T(0.5) * (q0 + qp1) - div6(d2lim);
  }
  return qf;
}

// extremum-preserving limiter of one cell's parabola (src/recon.hpp:104-127)
template <class T> CHQ_HD void ppmx_limit(T qm2, T qm1, T q, T qp1, T qp2, T &qL, T &qR) {
  const T C = T(1.25);
  const T dqm = q - qL, dqp = qR - q;
  const bool extremum = (dqm * dqp <= T(0)) || ((qp1 - q) * (q - qm1) <= T(0));
  if (extremum) {
    const T d2 = T(6) * ((qL + qR) - T(2) * q);
    const T d2c = (qm1 + qp1) - T(2) * q;
    const T d2l = (qm2 + q) - T(2) * qm1;
    const T d2r = (q + qp2) - T(2) * qp1;
    T d2lim = T(0);
    if (d2 * d2c > T(0) && d2 * d2l > T(0) && d2 * d2r > T(0))
      d2lim = sgn(d2) * fmin_(fmin_(C * fabs_(d2l), C * fabs_(d2r)), fmin_(C * fabs_(d2c), fabs_(d2)));
    const T rho = (fabs_(d2) > T(1e-12) * (fabs_(q) + fabs_(qm1) + fabs_(qp1)) + Tiny<T>::v) ? divz(d2lim, d2) : T(0);
    if (rho < T(1) - T(1e-12)) {
      qL = q - rho * dqm;
      qR = q + rho * dqp;
    }
  } else {
    if (fabs_(dqm) >= T(2) * fabs_(dqp)) qL = q - T(2) * dqp;
    if (fabs_(dqp) >= T(2) * fabs_(dqm)) qR = q + T(2) * dqm;
  }
}

// WENO-Z (Borges et al. 2008) right-interface value of the cell with stencil
// (f_{-2}, f_{-1}, f_0, f_1, f_2) (src/recon.hpp:144-164)
template <class T> CHQ_HD T wenoz_right(T fm2, T fm1, T f0, T fp1, T fp2) {
  const T eps = Tiny<T>::weno_eps;
  const T c13 = T(13) / T(12);
  const T b0 = c13 * sqr((fm2 + f0) - T(2) * fm1) + T(0.25) * sqr((T(3) * f0 + fm2) - T(4) * fm1);
  const T b1 = c13 * sqr((fm1 + fp1) - T(2) * f0) + T(0.25) * sqr(fm1 - fp1);
  const T b2 = c13 * sqr((fp2 + f0) - T(2) * fp1) + T(0.25) * sqr((T(3) * f0 + fp2) - T(4) * fp1);
  const T tau = fabs_(b0 - b2);
  const T a0 = T(0.1) * (T(1) + divz(tau, b0 + eps));
  const T a1 = T(0.6) * (T(1) + divz(tau, b1 + eps));
  const T a2 = T(0.3) * (T(1) + divz(tau, b2 + eps));
  const T inv = T(1) / (a0 + a1 + a2);
  const T q0 = div6(T(2) * fm2 - T(7) * fm1 + T(11) * f0);
  const T q1 = div6(-fm1 + T(5) * f0 + T(2) * fp1);
  const T q2 = div6(T(2) * f0 + T(5) * fp1 - fp2);
  return inv * (a0 * q0 + a1 * q1 + a2 * q2);
}

// Both interface values of one cell: aR = wenoz_right(q_{c-2..c+2}) and aL = the same
// formula on the mirrored stencil. Mirroring maps the smoothness indicators (b0, b1, b2) to
// (b2, b1, b0) with bitwise-equal values (the sums are commutative and a square does not see
// the sign), and tau to itself, so both sides share the three indicators and the three
// quotients tau / (b + eps): 5 divisions per cell instead of 8, same results bit for bit.
template <class T> CHQ_HD void wenoz_cell(const T q[5], T &aL, T &aR) {
  const T eps = Tiny<T>::weno_eps;
  const T c13 = T(13) / T(12);
  const T b0 = c13 * sqr((q[0] + q[2]) - T(2) * q[1]) + T(0.25) * sqr((T(3) * q[2] + q[0]) - T(4) * q[1]);
  const T b1 = c13 * sqr((q[1] + q[3]) - T(2) * q[2]) + T(0.25) * sqr(q[1] - q[3]);
  const T b2 = c13 * sqr((q[4] + q[2]) - T(2) * q[3]) + T(0.25) * sqr((T(3) * q[2] + q[4]) - T(4) * q[3]);
  const T tau = fabs_(b0 - b2);
  const T d0 = T(1) + divz(tau, b0 + eps);
  const T d1 = T(1) + divz(tau, b1 + eps);
  const T d2 = T(1) + divz(tau, b2 + eps);
  {
    const T a0 = T(0.1) * d0, a1 = T(0.6) * d1, a2 = T(0.3) * d2;
    const T inv = T(1) / (a0 + a1 + a2);
    const T r0 = div6(T(2) * q[0] - T(7) * q[1] + T(11) * q[2]);
    const T r1 = div6(-q[1] + T(5) * q[2] + T(2) * q[3]);
    const T r2 = div6(T(2) * q[2] + T(5) * q[3] - q[4]);
    aR = inv * (a0 * r0 + a1 * r1 + a2 * r2);
  }
  {
    const T a0 = T(0.1) * d2, a1 = T(0.6) * d1, a2 = T(0.3) * d0;
    const T inv = T(1) / (a0 + a1 + a2);
    const T r0 = div6(T(2) * q[4] - T(7) * q[3] + T(11) * q[2]);
    const T r1 = div6(-q[3] + T(5) * q[2] + T(2) * q[1]);
    const T r2 = div6(T(2) * q[2] + T(5) * q[1] - q[0]);
    aL = inv * (a0 * r0 + a1 * r1 + a2 * r2);
  }
}

// CW84 flattening coefficient of the cell with pressures p5 = p_{c-2..c+2} and normal
// velocities um1 = u_{c-1}, up1 = u_{c+1} (src/recon.hpp:179-187)
template <class T> CHQ_HD T flattening(const T p5[5], T um1, T up1) {
  const T dp = p5[3] - p5[1];
  const T dp2 = p5[4] - p5[0];
  const T pmin = fmin_(p5[1], p5[3]);
  const bool strong = (fabs_(dp) > T(0.33) * pmin) && (um1 > up1);
  if (!strong) return T(0);
  const T ratio = (fabs_(dp2) > Tiny<T>::v) ? dp / dp2 : T(0);
  return fmin_(T(1), fmax_(T(0), T(10) * (ratio - T(0.75))));
}

// Number of stencil cells each side of the centre that scheme R reads.
template <int R> struct Reach { static constexpr int v = (R == R_DC) ? 0 : (R == R_PLM) ? 1 : 2; };

// Per-cell reconstruction: q5[0..4] = q_{c-2..c+2} (only q5[1..3] for PLM, q5[2] for DC).
// aL = value at the cell's left face (face c), aR = value at its right face (face c+1).
template <int R, class T> CHQ_HD void recon_cell(const T q5[5], T &aL, T &aR) {
  if constexpr (R == R_DC) {
    aL = q5[2];
    aR = q5[2];
  } else if constexpr (R == R_PLM) {
    const T s = vl_slope(q5[1], q5[2], q5[3]);
    aR = q5[2] + T(0.5) * s;
    aL = q5[2] - T(0.5) * s;
  } else if constexpr (R == R_PPM) {
    const T sm = mc_slope(q5[0], q5[1], q5[2]);
    const T s0 = mc_slope(q5[1], q5[2], q5[3]);
    const T sp = mc_slope(q5[2], q5[3], q5[4]);
    aL = ppm_face(q5[1], q5[2], sm, s0);
    aR = ppm_face(q5[2], q5[3], s0, sp);
    ppm_limit(q5[2], aL, aR);
  } else if constexpr (R == R_PPMX) {
    aL = ppmx_face(q5[0], q5[1], q5[2], q5[3]);
    aR = ppmx_face(q5[1], q5[2], q5[3], q5[4]);
    ppmx_limit(q5[0], q5[1], q5[2], q5[3], q5[4], aL, aR);
  } else {
    wenoz_cell(q5, aL, aR);
  }
}

}  // namespace chq
