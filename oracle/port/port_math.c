/* Oracle (test infrastructure): point functions of the path restated in C — face
 * reconstruction (src/recon.hpp), the HLLE / HLLD / LHLLD Riemann solvers (src/riemann.hpp)
 * and the primitive-variable MHD eigensystem (src/eigen_mhd.hpp). Operation order follows
 * the reference exactly (compiled with -ffp-contract=off), so results are bitwise equal. */
#include <math.h>
#include <string.h>
#include "port.h"
#include "port_internal.h"

static double sq(double x) { return x * x; }
double port_sign(double x) { return (x > 0.0) ? 1.0 : ((x < 0.0) ? -1.0 : 0.0); }

/* src/recon.hpp:14-18 */
static double slope_vl(double qm, double q0, double qp) {
  double dl = q0 - qm, dr = qp - q0, d2 = dl * dr;
  return (d2 > 0.0) ? 2.0 * d2 / (dl + dr) : 0.0;
}
/* src/recon.hpp:21-27 */
static double slope_mc(double qm, double q0, double qp) {
  double dl = q0 - qm, dr = qp - q0, dc, lim;
  if (dl * dr <= 0.0) return 0.0;
  dc = 0.5 * (qp - qm);
  lim = 2.0 * fmin(fabs(dl), fabs(dr));
  return port_sign(dc) * fmin(fabs(dc), lim);
}
/* src/recon.hpp:42-44 */
static double face_cw(double qa, double qb, double dqa, double dqb) { return 0.5 * (qa + qb) + (dqa - dqb) / 6.0; }
/* src/recon.hpp:47-57 */
static void limit_cw(double q, double *qL, double *qR) {
  double d, c, d2o6;
  if ((*qR - q) * (q - *qL) <= 0.0) { *qL = q; *qR = q; return; }
  d = *qR - *qL;
  c = q - 0.5 * (*qL + *qR);
  d2o6 = d * d / 6.0;
  if (d * c > d2o6) *qL = 3.0 * q - 2.0 * *qR;
  else if (d * c < -d2o6) *qR = 3.0 * q - 2.0 * *qL;
}
/* src/recon.hpp:85-100 */
static double face_x(double qm1, double q0, double qp1, double qp2) {
  const double C = 1.25;
  double qf = (7.0 / 12.0) * (q0 + qp1) - (1.0 / 12.0) * (qm1 + qp2);
  if ((qf - q0) * (qp1 - qf) < 0.0) {
    double d2 = 3.0 * ((q0 + qp1) - 2.0 * qf);
    double d2l = (qm1 + qp1) - 2.0 * q0, d2r = (q0 + qp2) - 2.0 * qp1, d2lim = 0.0;
    if (d2 * d2l > 0.0 && d2 * d2r > 0.0) d2lim = port_sign(d2) * fmin(fmin(C * fabs(d2l), C * fabs(d2r)), fabs(d2));
    qf = 0.5 * (q0 + qp1) - d2lim / 6.0;
  }
  return qf;
}
/* src/recon.hpp:104-127 */
static void limit_x(double qm2, double qm1, double q, double qp1, double qp2, double *qL, double *qR) {
  const double C = 1.25;
  double dqm = q - *qL, dqp = *qR - q;
  int ext = (dqm * dqp <= 0.0) || ((qp1 - q) * (q - qm1) <= 0.0);
  if (ext) {
    double d2 = 6.0 * ((*qL + *qR) - 2.0 * q);
    double d2c = (qm1 + qp1) - 2.0 * q, d2l = (qm2 + q) - 2.0 * qm1, d2r = (q + qp2) - 2.0 * qp1;
    double d2lim = 0.0, rho;
    if (d2 * d2c > 0.0 && d2 * d2l > 0.0 && d2 * d2r > 0.0)
      d2lim = port_sign(d2) * fmin(fmin(C * fabs(d2l), C * fabs(d2r)), fmin(C * fabs(d2c), fabs(d2)));
    rho = (fabs(d2) > 1e-12 * (fabs(q) + fabs(qm1) + fabs(qp1)) + 1e-300) ? d2lim / d2 : 0.0;
    if (rho < 1.0 - 1e-12) { *qL = q - rho * dqm; *qR = q + rho * dqp; }
  } else {
    if (fabs(dqm) >= 2.0 * fabs(dqp)) *qL = q - 2.0 * dqp;
    if (fabs(dqp) >= 2.0 * fabs(dqm)) *qR = q + 2.0 * dqm;
  }
}
/* src/recon.hpp:144-164 */
static double weno_z(double fm2, double fm1, double f0, double fp1, double fp2) {
  const double eps = 1e-36, c13 = 13.0 / 12.0;
  double b0 = c13 * sq((fm2 + f0) - 2.0 * fm1) + 0.25 * sq((3.0 * f0 + fm2) - 4.0 * fm1);
  double b1 = c13 * sq((fm1 + fp1) - 2.0 * f0) + 0.25 * sq(fm1 - fp1);
  double b2 = c13 * sq((fp2 + f0) - 2.0 * fp1) + 0.25 * sq((3.0 * f0 + fp2) - 4.0 * fp1);
  double tau = fabs(b0 - b2);
  double a0 = 0.1 * (1.0 + tau / (b0 + eps)), a1 = 0.6 * (1.0 + tau / (b1 + eps)), a2 = 0.3 * (1.0 + tau / (b2 + eps));
  double inv = 1.0 / (a0 + a1 + a2);
  double q0 = (2.0 * fm2 - 7.0 * fm1 + 11.0 * f0) / 6.0;
  double q1 = (-fm1 + 5.0 * f0 + 2.0 * fp1) / 6.0;
  double q2 = (2.0 * f0 + 5.0 * fp1 - fp2) / 6.0;
  return inv * (a0 * q0 + a1 * q1 + a2 * q2);
}

/* per face from the 6-cell stencil q[0..5] = q_{i-3..i+2}: src/recon.hpp:29-171, 189-196 */
void port_recon(int scheme, const double q[6], double *ql, double *qr) {
  switch (scheme) {
    case 0: *ql = q[2]; *qr = q[3]; return;
    case 1:
      *ql = q[2] + 0.5 * slope_vl(q[1], q[2], q[3]);
      *qr = q[3] - 0.5 * slope_vl(q[2], q[3], q[4]);
      return;
    case 2: {
      double d1 = slope_mc(q[0], q[1], q[2]), d2 = slope_mc(q[1], q[2], q[3]);
      double d3 = slope_mc(q[2], q[3], q[4]), d4 = slope_mc(q[3], q[4], q[5]);
      double a = face_cw(q[1], q[2], d1, d2), b = face_cw(q[2], q[3], d2, d3), c = face_cw(q[3], q[4], d3, d4);
      double aL = a, aR = b, bL = b, bR = c;
      limit_cw(q[2], &aL, &aR);
      limit_cw(q[3], &bL, &bR);
      *ql = aR;
      *qr = bL;
      return;
    }
    case 4: {
      double a = face_x(q[0], q[1], q[2], q[3]), b = face_x(q[1], q[2], q[3], q[4]), c = face_x(q[2], q[3], q[4], q[5]);
      double aL = a, aR = b, bL = b, bR = c;
      limit_x(q[0], q[1], q[2], q[3], q[4], &aL, &aR);
      limit_x(q[1], q[2], q[3], q[4], q[5], &bL, &bR);
      *ql = aR;
      *qr = bL;
      return;
    }
    default:
      *ql = weno_z(q[0], q[1], q[2], q[3], q[4]);
      *qr = weno_z(q[5], q[4], q[3], q[2], q[1]);
  }
}

/* src/recon.hpp:179-187 */
double port_flattening(const double p[5], double um1, double up1) {
  double dp = p[3] - p[1], dp2 = p[4] - p[0], pmin = fmin(p[1], p[3]), ratio;
  if (!((fabs(dp) > 0.33 * pmin) && (um1 > up1))) return 0.0;
  ratio = (fabs(dp2) > 1e-300) ? dp / dp2 : 0.0;
  return fmin(1.0, fmax(0.0, 10.0 * (ratio - 0.75)));
}

/* ---- Riemann solvers: state s = (d, u, v, w, p, by, bz) ---- */
/* src/riemann.hpp:19-25 */
double port_cfast(const double *s, double bn, double gamma) {
  double bsq = bn * bn + s[5] * s[5] + s[6] * s[6], gp = gamma * s[4];
  double a = (gp + bsq) / s[0];
  double disc = a * a - 4.0 * gp * bn * bn / (s[0] * s[0]);
  return sqrt(0.5 * (a + sqrt(fmax(disc, 0.0))));
}
/* src/riemann.hpp:27-40 */
void port_pflux(const double *s, double bn, double gm1, double *e, double *pt, double f[7]) {
  double vsq = s[1] * s[1] + s[2] * s[2] + s[3] * s[3], bsq = bn * bn + s[5] * s[5] + s[6] * s[6], vb;
  *e = s[4] / gm1 + 0.5 * (s[0] * vsq + bsq);
  *pt = s[4] + 0.5 * bsq;
  vb = s[1] * bn + s[2] * s[5] + s[3] * s[6];
  f[0] = s[0] * s[1];
  f[1] = s[0] * s[1] * s[1] + *pt - bn * bn;
  f[2] = s[0] * s[1] * s[2] - bn * s[5];
  f[3] = s[0] * s[1] * s[3] - bn * s[6];
  f[4] = (*e + *pt) * s[1] - bn * vb;
  f[5] = s[5] * s[1] - bn * s[2];
  f[6] = s[6] * s[1] - bn * s[3];
}
/* src/riemann.hpp:44-51 */
double port_cflow(const double *s, double bn) {
  double vsq = s[1] * s[1] + s[2] * s[2] + s[3] * s[3];
  double casq = (bn * bn + s[5] * s[5] + s[6] * s[6]) / s[0], caxsq = bn * bn / s[0];
  double a = casq + vsq, disc = a * a - 4.0 * vsq * caxsq;
  return sqrt(0.5 * (a + sqrt(fmax(disc, 0.0))));
}
/* src/riemann.hpp:55-68 */
static void hlle(const double *L, const double *R, double bn, double gamma, double f[7]) {
  double fl[7], fr[7], el, er, ptl, ptr, cl, cr, sl, sr, inv;
  double ul[7], ur[7];
  int n;
  port_pflux(L, bn, gamma - 1.0, &el, &ptl, fl);
  port_pflux(R, bn, gamma - 1.0, &er, &ptr, fr);
  cl = port_cfast(L, bn, gamma);
  cr = port_cfast(R, bn, gamma);
  sl = fmin(L[1] - cl, R[1] - cr);
  sr = fmax(L[1] + cl, R[1] + cr);
  if (sl >= 0.0) { memcpy(f, fl, sizeof(fl)); return; }
  if (sr <= 0.0) { memcpy(f, fr, sizeof(fr)); return; }
  ul[0] = L[0]; ul[1] = L[0] * L[1]; ul[2] = L[0] * L[2]; ul[3] = L[0] * L[3]; ul[4] = el; ul[5] = L[5]; ul[6] = L[6];
  ur[0] = R[0]; ur[1] = R[0] * R[1]; ur[2] = R[0] * R[2]; ur[3] = R[0] * R[3]; ur[4] = er; ur[5] = R[5]; ur[6] = R[6];
  inv = 1.0 / (sr - sl);
  for (n = 0; n < 7; ++n) f[n] = (sr * fl[n] - sl * fr[n] + sl * sr * (ur[n] - ul[n])) * inv;
}
/* src/riemann.hpp:81-91 */
static void sflux(double d, double sm, double v, double w, double e, double by, double bz, double bn, double pts,
                  double f[7]) {
  double vb = (sm * bn + v * by) + w * bz;
  f[0] = d * sm;
  f[1] = (d * sm) * sm + (pts - bn * bn);
  f[2] = (d * sm) * v - bn * by;
  f[3] = (d * sm) * w - bn * bz;
  f[4] = (e + pts) * sm - bn * vb;
  f[5] = by * sm - bn * v;
  f[6] = bz * sm - bn * w;
}
/* src/riemann.hpp:96-234 */
static void hlld(const double *L, const double *R, double bn, double gamma, double f[7], double theta, double phi,
                 int lh) {
  double fl[7], fr[7], el, er, ptl, ptr, cl, cr, sl, sr;
  double bnsq, slml, srmr, dsl, dsr, iden, sm, pts, slms, dls, srms, drs;
  double vls, wls, byls, bzls, vrs, wrs, byrs, bzrs, vbl, vbls, vbr, vbrs, els, ers;
  double sqdl, sqdr, abn, sls, srs, fls[7], frs[7];
  int n;
  port_pflux(L, bn, gamma - 1.0, &el, &ptl, fl);
  port_pflux(R, bn, gamma - 1.0, &er, &ptr, fr);
  cl = port_cfast(L, bn, gamma);
  cr = port_cfast(R, bn, gamma);
  if (lh) {
    double cmax = fmax(cl, cr);
    sl = fmin(0.0, fmin(L[1], R[1]) - cmax);
    sr = fmax(0.0, fmax(L[1], R[1]) + cmax);
  } else {
    sl = fmin(L[1] - cl, R[1] - cr);
    sr = fmax(L[1] + cl, R[1] + cr);
  }
  if (sl >= 0.0) { memcpy(f, fl, sizeof(fl)); return; }
  if (sr <= 0.0) { memcpy(f, fr, sizeof(fr)); return; }
  bnsq = bn * bn;
  slml = sl - L[1];
  srmr = sr - R[1];
  dsl = L[0] * slml;
  dsr = R[0] * srmr;
  iden = 1.0 / (dsr - dsl);
  sm = ((dsr * R[1] - dsl * L[1]) + theta * (ptl - ptr)) * iden;
  pts = ((dsr * ptl - dsl * ptr) + (phi * ((L[0] * R[0]) * (srmr * slml))) * (R[1] - L[1])) * iden;
  slms = sl - sm;
  dls = dsl / slms;
  {
    double den = (L[0] * slml) * slms - bnsq, scale = fabs((L[0] * slml) * slms) + bnsq;
    if (fabs(den) <= 1e-12 * scale + 1e-300) { vls = L[2]; wls = L[3]; byls = L[5]; bzls = L[6]; }
    else {
      double nv = (bn * (sm - L[1])) / den, nb;
      vls = L[2] - L[5] * nv;
      wls = L[3] - L[6] * nv;
      nb = ((L[0] * slml) * slml - bnsq) / den;
      byls = L[5] * nb;
      bzls = L[6] * nb;
    }
  }
  vbl = (L[1] * bn + L[2] * L[5]) + L[3] * L[6];
  vbls = (sm * bn + vls * byls) + wls * bzls;
  els = (((slml * el - ptl * L[1]) + pts * sm) + bn * (vbl - vbls)) / slms;
  srms = sr - sm;
  drs = dsr / srms;
  {
    double den = (R[0] * srmr) * srms - bnsq, scale = fabs((R[0] * srmr) * srms) + bnsq;
    if (fabs(den) <= 1e-12 * scale + 1e-300) { vrs = R[2]; wrs = R[3]; byrs = R[5]; bzrs = R[6]; }
    else {
      double nv = (bn * (sm - R[1])) / den, nb;
      vrs = R[2] - R[5] * nv;
      wrs = R[3] - R[6] * nv;
      nb = ((R[0] * srmr) * srmr - bnsq) / den;
      byrs = R[5] * nb;
      bzrs = R[6] * nb;
    }
  }
  vbr = (R[1] * bn + R[2] * R[5]) + R[3] * R[6];
  vbrs = (sm * bn + vrs * byrs) + wrs * bzrs;
  ers = (((srmr * er - ptr * R[1]) + pts * sm) + bn * (vbr - vbrs)) / srms;
  sqdl = sqrt(dls);
  sqdr = sqrt(drs);
  abn = fabs(bn);
  sls = sm - abn / sqdl;
  srs = sm + abn / sqdr;
  {
    double uls[7] = {dls, dls * sm, dls * vls, dls * wls, els, byls, bzls};
    double urs[7] = {drs, drs * sm, drs * vrs, drs * wrs, ers, byrs, bzrs};
    double ul[7] = {L[0], L[0] * L[1], L[0] * L[2], L[0] * L[3], el, L[5], L[6]};
    double ur[7] = {R[0], R[0] * R[1], R[0] * R[2], R[0] * R[3], er, R[5], R[6]};
    double sg, inv, vss, wss, byss, bzss, vbss, elss, erss, flss[7], frss[7];
    if (lh) {
      sflux(dls, sm, vls, wls, els, byls, bzls, bn, pts, fls);
      sflux(drs, sm, vrs, wrs, ers, byrs, bzrs, bn, pts, frs);
    } else {
      for (n = 0; n < 7; ++n) { fls[n] = fl[n] + sl * (uls[n] - ul[n]); frs[n] = fr[n] + sr * (urs[n] - ur[n]); }
    }
    if (sls > 0.0) { memcpy(f, fls, sizeof(fls)); return; }
    if (srs < 0.0) { memcpy(f, frs, sizeof(frs)); return; }
    if (bnsq <= 1e-12 * (ptl + ptr)) {
      for (n = 0; n < 7; ++n) f[n] = (sm > 0.0) ? fls[n] : (sm < 0.0) ? frs[n] : 0.5 * (fls[n] + frs[n]);
      return;
    }
    sg = port_sign(bn);
    inv = 1.0 / (sqdl + sqdr);
    vss = ((sqdl * vls + sqdr * vrs) + (byrs - byls) * sg) * inv;
    wss = ((sqdl * wls + sqdr * wrs) + (bzrs - bzls) * sg) * inv;
    byss = ((sqdl * byrs + sqdr * byls) + (sqdl * sqdr) * ((vrs - vls) * sg)) * inv;
    bzss = ((sqdl * bzrs + sqdr * bzls) + (sqdl * sqdr) * ((wrs - wls) * sg)) * inv;
    vbss = (sm * bn + vss * byss) + wss * bzss;
    elss = els - sqdl * ((vbls - vbss) * sg);
    erss = ers + sqdr * ((vbrs - vbss) * sg);
    if (lh) {
      sflux(dls, sm, vss, wss, elss, byss, bzss, bn, pts, flss);
      sflux(drs, sm, vss, wss, erss, byss, bzss, bn, pts, frss);
    } else {
      double ulss[7] = {dls, dls * sm, dls * vss, dls * wss, elss, byss, bzss};
      double urss[7] = {drs, drs * sm, drs * vss, drs * wss, erss, byss, bzss};
      for (n = 0; n < 7; ++n) {
        flss[n] = fls[n] + sls * (ulss[n] - uls[n]);
        frss[n] = frs[n] + srs * (urss[n] - urs[n]);
      }
    }
    for (n = 0; n < 7; ++n) f[n] = (sm > 0.0) ? flss[n] : (sm < 0.0) ? frss[n] : 0.5 * (flss[n] + frss[n]);
  }
}

/* solver 0 HLLE, 1 HLLD, 2 HLLD with (theta, phi) and the LHLLD signal speeds */
void port_riemann(int solver, const double L[7], const double R[7], double bn, double gamma, double theta, double phi,
                  double f[7]) {
  if (solver == 0) hlle(L, R, bn, gamma, f);
  else if (solver == 1) hlld(L, R, bn, gamma, f, 1.0, 1.0, 0);
  else hlld(L, R, bn, gamma, f, theta, phi, 1);
}

/* src/eigen_mhd.hpp:14-82; w8 = (d, u, v, w, p, by, bz, bx); row-major 7x7 outputs */
void port_eigen(const double w8[8], double gamma, double Lm[49], double Rm[49]) {
  double d = w8[0], p = w8[4], by = w8[5], bz = w8[6], bx = w8[7];
  double sqrtd = sqrt(d), isqrtd = 1.0 / sqrtd, asq = gamma * p / d, a = sqrt(asq), casq = bx * bx / d;
  double bperpsq = by * by + bz * bz, ctsq = bperpsq / d, tsum = asq + casq + ctsq, tdif = asq + ctsq - casq;
  double disc = sqrt(fmax(tdif * tdif + 4.0 * ctsq * casq, 0.0));
  double cfsq = 0.5 * (tsum + disc), cssq = fmax(0.5 * (tsum - disc), 0.0), cf = sqrt(cfsq), cs = sqrt(cssq);
  double alf, als, bety, betz, s, cff, css, qf, qs, af, as, nrm, ncff, ncss, nqf, nqs, naf, nas;
#define R_(i, j) Rm[(i) * 7 + (j)]
#define L_(i, j) Lm[(i) * 7 + (j)]
  if (cfsq - cssq <= 1e-12 * cfsq) { alf = 1.0; als = 0.0; }
  else if (ctsq <= 1e-12 * (asq + casq)) {
    if (asq >= casq) { alf = 1.0; als = 0.0; } else { alf = 0.0; als = 1.0; }
  } else if (asq - cssq <= 0.0) { alf = 0.0; als = 1.0; }
  else if (cfsq - asq <= 0.0) { alf = 1.0; als = 0.0; }
  else { alf = sqrt((asq - cssq) / (cfsq - cssq)); als = sqrt((cfsq - asq) / (cfsq - cssq)); }
  if (bperpsq > 0.0) { double ib = 1.0 / sqrt(bperpsq); bety = by * ib; betz = bz * ib; }
  else { bety = 1.0 / sqrt(2.0); betz = bety; }
  s = (bx >= 0.0) ? 1.0 : -1.0;
  cff = cf * alf; css = cs * als; qf = cff * s; qs = css * s; af = a * alf * sqrtd; as = a * als * sqrtd;
  memset(Lm, 0, 49 * sizeof(double));
  memset(Rm, 0, 49 * sizeof(double));
  R_(0, 0) = d * alf; R_(0, 2) = d * als; R_(0, 3) = 1.0; R_(0, 4) = d * als; R_(0, 6) = d * alf;
  R_(1, 0) = -cff; R_(1, 2) = -css; R_(1, 4) = css; R_(1, 6) = cff;
  R_(2, 0) = qs * bety; R_(2, 1) = -betz; R_(2, 2) = -qf * bety; R_(2, 4) = qf * bety; R_(2, 5) = betz; R_(2, 6) = -qs * bety;
  R_(3, 0) = qs * betz; R_(3, 1) = bety; R_(3, 2) = -qf * betz; R_(3, 4) = qf * betz; R_(3, 5) = -bety; R_(3, 6) = -qs * betz;
  R_(4, 0) = d * alf * asq; R_(4, 2) = d * als * asq; R_(4, 4) = d * als * asq; R_(4, 6) = d * alf * asq;
  R_(5, 0) = as * bety; R_(5, 1) = -betz * s * sqrtd; R_(5, 2) = -af * bety; R_(5, 4) = -af * bety;
  R_(5, 5) = -betz * s * sqrtd; R_(5, 6) = as * bety;
  R_(6, 0) = as * betz; R_(6, 1) = bety * s * sqrtd; R_(6, 2) = -af * betz; R_(6, 4) = -af * betz;
  R_(6, 5) = bety * s * sqrtd; R_(6, 6) = as * betz;
  nrm = 0.5 / asq; ncff = nrm * cff; ncss = nrm * css; nqf = nrm * qf; nqs = nrm * qs;
  naf = nrm * af / d; nas = nrm * as / d;
  L_(0, 1) = -ncff; L_(0, 2) = nqs * bety; L_(0, 3) = nqs * betz; L_(0, 4) = nrm * alf / d; L_(0, 5) = nas * bety;
  L_(0, 6) = nas * betz;
  L_(1, 2) = -0.5 * betz; L_(1, 3) = 0.5 * bety; L_(1, 5) = -0.5 * betz * s * isqrtd; L_(1, 6) = 0.5 * bety * s * isqrtd;
  L_(2, 1) = -ncss; L_(2, 2) = -nqf * bety; L_(2, 3) = -nqf * betz; L_(2, 4) = nrm * als / d; L_(2, 5) = -naf * bety;
  L_(2, 6) = -naf * betz;
  L_(3, 0) = 1.0; L_(3, 4) = -1.0 / asq;
  L_(4, 1) = ncss; L_(4, 2) = nqf * bety; L_(4, 3) = nqf * betz; L_(4, 4) = nrm * als / d; L_(4, 5) = -naf * bety;
  L_(4, 6) = -naf * betz;
  L_(5, 2) = 0.5 * betz; L_(5, 3) = -0.5 * bety; L_(5, 5) = -0.5 * betz * s * isqrtd; L_(5, 6) = 0.5 * bety * s * isqrtd;
  L_(6, 1) = ncff; L_(6, 2) = -nqs * bety; L_(6, 3) = -nqs * betz; L_(6, 4) = nrm * alf / d; L_(6, 5) = nas * bety;
  L_(6, 6) = nas * betz;
#undef R_
#undef L_
}
