// chasqui_b200 — ideal-MHD Riemann solvers on one face, evaluated entirely in registers.
//
// States are in the face frame: u normal velocity, (v, w) transverse velocities, bn the
// face-normal field, (by, bz) transverse fields; magnetic pressure B^2/2.
//   HLLE  : Einfeldt (1988)                       (src/riemann.hpp:55-68)
//   HLLD  : Miyoshi & Kusano, JCP 208, 315 (2005)  (src/riemann.hpp:96-234)
//   LHLLD : HLLD with the shock-stability / low-dissipation factors and signal speeds of
//           Minoshima & Miyoshi (2021), star fluxes from the star states.
// The left and right halves are exact mirror copies and multi-term sums are grouped in
// mirror-image pairs, as in the reference, so that reflected inputs give bitwise-reflected
// fluxes (the reference's symmetry_test contract). Flux slots follow the reference:
// 0 mass, 1 normal momentum, 2/3 transverse momenta, 4 energy, 5/6 transverse fields.
#pragma once
#include "chq_common.cuh"

namespace chq {

enum : int { FD = 0, FMU = 1, FMV = 2, FMW = 3, FEN = 4, FBY = 5, FBZ = 6, NFLX = 7 };

template <class T> struct MState { T d, u, v, w, p, by, bz; };

// fast magnetosonic speed (src/riemann.hpp:19-25)
template <class T> CHQ_HD T fast_speed(const MState<T> &s, T bn, T gamma) {
  const T bsq = bn * bn + s.by * s.by + s.bz * s.bz;
  const T gp = gamma * s.p;
  const T a = (gp + bsq) / s.d;
  const T disc = a * a - divz(T(4) * gp * bn * bn, s.d * s.d);
  return sqrt_(T(0.5) * (a + sqrt_(fmax_(disc, T(0)))));
}

// physical flux, total energy and total pressure of a state (src/riemann.hpp:27-40)
template <class T> CHQ_HD void phys_flux(const MState<T> &s, T bn, T gm1, T &e, T &pt, T f[NFLX]) {
  const T vsq = s.u * s.u + s.v * s.v + s.w * s.w;
  const T bsq = bn * bn + s.by * s.by + s.bz * s.bz;
  e = s.p / gm1 + T(0.5) * (s.d * vsq + bsq);
  pt = s.p + T(0.5) * bsq;
  const T vdotb = s.u * bn + s.v * s.by + s.w * s.bz;
  f[FD] = s.d * s.u;
  f[FMU] = s.d * s.u * s.u + pt - bn * bn;
  f[FMV] = s.d * s.u * s.v - bn * s.by;
  f[FMW] = s.d * s.u * s.w - bn * s.bz;
  f[FEN] = (e + pt) * s.u - bn * vdotb;
  f[FBY] = s.by * s.u - bn * s.v;
  f[FBZ] = s.bz * s.u - bn * s.w;
}

// total energy and total pressure alone (the scalars phys_flux computes first)
template <class T> CHQ_HD void energy_ptot(const MState<T> &s, T bn, T gm1, T &e, T &pt) {
  const T vsq = s.u * s.u + s.v * s.v + s.w * s.w;
  const T bsq = bn * bn + s.by * s.by + s.bz * s.bz;
  e = s.p / gm1 + T(0.5) * (s.d * vsq + bsq);
  pt = s.p + T(0.5) * bsq;
}

// the flux vector of phys_flux from already computed e and pt
template <class T> CHQ_HD void flux_from(const MState<T> &s, T bn, T e, T pt, T f[NFLX]) {
  const T vdotb = s.u * bn + s.v * s.by + s.w * s.bz;
  f[FD] = s.d * s.u;
  f[FMU] = s.d * s.u * s.u + pt - bn * bn;
  f[FMV] = s.d * s.u * s.v - bn * s.by;
  f[FMW] = s.d * s.u * s.w - bn * s.bz;
  f[FEN] = (e + pt) * s.u - bn * vdotb;
  f[FBY] = s.by * s.u - bn * s.v;
  f[FBZ] = s.bz * s.u - bn * s.w;
}

// modified fast speed with the sound speed replaced by |v| (src/riemann.hpp:44-51)
template <class T> CHQ_HD T flow_speed_u(const MState<T> &s, T bn) {
  const T vsq = s.u * s.u + s.v * s.v + s.w * s.w;
  const T casq = divz(bn * bn + s.by * s.by + s.bz * s.bz, s.d);
  const T caxsq = divz(bn * bn, s.d);
  const T a = casq + vsq;
  const T disc = a * a - T(4) * vsq * caxsq;
  return sqrt_(T(0.5) * (a + sqrt_(fmax_(disc, T(0)))));
}

template <class T> CHQ_HD void hlle(const MState<T> &L, const MState<T> &R, T bn, T gamma, T gm1, T f[NFLX]) {
  // speeds first; the flux vectors are built only for the region that is selected
  const T cl = fast_speed(L, bn, gamma), cr = fast_speed(R, bn, gamma);
  const T sl = fmin_(L.u - cl, R.u - cr);
  const T sr = fmax_(L.u + cl, R.u + cr);
  T el, er, ptl, ptr;
  energy_ptot(L, bn, gm1, el, ptl);
  if (sl >= T(0)) {
    flux_from(L, bn, el, ptl, f);
    return;
  }
  energy_ptot(R, bn, gm1, er, ptr);
  if (sr <= T(0)) {
    flux_from(R, bn, er, ptr, f);
    return;
  }
  T fl[NFLX], fr[NFLX];
  flux_from(L, bn, el, ptl, fl);
  flux_from(R, bn, er, ptr, fr);
  const T ul[NFLX] = {L.d, L.d * L.u, L.d * L.v, L.d * L.w, el, L.by, L.bz};
  const T ur[NFLX] = {R.d, R.d * R.u, R.d * R.v, R.d * R.w, er, R.by, R.bz};
  const T inv = T(1) / (sr - sl);
#pragma unroll
  for (int n = 0; n < NFLX; ++n) f[n] = (sr * fl[n] - sl * fr[n] + sl * sr * (ur[n] - ul[n])) * inv;
}

// flux of an intermediate state with intermediate total pressure pts (src/riemann.hpp:81-91)
template <class T>
CHQ_HD void star_flux(T d, T sm, T v, T w, T e, T by, T bz, T bn, T pts, T f[NFLX]) {
  const T vdotb = (sm * bn + v * by) + w * bz;
  f[FD] = d * sm;
  f[FMU] = (d * sm) * sm + (pts - bn * bn);
  f[FMV] = (d * sm) * v - bn * by;
  f[FMW] = (d * sm) * w - bn * bz;
  f[FEN] = (e + pts) * sm - bn * vdotb;
  f[FBY] = by * sm - bn * v;
  f[FBZ] = bz * sm - bn * w;
}

// One side's single-star transverse velocity and field (MK05 eqs. 43-47); the left and
// right calls run the identical expression sequence.
template <class T>
CHQ_HD void star_side(const MState<T> &S, T slm, T sms, T sm, T bn, T bnsq, T &vs, T &ws, T &bys, T &bzs) {
  const T den = (S.d * slm) * sms - bnsq;
  const T scale = fabs_((S.d * slm) * sms) + bnsq;
  if (fabs_(den) <= T(1e-12) * scale + Tiny<T>::v) {
    vs = S.v;
    ws = S.w;
    bys = S.by;
    bzs = S.bz;
  } else {
    const T num_v = divz(bn * (sm - S.u), den);
    vs = S.v - S.by * num_v;
    ws = S.w - S.bz * num_v;
    const T num_b = ((S.d * slm) * slm - bnsq) / den;
    bys = S.by * num_b;
    bzs = S.bz * num_b;
  }
}

// single-star flux of one side: F + S (U* - U) (HLLD) or the star state's own flux (LHLLD)
template <bool LHLLD, class T>
CHQ_HD void side_star_flux(const MState<T> &S, T bn, T e, T pt, T s, T ds, T sm, T vs, T ws, T bys, T bzs, T es,
                           T pts, T f[NFLX]) {
  if constexpr (LHLLD) {
    star_flux(ds, sm, vs, ws, es, bys, bzs, bn, pts, f);
  } else {
    T fs[NFLX];
    flux_from(S, bn, e, pt, fs);
    const T us[NFLX] = {ds, ds * sm, ds * vs, ds * ws, es, bys, bzs};
    const T u[NFLX] = {S.d, S.d * S.u, S.d * S.v, S.d * S.w, e, S.by, S.bz};
#pragma unroll
    for (int n = 0; n < NFLX; ++n) f[n] = fs[n] + s * (us[n] - u[n]);
  }
}

// double-star flux of one side: F* + S* (U** - U*) (HLLD) or the ** state's own flux (LHLLD)
template <bool LHLLD, class T>
CHQ_HD void side_dstar_flux(const MState<T> &S, T bn, T e, T pt, T s, T ds, T sm, T vs, T ws, T bys, T bzs, T es,
                            T pts, T ss, T vss, T wss, T byss, T bzss, T ess, T f[NFLX]) {
  if constexpr (LHLLD) {
    star_flux(ds, sm, vss, wss, ess, byss, bzss, bn, pts, f);
  } else {
    T fs[NFLX];
    side_star_flux<false>(S, bn, e, pt, s, ds, sm, vs, ws, bys, bzs, es, pts, fs);
    const T us[NFLX] = {ds, ds * sm, ds * vs, ds * ws, es, bys, bzs};
    const T uss[NFLX] = {ds, ds * sm, ds * vss, ds * wss, ess, byss, bzss};
#pragma unroll
    for (int n = 0; n < NFLX; ++n) f[n] = fs[n] + ss * (uss[n] - us[n]);
  }
}

// Single-star (single) or double-star flux of the side `left` selects. The operands of the
// two sides are picked value by value, then one evaluation runs with exactly the expression
// sequence of side_star_flux / side_dstar_flux, so the result is bitwise the flux of that
// side. The left side's double-star energy is E*_L - sqrt(D*_L) (v*_L.B*_L - v**.B**) sgn(bn),
// the right side's E*_R + (the mirror term); x - t and x + (-t) are the same IEEE operation.
template <bool LHLLD, class T>
CHQ_HD void side_region_flux(bool left, bool single, const MState<T> &L, const MState<T> &R, T bn, T el, T er, T ptl,
                             T ptr, T sl, T sr, T dls, T drs, T sm, T vls, T vrs, T wls, T wrs, T byls, T byrs, T bzls,
                             T bzrs, T els, T ers, T pts, T sls, T srs, T sqdl, T sqdr, T vdotb_ls, T vdotb_rs, T sg,
                             T vss, T wss, T byss, T bzss, T vdotb_ss, T f[NFLX]) {
  const T ds = left ? dls : drs, vs = left ? vls : vrs, ws = left ? wls : wrs;
  const T bys = left ? byls : byrs, bzs = left ? bzls : bzrs, es = left ? els : ers;
  if constexpr (LHLLD) {
    if (single) {
      star_flux(ds, sm, vs, ws, es, bys, bzs, bn, pts, f);
    } else {
      const T t = (left ? sqdl : sqdr) * (((left ? vdotb_ls : vdotb_rs) - vdotb_ss) * sg);
      const T ess = es + (left ? -t : t);
      star_flux(ds, sm, vss, wss, ess, byss, bzss, bn, pts, f);
    }
  } else {
    const MState<T> S{left ? L.d : R.d, left ? L.u : R.u, left ? L.v : R.v, left ? L.w : R.w,
                      left ? L.p : R.p, left ? L.by : R.by, left ? L.bz : R.bz};
    const T e = left ? el : er, pt = left ? ptl : ptr, s = left ? sl : sr;
    side_star_flux<false>(S, bn, e, pt, s, ds, sm, vs, ws, bys, bzs, es, pts, f);
    if (!single) {
      const T t = (left ? sqdl : sqdr) * (((left ? vdotb_ls : vdotb_rs) - vdotb_ss) * sg);
      const T ess = es + (left ? -t : t);
      const T ss = left ? sls : srs;
      const T us[NFLX] = {ds, ds * sm, ds * vs, ds * ws, es, bys, bzs};
      const T uss[NFLX] = {ds, ds * sm, ds * vss, ds * wss, ess, byss, bzss};
#pragma unroll
      for (int n = 0; n < NFLX; ++n) f[n] = f[n] + ss * (uss[n] - us[n]);
    }
  }
}

template <bool LHLLD, class T>
CHQ_HD void hlld(const MState<T> &L, const MState<T> &R, T bn, T gamma, T gm1, T f[NFLX], T theta, T phi) {
  // speeds and the scalars of both sides first; flux vectors only for the selected region
  T el, er, ptl, ptr;
  energy_ptot(L, bn, gm1, el, ptl);
  energy_ptot(R, bn, gm1, er, ptr);
  const T cl = fast_speed(L, bn, gamma), cr = fast_speed(R, bn, gamma);
  T sl, sr;
  if constexpr (LHLLD) {
    const T cmax = fmax_(cl, cr);
    sl = fmin_(T(0), fmin_(L.u, R.u) - cmax);
    sr = fmax_(T(0), fmax_(L.u, R.u) + cmax);
  } else {
    sl = fmin_(L.u - cl, R.u - cr);
    sr = fmax_(L.u + cl, R.u + cr);
  }
  if (sl >= T(0)) {
    flux_from(L, bn, el, ptl, f);
    return;
  }
  if (sr <= T(0)) {
    flux_from(R, bn, er, ptr, f);
    return;
  }
  const T bnsq = bn * bn;
  const T slml = sl - L.u;
  const T srmr = sr - R.u;
  const T dsl = L.d * slml;
  const T dsr = R.d * srmr;
  const T iden = T(1) / (dsr - dsl);
  // contact speed and star total pressure (MK05 eqs. 38, 41)
  const T sm = ((dsr * R.u - dsl * L.u) + theta * (ptl - ptr)) * iden;
  const T pts = ((dsr * ptl - dsl * ptr) + (phi * ((L.d * R.d) * (srmr * slml))) * (R.u - L.u)) * iden;

  const T slms = sl - sm;
  const T dls = dsl / slms;
  T vls, wls, byls, bzls;
  star_side(L, slml, slms, sm, bn, bnsq, vls, wls, byls, bzls);
  const T vdotb_l = (L.u * bn + L.v * L.by) + L.w * L.bz;
  const T vdotb_ls = (sm * bn + vls * byls) + wls * bzls;
  const T els = (((slml * el - ptl * L.u) + pts * sm) + bn * (vdotb_l - vdotb_ls)) / slms;

  const T srms = sr - sm;
  const T drs = dsr / srms;
  T vrs, wrs, byrs, bzrs;
  star_side(R, srmr, srms, sm, bn, bnsq, vrs, wrs, byrs, bzrs);
  const T vdotb_r = (R.u * bn + R.v * R.by) + R.w * R.bz;
  const T vdotb_rs = (sm * bn + vrs * byrs) + wrs * bzrs;
  const T ers = (((srmr * er - ptr * R.u) + pts * sm) + bn * (vdotb_r - vdotb_rs)) / srms;

  // Alfven waves bounding the double-star region (MK05 eq. 51)
  const T sqdl = sqrt_(dls), sqdr = sqrt_(drs);
  const T abn = fabs_(bn);
  const T sls = sm - divz(abn, sqdl);
  const T srs = sm + divz(abn, sqdr);

  // Region of the face (strict inequalities: with S*_L = S*_R = 0 both sides are averaged):
  //   S*_L > 0           single-star flux of the left side
  //   S*_R < 0           single-star flux of the right side
  //   bn ~ 0             the double-star region collapses onto the contact: single-star flux
  //                      of the side the contact moves away from
  //   otherwise          double-star flux of that side
  // and both sides averaged when the contact speed is exactly zero (or not a number). The
  // side's operands are selected first and its flux is evaluated once, so the lanes of a
  // warp whose contacts move either way run one flux evaluation instead of one per side.
  const T bnsmall = T(1e-12) * (ptl + ptr);
  const bool star_l = sls > T(0);
  const bool star_r = !star_l && (srs < T(0));
  const bool single = star_l || star_r || (bnsq <= bnsmall);
  const bool pos = sm > T(0), neg = sm < T(0);
  const bool both = !star_l && !star_r && !pos && !neg;
  const bool left = star_l || (!star_r && (pos || both));
  // double-star states (MK05 eqs. 59-63)
  T sg = T(0), vss = T(0), wss = T(0), byss = T(0), bzss = T(0), vdotb_ss = T(0);
  if (!single) {
    sg = sgn(bn);
    const T inv = T(1) / (sqdl + sqdr);
    vss = ((sqdl * vls + sqdr * vrs) + (byrs - byls) * sg) * inv;
    wss = ((sqdl * wls + sqdr * wrs) + (bzrs - bzls) * sg) * inv;
    byss = ((sqdl * byrs + sqdr * byls) + (sqdl * sqdr) * ((vrs - vls) * sg)) * inv;
    bzss = ((sqdl * bzrs + sqdr * bzls) + (sqdl * sqdr) * ((wrs - wls) * sg)) * inv;
    vdotb_ss = (sm * bn + vss * byss) + wss * bzss;
  }
  side_region_flux<LHLLD>(left, single, L, R, bn, el, er, ptl, ptr, sl, sr, dls, drs, sm, vls, vrs, wls, wrs, byls,
                          byrs, bzls, bzrs, els, ers, pts, sls, srs, sqdl, sqdr, vdotb_ls, vdotb_rs, sg, vss, wss,
                          byss, bzss, vdotb_ss, f);
  if (both) {
    T fb[NFLX];
    side_region_flux<LHLLD>(false, single, L, R, bn, el, er, ptl, ptr, sl, sr, dls, drs, sm, vls, vrs, wls, wrs,
                            byls, byrs, bzls, bzrs, els, ers, pts, sls, srs, sqdl, sqdr, vdotb_ls, vdotb_rs, sg, vss,
                            wss, byss, bzss, vdotb_ss, fb);
#pragma unroll
    for (int n = 0; n < NFLX; ++n) f[n] = T(0.5) * (f[n] + fb[n]);
  }
}

}  // namespace chq
