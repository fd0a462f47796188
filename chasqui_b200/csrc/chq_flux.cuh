// chasqui_b200 — K1: the fused face-flux kernel of one Runge-Kutta stage.
//
// Per face: reconstruct both sides from the primitives, apply flattening and the
// donor-cell floor fallback, optionally the low-Mach velocity blend, solve the Riemann
// problem in registers and write the 6 conserved fluxes plus the two face EMF components
// (E_t2 = -F(B_t1), E_t1 = +F(B_t2)). Same face ranges and outputs as the reference's
// Fluxes<DIR,R,S> (src/physics.hpp:66-226); the left/right face states never leave the SM.
//
// Work decomposition (one launch covers all three directions):
//   x-sweep : one warp = 32 consecutive cells of a row; lane l computes the (aL, aR) pair
//             of its cell once and receives its left neighbour's aR by __shfl_up_sync, so a
//             warp emits 31 faces and no cell parabola is evaluated twice.
//   y/z-sweep: lanes run along i (fully coalesced rows); each thread marches `seglen` faces
//             along the sweep direction, carrying the previous cell's aR in registers.
// Warps for z come first, then y, then x, so that the short x warps fill the tail.
#pragma once
#include "chq_common.cuh"
#include "chq_recon.cuh"
#include "chq_riemann.cuh"
#include "chq_eigen.cuh"

namespace chq {

struct StepCtl;   // device-resident time-step control (chq_ctl.cuh)

template <class P> struct FluxArgs {
  Geom g;
  EOSp eos;
  const P *w;          // primitives, 6 components
  const P *bcc;        // cell-centred B, 3 components
  const double *bn[3]; // face-normal field of the stage's current state, per direction
  P *flx[3];           // fluxes, 6 components, per direction
  P *et2[3];           // E_{t2} on faces of each direction (e3x1, e1x2, e2x3)
  P *et1[3];           // E_{t1} on faces of each direction (e2x1, e3x2, e1x3)
  int flatten, low_mach;
  double lhlld_phi;
  // inclusive face ranges per direction: lo[dir][0..2] = (k, j, i)
  int lo[3][3], hi[3][3];
  int active[3];
  int seglen;          // faces per thread along y/z sweeps
  long nwarp[3];       // warps per direction
  int nseg[3];         // segments along the sweep (x: 31-face segments)
  int nchunk;          // 32-wide i chunks for y/z sweeps (aligned to i = 0)
  const int *skip;     // optional device flag: nonzero -> kernel returns immediately
};

// ---------------------------------------------------------------------------------------
// Cell work: the (aL, aR) pair of cell `lc` (linear index) for the 8 reconstructed
// quantities (d, u, v, w, p, by, bz, s) in the frame of direction DIR.
template <int DIR, int R, bool CHAR, class P>
CHQ_D void cell_states(const FluxArgs<P> &A, long lc, P aL[8], P aR[8]) {
  constexpr int IVU = IVX + DIR, IVV = IVX + (DIR + 1) % 3, IVW = IVX + (DIR + 2) % 3;
  constexpr int IBT1 = (DIR + 1) % 3, IBT2 = (DIR + 2) % 3;
  constexpr int RE = Reach<R>::v;
  const long vs = A.g.vstride;
  const long st = (DIR == 0) ? 1 : (DIR == 1) ? A.g.sj : A.g.sk;
  const P *src[8] = {A.w + IDN * vs, A.w + IVU * vs, A.w + IVV * vs, A.w + IVW * vs,
                     A.w + IPR * vs, A.bcc + IBT1 * vs, A.bcc + IBT2 * vs, A.w + IENT * vs};
  P q[8][5];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
#pragma unroll
    for (int m = -RE; m <= RE; ++m) q[n][2 + m] = ldg(src[n] + lc + m * st);
#pragma unroll
    for (int m = RE + 1; m <= 2; ++m) { q[n][2 + m] = q[n][2 + RE]; q[n][2 - m] = q[n][2 - RE]; }
  }
  if constexpr (!CHAR || R == R_DC) {
#pragma unroll
    for (int n = 0; n < 7; ++n) recon_cell<R>(q[n], aL[n], aR[n]);
  } else {
    // characteristic projection with this cell's own eigenvectors (src/physics.hpp:108-150)
    Eigen7<P> E;
    const P bx = ldg(A.bcc + DIR * vs + lc);
    eigensystem<P>(q[0][2], q[4][2], q[5][2], q[6][2], bx, P(A.eos.gamma), E);
    P cL[7], cR[7];
#pragma unroll
    for (int kk = 0; kk < 7; ++kk) {
      P c5[5];
#pragma unroll
      for (int m = 2 - RE; m <= 2 + RE; ++m) {
        P acc = P(0);
#pragma unroll
        for (int n = 0; n < 7; ++n) acc += E.L[kk][n] * q[n][m];
        c5[m] = acc;
      }
#pragma unroll
      for (int m = RE + 1; m <= 2; ++m) { c5[2 + m] = c5[2 + RE]; c5[2 - m] = c5[2 - RE]; }
      recon_cell<R>(c5, cL[kk], cR[kk]);
    }
#pragma unroll
    for (int n = 0; n < 7; ++n) {
      P accL = P(0), accR = P(0);
#pragma unroll
      for (int kk = 0; kk < 7; ++kk) {
        accL += E.R[n][kk] * cL[kk];
        accR += E.R[n][kk] * cR[kk];
      }
      aL[n] = accL;
      aR[n] = accR;
    }
  }
  recon_cell<R>(q[7], aL[7], aR[7]);   // entropy scalar, always primitive
  if constexpr (R == R_PPM || R == R_PPMX || R == R_WENOZ) {
    if (A.flatten) {
      const P f = flattening<P>(q[4], q[1][1], q[1][3]);
      if (f > P(0)) {
#pragma unroll
        for (int n = 0; n < 8; ++n) {
          aL[n] += f * (q[n][2] - aL[n]);
          aR[n] += f * (q[n][2] - aR[n]);
        }
      }
    }
  }
  // donor-cell fallback of a side that reconstructed to rho <= floor or p <= floor
  const P dfl = P(A.eos.dfloor), pfl = P(A.eos.pfloor);
  if (aL[0] <= dfl || aL[4] <= pfl) {
#pragma unroll
    for (int n = 0; n < 8; ++n) aL[n] = q[n][2];
  }
  if (aR[0] <= dfl || aR[4] <= pfl) {
#pragma unroll
    for (int n = 0; n < 8; ++n) aR[n] = q[n][2];
  }
}

// ---------------------------------------------------------------------------------------
// Face work: Riemann solve of the face `lf` (between cells lf - stride and lf).
template <int DIR, int S, class P>
CHQ_D void face_flux(const FluxArgs<P> &A, long lf, const P wl[8], const P wr[8]) {
  constexpr int IVU = IVX + DIR, IVV = IVX + (DIR + 1) % 3, IVW = IVX + (DIR + 2) % 3;
  const long vs = A.g.vstride;
  const P gamma = P(A.eos.gamma), gm1 = P(A.eos.gm1);
  MState<P> L{wl[0], wl[1], wl[2], wl[3], wl[4], wl[5], wl[6]};
  MState<P> R{wr[0], wr[1], wr[2], wr[3], wr[4], wr[5], wr[6]};
  const P b_n = P(A.bn[DIR][lf]);
  if (A.low_mach) {
    // Thornber et al. (2008) blend of the normal velocities (src/physics.hpp:170-178)
    const P cl = fast_speed(L, b_n, gamma), cr = fast_speed(R, b_n, gamma);
    const P z = fmin_(P(1), fmax_(fabs_(L.u) / cl, fabs_(R.u) / cr));
    const P um = P(0.5) * (L.u + R.u), ud = P(0.5) * (z * (L.u - R.u));
    L.u = um + ud;
    R.u = um - ud;
  }
  P f[NFLX];
  if constexpr (S == S_HLLD) {
    hlld<false>(L, R, b_n, gamma, gm1, f, P(1), P(1));
  } else if constexpr (S == S_LHLLD) {
    // shock detector theta and low-Mach factor phi (src/physics.hpp:183-211)
    constexpr int t1 = (DIR + 1) % 3, t2 = (DIR + 2) % 3;
    const long st = (DIR == 0) ? 1 : (DIR == 1) ? A.g.sj : A.g.sk;
    const long s1 = (t1 == 0) ? 1 : (t1 == 1) ? A.g.sj : A.g.sk;
    const long s2 = (t2 == 0) ? 1 : (t2 == 1) ? A.g.sj : A.g.sk;
    const bool has_t1 = (t1 == 0) || (t1 == 1 && A.g.two_d) || (t1 == 2 && A.g.three_d);
    const bool has_t2 = (t2 == 0) || (t2 == 1 && A.g.two_d) || (t2 == 2 && A.g.three_d);
    const long lL = lf - st;
    const P cfmax = fmax_(fast_speed(L, b_n, gamma), fast_speed(R, b_n, gamma));
    const P *wu = A.w + IVU * vs, *wv = A.w + IVV * vs, *ww = A.w + IVW * vs;
    const P du = ldg(wu + lf) - ldg(wu + lL);
    P dvw = P(0);
    if (has_t1) {
      const P d1 = fmin_(fmin_(ldg(wv + lL) - ldg(wv + lL - s1), ldg(wv + lL + s1) - ldg(wv + lL)),
                         fmin_(ldg(wv + lf) - ldg(wv + lf - s1), ldg(wv + lf + s1) - ldg(wv + lf)));
      dvw = fmin_(dvw, d1);
    }
    if (has_t2) {
      const P d2 = fmin_(fmin_(ldg(ww + lL) - ldg(ww + lL - s2), ldg(ww + lL + s2) - ldg(ww + lL)),
                         fmin_(ldg(ww + lf) - ldg(ww + lf - s2), ldg(ww + lf + s2) - ldg(ww + lf)));
      dvw = fmin_(dvw, d2);
    }
    const P ratio = fmin_(P(1), (-fmin_(du, P(0)) + cfmax) / (-dvw + cfmax));
    const P r2 = ratio * ratio;
    const P theta = r2 * r2;
    const P chi = fmin_(P(1), fmax_(flow_speed_u(L, b_n), flow_speed_u(R, b_n)) / cfmax);
    const P phi = (A.lhlld_phi >= 0.0) ? P(A.lhlld_phi) : chi * (P(2) - chi);
    hlld<true>(L, R, b_n, gamma, gm1, f, theta, phi);
  } else {
    hlle(L, R, b_n, gamma, gm1, f);
  }
  P *flx = A.flx[DIR];
  flx[IDN * vs + lf] = f[FD];
  flx[IVU * vs + lf] = f[FMU];
  flx[IVV * vs + lf] = f[FMV];
  flx[IVW * vs + lf] = f[FMW];
  flx[IEN * vs + lf] = f[FEN];
  // entropy flux upwinded with the mass flux, averaged at an exact zero
  const P sl = wl[7], sr = wr[7];
  flx[IENT * vs + lf] = (f[FD] > P(0)) ? f[FD] * sl : (f[FD] < P(0)) ? f[FD] * sr : P(0.5) * (f[FD] * (sl + sr));
  A.et2[DIR][lf] = -f[FBY];
  A.et1[DIR][lf] = f[FBZ];
}

// ---------------------------------------------------------------------------------------
template <int R, int S, bool CHAR, class P>
CHQ_D void sweep_x(const FluxArgs<P> &A, long wid) {
  const int lane = threadIdx.x & 31;
  const int nseg = A.nseg[0];
  const long row = wid / nseg;
  const int seg = (int)(wid - row * nseg);
  const int nj = A.hi[0][1] - A.lo[0][1] + 1;
  const int k = A.lo[0][0] + (int)(row / nj);
  const int j = A.lo[0][1] + (int)(row - (long)(row / nj) * nj);
  const int c = A.lo[0][2] - 1 + 31 * seg + lane;   // this lane's cell
  const bool have = (c <= A.hi[0][2]);
  P aL[8], aR[8];
  const long lc = A.g.idx(k, j, c);
  if (have) cell_states<0, R, CHAR, P>(A, lc, aL, aR);
  P wl[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) wl[n] = __shfl_up_sync(0xffffffffu, aR[n], 1);
  if (have && lane > 0) face_flux<0, S, P>(A, lc, wl, aL);
}

template <int DIR, int R, int S, bool CHAR, class P>
CHQ_D void sweep_yz(const FluxArgs<P> &A, long wid) {
  const int lane = threadIdx.x & 31;
  const int nseg = A.nseg[DIR];
  const int nchunk = A.nchunk;
  // warp id -> (outer transverse index, segment, i chunk)
  const int chunk = (int)(wid % nchunk);
  const long rest = wid / nchunk;
  const int seg = (int)(rest % nseg);
  const int outer = (int)(rest / nseg);
  const int i = 32 * chunk + lane;
  if (i < A.lo[DIR][2] || i > A.hi[DIR][2]) return;
  const int f0 = A.lo[DIR][DIR == 1 ? 1 : 0] + A.seglen * seg;
  const int f1 = min(f0 + A.seglen - 1, A.hi[DIR][DIR == 1 ? 1 : 0]);
  const long st = (DIR == 1) ? A.g.sj : A.g.sk;
  long lc;
  if (DIR == 1) lc = A.g.idx(A.lo[1][0] + outer, f0 - 1, i);
  else lc = A.g.idx(f0 - 1, A.lo[2][1] + outer, i);
  P aL[8], aR[8], wl[8];
  cell_states<DIR, R, CHAR, P>(A, lc, aL, aR);
#pragma unroll
  for (int n = 0; n < 8; ++n) wl[n] = aR[n];
  for (int f = f0; f <= f1; ++f) {
    lc += st;
    cell_states<DIR, R, CHAR, P>(A, lc, aL, aR);
    face_flux<DIR, S, P>(A, lc, wl, aL);
#pragma unroll
    for (int n = 0; n < 8; ++n) wl[n] = aR[n];
  }
}

template <int R, int S, bool CHAR, class P>
__global__ void __launch_bounds__(128) flux_kernel(const FluxArgs<P> A) {
  if (A.skip && *A.skip) return;
  const long wid = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (wid < A.nwarp[2]) {
    sweep_yz<2, R, S, CHAR, P>(A, wid);
  } else if (wid < A.nwarp[2] + A.nwarp[1]) {
    sweep_yz<1, R, S, CHAR, P>(A, wid - A.nwarp[2]);
  } else if (wid < A.nwarp[2] + A.nwarp[1] + A.nwarp[0]) {
    sweep_x<R, S, CHAR, P>(A, wid - A.nwarp[2] - A.nwarp[1]);
  }
}

}  // namespace chq
