// chasqui_b200 — K1: the fused face-flux kernel of one Runge-Kutta stage.
//
// Per face: reconstruct both sides from the primitives, apply flattening and the
// donor-cell floor fallback, optionally the low-Mach velocity blend, solve the Riemann
// problem in registers and write the 6 conserved fluxes plus the two face EMF components
// (E_t2 = -F(B_t1), E_t1 = +F(B_t2)). Same face ranges and outputs as the reference's
// Fluxes<DIR,R,S> (src/physics.hpp:66-226); the left/right face states never leave the SM.
//
// Work decomposition, two launches per stage:
//   flux_x_kernel : one warp = 32 consecutive cells of a row; lane l computes the (aL, aR)
//             pair of its cell once (stencil from L1) and receives its left neighbour's aR by
//             __shfl_up_sync, so a warp emits 31 faces and no cell parabola is evaluated twice
//             (PPM: slopes and unlimited interface values are shared between lanes too, and a
//             warp emits 29 faces).
//   flux_yz_kernel: lanes run along i (fully coalesced rows); each thread marches `seglen`
//             faces along y or z with its stencil in a shared-memory window that cp.async
//             refills one cell ahead, and parks the previous cell's aR in shared memory
//             during the Riemann solve (PPM: the march carries each quantity's slope and
//             unlimited interface value to the next cell). z warps come first, then y.
// The batched forms (flux_x_batched, flux_yz_batched) run the same sweeps for many meshes.
#pragma once
#include <cuda.h>   // CUtensorMap (the TMA descriptor type; no driver call is made from here)
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
  int nseg[3];         // segments along the sweep (x: XFaces-face segments)
  int nchunk;          // 32-wide i chunks for y/z sweeps (aligned to i = 0)
  int xvar;            // x-sweep kernel variant (register cap, FluxMinBlocks); picked by the autotuner
  const int *skip;     // optional device flag: nonzero -> kernel returns immediately
  int yzvar;           // y/z staging of the FP64 streaming-PPM march: 0 cp.async, 1 TMA (autotuner)
  const void *yzmaps;  // host copy of the two tensor maps of the TMA staging (YzMaps), or null
  int *err;            // device error word: a TMA wait that gave up sets it (and its warp stops)
};

// Tensor maps of the TMA staging: the primitives w (6 components) and the centred field bcc
// (3 components) of one mesh as 4-D tensors (i over the row pitch, j, k, component), boxes of
// one 32-cell row segment of one component.
struct YzMaps {
  CUtensorMap w, b;
};

// ---------------------------------------------------------------------------------------
// Per-direction views: the 8 reconstructed quantities (d, u, v, w, p, by, bz, s) of the
// frame of direction d and the output slots of its faces. Built once per warp; the
// arithmetic is identical for every direction, so one code copy serves the y and z sweeps.
template <class P> struct DirView {
  const P *src[8];     // cell fields in face-frame order
  const P *bx;         // cell-centred normal field (characteristic projection)
  int st;              // stride along the sweep (offsets within a component fit in 32 bits)
  int s1, s2;          // strides of the two transverse directions (LHLLD detector)
  int has1, has2;
  const double *bn;    // face-normal field of the stage's current state
  P *out[8];           // flux slots (d, u, v, w, E, s) then E_t2, E_t1
};

template <class P> CHQ_D DirView<P> dir_view(const FluxArgs<P> &A, int d) {
  DirView<P> v;
  const long vs = A.g.vstride;
  const int ivu = IVX + d, ivv = IVX + (d + 1) % 3, ivw = IVX + (d + 2) % 3;
  const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
  const int strides[3] = {1, (int)A.g.sj, (int)A.g.sk};
  v.src[0] = A.w + IDN * vs;
  v.src[1] = A.w + ivu * vs;
  v.src[2] = A.w + ivv * vs;
  v.src[3] = A.w + ivw * vs;
  v.src[4] = A.w + IPR * vs;
  v.src[5] = A.bcc + t1 * vs;
  v.src[6] = A.bcc + t2 * vs;
  v.src[7] = A.w + IENT * vs;
  v.bx = A.bcc + d * vs;
  v.st = strides[d];
  v.s1 = strides[t1];
  v.s2 = strides[t2];
  v.has1 = (t1 == 0) || (t1 == 1 && A.g.two_d) || (t1 == 2 && A.g.three_d);
  v.has2 = (t2 == 0) || (t2 == 1 && A.g.two_d) || (t2 == 2 && A.g.three_d);
  v.bn = A.bn[d];
  P *f = A.flx[d];
  v.out[0] = f + IDN * vs;
  v.out[1] = f + ivu * vs;
  v.out[2] = f + ivv * vs;
  v.out[3] = f + ivw * vs;
  v.out[4] = f + IEN * vs;
  v.out[5] = f + IENT * vs;
  v.out[6] = A.et2[d];
  v.out[7] = A.et1[d];
  return v;
}

// ---------------------------------------------------------------------------------------
// Flattening toward the cell value (PPM, PPMX, WENO-Z; src/recon.hpp:179-187 applied as in
// src/physics.hpp:152-162) and the donor-cell fallback of a side that reconstructed to
// rho <= floor or p <= floor, on the cell's (aL, aR) pairs of the 8 quantities.
template <int R, class P>
CHQ_D void finish_states(const FluxArgs<P> &A, P aL[8], P aR[8], const P qc[8], const P p5[5], P um1, P up1) {
  if constexpr (R == R_PPM || R == R_PPMX || R == R_WENOZ) {
    if (A.flatten) {
      const P f = flattening<P>(p5, um1, up1);
      if (f > P(0)) {
#pragma unroll
        for (int n = 0; n < 8; ++n) {
          aL[n] += f * (qc[n] - aL[n]);
          aR[n] += f * (qc[n] - aR[n]);
        }
      }
    }
  }
  const P dfl = P(A.eos.dfloor), pfl = P(A.eos.pfloor);
  if (aL[0] <= dfl || aL[4] <= pfl) {
#pragma unroll
    for (int n = 0; n < 8; ++n) aL[n] = qc[n];
  }
  if (aR[0] <= dfl || aR[4] <= pfl) {
#pragma unroll
    for (int n = 0; n < 8; ++n) aR[n] = qc[n];
  }
}

// ---------------------------------------------------------------------------------------
// Cell work: the (aL, aR) pair of cell `lc` (linear index) for the 8 reconstructed
// quantities in the frame of the view's direction. Each quantity is reconstructed as soon
// as its stencil is loaded, so only the cell values (for flattening and the floor
// fallback) stay live across quantities.
template <int R, bool CHAR, class P, class Stencil>
CHQ_D void cell_states_from(const FluxArgs<P> &A, const DirView<P> &V, int lc, P aL[8], P aR[8], const Stencil &ld) {
  constexpr int RE = Reach<R>::v;
  P qc[8];
  P p5[5], um1 = P(0), up1 = P(0);
  if constexpr (!CHAR || R == R_DC) {
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      P q5[5];
      ld(n, q5);
#pragma unroll
      for (int m = RE + 1; m <= 2; ++m) { q5[2 + m] = q5[2 + RE]; q5[2 - m] = q5[2 - RE]; }
      recon_cell<R>(q5, aL[n], aR[n]);
      qc[n] = q5[2];
      if (n == 1) { um1 = q5[1]; up1 = q5[3]; }
      if (n == 4) {
#pragma unroll
        for (int m = 0; m < 5; ++m) p5[m] = q5[m];
      }
    }
  } else {
    // characteristic projection with this cell's own eigenvectors (src/physics.hpp:108-150)
    P q[7][5];
#pragma unroll
    for (int n = 0; n < 7; ++n) {
      ld(n, q[n]);
#pragma unroll
      for (int m = RE + 1; m <= 2; ++m) { q[n][2 + m] = q[n][2 + RE]; q[n][2 - m] = q[n][2 - RE]; }
      qc[n] = q[n][2];
    }
    um1 = q[1][1];
    up1 = q[1][3];
#pragma unroll
    for (int m = 0; m < 5; ++m) p5[m] = q[4][m];
    Eigen7<P> E;
    eigensystem<P>(q[0][2], q[4][2], q[5][2], q[6][2], ldg(V.bx + lc), P(A.eos.gamma), E);
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
    // entropy scalar, always primitive
    P q5[5];
    ld(7, q5);
#pragma unroll
    for (int m = RE + 1; m <= 2; ++m) { q5[2 + m] = q5[2 + RE]; q5[2 - m] = q5[2 - RE]; }
    recon_cell<R>(q5, aL[7], aR[7]);
    qc[7] = q5[2];
  }
  finish_states<R, P>(A, aL, aR, qc, p5, um1, up1);
}

// Stencil sources of cell_states_from: q5[2-RE .. 2+RE] of quantity n of the cell.
// Global: cached loads along the sweep (the x-sweep, whose stencil lies in the lanes' lines).
template <int RE, class P> struct GlobalStencil {
  const DirView<P> &V;
  int lc;
  CHQ_D void operator()(int n, P q5[5]) const {
#pragma unroll
    for (int m = -RE; m <= RE; ++m) q5[2 + m] = ldg(V.src[n] + lc + m * V.st);
  }
};

template <int R, bool CHAR, class P>
CHQ_D void cell_states(const FluxArgs<P> &A, const DirView<P> &V, int lc, P aL[8], P aR[8]) {
  cell_states_from<R, CHAR, P>(A, V, lc, aL, aR, GlobalStencil<Reach<R>::v, P>{V, lc});
}

// asynchronous global -> shared copies of one element (cp.async, completed per thread)
CHQ_D void cp_async_elem(double *dst, const double *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
CHQ_D void cp_async_elem(float *dst, const float *src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}
CHQ_D void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
CHQ_D void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Tensor-memory-access (TMA) staging: an mbarrier in shared memory counts the bytes the
// bulk tensor copies deliver (complete_tx); threads wait on its phase parity.
CHQ_D unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
CHQ_D void mbar_init(unsigned long long *mb, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(mb)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
CHQ_D void mbar_expect_tx(unsigned long long *mb, unsigned bytes) {
  asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_addr(mb)),
               "r"(bytes)
               : "memory");
}
// bounded wait for the phase of the given parity; false when the limit ran out
CHQ_D bool mbar_wait(unsigned long long *mb, unsigned parity) {
  const unsigned a = smem_addr(mb);
  for (int it = 0; it < (1 << 24); ++it) {
    unsigned ok = 0;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok)
                 : "r"(a), "r"(parity)
                 : "memory");
    if (ok) return true;
  }
  return false;
}
// generic-proxy accesses of shared memory before the async-proxy writes that follow
CHQ_D void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// one box of a 4-D tensor map over this GPU's own memory into this CTA's shared memory only,
// completing on mb
CHQ_D void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, unsigned long long *mb) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(mb))
      : "memory");
}

// Threads per block of the y/z kernels (the stride of their shared-memory columns).
#ifndef CHQ_FLUXYZ_THREADS
#define CHQ_FLUXYZ_THREADS 128
#endif
constexpr int kYzThreads = CHQ_FLUXYZ_THREADS;

// Marching window: one shared-memory column per thread and quantity, 2RE+1 slots. For the
// current cell c, slots 0..2RE-1 hold q[c-RE .. c+RE-1] and slot 2RE holds q[c+RE], copied
// asynchronously one step earlier. Reading the stencil shifts the window down by one slot
// (every slot value is consumed by that shift before the next copy into slot 2RE is issued,
// so the copy cannot overtake the read) and starts the copy of q[c+RE+1] for the next cell.
template <int RE, class P> struct WindowStencil {
  P *col;            // this thread's column: slot m of quantity n at col[(n*(2RE+1) + m) * kYzThreads]
  const DirView<P> &V;
  int lc;
  bool prefetch;     // false on the last cell of the march
  CHQ_D void operator()(int n, P q5[5]) const {
    P *w = col + n * (2 * RE + 1) * kYzThreads;
#pragma unroll
    for (int m = 0; m <= 2 * RE; ++m) q5[2 - RE + m] = w[m * kYzThreads];
#pragma unroll
    for (int m = 0; m < 2 * RE; ++m) w[m * kYzThreads] = q5[3 - RE + m];
    if (prefetch) cp_async_elem(w + 2 * RE * kYzThreads, V.src[n] + lc + (RE + 1) * V.st);
  }
};

// ---------------------------------------------------------------------------------------
// Face work: Riemann solve of the face `lf` (between cells lf - stride and lf).
// b_n: the face-normal field of the face (a sweep that prefetched it passes it in).
template <int S, class P>
CHQ_D void face_flux(const FluxArgs<P> &A, const DirView<P> &V, int lf, const P wl[8], const P wr[8], const P b_n) {
  const P gamma = P(A.eos.gamma), gm1 = P(A.eos.gm1);
  MState<P> L{wl[0], wl[1], wl[2], wl[3], wl[4], wl[5], wl[6]};
  MState<P> R{wr[0], wr[1], wr[2], wr[3], wr[4], wr[5], wr[6]};
  if (A.low_mach) {
    // Thornber et al. (2008) blend of the normal velocities (src/physics.hpp:170-178)
    const P cl = fast_speed(L, b_n, gamma), cr = fast_speed(R, b_n, gamma);
    const P z = fmin_(P(1), fmax_(divz(fabs_(L.u), cl), divz(fabs_(R.u), cr)));
    const P um = P(0.5) * (L.u + R.u), ud = P(0.5) * (z * (L.u - R.u));
    L.u = um + ud;
    R.u = um - ud;
  }
  P f[NFLX];
  if constexpr (S == S_HLLD) {
    hlld<false>(L, R, b_n, gamma, gm1, f, P(1), P(1));
  } else if constexpr (S == S_LHLLD) {
    // shock detector theta and low-Mach factor phi (src/physics.hpp:183-211)
    const int lL = lf - V.st;
    const P cfmax = fmax_(fast_speed(L, b_n, gamma), fast_speed(R, b_n, gamma));
    const P *wu = V.src[1], *wv = V.src[2], *ww = V.src[3];
    const int s1 = V.s1, s2 = V.s2;
    const P du = ldg(wu + lf) - ldg(wu + lL);
    P dvw = P(0);
    if (V.has1) {
      const P d1 = fmin_(fmin_(ldg(wv + lL) - ldg(wv + lL - s1), ldg(wv + lL + s1) - ldg(wv + lL)),
                         fmin_(ldg(wv + lf) - ldg(wv + lf - s1), ldg(wv + lf + s1) - ldg(wv + lf)));
      dvw = fmin_(dvw, d1);
    }
    if (V.has2) {
      const P d2 = fmin_(fmin_(ldg(ww + lL) - ldg(ww + lL - s2), ldg(ww + lL + s2) - ldg(ww + lL)),
                         fmin_(ldg(ww + lf) - ldg(ww + lf - s2), ldg(ww + lf + s2) - ldg(ww + lf)));
      dvw = fmin_(dvw, d2);
    }
    const P ratio = fmin_(P(1), (-fmin_(du, P(0)) + cfmax) / (-dvw + cfmax));
    const P r2 = ratio * ratio;
    const P theta = r2 * r2;
    const P chi = fmin_(P(1), divz(fmax_(flow_speed_u(L, b_n), flow_speed_u(R, b_n)), cfmax));
    const P phi = (A.lhlld_phi >= 0.0) ? P(A.lhlld_phi) : chi * (P(2) - chi);
    hlld<true>(L, R, b_n, gamma, gm1, f, theta, phi);
  } else {
    hlle(L, R, b_n, gamma, gm1, f);
  }
  V.out[0][lf] = f[FD];
  V.out[1][lf] = f[FMU];
  V.out[2][lf] = f[FMV];
  V.out[3][lf] = f[FMW];
  V.out[4][lf] = f[FEN];
  // entropy flux upwinded with the mass flux, averaged at an exact zero
  const P sl = wl[7], sr = wr[7];
  V.out[5][lf] = (f[FD] > P(0)) ? f[FD] * sl : (f[FD] < P(0)) ? f[FD] * sr : P(0.5) * (f[FD] * (sl + sr));
  V.out[6][lf] = -f[FBY];
  V.out[7][lf] = f[FBZ];
}
template <int S, class P>
CHQ_D void face_flux(const FluxArgs<P> &A, const DirView<P> &V, int lf, const P wl[8], const P wr[8]) {
  face_flux<S, P>(A, V, lf, wl, wr, P(V.bn[lf]));
}

// ---------------------------------------------------------------------------------------
template <int R, int S, bool CHAR, class P>
CHQ_D void sweep_x(const FluxArgs<P> &A, int wid) {
  const int lane = threadIdx.x & 31;
  const int nseg = A.nseg[0];
  const int row = wid / nseg;
  const int seg = (int)(wid - row * nseg);
  const int nj = A.hi[0][1] - A.lo[0][1] + 1;
  const int k = A.lo[0][0] + (int)(row / nj);
  const int j = A.lo[0][1] + (row - (row / nj) * nj);
  const int c = A.lo[0][2] - 1 + 31 * seg + lane;   // this lane's cell
  const bool have = (c <= A.hi[0][2]);
  const DirView<P> V = dir_view(A, 0);
  P aL[8], aR[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) { aL[n] = P(0); aR[n] = P(0); }
  const int lc = A.g.idx32(k, j, c);
  const P bnf = have ? P(ldg(V.bn + lc)) : P(0);   // loaded before the reconstruction
  if (have) cell_states<R, CHAR, P>(A, V, lc, aL, aR);
  P wl[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) wl[n] = __shfl_up_sync(0xffffffffu, aR[n], 1);
  if (have && lane > 0) face_flux<S, P>(A, V, lc, wl, aL, bnf);
}

// Faces per x-sweep warp: 31 in the per-cell form (lane 0 contributes only its right state),
// 29 in the streaming PPM form below (lanes 0 and 31 contribute only their slope and interface
// value, so the states of lanes 1..30 are complete and lanes 2..30 emit faces).
template <int R, bool CHAR> struct XFaces { static constexpr int v = (R == R_PPM && !CHAR) ? 29 : 31; };

// Streaming PPM (CW84, src/recon.hpp:21-78) along a row of 32 cells, one per lane. The
// reference evaluates, for face i, the limited parabolas of cells i-1 and i from their
// monotonised slopes and unlimited interface values, so each slope is evaluated three times
// and each unlimited interface value twice over a row. Here lane c evaluates its own slope
// s_c and the unlimited value at its right interface F_{c+1/2} once; the slope of cell c+1
// and the value F_{c-1/2} come from the neighbouring lanes by warp shuffle. The operands of
// every expression are the reference's, so the limited states are bitwise the same.
template <int S, class P>
CHQ_D void sweep_x_ppm(const FluxArgs<P> &A, int wid) {
  const int lane = threadIdx.x & 31;
  const int nseg = A.nseg[0];
  const int row = wid / nseg;
  const int seg = (int)(wid - row * nseg);
  const int nj = A.hi[0][1] - A.lo[0][1] + 1;
  const int k = A.lo[0][0] + (int)(row / nj);
  const int j = A.lo[0][1] + (row - (row / nj) * nj);
  const int c = A.lo[0][2] - 2 + 29 * seg + lane;   // this lane's cell
  // lanes past the row's last face (and lane 0's stencil at the row start) read clamped
  // indices inside the row; their states are never used
  const int last = A.g.ni - 1;
  const int cm2 = max(c - 2, 0), cm1 = max(c - 1, 0), c0 = min(c, last), cp1 = min(c + 1, last),
            cp2 = min(c + 2, last);
  const int base = A.g.idx32(k, j, 0);
  const DirView<P> V = dir_view(A, 0);
  const P bnf = P(ldg(V.bn + base + c0));   // this lane's face-normal field, loaded before the reconstruction
  P aL[8], aR[8], qc[8], p5[5], um1 = P(0), up1 = P(0);
  // every stencil load of the lane is issued before any arithmetic: a warp handles one row
  // segment, so nothing else hides the latency of its loads (measured: the x sweep ~20 %
  // faster in FP64 than with the loads interleaved with each quantity's reconstruction)
  P QM[8], Q0[8], QP[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const P *src = V.src[n] + base;
    QM[n] = ldg(src + cm1);
    Q0[n] = ldg(src + c0);
    QP[n] = ldg(src + cp1);
  }
  const P pm2 = ldg(V.src[4] + base + cm2), pp2 = ldg(V.src[4] + base + cp2);
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const P qm = QM[n], q0 = Q0[n], qp = QP[n];
    const P sc = mc_slope(qm, q0, qp);
    const P sp = __shfl_down_sync(0xffffffffu, sc, 1);    // s_{c+1}
    const P fp = ppm_face(q0, qp, sc, sp);                 // F_{c+1/2}, unlimited
    P l = __shfl_up_sync(0xffffffffu, fp, 1), r = fp;     // F_{c-1/2}
    ppm_limit(q0, l, r);
    aL[n] = l;
    aR[n] = r;
    qc[n] = q0;
    if (n == 1) { um1 = qm; up1 = qp; }
    if (n == 4) { p5[0] = pm2; p5[1] = qm; p5[2] = q0; p5[3] = qp; p5[4] = pp2; }
  }
  finish_states<R_PPM, P>(A, aL, aR, qc, p5, um1, up1);
  P wl[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) wl[n] = __shfl_up_sync(0xffffffffu, aR[n], 1);
  if (lane >= 2 && lane <= 30 && c <= A.hi[0][2]) face_flux<S, P>(A, V, base + c, wl, aL, bnf);
}

// Streaming PPM along a y/z march. Each thread's shared-memory column keeps, per quantity,
// q_c, q_{c+1}, q_{c+2} (the last copied asynchronously one cell ahead), the slope s_c and
// the unlimited interface value F_{c-1/2} computed at the previous cell; the velocity adds
// u_{c-1} and the pressure p_{c-2}, p_{c-1} (flattening). A cell then evaluates one slope
// (s_{c+1}) and one interface value (F_{c+1/2}) per quantity instead of three and two, with
// the reference's operands (bitwise the same limited states as the per-cell form). In FP64
// the face-normal field of the next face is copied asynchronously one cell ahead as well,
// into one of two slots per thread (alternating, so a copy never lands in the slot being
// read), instead of a load at the Riemann solve.
struct PpmWin {
  static constexpr int nslot = 43;
  enum : int { Q0 = 0, Q1 = 1, Q2 = 2, S = 3, F = 4, X1 = 5, X2 = 6 };
  CHQ_HD static constexpr int off(int n) {
    return (n == 0) ? 0 : (n == 1) ? 5 : (n == 2) ? 11 : (n == 3) ? 16 : (n == 4) ? 21 : (n == 5) ? 28 : (n == 6) ? 33 : 38;
  }
};

// TMA (FP64 only, maps and mbar given): instead of one cp.async per quantity and thread, one
// lane of the warp issues, one cell ahead, eight bulk tensor copies of the next cell's 32-wide
// row of each quantity straight into the warp's rows of the window's q_{c+2} slots; the warp
// waits on its mbarrier's phase. Same slots, same values: the states are bitwise those of the
// cp.async form.
template <int S, class P, bool TMA = false>
CHQ_D void sweep_yz_ppm(const FluxArgs<P> &A, int d, int wid, P *park, P *win, const YzMaps *maps = nullptr,
                        unsigned long long *mbar = nullptr) {
  const int lane = threadIdx.x & 31;
  const int nseg = A.nseg[d];
  const int nchunk = A.nchunk;
  const int chunk = (int)(wid % nchunk);
  const int rest = wid / nchunk;
  const int seg = (int)(rest % nseg);
  const int outer = (int)(rest / nseg);
  const int i = 32 * chunk + lane;
  const bool act = !(i < A.lo[d][2] || i > A.hi[d][2]);
  unsigned mask = 0xffffffffu;
  bool leader = false;
  if constexpr (TMA) {
    mask = __ballot_sync(0xffffffffu, act);
    leader = act && (lane == __ffs(mask) - 1);
  }
  if (!act) return;
  const int sweep_lo = (d == 1) ? A.lo[1][1] : A.lo[2][0];
  const int sweep_hi = (d == 1) ? A.hi[1][1] : A.hi[2][0];
  const int f0 = sweep_lo + A.seglen * seg;
  const int f1 = min(f0 + A.seglen - 1, sweep_hi);
  const DirView<P> V = dir_view(A, d);
  const int st = V.st;
  int lc = (d == 1) ? A.g.idx32(A.lo[1][0] + outer, f0 - 1, i) : A.g.idx32(f0 - 1, A.lo[2][1] + outer, i);
  const int t = threadIdx.x;
  P *col = win + t;
  constexpr bool PFB = (sizeof(P) == 8);
  double *bnw = reinterpret_cast<double *>(win + PpmWin::nslot * kYzThreads) + t;
  // TMA staging: this warp's mbarrier, its rows of the q_{c+2} slots, the tensor coordinates
  unsigned long long *mb = TMA ? mbar + (t >> 5) : nullptr;
  unsigned phase = 0;
  const int outer_idx = (d == 1) ? A.lo[1][0] + outer : A.lo[2][1] + outer;
  auto issue = [&](int pos) {   // the rows of the cell at sweep position pos, all 8 quantities
    mbar_expect_tx(mb, 8u * 32u * (unsigned)sizeof(P));
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      // component of quantity n in w (0, 1, 2, 3, 4, 7) or bcc (5, 6), as dir_view orders them
      const int comp = (n == 0) ? IDN : (n == 1) ? IVX + d : (n == 2) ? IVX + (d + 1) % 3 : (n == 3) ? IVX + (d + 2) % 3
                     : (n == 4) ? IPR : (n == 5) ? (d + 1) % 3 : (n == 6) ? (d + 2) % 3 : IENT;
      const CUtensorMap *map = (n == 5 || n == 6) ? &maps->b : &maps->w;
      P *row = win + (PpmWin::off(n) + PpmWin::Q2) * kYzThreads + (t & ~31);
      if (d == 1) tma_load_4d(row, map, 32 * chunk, pos, outer_idx, comp, mb);
      else tma_load_4d(row, map, 32 * chunk, outer_idx, pos, comp, mb);
    }
  };
  if constexpr (TMA) {
    if (leader) mbar_init(mb, 1);
    __syncwarp(mask);
  }
#define CHQ_SLOT(n, k) col[(PpmWin::off(n) + PpmWin::k) * kYzThreads]
  // cell f0-1: its slope, its left interface value and the window, from direct loads
#pragma unroll
  for (int n = 0; n < 8; ++n) {
    const P *src = V.src[n] + lc;
    const P qm2 = ldg(src - 2 * st), qm1 = ldg(src - st), q0 = ldg(src), qp1 = ldg(src + st);
    const P sm = mc_slope(qm2, qm1, q0), sc = mc_slope(qm1, q0, qp1);
    CHQ_SLOT(n, Q0) = q0;
    CHQ_SLOT(n, Q1) = qp1;
    CHQ_SLOT(n, S) = sc;
    CHQ_SLOT(n, F) = ppm_face(qm1, q0, sm, sc);
    if (n == 1) CHQ_SLOT(1, X1) = qm1;
    if (n == 4) {
      CHQ_SLOT(4, X1) = qm2;
      CHQ_SLOT(4, X2) = qm1;
    }
    if constexpr (!TMA) cp_async_elem(&CHQ_SLOT(n, Q2), src + 2 * st);
  }
  cp_async_commit();
  if constexpr (TMA) {
    if (leader) issue(f0 + 1);
  }
  P wl[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) wl[n] = P(0);
  for (int f = f0 - 1; f <= f1; ++f, lc += st) {
    cp_async_wait_all();
    if constexpr (TMA) {
      // q_{c+2} rows of this cell: the warp gives up together if the copies never land
      const bool ok = __all_sync(mask, mbar_wait(mb, phase & 1u));
      ++phase;
      if (!ok) {
        if (leader && A.err) atomicExch(A.err, 3);
        return;
      }
    }
    const bool pre = (f < f1);
    P bnv = P(0);
    if constexpr (PFB) {
      if (f >= f0) bnv = P(bnw[(f & 1) * kYzThreads]);
      if (pre) cp_async_elem(bnw + ((f + 1) & 1) * kYzThreads, V.bn + lc + st);
    }
    P aL[8], aR[8], qc[8], p5[5], um1 = P(0), up1 = P(0);
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      const P q0 = CHQ_SLOT(n, Q0), q1 = CHQ_SLOT(n, Q1), q2 = CHQ_SLOT(n, Q2);
      const P sc = CHQ_SLOT(n, S), fm = CHQ_SLOT(n, F);
      const P sp = mc_slope(q0, q1, q2);          // s_{c+1}
      const P fp = ppm_face(q0, q1, sc, sp);      // F_{c+1/2}, unlimited
      P l = fm, r = fp;
      ppm_limit(q0, l, r);
      aL[n] = l;
      aR[n] = r;
      qc[n] = q0;
      if (n == 1) {
        um1 = CHQ_SLOT(1, X1);
        up1 = q1;
        CHQ_SLOT(1, X1) = q0;
      }
      if (n == 4) {
        p5[0] = CHQ_SLOT(4, X1);
        p5[1] = CHQ_SLOT(4, X2);
        p5[2] = q0;
        p5[3] = q1;
        p5[4] = q2;
        CHQ_SLOT(4, X1) = p5[1];
        CHQ_SLOT(4, X2) = q0;
      }
      CHQ_SLOT(n, Q0) = q1;
      CHQ_SLOT(n, Q1) = q2;
      CHQ_SLOT(n, S) = sp;
      CHQ_SLOT(n, F) = fp;
      if constexpr (!TMA) {
        if (pre) cp_async_elem(&CHQ_SLOT(n, Q2), V.src[n] + lc + 3 * st);
      }
    }
    cp_async_commit();
    if constexpr (TMA) {
      if (pre) {
        __syncwarp(mask);   // every lane has read its q_{c+2} slots before the copies overwrite them
        if (leader) {
          fence_proxy_async();
          issue(f + 3);
        }
      }
    }
    finish_states<R_PPM, P>(A, aL, aR, qc, p5, um1, up1);
#pragma unroll
    for (int n = 0; n < 8; ++n) park[n * kYzThreads + t] = aR[n];
    if (f >= f0) {
      if constexpr (PFB) face_flux<S, P>(A, V, lc, wl, aL, bnv);
      else face_flux<S, P>(A, V, lc, wl, aL);
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) wl[n] = park[n * kYzThreads + t];
  }
#undef CHQ_SLOT
}

// y (d = 1) or z (d = 2) sweep: one code copy, direction in the view. The right state
// carried to the next face is parked in this thread's shared-memory slot during the
// Riemann solve, which keeps it out of the registers at the solver's peak. With WIN the
// stencil comes from the thread's marching window in shared memory (WindowStencil): one
// asynchronous copy per quantity and cell, issued a whole cell ahead, instead of 2RE+1
// cached loads whose lines a y/z march cannot keep in L1.
template <int R, int S, bool CHAR, bool WIN, class P>
CHQ_D void sweep_yz(const FluxArgs<P> &A, int d, int wid, P *park, P *win) {
  if constexpr (R == R_PPM && !CHAR && WIN) {
    sweep_yz_ppm<S, P>(A, d, wid, park, win);
    return;
  }
  const int lane = threadIdx.x & 31;
  const int nseg = A.nseg[d];
  const int nchunk = A.nchunk;
  const int chunk = (int)(wid % nchunk);
  const int rest = wid / nchunk;
  const int seg = (int)(rest % nseg);
  const int outer = (int)(rest / nseg);
  const int i = 32 * chunk + lane;
  if (i < A.lo[d][2] || i > A.hi[d][2]) return;
  const int sweep_lo = (d == 1) ? A.lo[1][1] : A.lo[2][0];
  const int sweep_hi = (d == 1) ? A.hi[1][1] : A.hi[2][0];
  const int f0 = sweep_lo + A.seglen * seg;
  const int f1 = min(f0 + A.seglen - 1, sweep_hi);
  const DirView<P> V = dir_view(A, d);
  // cell f0-1 first (its right state only), then cell f and face f for f = f0..f1; one copy
  // of the cell code in the loop keeps the kernel's instruction footprint small
  int lc = (d == 1) ? A.g.idx32(A.lo[1][0] + outer, f0 - 1, i) : A.g.idx32(f0 - 1, A.lo[2][1] + outer, i);
  P wl[8];
#pragma unroll
  for (int n = 0; n < 8; ++n) wl[n] = P(0);
  const int t = threadIdx.x;
  constexpr int RE = Reach<R>::v;
  constexpr bool use_win = WIN && (RE > 0);
  P *col = use_win ? win + t : nullptr;
  // FP64: the next face's normal field copied one cell ahead into two alternating slots
  // after the window (as in the streaming-PPM march)
  constexpr bool PFB = use_win && (sizeof(P) == 8);
  double *bnw = PFB ? reinterpret_cast<double *>(win + 8 * (2 * RE + 1) * kYzThreads) + t : nullptr;
  if constexpr (use_win) {
    // window of cell f0-1: q[c-RE .. c+RE-1] now, q[c+RE] asynchronously
#pragma unroll
    for (int n = 0; n < 8; ++n) {
      P *w = col + n * (2 * RE + 1) * kYzThreads;
#pragma unroll
      for (int m = 0; m < 2 * RE; ++m) w[m * kYzThreads] = ldg(V.src[n] + lc + (m - RE) * V.st);
      cp_async_elem(w + 2 * RE * kYzThreads, V.src[n] + lc + RE * V.st);
    }
    cp_async_commit();
  }
  for (int f = f0 - 1; f <= f1; ++f, lc += V.st) {
    P aL[8], aR[8];
    P bnv = P(0);
    if constexpr (use_win) {
      cp_async_wait_all();
      if constexpr (PFB) {
        if (f >= f0) bnv = P(bnw[(f & 1) * kYzThreads]);
        if (f < f1) cp_async_elem(bnw + ((f + 1) & 1) * kYzThreads, V.bn + lc + V.st);
      }
      cell_states_from<R, CHAR, P>(A, V, lc, aL, aR, WindowStencil<RE, P>{col, V, lc, f < f1});
      cp_async_commit();
    } else {
      cell_states<R, CHAR, P>(A, V, lc, aL, aR);
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) park[n * kYzThreads + t] = aR[n];
    if (f >= f0) {
      if constexpr (PFB) face_flux<S, P>(A, V, lc, wl, aL, bnv);
      else face_flux<S, P>(A, V, lc, wl, aL);
    }
#pragma unroll
    for (int n = 0; n < 8; ++n) wl[n] = park[n * kYzThreads + t];
  }
}

// Resident 128-thread blocks per SM the x-sweep kernel is compiled for (register cap), in two
// variants that the autotuner chooses between per scheme, precision and mesh: V = 0 at 5
// (FP64, 96 registers) / 10 (FP32, 48 registers) blocks, V = 1 at 6 / 12 blocks (more
// resident warps to hide the FP64 / FP32 latency, fewer registers, some spilling to L1).
#ifndef CHQ_FLUX_MINB_D
#define CHQ_FLUX_MINB_D 5
#endif
#ifndef CHQ_FLUX_MINB_F
#define CHQ_FLUX_MINB_F 10
#endif
template <class P, int V = 0> struct FluxMinBlocks {
  static constexpr int v = (sizeof(P) == 8) ? CHQ_FLUX_MINB_D + V : CHQ_FLUX_MINB_F + 2 * V;
};
constexpr int kFluxXVariants = 2;

// Single-mesh launches split by sweep: the x-sweep kernel needs no shared window, so it keeps
// the full L1 and the register cap above; the y/z kernel holds 8 + 8(2RE+1) shared columns
// per thread (48 KB per block in FP64 PPM / PPMX / WENO-Z), which sets its residency.
#ifndef CHQ_FLUXYZ_MINB_D
#define CHQ_FLUXYZ_MINB_D 4
#endif
#ifndef CHQ_FLUXYZ_MINB_F
#define CHQ_FLUXYZ_MINB_F 8
#endif
template <class P> struct FluxYzMinBlocks { static constexpr int v = (sizeof(P) == 8) ? CHQ_FLUXYZ_MINB_D : CHQ_FLUXYZ_MINB_F; };

template <int R, class P> __host__ __device__ constexpr size_t flux_yz_smem() {
  // park (8) + window: streaming PPM 43 slots (the characteristic PPM form uses 40 of them),
  // otherwise 8 quantities x (2 reach + 1); in FP64 every windowed march adds two face-field slots
  return (size_t)(8 + ((R == R_PPM) ? PpmWin::nslot : (Reach<R>::v > 0) ? 8 * (2 * Reach<R>::v + 1) : 0)) *
             kYzThreads * sizeof(P) +
         ((Reach<R>::v > 0 && sizeof(P) == 8) ? 2 * kYzThreads * sizeof(double) : 0);
}

template <int R, int S, bool CHAR, class P, int V = 0>
__global__ void __launch_bounds__(128, (FluxMinBlocks<P, V>::v)) flux_x_kernel(const FluxArgs<P> A) {
  if (A.skip && *A.skip) return;
  const int wid = (int)blockIdx.x * 4 + (int)(threadIdx.x >> 5);
  if (wid < (int)A.nwarp[0]) {
    if constexpr (R == R_PPM && !CHAR) sweep_x_ppm<S, P>(A, wid);
    else sweep_x<R, S, CHAR, P>(A, wid);
  }
}

template <int R, int S, bool CHAR, class P>
__global__ void __launch_bounds__(kYzThreads, FluxYzMinBlocks<P>::v) flux_yz_kernel(const FluxArgs<P> A) {
  extern __shared__ __align__(16) unsigned char flux_dsm[];
  P *park = reinterpret_cast<P *>(flux_dsm);
  P *win = park + 8 * kYzThreads;
  if (A.skip && *A.skip) return;
  const int wid = (int)blockIdx.x * (kYzThreads / 32) + (int)(threadIdx.x >> 5);
  const int nz = (int)A.nwarp[2], nyz = (int)(A.nwarp[2] + A.nwarp[1]);
  if (wid < nz) sweep_yz<R, S, CHAR, true, P>(A, 2, wid, park, win);
  else if (wid < nyz) sweep_yz<R, S, CHAR, true, P>(A, 1, wid - nz, park, win);
}

// The FP64 streaming-PPM y/z kernel with TMA staging (FluxArgs::yzvar = 1): dynamic shared
// memory of flux_yz_kernel plus one mbarrier per warp; the tensor maps are kernel parameters.
constexpr size_t flux_yz_tma_smem() { return flux_yz_smem<R_PPM, double>() + (kYzThreads / 32) * sizeof(unsigned long long); }

template <int S>
__global__ void __launch_bounds__(kYzThreads, FluxYzMinBlocks<double>::v)
    flux_yz_tma_kernel(const __grid_constant__ FluxArgs<double> A, const __grid_constant__ YzMaps maps) {
  extern __shared__ __align__(128) unsigned char flux_tma_dsm[];
  double *park = reinterpret_cast<double *>(flux_tma_dsm);
  double *win = park + 8 * kYzThreads;
  unsigned long long *mbar = reinterpret_cast<unsigned long long *>(flux_tma_dsm + flux_yz_smem<R_PPM, double>());
  if (A.skip && *A.skip) return;
  const int wid = (int)blockIdx.x * (kYzThreads / 32) + (int)(threadIdx.x >> 5);
  const int nz = (int)A.nwarp[2], nyz = (int)(A.nwarp[2] + A.nwarp[1]);
  if (wid < nz) sweep_yz_ppm<S, double, true>(A, 2, wid, park, win, &maps, mbar);
  else if (wid < nyz) sweep_yz_ppm<S, double, true>(A, 1, wid - nz, park, win, &maps, mbar);
}

// batched forms: the blocks of many meshes in one launch per sweep kind (chq_batch); each
// block copies its mesh's arguments to shared memory first
template <int R, int S, bool CHAR, class P, int V = 0>
__global__ void __launch_bounds__(128, (FluxMinBlocks<P, V>::v)) flux_x_batched(const FluxArgs<P> *args, const BatchSlot *slots, int n) {
  __shared__ __align__(16) unsigned char sa[sizeof(FluxArgs<P>)];
  const int j = batch_job(slots, n, blockIdx.x);
  const FluxArgs<P> &A = stage_args(args, j, sa);
  if (A.skip && *A.skip) return;
  const int wid = (int)(blockIdx.x - slots[j].off) * 4 + (int)(threadIdx.x >> 5);
  if (wid < (int)A.nwarp[0]) {
    if constexpr (R == R_PPM && !CHAR) sweep_x_ppm<S, P>(A, wid);
    else sweep_x<R, S, CHAR, P>(A, wid);
  }
}

template <int R, class P> __host__ __device__ constexpr size_t flux_yz_batched_smem() {
  return flux_yz_smem<R, P>() + (sizeof(FluxArgs<P>) + 15) / 16 * 16;
}

template <int R, int S, bool CHAR, class P>
__global__ void __launch_bounds__(kYzThreads, FluxYzMinBlocks<P>::v) flux_yz_batched(const FluxArgs<P> *args, const BatchSlot *slots, int n) {
  extern __shared__ __align__(16) unsigned char flux_dsm[];
  P *park = reinterpret_cast<P *>(flux_dsm);
  P *win = park + 8 * kYzThreads;
  const int j = batch_job(slots, n, blockIdx.x);
  const FluxArgs<P> &A = stage_args(args, j, flux_dsm + flux_yz_smem<R, P>());
  if (A.skip && *A.skip) return;
  const int wid = (int)(blockIdx.x - slots[j].off) * (kYzThreads / 32) + (int)(threadIdx.x >> 5);
  const int nz = (int)A.nwarp[2], nyz = (int)(A.nwarp[2] + A.nwarp[1]);
  if (wid < nz) sweep_yz<R, S, CHAR, true, P>(A, 2, wid, park, win);
  else if (wid < nyz) sweep_yz<R, S, CHAR, true, P>(A, 1, wid - nz, park, win);
}

}  // namespace chq
