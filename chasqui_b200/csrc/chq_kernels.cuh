// chasqui_b200 — the stage kernels other than the face fluxes:
//   K2  corner_emf_kernel   upwind edge EMFs (Gardiner & Stone 2005)   src/physics.hpp:228-297
//   K3  update_kernel       RK combination + flux divergence + CT     src/physics.hpp:299-348
//       fofc_flag_kernel    FOFC test of the tentative state + count   src/fofc.hpp:17-43
//       fofc_repair_kernel  DC + HLLE fluxes on faces of flagged cells  src/fofc.hpp:46-95
//       limit_kernel        Hu-Adams-Shu positivity flux limiter        src/positivity.hpp:25-88
//   K4  bc_kernel<dir>      periodic / outflow / reflect ghost fill     src/physics.hpp:354-432
//   K5  c2p_kernel          con2prim + centred B + cell EMF + dt min    src/physics.hpp:437-494
//       history kernels     the .hst sums and div B                     src/output.hpp:91-119
// P is the storage/arithmetic type of primitives, fluxes and EMFs (double in the FP64 form,
// float in the mixed form); conserved variables and face fields are always double.
#pragma once
#include "chq_common.cuh"
#include "chq_riemann.cuh"
#include "chq_ctl.cuh"
#include "chq_diffusion.cuh"

namespace chq {

// ---------------------------------------------------------------------------------------
// K2
template <class P> struct EmfArgs {
  Geom g;
  const P *f1, *f2, *f3;                           // mass flux = component 0 of each
  const P *e2x1, *e3x1, *e1x2, *e3x2, *e1x3, *e2x3;
  const P *ecc;
  P *e1, *e2, *e3;
  const int *done;   // skip when nonzero
  const int *need;   // run only when *need != 0 (FOFC re-run); null = always
  const int *list;   // FOFC re-run: the stage's flagged cells (count *need, first `cap` listed)
  int cap;
};

template <class P> CHQ_D P upwind(P flux, P left, P right) {
  const P tol = P(1e-14);
  return (flux > tol) ? left : (flux < -tol) ? right : P(0.5) * (left + right);
}

// The edge EMFs stored at point (k, j, i): E1 at (k-1/2, j-1/2, i), E2 at (k-1/2, j, i-1/2),
// E3 at (k, j-1/2, i-1/2), each where it is in range (src/physics.hpp:242-297).
template <class P> CHQ_D void corner_point(const EmfArgs<P> &A, int k, int j, int i) {
  const Geom &g = A.g;
  const long vs = g.vstride;
  const long sj = g.sj, sk = g.sk;
  if (i > g.ie + 1) return;
  const long l = g.idx(k, j, i);
  if (g.three_d) {
    if (j > g.je + 1 || k > g.ke + 1) return;
    const P *c0 = A.ecc, *c1 = A.ecc + vs, *c2 = A.ecc + 2 * vs;
    if (i <= g.ie) {   // E1 on x1-edges (k-1/2, j-1/2, i)
      const P l3 = upwind(ldg(A.f2 + l - sk), ldg(A.e1x3 + l - sj) - ldg(c0 + l - sk - sj), ldg(A.e1x3 + l) - ldg(c0 + l - sk));
      const P r3 = upwind(ldg(A.f2 + l), ldg(A.e1x3 + l - sj) - ldg(c0 + l - sj), ldg(A.e1x3 + l) - ldg(c0 + l));
      const P l2 = upwind(ldg(A.f3 + l - sj), ldg(A.e1x2 + l - sk) - ldg(c0 + l - sk - sj), ldg(A.e1x2 + l) - ldg(c0 + l - sj));
      const P r2 = upwind(ldg(A.f3 + l), ldg(A.e1x2 + l - sk) - ldg(c0 + l - sk), ldg(A.e1x2 + l) - ldg(c0 + l));
      A.e1[l] = P(0.25) * (((l3 + r3) + (l2 + r2)) + ((ldg(A.e1x2 + l - sk) + ldg(A.e1x2 + l)) + (ldg(A.e1x3 + l - sj) + ldg(A.e1x3 + l))));
    }
    if (j <= g.je) {   // E2 on x2-edges (k-1/2, j, i-1/2)
      const P l3 = upwind(ldg(A.f1 + l - sk), ldg(A.e2x3 + l - 1) - ldg(c1 + l - sk - 1), ldg(A.e2x3 + l) - ldg(c1 + l - sk));
      const P r3 = upwind(ldg(A.f1 + l), ldg(A.e2x3 + l - 1) - ldg(c1 + l - 1), ldg(A.e2x3 + l) - ldg(c1 + l));
      const P l1 = upwind(ldg(A.f3 + l - 1), ldg(A.e2x1 + l - sk) - ldg(c1 + l - sk - 1), ldg(A.e2x1 + l) - ldg(c1 + l - 1));
      const P r1 = upwind(ldg(A.f3 + l), ldg(A.e2x1 + l - sk) - ldg(c1 + l - sk), ldg(A.e2x1 + l) - ldg(c1 + l));
      A.e2[l] = P(0.25) * (((l3 + r3) + (l1 + r1)) + ((ldg(A.e2x3 + l - 1) + ldg(A.e2x3 + l)) + (ldg(A.e2x1 + l - sk) + ldg(A.e2x1 + l))));
    }
    if (k <= g.ke) {   // E3 on x3-edges (k, j-1/2, i-1/2)
      const P l2 = upwind(ldg(A.f1 + l - sj), ldg(A.e3x2 + l - 1) - ldg(c2 + l - sj - 1), ldg(A.e3x2 + l) - ldg(c2 + l - sj));
      const P r2 = upwind(ldg(A.f1 + l), ldg(A.e3x2 + l - 1) - ldg(c2 + l - 1), ldg(A.e3x2 + l) - ldg(c2 + l));
      const P l1 = upwind(ldg(A.f2 + l - 1), ldg(A.e3x1 + l - sj) - ldg(c2 + l - sj - 1), ldg(A.e3x1 + l) - ldg(c2 + l - 1));
      const P r1 = upwind(ldg(A.f2 + l), ldg(A.e3x1 + l - sj) - ldg(c2 + l - sj), ldg(A.e3x1 + l) - ldg(c2 + l));
      A.e3[l] = P(0.25) * (((l2 + r2) + (l1 + r1)) + ((ldg(A.e3x2 + l - 1) + ldg(A.e3x2 + l)) + (ldg(A.e3x1 + l - sj) + ldg(A.e3x1 + l))));
    }
  } else {
    // 2D / 1D: E1 and E2 live on x3-edges that coincide with the x2- and x1-faces
    if (j > g.je + 1) return;
    const P a = ldg(A.e1x2 + l), b = ldg(A.e2x1 + l);
    A.e1[l] = a; A.e1[l + sk] = a;
    A.e2[l] = b; A.e2[l + sk] = b;
    if (!g.two_d) {
      if (j == g.js) {
        const P c = ldg(A.e3x1 + l);
        A.e3[l] = c;
        A.e3[l + sj] = c;
      }
    } else {
      const P *c2 = A.ecc + 2 * vs;
      const P l2 = upwind(ldg(A.f1 + l - sj), ldg(A.e3x2 + l - 1) - ldg(c2 + l - sj - 1), ldg(A.e3x2 + l) - ldg(c2 + l - sj));
      const P r2 = upwind(ldg(A.f1 + l), ldg(A.e3x2 + l - 1) - ldg(c2 + l - 1), ldg(A.e3x2 + l) - ldg(c2 + l));
      const P l1 = upwind(ldg(A.f2 + l - 1), ldg(A.e3x1 + l - sj) - ldg(c2 + l - sj - 1), ldg(A.e3x1 + l) - ldg(c2 + l - 1));
      const P r1 = upwind(ldg(A.f2 + l), ldg(A.e3x1 + l - sj) - ldg(c2 + l - sj), ldg(A.e3x1 + l) - ldg(c2 + l));
      A.e3[l] = P(0.25) * (((l2 + r2) + (l1 + r1)) + ((ldg(A.e3x2 + l - 1) + ldg(A.e3x2 + l)) + (ldg(A.e3x1 + l - sj) + ldg(A.e3x1 + l))));
    }
  }
}

template <class P> CHQ_D void corner_emf_body(const EmfArgs<P> &A, int bx, int by, int bz) {
  if (A.done && *A.done) return;
  if (A.need && *A.need == 0) return;
  const Geom &g = A.g;
  corner_point<P>(A, g.ks + bz, g.js + by * (int)blockDim.y + (int)threadIdx.y, g.is + bx * (int)blockDim.x + (int)threadIdx.x);
}

template <class P> __global__ void __launch_bounds__(256) corner_emf_kernel(const EmfArgs<P> A) { corner_emf_body<P>(A, blockIdx.x, blockIdx.y, blockIdx.z); }

// FOFC re-run of the corner EMFs (no explicit diffusion: the edges are overwritten, never
// accumulated). A repaired face is a face of a listed cell and only the edges of the repaired
// faces see new inputs, so recomputing the points of the listed cells' edges (k..k+1, j..j+1,
// i..i+1; k..k only below 3D) gives every edge the value a full re-run gives it; the other
// edges keep values equal to it. Without a usable list every point is recomputed.
template <class P> CHQ_D void corner_rerun_body(const EmfArgs<P> &A, int bx, int nbx) {
  if (A.done && *A.done) return;
  const int nb = *A.need;
  if (nb == 0) return;
  const Geom &g = A.g;
  const int tid = bx * (int)blockDim.x + (int)threadIdx.x, nth = nbx * (int)blockDim.x;
  const int nzk = g.three_d ? 2 : 1;
  if (A.list && nb > 0 && nb <= A.cap) {
    const int per = 4 * nzk, sj = (int)g.sj, sk = (int)g.sk;
    for (int it = tid; it < per * nb; it += nth) {
      const int q = it / per, p = it - per * q;
      const int c = A.list[q];
      const int k = c / sk, r = c - k * sk, j = r / sj, i = r - j * sj;
      corner_point<P>(A, k + (p >> 2), j + ((p >> 1) & 1), i + (p & 1));
    }
    return;
  }
  const int ni = g.ie + 2 - g.is, nj = g.je + 2 - g.js, nk = g.three_d ? g.ke + 2 - g.ks : 1;
  const long tot = (long)ni * nj * nk;
  for (long t = tid; t < tot; t += nth) {
    const int i = g.is + (int)(t % ni);
    const long r = t / ni;
    corner_point<P>(A, g.ks + (int)(r / nj), g.js + (int)(r % nj), i);
  }
}

template <class P> __global__ void __launch_bounds__(256) corner_rerun_kernel(const EmfArgs<P> A) {
  corner_rerun_body<P>(A, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------------------
// K3. Each thread owns one (k, j, i) of the face/edge frame: the cell update when (k, j, i)
// is an active cell and the x1/x2/x3 face updates when it is an active face. The reads of
// ua/ub/b?a/b?b precede this thread's writes to the same elements and no other thread
// touches them, so the RK aliasing of out with a or b is safe.
// gravity source of the update epilogue (src/srcterms.hpp:10-41)
struct GravityP {
  int on, point;
  double g1, g2, g3, gm, x0, y0, z0, rsoft;
};

template <class P> struct UpdateArgs {
  Geom g;
  GravityP grav;
  const P *w;                // stage primitives (gravity only)
  EOSp eos;
  const P *f1, *f2, *f3, *e1, *e2, *e3;
  const double *ua, *ub;
  double *uout;
  const double *b1a, *b2a, *b3a, *b1b, *b2b, *b3b;
  double *b1o, *b2o, *b3o;
  double g0, g1, beta_dt;    // used when beta_dt_dev is null
  const double *beta_dt_dev; // device beta*dt of this stage (StepCtl::beta_dt[s])
  double idx1, idx2, idx3;
  const int *done;
  const int *need;           // run only when *need > need_min (FOFC re-run); null = always
  int need_min;
  const int *list;           // flagged cells of the stage (update_rerun_listed_kernel)
  int cap;                   // list capacity
};

// new face fields; curl of the edge EMFs (src/physics.hpp:327-347)
template <class P> CHQ_D double new_b1(const UpdateArgs<P> &A, long l, double g0, double g1, double bdt) {
  const Geom &g = A.g;
  double curl = 0.0;
  if (g.two_d) curl += ((double)ldg(A.e3 + l + g.sj) - (double)ldg(A.e3 + l)) * A.idx2;
  if (g.three_d) curl -= ((double)ldg(A.e2 + l + g.sk) - (double)ldg(A.e2 + l)) * A.idx3;
  return g0 * A.b1a[l] + g1 * A.b1b[l] - bdt * curl;
}
template <class P> CHQ_D double new_b2(const UpdateArgs<P> &A, long l, double g0, double g1, double bdt) {
  const Geom &g = A.g;
  double curl = -((double)ldg(A.e3 + l + 1) - (double)ldg(A.e3 + l)) * A.idx1;
  if (g.three_d) curl += ((double)ldg(A.e1 + l + g.sk) - (double)ldg(A.e1 + l)) * A.idx3;
  return g0 * A.b2a[l] + g1 * A.b2b[l] - bdt * curl;
}
template <class P> CHQ_D double new_b3(const UpdateArgs<P> &A, long l, double g0, double g1, double bdt) {
  const Geom &g = A.g;
  double curl = ((double)ldg(A.e2 + l + 1) - (double)ldg(A.e2 + l)) * A.idx1;
  if (g.two_d) curl -= ((double)ldg(A.e1 + l + g.sj) - (double)ldg(A.e1 + l)) * A.idx2;
  return g0 * A.b3a[l] + g1 * A.b3b[l] - bdt * curl;
}

// GRAV: compile the gravity epilogue (a separate instantiation keeps the plain update's
// register count, and with it its occupancy, unchanged)
// The update of one point (k, j, i) of the face/edge frame, is <= i <= ie+1 (and so on).
template <class P, bool GRAV = false> CHQ_D void update_point(const UpdateArgs<P> &A, int k, int j, int i, double bdt) {
  const Geom &g = A.g;
  const double g0 = A.g0, g1 = A.g1;
  const long l = g.idx(k, j, i);
  const long vs = g.vstride;
  const bool cell = (i <= g.ie && j <= g.je && k <= g.ke);
  double un[NVAR];
  if (cell) {
#pragma unroll
    for (int n = 0; n < NVAR; ++n) {
      const long ln = n * vs + l;
      double divf = ((double)ldg(A.f1 + ln + 1) - (double)ldg(A.f1 + ln)) * A.idx1;
      if (g.two_d) divf += ((double)ldg(A.f2 + ln + g.sj) - (double)ldg(A.f2 + ln)) * A.idx2;
      if (g.three_d) divf += ((double)ldg(A.f3 + ln + g.sk) - (double)ldg(A.f3 + ln)) * A.idx3;
      un[n] = g0 * A.ua[ln] + g1 * A.ub[ln] - bdt * divf;
    }
    if (GRAV && A.grav.on) {
      // ApplyGravity on the updated state with the stage primitives and beta*dt
      const GravityP &gr = A.grav;
      double a1 = gr.g1, a2 = gr.g2, a3 = gr.g3;
      if (gr.point) {
        const double dx = (g.x1min + (i - g.is + 0.5) * g.dx1) - gr.x0;
        const double dy = g.two_d ? (g.x2min + (j - g.js + 0.5) * g.dx2) - gr.y0 : 0.0;
        const double dz = g.three_d ? (g.x3min + (k - g.ks + g.koff + 0.5) * g.dx3) - gr.z0 : 0.0;
        const double r2 = dx * dx + dy * dy + dz * dz + gr.rsoft * gr.rsoft;
        const double f = -gr.gm / (r2 * sqrt(r2));
        a1 += f * dx;
        a2 += f * dy;
        a3 += f * dz;
      }
      const double d = (double)A.w[IDN * vs + l];
      un[IM1] += bdt * d * a1;
      un[IM2] += bdt * d * a2;
      un[IM3] += bdt * d * a3;
      un[IEN] += bdt * d * ((double)A.w[IVX * vs + l] * a1 + (double)A.w[IVY * vs + l] * a2 + (double)A.w[IVZ * vs + l] * a3);
    }
  }
  double nb1 = 0, nb2 = 0, nb3 = 0;
  if (j <= g.je && k <= g.ke) nb1 = new_b1(A, l, g0, g1, bdt);
  if (i <= g.ie && k <= g.ke && (g.two_d || j == g.js)) nb2 = new_b2(A, l, g0, g1, bdt);
  if (i <= g.ie && j <= g.je && (g.three_d || k == g.ks)) nb3 = new_b3(A, l, g0, g1, bdt);
  if (cell) {
#pragma unroll
    for (int n = 0; n < NVAR; ++n) A.uout[n * vs + l] = un[n];
  }
  if (j <= g.je && k <= g.ke) A.b1o[l] = nb1;
  if (i <= g.ie && k <= g.ke && (g.two_d || j == g.js)) {
    A.b2o[l] = nb2;
    if (!g.two_d) A.b2o[l + g.sj] = nb2;
  }
  if (i <= g.ie && j <= g.je && (g.three_d || k == g.ks)) {
    A.b3o[l] = nb3;
    if (!g.three_d) A.b3o[l + g.sk] = nb3;
  }
}

template <class P, bool GRAV = false> CHQ_D void update_body(const UpdateArgs<P> &A, int bx, int by, int bz) {
  if (A.done && *A.done) return;
  if (A.need && *A.need <= A.need_min) return;
  const Geom &g = A.g;
  const int i = g.is + bx * blockDim.x + threadIdx.x;
  const int j = g.js + by * blockDim.y + threadIdx.y;
  const int k = g.ks + bz;
  if (i > g.ie + 1 || j > g.je + 1 || k > g.ke + 1) return;
  update_point<P, GRAV>(A, k, j, i, A.beta_dt_dev ? *A.beta_dt_dev : A.beta_dt);
}

template <class P, bool GRAV> __global__ void __launch_bounds__(256) update_kernel(const UpdateArgs<P> A) {
  update_body<P, GRAV>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

// FOFC re-run of the update in a stage whose b-weight is zero and whose output is the
// b-state (the first stage of RK2, RK3 and SSPRK(4,3): out = u1 = ub, g1 = 0; src/main.cpp:68-91
// re-runs Update over every cell). There the re-run computes g0 ua + 0 ub - bdt div with ub
// the first pass's output: 0 ub is a zero, and the sum equals the first pass's value wherever
// the divergence and the curl are unchanged (a zero's sign can only matter when ua is -0, and
// then the first pass's output carries the sign the re-run reproduces). Only points whose
// fluxes or edge EMFs were repaired change: the listed cells and their face neighbours, and
// the faces next to the listed cells' edges, all inside the 3x3x3 points around each listed
// cell. A point shared by two listed cells is recomputed twice with equal results. A cell
// whose first-pass state was not finite keeps it (the full re-run would give NaN there too,
// or for an infinite state NaN instead of the infinity). Without a usable list (count above
// the capacity) this kernel does nothing and update_kernel with need_min = cap re-runs every
// point.
template <class P, bool GRAV> __global__ void __launch_bounds__(256) update_rerun_listed_kernel(const UpdateArgs<P> A) {
  if (A.done && *A.done) return;
  const int nb = *A.need;
  if (nb <= 0 || nb > A.cap) return;
  const Geom &g = A.g;
  const double bdt = A.beta_dt_dev ? *A.beta_dt_dev : A.beta_dt;
  const int tid = (int)(blockIdx.x * blockDim.x + threadIdx.x), nth = (int)(gridDim.x * blockDim.x);
  {
    const int rj = g.two_d ? 3 : 1, rk = g.three_d ? 3 : 1, per = 3 * rj * rk;
    const int sj = (int)g.sj, sk = (int)g.sk;
    for (int it = tid; it < per * nb; it += nth) {
      const int q = it / per, p = it - per * q;
      const int c = A.list[q];
      const int kc = c / sk, r = c - kc * sk, jc = r / sj, ic = r - jc * sj;
      const int i = ic + p % 3 - 1;
      const int j = jc + (p / 3) % rj - (rj >> 1);
      const int k = kc + p / (3 * rj) - (rk >> 1);
      if (i < g.is || i > g.ie + 1 || j < g.js || j > g.je + 1 || k < g.ks || k > g.ke + 1) continue;
      update_point<P, GRAV>(A, k, j, i, bdt);
    }
  }
}

// ---------------------------------------------------------------------------------------
// Optically thin cooling after the step (src/srcterms.hpp:43-71): dT/dt = -(gamma-1) rho
// lambda0 T^alpha integrated exactly over this cycle's dt (read from the step control) with
// the primitives of the step's end state, applied to the conserved energy of active cells.
template <class P> struct CoolArgs {
  Geom g;
  double gm1, lambda0, alpha, tfloor;
  double *u;
  const P *w;
  const double *dt;
  const int *done;
};

template <class P> CHQ_D void cooling_body(const CoolArgs<P> &A, int bx, int by, int bz) {
  if (A.done && *A.done) return;
  const Geom &g = A.g;
  const int i = g.is + bx * blockDim.x + threadIdx.x;
  const int j = g.js + by * blockDim.y + threadIdx.y;
  const int k = g.ks + bz;
  if (i > g.ie || j > g.je || k > g.ke) return;
  const long vs = g.vstride, l = g.idx(k, j, i);
  const double dt = *A.dt;
  const double d = (double)A.w[IDN * vs + l], p = (double)A.w[IPR * vs + l];
  const double t0 = p / d;
  const double cc = A.gm1 * d * A.lambda0;
  double t1;
  if (fabs(A.alpha - 1.0) < 1e-12) {
    t1 = t0 * exp(-cc * dt);
  } else {
    const double e = 1.0 - A.alpha;
    const double base = pow(t0, e) + (A.alpha - 1.0) * cc * dt;
    t1 = (base > 0.0) ? pow(base, 1.0 / e) : A.tfloor;
  }
  t1 = fmax(t1, A.tfloor);
  A.u[IEN * vs + l] += d * (t1 - t0) / A.gm1;
}

template <class P> __global__ void __launch_bounds__(256) cooling_kernel(const CoolArgs<P> A) {
  cooling_body<P>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------------------
// FOFC flag of the tentative state (src/fofc.hpp:17-43): rho <= dfloor or p <= pfloor,
// written for every active cell, with a warp-aggregated count into *nbad. The flagged cells'
// linear indices are also appended to `list` (the first `cap` of them), so that the repair
// visits only their faces.
struct FlagArgs {
  Geom g;
  EOSp eos;
  const double *u, *b1, *b2, *b3;
  int *flag;
  int *nbad;
  const int *done;
  int *list;
  int cap;
};

CHQ_D void fofc_flag_body(const FlagArgs &A, int bx, int by, int bz) {
  if (A.done && *A.done) return;
  const Geom &g = A.g;
  const int i = g.is + bx * blockDim.x + threadIdx.x;
  const int j = g.js + by * blockDim.y + threadIdx.y;
  const int k = g.ks + bz;
  int bad = 0;
  if (i <= g.ie && j <= g.je) {
    const long vs = g.vstride;
    const long l = g.idx(k, j, i);
    const double bx = 0.5 * (A.b1[l] + A.b1[l + 1]);
    const double by = g.two_d ? 0.5 * (A.b2[l] + A.b2[l + g.sj]) : A.b2[l];
    const double bz = g.three_d ? 0.5 * (A.b3[l] + A.b3[l + g.sk]) : A.b3[l];
    const double d = A.u[IDN * vs + l];
    bool b = (d <= A.eos.dfloor);
    if (!b) {
      const double ke = divz(0.5 * (sqr(A.u[IM1 * vs + l]) + sqr(A.u[IM2 * vs + l]) + sqr(A.u[IM3 * vs + l])), d);
      const double eint = A.u[IEN * vs + l] - ke - 0.5 * (bx * bx + by * by + bz * bz);
      double p = A.eos.gm1 * eint;
      if (A.eos.dual_energy && eint < A.eos.de_eta * fabs(A.u[IEN * vs + l]))
        p = (A.u[IENT * vs + l] / d) * pow(d, A.eos.gamma);
      b = (p <= A.eos.pfloor);
    }
    bad = b ? 1 : 0;
    A.flag[l] = bad;
  }
  // blockDim.x == 32: the lane is threadIdx.x
  const unsigned m = __ballot_sync(0xffffffffu, bad != 0);
  if (m) {
    int base = 0;
    if (threadIdx.x == 0) base = atomicAdd(A.nbad, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (bad && A.list) {
      const int pos = base + __popc(m & ((1u << threadIdx.x) - 1u));
      if (pos < A.cap) A.list[pos] = g.idx32(k, j, i);
    }
  }
}

__global__ void __launch_bounds__(256) fofc_flag_kernel(const FlagArgs A) { fofc_flag_body(A, blockIdx.x, blockIdx.y, blockIdx.z); }

// ---------------------------------------------------------------------------------------
// FOFC repair: first-order (donor cell) HLLE fluxes on faces touching a flagged cell,
// from the stage-start primitives (src/fofc.hpp:46-95). One launch, all directions. With
// the flag kernel's cell list (count *need <= cap) the launch visits the six faces of each
// listed cell only; otherwise it scans every face, as the reference's loop does.
template <class P> struct RepairArgs {
  Geom g;
  EOSp eos;
  const P *w, *bcc;
  const double *bn[3];
  P *flx[3], *et2[3], *et1[3];
  const int *flag;
  int lo[3][3], hi[3][3];   // flux face ranges per direction (k, j, i)
  long nface[3];
  const int *done;
  const int *need;
  int has_diff;             // re-add the diffusive fluxes on repaired active faces
  DiffArgs<P> diff;
  const int *list;          // flagged cells (linear indices) of this stage, or null
  int cap;                  // list capacity
  int kext[2];              // z slab: the ghost plane below / above holds the neighbouring slab's flags
};

template <int DIR, class P> CHQ_D void repair_face(const RepairArgs<P> &A, int k, int j, int i) {
  const Geom &g = A.g;
  constexpr int IVU = IVX + DIR, IVV = IVX + (DIR + 1) % 3, IVW = IVX + (DIR + 2) % 3;
  constexpr int IBT1 = (DIR + 1) % 3, IBT2 = (DIR + 2) % 3;
  const int kL = k - (DIR == 2), jL = j - (DIR == 1), iL = i - (DIR == 0);
  // cells of the mesh (with a z slab's neighbouring planes, which are cells of the whole mesh)
  auto inside = [&](int kk, int jj, int ii) {
    return (ii >= g.is && ii <= g.ie && jj >= g.js && jj <= g.je && kk >= g.ks - A.kext[0] && kk <= g.ke + A.kext[1]);
  };
  const long l = g.idx(k, j, i), lL = g.idx(kL, jL, iL);
  const bool fr = inside(k, j, i) && A.flag[l];
  const bool fl = inside(kL, jL, iL) && A.flag[lL];
  if (!(fl || fr)) return;
  const long vs = g.vstride;
  MState<P> L{A.w[IDN * vs + lL], A.w[IVU * vs + lL], A.w[IVV * vs + lL], A.w[IVW * vs + lL], A.w[IPR * vs + lL],
              A.bcc[IBT1 * vs + lL], A.bcc[IBT2 * vs + lL]};
  MState<P> R{A.w[IDN * vs + l], A.w[IVU * vs + l], A.w[IVV * vs + l], A.w[IVW * vs + l], A.w[IPR * vs + l],
              A.bcc[IBT1 * vs + l], A.bcc[IBT2 * vs + l]};
  P f[NFLX];
  hlle(L, R, P(A.bn[DIR][l]), P(A.eos.gamma), P(A.eos.gm1), f);
  P *flx = A.flx[DIR];
  flx[IDN * vs + l] = f[FD];
  flx[IVU * vs + l] = f[FMU];
  flx[IVV * vs + l] = f[FMV];
  flx[IVW * vs + l] = f[FMW];
  flx[IEN * vs + l] = f[FEN];
  const P sL = A.w[IENT * vs + lL], sR = A.w[IENT * vs + l];
  flx[IENT * vs + l] = (f[FD] > P(0)) ? f[FD] * sL : (f[FD] < P(0)) ? f[FD] * sR : P(0.5) * (f[FD] * (sL + sR));
  A.et2[DIR][l] = -f[FBY];
  A.et1[DIR][l] = f[FBZ];
  // diffusive fluxes exist only on the faces of active cells (src/fofc.hpp:89-93)
  if (A.has_diff) {
    const bool af = (DIR == 0) ? (i >= g.is && i <= g.ie + 1 && j >= g.js && j <= g.je && k >= g.ks && k <= g.ke)
                  : (DIR == 1) ? (j >= g.js && j <= g.je + 1 && i >= g.is && i <= g.ie && k >= g.ks && k <= g.ke)
                               : (k >= g.ks && k <= g.ke + 1 && i >= g.is && i <= g.ie && j >= g.js && j <= g.je);
    if (af) diff_face<DIR, P>(A.diff, k, j, i);
  }
}

template <class P> CHQ_D void repair_in_range(const RepairArgs<P> &A, int d, int k, int j, int i) {
  if (k < A.lo[d][0] || k > A.hi[d][0] || j < A.lo[d][1] || j > A.hi[d][1] || i < A.lo[d][2] || i > A.hi[d][2]) return;
  if (d == 0) repair_face<0, P>(A, k, j, i);
  else if (d == 1) repair_face<1, P>(A, k, j, i);
  else repair_face<2, P>(A, k, j, i);
}

// block bx of nbx blocks (grid-stride over the work)
template <class P> CHQ_D void fofc_repair_body(const RepairArgs<P> &A, int bx, int nbx) {
  if (A.done && *A.done) return;
  const int nb = A.need ? *A.need : -1;
  if (nb == 0) return;
  const int tid = bx * (int)blockDim.x + (int)threadIdx.x, nth = nbx * (int)blockDim.x;
  const Geom &g = A.g;
  if (A.list && nb > 0 && nb <= A.cap) {
    // item = 6 * cell + 2 * direction + side. A face between two flagged cells belongs to the
    // upper cell's low side only, so every face is written once (the diffusive flux is added
    // to the repaired one, which must not happen twice).
    const int sj = (int)g.sj, sk = (int)g.sk;
    for (int it = tid; it < 6 * nb; it += nth) {
      const int q = it / 6, f = it - 6 * q, d = f >> 1;
      if (A.nface[d] == 0) continue;
      const int c = A.list[q];
      int k = c / sk;
      const int r = c - k * sk;
      int j = r / sj;
      int i = r - j * sj;
      if (f & 1) {
        const int kn = k + (d == 2), jn = j + (d == 1), in = i + (d == 0);
        if (in <= g.ie && jn <= g.je && kn <= g.ke && A.flag[g.idx32(kn, jn, in)]) continue;
        k = kn;
        j = jn;
        i = in;
      }
      repair_in_range<P>(A, d, k, j, i);
    }
    return;
  }
#pragma unroll 1
  for (int d = 0; d < 3; ++d) {
    const int ni = A.hi[d][2] - A.lo[d][2] + 1, nj = A.hi[d][1] - A.lo[d][1] + 1;
    for (long t = tid; t < A.nface[d]; t += nth) {
      const int i = A.lo[d][2] + (int)(t % ni);
      const long r = t / ni;
      const int j = A.lo[d][1] + (int)(r % nj);
      const int k = A.lo[d][0] + (int)(r / nj);
      repair_in_range<P>(A, d, k, j, i);
    }
  }
}

template <class P> __global__ void __launch_bounds__(256) fofc_repair_kernel(const RepairArgs<P> A) {
  fofc_repair_body<P>(A, blockIdx.x, gridDim.x);
}

// ---------------------------------------------------------------------------------------
// Positivity flux limiter (Hu, Adams & Shu 2013) on the active faces of each direction.
template <class P> struct LimitArgs {
  Geom g;
  EOSp eos;
  const P *w, *bcc;
  P *flx[3];
  double two_ndim;              // 2 * ndim
  double dx[3];
  double beta_dt;
  const double *beta_dt_dev;
  int lo[3][3], hi[3][3];
  long nface[3];
  long long *count;
  const int *done;
  // limited faces counted per direction only for k in [kcount[d][0], kcount[d][1]]: a z slab
  // also limits the transverse faces of the ghost plane next to another slab (their mass
  // fluxes steer that plane's edge EMFs), which the neighbouring slab owns and counts
  int kcount[3][2];
};

template <class P> CHQ_D void cell_flux6(const MState<P> &s, P bn, P sent, P gm1, P gamma, P fc[6], P uc[6], P &cf) {
  P f[NFLX], e, pt;
  phys_flux(s, bn, gm1, e, pt, f);
  fc[0] = f[FD]; fc[1] = f[FMU]; fc[2] = f[FMV]; fc[3] = f[FMW]; fc[4] = f[FEN]; fc[5] = f[FD] * sent;
  uc[0] = s.d; uc[1] = s.d * s.u; uc[2] = s.d * s.v; uc[3] = s.d * s.w; uc[4] = e; uc[5] = s.d * sent;
  cf = fast_speed(s, bn, gamma);
}

template <int DIR, class P> CHQ_D int limit_face(const LimitArgs<P> &A, int k, int j, int i, double bdt) {
  const Geom &g = A.g;
  constexpr int IVU = IVX + DIR, IVV = IVX + (DIR + 1) % 3, IVW = IVX + (DIR + 2) % 3;
  constexpr int IBT1 = (DIR + 1) % 3, IBT2 = (DIR + 2) % 3;
  const long vs = g.vstride;
  const int kL = k - (DIR == 2), jL = j - (DIR == 1), iL = i - (DIR == 0);
  const long l = g.idx(k, j, i), lL = g.idx(kL, jL, iL);
  const P gamma = P(A.eos.gamma), gm1 = P(A.eos.gm1);
  // lam2 = 2 ndim beta_dt / dx, in the reference's order ((2*ndim)*beta_dt)/dx
  const P lam2 = P((A.two_ndim * bdt) / A.dx[DIR]);
  MState<P> L{A.w[IDN * vs + lL], A.w[IVU * vs + lL], A.w[IVV * vs + lL], A.w[IVW * vs + lL], A.w[IPR * vs + lL],
              A.bcc[IBT1 * vs + lL], A.bcc[IBT2 * vs + lL]};
  MState<P> R{A.w[IDN * vs + l], A.w[IVU * vs + l], A.w[IVV * vs + l], A.w[IVW * vs + l], A.w[IPR * vs + l],
              A.bcc[IBT1 * vs + l], A.bcc[IBT2 * vs + l]};
  const P bnL = A.bcc[DIR * vs + lL], bnR = A.bcc[DIR * vs + l];
  P fL[6], fR[6], uL[6], uR[6], cfL, cfR;
  cell_flux6(L, bnL, A.w[IENT * vs + lL], gm1, gamma, fL, uL, cfL);
  cell_flux6(R, bnR, A.w[IENT * vs + l], gm1, gamma, fR, uR, cfR);
  const P alpha = fmax_(fabs_(L.u) + cfL, fabs_(R.u) + cfR);
  const int nv[6] = {IDN, IVU, IVV, IVW, IEN, IENT};
  P fho[6], flf[6];
  P *flx = A.flx[DIR];
#pragma unroll
  for (int n = 0; n < 6; ++n) {
    fho[n] = flx[nv[n] * vs + l];
    flf[n] = P(0.5) * (fL[n] + fR[n]) - P(0.5) * (alpha * (uR[n] - uL[n]));
  }
  const P emL = P(0.5) * (bnL * bnL + L.by * L.by + L.bz * L.bz);
  const P emR = P(0.5) * (bnR * bnR + R.by * R.by + R.bz * R.bz);
  const P dfl = P(A.eos.dfloor), pfl = P(A.eos.pfloor), deta = P(A.eos.de_eta);
  auto ok = [&](P th) {
    P f[6];
#pragma unroll
    for (int n = 0; n < 6; ++n) f[n] = flf[n] + th * (fho[n] - flf[n]);
    P a[5], b[5];
#pragma unroll
    for (int n = 0; n < 5; ++n) {
      a[n] = uL[n] - lam2 * (f[n] - fL[n]);
      b[n] = uR[n] + lam2 * (f[n] - fR[n]);
    }
    if (a[0] < dfl || b[0] < dfl) return false;
    const P ea = a[4] - divz(P(0.5) * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]), a[0]) - emL;
    const P eb = b[4] - divz(P(0.5) * (b[1] * b[1] + b[2] * b[2] + b[3] * b[3]), b[0]) - emR;
    P pa = gm1 * ea, pb = gm1 * eb;
    if (A.eos.dual_energy) {
      const P sa = (uL[5] - lam2 * (f[5] - fL[5])) / a[0], sb = (uR[5] + lam2 * (f[5] - fR[5])) / b[0];
      if (ea < deta * fabs_(a[4])) pa = sa * P(pow((double)a[0], A.eos.gamma));
      if (eb < deta * fabs_(b[4])) pb = sb * P(pow((double)b[0], A.eos.gamma));
    }
    return (pa >= pfl && pb >= pfl);
  };
  if (ok(P(1))) return 0;
  P lo = P(0), hi = P(1);
  for (int it = 0; it < 12; ++it) {
    const P mid = P(0.5) * (lo + hi);
    if (ok(mid)) lo = mid; else hi = mid;
  }
  const P th = lo;
#pragma unroll
  for (int n = 0; n < 6; ++n) flx[nv[n] * vs + l] = flf[n] + th * (fho[n] - flf[n]);
  return 1;
}

template <class P> CHQ_D void limit_body(const LimitArgs<P> &A, int bx) {
  if (A.done && *A.done) return;
  const double bdt = A.beta_dt_dev ? *A.beta_dt_dev : A.beta_dt;
  int t = bx * (int)blockDim.x + (int)threadIdx.x;
  int lim = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (t >= 0 && t < A.nface[d]) {
      const int ni = A.hi[d][2] - A.lo[d][2] + 1, nj = A.hi[d][1] - A.lo[d][1] + 1;
      const int i = A.lo[d][2] + (int)(t % ni);
      const int r = t / ni;
      const int j = A.lo[d][1] + (int)(r % nj);
      const int k = A.lo[d][0] + (int)(r / nj);
      if (d == 0) lim = limit_face<0, P>(A, k, j, i, bdt);
      else if (d == 1) lim = limit_face<1, P>(A, k, j, i, bdt);
      else lim = limit_face<2, P>(A, k, j, i, bdt);
      if (k < A.kcount[d][0] || k > A.kcount[d][1]) lim = 0;
      t = -1;
    } else if (t >= 0) {
      t -= (int)A.nface[d];
    }
  }
  const unsigned m = __ballot_sync(__activemask(), lim != 0);
  if (m && (threadIdx.x & 31) == (__ffs(__activemask()) - 1)) atomicAdd((unsigned long long *)A.count, (unsigned long long)__popc(m));
}

template <class P> __global__ void __launch_bounds__(256) limit_kernel(const LimitArgs<P> A) { limit_body<P>(A, blockIdx.x); }

// ---------------------------------------------------------------------------------------
// K4 ghost fill; DIR selects the x1, x2 or x3 slabs. Must run x1, x2, x3 in order.
struct BcArgs {
  Geom g;
  double *u, *b1, *b2, *b3;
  int bc;
  const int *done;
  int zside;   // z sweep: bit 0 fills the lower ghosts, bit 1 the upper ones (a z slab's peer sides get halos instead)
};

template <int DIR> CHQ_D void bc_body(const BcArgs &A, int bx) {
  if (A.done && *A.done) return;
  const Geom &g = A.g;
  const long vs = g.vstride;
  const double sgn = (A.bc == BC_REFLECT) ? -1.0 : 1.0;
  if (DIR == 0) {
    // threads over (k in [0,nk], j in [0,nj], gh in [0,ng))
    const int t = bx * (int)blockDim.x + (int)threadIdx.x;
    const int gh = (int)(t % g.ng);
    const int r = t / g.ng;
    const int j = (int)(r % (g.nj + 1));
    const int k = (int)(r / (g.nj + 1));
    if (k > g.nk) return;
    const int il = gh, ir = g.ie + 1 + gh;
    const int srcl = (A.bc == 0) ? il + g.nx1 : (A.bc == 1) ? g.is : 2 * g.is - 1 - il;
    const int srcr = (A.bc == 0) ? ir - g.nx1 : (A.bc == 1) ? g.ie : 2 * g.ie + 1 - ir;
    const long row = g.idx(k, j, 0);
    if (k < g.nk && j < g.nj) {
#pragma unroll
      for (int n = 0; n < NVAR; ++n) {
        const double f = (n == IM1) ? sgn : 1.0;
        A.u[n * vs + row + il] = f * A.u[n * vs + row + srcl];
        A.u[n * vs + row + ir] = f * A.u[n * vs + row + srcr];
      }
      A.b2[row + il] = A.b2[row + srcl]; A.b2[row + ir] = A.b2[row + srcr];
      A.b3[row + il] = A.b3[row + srcl]; A.b3[row + ir] = A.b3[row + srcr];
    }
    const int fl = gh, fr = g.ie + 2 + gh;
    if (A.bc == 0) { A.b1[row + fl] = A.b1[row + fl + g.nx1]; A.b1[row + fr] = A.b1[row + fr - g.nx1]; }
    else if (A.bc == 1) { A.b1[row + fl] = A.b1[row + g.is]; A.b1[row + fr] = A.b1[row + g.ie + 1]; }
    else { A.b1[row + fl] = -A.b1[row + 2 * g.is - fl]; A.b1[row + fr] = -A.b1[row + 2 * (g.ie + 1) - fr]; }
    if (A.bc == 0 && gh == 0) A.b1[row + g.ie + 1] = A.b1[row + g.is];
  } else if (DIR == 1) {
    // threads over (k in [0,nk], gh in [0,ng), i in [0,ni])
    const int t = bx * (int)blockDim.x + (int)threadIdx.x;
    const int i = (int)(t % (g.ni + 1));
    const int r = t / (g.ni + 1);
    const int gh = (int)(r % g.ng);
    const int k = (int)(r / g.ng);
    if (k > g.nk) return;
    const int jl = gh, jr = g.je + 1 + gh;
    const int srcl = (A.bc == 0) ? jl + g.nx2 : (A.bc == 1) ? g.js : 2 * g.js - 1 - jl;
    const int srcr = (A.bc == 0) ? jr - g.nx2 : (A.bc == 1) ? g.je : 2 * g.je + 1 - jr;
    const long ljl = g.idx(k, jl, i), ljr = g.idx(k, jr, i), lsl = g.idx(k, srcl, i), lsr = g.idx(k, srcr, i);
    if (k < g.nk && i < g.ni) {
#pragma unroll
      for (int n = 0; n < NVAR; ++n) {
        const double f = (n == IM2) ? sgn : 1.0;
        A.u[n * vs + ljl] = f * A.u[n * vs + lsl];
        A.u[n * vs + ljr] = f * A.u[n * vs + lsr];
      }
      A.b3[ljl] = A.b3[lsl]; A.b3[ljr] = A.b3[lsr];
    }
    if (k < g.nk) { A.b1[ljl] = A.b1[lsl]; A.b1[ljr] = A.b1[lsr]; }
    const int fl = gh, fr = g.je + 2 + gh;
    const long lfl = g.idx(k, fl, i), lfr = g.idx(k, fr, i);
    if (A.bc == 0) { A.b2[lfl] = A.b2[g.idx(k, fl + g.nx2, i)]; A.b2[lfr] = A.b2[g.idx(k, fr - g.nx2, i)]; }
    else if (A.bc == 1) { A.b2[lfl] = A.b2[g.idx(k, g.js, i)]; A.b2[lfr] = A.b2[g.idx(k, g.je + 1, i)]; }
    else { A.b2[lfl] = -A.b2[g.idx(k, 2 * g.js - fl, i)]; A.b2[lfr] = -A.b2[g.idx(k, 2 * (g.je + 1) - fr, i)]; }
    if (A.bc == 0 && gh == 0) A.b2[g.idx(k, g.je + 1, i)] = A.b2[g.idx(k, g.js, i)];
  } else {
    // threads over (gh in [0,ng), j in [0,nj], i in [0,ni])
    const int t = bx * (int)blockDim.x + (int)threadIdx.x;
    const int i = (int)(t % (g.ni + 1));
    const int r = t / (g.ni + 1);
    const int j = (int)(r % (g.nj + 1));
    const int gh = (int)(r / (g.nj + 1));
    if (gh >= g.ng) return;
    const int kl = gh, kr = g.ke + 1 + gh;
    const int srcl = (A.bc == 0) ? kl + g.nx3 : (A.bc == 1) ? g.ks : 2 * g.ks - 1 - kl;
    const int srcr = (A.bc == 0) ? kr - g.nx3 : (A.bc == 1) ? g.ke : 2 * g.ke + 1 - kr;
    const long lkl = g.idx(kl, j, i), lkr = g.idx(kr, j, i), lsl = g.idx(srcl, j, i), lsr = g.idx(srcr, j, i);
    const bool lo = (A.zside & 1) != 0, hi = (A.zside & 2) != 0;
    if (j < g.nj && i < g.ni) {
#pragma unroll
      for (int n = 0; n < NVAR; ++n) {
        const double f = (n == IM3) ? sgn : 1.0;
        if (lo) A.u[n * vs + lkl] = f * A.u[n * vs + lsl];
        if (hi) A.u[n * vs + lkr] = f * A.u[n * vs + lsr];
      }
    }
    if (lo) { A.b1[lkl] = A.b1[lsl]; A.b2[lkl] = A.b2[lsl]; }
    if (hi) { A.b1[lkr] = A.b1[lsr]; A.b2[lkr] = A.b2[lsr]; }
    const int fl = gh, fr = g.ke + 2 + gh;
    const long lfl = g.idx(fl, j, i), lfr = g.idx(fr, j, i);
    if (A.bc == 0) {
      if (lo) A.b3[lfl] = A.b3[g.idx(fl + g.nx3, j, i)];
      if (hi) A.b3[lfr] = A.b3[g.idx(fr - g.nx3, j, i)];
    } else if (A.bc == 1) {
      if (lo) A.b3[lfl] = A.b3[g.idx(g.ks, j, i)];
      if (hi) A.b3[lfr] = A.b3[g.idx(g.ke + 1, j, i)];
    } else {
      if (lo) A.b3[lfl] = -A.b3[g.idx(2 * g.ks - fl, j, i)];
      if (hi) A.b3[lfr] = -A.b3[g.idx(2 * (g.ke + 1) - fr, j, i)];
    }
    if (A.bc == 0 && gh == 0 && lo && hi) A.b3[g.idx(g.ke + 1, j, i)] = A.b3[g.idx(g.ks, j, i)];
  }
}

template <int DIR> __global__ void __launch_bounds__(256) bc_kernel(const BcArgs A) { bc_body<DIR>(A, blockIdx.x); }

// Halo exchange of z slabs (chq_slab_pack / chq_slab_unpack): contiguous spans of 8-byte
// words copied between a slab's planes and a packed buffer, one grid row (blockIdx.y) per span.
constexpr int kHaloSpans = 12;
struct HaloArgs {
  unsigned long long *dst[kHaloSpans];
  const unsigned long long *src[kHaloSpans];
  long words[kHaloSpans];
  int nspan;
};
__global__ void __launch_bounds__(256) halo_copy_kernel(const HaloArgs A) {
  const int q = (int)blockIdx.y;
  if (q >= A.nspan) return;
  unsigned long long *d = A.dst[q];
  const unsigned long long *src = A.src[q];
  const long n = A.words[q];
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long)gridDim.x * blockDim.x) d[t] = src[t];
}

// ---------------------------------------------------------------------------------------
// K5
// .hst rows recorded on the device (chq_history_record): the con2prim of each cycle's final
// state also reduces the history sums (src/output.hpp:91-119) when that cycle reaches the next
// output time, and the row is appended to a ring the host drains.
struct HstRec {
  int due;                  // this cycle's final state is an output (set after ctl_begin)
  int count, cap, lost;     // rows in the ring, its capacity, rows dropped on a full ring
  double next, dt_hst, eps; // next output time, interval, tolerance (src/main.cpp:212)
  double vol, ncell, idx1, idx2, idx3;
  long nblk, nfold;         // K5 blocks (partials), second-level partials
  double *part, *fold;      // nblk x 10, nfold x 10
  double *rows;             // cap x 12: t, dt, mass mom1 mom2 mom3 etot ekin emag eint divB_max divB_L1
};

template <class P> struct C2pArgs {
  Geom g;
  EOSp eos;
  double *u;
  const double *b1, *b2, *b3;
  P *w, *bcc, *ecc;
  int compute_dt;
  unsigned long long *mdt_bits;   // atomic min of dt over active cells
  StepCtl *ctl;                   // when set: fold the FOFC count and reset it (block 0)
  const int *done;
  const HstRec *hst;              // K5 of a cycle's final state with recording on (HST form)
};

CHQ_D double hsq(double x) { return x * x; }

template <class P, bool HST = false> CHQ_D void c2p_body(const C2pArgs<P> &A, int bx, int by, int bz) {
  if (A.done && *A.done) return;
  // history terms of this thread's cell (active cells, output cycles, HST form only)
  double hv[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const bool hdue = HST && A.hst->due;
  const Geom &g = A.g;
  if (A.ctl && bx == 0 && by == 0 && bz == 0 && threadIdx.x == 0 && threadIdx.y == 0) {
    A.ctl->fofc_count += A.ctl->nbad;
    A.ctl->nbad = 0;
  }
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz;
  double mdt = __longlong_as_double(0x7ff0000000000000LL);   // +inf
  if (i < g.ni && j < g.nj && k < g.nk) {
    const long vs = g.vstride;
    const long l = g.idx(k, j, i);
    const double bx = 0.5 * (A.b1[l] + A.b1[l + 1]);
    const double by = g.two_d ? 0.5 * (A.b2[l] + A.b2[l + g.sj]) : A.b2[l];
    const double bz = g.three_d ? 0.5 * (A.b3[l] + A.b3[l + g.sk]) : A.b3[l];
    const EOSp &e = A.eos;
    const double d = fmax(A.u[IDN * vs + l], e.dfloor);
    const double id = 1.0 / d;
    const double vx = A.u[IM1 * vs + l] * id, vy = A.u[IM2 * vs + l] * id, vz = A.u[IM3 * vs + l] * id;
    const double bsq = bx * bx + by * by + bz * bz;
    const double ke = 0.5 * d * (vx * vx + vy * vy + vz * vz);
    const double etot = A.u[IEN * vs + l];
    const double eint = etot - ke - 0.5 * bsq;
    double p = e.gm1 * eint;
    double sent = A.u[IENT * vs + l] * id;
    double en = etot;   // the energy left in u
    if (e.dual_energy && eint < e.de_eta * fabs(etot)) {
      p = sent * pow(d, e.gamma);
      p = fmax(p, e.pfloor);
      en = ke + 0.5 * bsq + p / e.gm1;
      A.u[IEN * vs + l] = en;
    } else {
      p = fmax(p, e.pfloor);
      sent = p / pow(d, e.gamma);
      A.u[IENT * vs + l] = d * sent;
    }
    A.w[IDN * vs + l] = P(d);
    A.w[IVX * vs + l] = P(vx);
    A.w[IVY * vs + l] = P(vy);
    A.w[IVZ * vs + l] = P(vz);
    A.w[IPR * vs + l] = P(p);
    A.w[IENT * vs + l] = P(sent);
    A.bcc[0 * vs + l] = P(bx);
    A.bcc[1 * vs + l] = P(by);
    A.bcc[2 * vs + l] = P(bz);
    A.ecc[0 * vs + l] = P(vz * by - vy * bz);
    A.ecc[1 * vs + l] = P(vx * bz - vz * bx);
    A.ecc[2 * vs + l] = P(vy * bx - vx * by);
    if (A.compute_dt && i >= g.is && i <= g.ie && j >= g.js && j <= g.je && k >= g.ks && k <= g.ke) {
      const double gp = e.gamma * p;
      const double a = (gp + bsq) * id;
      auto cf = [&](double bn) {
        const double disc = a * a - 4.0 * gp * bn * bn * id * id;
        return sqrt(0.5 * (a + sqrt(fmax(disc, 0.0))));
      };
      double dt = g.dx1 / (fabs(vx) + cf(bx));
      if (g.two_d) dt = fmin(dt, g.dx2 / (fabs(vy) + cf(by)));
      if (g.three_d) dt = fmin(dt, g.dx3 / (fabs(vz) + cf(bz)));
      mdt = dt;
    }
    if (hdue && i >= g.is && i <= g.ie && j >= g.js && j <= g.je && k >= g.ks && k <= g.ke) {
      // the stored (P) primitives and centred field, as the separate history pass reads them
      const double wd = (double)P(d), wx = (double)P(vx), wy = (double)P(vy), wz = (double)P(vz);
      const double cx = (double)P(bx), cy = (double)P(by), cz = (double)P(bz);
      const HstRec &H = *A.hst;
      hv[0] = A.u[IDN * vs + l];
      hv[1] = A.u[IM1 * vs + l];
      hv[2] = A.u[IM2 * vs + l];
      hv[3] = A.u[IM3 * vs + l];
      hv[4] = en;
      hv[5] = 0.5 * wd * (hsq(wx) + hsq(wy) + hsq(wz));
      hv[6] = 0.5 * (hsq(cx) + hsq(cy) + hsq(cz));
      hv[7] = en - 0.5 * wd * (hsq(wx) + hsq(wy) + hsq(wz)) - 0.5 * (hsq(cx) + hsq(cy) + hsq(cz));
      double db = (A.b1[l + 1] - A.b1[l]) * H.idx1;
      if (g.two_d) db += (A.b2[l + g.sj] - A.b2[l]) * H.idx2;
      if (g.three_d) db += (A.b3[l + g.sk] - A.b3[l]) * H.idx3;
      hv[8] = fabs(db);
      hv[9] = fabs(db);
    }
  }
  if (A.compute_dt) block_min_pos(A.mdt_bits, mdt);   // one atomic per block (the whole block is here)
  if (hdue) {
    // fixed-order block partial. Warp level: a butterfly over the ten values padded to 16.
    // At each xor step every lane keeps half of its values, sends the other half to its
    // partner and combines (value 8 is a maximum, the rest sums), so 8 + 4 + 2 + 1 + 1
    // shuffles replace ten separate 5-step reductions; afterwards lanes 2q and 2q + 1 hold
    // value q of the warp. Then the block's 8 warps in order.
    __shared__ double hs[10][8];
    const int lane = threadIdx.x, wid = threadIdx.y;   // blockDim (32, 8)
    double v[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = (q < 10) ? hv[q] : 0.0;
    int base = 0;   // value index of v[0] on this lane
#pragma unroll
    for (int half = 8; half >= 1; half >>= 1) {
      const bool up = (lane & (2 * half)) != 0;   // this lane keeps the upper half
#pragma unroll
      for (int q = 0; q < half; ++q) {
        const double keep = up ? v[half + q] : v[q];
        const double give = up ? v[q] : v[half + q];
        const double got = __shfl_xor_sync(0xffffffffu, give, 2 * half);
        const int idx = base + (up ? half : 0) + q;
        v[q] = (idx == 8) ? fmax(keep, got) : keep + got;
      }
      base += up ? half : 0;
    }
    {
      const double got = __shfl_xor_sync(0xffffffffu, v[0], 1);
      v[0] = (base == 8) ? fmax(v[0], got) : v[0] + got;
    }
    if ((lane & 1) == 0 && base < 10) hs[base][wid] = v[0];
    __syncthreads();
    if (wid == 0 && lane < 10) {
      double r = hs[lane][0];
      for (int w = 1; w < 8; ++w) r = (lane == 8) ? fmax(r, hs[lane][w]) : r + hs[lane][w];
      const long b = ((long)bz * gridDim.y + by) * gridDim.x + bx;
      A.hst->part[b * 10 + lane] = r;
    }
  }
}

template <class P, bool HST = false>
__global__ void __launch_bounds__(256) c2p_kernel(const C2pArgs<P> A) { c2p_body<P, HST>(A, blockIdx.x, blockIdx.y, blockIdx.z); }

// Output test of the cycle just begun: its end time t + dt reaches the next output time
// (the driver's check after t += dt, src/main.cpp:212-223).
__global__ void hst_due_kernel(const StepCtl *c, HstRec *h) {
  h->due = (!c->done && c->t + c->dt >= h->next - h->eps) ? 1 : 0;
}

// Fixed-order folds of the K5 partials: block f of hst_fold_kernel folds its contiguous range
// (warp q: value q, lanes strided, then a shuffle tree), hst_commit_kernel folds the block
// results the same way and appends the scaled row (t, dt, sums) after ctl_end has advanced t.
CHQ_D double hst_fold_range(const double *src, long lo, long hi, int q, int lane) {
  double r = 0.0;
  for (long b = lo + lane; b < hi; b += 32) r = (q == 8) ? fmax(r, src[b * 10 + q]) : r + src[b * 10 + q];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double x = __shfl_down_sync(0xffffffffu, r, o);
    r = (q == 8) ? fmax(r, x) : r + x;
  }
  return r;
}
__global__ void __launch_bounds__(320) hst_fold_kernel(HstRec *h) {
  if (!h->due) return;
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long per = (h->nblk + h->nfold - 1) / h->nfold;
  const long lo = (long)blockIdx.x * per, hi = min(h->nblk, lo + per);
  const double r = hst_fold_range(h->part, lo, hi, q, lane);
  if (lane == 0) h->fold[(long)blockIdx.x * 10 + q] = r;
}
__global__ void __launch_bounds__(320) hst_commit_kernel(const StepCtl *c, HstRec *h) {
  if (!h->due) return;
  __shared__ double v[10];
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const double r = hst_fold_range(h->fold, 0, h->nfold, q, lane);
  if (lane == 0) v[q] = r;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (h->count < h->cap) {
      double *row = h->rows + (long)h->count * 12;
      row[0] = c->t;
      row[1] = c->dt;
      for (int n = 0; n < 8; ++n) row[2 + n] = v[n] * h->vol;
      row[10] = v[8];
      row[11] = v[9] / h->ncell;
      h->count += 1;
    } else {
      h->lost += 1;
    }
    h->next += h->dt_hst;
    h->due = 0;
  }
}

// ---------------------------------------------------------------------------------------
// Batched forms: the same bodies, one launch over the blocks of many meshes (chq_batch).
template <class P> __global__ void __launch_bounds__(256) corner_emf_batched(const EmfArgs<P> *args, const BatchSlot *slots, int n) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(EmfArgs<P>)];
  const EmfArgs<P> &A = stage_args(args, j, sa);
  corner_emf_body<P>(A, bx, by, bz);
}
template <class P> __global__ void __launch_bounds__(256) corner_rerun_batched(const EmfArgs<P> *args, const BatchSlot *slots, int n) {
  const int j = batch_job(slots, n, blockIdx.x);
  __shared__ __align__(16) unsigned char sa[sizeof(EmfArgs<P>)];
  const EmfArgs<P> &A = stage_args(args, j, sa);
  corner_rerun_body<P>(A, (int)(blockIdx.x - slots[j].off), slots[j].gx);
}
template <class P, bool GRAV> __global__ void __launch_bounds__(256) update_batched(const UpdateArgs<P> *args, const BatchSlot *slots, int n) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(UpdateArgs<P>)];
  const UpdateArgs<P> &A = stage_args(args, j, sa);
  update_body<P, GRAV>(A, bx, by, bz);
}
__global__ void __launch_bounds__(256) fofc_flag_batched(const FlagArgs *args, const BatchSlot *slots, int n) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(FlagArgs)];
  const FlagArgs &A = stage_args(args, j, sa);
  fofc_flag_body(A, bx, by, bz);
}
template <class P> __global__ void __launch_bounds__(256) fofc_repair_batched(const RepairArgs<P> *args, const BatchSlot *slots, int n) {
  const int j = batch_job(slots, n, blockIdx.x);
  __shared__ __align__(16) unsigned char sa[sizeof(RepairArgs<P>)];
  const RepairArgs<P> &A = stage_args(args, j, sa);
  fofc_repair_body<P>(A, (int)(blockIdx.x - slots[j].off), slots[j].gx);
}
template <class P> __global__ void __launch_bounds__(256) limit_batched(const LimitArgs<P> *args, const BatchSlot *slots, int n) {
  const int j = batch_job(slots, n, blockIdx.x);
  __shared__ __align__(16) unsigned char sa[sizeof(LimitArgs<P>)];
  const LimitArgs<P> &A = stage_args(args, j, sa);
  limit_body<P>(A, (int)(blockIdx.x - slots[j].off));
}
template <int DIR> __global__ void __launch_bounds__(256) bc_batched(const BcArgs *args, const BatchSlot *slots, int n) {
  const int j = batch_job(slots, n, blockIdx.x);
  __shared__ __align__(16) unsigned char sa[sizeof(BcArgs)];
  const BcArgs &A = stage_args(args, j, sa);
  bc_body<DIR>(A, (int)(blockIdx.x - slots[j].off));
}
template <class P> __global__ void __launch_bounds__(256) c2p_batched(const C2pArgs<P> *args, const BatchSlot *slots, int n) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(C2pArgs<P>)];
  const C2pArgs<P> &A = stage_args(args, j, sa);
  c2p_body<P>(A, bx, by, bz);
}
template <class P> __global__ void __launch_bounds__(256) cooling_batched(const CoolArgs<P> *args, const BatchSlot *slots, int n) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(CoolArgs<P>)];
  const CoolArgs<P> &A = stage_args(args, j, sa);
  cooling_body<P>(A, bx, by, bz);
}

}  // namespace chq
