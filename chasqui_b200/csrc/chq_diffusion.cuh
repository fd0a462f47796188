// chasqui_b200 — explicit non-ideal terms and the RKL2 super-time-stepping operator.
//
//   diff_flux_body   viscous (mu = rho nu), conductive (q = -kappa grad T, T = p/rho) and
//                    resistive-Poynting fluxes added on the active faces of one direction
//                    (src/diffusion.hpp:48-139)
//   resistive_emf    eta J added to the edge EMFs, J = curl B on edges from the face fields
//                    (src/diffusion.hpp:23-45, 142-156)
//   rho_min          the minimum density of the active cells, for the parabolic time step
//                    dt <= dx_min^2 / (2 ndim max(nu, eta, kappa (gamma-1)/rho_min))
//                    (src/diffusion.hpp:159-174)
//   sts_div_body     M(U) = -div F_diff and M(B) = -curl(eta J) on cells and faces
//                    (src/sts.hpp:43-90)
//   sts_combine      Y = ((a x + b y) + c z) + (d p + e q) on active cells and faces
//                    (src/sts.hpp:93-107)
// Expressions keep the reference's operation order (bitwise parity in the FP64 form).
#pragma once
#include "chq_common.cuh"
#include "chq_ctl.cuh"

namespace chq {

struct DiffCoef {
  double nu, kappa, eta;
};

// current density on edges (src/diffusion.hpp:25-45)
struct CurlB {
  const double *b1, *b2, *b3;
  double idx1, idx2, idx3;
  int two_d, three_d;
  long sj, sk;
  CHQ_D double J1(long l) const {
    double j1 = 0.0;
    if (two_d) j1 += (b3[l] - b3[l - sj]) * idx2;
    if (three_d) j1 -= (b2[l] - b2[l - sk]) * idx3;
    return j1;
  }
  CHQ_D double J2(long l) const {
    double j2 = -(b3[l] - b3[l - 1]) * idx1;
    if (three_d) j2 += (b1[l] - b1[l - sk]) * idx3;
    return j2;
  }
  CHQ_D double J3(long l) const {
    double j3 = (b2[l] - b2[l - 1]) * idx1;
    if (two_d) j3 -= (b1[l] - b1[l - sj]) * idx2;
    return j3;
  }
};

template <class P> struct DiffArgs {
  Geom g;
  DiffCoef c;
  const P *w, *bcc;
  P *flx[3];
  CurlB J;
  int lo[3][3], hi[3][3];   // active face ranges per direction (k, j, i)
  long nface[3];
  const int *done;
};

// add the diffusive fluxes of face (k, j, i) of direction DIR (FaceCtx::Add)
template <int DIR, class P> CHQ_D void diff_face(const DiffArgs<P> &A, int k, int j, int i) {
  const Geom &g = A.g;
  constexpr int IVU = IVX + DIR, IVV = IVX + (DIR + 1) % 3, IVW = IVX + (DIR + 2) % 3;
  constexpr int t1 = (DIR + 1) % 3, t2 = (DIR + 2) % 3;
  const long vs = g.vstride;
  const long st[3] = {1, g.sj, g.sk};
  const long s1 = st[t1], s2 = st[t2];
  const bool has_t1 = (t1 == 0) || (t1 == 1 && g.two_d) || (t1 == 2 && g.three_d);
  const bool has_t2 = (t2 == 0) || (t2 == 1 && g.two_d) || (t2 == 2 && g.three_d);
  const double idx[3] = {1.0 / g.dx1, 1.0 / g.dx2, 1.0 / g.dx3};
  const double idn = idx[DIR], idt1 = idx[t1], idt2 = idx[t2];
  const long l = g.idx(k, j, i), lL = l - st[DIR];
  auto W = [&](int n, long q) { return (double)A.w[n * vs + q]; };
  P *flx = A.flx[DIR];
  if (A.c.nu > 0.0) {
    const double nu = A.c.nu;
    const double mu = nu * 0.5 * (W(IDN, lL) + W(IDN, l));
    const double dun = (W(IVU, l) - W(IVU, lL)) * idn;
    const double dvn = (W(IVV, l) - W(IVV, lL)) * idn;
    const double dwn = (W(IVW, l) - W(IVW, lL)) * idn;
    double dut1 = 0, dvt1 = 0, dut2 = 0, dwt2 = 0;
    if (has_t1) {
      dut1 = 0.25 * idt1 * ((W(IVU, l + s1) - W(IVU, l - s1)) + (W(IVU, lL + s1) - W(IVU, lL - s1)));
      dvt1 = 0.25 * idt1 * ((W(IVV, l + s1) - W(IVV, l - s1)) + (W(IVV, lL + s1) - W(IVV, lL - s1)));
    }
    if (has_t2) {
      dut2 = 0.25 * idt2 * ((W(IVU, l + s2) - W(IVU, l - s2)) + (W(IVU, lL + s2) - W(IVU, lL - s2)));
      dwt2 = 0.25 * idt2 * ((W(IVW, l + s2) - W(IVW, l - s2)) + (W(IVW, lL + s2) - W(IVW, lL - s2)));
    }
    const double divv = dun + dvt1 + dwt2;
    const double tnn = mu * (2.0 * dun - (2.0 / 3.0) * divv);
    const double tnt1 = mu * (dvn + dut1);
    const double tnt2 = mu * (dwn + dut2);
    const double uf = 0.5 * (W(IVU, lL) + W(IVU, l));
    const double vf = 0.5 * (W(IVV, lL) + W(IVV, l));
    const double wf = 0.5 * (W(IVW, lL) + W(IVW, l));
    flx[IVU * vs + l] = (P)((double)flx[IVU * vs + l] - tnn);
    flx[IVV * vs + l] = (P)((double)flx[IVV * vs + l] - tnt1);
    flx[IVW * vs + l] = (P)((double)flx[IVW * vs + l] - tnt2);
    flx[IEN * vs + l] = (P)((double)flx[IEN * vs + l] - (tnn * uf + tnt1 * vf + tnt2 * wf));
  }
  if (A.c.kappa > 0.0) {
    const double tL = W(IPR, lL) / W(IDN, lL), tR = W(IPR, l) / W(IDN, l);
    flx[IEN * vs + l] = (P)((double)flx[IEN * vs + l] - A.c.kappa * (tR - tL) * idn);
  }
  if (A.c.eta > 0.0) {
    const double eta = A.c.eta;
    const CurlB &J = A.J;
    double et1, et2;
    if (DIR == 0) {
      et1 = eta * 0.5 * (J.J2(l) + (has_t2 ? J.J2(l + g.sk) : J.J2(l)));
      et2 = eta * 0.5 * (J.J3(l) + (has_t1 ? J.J3(l + g.sj) : J.J3(l)));
    } else if (DIR == 1) {
      et1 = eta * 0.5 * (J.J3(l) + J.J3(l + 1));
      et2 = eta * 0.5 * (J.J1(l) + (has_t1 ? J.J1(l + g.sk) : J.J1(l)));
    } else {
      et1 = eta * 0.5 * (J.J1(l) + J.J1(l + g.sj));
      et2 = eta * 0.5 * (J.J2(l) + J.J2(l + 1));
    }
    const double bt1 = 0.5 * ((double)A.bcc[t1 * vs + lL] + (double)A.bcc[t1 * vs + l]);
    const double bt2 = 0.5 * ((double)A.bcc[t2 * vs + lL] + (double)A.bcc[t2 * vs + l]);
    flx[IEN * vs + l] = (P)((double)flx[IEN * vs + l] + (et1 * bt2 - et2 * bt1));
  }
}

template <class P> CHQ_D void diff_flux_body(const DiffArgs<P> &A, int bx) {
  if (A.done && *A.done) return;
  int t = bx * (int)blockDim.x + (int)threadIdx.x;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (t < A.nface[d]) {
      const int ni = A.hi[d][2] - A.lo[d][2] + 1, nj = A.hi[d][1] - A.lo[d][1] + 1;
      const int i = A.lo[d][2] + (int)(t % ni);
      const int r = t / ni;
      const int j = A.lo[d][1] + (int)(r % nj);
      const int k = A.lo[d][0] + (int)(r / nj);
      if (d == 0) diff_face<0, P>(A, k, j, i);
      else if (d == 1) diff_face<1, P>(A, k, j, i);
      else diff_face<2, P>(A, k, j, i);
      return;
    }
    t -= (int)A.nface[d];
  }
}

template <class P> __global__ void __launch_bounds__(256) diff_flux_kernel(const DiffArgs<P> A) { diff_flux_body<P>(A, blockIdx.x); }

template <class P> __global__ void __launch_bounds__(256) diff_flux_batched(const DiffArgs<P> *args, const BatchSlot *slots, int n) {
  const int j = batch_job(slots, n, blockIdx.x);
  __shared__ __align__(16) unsigned char sa[sizeof(DiffArgs<P>)];
  const DiffArgs<P> &A = stage_args(args, j, sa);
  diff_flux_body<P>(A, (int)(blockIdx.x - slots[j].off));
}

// eta J added to the edge EMFs (ResistiveEMF); threads over k in [ks, ku], j in [js, ju],
// i in [is, ie+1] with ku = ke+1 (3D) or ks+1, ju = je+1 (2D) or js+1
template <class P> struct ResEmfArgs {
  Geom g;
  double eta;
  CurlB J;
  P *e1, *e2, *e3;
  int ku, ju;
  const int *done;
  const int *need;   // when set: run only if *need != 0 (the FOFC re-run)
};

template <class P> CHQ_D void resistive_emf_body(const ResEmfArgs<P> &A, int bx, int by, int bz) {
  if (A.done && *A.done) return;
  if (A.need && *A.need == 0) return;
  const Geom &g = A.g;
  const int i = g.is + bx * blockDim.x + threadIdx.x;
  const int j = g.js + by * blockDim.y + threadIdx.y;
  const int k = g.ks + bz;
  if (i > g.ie + 1 || j > A.ju || k > A.ku) return;
  const long l = g.idx(k, j, i);
  if (i <= g.ie) A.e1[l] = (P)((double)A.e1[l] + A.eta * A.J.J1(l));
  if (j <= g.je || !g.two_d) A.e2[l] = (P)((double)A.e2[l] + A.eta * A.J.J2(l));
  if (k <= g.ke || !g.three_d) A.e3[l] = (P)((double)A.e3[l] + A.eta * A.J.J3(l));
}

template <class P> __global__ void __launch_bounds__(256) resistive_emf_kernel(const ResEmfArgs<P> A) {
  resistive_emf_body<P>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <class P> __global__ void __launch_bounds__(256) resistive_emf_batched(const ResEmfArgs<P> *args, const BatchSlot *slots, int n) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(ResEmfArgs<P>)];
  const ResEmfArgs<P> &A = stage_args(args, j, sa);
  resistive_emf_body<P>(A, bx, by, bz);
}

// minimum density over the active cells into *bits (atomic min of positive doubles)
template <class P> struct RhoMinArgs {
  Geom g;
  const P *w;
  unsigned long long *bits;
  const int *done;
};

template <class P> CHQ_D void rho_min_body(const RhoMinArgs<P> &A, int bx, int by, int bz) {
  const Geom &g = A.g;
  const P *w = A.w;
  unsigned long long *bits = A.bits;
  if (A.done && *A.done) return;
  const int i = g.is + bx * blockDim.x + threadIdx.x;
  const int j = g.js + by * blockDim.y + threadIdx.y;
  const int k = g.ks + bz;
  double v = __longlong_as_double(0x7ff0000000000000LL);
  if (i <= g.ie && j <= g.je) v = (double)w[g.idx(k, j, i)];
  block_min_pos(bits, v);   // one atomic per block (the whole block is here)
}

template <class P> __global__ void __launch_bounds__(256) rho_min_kernel(const RhoMinArgs<P> A) {
  rho_min_body<P>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

template <class P> __global__ void __launch_bounds__(256) rho_min_batched(const RhoMinArgs<P> *args, const BatchSlot *slots, int n) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(RhoMinArgs<P>)];
  const RhoMinArgs<P> &A = stage_args(args, j, sa);
  rho_min_body<P>(A, bx, by, bz);
}

// M(U) = -div F and M(B) = -curl E over the update ranges (sts_div)
template <class P> struct StsDivArgs {
  Geom g;
  const P *f1, *f2, *f3, *e1, *e2, *e3;
  double *mu, *mb1, *mb2, *mb3;
  double idx1, idx2, idx3;
  const int *done;   // batched RKL2: this member takes no stage here
};

template <class P> CHQ_D void sts_div_body(const StsDivArgs<P> &A, int bx, int by, int bz) {
  if (A.done && *A.done) return;
  const Geom &g = A.g;
  const int i = g.is + bx * blockDim.x + threadIdx.x;
  const int j = g.js + by * blockDim.y + threadIdx.y;
  const int k = g.ks + bz;
  if (i > g.ie + 1 || j > g.je + 1 || k > g.ke + 1) return;
  const long l = g.idx(k, j, i);
  const long vs = g.vstride;
  if (i <= g.ie && j <= g.je && k <= g.ke) {
    for (int n = 0; n < NVAR; ++n) {
      const long ln = n * vs + l;
      double d = ((double)A.f1[ln + 1] - (double)A.f1[ln]) * A.idx1;
      if (g.two_d) d += ((double)A.f2[ln + g.sj] - (double)A.f2[ln]) * A.idx2;
      if (g.three_d) d += ((double)A.f3[ln + g.sk] - (double)A.f3[ln]) * A.idx3;
      A.mu[ln] = -d;
    }
  }
  if (j <= g.je && k <= g.ke) {
    double c = 0.0;
    if (g.two_d) c += ((double)A.e3[l + g.sj] - (double)A.e3[l]) * A.idx2;
    if (g.three_d) c -= ((double)A.e2[l + g.sk] - (double)A.e2[l]) * A.idx3;
    A.mb1[l] = -c;
  }
  if (i <= g.ie && k <= g.ke && (g.two_d || j == g.js)) {
    double c = -((double)A.e3[l + 1] - (double)A.e3[l]) * A.idx1;
    if (g.three_d) c += ((double)A.e1[l + g.sk] - (double)A.e1[l]) * A.idx3;
    A.mb2[l] = -c;
    if (!g.two_d) A.mb2[l + g.sj] = -c;
  }
  if (i <= g.ie && j <= g.je && (g.three_d || k == g.ks)) {
    double c = ((double)A.e2[l + 1] - (double)A.e2[l]) * A.idx1;
    if (g.two_d) c -= ((double)A.e1[l + g.sj] - (double)A.e1[l]) * A.idx2;
    A.mb3[l] = -c;
    if (!g.three_d) A.mb3[l + g.sk] = -c;
  }
}

template <class P> __global__ void __launch_bounds__(256) sts_div_kernel(const StsDivArgs<P> A) {
  sts_div_body<P>(A, blockIdx.x, blockIdx.y, blockIdx.z);
}

// out = ((a x + b y) + c z) + (d p + e q) on active cells (6 components) and on the faces of
// the update range (3 face fields); coefficients in double as the reference's Real
struct StsCombArgs {
  Geom g;
  double a, b, c, d, e;
  double *out;
  const double *x, *y, *z, *p, *q;           // cell arrays (6 components)
  double *bo[3];
  const double *bx[3], *by[3], *bz[3], *bp[3], *bq[3];
  const int *done;   // batched RKL2: this member takes no stage here
};

// cf: the five coefficients (a, b, c, d, e)
CHQ_D void sts_combine_body(const StsCombArgs &A, const double *cf, int bx, int by, int bz) {
  if (A.done && *A.done) return;
  const Geom &g = A.g;
  const int i = g.is + bx * blockDim.x + threadIdx.x;
  const int j = g.js + by * blockDim.y + threadIdx.y;
  const int k = g.ks + bz;
  if (i > g.ie + 1 || j > g.je + 1 || k > g.ke + 1) return;
  const double a = cf[0], b = cf[1], c = cf[2], d = cf[3], e = cf[4];
  const long l = g.idx(k, j, i);
  if (i <= g.ie && j <= g.je && k <= g.ke) {
    for (int n = 0; n < NVAR; ++n) {
      const long q = n * g.vstride + l;
      A.out[q] = ((a * A.x[q] + b * A.y[q]) + c * A.z[q]) + (d * A.p[q] + e * A.q[q]);
    }
  }
  for (int f = 0; f < 3; ++f)
    A.bo[f][l] = ((a * A.bx[f][l] + b * A.by[f][l]) + c * A.bz[f][l]) + (d * A.bp[f][l] + e * A.bq[f][l]);
}

__global__ void __launch_bounds__(256) sts_combine_kernel(const StsCombArgs A) {
  const double cf[5] = {A.a, A.b, A.c, A.d, A.e};
  sts_combine_body(A, cf, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---- batched RKL2 stages (many meshes, one launch per kernel kind and stage) -----------
// Every member advances its own stage count s_m; at stage j the members with j > s_m (or a
// finished clock) skip: skip[m] is rewritten before each stage.
__global__ void sts_skip_kernel(int *skip, const int *nst, int n, int j) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n) skip[m] = (j > nst[m]) ? 1 : 0;
}

template <class P> __global__ void __launch_bounds__(256) sts_div_batched(const StsDivArgs<P> *args, const BatchSlot *slots, int n) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(StsDivArgs<P>)];
  const StsDivArgs<P> &A = stage_args(args, j, sa);
  sts_div_body<P>(A, bx, by, bz);
}

// coef: this stage's five coefficients of every member (member m at coef[5 m])
__global__ void __launch_bounds__(256) sts_combine_batched(const StsCombArgs *args, const BatchSlot *slots, int n,
                                                           const double *coef) {
  int bx, by, bz;
  const int j = batch_job(slots, n, blockIdx.x);
  batch_block(slots[j], blockIdx.x, bx, by, bz);
  __shared__ __align__(16) unsigned char sa[sizeof(StsCombArgs)];
  const StsCombArgs &A = stage_args(args, j, sa);
  sts_combine_body(A, coef + 5 * j, bx, by, bz);
}

// Whole-array copies and zero fills of up to six spans of 8-byte words per member, the
// member's blocks striding over each span (the RKL2 state copies and flux/EMF zeroing).
struct SpanArgs {
  unsigned long long *dst[6];
  const unsigned long long *src[6];   // null: zero fill
  long words[6];
  int nspan;
  const int *done;
};

// the same copies and zero fills for one mesh (all blocks of the launch)
__global__ void __launch_bounds__(256) span_kernel(const SpanArgs A) {
  for (int q = 0; q < A.nspan; ++q) {
    unsigned long long *d = A.dst[q];
    const unsigned long long *src = A.src[q];
    for (long w = (long)blockIdx.x * blockDim.x + threadIdx.x; w < A.words[q]; w += (long)gridDim.x * blockDim.x)
      d[w] = src ? src[w] : 0ull;
  }
}

__global__ void __launch_bounds__(256) span_batched(const SpanArgs *args, const BatchSlot *slots, int n) {
  const int j = batch_job(slots, n, blockIdx.x);
  __shared__ __align__(16) unsigned char sa[sizeof(SpanArgs)];
  const SpanArgs &A = stage_args(args, j, sa);
  if (A.done && *A.done) return;
  const long b = blockIdx.x - slots[j].off, nb = slots[j].gx;
  for (int q = 0; q < A.nspan; ++q) {
    unsigned long long *d = A.dst[q];
    const unsigned long long *src = A.src[q];
    for (long w = b * blockDim.x + threadIdx.x; w < A.words[q]; w += nb * blockDim.x) d[w] = src ? src[w] : 0ull;
  }
}

}  // namespace chq
