// chasqui_b200 — device-resident time-step control.
//
// The reference returns dt and the FOFC count to the host at every stage (src/main.cpp:247,
// src/fofc.hpp:17-43), which forces a host synchronisation per stage. Here both stay in
// device memory: kernels read this cycle's beta*dt from StepCtl and accumulate the FOFC and
// limiter counts into it, so whole cycles run back to back (and can be graph-captured)
// without the host. The host reads StepCtl only when asked.
#pragma once
#include "chq_common.cuh"

namespace chq {

struct StepCtl {
  double t, tlim, cfl, dt;
  double min_dt;                 // last completed dt reduction (before cfl)
  double beta_dt[4];             // beta_s * dt of each stage of the current cycle
  double beta[4], g0[4], g1[4];  // integrator table, written once by the host
  unsigned long long mdt_bits;   // running min of the c2p dt reduction (positive doubles order as integers)
  long long fofc_count, limiter_count;
  int nbad;                      // cells flagged by the FOFC test in the current stage
  int cycle, done, nstage, nlim;   // nlim >= 0: stop after that many cycles (time.nlim)
  int err;                       // nonzero: a kernel detected an invalid launch configuration
  // explicit diffusion: the parabolic time-step limit joins min_dt (src/diffusion.hpp:159-174)
  int diff_on, sts, ndim;
  double nu, eta, kappa, gm1, dxmin;
  unsigned long long rho_bits;   // min density of the active cells after the last con2prim
};

// dx_min^2 / (2 ndim max(nu, eta, kappa (gamma-1) / rho_min)) in the reference's order
CHQ_D double parabolic_dt(const StepCtl *c) {
  const double rho_min = __longlong_as_double((long long)c->rho_bits);
  const double chi = (c->kappa > 0) ? c->kappa * c->gm1 / rho_min : 0.0;
  const double dmax = fmax(fmax(c->nu, c->eta), chi);
  return c->dxmin * c->dxmin / (2.0 * c->ndim * dmax);
}

// Start of a cycle: dt = cfl * min_dt, clamped to reach tlim exactly (src/main.cpp:246-248).
__global__ void ctl_begin_kernel(StepCtl *c, int nlim_left);
// End of a cycle: t += dt, ++cycle, min_dt from this cycle's reduction (src/main.cpp:291-292).
__global__ void ctl_end_kernel(StepCtl *c);

CHQ_D void atomic_min_pos(unsigned long long *bits, double v) {
  // non-negative doubles (and +inf / NaN above them) order like their bit patterns
  atomicMin(bits, (unsigned long long)__double_as_longlong(v));
}

// Minimum of v over the block into *bits with one atomic per block: warp shuffles, then the
// warps' minima through shared memory. Every thread of the block must call it (it holds a
// barrier); blocks of at most 32 warps. The result is the same as one atomic per thread.
CHQ_D void block_min_pos(unsigned long long *bits, double v) {
  __shared__ double wmin[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int tid = (int)(threadIdx.z * blockDim.y + threadIdx.y) * (int)blockDim.x + (int)threadIdx.x;
  const int nw = (int)((blockDim.x * blockDim.y * blockDim.z + 31) / 32);
  if ((tid & 31) == 0) wmin[tid >> 5] = v;
  __syncthreads();
  if (tid == 0) {
    double m = wmin[0];
    for (int w = 1; w < nw; ++w) m = fmin(m, wmin[w]);
    atomic_min_pos(bits, m);
  }
}

}  // namespace chq
