// chasqui_b200 — instantiation unit of the face-flux kernel for one (precision, scheme).
// Compiled once per pair with -DCHQ_P=<double|float> -DCHQ_R=<0..4>.
#include "chq_launch.h"

#ifndef CHQ_P
#error "CHQ_P must be defined (double or float)"
#endif
#ifndef CHQ_R
#error "CHQ_R must be defined (reconstruction enum)"
#endif

namespace chq {

template <int S, bool C>
static cudaError_t go(const FluxArgs<CHQ_P> &a, unsigned nblocks, cudaStream_t s) {
  flux_kernel<CHQ_R, S, C, CHQ_P><<<nblocks, 128, 0, s>>>(a);
  return cudaGetLastError();
}

template <>
cudaError_t launch_flux<CHQ_P, CHQ_R>(const FluxArgs<CHQ_P> &a, int rsolver, int charac, unsigned nblocks,
                                       cudaStream_t s) {
  if (nblocks == 0) return cudaSuccess;
  const bool c = (charac != 0) && (CHQ_R != R_DC);
  switch (rsolver) {
    case S_HLLE: return c ? go<S_HLLE, true>(a, nblocks, s) : go<S_HLLE, false>(a, nblocks, s);
    case S_HLLD: return c ? go<S_HLLD, true>(a, nblocks, s) : go<S_HLLD, false>(a, nblocks, s);
    case S_LHLLD: return c ? go<S_LHLLD, true>(a, nblocks, s) : go<S_LHLLD, false>(a, nblocks, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int S, bool C>
static cudaError_t gob(const FluxArgs<CHQ_P> *a, const BatchSlot *sl, int n, unsigned nblocks, cudaStream_t s) {
  flux_batched<CHQ_R, S, C, CHQ_P><<<nblocks, 128, 0, s>>>(a, sl, n);
  return cudaGetLastError();
}

template <>
cudaError_t launch_flux_batched<CHQ_P, CHQ_R>(const FluxArgs<CHQ_P> *a, const BatchSlot *sl, int n, int rsolver,
                                               int charac, unsigned nblocks, cudaStream_t s) {
  if (nblocks == 0) return cudaSuccess;
  const bool c = (charac != 0) && (CHQ_R != R_DC);
  switch (rsolver) {
    case S_HLLE: return c ? gob<S_HLLE, true>(a, sl, n, nblocks, s) : gob<S_HLLE, false>(a, sl, n, nblocks, s);
    case S_HLLD: return c ? gob<S_HLLD, true>(a, sl, n, nblocks, s) : gob<S_HLLD, false>(a, sl, n, nblocks, s);
    case S_LHLLD: return c ? gob<S_LHLLD, true>(a, sl, n, nblocks, s) : gob<S_LHLLD, false>(a, sl, n, nblocks, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int S, bool C>
static int regs() {
  cudaFuncAttributes at{};
  if (cudaFuncGetAttributes(&at, flux_kernel<CHQ_R, S, C, CHQ_P>) != cudaSuccess) return -1;
  return at.numRegs;
}

template <>
int flux_regs<CHQ_P, CHQ_R>(int rsolver, int charac) {
  const bool c = (charac != 0) && (CHQ_R != R_DC);
  switch (rsolver) {
    case S_HLLE: return c ? regs<S_HLLE, true>() : regs<S_HLLE, false>();
    case S_HLLD: return c ? regs<S_HLLD, true>() : regs<S_HLLD, false>();
    case S_LHLLD: return c ? regs<S_LHLLD, true>() : regs<S_LHLLD, false>();
    default: return -1;
  }
}

}  // namespace chq
