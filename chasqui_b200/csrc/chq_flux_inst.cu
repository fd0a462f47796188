// chasqui_b200 — instantiation unit of the face-flux kernel for one (precision, scheme).
// Compiled once per pair with -DCHQ_P=<double|float> -DCHQ_R=<0..4>.
#include <cstring>
#include "chq_launch.h"

#ifndef CHQ_P
#error "CHQ_P must be defined (double or float)"
#endif
#ifndef CHQ_R
#error "CHQ_R must be defined (reconstruction enum)"
#endif

namespace chq {

// per-device one-time opt-in to the dynamic shared memory of a y/z kernel
template <class K>
static cudaError_t allow_smem(K kern, size_t smem, bool *ready) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && ready[dev]) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  if (e == cudaSuccess && dev >= 0 && dev < 64) ready[dev] = true;
  return e;
}

// y/z sweeps (shared marching window, dynamic shared memory) then the x-sweep, one stream
template <int S, bool C>
static cudaError_t go(const FluxArgs<CHQ_P> &a, unsigned, cudaStream_t s) {
  constexpr int wpb = kYzThreads / 32;
  const unsigned nyz = (unsigned)((a.nwarp[1] + a.nwarp[2] + wpb - 1) / wpb), nx = (unsigned)((a.nwarp[0] + 3) / 4);
  bool yz_done = false;
  if constexpr (CHQ_R == R_PPM && !C && sizeof(CHQ_P) == 8) {
    // TMA staging of the streaming-PPM march (picked by the autotuner; FP64 only)
    if (nyz && a.yzvar == 1 && a.yzmaps) {
      constexpr size_t smem = flux_yz_tma_smem();
      static bool ready_tma[64] = {};
      const cudaError_t ea = allow_smem(flux_yz_tma_kernel<S>, smem, ready_tma);
      if (ea != cudaSuccess) return ea;
      YzMaps maps;
      std::memcpy(&maps, a.yzmaps, sizeof(maps));
      flux_yz_tma_kernel<S><<<nyz, kYzThreads, smem, s>>>(a, maps);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) return e;
      yz_done = true;
    }
  }
  if (nyz && !yz_done) {
    constexpr size_t smem = flux_yz_smem<CHQ_R, CHQ_P>();
    static bool ready[64] = {};
    const cudaError_t ea = allow_smem(flux_yz_kernel<CHQ_R, S, C, CHQ_P>, smem, ready);
    if (ea != cudaSuccess) return ea;
    flux_yz_kernel<CHQ_R, S, C, CHQ_P><<<nyz, kYzThreads, smem, s>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (nx) {
    if (a.xvar) flux_x_kernel<CHQ_R, S, C, CHQ_P, 1><<<nx, 128, 0, s>>>(a);
    else flux_x_kernel<CHQ_R, S, C, CHQ_P, 0><<<nx, 128, 0, s>>>(a);
  }
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
static cudaError_t gob(const FluxArgs<CHQ_P> *a, const BatchSlot *sx, const BatchSlot *syz, int n, unsigned nbx,
                       unsigned nbyz, int xvar, cudaStream_t s) {
  if (nbyz) {
    constexpr size_t smem = flux_yz_batched_smem<CHQ_R, CHQ_P>();
    static bool ready[64] = {};
    const cudaError_t e = allow_smem(flux_yz_batched<CHQ_R, S, C, CHQ_P>, smem, ready);
    if (e != cudaSuccess) return e;
    flux_yz_batched<CHQ_R, S, C, CHQ_P><<<nbyz, kYzThreads, smem, s>>>(a, syz, n);
    const cudaError_t e2 = cudaGetLastError();
    if (e2 != cudaSuccess) return e2;
  }
  if (nbx) {
    if (xvar) flux_x_batched<CHQ_R, S, C, CHQ_P, 1><<<nbx, 128, 0, s>>>(a, sx, n);
    else flux_x_batched<CHQ_R, S, C, CHQ_P, 0><<<nbx, 128, 0, s>>>(a, sx, n);
  }
  return cudaGetLastError();
}

template <>
cudaError_t launch_flux_batched<CHQ_P, CHQ_R>(const FluxArgs<CHQ_P> *a, const BatchSlot *sx, const BatchSlot *syz, int n,
                                               int rsolver, int charac, unsigned nbx, unsigned nbyz, int xvar,
                                               cudaStream_t s) {
  if (nbx == 0 && nbyz == 0) return cudaSuccess;
  const bool c = (charac != 0) && (CHQ_R != R_DC);
  switch (rsolver) {
    case S_HLLE: return c ? gob<S_HLLE, true>(a, sx, syz, n, nbx, nbyz, xvar, s) : gob<S_HLLE, false>(a, sx, syz, n, nbx, nbyz, xvar, s);
    case S_HLLD: return c ? gob<S_HLLD, true>(a, sx, syz, n, nbx, nbyz, xvar, s) : gob<S_HLLD, false>(a, sx, syz, n, nbx, nbyz, xvar, s);
    case S_LHLLD: return c ? gob<S_LHLLD, true>(a, sx, syz, n, nbx, nbyz, xvar, s) : gob<S_LHLLD, false>(a, sx, syz, n, nbx, nbyz, xvar, s);
    default: return cudaErrorInvalidValue;
  }
}

template <int S, bool C>
static int regs() {
  cudaFuncAttributes at{};
  if (cudaFuncGetAttributes(&at, flux_yz_kernel<CHQ_R, S, C, CHQ_P>) != cudaSuccess) return -1;
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
