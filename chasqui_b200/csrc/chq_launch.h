// chasqui_b200 — host-side launchers of the face-flux kernel, one translation unit per
// (precision, reconstruction) pair so that the 30 solver/characteristic variants of each
// compile in parallel.
#pragma once
#include "chq_flux.cuh"

namespace chq {

template <class P, int R>
cudaError_t launch_flux(const FluxArgs<P> &a, int rsolver, int charac, unsigned nblocks, cudaStream_t s);

// x-sweep blocks and y/z-sweep blocks of many meshes, with one slot table each
template <class P, int R>
cudaError_t launch_flux_batched(const FluxArgs<P> *args, const BatchSlot *slots_x, const BatchSlot *slots_yz, int njobs,
                                int rsolver, int charac, unsigned nblocks_x, unsigned nblocks_yz, int xvar,
                                cudaStream_t s);

// registers per thread of the instantiated y/z kernel (for the launch report)
template <class P, int R>
int flux_regs(int rsolver, int charac);

}  // namespace chq
