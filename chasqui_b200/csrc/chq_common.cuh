// chasqui_b200 — device data layout, geometry and scalar helpers shared by every kernel.
//
// Layout in HBM. Every field (cell, face or edge centred) lives in one common 3-D frame of
// (nk+1) planes x (nj+1) rows x `pitch` elements, pitch = ni+1 rounded up to 32 elements, so
// a single linear index serves cells, faces and edges with the reference's left-face /
// lower-edge convention (src/mesh.hpp:3-9). Multi-component fields (u, w, bcc, ecc, fluxes)
// stack their components `vstride` elements apart. Rows start on 256-byte boundaries, which
// keeps every warp's row access fully coalesced and every row a legal TMA/bulk-copy start.
// Conversion to and from the reference's packed (nk,nj,ni) / (nk+1,nj+1,ni+1) arrays happens
// only at the C-ABI upload/download boundary.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include <math.h>
#include "chq_divide.cuh"

#define CHQ_HD __host__ __device__ __forceinline__
#define CHQ_D __device__ __forceinline__

namespace chq {

// variable slots: src/defs.hpp:16-20
enum : int { IDN = 0, IM1 = 1, IM2 = 2, IM3 = 3, IEN = 4, IENT = 5, NVAR = 6 };
enum : int { IVX = 1, IVY = 2, IVZ = 3, IPR = 4 };
// reconstruction, Riemann solver and boundary enums keep the reference's values
// (src/defs.hpp:35-37, src/physics.hpp:20)
enum : int { R_DC = 0, R_PLM = 1, R_PPM = 2, R_WENOZ = 3, R_PPMX = 4 };
enum : int { S_HLLE = 0, S_HLLD = 1, S_LHLLD = 2 };
enum : int { BC_PERIODIC = 0, BC_OUTFLOW = 1, BC_REFLECT = 2 };

struct Geom {
  int nx1, nx2, nx3, ng;
  int ni, nj, nk;
  int is, ie, js, je, ks, ke;
  int two_d, three_d;
  double x1min, x2min, x3min, x1max, x2max, x3max;
  double dx1, dx2, dx3;
  // global index of this mesh's first active plane minus ks: 0 for a whole mesh, the slab's
  // first plane for one z slab of a decomposed mesh (coordinates and seeded noise use it)
  int koff;
  // device frame strides (elements)
  long sj;        // row pitch
  long sk;        // plane stride = (nj+1) * sj
  long vstride;   // component stride of multi-component fields
  long nelem;     // elements of one component (= vstride)
  CHQ_HD long idx(int k, int j, int i) const { return (long)k * sk + (long)j * sj + i; }
  // 32-bit form for offsets within one component (vstride < 2^31 is checked at mesh creation)
  CHQ_HD int idx32(int k, int j, int i) const { return k * (int)sk + j * (int)sj + i; }
};

struct EOSp {
  double gamma, gm1, dfloor, pfloor, de_eta;
  int dual_energy;
};

template <class T> CHQ_HD T sqr(T x) { return x * x; }
template <class T> CHQ_HD T sgn(T x) { return (x > T(0)) ? T(1) : ((x < T(0)) ? T(-1) : T(0)); }

CHQ_HD double fmin_(double a, double b) { return fmin(a, b); }
CHQ_HD float fmin_(float a, float b) { return fminf(a, b); }
CHQ_HD double fmax_(double a, double b) { return fmax(a, b); }
CHQ_HD float fmax_(float a, float b) { return fmaxf(a, b); }
CHQ_HD double fabs_(double a) { return fabs(a); }
CHQ_HD float fabs_(float a) { return fabsf(a); }
CHQ_HD double sqrt_(double a) { return sqrt(a); }
CHQ_HD float sqrt_(float a) { return sqrtf(a); }
CHQ_HD double pow_(double a, double b) { return pow(a, b); }

// smallest positive constants of the reference's double arithmetic; in the FP32 form they
// flush to zero exactly as the reference's single-precision build does (src/recon.hpp:117,185,
// src/riemann.hpp:134,156)
template <class T> struct Tiny;
template <> struct Tiny<double> { static constexpr double v = 1e-300; static constexpr double weno_eps = 1e-36; };
template <> struct Tiny<float> { static constexpr float v = 0.0f; static constexpr float weno_eps = 1e-20f; };

// read-only cached load
template <class T> CHQ_D T ldg(const T *p) { return __ldg(p); }

// Batched launches: one launch covers the blocks of many meshes. Job j owns the launch
// blocks [off, off + gx*gy*gz) of the 1-D grid and sees them as its own (gx, gy, gz) grid.
struct BatchSlot {
  long off;
  int gx, gy, gz, pad;
};

// the job whose block range holds launch block b (offsets are prefix sums; jobs without
// blocks share the next job's offset and are skipped)
CHQ_D int batch_job(const BatchSlot *s, int n, long b) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (s[mid].off <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Job j's argument struct copied into the block's shared memory by all threads, so that the
// batched bodies read their fields with uniform shared loads (the single-mesh kernels read
// them from the constant bank) instead of holding a private copy in registers or local memory.
template <class A> CHQ_D const A &stage_args(const A *args, int j, void *smem) {
  static_assert(sizeof(A) % 4 == 0, "argument structs are word-sized");
  const unsigned *src = reinterpret_cast<const unsigned *>(args + j);
  unsigned *dst = static_cast<unsigned *>(smem);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int t = (threadIdx.z * blockDim.y + threadIdx.y) * blockDim.x + threadIdx.x;
  for (int q = t; q < (int)(sizeof(A) / 4); q += nt) dst[q] = __ldg(src + q);
  __syncthreads();
  return *static_cast<const A *>(smem);
}

CHQ_D void batch_block(const BatchSlot &sl, long b, int &bx, int &by, int &bz) {
  const long loc = b - sl.off;
  bx = (int)(loc % sl.gx);
  by = (int)((loc / sl.gx) % sl.gy);
  bz = (int)(loc / ((long)sl.gx * sl.gy));
}

}  // namespace chq
