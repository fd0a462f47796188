// chasqui_b200 — history sums without any device allocation.
//
// chq_history() reduces into scratch that chq_mesh_create() allocated. Some callers cannot
// allocate device memory at all: an application whose memory is owned by its own pool or
// framework allocator (for instance a Kokkos code that keeps its fields in Views and
// forbids other allocations), code that must not trigger the implicit device
// synchronisation of cudaMalloc/cudaFree inside a timed or latency-critical loop, or a
// monitoring hook that only receives pointers to someone else's state. For them,
// chq_history_noalloc() works on caller-owned device arrays in the reference's packed
// layout and keeps its block partials in the fixed file-scope array below.
//
// Scratch: kNoallocMaxUnits partial rows of 10 doubles (~640 KiB), plus 10 result slots.
// One "unit" is one k-plane x 128-row slab of active cells, so a mesh needs
// nx3 * ceil(nx2 / 128) units; larger meshes are rejected with CHQ_ERR_ARG. Every device
// that loads this library holds the array until the process exits. All calls share it and
// it keeps the last call's contents; each call overwrites every slot it reads, so nothing
// needs clearing, but calls that overlap on the GPU (other streams, other host threads on
// the same device) race on it and must be serialised by the caller.
#include <cuda_runtime.h>
#include <string>
#include "chq.h"

namespace chq {
void set_last_error(const std::string &msg);   // chq_mesh.cu: the message behind chq_last_error()
}

namespace {

constexpr int kNoallocMaxUnits = 8192;
constexpr int kRowsPerUnit = 128;
constexpr int kNoallocSlots = kNoallocMaxUnits * 10 + 16;

static __device__ __align__(256) double g_noalloc_scratch[kNoallocSlots];

// Host code never dereferences g_noalloc_scratch: in host code the name is a stand-in, not a
// device address. Each call asks the runtime for the array's address in the calling thread's
// current context (cudaGetSymbolAddress allocates nothing). The address is not cached: after
// a cudaDeviceReset, or in another context on the same device, the module is loaded anew at
// another address, and a cached pointer would be stale.


struct Dims {
  int nx1, nx2, nx3, ng, ni, nj, nk, is, js, ks, two_d, three_d, nch;
  double idx1, idx2, idx3;
};

__global__ void __launch_bounds__(256) hst_units_kernel(Dims d, const double *u, const double *b1, const double *b2,
                                                        const double *b3, double *scratch) {
  __shared__ double sm[10][8];
  const int unit = blockIdx.x;
  const int k = d.ks + unit / d.nch;
  const int j0 = d.js + (unit % d.nch) * kRowsPerUnit;
  const int nrows = min(kRowsPerUnit, d.js + d.nx2 - j0);
  const long ncell = (long)d.nk * d.nj * d.ni;
  const long fj = d.ni + 1, fk = (long)(d.nj + 1) * (d.ni + 1);
  double v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (long c = threadIdx.x; c < (long)nrows * d.nx1; c += blockDim.x) {
    const int j = j0 + (int)(c / d.nx1);
    const int i = d.is + (int)(c % d.nx1);
    const long l = ((long)k * d.nj + j) * d.ni + i;
    const long f = k * fk + j * fj + i;
    const double rho = u[l];
    const double id = 1.0 / rho;
    const double vx = u[ncell + l] * id, vy = u[2 * ncell + l] * id, vz = u[3 * ncell + l] * id;
    const double bx = 0.5 * (b1[f] + b1[f + 1]);
    const double by = d.two_d ? 0.5 * (b2[f] + b2[f + fj]) : b2[f];
    const double bz = d.three_d ? 0.5 * (b3[f] + b3[f + fk]) : b3[f];
    const double ek = 0.5 * rho * (vx * vx + vy * vy + vz * vz);
    const double em = 0.5 * (bx * bx + by * by + bz * bz);
    const double e = u[4 * ncell + l];
    v[0] += rho;
    v[1] += u[ncell + l];
    v[2] += u[2 * ncell + l];
    v[3] += u[3 * ncell + l];
    v[4] += e;
    v[5] += ek;
    v[6] += em;
    v[7] += e - ek - em;
    double db = (b1[f + 1] - b1[f]) * d.idx1;
    if (d.two_d) db += (b2[f + fj] - b2[f]) * d.idx2;
    if (d.three_d) db += (b3[f + fk] - b3[f]) * d.idx3;
    v[8] = fmax(v[8], fabs(db));
    v[9] += fabs(db);
  }
#pragma unroll
  for (int q = 0; q < 10; ++q)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double x = __shfl_down_sync(0xffffffffu, v[q], o);
      v[q] = (q == 8) ? fmax(v[q], x) : v[q] + x;
    }
  if ((threadIdx.x & 31) == 0)
    for (int q = 0; q < 10; ++q) sm[q][threadIdx.x >> 5] = v[q];
  __syncthreads();
  if (threadIdx.x < 10) {
    double s = sm[threadIdx.x][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) s = (threadIdx.x == 8) ? fmax(s, sm[threadIdx.x][w]) : s + sm[threadIdx.x][w];
    scratch[(long)unit * 10 + threadIdx.x] = s;
  }
}

__global__ void hst_units_final_kernel(const double *scratch, int nunits, double *res) {
  const int q = threadIdx.x;
  if (q >= 10) return;
  double s = 0.0;
  for (int b = 0; b < nunits; ++b) s = (q == 8) ? fmax(s, scratch[(long)b * 10 + q]) : s + scratch[(long)b * 10 + q];
  res[q] = s;
}

int err(int code, const std::string &m) {
  chq::set_last_error(m);
  return code;
}

}  // namespace

extern "C" CHQ_API int chq_history_noalloc(int nx1, int nx2, int nx3, int ng, double dx1, double dx2, double dx3,
                                           const double *u, const double *b1, const double *b2, const double *b3,
                                           double out[10], void *stream) {
  if (nx1 < 1 || nx2 < 1 || nx3 < 1 || ng < 1) return err(CHQ_ERR_ARG, "chq_history_noalloc: bad mesh size");
  if (nx2 == 1 && nx3 > 1) return err(CHQ_ERR_ARG, "chq_history_noalloc: nx3 > 1 requires nx2 > 1");
  const long nch = (nx2 + kRowsPerUnit - 1) / kRowsPerUnit;
  const long nunits = (long)nx3 * nch;
  if (nunits > kNoallocMaxUnits)
    return err(CHQ_ERR_ARG, "chq_history_noalloc: mesh too large for the fixed scratch (nx3 * ceil(nx2/128) = " +
                                std::to_string(nunits) + " > " + std::to_string(kNoallocMaxUnits) + ")");
  if (!u || !b1 || !b2 || !b3 || !out) return err(CHQ_ERR_ARG, "chq_history_noalloc: null pointer");
  // the static array's device address in the current context (the first call on a device
  // also loads this module there: the set-up step)
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return err(CHQ_ERR_CUDA, std::string("chq_history_noalloc set-up: ") +
                                 (e != cudaSuccess ? cudaGetErrorString(e) : "no device address"));
  double *scratch = static_cast<double *>(p);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  Dims d;
  d.nx1 = nx1; d.nx2 = nx2; d.nx3 = nx3; d.ng = ng;
  d.ni = nx1 + 2 * ng;
  d.nj = (nx2 > 1) ? nx2 + 2 * ng : 1;
  d.nk = (nx3 > 1) ? nx3 + 2 * ng : 1;
  d.is = ng;
  d.js = (nx2 > 1) ? ng : 0;
  d.ks = (nx3 > 1) ? ng : 0;
  d.two_d = nx2 > 1;
  d.three_d = nx3 > 1;
  d.nch = (int)nch;
  d.idx1 = 1.0 / dx1; d.idx2 = 1.0 / dx2; d.idx3 = 1.0 / dx3;
  hst_units_kernel<<<(unsigned)nunits, 256, 0, s>>>(d, u, b1, b2, b3, scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) return err(CHQ_ERR_CUDA, std::string("chq_history_noalloc: ") + cudaGetErrorString(e));
  double *res = scratch + (long)kNoallocMaxUnits * 10;
  hst_units_final_kernel<<<1, 32, 0, s>>>(scratch, (int)nunits, res);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, res, 10 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return err(CHQ_ERR_CUDA, std::string("chq_history_noalloc: ") + cudaGetErrorString(e));
  const double vol = dx1 * (d.two_d ? dx2 : 1.0) * (d.three_d ? dx3 : 1.0);
  for (int q = 0; q < 8; ++q) out[q] *= vol;
  out[9] /= (double)nx1 * nx2 * nx3;
  return CHQ_OK;
}
