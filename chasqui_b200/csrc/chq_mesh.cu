// chasqui_b200 — device mesh, stage orchestration and the C ABI declared in include/chq.h.
//
// One chq_mesh owns every field of one simulation in a single device allocation, laid out
// in the common padded frame described in chq_common.cuh. The stage sequence is the
// reference's Stage() (src/main.cpp:46-93) with the host synchronisations removed: the
// time step, the FOFC decision and all counters live in a device StepCtl.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include "chq.h"
#include "chq_common.cuh"
#include "chq_ctl.cuh"
#include "chq_kernels.cuh"
#include "chq_launch.h"
#include "chq_pgen.cuh"

using namespace chq;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char *where, int line = 0) {
  std::string at = where;
  if (line > 0) at += " (chq_mesh.cu:" + std::to_string(line) + ")";
  return fail(CHQ_ERR_CUDA, at + ": " + cudaGetErrorString(e));
}
#define CHQ_CUDA(call)                                             \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call, __LINE__);  \
  } while (0)

}  // namespace

namespace chq {
void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace chq

// ---------------------------------------------------------------------------------------
// device control kernels
namespace chq {
CHQ_D void ctl_begin(StepCtl *c) {
  if (c->done) return;
  if (!(c->t < c->tlim) || (c->nlim >= 0 && c->cycle >= c->nlim)) { c->done = 1; return; }
  double dt = c->cfl * c->min_dt;
  if (c->t + dt > c->tlim) dt = c->tlim - c->t;
  c->dt = dt;
  for (int s = 0; s < c->nstage; ++s) c->beta_dt[s] = c->beta[s] * dt;
  c->mdt_bits = 0x7ff0000000000000ULL;
  c->rho_bits = 0x7ff0000000000000ULL;
}
CHQ_D void ctl_end(StepCtl *c) {
  if (c->done) return;
  c->t += c->dt;
  c->cycle += 1;
  c->min_dt = __longlong_as_double((long long)c->mdt_bits);
  if (c->diff_on && !c->sts) c->min_dt = fmin(c->min_dt, parabolic_dt(c));
}
__global__ void ctl_begin_kernel(StepCtl *c, int) { ctl_begin(c); }
__global__ void ctl_end_kernel(StepCtl *c) { ctl_end(c); }
__global__ void ctl_begin_batched(StepCtl *const *c, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) ctl_begin(c[j]);
}
__global__ void ctl_end_batched(StepCtl *const *c, int n) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) ctl_end(c[j]);
}
__global__ void batch_status_kernel(StepCtl *const *c, int n, double *out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) {
    out[3 * j] = c[j]->t;
    out[3 * j + 1] = (double)c[j]->cycle;
    out[3 * j + 2] = (double)c[j]->done;
  }
}
__global__ void ctl_prime_kernel(StepCtl *c, double t) {
  c->t = t;
  c->done = 0;
  c->cycle = 0;
  c->nbad = 0;
  c->fofc_count = 0;
  c->limiter_count = 0;
  c->mdt_bits = 0x7ff0000000000000ULL;
  c->rho_bits = 0x7ff0000000000000ULL;
}
__global__ void ctl_take_dt_kernel(StepCtl *c) {
  c->min_dt = __longlong_as_double((long long)c->mdt_bits);
  if (c->diff_on && !c->sts) c->min_dt = fmin(c->min_dt, parabolic_dt(c));
}
__global__ void reset_rho_kernel(StepCtl *c) { c->rho_bits = 0x7ff0000000000000ULL; }
__global__ void reset_bits_kernel(unsigned long long *b) { *b = 0x7ff0000000000000ULL; }
}  // namespace chq

// ---------------------------------------------------------------------------------------
// history: two-pass deterministic reduction (block partials in scratch, then one block)
namespace chq {
template <class P>
__global__ void __launch_bounds__(256) hst_partial_kernel(Geom g, const double *u, const P *w, const P *bcc,
                                                          const double *b1, const double *b2, const double *b3,
                                                          double idx1, double idx2, double idx3, double *part) {
  __shared__ double sm[10][8];
  double v[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  const long ncell = (long)g.nx1 * g.nx2 * g.nx3;
  const long vs = g.vstride;
  for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < ncell; c += (long)gridDim.x * blockDim.x) {
    const int i = g.is + (int)(c % g.nx1);
    const long r = c / g.nx1;
    const int j = g.js + (int)(r % g.nx2);
    const int k = g.ks + (int)(r / g.nx2);
    const long l = g.idx(k, j, i);
    const double d = (double)w[IDN * vs + l];
    const double vx = (double)w[IVX * vs + l], vy = (double)w[IVY * vs + l], vz = (double)w[IVZ * vs + l];
    const double bx = (double)bcc[l], by = (double)bcc[vs + l], bz = (double)bcc[2 * vs + l];
    v[0] += u[IDN * vs + l];
    v[1] += u[IM1 * vs + l];
    v[2] += u[IM2 * vs + l];
    v[3] += u[IM3 * vs + l];
    v[4] += u[IEN * vs + l];
    const double ek = 0.5 * d * (sqr(vx) + sqr(vy) + sqr(vz));
    const double em = 0.5 * (sqr(bx) + sqr(by) + sqr(bz));
    v[5] += ek;
    v[6] += em;
    v[7] += u[IEN * vs + l] - 0.5 * d * (sqr(vx) + sqr(vy) + sqr(vz)) - 0.5 * (sqr(bx) + sqr(by) + sqr(bz));
    double db = (b1[l + 1] - b1[l]) * idx1;
    if (g.two_d) db += (b2[l + g.sj] - b2[l]) * idx2;
    if (g.three_d) db += (b3[l + g.sk] - b3[l]) * idx3;
    v[8] = fmax(v[8], fabs(db));
    v[9] += fabs(db);
  }
  // fixed-order tree: warp shuffles, then warps in order
#pragma unroll
  for (int q = 0; q < 10; ++q) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double x = __shfl_down_sync(0xffffffffu, v[q], o);
      v[q] = (q == 8) ? fmax(v[q], x) : v[q] + x;
    }
  }
  const int wid = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0)
    for (int q = 0; q < 10; ++q) sm[q][wid] = v[q];
  __syncthreads();
  if (threadIdx.x < 10) {
    double s = sm[threadIdx.x][0];
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) s = (threadIdx.x == 8) ? fmax(s, sm[threadIdx.x][q]) : s + sm[threadIdx.x][q];
    part[(long)blockIdx.x * 10 + threadIdx.x] = s;
  }
}
__global__ void hst_final_kernel(const double *part, int nblk, double *out) {
  const int q = threadIdx.x;
  if (q >= 10) return;
  double s = (q == 8) ? 0.0 : 0.0;
  for (int b = 0; b < nblk; ++b) s = (q == 8) ? fmax(s, part[b * 10 + q]) : s + part[b * 10 + q];
  out[q] = s;
}
}  // namespace chq

// ---------------------------------------------------------------------------------------
struct chq_mesh {
  chq_config cfg;
  Geom g;
  EOSp eos;
  int nstage;
  int mixed;
  size_t psize;            // bytes of one P element
  cudaStream_t stream = nullptr;
  char *slab = nullptr;
  size_t slab_bytes = 0;
  double *u[2];
  double *bf[2][3];
  void *w, *bcc, *ecc, *flx[3], *et2[3], *et1[3], *e[3];
  int *flag;
  // chq_run_host_async jobs: uploads on up_stream, at most two in flight (oldest = hj_head)
  int device = 0;                          // the device the mesh was created on
  cudaStream_t up_stream = nullptr, down_stream = nullptr;   // the device's shared copy lanes
  cudaEvent_t up_ready = nullptr, prev_done = nullptr, hj_evt[2] = {nullptr, nullptr};
  void *hj_clk[2] = {nullptr, nullptr};   // pinned copies of the clock after each job's cycles
  int hj_head = 0, hj_count = 0;
  int *bad_list;   // this stage's flagged cells (first bad_cap), filled by the flag kernel
  int bad_cap;     // kBadCap; CHQ_FOFC_LIST_CAP in the environment lowers it (0: always scan)
  StepCtl *ctl;            // device
  double *hst_part, *hst_out;
  int hst_blocks;
  HstRec *hrec = nullptr;  // device .hst recording (chq_history_record): header, partials, rows
  long hrec_nfold = 0;
  int hrec_cap = 0;
  // flux launch geometry
  int lo[3][3], hi[3][3], active[3];
  int act_lo[3][3], act_hi[3][3];
  int seglen;
  int xvar = 0;   // x-sweep kernel variant (register cap), chq_autotune
  // y/z staging of the FP64 streaming-PPM march: 0 cp.async, 1 TMA (chq_autotune_yz); the
  // tensor maps over w and bcc are encoded at creation when the driver offers the encoder
  int yzvar = 0;
  bool tma_ok = false;
  YzMaps tmaps;
  // z slab of a decomposed mesh (chq_slab_create): the lower / upper z side borders another
  // slab (its ghosts come from chq_slab_unpack, not from the boundary kernel); slab geometry
  int zpeer[2] = {0, 0};
  int slab_rank = 0, slab_count = 1;
  // the FOFC repair reads the flags of the ghost plane below / above: only across an internal
  // slab boundary (at the periodic wrap the whole mesh's ghost cells are never flagged cells)
  int fofc_ext[2] = {0, 0};
  // RKL2 work arrays (cfg.sts only): Y0..Y2, M0, Mj on cells; their face-field twins
  double *sy[3] = {}, *sm0 = nullptr, *smj = nullptr;
  double *sb[3][3] = {}, *smb0[3] = {}, *smbj[3] = {};
  bool diff = false;
  long long sts_stages = 0;
  // set while the mesh is a member of a batch: the batch's end-of-cycles event, which every
  // operation on the mesh's own stream waits for (not owned by the mesh)
  cudaEvent_t batch_evt = nullptr;
  // output snapshot (chq_snapshot): device copy area, its stream and events, pending items
  struct SnapItem {
    double *host;
    long n;
    int ncomp, face;
    size_t es;
    int isint;
    char *copy;
    std::vector<unsigned char> tmp;   // host staging when the device element is not double
  };
  char *snap = nullptr;
  size_t snap_bytes = 0;
  double *stage_buf = nullptr;   // four upload staging slots (packed host layout), allocated on first upload
  cudaEvent_t stage_copied[4] = {}, stage_unpacked[4] = {};
  unsigned long long stage_seq = 0;   // chunks staged so far (slot = seq % 4)
  cudaStream_t unpack_stream = nullptr;   // the device's shared unpack lane (host jobs)
  // whole-cycle CUDA graph of chq_cycles on the mesh stream (built after one plain cycle)
  cudaGraph_t cyc_graph = nullptr;
  cudaGraphExec_t cyc_exec = nullptr;
  long long cyc_launches = 0;   // kernels in one captured cycle
  bool cyc_warm = false;        // a plain cycle has run (first-launch attribute set-up done)
  cudaStream_t snap_stream = nullptr;
  cudaEvent_t snap_taken = nullptr, snap_landed = nullptr;
  std::vector<SnapItem> snap_items;
  bool snap_pending = false;
  // timing
  cudaEvent_t slots[8] = {};
  bool prof = false;
  struct Pend { int kind; cudaEvent_t b, e; };
  std::vector<Pend> pending;
  std::vector<cudaEvent_t> pool;
  long long nlaunch = 0;
  double prof_ms[CHQ_NPROF] = {};
  long long prof_n[CHQ_NPROF] = {};
};

namespace {

// Mesh slabs and batch tables come from one stream-ordered memory pool per device. cudaFree
// waits for the whole device, so a server that retired a job while others ran stalled them
// all; a pool free is ordered on one stream only, and up to kPoolKeepBytes of freed blocks
// stay in the pool for the next job's mesh (beyond that the pool returns memory to the
// device at the next synchronisation).
const uint64_t kPoolKeepBytes = 16ull << 30;

cudaMemPool_t device_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) return nullptr;
    uint64_t keep = kPoolKeepBytes;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[dev] = p;
  }
  return pools[dev];
}

// stream-ordered allocation from the device's pool (the device's default pool if the
// library's own could not be created)
cudaError_t pool_alloc(void **ptr, size_t bytes, cudaStream_t s) {
  cudaMemPool_t p = device_pool();
  return p ? cudaMallocFromPoolAsync(ptr, bytes, p, s) : cudaMallocAsync(ptr, bytes, s);
}

const int kHstBlocks = 1184;   // 8 blocks per SM on 148 SMs
const size_t kBadCap = 1 << 16;            // flagged cells listed per stage
const long kRepairBlocks = 1184;           // repair grid of one mesh
const long kRepairBlocksBatched = 148;     // repair blocks per mesh of a batch

// bytes of one mesh slab: 18 double fields (u0, u1, 6 face fields), 39 fields of the
// primitive type, the int flags, the control block and the history scratch
size_t slab_size(size_t nel, size_t psize, bool sts) {
  auto up = [](size_t x) { return (x + 255) / 256 * 256; };
  // RKL2: 5 cell arrays of 6 components and 5 x 3 face fields, all double
  const size_t sts_fields = sts ? 45 : 0;
  return nel * sizeof(double) * (18 + sts_fields) + nel * psize * 39 + up(nel * sizeof(int)) +
         up(kBadCap * sizeof(int)) + up(sizeof(StepCtl)) + up((size_t)(kHstBlocks * 10 + 16) * sizeof(double));
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// reference stage table (src/main.cpp:250-268)
void stage_table(int nstage, int s, double &g0, double &g1, double &beta, int &cur, int &out) {
  if (nstage == 1) { g0 = 1; g1 = 0; beta = 1; cur = 0; out = 0; }
  else if (nstage == 2) {
    if (s == 1) { g0 = 1; g1 = 0; beta = 1; cur = 0; out = 1; }
    else { g0 = 0.5; g1 = 0.5; beta = 0.5; cur = 1; out = 0; }
  } else if (nstage == 3) {
    if (s == 1) { g0 = 1; g1 = 0; beta = 1; cur = 0; out = 1; }
    else if (s == 2) { g0 = 0.75; g1 = 0.25; beta = 0.25; cur = 1; out = 1; }
    else { g0 = 1.0 / 3.0; g1 = 2.0 / 3.0; beta = 2.0 / 3.0; cur = 1; out = 0; }
  } else {
    if (s == 1) { g0 = 1; g1 = 0; beta = 0.5; cur = 0; out = 1; }
    else if (s == 2) { g0 = 0; g1 = 1; beta = 0.5; cur = 1; out = 1; }
    else if (s == 3) { g0 = 2.0 / 3.0; g1 = 1.0 / 3.0; beta = 1.0 / 6.0; cur = 1; out = 1; }
    else { g0 = 0; g1 = 1; beta = 0.5; cur = 1; out = 0; }
  }
}

cudaStream_t S(chq_mesh *m, void *s) {
  cudaStream_t st = s ? static_cast<cudaStream_t>(s) : m->stream;
  if (m->batch_evt) cudaStreamWaitEvent(st, m->batch_evt, 0);
  return st;
}

template <class P> P *as(void *p) { return static_cast<P *>(p); }

cudaEvent_t pool_event(chq_mesh *m) {
  if (!m->pool.empty()) {
    cudaEvent_t e = m->pool.back();
    m->pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// CUDA-event timing of one kernel kind around a launch sequence (when profiling is on)
struct Prof {
  chq_mesh *m;
  int kind;
  cudaStream_t s;
  cudaEvent_t b = nullptr;
  Prof(chq_mesh *m_, int k, cudaStream_t s_) : m(m_), kind(k), s(s_) {
    if (m->prof) {
      b = pool_event(m);
      cudaEventRecord(b, s);
    }
  }
  ~Prof() {
    if (m->prof && b) {
      cudaEvent_t e = pool_event(m);
      cudaEventRecord(e, s);
      m->pending.push_back({kind, b, e});
    }
  }
};
enum { PK_FLUX = 0, PK_CORNER = 1, PK_UPDATE = 2, PK_FLAG = 3, PK_REPAIR = 4, PK_BC = 5, PK_C2P = 6, PK_LIMIT = 7,
       PK_CTL = 8, PK_DIFF = 9, PK_STS = 10 };

// ---- fluxes --------------------------------------------------------------------------
template <class P>
FluxArgs<P> flux_args(chq_mesh *m, int cur, unsigned dirmask) {
  FluxArgs<P> a{};
  a.g = m->g;
  a.eos = m->eos;
  a.w = as<P>(m->w);
  a.bcc = as<P>(m->bcc);
  for (int d = 0; d < 3; ++d) {
    a.bn[d] = m->bf[cur][d];
    a.flx[d] = as<P>(m->flx[d]);
    a.et2[d] = as<P>(m->et2[d]);
    a.et1[d] = as<P>(m->et1[d]);
    for (int q = 0; q < 3; ++q) { a.lo[d][q] = m->lo[d][q]; a.hi[d][q] = m->hi[d][q]; }
    a.active[d] = m->active[d] && ((dirmask >> d) & 1);
  }
  a.flatten = m->cfg.flatten;
  a.low_mach = m->cfg.low_mach;
  a.lhlld_phi = m->cfg.lhlld_phi;
  a.seglen = m->seglen;
  a.xvar = m->xvar;
  a.yzvar = m->tma_ok ? m->yzvar : 0;
  a.yzmaps = m->tma_ok ? &m->tmaps : nullptr;
  a.err = &m->ctl->err;
  a.nchunk = (m->g.ni + 1 + 31) / 32;
  // x: rows x segments of XFaces faces (29 for streaming PPM, else 31); y/z: i chunks x
  // outer x segments
  const int xf = (m->cfg.recon == R_PPM && !m->cfg.characteristic) ? XFaces<R_PPM, false>::v : XFaces<R_DC, false>::v;
  a.nseg[0] = (m->hi[0][2] - m->lo[0][2] + 1 + xf - 1) / xf;
  a.nwarp[0] = a.active[0] ? (long)(m->hi[0][0] - m->lo[0][0] + 1) * (m->hi[0][1] - m->lo[0][1] + 1) * a.nseg[0] : 0;
  a.nseg[1] = (m->hi[1][1] - m->lo[1][1] + 1 + a.seglen - 1) / a.seglen;
  a.nwarp[1] = a.active[1] ? (long)a.nchunk * (m->hi[1][0] - m->lo[1][0] + 1) * a.nseg[1] : 0;
  a.nseg[2] = (m->hi[2][0] - m->lo[2][0] + 1 + a.seglen - 1) / a.seglen;
  a.nwarp[2] = a.active[2] ? (long)a.nchunk * (m->hi[2][1] - m->lo[2][1] + 1) * a.nseg[2] : 0;
  a.skip = nullptr;
  return a;
}

template <class P>
cudaError_t launch_flux_any(const FluxArgs<P> &a, int recon, int rsolver, int charac, cudaStream_t s) {
  const long warps = a.nwarp[0] + a.nwarp[1] + a.nwarp[2];
  const unsigned nblocks = (unsigned)((warps + 3) / 4);
  switch (recon) {
    case R_DC: return launch_flux<P, R_DC>(a, rsolver, charac, nblocks, s);
    case R_PLM: return launch_flux<P, R_PLM>(a, rsolver, charac, nblocks, s);
    case R_PPM: return launch_flux<P, R_PPM>(a, rsolver, charac, nblocks, s);
    case R_PPMX: return launch_flux<P, R_PPMX>(a, rsolver, charac, nblocks, s);
    case R_WENOZ: return launch_flux<P, R_WENOZ>(a, rsolver, charac, nblocks, s);
    default: return cudaErrorInvalidValue;
  }
}

int do_fluxes(chq_mesh *m, int cur, unsigned dirmask, const int *done, cudaStream_t s) {
  cudaError_t e;
  m->nlaunch += 1;
  if (m->mixed) {
    FluxArgs<float> a = flux_args<float>(m, cur, dirmask);
    a.skip = done;
    e = launch_flux_any(a, m->cfg.recon, m->cfg.rsolver, m->cfg.characteristic, s);
  } else {
    FluxArgs<double> a = flux_args<double>(m, cur, dirmask);
    a.skip = done;
    e = launch_flux_any(a, m->cfg.recon, m->cfg.rsolver, m->cfg.characteristic, s);
  }
  if (e != cudaSuccess) return cuda_fail(e, "flux_kernel launch");
  return CHQ_OK;
}

// ---- corner EMF ----------------------------------------------------------------------
struct Launch3 {
  dim3 grid, block;
};

template <class P>
EmfArgs<P> corner_args(chq_mesh *m, const int *done, const int *need) {
  const Geom &g = m->g;
  EmfArgs<P> a{};
  a.g = g;
  a.f1 = as<P>(m->flx[0]); a.f2 = as<P>(m->flx[1]); a.f3 = as<P>(m->flx[2]);
  a.e2x1 = as<P>(m->et1[0]); a.e3x1 = as<P>(m->et2[0]);
  a.e1x2 = as<P>(m->et2[1]); a.e3x2 = as<P>(m->et1[1]);
  a.e1x3 = as<P>(m->et1[2]); a.e2x3 = as<P>(m->et2[2]);
  a.ecc = as<P>(m->ecc);
  a.e1 = as<P>(m->e[0]); a.e2 = as<P>(m->e[1]); a.e3 = as<P>(m->e[2]);
  a.done = done;
  a.need = need;
  a.list = m->bad_list;
  a.cap = m->bad_cap;
  return a;
}

Launch3 corner_grid(const chq_mesh *m) {
  const Geom &g = m->g;
  const int nxi = g.ie + 2 - g.is, nyj = g.je + 2 - g.js;
  const int nzk = g.three_d ? g.ke + 2 - g.ks : 1;
  return {dim3((nxi + 31) / 32, (nyj + 7) / 8, nzk), dim3(32, 8)};
}

template <class P>
int do_corner(chq_mesh *m, const int *done, const int *need, cudaStream_t s) {
  const EmfArgs<P> a = corner_args<P>(m, done, need);
  const Launch3 L = corner_grid(m);
  m->nlaunch += 1;
  corner_emf_kernel<P><<<L.grid, L.block, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

Launch3 repair_grid(long faces, long max_blocks);

// FOFC re-run of the corner EMFs over the edges of the flagged cells only (need = the
// device count of flagged cells); grid-stride, at most kRepairBlocks blocks
template <class P>
int do_corner_rerun(chq_mesh *m, const int *done, const int *need, cudaStream_t s) {
  const EmfArgs<P> a = corner_args<P>(m, done, need);
  const Geom &g = m->g;
  const long pts = (long)(g.ie + 2 - g.is) * (g.je + 2 - g.js) * (g.three_d ? g.ke + 2 - g.ks : 1);
  m->nlaunch += 1;
  corner_rerun_kernel<P><<<repair_grid(pts, kRepairBlocks).grid, 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

// ---- update --------------------------------------------------------------------------
template <class P>
UpdateArgs<P> update_args(chq_mesh *m, int out, double g0, double g1, double bdt, const double *bdt_dev,
                          const int *done, const int *need) {
  const Geom &g = m->g;
  UpdateArgs<P> a{};
  a.g = g;
  a.eos = m->eos;
  a.f1 = as<P>(m->flx[0]); a.f2 = as<P>(m->flx[1]); a.f3 = as<P>(m->flx[2]);
  a.e1 = as<P>(m->e[0]); a.e2 = as<P>(m->e[1]); a.e3 = as<P>(m->e[2]);
  a.ua = m->u[0]; a.ub = m->u[1]; a.uout = m->u[out];
  a.b1a = m->bf[0][0]; a.b2a = m->bf[0][1]; a.b3a = m->bf[0][2];
  a.b1b = m->bf[1][0]; a.b2b = m->bf[1][1]; a.b3b = m->bf[1][2];
  a.b1o = m->bf[out][0]; a.b2o = m->bf[out][1]; a.b3o = m->bf[out][2];
  a.g0 = g0; a.g1 = g1; a.beta_dt = bdt; a.beta_dt_dev = bdt_dev;
  a.idx1 = 1.0 / g.dx1; a.idx2 = 1.0 / g.dx2; a.idx3 = 1.0 / g.dx3;
  a.done = done;
  a.need = need;
  const chq_config &c = m->cfg;
  a.grav = GravityP{(c.gravity_uniform || c.gravity_point) ? 1 : 0, c.gravity_point ? 1 : 0,
                    c.gravity_uniform ? c.g1 : 0.0, c.gravity_uniform ? c.g2 : 0.0, c.gravity_uniform ? c.g3 : 0.0,
                    c.gm, c.gx0, c.gy0, c.gz0, c.rsoft};
  a.w = as<P>(m->w);
  return a;
}

Launch3 update_grid(const chq_mesh *m) {
  const Geom &g = m->g;
  const int nxi = g.ie + 2 - g.is, nyj = g.je + 2 - g.js, nzk = g.ke + 2 - g.ks;
  return {dim3((nxi + 31) / 32, (nyj + 7) / 8, nzk), dim3(32, 8)};
}

template <class P>
int do_update(chq_mesh *m, int out, double g0, double g1, double bdt, const double *bdt_dev, const int *done,
              const int *need, cudaStream_t s) {
  const UpdateArgs<P> a = update_args<P>(m, out, g0, g1, bdt, bdt_dev, done, need);
  const Launch3 L = update_grid(m);
  m->nlaunch += 1;
  if (a.grav.on) update_kernel<P, true><<<L.grid, L.block, 0, s>>>(a);
  else update_kernel<P, false><<<L.grid, L.block, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

// FOFC re-run of the update (need = the device count of flagged cells). In a stage with
// g1 = 0 whose output is the b-state only the points around the listed cells change
// (update_rerun_listed_kernel); every other stage re-runs the whole update, as the reference.
template <class P>
int do_update_rerun(chq_mesh *m, int out, double g0, double g1, double bdt, const double *bdt_dev, const int *done,
                    const int *need, cudaStream_t s) {
  if (!(g1 == 0.0 && out == 1) || m->bad_cap <= 0) return do_update<P>(m, out, g0, g1, bdt, bdt_dev, done, need, s);
  UpdateArgs<P> a = update_args<P>(m, out, g0, g1, bdt, bdt_dev, done, need);
  a.list = m->bad_list;
  a.cap = m->bad_cap;
  const Geom &g = m->g;
  const int per = 3 * (g.two_d ? 3 : 1) * (g.three_d ? 3 : 1);
  const dim3 grid = repair_grid((long)per * m->bad_cap, kRepairBlocks).grid;
  m->nlaunch += 2;
  if (a.grav.on) update_rerun_listed_kernel<P, true><<<grid, 256, 0, s>>>(a);
  else update_rerun_listed_kernel<P, false><<<grid, 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  // list overflow (count above the capacity): the whole update, as in the other stages
  a.need_min = m->bad_cap;
  const Launch3 L = update_grid(m);
  if (a.grav.on) update_kernel<P, true><<<L.grid, L.block, 0, s>>>(a);
  else update_kernel<P, false><<<L.grid, L.block, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

FlagArgs flag_args(chq_mesh *m, int buf, int *nbad_dev, const int *done) {
  const Geom &g = m->g;
  FlagArgs a{};
  a.g = g;
  a.eos = m->eos;
  a.u = m->u[buf];
  a.b1 = m->bf[buf][0]; a.b2 = m->bf[buf][1]; a.b3 = m->bf[buf][2];
  a.flag = m->flag;
  a.nbad = nbad_dev;
  a.done = done;
  a.list = m->bad_list;
  a.cap = m->bad_cap;
  return a;
}

Launch3 flag_grid(const chq_mesh *m) {
  const Geom &g = m->g;
  return {dim3((g.nx1 + 31) / 32, (g.je - g.js + 1 + 7) / 8, g.ke - g.ks + 1), dim3(32, 8)};
}

int do_flag(chq_mesh *m, int buf, int *nbad_dev, const int *done, cudaStream_t s) {
  const FlagArgs a = flag_args(m, buf, nbad_dev, done);
  const Launch3 L = flag_grid(m);
  m->nlaunch += 1;
  fofc_flag_kernel<<<L.grid, L.block, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

template <class P>
RepairArgs<P> repair_args(chq_mesh *m, int cur, unsigned dirmask, const int *done, const int *need, long &tot) {
  RepairArgs<P> a{};
  a.g = m->g;
  a.eos = m->eos;
  a.w = as<P>(m->w);
  a.bcc = as<P>(m->bcc);
  tot = 0;
  for (int d = 0; d < 3; ++d) {
    a.bn[d] = m->bf[cur][d];
    a.flx[d] = as<P>(m->flx[d]);
    a.et2[d] = as<P>(m->et2[d]);
    a.et1[d] = as<P>(m->et1[d]);
    for (int q = 0; q < 3; ++q) { a.lo[d][q] = m->lo[d][q]; a.hi[d][q] = m->hi[d][q]; }
    const bool on = m->active[d] && ((dirmask >> d) & 1);
    a.nface[d] = on ? (long)(m->hi[d][0] - m->lo[d][0] + 1) * (m->hi[d][1] - m->lo[d][1] + 1) * (m->hi[d][2] - m->lo[d][2] + 1) : 0;
    tot += a.nface[d];
  }
  a.flag = m->flag;
  a.done = done;
  a.need = need;
  a.list = m->bad_list;
  a.cap = m->bad_cap;
  a.kext[0] = m->fofc_ext[0];
  a.kext[1] = m->fofc_ext[1];
  return a;
}

// repair grid: grid-stride, at most kRepairBlocks blocks of 256 (a listed repair touches a
// few faces; the full scan is the rare fallback)
Launch3 repair_grid(long faces, long max_blocks) {
  return {dim3((unsigned)std::max(1L, std::min((faces + 255) / 256, max_blocks))), dim3(256)};
}

template <class P>
int do_repair(chq_mesh *m, int cur, unsigned dirmask, const int *done, const int *need, cudaStream_t s) {
  long tot = 0;
  const RepairArgs<P> a = repair_args<P>(m, cur, dirmask, done, need, tot);
  if (tot == 0) return CHQ_OK;
  m->nlaunch += 1;
  fofc_repair_kernel<P><<<repair_grid(tot, kRepairBlocks).grid, 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

template <class P>
LimitArgs<P> limit_args(chq_mesh *m, unsigned dirmask, double bdt, const double *bdt_dev, long long *count_dev,
                        const int *done, long &tot) {
  const Geom &g = m->g;
  LimitArgs<P> a{};
  a.g = g;
  a.eos = m->eos;
  a.w = as<P>(m->w);
  a.bcc = as<P>(m->bcc);
  const int ndim = 1 + g.two_d + g.three_d;
  a.two_ndim = 2.0 * ndim;
  a.dx[0] = g.dx1; a.dx[1] = g.dx2; a.dx[2] = g.dx3;
  a.beta_dt = bdt;
  a.beta_dt_dev = bdt_dev;
  tot = 0;
  for (int d = 0; d < 3; ++d) {
    a.flx[d] = as<P>(m->flx[d]);
    for (int q = 0; q < 3; ++q) { a.lo[d][q] = m->act_lo[d][q]; a.hi[d][q] = m->act_hi[d][q]; }
    a.kcount[d][0] = a.lo[d][0];
    a.kcount[d][1] = a.hi[d][0];
    if (d < 2) {
      // across an internal slab boundary the transverse faces of the ghost plane are active
      // faces of the whole mesh
      a.lo[d][0] -= m->fofc_ext[0];
      a.hi[d][0] += m->fofc_ext[1];
    } else if (m->fofc_ext[1]) {
      a.kcount[d][1] -= 1;   // the face shared with the upper slab is counted there
    }
    const bool on = m->active[d] && ((dirmask >> d) & 1);
    a.nface[d] = on ? (long)(a.hi[d][0] - a.lo[d][0] + 1) * (a.hi[d][1] - a.lo[d][1] + 1) * (a.hi[d][2] - a.lo[d][2] + 1) : 0;
    tot += a.nface[d];
  }
  a.count = count_dev;
  a.done = done;
  return a;
}

template <class P>
int do_limit(chq_mesh *m, unsigned dirmask, double bdt, const double *bdt_dev, long long *count_dev, const int *done,
             cudaStream_t s) {
  long tot = 0;
  const LimitArgs<P> a = limit_args<P>(m, dirmask, bdt, bdt_dev, count_dev, done, tot);
  if (tot == 0) return CHQ_OK;
  m->nlaunch += 1;
  limit_kernel<P><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

BcArgs bc_args(chq_mesh *m, int buf, const int *done, int dir) {
  BcArgs a{};
  a.g = m->g;
  a.u = m->u[buf];
  a.b1 = m->bf[buf][0]; a.b2 = m->bf[buf][1]; a.b3 = m->bf[buf][2];
  a.done = done;
  a.bc = (dir == 0) ? m->cfg.bc1 : (dir == 1) ? m->cfg.bc2 : m->cfg.bc3;
  a.zside = 3;
  return a;
}

// threads of the ghost-fill launch of one direction (0 when the direction is inactive)
long bc_threads(const chq_mesh *m, int dir) {
  const Geom &g = m->g;
  if (dir == 0) return (long)(g.nk + 1) * (g.nj + 1) * g.ng;
  if (dir == 1) return g.two_d ? (long)(g.nk + 1) * g.ng * (g.ni + 1) : 0;
  return g.three_d ? (long)g.ng * (g.nj + 1) * (g.ni + 1) : 0;
}

int do_bc_ptr(chq_mesh *m, double *u, double *b1, double *b2, double *b3, const int *done, cudaStream_t s) {
  const Geom &g = m->g;
  BcArgs a{};
  a.g = g;
  a.u = u;
  a.b1 = b1; a.b2 = b2; a.b3 = b3;
  a.done = done;
  a.bc = m->cfg.bc1;
  long n = (long)(g.nk + 1) * (g.nj + 1) * g.ng;
  m->nlaunch += 1;
  bc_kernel<0><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  if (g.two_d) {
    a.bc = m->cfg.bc2;
    n = (long)(g.nk + 1) * g.ng * (g.ni + 1);
    m->nlaunch += 1;
    bc_kernel<1><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
    CHQ_CUDA(cudaGetLastError());
  }
  // a z slab's peer sides receive halos from the neighbouring slabs instead (chq_slab_unpack)
  a.zside = (m->zpeer[0] ? 0 : 1) | (m->zpeer[1] ? 0 : 2);
  if (g.three_d && a.zside) {
    a.bc = m->cfg.bc3;
    n = (long)g.ng * (g.nj + 1) * (g.ni + 1);
    m->nlaunch += 1;
    bc_kernel<2><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a);
    CHQ_CUDA(cudaGetLastError());
  }
  return CHQ_OK;
}

int do_bc(chq_mesh *m, int buf, const int *done, cudaStream_t s) {
  return do_bc_ptr(m, m->u[buf], m->bf[buf][0], m->bf[buf][1], m->bf[buf][2], done, s);
}

template <class P>
C2pArgs<P> c2p_args_ptr(chq_mesh *m, double *u, const double *b1, const double *b2, const double *b3, int compute_dt,
                        unsigned long long *bits, StepCtl *fold, const int *done) {
  const Geom &g = m->g;
  C2pArgs<P> a{};
  a.g = g;
  a.eos = m->eos;
  a.u = u;
  a.b1 = b1; a.b2 = b2; a.b3 = b3;
  a.w = as<P>(m->w); a.bcc = as<P>(m->bcc); a.ecc = as<P>(m->ecc);
  a.compute_dt = compute_dt;
  a.mdt_bits = bits;
  a.ctl = fold;
  a.done = done;
  return a;
}

template <class P>
C2pArgs<P> c2p_args(chq_mesh *m, int buf, int compute_dt, unsigned long long *bits, StepCtl *fold, const int *done) {
  return c2p_args_ptr<P>(m, m->u[buf], m->bf[buf][0], m->bf[buf][1], m->bf[buf][2], compute_dt, bits, fold, done);
}

Launch3 c2p_grid(const chq_mesh *m) {
  const Geom &g = m->g;
  return {dim3((g.ni + 31) / 32, (g.nj + 7) / 8, g.nk), dim3(32, 8)};
}

template <class P>
int launch_c2p(chq_mesh *m, const C2pArgs<P> &a, cudaStream_t s) {
  const Launch3 L = c2p_grid(m);
  m->nlaunch += 1;
  c2p_kernel<P><<<L.grid, L.block, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

template <class P>
int do_c2p(chq_mesh *m, int buf, int compute_dt, unsigned long long *bits, StepCtl *fold, const int *done,
           cudaStream_t s) {
  return launch_c2p<P>(m, c2p_args<P>(m, buf, compute_dt, bits, fold, done), s);
}

// K5 of a cycle's final state (u0, with the dt reduction); with .hst recording on, the form
// that also reduces the history sums when the cycle is an output
template <class P>
int do_c2p_end(chq_mesh *m, const int *done, cudaStream_t s) {
  if (!m->hrec) return do_c2p<P>(m, 0, 1, &m->ctl->mdt_bits, m->ctl, done, s);
  C2pArgs<P> a = c2p_args<P>(m, 0, 1, &m->ctl->mdt_bits, m->ctl, done);
  a.hst = m->hrec;
  const Launch3 L = c2p_grid(m);
  m->nlaunch += 1;
  c2p_kernel<P, true><<<L.grid, L.block, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

// ---- explicit diffusion (src/diffusion.hpp) --------------------------------------------
CurlB curl_of(const chq_mesh *m, const double *b1, const double *b2, const double *b3) {
  const Geom &g = m->g;
  CurlB J{};
  J.b1 = b1; J.b2 = b2; J.b3 = b3;
  J.idx1 = 1.0 / g.dx1; J.idx2 = 1.0 / g.dx2; J.idx3 = 1.0 / g.dx3;
  J.two_d = g.two_d; J.three_d = g.three_d;
  J.sj = g.sj; J.sk = g.sk;
  return J;
}

template <class P>
DiffArgs<P> diff_args(chq_mesh *m, const double *b1, const double *b2, const double *b3, const int *done, long &tot) {
  DiffArgs<P> a{};
  a.g = m->g;
  a.c = DiffCoef{m->cfg.nu, m->cfg.kappa, m->cfg.eta};
  a.w = as<P>(m->w);
  a.bcc = as<P>(m->bcc);
  a.J = curl_of(m, b1, b2, b3);
  tot = 0;
  for (int d = 0; d < 3; ++d) {
    a.flx[d] = as<P>(m->flx[d]);
    for (int q = 0; q < 3; ++q) { a.lo[d][q] = m->act_lo[d][q]; a.hi[d][q] = m->act_hi[d][q]; }
    a.nface[d] = m->active[d] ? (long)(a.hi[d][0] - a.lo[d][0] + 1) * (a.hi[d][1] - a.lo[d][1] + 1) * (a.hi[d][2] - a.lo[d][2] + 1) : 0;
    tot += a.nface[d];
  }
  a.done = done;
  return a;
}

template <class P> RhoMinArgs<P> rho_min_args(chq_mesh *m, const int *done) {
  return RhoMinArgs<P>{m->g, as<P>(m->w), &m->ctl->rho_bits, done};
}

// grid of the kernels over the active cells (rho_min, cooling)
Launch3 active_grid(const chq_mesh *m) {
  const Geom &g = m->g;
  return {dim3((unsigned)((g.nx1 + 31) / 32), (unsigned)((g.je - g.js + 1 + 7) / 8), (unsigned)(g.ke - g.ks + 1)), dim3(32, 8)};
}

// diffusive fluxes of every active direction in one launch (diffusion::Fluxes<0..2>)
template <class P>
int do_diff(chq_mesh *m, const double *b1, const double *b2, const double *b3, const int *done, cudaStream_t s) {
  long tot = 0;
  const DiffArgs<P> a = diff_args<P>(m, b1, b2, b3, done, tot);
  if (tot == 0) return CHQ_OK;
  m->nlaunch += 1;
  diff_flux_kernel<P><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

template <class P>
ResEmfArgs<P> res_emf_args(chq_mesh *m, const double *b1, const double *b2, const double *b3, const int *done,
                           const int *need) {
  const Geom &g = m->g;
  ResEmfArgs<P> a{};
  a.g = g;
  a.eta = m->cfg.eta;
  a.J = curl_of(m, b1, b2, b3);
  a.e1 = as<P>(m->e[0]); a.e2 = as<P>(m->e[1]); a.e3 = as<P>(m->e[2]);
  a.ku = g.three_d ? g.ke + 1 : g.ks + 1;
  a.ju = g.two_d ? g.je + 1 : g.js + 1;
  a.done = done;
  a.need = need;
  return a;
}

// the resistive EMF grid; empty without resistivity
Launch3 res_emf_grid(const chq_mesh *m) {
  const Geom &g = m->g;
  if (!(m->cfg.eta > 0.0)) return {dim3(0, 1, 1), dim3(32, 8)};
  const int ku = g.three_d ? g.ke + 1 : g.ks + 1, ju = g.two_d ? g.je + 1 : g.js + 1;
  return {dim3((unsigned)((g.ie + 2 - g.is + 31) / 32), (unsigned)((ju - g.js + 1 + 7) / 8), (unsigned)(ku - g.ks + 1)),
          dim3(32, 8)};
}

// eta J added to the edge EMFs (diffusion::ResistiveEMF); a no-op without resistivity
template <class P>
int do_res_emf(chq_mesh *m, const double *b1, const double *b2, const double *b3, const int *done, const int *need,
               cudaStream_t s) {
  if (!(m->cfg.eta > 0.0)) return CHQ_OK;
  const ResEmfArgs<P> a = res_emf_args<P>(m, b1, b2, b3, done, need);
  m->nlaunch += 1;
  resistive_emf_kernel<P><<<res_emf_grid(m).grid, dim3(32, 8), 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

// cooling of the step's end state u0 over this cycle's dt (srcterms::ApplyCooling)
template <class P> CoolArgs<P> cool_args(chq_mesh *m, const int *done) {
  CoolArgs<P> a{};
  a.g = m->g;
  a.gm1 = m->cfg.gamma - 1.0;
  a.lambda0 = m->cfg.lambda0;
  a.alpha = m->cfg.cool_alpha;
  a.tfloor = m->cfg.tfloor;
  a.u = m->u[0];
  a.w = as<P>(m->w);
  a.dt = &m->ctl->dt;
  a.done = done;
  return a;
}

template <class P>
int do_cooling(chq_mesh *m, const int *done, cudaStream_t s) {
  const Geom &g = m->g;
  CoolArgs<P> a{};
  a.g = g;
  a.gm1 = m->cfg.gamma - 1.0;
  a.lambda0 = m->cfg.lambda0;
  a.alpha = m->cfg.cool_alpha;
  a.tfloor = m->cfg.tfloor;
  a.u = m->u[0];
  a.w = as<P>(m->w);
  a.dt = &m->ctl->dt;
  a.done = done;
  const dim3 grid((unsigned)((g.nx1 + 31) / 32), (unsigned)((g.je - g.js + 1 + 7) / 8), (unsigned)(g.ke - g.ks + 1));
  m->nlaunch += 1;
  cooling_kernel<P><<<grid, dim3(32, 8), 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

// minimum density of the active cells into StepCtl::rho_bits (diffusion::TimeStep's reduction)
template <class P>
int do_rho_min(chq_mesh *m, const int *done, cudaStream_t s) {
  const Geom &g = m->g;
  const dim3 grid((unsigned)((g.nx1 + 31) / 32), (unsigned)((g.je - g.js + 1 + 7) / 8), (unsigned)(g.ke - g.ks + 1));
  m->nlaunch += 1;
  rho_min_kernel<P><<<grid, dim3(32, 8), 0, s>>>(rho_min_args<P>(m, done));
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

#define DISPATCH_P(m, call) ((m)->mixed ? call<float> : call<double>)

// FOFC repair with the diffusive fluxes re-added on repaired active faces when `with_diff`
template <class P>
int do_repair_d(chq_mesh *m, int cur, bool with_diff, const int *done, const int *need, cudaStream_t s) {
  long tot = 0;
  RepairArgs<P> a = repair_args<P>(m, cur, 7u, done, need, tot);
  if (tot == 0) return CHQ_OK;
  if (with_diff) {
    long nd = 0;
    a.has_diff = 1;
    a.diff = diff_args<P>(m, m->bf[cur][0], m->bf[cur][1], m->bf[cur][2], done, nd);
  }
  m->nlaunch += 1;
  fofc_repair_kernel<P><<<repair_grid(tot, kRepairBlocks).grid, 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

// One RK stage (src/main.cpp:46-93) with all decisions on the device. With explicit
// diffusion (diffusion.sts off) the diffusive fluxes join the hyperbolic ones before the
// limiter and eta J joins the corner EMFs before the update, also in the FOFC re-run.
// First part: fluxes through the update and the FOFC flags (the FOFC count is complete
// when it ends; a z slab adds the other slabs' counts before the second part).
int run_stage_a(chq_mesh *m, int cur, int out, double g0, double g1, double bdt, const double *bdt_dev,
                const int *done, cudaStream_t s) {
  int rc;
  const bool dstage = m->diff && !m->cfg.sts;
  const double *bc1 = m->bf[cur][0], *bc2 = m->bf[cur][1], *bc3 = m->bf[cur][2];
  {
    Prof p(m, PK_FLUX, s);
    if ((rc = do_fluxes(m, cur, 7u, done, s))) return rc;
  }
  if (dstage) {
    Prof p(m, PK_DIFF, s);
    if ((rc = DISPATCH_P(m, do_diff)(m, bc1, bc2, bc3, done, s))) return rc;
  }
  if (m->cfg.flux_limiter) {
    Prof p(m, PK_LIMIT, s);
    if ((rc = DISPATCH_P(m, do_limit)(m, 7u, bdt, bdt_dev, &m->ctl->limiter_count, done, s))) return rc;
  }
  {
    Prof p(m, PK_CORNER, s);
    if ((rc = DISPATCH_P(m, do_corner)(m, done, nullptr, s))) return rc;
  }
  if (dstage) {
    Prof p(m, PK_DIFF, s);
    if ((rc = DISPATCH_P(m, do_res_emf)(m, bc1, bc2, bc3, done, nullptr, s))) return rc;
  }
  {
    Prof p(m, PK_UPDATE, s);
    if ((rc = DISPATCH_P(m, do_update)(m, out, g0, g1, bdt, bdt_dev, done, nullptr, s))) return rc;
  }
  if (m->cfg.fofc) {
    Prof p(m, PK_FLAG, s);
    if ((rc = do_flag(m, out, &m->ctl->nbad, done, s))) return rc;
  }
  return CHQ_OK;
}

// Second part: the FOFC repair and re-runs when cells were flagged, then the ghost fill.
int run_stage_b(chq_mesh *m, int cur, int out, double g0, double g1, double bdt, const double *bdt_dev,
                const int *done, cudaStream_t s) {
  int rc;
  const bool dstage = m->diff && !m->cfg.sts;
  const double *bc1 = m->bf[cur][0], *bc2 = m->bf[cur][1], *bc3 = m->bf[cur][2];
  if (m->cfg.fofc) {
    int *nbad = &m->ctl->nbad;
    Prof p(m, PK_REPAIR, s);
    if (m->mixed) rc = do_repair_d<float>(m, cur, dstage, done, nbad, s);
    else rc = do_repair_d<double>(m, cur, dstage, done, nbad, s);
    if (rc) return rc;
    // with explicit diffusion eta J is added to every edge afterwards, so every edge is redone
    if (dstage) rc = DISPATCH_P(m, do_corner)(m, done, nbad, s);
    else rc = DISPATCH_P(m, do_corner_rerun)(m, done, nbad, s);
    if (rc) return rc;
    if (dstage && (rc = DISPATCH_P(m, do_res_emf)(m, bc1, bc2, bc3, done, nbad, s))) return rc;
    if ((rc = DISPATCH_P(m, do_update_rerun)(m, out, g0, g1, bdt, bdt_dev, done, nbad, s))) return rc;
  }
  Prof p(m, PK_BC, s);
  return do_bc(m, out, done, s);
}

int run_stage(chq_mesh *m, int cur, int out, double g0, double g1, double bdt, const double *bdt_dev,
              const int *done, cudaStream_t s) {
  const int rc = run_stage_a(m, cur, out, g0, g1, bdt, bdt_dev, done, s);
  return rc ? rc : run_stage_b(m, cur, out, g0, g1, bdt, bdt_dev, done, s);
}

// ---- RKL2 super-time-stepping (src/sts.hpp) ---------------------------------------------
// Number of RKL2 stages covering tau under the parabolic limit dt_par (sts::Stages).
int sts_stage_count(double tau, double dt_par) {
  const double r = tau / dt_par;
  const int s = static_cast<int>(std::ceil(0.5 * (-1.0 + std::sqrt(9.0 + 16.0 * r))));
  return (s < 2) ? 2 : s;
}

double sts_b(int j) { return (j <= 2) ? 1.0 / 3.0 : (double(j) * j + j - 2.0) / (2.0 * j * (j + 1.0)); }

struct StsState {
  double *u;
  double *b[3];
};

// M(U, B) of (cell state whose primitives are in w, face fields b) into (mu, mb): zeroed
// flux and EMF arrays, the diffusive fluxes, eta J, then -div F and -curl E (sts::Operator)
// one launch for up to six whole-array copies or zero fills of one mesh
int launch_spans(chq_mesh *m, const SpanArgs &a, cudaStream_t s) {
  long words = 0;
  for (int q = 0; q < a.nspan; ++q) words = std::max(words, a.words[q]);
  const unsigned blocks = (unsigned)std::max(1L, std::min(1184L, (words + 1023) / 1024));
  m->nlaunch += 1;
  span_kernel<<<blocks, 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

template <class P>
int sts_operator(chq_mesh *m, double *const b[3], double *mu, double *const mb[3], cudaStream_t s) {
  const Geom &g = m->g;
  {
    SpanArgs z{};   // the flux and EMF arrays start from zero (sts::Operator)
    for (int d = 0; d < 3; ++d) {
      z.dst[d] = (unsigned long long *)m->flx[d];
      z.words[d] = NVAR * (long)g.vstride * (long)m->psize / 8;
      z.dst[3 + d] = (unsigned long long *)m->e[d];
      z.words[3 + d] = (long)g.vstride * (long)m->psize / 8;
    }
    z.nspan = 6;
    if (int rc = launch_spans(m, z, s)) return rc;
  }
  int rc = do_diff<P>(m, b[0], b[1], b[2], nullptr, s);
  if (rc) return rc;
  if ((rc = do_res_emf<P>(m, b[0], b[1], b[2], nullptr, nullptr, s))) return rc;
  StsDivArgs<P> a{};
  a.g = g;
  a.f1 = as<P>(m->flx[0]); a.f2 = as<P>(m->flx[1]); a.f3 = as<P>(m->flx[2]);
  a.e1 = as<P>(m->e[0]); a.e2 = as<P>(m->e[1]); a.e3 = as<P>(m->e[2]);
  a.mu = mu;
  a.mb1 = mb[0]; a.mb2 = mb[1]; a.mb3 = mb[2];
  a.idx1 = 1.0 / g.dx1; a.idx2 = 1.0 / g.dx2; a.idx3 = 1.0 / g.dx3;
  const Launch3 L = update_grid(m);
  m->nlaunch += 1;
  sts_div_kernel<P><<<L.grid, L.block, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

// out = ((a x + b y) + c z) + (d p + e q) on active cells and update-range faces (sts::Combine)
int sts_combine(chq_mesh *m, const StsState &out, double a, const StsState &x, double b, const StsState &y, double c,
                const StsState &z, double d, const double *p, double *const pb[3], double e, const double *q,
                double *const qb[3], cudaStream_t s) {
  StsCombArgs A{};
  A.g = m->g;
  A.a = a; A.b = b; A.c = c; A.d = d; A.e = e;
  A.out = out.u; A.x = x.u; A.y = y.u; A.z = z.u; A.p = p; A.q = q;
  for (int k = 0; k < 3; ++k) {
    A.bo[k] = out.b[k]; A.bx[k] = x.b[k]; A.by[k] = y.b[k]; A.bz[k] = z.b[k]; A.bp[k] = pb[k]; A.bq[k] = qb[k];
  }
  const Launch3 L = update_grid(m);
  m->nlaunch += 1;
  sts_combine_kernel<<<L.grid, L.block, 0, s>>>(A);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

// Advance the diffusive terms over tau from (u0, b?f0), result back in them (sts::Advance).
// u1 / b?f1 serve as the fourth rotating buffer, as in the reference.
template <class P>
int sts_advance(chq_mesh *m, double tau, double dt_par, cudaStream_t s, int &nst) {
  const Geom &g = m->g;
  const size_t ub = (size_t)g.vstride * sizeof(double) * NVAR, fb = (size_t)g.vstride * sizeof(double);
  nst = sts_stage_count(tau, dt_par);
  const int ns = nst;
  const double w1 = 4.0 / (double(ns) * ns + ns - 2.0);
  StsState Y0{m->sy[0], {m->sb[0][0], m->sb[0][1], m->sb[0][2]}};
  StsState Y1{m->sy[1], {m->sb[1][0], m->sb[1][1], m->sb[1][2]}};
  StsState Y2{m->sy[2], {m->sb[2][0], m->sb[2][1], m->sb[2][2]}};
  StsState spare{m->u[1], {m->bf[1][0], m->bf[1][1], m->bf[1][2]}};
  double *M0 = m->sm0, *Mj = m->smj;
  double *MB0[3] = {m->smb0[0], m->smb0[1], m->smb0[2]}, *MBj[3] = {m->smbj[0], m->smbj[1], m->smbj[2]};
  int rc;
  // Y0 = (u0, b?f0) and, at the end, (u0, b?f0) = Y_s: whole arrays, one launch each
  auto copy = [&](double *du, double *const db[3], const double *su, const double *const sb[3]) {
    SpanArgs c{};
    c.dst[0] = (unsigned long long *)du;
    c.src[0] = (const unsigned long long *)su;
    c.words[0] = (long)(ub / 8);
    for (int k = 0; k < 3; ++k) {
      c.dst[1 + k] = (unsigned long long *)db[k];
      c.src[1 + k] = (const unsigned long long *)sb[k];
      c.words[1 + k] = (long)(fb / 8);
    }
    c.nspan = 4;
    return launch_spans(m, c, s);
  };
  if ((rc = copy(Y0.u, Y0.b, m->u[0], m->bf[0]))) return rc;
  if ((rc = launch_c2p<P>(m, c2p_args_ptr<P>(m, Y0.u, Y0.b[0], Y0.b[1], Y0.b[2], 0, nullptr, nullptr, nullptr), s)))
    return rc;
  if ((rc = sts_operator<P>(m, Y0.b, M0, MB0, s))) return rc;
  const double mt1 = double(sts_b(1) * w1) * tau;
  if ((rc = sts_combine(m, Y1, 1.0, Y0, 0.0, Y0, 0.0, Y0, mt1, M0, MB0, 0.0, M0, MB0, s))) return rc;
  if ((rc = do_bc_ptr(m, Y1.u, Y1.b[0], Y1.b[1], Y1.b[2], nullptr, s))) return rc;
  StsState yjm2 = Y0, yjm1 = Y1, yj = Y2;
  for (int j = 2; j <= ns; ++j) {
    const double b_j = sts_b(j), b_jm1 = sts_b(j - 1), b_jm2 = sts_b(j - 2);
    const double mu = (2.0 * j - 1.0) / j * b_j / b_jm1;
    const double nu = -(j - 1.0) / j * b_j / b_jm2;
    const double mut = mu * w1;
    const double gt = -(1.0 - b_jm1) * mut;
    if ((rc = launch_c2p<P>(m, c2p_args_ptr<P>(m, yjm1.u, yjm1.b[0], yjm1.b[1], yjm1.b[2], 0, nullptr, nullptr,
                                               nullptr), s)))
      return rc;
    if ((rc = sts_operator<P>(m, yjm1.b, Mj, MBj, s))) return rc;
    if ((rc = sts_combine(m, yj, mu, yjm1, nu, yjm2, 1.0 - mu - nu, Y0, mut * tau, Mj, MBj, gt * tau, M0, MB0, s)))
      return rc;
    if ((rc = do_bc_ptr(m, yj.u, yj.b[0], yj.b[1], yj.b[2], nullptr, s))) return rc;
    const StsState freed = (j == 2) ? spare : yjm2;
    yjm2 = yjm1;
    yjm1 = yj;
    yj = freed;
  }
  return copy(m->u[0], m->bf[0], yjm1.u, yjm1.b);
}

// dx_min^2 / (2 ndim max(nu, eta, chi)) on the host, same operations as parabolic_dt
double host_parabolic_dt(const chq_mesh *m, double rho_min) {
  const Geom &g = m->g;
  const int ndim = 1 + g.two_d + g.three_d;
  double dxmin = g.dx1;
  if (g.two_d) dxmin = std::fmin(dxmin, g.dx2);
  if (g.three_d) dxmin = std::fmin(dxmin, g.dx3);
  const double kappa = m->cfg.kappa, gm1 = m->cfg.gamma - 1.0;
  const double chi = (kappa > 0) ? kappa * gm1 / rho_min : 0.0;
  const double dmax = std::fmax(std::fmax(m->cfg.nu, m->cfg.eta), chi);
  return dxmin * dxmin / (2.0 * ndim * dmax);
}

// ---- layout conversion ---------------------------------------------------------------
struct FieldRef {
  void *base;
  int ncomp;
  int face;      // 1: (nk+1, nj+1, ni+1) shape; 0: cell shape
  int isp;       // 1: element type is P (float in the mixed form); 0: double
  int isint;     // the int flag array
};

bool field_by_name(chq_mesh *m, const char *n, FieldRef &f) {
  struct E { const char *name; void *base; int ncomp, face, isp, isint; };
  const E tab[] = {
      {"u0", m->u[0], 6, 0, 0, 0},      {"u1", m->u[1], 6, 0, 0, 0},      {"w", m->w, 6, 0, 1, 0},
      {"bcc", m->bcc, 3, 0, 1, 0},      {"ecc", m->ecc, 3, 0, 1, 0},      {"b1f0", m->bf[0][0], 1, 1, 0, 0},
      {"b2f0", m->bf[0][1], 1, 1, 0, 0}, {"b3f0", m->bf[0][2], 1, 1, 0, 0}, {"b1f1", m->bf[1][0], 1, 1, 0, 0},
      {"b2f1", m->bf[1][1], 1, 1, 0, 0}, {"b3f1", m->bf[1][2], 1, 1, 0, 0}, {"f1", m->flx[0], 6, 1, 1, 0},
      {"f2", m->flx[1], 6, 1, 1, 0},     {"f3", m->flx[2], 6, 1, 1, 0},     {"e2x1", m->et1[0], 1, 1, 1, 0},
      {"e3x1", m->et2[0], 1, 1, 1, 0},   {"e1x2", m->et2[1], 1, 1, 1, 0},   {"e3x2", m->et1[1], 1, 1, 1, 0},
      {"e1x3", m->et1[2], 1, 1, 1, 0},   {"e2x3", m->et2[2], 1, 1, 1, 0},   {"e1", m->e[0], 1, 1, 1, 0},
      {"e2", m->e[1], 1, 1, 1, 0},       {"e3", m->e[2], 1, 1, 1, 0},       {"flag", m->flag, 1, 0, 0, 1},
  };
  for (const E &e : tab)
    if (!std::strcmp(e.name, n)) { f = FieldRef{e.base, e.ncomp, e.face, e.isp, e.isint}; return true; }
  return false;
}

long field_size(const chq_mesh *m, const FieldRef &f) {
  const Geom &g = m->g;
  return f.face ? (long)f.ncomp * (g.nk + 1) * (g.nj + 1) * (g.ni + 1) : (long)f.ncomp * g.nk * g.nj * g.ni;
}

// element size on the device
size_t field_esize(const chq_mesh *m, const FieldRef &f) {
  if (f.isint) return sizeof(int);
  if (f.isp && m->mixed) return sizeof(float);
  return sizeof(double);
}

// Packed host planes -> the device frame: nz planes of ny rows of nx doubles, starting at
// plane k0 of one component (dst = component base). Host-to-device copies of contiguous
// packed data run at the link's full rate (the row-pitched 3-D copy reached ~60 % of it on
// a B200 host link), so uploads go through a device staging buffer and this kernel.
__global__ void __launch_bounds__(256) unpack_planes_kernel(const double *src, double *dst, int nx, int ny, int nz,
                                                            long sj, long sk, int k0) {
  const long total = (long)nx * ny * nz;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const int i = (int)(q % nx);
    const long r = q / nx;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny) + k0;
    dst[(long)k * sk + (long)j * sj + i] = src[q];
  }
}

// The device frame -> packed host planes of ncomp components (the inverse of the unpack):
// downloads of contiguous packed data run at the link's full rate.
template <class T>
__global__ void __launch_bounds__(256) pack_planes_kernel(const T *src, T *dst, int ncomp, int nx, int ny, int nz,
                                                          long sj, long sk, long vstride) {
  const long plane3 = (long)nx * ny * nz, total = plane3 * ncomp;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const int c = (int)(q / plane3);
    const long r0 = q - c * plane3;
    const int i = (int)(r0 % nx);
    const long r = r0 / nx;
    const int j = (int)(r % ny);
    const int k = (int)(r / ny);
    dst[q] = src[c * vstride + (long)k * sk + (long)j * sj + i];
  }
}

// The cell data of the reference's VTK dump (src/output.hpp:71-84) built on the device: rho,
// prs, vx1, vx2, vx3, Bx1, Bx2, Bx3 over the active cells, i fastest, each value rounded to
// float and stored big-endian, so the host writes the downloaded bytes as they are.
template <class P>
__global__ void __launch_bounds__(256) vtk_cells_kernel(Geom g, const P *w, const P *bcc, unsigned *dst) {
  const long ncell = (long)g.nx1 * g.nx2 * g.nx3, total = 8 * ncell, vs = g.vstride;
  for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < total; q += (long)gridDim.x * blockDim.x) {
    const int c = (int)(q / ncell);
    const long r0 = q - c * ncell;
    const int i = g.is + (int)(r0 % g.nx1);
    const long r = r0 / g.nx1;
    const int j = g.js + (int)(r % g.nx2);
    const int k = g.ks + (int)(r / g.nx2);
    const long l = g.idx(k, j, i);
    const P v = (c == 0) ? w[IDN * vs + l] : (c == 1) ? w[IPR * vs + l] : (c < 5) ? w[(c - 1) * vs + l]
                                                                          : bcc[(c - 5) * vs + l];
    const float f = (float)v;
    dst[q] = __byte_perm(__float_as_uint(f), 0u, 0x0123u);
  }
}

const size_t kStageBytes = 64ull << 20;   // per staging slot; planes per chunk: as many as fit
const int kStageSlots = 4;

// make s wait until every staging slot's last unpack (and so its copy) is done
int stage_fence(chq_mesh *m, cudaStream_t s) {
  for (int q = 0; q < kStageSlots; ++q)
    if (m->stage_unpacked[q]) CHQ_CUDA(cudaStreamWaitEvent(s, m->stage_unpacked[q], 0));
  return CHQ_OK;
}


// Upload of one double component in plane chunks through kStageSlots staging slots: copy
// chunk c into slot c % kStageSlots, unpack it, and copy the next chunks into the other slots
// meanwhile. On the host-job upload lane the copies run on s and the unpacks on the unpack
// lane, so the link does not wait while an unpack kernel waits for SMs that a running cycle
// holds; on any other stream both run on s.
int upload_staged(chq_mesh *m, char *dev, const double *hst, int nx, int ny, int nz, cudaStream_t s) {
  const Geom &g = m->g;
  if (!m->stage_buf) {
    cudaError_t e = cudaMalloc(&m->stage_buf, kStageSlots * kStageBytes);
    if (e != cudaSuccess) return fail(CHQ_ERR_NOMEM, std::string("upload staging: ") + cudaGetErrorString(e));
    for (int q = 0; q < kStageSlots && e == cudaSuccess; ++q) {
      e = cudaEventCreateWithFlags(&m->stage_copied[q], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->stage_unpacked[q], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) return cuda_fail(e, "upload staging events");
  }
  const bool lane = m->up_stream && s == m->up_stream;
  cudaStream_t us = lane ? m->unpack_stream : s;
  if (!lane) {
    const int rc = stage_fence(m, s);   // a queued host job may still be uploading through the slots
    if (rc) return rc;
  }
  const size_t plane = (size_t)nx * ny;   // plane * sizeof(double) <= kStageBytes (caller)
  const int per = (int)(kStageBytes / (plane * sizeof(double)));
  for (int k0 = 0; k0 < nz; k0 += per) {
    const int nzc = std::min(per, nz - k0);
    const int slot = (int)(m->stage_seq++ % kStageSlots);
    double *buf = m->stage_buf + (size_t)slot * (kStageBytes / sizeof(double));
    CHQ_CUDA(cudaStreamWaitEvent(s, m->stage_unpacked[slot], 0));   // the slot's last unpack is done
    CHQ_CUDA(cudaMemcpyAsync(buf, hst + (size_t)k0 * plane, (size_t)nzc * plane * sizeof(double),
                             cudaMemcpyHostToDevice, s));
    CHQ_CUDA(cudaEventRecord(m->stage_copied[slot], s));
    CHQ_CUDA(cudaStreamWaitEvent(us, m->stage_copied[slot], 0));
    const long tot = (long)nzc * plane;
    const unsigned blocks = (unsigned)std::min<long>((tot + 255) / 256, 148L * 16);
    m->nlaunch += 1;
    unpack_planes_kernel<<<blocks, 256, 0, us>>>(buf, reinterpret_cast<double *>(dev), nx, ny, nzc, g.sj, g.sk, k0);
    CHQ_CUDA(cudaGetLastError());
    CHQ_CUDA(cudaEventRecord(m->stage_unpacked[slot], us));
  }
  return CHQ_OK;
}

// sync = false: leave the copies queued on s (double fields only; no host conversion)
int transfer(chq_mesh *m, const char *name, double *host, long n, bool up, cudaStream_t s, bool sync = true) {
  FieldRef f;
  if (!field_by_name(m, name, f)) return fail(CHQ_ERR_ARG, std::string("unknown field: ") + name);
  if (field_size(m, f) != n) return fail(CHQ_ERR_ARG, std::string("size mismatch for field ") + name);
  const Geom &g = m->g;
  const int nx = f.face ? g.ni + 1 : g.ni, ny = f.face ? g.nj + 1 : g.nj, nz = f.face ? g.nk + 1 : g.nk;
  const size_t es = field_esize(m, f);
  // stage through a host buffer of the device element type when it is not double
  std::vector<unsigned char> tmp;
  void *hptr = host;
  if (!sync && (es != sizeof(double) || f.isint))
    return fail(CHQ_ERR_ARG, std::string("field ") + name + " needs a host conversion; it cannot be queued");
  if (es != sizeof(double) || f.isint) {
    tmp.resize((size_t)n * es);
    hptr = tmp.data();
    if (up) {
      for (long q = 0; q < n; ++q) {
        if (f.isint) reinterpret_cast<int *>(hptr)[q] = (int)host[q];
        else reinterpret_cast<float *>(hptr)[q] = (float)host[q];
      }
    }
  }
  for (int c = 0; c < f.ncomp; ++c) {
    cudaMemcpy3DParms p{};
    char *dev = static_cast<char *>(f.base) + (size_t)c * g.vstride * es;
    char *hst = static_cast<char *>(hptr) + (size_t)c * nx * ny * nz * es;
    // (a plane larger than the staging buffer takes the pitched copy below)
    if (up && es == sizeof(double) && !f.isint && (size_t)nx * ny * sizeof(double) <= kStageBytes) {
      const int rc = upload_staged(m, dev, reinterpret_cast<const double *>(hst), nx, ny, nz, s);
      if (rc) return rc;
      continue;
    }
    cudaPitchedPtr dp = make_cudaPitchedPtr(dev, (size_t)g.sj * es, (size_t)nx * es, (size_t)(g.nj + 1));
    cudaPitchedPtr hp = make_cudaPitchedPtr(hst, (size_t)nx * es, (size_t)nx * es, (size_t)ny);
    p.extent = make_cudaExtent((size_t)nx * es, (size_t)ny, (size_t)nz);
    if (up) { p.srcPtr = hp; p.dstPtr = dp; p.kind = cudaMemcpyHostToDevice; }
    else { p.srcPtr = dp; p.dstPtr = hp; p.kind = cudaMemcpyDeviceToHost; }
    CHQ_CUDA(cudaMemcpy3DAsync(&p, s));
  }
  if (!sync) return CHQ_OK;
  CHQ_CUDA(cudaStreamSynchronize(s));
  if (!up && hptr != host) {
    for (long q = 0; q < n; ++q) {
      if (f.isint) host[q] = (double)reinterpret_cast<int *>(hptr)[q];
      else host[q] = (double)reinterpret_cast<float *>(hptr)[q];
    }
  }
  return CHQ_OK;
}

}  // namespace


// =======================================================================================
// Batched stepping: the meshes of one class (same precision, reconstruction, Riemann
// solver, characteristic flag, integrator, FOFC and limiter switches) advance together with
// one launch per kernel kind per stage. Each mesh keeps its own StepCtl (dt, clock, FOFC
// decision), so results are identical to stepping it alone.
struct chq_batch {
  std::vector<chq_mesh *> jobs;
  int mixed = 0, recon = 0, rsolver = 0, charac = 0, nstage = 0, fofc = 0, limiter = 0;
  int xvar = 0;   // x-sweep kernel variant of the batched flux launch (chq_batch_autotune)
  cudaStream_t stream = nullptr;
  char *dev = nullptr;
  struct Kind {
    BatchSlot *slots = nullptr;
    long nblocks = 0;
  };
  Kind k_flux, k_flux_yz, k_corner, k_update, k_flag, k_repair, k_limit, k_bc[3], k_c2p;
  // source terms and diffusion (every member or none): with explicit diffusion (diff) the
  // stage adds the diffusive fluxes after K1 and eta J after the corner EMFs; gravity runs in
  // the update epilogue; cooling is split after the step
  int diff = 0, grav = 0, cool = 0;
  int sts = 0;   // RKL2 members: super-time-stepping stages batched after the hyperbolic stages
  Kind k_diff, k_res, k_rho, k_cool, k_corner_rerun;
  // batched RKL2 stages: argument tables per state buffer (Y0, Y1, Y2, u1) and per stage form,
  // built once; stage counts, coefficients and the final copies are uploaded every cycle
  Kind k_span;
  void *a_sts_c2p[4] = {}, *a_sts_diff[4] = {}, *a_sts_res[4] = {}, *a_sts_div[2] = {}, *a_sts_comb[5] = {},
       *a_sts_bc[4][3] = {}, *a_sts_zero = nullptr, *a_sts_copy0 = nullptr;
  int *sts_skip = nullptr;   // per member: skip the current RKL2 stage
  char *sts_dyn = nullptr;   // per cycle: stage counts | coefficients | final copies
  size_t sts_dyn_bytes = 0;
  void *a_diff[4] = {}, *a_res[4] = {}, *a_res_need[4] = {};
  void *a_rho = nullptr, *a_cool = nullptr, *a_c2p_split[2] = {}, *a_bc0[3] = {};
  void *a_flux[4] = {}, *a_update[4] = {}, *a_update_need[4] = {}, *a_repair[4] = {}, *a_limit[4] = {},
       *a_c2p[4] = {}, *a_flag[4] = {}, *a_bc[4][3] = {};
  void *a_corner = nullptr, *a_corner_need = nullptr;
  StepCtl **ctls = nullptr;
  double *status = nullptr;
  cudaEvent_t done_evt = nullptr;   // recorded after every chq_batch_cycles call
  bool use_graph = false;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long nlaunch = 0;
  long long per_cycle = 0;   // launches in one captured cycle
};

namespace {

struct HostTable {
  std::vector<char> b;
  size_t push(const void *p, size_t n) {
    const size_t off = (b.size() + 255) & ~size_t(255);
    b.resize(off + n);
    std::memcpy(b.data() + off, p, n);
    return off;
  }
};

template <class T>
size_t push_vec(HostTable &h, const std::vector<T> &v) {
  return h.push(v.data(), v.size() * sizeof(T));
}

template <class F>
size_t slots_of(HostTable &h, const std::vector<chq_mesh *> &jobs, F grid, long &total) {
  std::vector<BatchSlot> v(jobs.size());
  long off = 0;
  for (size_t j = 0; j < jobs.size(); ++j) {
    const Launch3 L = grid(jobs[j]);
    v[j] = BatchSlot{off, (int)L.grid.x, (int)L.grid.y, (int)L.grid.z, 0};
    off += (long)L.grid.x * L.grid.y * L.grid.z;
  }
  total = off;
  return push_vec(h, v);
}

Launch3 linear(long threads, int per) { return {dim3((unsigned)((threads + per - 1) / per), 1, 1), dim3(per)}; }

template <class P>
int batch_build(chq_batch *B) {
  HostTable h;
  const std::vector<chq_mesh *> &J = B->jobs;
  const int n = (int)J.size();
  size_t o_flux_s, o_corner_s, o_update_s, o_flag_s, o_repair_s, o_limit_s, o_bc_s[3], o_c2p_s;
  o_flux_s = slots_of(h, J, [](chq_mesh *m) {
    const FluxArgs<P> a = flux_args<P>(m, 0, 7u);
    return linear(a.nwarp[0] * 32, 128);
  }, B->k_flux.nblocks);
  const size_t o_flux_yz_s = slots_of(h, J, [](chq_mesh *m) {
    const FluxArgs<P> a = flux_args<P>(m, 0, 7u);
    return linear((a.nwarp[1] + a.nwarp[2]) * 32, kYzThreads);
  }, B->k_flux_yz.nblocks);
  o_corner_s = slots_of(h, J, [](chq_mesh *m) { return corner_grid(m); }, B->k_corner.nblocks);
  o_update_s = slots_of(h, J, [](chq_mesh *m) { return update_grid(m); }, B->k_update.nblocks);
  o_flag_s = slots_of(h, J, [](chq_mesh *m) { return flag_grid(m); }, B->k_flag.nblocks);
  o_repair_s = slots_of(h, J, [](chq_mesh *m) {
    long tot = 0;
    repair_args<P>(m, 0, 7u, nullptr, nullptr, tot);
    return repair_grid(tot, kRepairBlocksBatched);
  }, B->k_repair.nblocks);
  o_limit_s = slots_of(h, J, [](chq_mesh *m) {
    long tot = 0;
    limit_args<P>(m, 7u, 0.0, nullptr, nullptr, nullptr, tot);
    return linear(tot, 256);
  }, B->k_limit.nblocks);
  for (int d = 0; d < 3; ++d)
    o_bc_s[d] = slots_of(h, J, [d](chq_mesh *m) { return linear(bc_threads(m, d), 256); }, B->k_bc[d].nblocks);
  o_c2p_s = slots_of(h, J, [](chq_mesh *m) { return c2p_grid(m); }, B->k_c2p.nblocks);
  const size_t o_diff_s = slots_of(h, J, [](chq_mesh *m) {
    long tot = 0;
    if (m->diff) diff_args<P>(m, m->bf[0][0], m->bf[0][1], m->bf[0][2], nullptr, tot);
    return linear(tot, 256);
  }, B->k_diff.nblocks);
  const size_t o_res_s = slots_of(h, J, [](chq_mesh *m) { return res_emf_grid(m); }, B->k_res.nblocks);
  const size_t o_crr_s = slots_of(h, J, [](chq_mesh *m) {
    const Geom &g = m->g;
    const long pts = (long)(g.ie + 2 - g.is) * (g.je + 2 - g.js) * (g.three_d ? g.ke + 2 - g.ks : 1);
    return repair_grid(pts, kRepairBlocksBatched);
  }, B->k_corner_rerun.nblocks);
  const size_t o_rho_s = slots_of(h, J, [](chq_mesh *m) {
    return m->diff ? active_grid(m) : Launch3{dim3(0, 1, 1), dim3(32, 8)};
  }, B->k_rho.nblocks);
  const size_t o_cool_s = slots_of(h, J, [](chq_mesh *m) {
    return m->cfg.cooling ? active_grid(m) : Launch3{dim3(0, 1, 1), dim3(32, 8)};
  }, B->k_cool.nblocks);

  std::vector<EmfArgs<P>> corner(n), corner_need(n);
  std::vector<StepCtl *> ctls(n);
  for (int j = 0; j < n; ++j) {
    chq_mesh *m = J[j];
    corner[j] = corner_args<P>(m, &m->ctl->done, nullptr);
    corner_need[j] = corner_args<P>(m, &m->ctl->done, &m->ctl->nbad);
    ctls[j] = m->ctl;
  }
  const size_t o_corner = push_vec(h, corner), o_corner_need = push_vec(h, corner_need), o_ctls = push_vec(h, ctls);
  size_t o_flux[4], o_update[4], o_update_need[4], o_flag[4], o_repair[4], o_limit[4], o_bc[4][3], o_c2p[4];
  size_t o_diff[4] = {}, o_res[4] = {}, o_res_need[4] = {};
  // the cooling split: con2prim of u0 without and with the dt, cooling, boundaries of u0
  std::vector<RhoMinArgs<P>> rho(n);
  std::vector<CoolArgs<P>> cool(n);
  std::vector<C2pArgs<P>> split0(n), split1(n);
  std::vector<BcArgs> bc0[3] = {std::vector<BcArgs>(n), std::vector<BcArgs>(n), std::vector<BcArgs>(n)};
  for (int j = 0; j < n; ++j) {
    chq_mesh *m = J[j];
    StepCtl *c = m->ctl;
    rho[j] = rho_min_args<P>(m, &c->done);
    cool[j] = cool_args<P>(m, &c->done);
    split0[j] = c2p_args<P>(m, 0, 0, &c->mdt_bits, c, &c->done);
    split1[j] = c2p_args<P>(m, 0, 1, &c->mdt_bits, c, &c->done);
    for (int d = 0; d < 3; ++d) bc0[d][j] = bc_args(m, 0, &c->done, d);
  }
  const size_t o_rho = push_vec(h, rho), o_cool = push_vec(h, cool), o_split0 = push_vec(h, split0),
               o_split1 = push_vec(h, split1);
  size_t o_bc0[3];
  for (int d = 0; d < 3; ++d) o_bc0[d] = push_vec(h, bc0[d]);
  for (int st = 1; st <= B->nstage; ++st) {
    double g0, g1, beta;
    int cur, out;
    stage_table(B->nstage, st, g0, g1, beta, cur, out);
    const bool last = (st == B->nstage);
    std::vector<FluxArgs<P>> fa(n);
    std::vector<UpdateArgs<P>> ua(n), uan(n);
    std::vector<FlagArgs> fl(n);
    std::vector<RepairArgs<P>> ra(n);
    std::vector<LimitArgs<P>> la(n);
    std::vector<BcArgs> bc[3] = {std::vector<BcArgs>(n), std::vector<BcArgs>(n), std::vector<BcArgs>(n)};
    std::vector<C2pArgs<P>> ca(n);
    std::vector<DiffArgs<P>> da(n);
    std::vector<ResEmfArgs<P>> ea(n), ean(n);
    for (int j = 0; j < n; ++j) {
      chq_mesh *m = J[j];
      StepCtl *c = m->ctl;
      const double *bc1 = m->bf[cur][0], *bc2 = m->bf[cur][1], *bc3 = m->bf[cur][2];
      long nd = 0;
      da[j] = diff_args<P>(m, bc1, bc2, bc3, &c->done, nd);
      ea[j] = res_emf_args<P>(m, bc1, bc2, bc3, &c->done, nullptr);
      ean[j] = res_emf_args<P>(m, bc1, bc2, bc3, &c->done, &c->nbad);
      fa[j] = flux_args<P>(m, cur, 7u);
      fa[j].skip = &c->done;
      ua[j] = update_args<P>(m, out, g0, g1, 0.0, &c->beta_dt[st - 1], &c->done, nullptr);
      uan[j] = update_args<P>(m, out, g0, g1, 0.0, &c->beta_dt[st - 1], &c->done, &c->nbad);
      fl[j] = flag_args(m, out, &c->nbad, &c->done);
      long tot = 0;
      ra[j] = repair_args<P>(m, cur, 7u, &c->done, &c->nbad, tot);
      if (m->diff && !m->cfg.sts) {
        ra[j].has_diff = 1;
        ra[j].diff = da[j];
      }
      la[j] = limit_args<P>(m, 7u, 0.0, &c->beta_dt[st - 1], &c->limiter_count, &c->done, tot);
      for (int d = 0; d < 3; ++d) bc[d][j] = bc_args(m, out, &c->done, d);
      const bool split = m->cfg.cooling || (m->diff && m->cfg.sts);
      ca[j] = c2p_args<P>(m, out, (last && !split) ? 1 : 0, &c->mdt_bits, c, &c->done);
    }
    o_diff[st - 1] = push_vec(h, da);
    o_res[st - 1] = push_vec(h, ea);
    o_res_need[st - 1] = push_vec(h, ean);
    o_flux[st - 1] = push_vec(h, fa);
    o_update[st - 1] = push_vec(h, ua);
    o_update_need[st - 1] = push_vec(h, uan);
    o_flag[st - 1] = push_vec(h, fl);
    o_repair[st - 1] = push_vec(h, ra);
    o_limit[st - 1] = push_vec(h, la);
    for (int d = 0; d < 3; ++d) o_bc[st - 1][d] = push_vec(h, bc[d]);
    o_c2p[st - 1] = push_vec(h, ca);
  }
  // batched RKL2 stages (src/sts.hpp:111-157 per member): the state buffers of stage j rotate
  // as in the reference, the same way for every member, so their tables are fixed
  size_t o_span_s = 0, o_sts_c2p[4] = {}, o_sts_diff[4] = {}, o_sts_res[4] = {}, o_sts_div[2] = {}, o_sts_comb[5] = {},
         o_sts_bc[4][3] = {}, o_sts_zero = 0, o_sts_copy0 = 0;
  if (B->sts) {
    cudaError_t e0 = cudaMalloc(&B->sts_skip, sizeof(int) * (size_t)n);
    if (e0 == cudaSuccess) e0 = cudaMemset(B->sts_skip, 0, sizeof(int) * (size_t)n);
    // the memset runs on the legacy default stream, which the batch's non-blocking stream does
    // not wait for: complete it before any batch kernel can read the flags
    if (e0 == cudaSuccess) e0 = cudaStreamSynchronize(cudaStreamLegacy);
    if (e0 != cudaSuccess) return cuda_fail(e0, "batch RKL2 flags");
    o_span_s = slots_of(h, J, [](chq_mesh *m) {
      const long words = (long)(3 * NVAR + 3) * (long)m->g.vstride * (long)m->psize / 8;
      return Launch3{dim3((unsigned)std::max(1L, std::min(1184L, (words + 4095) / 4096)), 1, 1), dim3(256)};
    }, B->k_span.nblocks);
    std::vector<C2pArgs<P>> c2(n);
    std::vector<DiffArgs<P>> df(n);
    std::vector<ResEmfArgs<P>> rs(n);
    std::vector<StsDivArgs<P>> dv(n);
    std::vector<StsCombArgs> cb(n);
    std::vector<BcArgs> bb(n);
    auto U = [](chq_mesh *m, int b) { return b < 3 ? m->sy[b] : m->u[1]; };
    auto BF = [](chq_mesh *m, int b, int d) { return b < 3 ? m->sb[b][d] : m->bf[1][d]; };
    for (int b = 0; b < 4; ++b) {
      for (int j = 0; j < n; ++j) {
        chq_mesh *m = J[j];
        const int *skip = B->sts_skip + j;
        long nd = 0;
        c2[j] = c2p_args_ptr<P>(m, U(m, b), BF(m, b, 0), BF(m, b, 1), BF(m, b, 2), 0, nullptr, nullptr, skip);
        df[j] = diff_args<P>(m, BF(m, b, 0), BF(m, b, 1), BF(m, b, 2), skip, nd);
        rs[j] = res_emf_args<P>(m, BF(m, b, 0), BF(m, b, 1), BF(m, b, 2), skip, nullptr);
      }
      o_sts_c2p[b] = push_vec(h, c2);
      o_sts_diff[b] = push_vec(h, df);
      o_sts_res[b] = push_vec(h, rs);
      for (int d = 0; d < 3; ++d) {
        for (int j = 0; j < n; ++j) {
          bb[j] = bc_args(J[j], 0, B->sts_skip + j, d);
          bb[j].u = U(J[j], b);
          bb[j].b1 = BF(J[j], b, 0); bb[j].b2 = BF(J[j], b, 1); bb[j].b3 = BF(J[j], b, 2);
        }
        o_sts_bc[b][d] = push_vec(h, bb);
      }
    }
    for (int v = 0; v < 2; ++v) {   // M0 (first stage) or Mj
      for (int j = 0; j < n; ++j) {
        chq_mesh *m = J[j];
        const Geom &g = m->g;
        StsDivArgs<P> a{};
        a.g = g;
        a.f1 = as<P>(m->flx[0]); a.f2 = as<P>(m->flx[1]); a.f3 = as<P>(m->flx[2]);
        a.e1 = as<P>(m->e[0]); a.e2 = as<P>(m->e[1]); a.e3 = as<P>(m->e[2]);
        a.mu = v ? m->smj : m->sm0;
        a.mb1 = v ? m->smbj[0] : m->smb0[0]; a.mb2 = v ? m->smbj[1] : m->smb0[1]; a.mb3 = v ? m->smbj[2] : m->smb0[2];
        a.idx1 = 1.0 / g.dx1; a.idx2 = 1.0 / g.dx2; a.idx3 = 1.0 / g.dx3;
        a.done = B->sts_skip + j;
        dv[j] = a;
      }
      o_sts_div[v] = push_vec(h, dv);
    }
    // (out, x, y) buffers of the five stage forms: stage 1, stage 2, then j = 3, 4, 5 mod 3
    const int form[5][3] = {{1, 0, 0}, {2, 1, 0}, {3, 2, 1}, {1, 3, 2}, {2, 1, 3}};
    for (int v = 0; v < 5; ++v) {
      for (int j = 0; j < n; ++j) {
        chq_mesh *m = J[j];
        StsCombArgs a{};
        a.g = m->g;
        a.out = U(m, form[v][0]); a.x = U(m, form[v][1]); a.y = U(m, form[v][2]); a.z = U(m, 0);
        a.p = v ? m->smj : m->sm0;
        a.q = m->sm0;
        for (int d = 0; d < 3; ++d) {
          a.bo[d] = BF(m, form[v][0], d); a.bx[d] = BF(m, form[v][1], d); a.by[d] = BF(m, form[v][2], d);
          a.bz[d] = BF(m, 0, d);
          a.bp[d] = v ? m->smbj[d] : m->smb0[d];
          a.bq[d] = m->smb0[d];
        }
        a.done = B->sts_skip + j;
        cb[j] = a;
      }
      o_sts_comb[v] = push_vec(h, cb);
    }
    std::vector<SpanArgs> zero(n), copy0(n);
    for (int j = 0; j < n; ++j) {   // flux and EMF zero fill; Y0 = (u0, b?f0)
      chq_mesh *m = J[j];
      const long vs = (long)m->g.vstride;
      SpanArgs z{}, c{};
      for (int d = 0; d < 3; ++d) {
        z.dst[d] = (unsigned long long *)m->flx[d];
        z.words[d] = NVAR * vs * (long)m->psize / 8;
        z.dst[3 + d] = (unsigned long long *)m->e[d];
        z.words[3 + d] = vs * (long)m->psize / 8;
      }
      z.nspan = 6;
      z.done = B->sts_skip + j;
      zero[j] = z;
      c.dst[0] = (unsigned long long *)m->sy[0];
      c.src[0] = (const unsigned long long *)m->u[0];
      c.words[0] = NVAR * vs;
      for (int d = 0; d < 3; ++d) {
        c.dst[1 + d] = (unsigned long long *)m->sb[0][d];
        c.src[1 + d] = (const unsigned long long *)m->bf[0][d];
        c.words[1 + d] = vs;
      }
      c.nspan = 4;
      c.done = &m->ctl->done;
      copy0[j] = c;
    }
    o_sts_zero = push_vec(h, zero);
    o_sts_copy0 = push_vec(h, copy0);
  }
  const size_t o_status = h.push(std::vector<double>(3 * n + 1).data(), (3 * n + 1) * sizeof(double));
  // allocated and uploaded on the legacy default stream, which then completes both
  cudaError_t e = pool_alloc(reinterpret_cast<void **>(&B->dev), h.b.size(), cudaStreamLegacy);
  if (e != cudaSuccess) return fail(CHQ_ERR_NOMEM, std::string("batch tables: ") + cudaGetErrorString(e));
  e = cudaMemcpy(B->dev, h.b.data(), h.b.size(), cudaMemcpyHostToDevice);
  // from pageable memory cudaMemcpy may return before the transfer has landed, and the
  // batch's non-blocking stream does not wait for the legacy default stream that carries it:
  // complete it before any batch kernel can read the tables
  if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
  if (e != cudaSuccess) return cuda_fail(e, "batch tables upload");
  char *d = B->dev;
  B->k_flux.slots = (BatchSlot *)(d + o_flux_s);
  B->k_flux_yz.slots = (BatchSlot *)(d + o_flux_yz_s);
  B->k_corner.slots = (BatchSlot *)(d + o_corner_s);
  B->k_update.slots = (BatchSlot *)(d + o_update_s);
  B->k_flag.slots = (BatchSlot *)(d + o_flag_s);
  B->k_repair.slots = (BatchSlot *)(d + o_repair_s);
  B->k_limit.slots = (BatchSlot *)(d + o_limit_s);
  for (int q = 0; q < 3; ++q) B->k_bc[q].slots = (BatchSlot *)(d + o_bc_s[q]);
  B->k_c2p.slots = (BatchSlot *)(d + o_c2p_s);
  B->a_corner = d + o_corner;
  B->a_corner_need = d + o_corner_need;
  B->ctls = (StepCtl **)(d + o_ctls);
  B->status = (double *)(d + o_status);
  B->k_diff.slots = (BatchSlot *)(d + o_diff_s);
  B->k_res.slots = (BatchSlot *)(d + o_res_s);
  B->k_corner_rerun.slots = (BatchSlot *)(d + o_crr_s);
  B->k_rho.slots = (BatchSlot *)(d + o_rho_s);
  B->k_cool.slots = (BatchSlot *)(d + o_cool_s);
  B->a_rho = d + o_rho;
  B->a_cool = d + o_cool;
  B->a_c2p_split[0] = d + o_split0;
  B->a_c2p_split[1] = d + o_split1;
  for (int q = 0; q < 3; ++q) B->a_bc0[q] = d + o_bc0[q];
  if (B->sts) {
    B->k_span.slots = (BatchSlot *)(d + o_span_s);
    for (int b = 0; b < 4; ++b) {
      B->a_sts_c2p[b] = d + o_sts_c2p[b];
      B->a_sts_diff[b] = d + o_sts_diff[b];
      B->a_sts_res[b] = d + o_sts_res[b];
      for (int q = 0; q < 3; ++q) B->a_sts_bc[b][q] = d + o_sts_bc[b][q];
    }
    for (int v = 0; v < 2; ++v) B->a_sts_div[v] = d + o_sts_div[v];
    for (int v = 0; v < 5; ++v) B->a_sts_comb[v] = d + o_sts_comb[v];
    B->a_sts_zero = d + o_sts_zero;
    B->a_sts_copy0 = d + o_sts_copy0;
  }
  for (int st = 0; st < B->nstage; ++st) {
    B->a_diff[st] = d + o_diff[st];
    B->a_res[st] = d + o_res[st];
    B->a_res_need[st] = d + o_res_need[st];
    B->a_flux[st] = d + o_flux[st];
    B->a_update[st] = d + o_update[st];
    B->a_update_need[st] = d + o_update_need[st];
    B->a_flag[st] = d + o_flag[st];
    B->a_repair[st] = d + o_repair[st];
    B->a_limit[st] = d + o_limit[st];
    for (int q = 0; q < 3; ++q) B->a_bc[st][q] = d + o_bc[st][q];
    B->a_c2p[st] = d + o_c2p[st];
  }
  return CHQ_OK;
}

template <class P>
cudaError_t batch_flux(const chq_batch *B, const FluxArgs<P> *args, cudaStream_t s) {
  const int n = (int)B->jobs.size();
  const unsigned nbx = (unsigned)B->k_flux.nblocks, nbyz = (unsigned)B->k_flux_yz.nblocks;
  const BatchSlot *sx = B->k_flux.slots, *syz = B->k_flux_yz.slots;
  switch (B->recon) {
    case R_DC: return launch_flux_batched<P, R_DC>(args, sx, syz, n, B->rsolver, B->charac, nbx, nbyz, B->xvar, s);
    case R_PLM: return launch_flux_batched<P, R_PLM>(args, sx, syz, n, B->rsolver, B->charac, nbx, nbyz, B->xvar, s);
    case R_PPM: return launch_flux_batched<P, R_PPM>(args, sx, syz, n, B->rsolver, B->charac, nbx, nbyz, B->xvar, s);
    case R_PPMX: return launch_flux_batched<P, R_PPMX>(args, sx, syz, n, B->rsolver, B->charac, nbx, nbyz, B->xvar, s);
    case R_WENOZ: return launch_flux_batched<P, R_WENOZ>(args, sx, syz, n, B->rsolver, B->charac, nbx, nbyz, B->xvar, s);
    default: return cudaErrorInvalidValue;
  }
}

// The RKL2 part of a batched cycle (src/main.cpp:274-281, src/sts.hpp:111-157). Each member's
// stage count is a host decision on its dt and density minimum, so the batch stream is
// synchronised once; then stage j of every member runs in one launch per kernel kind (members
// with fewer stages skip), the coefficients read from a per-cycle table, and each member's
// result is copied back from the buffer its last stage wrote.
template <class P>
int batch_sts(chq_batch *B, cudaStream_t s, long long &L) {
  const int n = (int)B->jobs.size();
  std::vector<StepCtl> h(n);
  for (int j = 0; j < n; ++j)
    CHQ_CUDA(cudaMemcpyAsync(&h[j], B->jobs[j]->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s));
  CHQ_CUDA(cudaStreamSynchronize(s));
  std::vector<int> nst(n, 0);
  int smax = 0;
  for (int j = 0; j < n; ++j) {
    if (h[j].done) continue;
    double rho_min;
    std::memcpy(&rho_min, &h[j].rho_bits, sizeof(rho_min));
    nst[j] = sts_stage_count(h[j].dt, host_parabolic_dt(B->jobs[j], rho_min));
    smax = std::max(smax, nst[j]);
  }
  if (smax == 0) return CHQ_OK;
  // buffer written by stage j (0: Y0): Y1, Y2, then u1, Y1, Y2, ... (the reference's rotation)
  auto wrote = [](int j) { return j == 0 ? 0 : j == 1 ? 1 : j == 2 ? 2 : (j % 3 == 0) ? 3 : (j % 3 == 1) ? 1 : 2; };
  // per-cycle table: stage counts | coefficients (stage j, member m: 5 doubles) | final copies
  const size_t o_coef = align_up(sizeof(int) * (size_t)n, 256);
  const size_t o_fin = align_up(o_coef + sizeof(double) * 5 * (size_t)n * smax, 256);
  const size_t bytes = o_fin + sizeof(SpanArgs) * (size_t)n;
  std::vector<char> tab(bytes, 0);
  std::memcpy(tab.data(), nst.data(), sizeof(int) * (size_t)n);
  double *coef = reinterpret_cast<double *>(tab.data() + o_coef);
  SpanArgs *fin = reinterpret_cast<SpanArgs *>(tab.data() + o_fin);
  for (int j = 0; j < n; ++j) {
    chq_mesh *m = B->jobs[j];
    const long vs = (long)m->g.vstride;
    const int ns = nst[j];
    if (ns) {
      const double tau = h[j].dt;
      const double w1 = 4.0 / (double(ns) * ns + ns - 2.0);
      double *c = coef + 5 * (size_t)j;
      c[0] = 1.0; c[1] = 0.0; c[2] = 0.0; c[3] = double(sts_b(1) * w1) * tau; c[4] = 0.0;
      for (int st = 2; st <= ns; ++st) {
        const double b_j = sts_b(st), b_jm1 = sts_b(st - 1), b_jm2 = sts_b(st - 2);
        const double mu = (2.0 * st - 1.0) / st * b_j / b_jm1;
        const double nu = -(st - 1.0) / st * b_j / b_jm2;
        const double mut = mu * w1;
        const double gt = -(1.0 - b_jm1) * mut;
        c = coef + 5 * ((size_t)(st - 1) * n + j);
        c[0] = mu; c[1] = nu; c[2] = 1.0 - mu - nu; c[3] = mut * tau; c[4] = gt * tau;
      }
    }
    const int b = wrote(ns);
    SpanArgs &f = fin[j];
    f.dst[0] = (unsigned long long *)m->u[0];
    f.src[0] = (const unsigned long long *)(b < 3 ? m->sy[b] : m->u[1]);
    f.words[0] = NVAR * vs;
    for (int d = 0; d < 3; ++d) {
      f.dst[1 + d] = (unsigned long long *)m->bf[0][d];
      f.src[1 + d] = (const unsigned long long *)(b < 3 ? m->sb[b][d] : m->bf[1][d]);
      f.words[1 + d] = vs;
    }
    f.nspan = 4;
    f.done = &m->ctl->done;
    m->sts_stages += ns;
  }
  if (bytes > B->sts_dyn_bytes) {
    if (B->sts_dyn) CHQ_CUDA(cudaFree(B->sts_dyn));
    B->sts_dyn = nullptr;
    B->sts_dyn_bytes = 0;
    CHQ_CUDA(cudaMalloc(&B->sts_dyn, bytes));
    B->sts_dyn_bytes = bytes;
  }
  CHQ_CUDA(cudaMemcpyAsync(B->sts_dyn, tab.data(), bytes, cudaMemcpyHostToDevice, s));
  CHQ_CUDA(cudaStreamSynchronize(s));   // the host table is freed on return
  const int *nst_dev = reinterpret_cast<const int *>(B->sts_dyn);
  const double *coef_dev = reinterpret_cast<const double *>(B->sts_dyn + o_coef);
  const dim3 b2(32, 8);
  const unsigned nspan = (unsigned)B->k_span.nblocks;
  span_batched<<<nspan, 256, 0, s>>>((const SpanArgs *)B->a_sts_copy0, B->k_span.slots, n);
  CHQ_CUDA(cudaGetLastError());
  ++L;
  for (int st = 1; st <= smax; ++st) {
    const int bi = wrote(st - 1), bo = wrote(st);
    const int form = st == 1 ? 0 : st == 2 ? 1 : 2 + (st % 3);
    sts_skip_kernel<<<(n + 127) / 128, 128, 0, s>>>(B->sts_skip, nst_dev, n, st);
    c2p_batched<P><<<(unsigned)B->k_c2p.nblocks, b2, 0, s>>>((const C2pArgs<P> *)B->a_sts_c2p[bi], B->k_c2p.slots, n);
    span_batched<<<nspan, 256, 0, s>>>((const SpanArgs *)B->a_sts_zero, B->k_span.slots, n);
    CHQ_CUDA(cudaGetLastError());
    L += 3;
    if (B->k_diff.nblocks) {
      diff_flux_batched<P><<<(unsigned)B->k_diff.nblocks, 256, 0, s>>>((const DiffArgs<P> *)B->a_sts_diff[bi],
                                                                        B->k_diff.slots, n);
      ++L;
    }
    if (B->k_res.nblocks) {
      resistive_emf_batched<P><<<(unsigned)B->k_res.nblocks, b2, 0, s>>>((const ResEmfArgs<P> *)B->a_sts_res[bi],
                                                                         B->k_res.slots, n);
      ++L;
    }
    sts_div_batched<P><<<(unsigned)B->k_update.nblocks, b2, 0, s>>>((const StsDivArgs<P> *)B->a_sts_div[st == 1 ? 0 : 1],
                                                                      B->k_update.slots, n);
    sts_combine_batched<<<(unsigned)B->k_update.nblocks, b2, 0, s>>>((const StsCombArgs *)B->a_sts_comb[form],
                                                                      B->k_update.slots, n,
                                                                      coef_dev + 5 * (size_t)(st - 1) * n);
    CHQ_CUDA(cudaGetLastError());
    L += 2;
    if (B->k_bc[0].nblocks) bc_batched<0><<<(unsigned)B->k_bc[0].nblocks, 256, 0, s>>>((const BcArgs *)B->a_sts_bc[bo][0], B->k_bc[0].slots, n);
    if (B->k_bc[1].nblocks) bc_batched<1><<<(unsigned)B->k_bc[1].nblocks, 256, 0, s>>>((const BcArgs *)B->a_sts_bc[bo][1], B->k_bc[1].slots, n);
    if (B->k_bc[2].nblocks) bc_batched<2><<<(unsigned)B->k_bc[2].nblocks, 256, 0, s>>>((const BcArgs *)B->a_sts_bc[bo][2], B->k_bc[2].slots, n);
    CHQ_CUDA(cudaGetLastError());
    L += (B->k_bc[0].nblocks > 0) + (B->k_bc[1].nblocks > 0) + (B->k_bc[2].nblocks > 0);
  }
  span_batched<<<nspan, 256, 0, s>>>((const SpanArgs *)(B->sts_dyn + o_fin), B->k_span.slots, n);
  CHQ_CUDA(cudaGetLastError());
  ++L;
  // the boundaries of the result in u0 / b?f0 (src/main.cpp:280)
  if (B->k_bc[0].nblocks) bc_batched<0><<<(unsigned)B->k_bc[0].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc0[0], B->k_bc[0].slots, n);
  if (B->k_bc[1].nblocks) bc_batched<1><<<(unsigned)B->k_bc[1].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc0[1], B->k_bc[1].slots, n);
  if (B->k_bc[2].nblocks) bc_batched<2><<<(unsigned)B->k_bc[2].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc0[2], B->k_bc[2].slots, n);
  CHQ_CUDA(cudaGetLastError());
  L += (B->k_bc[0].nblocks > 0) + (B->k_bc[1].nblocks > 0) + (B->k_bc[2].nblocks > 0);
  return CHQ_OK;
}

// one cycle of every member: the launch sequence of chq_cycles, batched
template <class P>
int batch_cycle(chq_batch *B, cudaStream_t s) {
  const int n = (int)B->jobs.size();
  const dim3 b2(32, 8);
  long long &L = B->nlaunch;
  ctl_begin_batched<<<(n + 127) / 128, 128, 0, s>>>(B->ctls, n);
  CHQ_CUDA(cudaGetLastError());
  ++L;
  for (int st = 0; st < B->nstage; ++st) {
    CHQ_CUDA(batch_flux<P>(B, (const FluxArgs<P> *)B->a_flux[st], s));
    ++L;
    if (B->diff && B->k_diff.nblocks) {
      diff_flux_batched<P><<<(unsigned)B->k_diff.nblocks, 256, 0, s>>>((const DiffArgs<P> *)B->a_diff[st], B->k_diff.slots, n);
      CHQ_CUDA(cudaGetLastError());
      ++L;
    }
    if (B->limiter && B->k_limit.nblocks) {
      limit_batched<P><<<(unsigned)B->k_limit.nblocks, 256, 0, s>>>((const LimitArgs<P> *)B->a_limit[st], B->k_limit.slots, n);
      CHQ_CUDA(cudaGetLastError());
      ++L;
    }
    auto update = [&](const void *args) -> cudaError_t {
      if (B->grav)
        update_batched<P, true><<<(unsigned)B->k_update.nblocks, b2, 0, s>>>((const UpdateArgs<P> *)args, B->k_update.slots, n);
      else
        update_batched<P, false><<<(unsigned)B->k_update.nblocks, b2, 0, s>>>((const UpdateArgs<P> *)args, B->k_update.slots, n);
      ++L;
      return cudaGetLastError();
    };
    auto res_emf = [&](const void *args) -> cudaError_t {
      if (!B->diff || !B->k_res.nblocks) return cudaSuccess;
      resistive_emf_batched<P><<<(unsigned)B->k_res.nblocks, b2, 0, s>>>((const ResEmfArgs<P> *)args, B->k_res.slots, n);
      ++L;
      return cudaGetLastError();
    };
    corner_emf_batched<P><<<(unsigned)B->k_corner.nblocks, b2, 0, s>>>((const EmfArgs<P> *)B->a_corner, B->k_corner.slots, n);
    CHQ_CUDA(cudaGetLastError());
    ++L;
    CHQ_CUDA(res_emf(B->a_res[st]));
    CHQ_CUDA(update(B->a_update[st]));
    if (B->fofc) {
      fofc_flag_batched<<<(unsigned)B->k_flag.nblocks, b2, 0, s>>>((const FlagArgs *)B->a_flag[st], B->k_flag.slots, n);
      CHQ_CUDA(cudaGetLastError());
      fofc_repair_batched<P><<<(unsigned)B->k_repair.nblocks, 256, 0, s>>>((const RepairArgs<P> *)B->a_repair[st], B->k_repair.slots, n);
      CHQ_CUDA(cudaGetLastError());
      // (with explicit diffusion eta J is added to every edge afterwards: every edge is redone)
      if (B->diff)
        corner_emf_batched<P><<<(unsigned)B->k_corner.nblocks, b2, 0, s>>>((const EmfArgs<P> *)B->a_corner_need, B->k_corner.slots, n);
      else
        corner_rerun_batched<P><<<(unsigned)B->k_corner_rerun.nblocks, 256, 0, s>>>((const EmfArgs<P> *)B->a_corner_need, B->k_corner_rerun.slots, n);
      CHQ_CUDA(cudaGetLastError());
      L += 3;
      CHQ_CUDA(res_emf(B->a_res_need[st]));
      CHQ_CUDA(update(B->a_update_need[st]));
    }
    bc_batched<0><<<(unsigned)B->k_bc[0].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc[st][0], B->k_bc[0].slots, n);
    CHQ_CUDA(cudaGetLastError());
    ++L;
    if (B->k_bc[1].nblocks) {
      bc_batched<1><<<(unsigned)B->k_bc[1].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc[st][1], B->k_bc[1].slots, n);
      CHQ_CUDA(cudaGetLastError());
      ++L;
    }
    if (B->k_bc[2].nblocks) {
      bc_batched<2><<<(unsigned)B->k_bc[2].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc[st][2], B->k_bc[2].slots, n);
      CHQ_CUDA(cudaGetLastError());
      ++L;
    }
    c2p_batched<P><<<(unsigned)B->k_c2p.nblocks, b2, 0, s>>>((const C2pArgs<P> *)B->a_c2p[st], B->k_c2p.slots, n);
    CHQ_CUDA(cudaGetLastError());
    ++L;
    if (st == B->nstage - 1 && ((B->diff && !B->cool) || B->sts)) {
      rho_min_batched<P><<<(unsigned)B->k_rho.nblocks, b2, 0, s>>>((const RhoMinArgs<P> *)B->a_rho, B->k_rho.slots, n);
      CHQ_CUDA(cudaGetLastError());
      ++L;
    }
  }
  if (B->sts) {
    const int rc = batch_sts<P>(B, s, L);
    if (rc) return rc;
  }
  if (B->cool) {
    // operator-split cooling of u0 after the step (src/main.cpp:272-290)
    c2p_batched<P><<<(unsigned)B->k_c2p.nblocks, b2, 0, s>>>((const C2pArgs<P> *)B->a_c2p_split[0], B->k_c2p.slots, n);
    CHQ_CUDA(cudaGetLastError());
    cooling_batched<P><<<(unsigned)B->k_cool.nblocks, b2, 0, s>>>((const CoolArgs<P> *)B->a_cool, B->k_cool.slots, n);
    CHQ_CUDA(cudaGetLastError());
    L += 2;
    for (int q = 0; q < 3; ++q) {
      if (!B->k_bc[q].nblocks) continue;
      if (q == 0) bc_batched<0><<<(unsigned)B->k_bc[0].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc0[0], B->k_bc[0].slots, n);
      if (q == 1) bc_batched<1><<<(unsigned)B->k_bc[1].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc0[1], B->k_bc[1].slots, n);
      if (q == 2) bc_batched<2><<<(unsigned)B->k_bc[2].nblocks, 256, 0, s>>>((const BcArgs *)B->a_bc0[2], B->k_bc[2].slots, n);
      CHQ_CUDA(cudaGetLastError());
      ++L;
    }
  }
  if (B->cool || B->sts) {
    c2p_batched<P><<<(unsigned)B->k_c2p.nblocks, b2, 0, s>>>((const C2pArgs<P> *)B->a_c2p_split[1], B->k_c2p.slots, n);
    CHQ_CUDA(cudaGetLastError());
    ++L;
    if (B->diff) {
      rho_min_batched<P><<<(unsigned)B->k_rho.nblocks, b2, 0, s>>>((const RhoMinArgs<P> *)B->a_rho, B->k_rho.slots, n);
      CHQ_CUDA(cudaGetLastError());
      ++L;
    }
  }
  ctl_end_batched<<<(n + 127) / 128, 128, 0, s>>>(B->ctls, n);
  CHQ_CUDA(cudaGetLastError());
  ++L;
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

void batch_free(chq_batch *B) {
  if (B->stream) cudaStreamSynchronize(B->stream);
  for (chq_mesh *m : B->jobs)
    if (m && B->done_evt && m->batch_evt == B->done_evt) m->batch_evt = nullptr;
  if (B->done_evt) cudaEventDestroy(B->done_evt);
  B->done_evt = nullptr;
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  if (B->dev) cudaFreeAsync(B->dev, cudaStreamLegacy);   // the batch's stream has drained
  if (B->sts_skip) cudaFree(B->sts_skip);
  if (B->sts_dyn) cudaFree(B->sts_dyn);
  B->sts_skip = nullptr;
  B->sts_dyn = nullptr;
  B->sts_dyn_bytes = 0;
  if (B->stream) cudaStreamDestroy(B->stream);
  B->exec = nullptr;
  B->graph = nullptr;
  B->dev = nullptr;
  B->stream = nullptr;
}

}  // namespace

// =======================================================================================
extern "C" {

const char *chq_last_error(void) { return g_err.c_str(); }

void chq_config_defaults(chq_config *c) {
  std::memset(c, 0, sizeof(*c));
  c->nx1 = 64; c->nx2 = 1; c->nx3 = 1;
  c->nghost = 0;
  c->x1min = 0; c->x1max = 1; c->x2min = 0; c->x2max = 1; c->x3min = 0; c->x3max = 1;
  c->recon = CHQ_RECON_PPM;
  c->rsolver = CHQ_RS_HLLD;
  c->integrator = 3;
  c->bc1 = c->bc2 = c->bc3 = CHQ_BC_PERIODIC;
  c->gamma = 5.0 / 3.0;
  c->dfloor = 1.0e-10;
  c->pfloor = 1.0e-12;
  c->cfl = 0.3;
  c->de_eta = 1.0e-3;
  c->lhlld_phi = -1.0;
  c->flatten = 1;
  c->fofc = 1;
  c->precision = CHQ_FP64;
  c->tlim = 1.0;
  c->nlim = -1;
  c->cool_alpha = 1.0;
}

}  // extern "C"

namespace {
// The driver's tensor-map encoder, looked up once through the runtime (no -lcuda link).
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  if (!tried) {
    tried = true;
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor maps of the FP64 y/z TMA staging over this mesh's own w (6 components) and bcc (3):
// 4-D (i over the row pitch, j, k, component), box = one 32-cell row segment of one component.
// The base addresses are 256-byte aligned, strides are multiples of 256 bytes and every box
// starts at i = 32 * chunk (256 bytes), which the bulk tensor copy requires (16 bytes).
bool encode_yz_maps(chq_mesh *m) {
  const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
  if (!enc) return false;
  const Geom &g = m->g;
  const cuuint64_t stride[3] = {(cuuint64_t)g.sj * 8, (cuuint64_t)g.sk * 8, (cuuint64_t)g.vstride * 8};
  const cuuint32_t box[4] = {32, 1, 1, 1}, estr[4] = {1, 1, 1, 1};
  const cuuint64_t dw[4] = {(cuuint64_t)g.sj, (cuuint64_t)g.nj + 1, (cuuint64_t)g.nk + 1, 6};
  const cuuint64_t db[4] = {(cuuint64_t)g.sj, (cuuint64_t)g.nj + 1, (cuuint64_t)g.nk + 1, 3};
  CUresult r = enc(&m->tmaps.w, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, m->w, dw, stride, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r == CUDA_SUCCESS)
    r = enc(&m->tmaps.b, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, m->bcc, db, stride, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

// the TMA staging variant exists for FP64 streaming PPM (no characteristic projection)
bool yz_tma_applies(const chq_mesh *m) {
  return m->tma_ok && !m->mixed && m->cfg.recon == R_PPM && !m->cfg.characteristic;
}

namespace {
// A whole mesh (nslab = 1) or z slab `rank` of `nslab` equal slabs of the mesh cfg describes:
// the slab holds nx3 / nslab active planes, keeps the whole mesh's x3 extent, cell width and
// coordinates (Geom::koff), and marks the z sides that border another slab.
int mesh_create_impl(const chq_config *cfg, int nslab, int rank, chq_mesh **out) {
  if (!cfg || !out) return fail(CHQ_ERR_ARG, "null argument");
  *out = nullptr;
  chq_config cl = *cfg;
  if (nslab > 1) {
    if (cfg->nx3 < 2 || cfg->nx3 % nslab != 0) return fail(CHQ_ERR_ARG, "z slabs: nx3 must be a multiple of the slab count");
    cl.nx3 = cfg->nx3 / nslab;
  }
  const chq_config &c = cl;
  if (c.nx1 < 1 || c.nx2 < 1 || c.nx3 < 1) return fail(CHQ_ERR_ARG, "nx must be >= 1");
  if (c.nx2 == 1 && c.nx3 > 1) return fail(CHQ_ERR_ARG, "nx3 > 1 requires nx2 > 1");
  if (c.recon < 0 || c.recon > 4) return fail(CHQ_ERR_ARG, "unknown reconstruction");
  if (c.rsolver < 0 || c.rsolver > 2) return fail(CHQ_ERR_ARG, "unknown Riemann solver");
  if (c.integrator < 1 || c.integrator > 4) return fail(CHQ_ERR_ARG, "unknown integrator");
  if (c.precision != CHQ_FP64 && c.precision != CHQ_MIXED) return fail(CHQ_ERR_ARG, "unknown precision");
  const int bcs[3] = {c.bc1, c.bc2, c.bc3};
  for (int q = 0; q < 3; ++q)
    if (bcs[q] < 0 || bcs[q] > 2) return fail(CHQ_ERR_ARG, "unknown boundary condition");
  const bool wide = (c.recon == CHQ_RECON_PPM || c.recon == CHQ_RECON_PPMX || c.recon == CHQ_RECON_WENOZ);
  const int ng_min = wide ? 3 : 2;
  const int ng = (c.nghost > 0) ? c.nghost : ng_min;
  if (ng < ng_min) return fail(CHQ_ERR_ARG, "nghost too small for the reconstruction method");
  if (c.nu < 0 || c.kappa < 0 || c.eta < 0) return fail(CHQ_ERR_ARG, "diffusion coefficients must be >= 0");
  if (nslab > 1) {
    if (c.nx3 < ng) return fail(CHQ_ERR_ARG, "z slabs: each slab needs at least nghost planes");
    if (c.sts || c.cooling) return fail(CHQ_ERR_ARG, "z slabs: RKL2 super-time-stepping and cooling are not supported");
  }

  chq_mesh *m = new chq_mesh;
  cudaGetDevice(&m->device);
  m->cfg = c;
  m->cfg.nghost = ng;
  Geom &g = m->g;
  g.nx1 = c.nx1; g.nx2 = c.nx2; g.nx3 = c.nx3; g.ng = ng;
  g.ni = c.nx1 + 2 * ng;
  g.nj = (c.nx2 > 1) ? c.nx2 + 2 * ng : 1;
  g.nk = (c.nx3 > 1) ? c.nx3 + 2 * ng : 1;
  g.is = ng; g.ie = ng + c.nx1 - 1;
  g.js = (c.nx2 > 1) ? ng : 0; g.je = (c.nx2 > 1) ? ng + c.nx2 - 1 : 0;
  g.ks = (c.nx3 > 1) ? ng : 0; g.ke = (c.nx3 > 1) ? ng + c.nx3 - 1 : 0;
  g.two_d = (c.nx2 > 1);
  g.three_d = (c.nx3 > 1);
  g.x1min = c.x1min; g.x2min = c.x2min; g.x3min = c.x3min;
  g.x1max = c.x1max; g.x2max = c.x2max; g.x3max = c.x3max;
  g.dx1 = (c.x1max - c.x1min) / c.nx1;
  g.dx2 = (c.x2max - c.x2min) / c.nx2;
  g.dx3 = (c.x3max - c.x3min) / c.nx3;
  g.koff = 0;
  if (nslab > 1) {
    // the whole mesh's cell width and the global index of this slab's first plane
    g.dx3 = (c.x3max - c.x3min) / cfg->nx3;
    g.koff = rank * c.nx3;
    m->slab_rank = rank;
    m->slab_count = nslab;
    m->zpeer[0] = (rank > 0 || c.bc3 == CHQ_BC_PERIODIC) ? 1 : 0;
    m->zpeer[1] = (rank < nslab - 1 || c.bc3 == CHQ_BC_PERIODIC) ? 1 : 0;
    m->fofc_ext[0] = (rank > 0) ? 1 : 0;
    m->fofc_ext[1] = (rank < nslab - 1) ? 1 : 0;
  }
  g.sj = (long)align_up((size_t)g.ni + 1, 32);
  g.sk = (long)(g.nj + 1) * g.sj;
  g.vstride = (long)align_up((size_t)(g.nk + 1) * g.sk, 64);
  // kernels index within one component with 32-bit offsets (any mesh that fits in HBM does)
  if (g.vstride >= (1L << 31) - 64) {
    delete m;
    return fail(CHQ_ERR_ARG, "mesh too large: one component exceeds 2^31 elements");
  }
  g.nelem = g.vstride;
  m->eos = EOSp{c.gamma, c.gamma - 1.0, c.dfloor, c.pfloor, c.de_eta, c.dual_energy};
  m->nstage = c.integrator;
  m->mixed = (c.precision == CHQ_MIXED);
  m->psize = m->mixed ? sizeof(float) : sizeof(double);

  // flux face ranges (src/physics.hpp:85-88) and active face ranges (src/positivity.hpp:32-33)
  for (int d = 0; d < 3; ++d) {
    int il = g.is, iu = g.ie, jl = g.js, ju = g.je, kl = g.ks, ku = g.ke;
    if (d == 0) iu = g.ie + 1; else if (g.nx1 > 1) { il = g.is - 1; iu = g.ie + 1; }
    if (d == 1) ju = g.je + 1; else if (g.two_d) { jl = g.js - 1; ju = g.je + 1; }
    if (d == 2) ku = g.ke + 1; else if (g.three_d) { kl = g.ks - 1; ku = g.ke + 1; }
    m->lo[d][0] = kl; m->lo[d][1] = jl; m->lo[d][2] = il;
    m->hi[d][0] = ku; m->hi[d][1] = ju; m->hi[d][2] = iu;
    m->act_lo[d][0] = g.ks; m->act_lo[d][1] = g.js; m->act_lo[d][2] = g.is;
    m->act_hi[d][0] = (d == 2) ? g.ke + 1 : g.ke;
    m->act_hi[d][1] = (d == 1) ? g.je + 1 : g.je;
    m->act_hi[d][2] = (d == 0) ? g.ie + 1 : g.ie;
  }
  m->active[0] = 1;
  m->active[1] = g.two_d;
  m->active[2] = g.three_d;
  // default march length: the longest of 16, 8, 4 that still gives the y/z sweeps a full
  // device of threads (148 SMs x 1024), so that small meshes are not one long serial march
  // per thread (chq_autotune measures instead)
  {
    const long lanes = (long)((g.ni + 1 + 31) / 32) * 32;
    m->seglen = 4;
    for (int L : {16, 8}) {
      long threads = 0;
      if (g.two_d) threads += lanes * (m->hi[1][0] - m->lo[1][0] + 1) * ((m->hi[1][1] - m->lo[1][1] + 1 + L - 1) / L);
      if (g.three_d) threads += lanes * (m->hi[2][1] - m->lo[2][1] + 1) * ((m->hi[2][0] - m->lo[2][0] + 1 + L - 1) / L);
      if (threads >= 148L * 1024) {
        m->seglen = L;
        break;
      }
    }
  }

  // one slab: doubles (u0, u1: 6 each; 6 face fields), P fields (w 6, bcc 3, ecc 3,
  // fluxes 18, face EMFs 6, edge EMFs 3), the int flag array, control block and scratch
  const size_t nel = (size_t)g.vstride;
  const size_t dbytes = nel * sizeof(double), pbytes = nel * m->psize, ibytes = align_up(nel * sizeof(int), 256);
  m->hst_blocks = kHstBlocks;
  const size_t ctl_bytes = align_up(sizeof(StepCtl), 256);
  m->slab_bytes = slab_size(nel, m->psize, c.sts != 0);
  cudaError_t e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = pool_alloc(reinterpret_cast<void **>(&m->slab), m->slab_bytes, m->stream);
  if (e != cudaSuccess) {
    if (m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return fail(CHQ_ERR_NOMEM, std::string("device allocation of the mesh failed: ") + cudaGetErrorString(e));
  }
  char *p = m->slab;
  m->u[0] = (double *)p; p += dbytes * 6;
  m->u[1] = (double *)p; p += dbytes * 6;
  for (int b = 0; b < 2; ++b)
    for (int d = 0; d < 3; ++d) { m->bf[b][d] = (double *)p; p += dbytes; }
  m->w = p; p += pbytes * 6;
  m->bcc = p; p += pbytes * 3;
  m->ecc = p; p += pbytes * 3;
  for (int d = 0; d < 3; ++d) { m->flx[d] = p; p += pbytes * 6; }
  for (int d = 0; d < 3; ++d) { m->et2[d] = p; p += pbytes; m->et1[d] = p; p += pbytes; }
  for (int d = 0; d < 3; ++d) { m->e[d] = p; p += pbytes; }
  m->flag = (int *)p; p += ibytes;
  m->bad_list = (int *)p; p += align_up(kBadCap * sizeof(int), 256);
  m->bad_cap = (int)kBadCap;
  if (const char *cap = std::getenv("CHQ_FOFC_LIST_CAP")) m->bad_cap = std::max(0, std::min(std::atoi(cap), (int)kBadCap));
  // a slab's FOFC repair also reads the flags of the neighbouring slabs' boundary planes,
  // which are not in its own cell list: slabs repair by scanning every face
  if (nslab > 1) m->bad_cap = 0;
  m->ctl = (StepCtl *)p; p += ctl_bytes;
  m->hst_part = (double *)p;
  m->hst_out = m->hst_part + (size_t)m->hst_blocks * 10;
  p += align_up((size_t)(kHstBlocks * 10 + 16) * sizeof(double), 256);
  if (c.sts) {
    for (int q = 0; q < 3; ++q) { m->sy[q] = (double *)p; p += dbytes * 6; }
    m->sm0 = (double *)p; p += dbytes * 6;
    m->smj = (double *)p; p += dbytes * 6;
    for (int q = 0; q < 3; ++q)
      for (int d = 0; d < 3; ++d) { m->sb[q][d] = (double *)p; p += dbytes; }
    for (int d = 0; d < 3; ++d) { m->smb0[d] = (double *)p; p += dbytes; }
    for (int d = 0; d < 3; ++d) { m->smbj[d] = (double *)p; p += dbytes; }
  }
  m->diff = (c.nu > 0 || c.kappa > 0 || c.eta > 0);
  e = cudaMemsetAsync(m->slab, 0, m->slab_bytes, m->stream);
  if (e == cudaSuccess) {
    StepCtl h{};
    h.tlim = c.tlim;
    h.nlim = c.nlim;
    h.diff_on = (c.nu > 0 || c.kappa > 0 || c.eta > 0) ? 1 : 0;
    h.sts = c.sts ? 1 : 0;
    h.ndim = 1 + g.two_d + g.three_d;
    h.nu = c.nu;
    h.eta = c.eta;
    h.kappa = c.kappa;
    h.gm1 = c.gamma - 1.0;
    h.dxmin = g.dx1;
    if (g.two_d) h.dxmin = std::fmin(h.dxmin, g.dx2);
    if (g.three_d) h.dxmin = std::fmin(h.dxmin, g.dx3);
    h.rho_bits = 0x7ff0000000000000ULL;
    h.cfl = c.cfl;
    h.nstage = m->nstage;
    h.mdt_bits = 0x7ff0000000000000ULL;
    for (int s = 1; s <= m->nstage; ++s) {
      int cur, o;
      stage_table(m->nstage, s, h.g0[s - 1], h.g1[s - 1], h.beta[s - 1], cur, o);
    }
    e = cudaMemcpyAsync(m->ctl, &h, sizeof(h), cudaMemcpyHostToDevice, m->stream);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) {
    chq_mesh_destroy(m);
    return cuda_fail(e, "mesh initialisation");
  }
  if (!m->mixed && g.two_d) m->tma_ok = encode_yz_maps(m);
  *out = m;
  return CHQ_OK;
}
}  // namespace

extern "C" {

int chq_mesh_create(const chq_config *cfg, chq_mesh **out) { return mesh_create_impl(cfg, 1, 0, out); }

int chq_slab_create(const chq_config *cfg, int nslab, int rank, chq_mesh **out) {
  if (nslab < 1 || rank < 0 || rank >= nslab) return fail(CHQ_ERR_ARG, "z slabs: rank out of range");
  return mesh_create_impl(cfg, nslab, rank, out);
}

int chq_mesh_destroy(chq_mesh *m) {
  if (!m) return CHQ_OK;
  if (m->batch_evt) cudaEventSynchronize(m->batch_evt);
  if (m->stream) cudaStreamSynchronize(m->stream);
  // (the copy lanes are shared by the device's meshes and stay; wait for this mesh's copies)
  if (m->up_stream) cudaStreamSynchronize(m->up_stream);
  if (m->unpack_stream) cudaStreamSynchronize(m->unpack_stream);
  if (m->down_stream) cudaStreamSynchronize(m->down_stream);
  for (int q = 0; q < 4; ++q) {
    if (m->stage_copied[q]) cudaEventDestroy(m->stage_copied[q]);
    if (m->stage_unpacked[q]) cudaEventDestroy(m->stage_unpacked[q]);
  }
  for (cudaEvent_t e : {m->up_ready, m->prev_done, m->hj_evt[0], m->hj_evt[1]})
    if (e) cudaEventDestroy(e);
  for (void *p : m->hj_clk)
    if (p) cudaFreeHost(p);
  if (m->snap_stream) {
    cudaStreamSynchronize(m->snap_stream);
    cudaStreamDestroy(m->snap_stream);
  }
  if (m->snap_taken) cudaEventDestroy(m->snap_taken);
  if (m->snap_landed) cudaEventDestroy(m->snap_landed);
  if (m->snap) cudaFree(m->snap);
  if (m->stage_buf) cudaFree(m->stage_buf);
  if (m->hrec) cudaFree(m->hrec);
  if (m->cyc_exec) cudaGraphExecDestroy(m->cyc_exec);
  if (m->cyc_graph) cudaGraphDestroy(m->cyc_graph);
  for (auto &p : m->pending) { m->pool.push_back(p.b); m->pool.push_back(p.e); }
  for (cudaEvent_t e : m->pool) cudaEventDestroy(e);
  for (cudaEvent_t e : m->slots) if (e) cudaEventDestroy(e);
  // every stream that used the slab has drained (above): return it to the pool in the mesh
  // stream's order, without waiting for the rest of the device
  if (m->slab) cudaFreeAsync(m->slab, m->stream);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
  return CHQ_OK;
}

int chq_mesh_dims(const chq_mesh *m, int dims[10]) {
  if (!m || !dims) return fail(CHQ_ERR_ARG, "null argument");
  const Geom &g = m->g;
  const int v[10] = {g.nx1, g.nx2, g.nx3, g.ng, g.ni, g.nj, g.nk, m->nstage, g.two_d, g.three_d};
  std::memcpy(dims, v, sizeof(v));
  return CHQ_OK;
}

long long chq_mesh_bytes(const chq_mesh *m) { return m ? (long long)m->slab_bytes : 0; }

long long chq_config_bytes(const chq_config *c) {
  if (!c || c->nx1 < 1 || c->nx2 < 1 || c->nx3 < 1) return -1;
  const bool wide = (c->recon == CHQ_RECON_PPM || c->recon == CHQ_RECON_PPMX || c->recon == CHQ_RECON_WENOZ);
  const int ng = (c->nghost > 0) ? c->nghost : (wide ? 3 : 2);
  const long ni = c->nx1 + 2 * ng, nj = (c->nx2 > 1) ? c->nx2 + 2 * ng : 1, nk = (c->nx3 > 1) ? c->nx3 + 2 * ng : 1;
  const size_t sj = align_up((size_t)ni + 1, 32);
  const size_t nel = align_up((size_t)(nk + 1) * (nj + 1) * sj, 64);
  return (long long)slab_size(nel, c->precision == CHQ_MIXED ? sizeof(float) : sizeof(double), c->sts != 0);
}

int chq_init_problem(chq_mesh *m, int problem, const double *prm, int nprm, void *stream) {
  if (!m || (nprm > 0 && !prm) || nprm < 0 || nprm > 12) return fail(CHQ_ERR_ARG, "bad argument");
  static const int need[3] = {1, 7, 7};
  if (problem < 0 || problem > 2) return fail(CHQ_ERR_ARG, "unknown problem generator");
  if (nprm < need[problem]) return fail(CHQ_ERR_ARG, "too few problem parameters");
  PgenArgs a{};
  a.g = m->g;
  a.problem = problem;
  a.gamma = m->cfg.gamma;
  for (int q = 0; q < nprm; ++q) a.prm[q] = prm[q];
  if (problem == PG_BLAST) {
    // the same operations as the host generator (chasqui_b200/ics.py blast_noise)
    const double ang = prm[4] * M_PI / 180.0, b0 = prm[3];
    double bx = b0 * std::cos(ang), by = b0 * std::sin(ang);
    if (std::fabs(bx) < 1e-14 * b0) bx = 0.0;
    if (std::fabs(by) < 1e-14 * b0) by = 0.0;
    a.bxy[0] = bx;
    a.bxy[1] = by;
  }
  if (problem == PG_CPAW) {
    // wavevector 2 pi (m1/L1, m2/L2, m3/L3) = 2 pi |mv| e1, with the host generator's
    // operation order (chasqui_b200/ics.py cpaw_oblique: e1 = m/|m|, k = 2 pi |m|)
    const double L[3] = {m->g.x1max - m->g.x1min, m->g.x2max - m->g.x2min, m->g.x3max - m->g.x3min};
    double mv[3];
    for (int q = 0; q < 3; ++q) mv[q] = prm[q] / L[q];
    const double nrm = std::sqrt(mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2]);
    if (!(nrm > 0.0)) return fail(CHQ_ERR_ARG, "cpaw: zero wavevector");
    for (int q = 0; q < 3; ++q) a.e1[q] = mv[q] / nrm;
    // e2 perpendicular to e1 (prefer the x-y plane), e3 = e1 x e2
    const double t[3] = {std::fabs(a.e1[2]) < 0.9 ? 0.0 : 1.0, 0.0, std::fabs(a.e1[2]) < 0.9 ? 1.0 : 0.0};
    double e2[3] = {t[1] * a.e1[2] - t[2] * a.e1[1], t[2] * a.e1[0] - t[0] * a.e1[2], t[0] * a.e1[1] - t[1] * a.e1[0]};
    const double n2 = std::sqrt(e2[0] * e2[0] + e2[1] * e2[1] + e2[2] * e2[2]);
    for (int q = 0; q < 3; ++q) a.e2[q] = e2[q] / n2;
    a.e3[0] = a.e1[1] * a.e2[2] - a.e1[2] * a.e2[1];
    a.e3[1] = a.e1[2] * a.e2[0] - a.e1[0] * a.e2[2];
    a.e3[2] = a.e1[0] * a.e2[1] - a.e1[1] * a.e2[0];
    a.kmag = 2.0 * M_PI * nrm;
  }
  a.u = m->u[0];
  a.b1 = m->bf[0][0];
  a.b2 = m->bf[0][1];
  a.b3 = m->bf[0][2];
  cudaStream_t s = S(m, stream);
  const Geom &g = m->g;
  const long nf = (long)(g.nk + 1) * (g.nj + 1) * (g.ni + 1), nc = (long)g.nk * g.nj * g.ni;
  pgen_faces_kernel<<<(unsigned)((nf + 255) / 256), 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  pgen_cells_kernel<<<(unsigned)((nc + 255) / 256), 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  m->nlaunch += 2;
  return CHQ_OK;
}

long chq_array_size(const chq_mesh *m, const char *name) {
  FieldRef f;
  if (m && name && !std::strcmp(name, "vtk")) return 4L * m->g.nx1 * m->g.nx2 * m->g.nx3;   // 8 floats per cell
  if (!m || !name || !field_by_name(const_cast<chq_mesh *>(m), name, f)) return -1;
  return field_size(m, f);
}

int chq_upload(chq_mesh *m, const char *name, const double *host, long n, void *stream) {
  if (!m || !name || !host) return fail(CHQ_ERR_ARG, "null argument");
  return transfer(m, name, const_cast<double *>(host), n, true, S(m, stream));
}

int chq_download(chq_mesh *m, const char *name, double *host, long n, void *stream) {
  if (!m || !name || !host) return fail(CHQ_ERR_ARG, "null argument");
  return transfer(m, name, host, n, false, S(m, stream));
}

int chq_snapshot_wait(chq_mesh *m) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  if (!m->snap_pending) return CHQ_OK;
  m->snap_pending = false;
  CHQ_CUDA(cudaEventSynchronize(m->snap_landed));
  for (auto &it : m->snap_items) {
    if (it.tmp.empty()) continue;
    for (long q = 0; q < it.n; ++q)
      it.host[q] = it.isint ? (double)reinterpret_cast<int *>(it.tmp.data())[q]
                            : (double)reinterpret_cast<float *>(it.tmp.data())[q];
  }
  m->snap_items.clear();
  return CHQ_OK;
}

namespace {
// Packs the named fields into the snapshot area in the host layout (a device-side copy
// behind the work queued on the mesh stream, once the previous snapshot's download has left
// the area), then downloads each with one linear copy on `down` (the snapshot stream when
// null); `items` describes the copies.
int snapshot_enqueue(chq_mesh *m, int nfields, const char *const *names, double *const *host, const long *n,
                     std::vector<chq_mesh::SnapItem> &items, cudaStream_t down) {
  const Geom &g = m->g;
  std::vector<FieldRef> fr(nfields);
  size_t need = 0;
  std::vector<char> vtk(nfields, 0);
  const long ncell = (long)g.nx1 * g.nx2 * g.nx3;
  for (int q = 0; q < nfields; ++q) {
    if (names[q] && host[q] && !std::strcmp(names[q], "vtk")) {
      if (n[q] != 4 * ncell) return fail(CHQ_ERR_ARG, "size mismatch for field vtk");
      vtk[q] = 1;
      need += align_up((size_t)ncell * 32, 256);
      continue;
    }
    if (!names[q] || !host[q] || !field_by_name(m, names[q], fr[q]))
      return fail(CHQ_ERR_ARG, std::string("unknown field: ") + (names[q] ? names[q] : "(null)"));
    if (field_size(m, fr[q]) != n[q]) return fail(CHQ_ERR_ARG, std::string("size mismatch for field ") + names[q]);
    const FieldRef &f = fr[q];
    const size_t nx = f.face ? g.ni + 1 : g.ni, ny = f.face ? g.nj + 1 : g.nj, nz = f.face ? g.nk + 1 : g.nk;
    need += align_up((size_t)f.ncomp * nx * ny * nz * field_esize(m, f), 256);
  }
  if (!m->snap_stream) {
    CHQ_CUDA(cudaStreamCreateWithFlags(&m->snap_stream, cudaStreamNonBlocking));
    CHQ_CUDA(cudaEventCreateWithFlags(&m->snap_taken, cudaEventDisableTiming));
    CHQ_CUDA(cudaEventCreateWithFlags(&m->snap_landed, cudaEventDisableTiming));
  }
  if (need > m->snap_bytes) {
    // (cudaFree waits for the device, so no download still reads the old area)
    if (m->snap) CHQ_CUDA(cudaFree(m->snap));
    m->snap = nullptr;
    m->snap_bytes = 0;
    const cudaError_t e = cudaMalloc(&m->snap, need);
    if (e != cudaSuccess) return fail(CHQ_ERR_NOMEM, std::string("snapshot area: ") + cudaGetErrorString(e));
    m->snap_bytes = need;
  }
  cudaStream_t s = S(m, nullptr);
  CHQ_CUDA(cudaStreamWaitEvent(s, m->snap_landed, 0));   // the previous download has left the area
  char *p = m->snap;
  items.clear();
  for (int q = 0; q < nfields; ++q) {
    if (vtk[q]) {
      const unsigned blocks = (unsigned)std::max(1L, std::min<long>((8 * ncell + 255) / 256, 148L * 16));
      m->nlaunch += 1;
      if (m->mixed)
        vtk_cells_kernel<float><<<blocks, 256, 0, s>>>(g, as<float>(m->w), as<float>(m->bcc), reinterpret_cast<unsigned *>(p));
      else
        vtk_cells_kernel<double><<<blocks, 256, 0, s>>>(g, as<double>(m->w), as<double>(m->bcc), reinterpret_cast<unsigned *>(p));
      CHQ_CUDA(cudaGetLastError());
      items.push_back(chq_mesh::SnapItem{host[q], n[q], 1, 0, sizeof(double), 0, p, {}});
      p += align_up((size_t)ncell * 32, 256);
      continue;
    }
    // packed into the snapshot area in the host layout
    const FieldRef &f = fr[q];
    const int nx = f.face ? g.ni + 1 : g.ni, ny = f.face ? g.nj + 1 : g.nj, nz = f.face ? g.nk + 1 : g.nk;
    const size_t es = field_esize(m, f), bytes = (size_t)f.ncomp * nx * ny * nz * es;
    const long tot = (long)f.ncomp * nx * ny * nz;
    const unsigned blocks = (unsigned)std::max(1L, std::min<long>((tot + 255) / 256, 148L * 16));
    m->nlaunch += 1;
    if (es == 8)
      pack_planes_kernel<unsigned long long><<<blocks, 256, 0, s>>>(static_cast<const unsigned long long *>(f.base),
          reinterpret_cast<unsigned long long *>(p), f.ncomp, nx, ny, nz, g.sj, g.sk, g.vstride);
    else
      pack_planes_kernel<unsigned><<<blocks, 256, 0, s>>>(static_cast<const unsigned *>(f.base),
          reinterpret_cast<unsigned *>(p), f.ncomp, nx, ny, nz, g.sj, g.sk, g.vstride);
    CHQ_CUDA(cudaGetLastError());
    chq_mesh::SnapItem it{host[q], n[q], f.ncomp, f.face, es, f.isint, p, {}};
    if (es != sizeof(double) || f.isint) it.tmp.resize((size_t)n[q] * es);
    items.push_back(std::move(it));
    p += align_up(bytes, 256);
  }
  if (!down) down = m->snap_stream;
  CHQ_CUDA(cudaEventRecord(m->snap_taken, s));
  CHQ_CUDA(cudaStreamWaitEvent(down, m->snap_taken, 0));
  for (auto &it : items) {
    void *hbase = it.tmp.empty() ? (void *)it.host : (void *)it.tmp.data();
    CHQ_CUDA(cudaMemcpyAsync(hbase, it.copy, (size_t)it.n * it.es, cudaMemcpyDeviceToHost, down));
  }
  CHQ_CUDA(cudaEventRecord(m->snap_landed, down));
  return CHQ_OK;
}
}  // namespace

int chq_snapshot(chq_mesh *m, int nfields, const char *const *names, double *const *host, const long *n) {
  if (!m || nfields < 1 || !names || !host || !n) return fail(CHQ_ERR_ARG, "bad argument");
  int rc = chq_snapshot_wait(m);
  if (rc) return rc;
  if ((rc = snapshot_enqueue(m, nfields, names, host, n, m->snap_items, nullptr))) return rc;
  m->snap_pending = true;
  return CHQ_OK;
}

int chq_fluxes(chq_mesh *m, int dir, int cur, void *stream) {
  if (!m || dir < 0 || dir > 2 || (cur != 0 && cur != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  if (!m->active[dir]) return fail(CHQ_ERR_ARG, "direction not active in this mesh");
  return do_fluxes(m, cur, 1u << dir, nullptr, S(m, stream));
}

int chq_fluxes_all(chq_mesh *m, int cur, void *stream) {
  if (!m || (cur != 0 && cur != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  return do_fluxes(m, cur, 7u, nullptr, S(m, stream));
}

int chq_corner_emf(chq_mesh *m, void *stream) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  return DISPATCH_P(m, do_corner)(m, nullptr, nullptr, S(m, stream));
}

int chq_update(chq_mesh *m, int out, double g0, double g1, double beta_dt, void *stream) {
  if (!m || (out != 0 && out != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  return DISPATCH_P(m, do_update)(m, out, g0, g1, beta_dt, nullptr, nullptr, nullptr, S(m, stream));
}

int chq_boundaries(chq_mesh *m, int buf, void *stream) {
  if (!m || (buf != 0 && buf != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  return do_bc(m, buf, nullptr, S(m, stream));
}

int chq_cons_to_prim(chq_mesh *m, int buf, int compute_dt, double *min_dt, void *stream) {
  if (!m || (buf != 0 && buf != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  cudaStream_t s = S(m, stream);
  unsigned long long *bits = &m->ctl->mdt_bits;
  if (compute_dt) {
    reset_bits_kernel<<<1, 1, 0, s>>>(bits);
    CHQ_CUDA(cudaGetLastError());
  }
  int rc = DISPATCH_P(m, do_c2p)(m, buf, compute_dt, bits, nullptr, nullptr, s);
  if (rc) return rc;
  if (compute_dt && min_dt) {
    unsigned long long h = 0;
    CHQ_CUDA(cudaMemcpyAsync(&h, bits, sizeof(h), cudaMemcpyDeviceToHost, s));
    CHQ_CUDA(cudaStreamSynchronize(s));
    std::memcpy(min_dt, &h, sizeof(double));
  }
  return CHQ_OK;
}

int chq_fofc_flag(chq_mesh *m, int buf, int *nbad, void *stream) {
  if (!m || (buf != 0 && buf != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  cudaStream_t s = S(m, stream);
  CHQ_CUDA(cudaMemsetAsync(&m->ctl->nbad, 0, sizeof(int), s));
  int rc = do_flag(m, buf, &m->ctl->nbad, nullptr, s);
  if (rc) return rc;
  if (nbad) {
    CHQ_CUDA(cudaMemcpyAsync(nbad, &m->ctl->nbad, sizeof(int), cudaMemcpyDeviceToHost, s));
    CHQ_CUDA(cudaStreamSynchronize(s));
  }
  return CHQ_OK;
}

int chq_fofc_repair(chq_mesh *m, int dir, int cur, void *stream) {
  if (!m || dir < 0 || dir > 2 || (cur != 0 && cur != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  if (!m->active[dir]) return fail(CHQ_ERR_ARG, "direction not active in this mesh");
  return DISPATCH_P(m, do_repair)(m, cur, 1u << dir, nullptr, nullptr, S(m, stream));
}

int chq_limit_fluxes(chq_mesh *m, int dir, double beta_dt, long *count, void *stream) {
  if (!m || dir < 0 || dir > 2) return fail(CHQ_ERR_ARG, "bad argument");
  if (!m->active[dir]) return fail(CHQ_ERR_ARG, "direction not active in this mesh");
  cudaStream_t s = S(m, stream);
  long long *cnt = &m->ctl->limiter_count;
  long long before = 0, after = 0;
  CHQ_CUDA(cudaMemcpyAsync(&before, cnt, sizeof(before), cudaMemcpyDeviceToHost, s));
  int rc = DISPATCH_P(m, do_limit)(m, 1u << dir, beta_dt, nullptr, cnt, nullptr, s);
  if (rc) return rc;
  CHQ_CUDA(cudaMemcpyAsync(&after, cnt, sizeof(after), cudaMemcpyDeviceToHost, s));
  CHQ_CUDA(cudaStreamSynchronize(s));
  if (count) *count += (long)(after - before);
  return CHQ_OK;
}

int chq_stage(chq_mesh *m, int cur, int out, double g0, double g1, double beta_dt, void *stream) {
  if (!m || (cur != 0 && cur != 1) || (out != 0 && out != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  if (m->slab_count > 1) return fail(CHQ_ERR_ARG, "a z slab steps through chq_slab_stage");
  cudaStream_t s = S(m, stream);
  CHQ_CUDA(cudaMemsetAsync(&m->ctl->nbad, 0, sizeof(int), s));
  return run_stage(m, cur, out, g0, g1, beta_dt, nullptr, nullptr, s);
}

int chq_prime(chq_mesh *m, double t, void *stream) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  if (m->slab_count > 1) return fail(CHQ_ERR_ARG, "a z slab is primed through chq_slab_prime");
  cudaStream_t s = S(m, stream);
  ctl_prime_kernel<<<1, 1, 0, s>>>(m->ctl, t);
  CHQ_CUDA(cudaGetLastError());
  int rc = do_bc(m, 0, nullptr, s);
  if (rc) return rc;
  rc = DISPATCH_P(m, do_c2p)(m, 0, 1, &m->ctl->mdt_bits, m->ctl, nullptr, s);
  if (rc) return rc;
  if (m->diff && !m->cfg.sts && (rc = DISPATCH_P(m, do_rho_min)(m, nullptr, s))) return rc;
  ctl_take_dt_kernel<<<1, 1, 0, s>>>(m->ctl);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

}  // extern "C"

namespace chq {
// n cycles as individual launches (the body of chq_cycles)
int plain_cycles(chq_mesh *m, int n, cudaStream_t s) {
  const int *done = &m->ctl->done;
  const bool sts = m->cfg.sts && m->diff;
  const bool cool = m->cfg.cooling != 0;
  // operator-split pieces after the hyperbolic step (src/main.cpp:272-290): RKL2 and
  // cooling; with either, the last stage's con2prim takes no dt and a final one does
  const bool split = sts || cool;
  for (int c = 0; c < n; ++c) {
    {
      Prof p(m, PK_CTL, s);
      ctl_begin_kernel<<<1, 1, 0, s>>>(m->ctl, 0);
      m->nlaunch += 1;
      if (m->hrec) {
        hst_due_kernel<<<1, 1, 0, s>>>(m->ctl, m->hrec);
        m->nlaunch += 1;
      }
    }
    CHQ_CUDA(cudaGetLastError());
    int rc;
    for (int st = 1; st <= m->nstage; ++st) {
      double g0, g1, beta;
      int cur, out;
      stage_table(m->nstage, st, g0, g1, beta, cur, out);
      rc = run_stage(m, cur, out, g0, g1, 0.0, &m->ctl->beta_dt[st - 1], done, s);
      if (rc) return rc;
      const bool last = (st == m->nstage);
      {
        Prof p(m, PK_C2P, s);
        rc = (last && !split) ? DISPATCH_P(m, do_c2p_end)(m, done, s)
                              : DISPATCH_P(m, do_c2p)(m, out, 0, &m->ctl->mdt_bits, m->ctl, done, s);
      }
      if (rc) return rc;
      if (last && m->diff && (!split || sts)) {
        Prof p(m, PK_DIFF, s);
        if ((rc = DISPATCH_P(m, do_rho_min)(m, done, s))) return rc;
      }
    }
    if (sts) {
      // the RKL2 stage count is a host decision: read dt and the density minimum here
      StepCtl h;
      CHQ_CUDA(cudaMemcpyAsync(&h, m->ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
      CHQ_CUDA(cudaStreamSynchronize(s));
      if (h.done) break;
      double rho_min;
      std::memcpy(&rho_min, &h.rho_bits, sizeof(rho_min));
      const double dt_par = host_parabolic_dt(m, rho_min);
      int nst = 0;
      {
        Prof p(m, PK_STS, s);
        rc = DISPATCH_P(m, sts_advance)(m, h.dt, dt_par, s, nst);
        if (!rc) rc = do_bc(m, 0, nullptr, s);
      }
      if (rc) return rc;
      m->sts_stages += nst;
    }
    if (cool) {
      Prof p(m, PK_C2P, s);
      if ((rc = DISPATCH_P(m, do_c2p)(m, 0, 0, &m->ctl->mdt_bits, m->ctl, done, s))) return rc;
      if ((rc = DISPATCH_P(m, do_cooling)(m, done, s))) return rc;
      if ((rc = do_bc(m, 0, done, s))) return rc;
    }
    if (split) {
      {
        Prof p(m, PK_C2P, s);
        if ((rc = DISPATCH_P(m, do_c2p_end)(m, done, s))) return rc;
      }
      if (m->diff && !sts) {
        Prof p(m, PK_DIFF, s);
        if ((rc = DISPATCH_P(m, do_rho_min)(m, done, s))) return rc;
      }
    }
    {
      Prof p(m, PK_CTL, s);
      ctl_end_kernel<<<1, 1, 0, s>>>(m->ctl);
      m->nlaunch += 1;
      if (m->hrec) {
        hst_fold_kernel<<<(unsigned)m->hrec_nfold, 320, 0, s>>>(m->hrec);
        hst_commit_kernel<<<1, 320, 0, s>>>(m->ctl, m->hrec);
        m->nlaunch += 2;
      }
    }
    CHQ_CUDA(cudaGetLastError());
  }
  return CHQ_OK;
}

// the mesh's own stream (the server records events behind a solo job's cycles on it)
cudaStream_t mesh_stream(chq_mesh *m) { return m->stream; }

// A copy of the step control queued behind the mesh's work, so that the server learns a solo
// job's clock without synchronising the stream (which would also wait for the next chunk).
size_t clock_bytes() { return sizeof(StepCtl); }
int clock_enqueue(chq_mesh *m, void *pinned) {
  CHQ_CUDA(cudaMemcpyAsync(pinned, m->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, m->stream));
  return CHQ_OK;
}
void clock_decode(const void *pinned, double *t, int *cycle) {
  const StepCtl *c = static_cast<const StepCtl *>(pinned);
  *t = c->t;
  *cycle = c->cycle;
}

void drop_cycle_graph(chq_mesh *m) {
  if (m->cyc_exec) cudaGraphExecDestroy(m->cyc_exec);
  if (m->cyc_graph) cudaGraphDestroy(m->cyc_graph);
  m->cyc_exec = nullptr;
  m->cyc_graph = nullptr;
}
}  // namespace chq

extern "C" {

// Whole cycles. Without RKL2 (whose stage count the host decides each cycle) and without
// per-kernel profiling, cycles on the mesh's own stream replay a CUDA graph of one cycle,
// captured after a first plain cycle: a cycle is ~70 small launches, and on small meshes
// their CPU cost exceeds the device time. The launch count of a replayed cycle is the
// captured one's.
int chq_cycles(chq_mesh *m, int n, void *stream) {
  if (!m || n < 0) return fail(CHQ_ERR_ARG, "bad argument");
  if (m->slab_count > 1) return fail(CHQ_ERR_ARG, "a z slab steps through chq_slab_begin / chq_slab_stage / chq_slab_end");
  cudaStream_t s = S(m, stream);
  const bool graphable = !(m->cfg.sts && m->diff) && !m->prof && (stream == nullptr || s == m->stream);
  if (!graphable || n == 0) return plain_cycles(m, n, s);
  int done_plain = 0;
  if (!m->cyc_warm) {
    const int rc = plain_cycles(m, 1, s);
    if (rc) return rc;
    m->cyc_warm = true;
    done_plain = 1;
  }
  if (done_plain == n) return CHQ_OK;
  if (!m->cyc_exec) {
    const long long l0 = m->nlaunch;
    CHQ_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    const int rc = plain_cycles(m, 1, s);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CHQ_CUDA(e);
    m->cyc_graph = g;
    CHQ_CUDA(cudaGraphInstantiate(&m->cyc_exec, m->cyc_graph, 0));
    m->cyc_launches = m->nlaunch - l0;   // the capture itself ran nothing
    m->nlaunch = l0;
  }
  for (int c = done_plain; c < n; ++c) CHQ_CUDA(cudaGraphLaunch(m->cyc_exec, s));
  m->nlaunch += m->cyc_launches * (n - done_plain);
  return CHQ_OK;
}

long long chq_sts_stages(const chq_mesh *m) { return m ? m->sts_stages : 0; }

int chq_clock(chq_mesh *m, double *t, int *cycle, double *dt, double *min_dt) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  StepCtl h;
  cudaStream_t s = S(m, nullptr);
  CHQ_CUDA(cudaMemcpyAsync(&h, m->ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
  CHQ_CUDA(cudaStreamSynchronize(s));
  if (t) *t = h.t;
  if (cycle) *cycle = h.cycle;
  if (dt) *dt = h.dt;
  if (min_dt) *min_dt = h.min_dt;
  return CHQ_OK;
}

int chq_counters(chq_mesh *m, long long *fofc, long long *limiter) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  StepCtl h;
  cudaStream_t s = S(m, nullptr);
  CHQ_CUDA(cudaMemcpyAsync(&h, m->ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
  CHQ_CUDA(cudaStreamSynchronize(s));
  if (fofc) *fofc = h.fofc_count + h.nbad;
  if (limiter) *limiter = h.limiter_count;
  return CHQ_OK;
}

int chq_history(chq_mesh *m, double out[10], void *stream) {
  if (!m || !out) return fail(CHQ_ERR_ARG, "null argument");
  cudaStream_t s = S(m, stream);
  const Geom &g = m->g;
  if (m->mixed)
    hst_partial_kernel<float><<<m->hst_blocks, 256, 0, s>>>(g, m->u[0], as<float>(m->w), as<float>(m->bcc), m->bf[0][0],
                                                            m->bf[0][1], m->bf[0][2], 1.0 / g.dx1, 1.0 / g.dx2,
                                                            1.0 / g.dx3, m->hst_part);
  else
    hst_partial_kernel<double><<<m->hst_blocks, 256, 0, s>>>(g, m->u[0], as<double>(m->w), as<double>(m->bcc),
                                                             m->bf[0][0], m->bf[0][1], m->bf[0][2], 1.0 / g.dx1,
                                                             1.0 / g.dx2, 1.0 / g.dx3, m->hst_part);
  CHQ_CUDA(cudaGetLastError());
  hst_final_kernel<<<1, 32, 0, s>>>(m->hst_part, m->hst_blocks, m->hst_out);
  CHQ_CUDA(cudaGetLastError());
  double h[10];
  CHQ_CUDA(cudaMemcpyAsync(h, m->hst_out, sizeof(h), cudaMemcpyDeviceToHost, s));
  CHQ_CUDA(cudaStreamSynchronize(s));
  const double vol = g.dx1 * (g.two_d ? g.dx2 : 1.0) * (g.three_d ? g.dx3 : 1.0);
  const double ncell = (double)g.nx1 * g.nx2 * g.nx3;
  for (int q = 0; q < 8; ++q) out[q] = h[q] * vol;
  out[8] = h[8];
  out[9] = h[9] / ncell;
  return CHQ_OK;
}

static_assert(sizeof(HstRec) <= 256, "HstRec header exceeds its slot");

int chq_history_record(chq_mesh *m, double dt_hst, double next, double eps, int capacity) {
  if (!m || capacity < 0) return fail(CHQ_ERR_ARG, "bad argument");
  if (capacity > 0 && !(dt_hst > 0)) return fail(CHQ_ERR_ARG, "history recording needs dt_hst > 0");
  cudaStream_t s = S(m, nullptr);
  CHQ_CUDA(cudaStreamSynchronize(s));
  drop_cycle_graph(m);   // the captured cycle has the old end-of-cycle launches
  if (m->hrec) {
    CHQ_CUDA(cudaFree(m->hrec));
    m->hrec = nullptr;
    m->hrec_cap = 0;
  }
  if (capacity == 0) return CHQ_OK;
  const Geom &g = m->g;
  const Launch3 L = c2p_grid(m);
  HstRec h{};
  h.cap = capacity;
  h.next = next;
  h.dt_hst = dt_hst;
  h.eps = eps;
  h.vol = g.dx1 * (g.two_d ? g.dx2 : 1.0) * (g.three_d ? g.dx3 : 1.0);
  h.ncell = (double)g.nx1 * g.nx2 * g.nx3;
  h.idx1 = 1.0 / g.dx1;
  h.idx2 = 1.0 / g.dx2;
  h.idx3 = 1.0 / g.dx3;
  h.nblk = (long)L.grid.x * L.grid.y * L.grid.z;
  h.nfold = std::min<long>(h.nblk, kHstBlocks);
  const size_t head = 256;
  const size_t bytes = head + sizeof(double) * ((size_t)h.nblk * 10 + (size_t)h.nfold * 10 + (size_t)capacity * 12);
  char *p = nullptr;
  CHQ_CUDA(cudaMalloc(&p, bytes));
  h.part = reinterpret_cast<double *>(p + head);
  h.fold = h.part + h.nblk * 10;
  h.rows = h.fold + h.nfold * 10;
  CHQ_CUDA(cudaMemcpy(p, &h, sizeof(h), cudaMemcpyHostToDevice));
  // landed before the mesh's non-blocking stream can read it (see batch_build)
  CHQ_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
  m->hrec = reinterpret_cast<HstRec *>(p);
  m->hrec_nfold = h.nfold;
  m->hrec_cap = capacity;
  return CHQ_OK;
}

int chq_history_drain(chq_mesh *m, double *rows, int max_rows, int *n, int *lost, double *next) {
  if (!m || max_rows < 0 || (max_rows > 0 && !rows)) return fail(CHQ_ERR_ARG, "bad argument");
  if (!m->hrec) return fail(CHQ_ERR_ARG, "history recording is off (chq_history_record)");
  cudaStream_t s = S(m, nullptr);
  HstRec h;
  CHQ_CUDA(cudaMemcpyAsync(&h, m->hrec, sizeof(h), cudaMemcpyDeviceToHost, s));
  CHQ_CUDA(cudaStreamSynchronize(s));
  const int k = std::min(h.count, max_rows);
  if (k > 0) CHQ_CUDA(cudaMemcpyAsync(rows, h.rows, sizeof(double) * 12 * (size_t)k, cudaMemcpyDeviceToHost, s));
  // rows that did not fit stay in the ring, oldest first, for the next drain
  std::vector<double> rest((size_t)(h.count - k) * 12);
  if (!rest.empty()) {
    CHQ_CUDA(cudaMemcpyAsync(rest.data(), h.rows + (size_t)k * 12, sizeof(double) * rest.size(),
                             cudaMemcpyDeviceToHost, s));
    CHQ_CUDA(cudaStreamSynchronize(s));
    CHQ_CUDA(cudaMemcpyAsync(h.rows, rest.data(), sizeof(double) * rest.size(), cudaMemcpyHostToDevice, s));
  }
  const int kept[3] = {h.count - k, h.cap, 0};   // count, cap, lost
  CHQ_CUDA(cudaMemcpyAsync(&m->hrec->count, kept, sizeof(kept), cudaMemcpyHostToDevice, s));
  CHQ_CUDA(cudaStreamSynchronize(s));
  if (n) *n = k;
  if (lost) *lost = h.lost;
  if (next) *next = h.next;
  return CHQ_OK;
}

int chq_run_host(chq_mesh *m, double *u, double *b1, double *b2, double *b3, int ncycles, double t0, void *stream) {
  if (!m || !u || !b1 || !b2 || !b3 || ncycles < 0) return fail(CHQ_ERR_ARG, "bad argument");
  cudaStream_t s = S(m, stream);
  int rc;
  if ((rc = transfer(m, "u0", u, chq_array_size(m, "u0"), true, s))) return rc;
  if ((rc = transfer(m, "b1f0", b1, chq_array_size(m, "b1f0"), true, s))) return rc;
  if ((rc = transfer(m, "b2f0", b2, chq_array_size(m, "b2f0"), true, s))) return rc;
  if ((rc = transfer(m, "b3f0", b3, chq_array_size(m, "b3f0"), true, s))) return rc;
  if ((rc = chq_prime(m, t0, s))) return rc;
  if ((rc = chq_cycles(m, ncycles, s))) return rc;
  int done_cycles = 0;
  if ((rc = transfer(m, "u0", u, chq_array_size(m, "u0"), false, s))) return rc;
  if ((rc = transfer(m, "b1f0", b1, chq_array_size(m, "b1f0"), false, s))) return rc;
  if ((rc = transfer(m, "b2f0", b2, chq_array_size(m, "b2f0"), false, s))) return rc;
  if ((rc = transfer(m, "b3f0", b3, chq_array_size(m, "b3f0"), false, s))) return rc;
  if ((rc = chq_clock(m, nullptr, &done_cycles, nullptr, nullptr))) return rc;
  return done_cycles;
}

namespace {
// Host jobs of all meshes on a device take turns, in submission order, on three lanes: one
// upload stream, the SMs (a job's cycles start after the previous job's cycles ended) and
// one download stream. Jobs on several meshes then never upload, compute or download all at
// once (which leaves the SMs idle while everything uploads), and one job's copies overlap
// another's cycles. The upload stream has the highest priority: its unpack kernels get SMs
// as soon as blocks of a running cycle retire. Lanes live as long as the process.
struct CopyLanes {
  cudaStream_t up = nullptr, unpack = nullptr, down = nullptr;
  cudaEvent_t computed = nullptr;   // recorded after the last queued host job's cycles
};
std::mutex g_lanes_mu;
CopyLanes g_lanes[64];

int copy_lanes(int device, CopyLanes &out) {
  if (device < 0 || device >= 64) return fail(CHQ_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lock(g_lanes_mu);
  CopyLanes &l = g_lanes[device];
  if (!l.up) {
    int least = 0, greatest = 0;
    CHQ_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CHQ_CUDA(cudaStreamCreateWithPriority(&l.up, cudaStreamNonBlocking, greatest));
    CHQ_CUDA(cudaStreamCreateWithPriority(&l.unpack, cudaStreamNonBlocking, greatest));
    CHQ_CUDA(cudaStreamCreateWithFlags(&l.down, cudaStreamNonBlocking));
    CHQ_CUDA(cudaEventCreateWithFlags(&l.computed, cudaEventDisableTiming));
  }
  out = l;
  return CHQ_OK;
}

// page-locked (cudaHostAlloc / cudaHostRegister) host memory: copies from it are asynchronous
bool page_locked(const void *p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}
}  // namespace

int chq_run_host_async(chq_mesh *m, double *u, double *b1, double *b2, double *b3, int ncycles, double t0) {
  if (!m || !u || !b1 || !b2 || !b3 || ncycles < 0) return fail(CHQ_ERR_ARG, "bad argument");
  if (m->hj_count == 2) return fail(CHQ_ERR_STATE, "two host jobs in flight on this mesh: call chq_run_host_wait first");
  for (const double *p : {u, b1, b2, b3})
    if (!page_locked(p)) return fail(CHQ_ERR_ARG, "chq_run_host_async needs page-locked host arrays (chq_host_alloc)");
  if (!m->up_stream) {
    CopyLanes l;
    const int rc0 = copy_lanes(m->device, l);
    if (rc0) return rc0;
    m->up_stream = l.up;
    m->unpack_stream = l.unpack;
    m->down_stream = l.down;
    CHQ_CUDA(cudaEventCreateWithFlags(&m->up_ready, cudaEventDisableTiming));
    CHQ_CUDA(cudaEventCreateWithFlags(&m->prev_done, cudaEventDisableTiming));
    for (int q = 0; q < 2; ++q) {
      CHQ_CUDA(cudaEventCreateWithFlags(&m->hj_evt[q], cudaEventDisableTiming));
      CHQ_CUDA(cudaHostAlloc(&m->hj_clk[q], sizeof(StepCtl), cudaHostAllocDefault));
    }
  }
  cudaStream_t s = m->stream;
  int rc;
  double *const arr[4] = {u, b1, b2, b3};
  const char *const names[4] = {"u0", "b1f0", "b2f0", "b3f0"};
  long sizes[4];
  for (int q = 0; q < 4; ++q) sizes[q] = chq_array_size(m, names[q]);
  // the upload waits for everything queued before it on the mesh stream (the previous job's
  // cycles and its copy into the snapshot area), not for that job's download
  CHQ_CUDA(cudaEventRecord(m->prev_done, s));
  CHQ_CUDA(cudaStreamWaitEvent(m->up_stream, m->prev_done, 0));
  for (int q = 0; q < 4; ++q)
    if ((rc = transfer(m, names[q], arr[q], sizes[q], true, m->up_stream, false))) return rc;
  if ((rc = stage_fence(m, m->up_stream))) return rc;   // up_ready then covers the unpacks
  CHQ_CUDA(cudaEventRecord(m->up_ready, m->up_stream));
  CHQ_CUDA(cudaStreamWaitEvent(s, m->up_ready, 0));
  CopyLanes l;
  if ((rc = copy_lanes(m->device, l))) return rc;
  {
    // the SM lane: after the previous host job's cycles (on any mesh of the device)
    std::lock_guard<std::mutex> lock(g_lanes_mu);
    CHQ_CUDA(cudaStreamWaitEvent(s, l.computed, 0));
    if ((rc = chq_prime(m, t0, s))) return rc;
    if ((rc = chq_cycles(m, ncycles, s))) return rc;
    CHQ_CUDA(cudaEventRecord(l.computed, s));
  }
  const int slot = (m->hj_head + m->hj_count) & 1;
  CHQ_CUDA(cudaMemcpyAsync(m->hj_clk[slot], m->ctl, sizeof(StepCtl), cudaMemcpyDeviceToHost, s));
  std::vector<chq_mesh::SnapItem> items;
  if ((rc = snapshot_enqueue(m, 4, names, arr, sizes, items, m->down_stream))) return rc;
  CHQ_CUDA(cudaEventRecord(m->hj_evt[slot], m->down_stream));
  ++m->hj_count;
  return CHQ_OK;
}

int chq_run_host_wait(chq_mesh *m, int *cycles) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  if (m->hj_count == 0) return fail(CHQ_ERR_STATE, "no host job in flight on this mesh");
  const int slot = m->hj_head;
  m->hj_head ^= 1;
  --m->hj_count;
  // the clock copy precedes the job's snapshot copy on the mesh stream, which precedes its
  // download on the snapshot stream
  CHQ_CUDA(cudaEventSynchronize(m->hj_evt[slot]));
  if (cycles) *cycles = static_cast<const StepCtl *>(m->hj_clk[slot])->cycle;
  return CHQ_OK;
}

int chq_set_device(int device) {
  CHQ_CUDA(cudaSetDevice(device));
  return CHQ_OK;
}

int chq_device_count(int *count) {
  if (!count) return fail(CHQ_ERR_ARG, "null argument");
  CHQ_CUDA(cudaGetDeviceCount(count));
  return CHQ_OK;
}

int chq_host_alloc(long long bytes, void **ptr) {
  if (!ptr || bytes <= 0) return fail(CHQ_ERR_ARG, "bad argument");
  cudaError_t e = cudaHostAlloc(ptr, (size_t)bytes, cudaHostAllocDefault);
  if (e != cudaSuccess) return fail(CHQ_ERR_NOMEM, std::string("pinned host allocation failed: ") + cudaGetErrorString(e));
  return CHQ_OK;
}

int chq_host_free(void *ptr) {
  if (ptr) CHQ_CUDA(cudaFreeHost(ptr));
  return CHQ_OK;
}

int chq_event_record(chq_mesh *m, int slot) {
  if (!m || slot < 0 || slot >= 8) return fail(CHQ_ERR_ARG, "bad argument");
  if (!m->slots[slot]) CHQ_CUDA(cudaEventCreate(&m->slots[slot]));
  CHQ_CUDA(cudaEventRecord(m->slots[slot], S(m, nullptr)));
  return CHQ_OK;
}

int chq_event_elapsed_between(chq_mesh *ma, int a, chq_mesh *mb, int b, float *ms) {
  if (!ma || !mb || !ms || a < 0 || a >= 8 || b < 0 || b >= 8 || !ma->slots[a] || !mb->slots[b])
    return fail(CHQ_ERR_ARG, "bad argument");
  CHQ_CUDA(cudaEventSynchronize(mb->slots[b]));
  CHQ_CUDA(cudaEventElapsedTime(ms, ma->slots[a], mb->slots[b]));
  return CHQ_OK;
}

int chq_event_elapsed(chq_mesh *m, int a, int b, float *ms) {
  if (!m || !ms || a < 0 || a >= 8 || b < 0 || b >= 8 || !m->slots[a] || !m->slots[b])
    return fail(CHQ_ERR_ARG, "bad argument");
  CHQ_CUDA(cudaEventSynchronize(m->slots[b]));
  CHQ_CUDA(cudaEventElapsedTime(ms, m->slots[a], m->slots[b]));
  return CHQ_OK;
}

bool grav_on(const chq_mesh *m) { return m->cfg.gravity_uniform || m->cfg.gravity_point; }
bool sts_on(const chq_mesh *m) { return m->diff && m->cfg.sts; }

// Argument tables from the members' current settings, the batch's stream and its completion
// event (members wait on it before work on their own streams).
static int batch_setup(chq_batch *B) {
  int rc = B->mixed ? batch_build<float>(B) : batch_build<double>(B);
  if (rc == CHQ_OK) {
    cudaError_t e = cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->done_evt, cudaEventDisableTiming);
    if (e != cudaSuccess) rc = cuda_fail(e, "batch stream");
  }
  if (rc != CHQ_OK) return rc;
  // an event that has never been recorded counts as complete, so members can wait on it now
  for (chq_mesh *m : B->jobs) m->batch_evt = B->done_evt;
  return CHQ_OK;
}

int chq_batch_create(chq_mesh *const *meshes, int n, chq_batch **out) {
  if (!meshes || n < 1 || !out) return fail(CHQ_ERR_ARG, "bad argument");
  *out = nullptr;
  const chq_mesh *a = meshes[0];
  for (int j = 0; j < n; ++j) {
    const chq_mesh *m = meshes[j];
    if (!m) return fail(CHQ_ERR_ARG, "null mesh in batch");
    if (m->slab_count > 1) return fail(CHQ_ERR_ARG, "a z slab cannot be a batch member");
    if (m->mixed != a->mixed || m->cfg.recon != a->cfg.recon || m->cfg.rsolver != a->cfg.rsolver ||
        m->cfg.characteristic != a->cfg.characteristic || m->nstage != a->nstage || m->cfg.fofc != a->cfg.fofc ||
        m->cfg.flux_limiter != a->cfg.flux_limiter)
      return fail(CHQ_ERR_ARG, "batch members must share precision, reconstruction, Riemann solver, "
                               "characteristic flag, integrator, FOFC and limiter switches");
    if (m->diff != a->diff || (m->cfg.cooling != 0) != (a->cfg.cooling != 0) || grav_on(m) != grav_on(a) ||
        sts_on(m) != sts_on(a))
      return fail(CHQ_ERR_ARG, "batch members must agree on diffusion, RKL2 super-time-stepping, cooling and "
                               "gravity (on or off; their coefficients may differ)");
    for (int q = 0; q < j; ++q)
      if (meshes[q] == m) return fail(CHQ_ERR_ARG, "a mesh appears twice in the batch");
  }
  chq_batch *B = new chq_batch;
  B->jobs.assign(meshes, meshes + n);
  B->mixed = a->mixed;
  B->recon = a->cfg.recon;
  B->rsolver = a->cfg.rsolver;
  B->charac = a->cfg.characteristic;
  B->nstage = a->nstage;
  B->fofc = a->cfg.fofc;
  B->limiter = a->cfg.flux_limiter;
  B->diff = (a->diff && !a->cfg.sts) ? 1 : 0;   // explicit diffusion inside the stages
  B->cool = a->cfg.cooling ? 1 : 0;
  B->grav = grav_on(a) ? 1 : 0;
  B->sts = sts_on(a) ? 1 : 0;
  B->xvar = a->xvar;   // the first member's x-sweep variant (chq_set_xvariant), as chq_batch_autotune sets it
  const int rc = batch_setup(B);
  if (rc != CHQ_OK) {
    batch_free(B);
    delete B;
    return rc;
  }
  *out = B;
  return CHQ_OK;
}

int chq_batch_destroy(chq_batch *B) {
  if (!B) return CHQ_OK;
  batch_free(B);
  delete B;
  return CHQ_OK;
}

int chq_batch_set_graph(chq_batch *B, int enable) {
  if (!B) return fail(CHQ_ERR_ARG, "null batch");
  B->use_graph = (enable != 0);
  return CHQ_OK;
}

int chq_batch_cycles(chq_batch *B, int n, void *stream) {
  if (!B || n < 0) return fail(CHQ_ERR_ARG, "bad argument");
  // members' own streams may still hold work (uploads, prime): order after them
  for (chq_mesh *m : B->jobs) CHQ_CUDA(cudaStreamSynchronize(m->stream));
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : B->stream;
  if (!B->use_graph || B->sts) {   // RKL2 batches take host decisions every cycle: no graph
    for (int c = 0; c < n; ++c) {
      const int rc = B->mixed ? batch_cycle<float>(B, s) : batch_cycle<double>(B, s);
      if (rc) return rc;
    }
    CHQ_CUDA(cudaEventRecord(B->done_evt, s));
    return CHQ_OK;
  }
  if (!B->exec) {
    // capture one cycle on the batch's own stream and keep the executable graph
    const long long l0 = B->nlaunch;
    CHQ_CUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = B->mixed ? batch_cycle<float>(B, B->stream) : batch_cycle<double>(B, B->stream);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(B->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    CHQ_CUDA(e);
    B->graph = g;
    CHQ_CUDA(cudaGraphInstantiate(&B->exec, B->graph, 0));
    B->per_cycle = B->nlaunch - l0;   // kernels in one cycle; the capture itself ran nothing
    B->nlaunch = l0;
  }
  for (int c = 0; c < n; ++c) CHQ_CUDA(cudaGraphLaunch(B->exec, s));
  B->nlaunch += B->per_cycle * n;
  CHQ_CUDA(cudaEventRecord(B->done_evt, s));
  return CHQ_OK;
}

int chq_batch_status(chq_batch *B, double *t, int *cycle, int *done) {
  if (!B) return fail(CHQ_ERR_ARG, "null batch");
  const int n = (int)B->jobs.size();
  batch_status_kernel<<<(n + 127) / 128, 128, 0, B->stream>>>(B->ctls, n, B->status);
  CHQ_CUDA(cudaGetLastError());
  std::vector<double> h(3 * n);
  CHQ_CUDA(cudaMemcpyAsync(h.data(), B->status, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, B->stream));
  CHQ_CUDA(cudaStreamSynchronize(B->stream));
  for (int j = 0; j < n; ++j) {
    if (t) t[j] = h[3 * j];
    if (cycle) cycle[j] = (int)h[3 * j + 1];
    if (done) done[j] = (int)h[3 * j + 2];
  }
  return CHQ_OK;
}

long long chq_batch_kernel_launches(const chq_batch *B) { return B ? B->nlaunch : 0; }


void *chq_batch_stream(chq_batch *B) { return B ? (void *)B->stream : nullptr; }

long long chq_kernel_launches(const chq_mesh *m) { return m ? m->nlaunch : 0; }

int chq_set_seglen(chq_mesh *m, int seglen) {
  if (!m || seglen < 1 || seglen > 1024) return fail(CHQ_ERR_ARG, "march length must be in [1, 1024]");
  if (seglen != m->seglen) drop_cycle_graph(m);
  m->seglen = seglen;
  return CHQ_OK;
}

int chq_get_seglen(const chq_mesh *m) { return m ? m->seglen : 0; }

int chq_set_xvariant(chq_mesh *m, int xvar) {
  if (!m || xvar < 0 || xvar >= CHQ_TUNE_NXVAR) return fail(CHQ_ERR_ARG, "x-sweep variant out of range");
  if (xvar != m->xvar) drop_cycle_graph(m);
  m->xvar = xvar;
  return CHQ_OK;
}

int chq_get_xvariant(const chq_mesh *m) { return m ? m->xvar : -1; }

int chq_set_yzvariant(chq_mesh *m, int yzvar) {
  if (!m || yzvar < 0 || yzvar > 1) return fail(CHQ_ERR_ARG, "y/z staging variant out of range");
  if (yzvar == 1 && !yz_tma_applies(m))
    return fail(CHQ_ERR_ARG, "TMA staging applies to 3-D FP64 meshes with PPM without characteristic projection");
  if (yzvar != m->yzvar) drop_cycle_graph(m);
  m->yzvar = yzvar;
  return CHQ_OK;
}

int chq_get_yzvariant(const chq_mesh *m) { return m ? m->yzvar : -1; }

}  // extern "C"

namespace {

// Device time of `reps` launches of `launch` after one warm-up launch, on stream s.
template <class F>
int time_launches(cudaStream_t s, int reps, F launch, double *ms) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  CHQ_CUDA(cudaEventCreate(&e0));
  cudaError_t e = cudaEventCreate(&e1);
  if (e != cudaSuccess) {
    cudaEventDestroy(e0);
    return cuda_fail(e, "autotune timing");
  }
  int rc = launch();
  if (rc == CHQ_OK) e = cudaEventRecord(e0, s);
  for (int r = 0; r < reps && rc == CHQ_OK && e == cudaSuccess; ++r) rc = launch();
  if (rc == CHQ_OK && e == cudaSuccess) e = cudaEventRecord(e1, s);
  float t = 0.f;
  if (rc == CHQ_OK && e == cudaSuccess) e = cudaEventSynchronize(e1);
  if (rc == CHQ_OK && e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc != CHQ_OK) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "autotune timing");
  *ms = t / reps;
  return CHQ_OK;
}

// Two-knob search shared by meshes and batches: the y/z march length over CHQ_TUNE_LENGTHS
// (x-sweep variant 0), then the x-sweep variants at the best length (the knobs act on
// different kernels). set(len, xvar) applies a candidate, run(&ms) times the flux launch.
template <class Set, class Run>
int tune_two_knobs(Set set, Run run, int nxvar, int *best_len, int *best_xvar, double ms_len[CHQ_TUNE_NLEN],
                   double ms_xvar[CHQ_TUNE_NXVAR]) {
  const int cand[CHQ_TUNE_NLEN] = CHQ_TUNE_LENGTHS;
  double best = 1e300;
  *best_len = cand[0];
  *best_xvar = 0;
  for (int q = 0; q < CHQ_TUNE_NLEN; ++q) {
    double t = 0.0;
    int rc = set(cand[q], 0);
    if (rc == CHQ_OK) rc = run(&t);
    if (rc != CHQ_OK) return rc;
    if (ms_len) ms_len[q] = t;
    if (t < best) {
      best = t;
      *best_len = cand[q];
    }
  }
  if (ms_xvar) {
    ms_xvar[0] = best;
    for (int v = nxvar; v < CHQ_TUNE_NXVAR; ++v) ms_xvar[v] = -1.0;
  }
  for (int v = 1; v < nxvar; ++v) {
    double t = 0.0;
    int rc = set(*best_len, v);
    if (rc == CHQ_OK) rc = run(&t);
    if (rc != CHQ_OK) return rc;
    if (ms_xvar) ms_xvar[v] = t;
    if (t < best) {
      best = t;
      *best_xvar = v;
    }
  }
  return set(*best_len, *best_xvar);
}

std::mutex g_tune_mu;
std::map<std::vector<long>, std::pair<int, int>> g_tune_cache;   // key -> (march length, x variant)

// x-sweep variants the tuner may pick. The FP64 form is compiled without multiply-add
// contraction, so both builds compute bit for bit the same fluxes; in the mixed form the
// compiler may contract the FP32 arithmetic differently in the two builds, which would make a
// job's rounding depend on the tuning (and a server job differ from the same job run alone),
// so the mixed form keeps variant 0.
int tune_xvariants(int mixed) { return mixed ? 1 : CHQ_TUNE_NXVAR; }

// batches of this many cells or more keep their members' launch settings untimed
constexpr long kBatchTuneMaxCells = 1L << 23;

}  // namespace

extern "C" {

int chq_autotune2(chq_mesh *m, int *seglen, int *xvar, double ms_len[CHQ_TUNE_NLEN],
                  double ms_xvar[CHQ_TUNE_NXVAR]) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  drop_cycle_graph(m);   // the captured cycle holds the old settings
  // per process: scheme, precision and mesh shape
  const std::vector<long> key = {0, m->mixed, m->cfg.recon, m->cfg.rsolver, m->cfg.characteristic,
                                 m->g.nx1, m->g.nx2, m->g.nx3};
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      m->seglen = it->second.first;
      m->xvar = it->second.second;
      if (seglen) *seglen = m->seglen;
      if (xvar) *xvar = m->xvar;
      if (ms_len)
        for (int q = 0; q < CHQ_TUNE_NLEN; ++q) ms_len[q] = -1.0;
      if (ms_xvar)
        for (int q = 0; q < CHQ_TUNE_NXVAR; ++q) ms_xvar[q] = -1.0;
      return CHQ_OK;
    }
  }
  cudaStream_t s = S(m, nullptr);
  const int keep_len = m->seglen, keep_x = m->xvar;
  int bl = keep_len, bx = keep_x;
  // fluxes are scratch: timing them leaves the state unchanged
  const int rc = tune_two_knobs(
      [&](int len, int v) {
        m->seglen = len;
        m->xvar = v;
        return CHQ_OK;
      },
      [&](double *t) { return time_launches(s, 3, [&] { return do_fluxes(m, 0, 7u, nullptr, s); }, t); },
      tune_xvariants(m->mixed), &bl, &bx, ms_len, ms_xvar);
  if (rc != CHQ_OK) {
    m->seglen = keep_len;
    m->xvar = keep_x;
    return rc;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = {bl, bx};
  }
  if (seglen) *seglen = bl;
  if (xvar) *xvar = bx;
  return CHQ_OK;
}

int chq_autotune(chq_mesh *m, int *seglen, double ms[CHQ_TUNE_NLEN]) {
  return chq_autotune2(m, seglen, nullptr, ms, nullptr);
}

int chq_autotune_yz(chq_mesh *m, int *yzvar, double ms[2]) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  if (ms) ms[0] = ms[1] = -1.0;
  if (!yz_tma_applies(m)) {
    if (yzvar) *yzvar = m->yzvar;
    return CHQ_OK;
  }
  drop_cycle_graph(m);
  cudaStream_t s = S(m, nullptr);
  double t[2] = {0.0, 0.0};
  const int keep = m->yzvar;
  for (int v = 0; v < 2; ++v) {
    m->yzvar = v;
    const int rc = time_launches(s, 3, [&] { return do_fluxes(m, 0, 7u, nullptr, s); }, &t[v]);
    if (rc != CHQ_OK) {
      m->yzvar = keep;
      return rc;
    }
  }
  // a TMA wait that gave up marks the step control: keep the cp.async form then
  StepCtl h;
  CHQ_CUDA(cudaMemcpyAsync(&h, m->ctl, sizeof(h), cudaMemcpyDeviceToHost, s));
  CHQ_CUDA(cudaStreamSynchronize(s));
  m->yzvar = (h.err == 0 && t[1] < t[0]) ? 1 : 0;
  if (ms) {
    ms[0] = t[0];
    ms[1] = t[1];
  }
  if (yzvar) *yzvar = m->yzvar;
  return CHQ_OK;
}

int chq_batch_autotune(chq_batch *B, int *seglen, int *xvar, double ms_len[CHQ_TUNE_NLEN],
                       double ms_xvar[CHQ_TUNE_NXVAR]) {
  if (!B || B->jobs.empty()) return fail(CHQ_ERR_ARG, "null or empty batch");
  // per process: scheme, precision, and the batch's size class (log2 of its cells and of its
  // member count), so that lanes of similar load share one measurement
  long cells = 0;
  for (const chq_mesh *m : B->jobs) cells += (long)m->g.nx1 * m->g.nx2 * m->g.nx3;
  const auto lg = [](long v) {
    int b = 0;
    while (v > 1) { v >>= 1; ++b; }
    return (long)b;
  };
  const std::vector<long> key = {1, B->mixed, B->recon, B->rsolver, B->charac, lg(cells), lg((long)B->jobs.size())};
  int bl = B->jobs[0]->seglen, bx = B->xvar;
  bool cached = false;
  if (cells >= kBatchTuneMaxCells) {
    // the members' own settings already fill the device: no timing (it would cost more than
    // it could gain over a short run); report them
    if (ms_len)
      for (int q = 0; q < CHQ_TUNE_NLEN; ++q) ms_len[q] = -1.0;
    if (ms_xvar)
      for (int q = 0; q < CHQ_TUNE_NXVAR; ++q) ms_xvar[q] = -1.0;
    if (seglen) *seglen = bl;
    if (xvar) *xvar = bx;
    return CHQ_OK;
  }
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    const auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      bl = it->second.first;
      bx = it->second.second;
      cached = true;
    }
  }
  // a new march length changes the flux launch geometry: rebuild the tables for it
  auto set = [&](int len, int v) -> int {
    bool same = (B->xvar == v);
    for (const chq_mesh *m : B->jobs) same = same && (m->seglen == len);
    if (same && B->dev) return CHQ_OK;
    batch_free(B);
    for (chq_mesh *m : B->jobs) {
      if (m->seglen != len) drop_cycle_graph(m);
      m->seglen = len;
      m->xvar = v;
    }
    B->xvar = v;
    return batch_setup(B);
  };
  if (cached) {
    if (ms_len)
      for (int q = 0; q < CHQ_TUNE_NLEN; ++q) ms_len[q] = -1.0;
    if (ms_xvar)
      for (int q = 0; q < CHQ_TUNE_NXVAR; ++q) ms_xvar[q] = -1.0;
  } else {
    // members' own streams may still hold work (uploads, prime): order after them
    for (chq_mesh *m : B->jobs) CHQ_CUDA(cudaStreamSynchronize(m->stream));
    const int rc = tune_two_knobs(
        set,
        [&](double *t) {
          return time_launches(B->stream, 3, [&]() -> int {
            const cudaError_t e = B->mixed ? batch_flux<float>(B, (const FluxArgs<float> *)B->a_flux[0], B->stream)
                                           : batch_flux<double>(B, (const FluxArgs<double> *)B->a_flux[0], B->stream);
            return (e == cudaSuccess) ? CHQ_OK : cuda_fail(e, "batched flux launch");
          }, t);
        },
        tune_xvariants(B->mixed), &bl, &bx, ms_len, ms_xvar);
    if (rc != CHQ_OK) return rc;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune_cache[key] = {bl, bx};
  }
  const int rc = set(bl, bx);
  if (rc != CHQ_OK) return rc;
  if (seglen) *seglen = bl;
  if (xvar) *xvar = bx;
  return CHQ_OK;
}

int chq_profile(chq_mesh *m, int enable) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  m->prof = (enable != 0);
  return CHQ_OK;
}

int chq_profile_read(chq_mesh *m, double ms[CHQ_NPROF], long long launches[CHQ_NPROF], int reset) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  CHQ_CUDA(cudaStreamSynchronize(m->stream));
  for (auto &p : m->pending) {
    float t = 0.f;
    if (cudaEventElapsedTime(&t, p.b, p.e) == cudaSuccess) {
      m->prof_ms[p.kind] += t;
      m->prof_n[p.kind] += 1;
    }
    m->pool.push_back(p.b);
    m->pool.push_back(p.e);
  }
  m->pending.clear();
  for (int k = 0; k < CHQ_NPROF; ++k) {
    if (ms) ms[k] = m->prof_ms[k];
    if (launches) launches[k] = m->prof_n[k];
    if (reset) { m->prof_ms[k] = 0; m->prof_n[k] = 0; }
  }
  return CHQ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// z slabs of one decomposed mesh (single-job multi-GPU domain decomposition). Each slab runs
// the stage of a whole mesh on its own planes; between the parts below the caller moves data
// between slabs (chq_slab_pack / chq_slab_unpack, and reductions of the step-control words
// chq_slab_ctl returns). Every part is asynchronous on `stream` (NULL = the mesh stream).
namespace {

int slab_check(chq_mesh *m) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  if (m->hrec) return fail(CHQ_ERR_ARG, "z slabs: device history recording is not supported");
  return CHQ_OK;
}

// spans of the halo message `what` for `side` (0: lower, 1: upper): pack = the planes the
// neighbour on that side needs, unpack = this slab's ghost planes that the neighbour on that
// side fills.
//   what 0: the state of buffer `buf` (the nghost planes the neighbour's ghosts hold);
//   what 1: the FOFC message of a stage whose output is buffer `buf`: the flags, b1 and b2 of
//           the boundary plane. The repair of the transverse faces on the ghost plane reads
//           the face-normal field of the stage's current state, which in a stage whose output
//           overwrites it (src/main.cpp:68-91) is the first update's output there.
int halo_spans(chq_mesh *m, int what, int buf, int side, bool pack, HaloArgs &a, long &words) {
  const Geom &g = m->g;
  const long sk = g.sk, vs = g.vstride, ng = g.ng;
  a = HaloArgs{};
  words = 0;
  auto add = [&](void *base, long first_plane, long nplanes, size_t esize) {
    a.src[a.nspan] = nullptr;
    a.dst[a.nspan] = reinterpret_cast<unsigned long long *>(static_cast<char *>(base) + (size_t)first_plane * sk * esize);
    a.words[a.nspan] = nplanes * sk * (long)esize / 8;
    words += a.words[a.nspan];
    ++a.nspan;
  };
  if ((what != 0 && what != 1) || (buf != 0 && buf != 1)) return fail(CHQ_ERR_ARG, "z slabs: unknown halo message");
  if (what == 1) {
    // the boundary plane (pack) or the ghost plane next to it (unpack)
    const long k = pack ? (side == 0 ? g.ks : g.ke) : (side == 0 ? g.ks - 1 : g.ke + 1);
    add(m->flag, k, 1, sizeof(int));
    add(m->bf[buf][0], k, 1, sizeof(double));
    add(m->bf[buf][1], k, 1, sizeof(double));
    return CHQ_OK;
  }
  // cell planes of u (6 components), b1, b2; face planes of b3
  long kc, kf, nf;
  if (pack) {
    kc = (side == 0) ? g.ks : g.ke + 1 - ng;
    kf = kc;
    nf = (side == 0) ? ng + 1 : ng;   // the lower neighbour also takes the shared face
  } else {
    kc = (side == 0) ? 0 : g.ke + 1;
    kf = kc;
    nf = (side == 0) ? ng : ng + 1;
  }
  for (int n = 0; n < NVAR; ++n) add(m->u[buf] + n * vs, kc, ng, sizeof(double));
  add(m->bf[buf][0], kc, ng, sizeof(double));
  add(m->bf[buf][1], kc, ng, sizeof(double));
  add(m->bf[buf][2], kf, nf, sizeof(double));
  return CHQ_OK;
}

int halo_copy(chq_mesh *m, int what, int buf, int side, bool pack, void *dev, cudaStream_t s) {
  if (side != 0 && side != 1) return fail(CHQ_ERR_ARG, "z slabs: side must be 0 or 1");
  if (!m->zpeer[side]) return fail(CHQ_ERR_ARG, "z slabs: no neighbouring slab on that side");
  // the FOFC message crosses internal slab boundaries only: at the periodic wrap the whole
  // mesh's repair sees ghost cells (never flagged) and the stage-start ghost fields
  if (what == 1 && !m->fofc_ext[side]) return CHQ_OK;
  if (!dev || (reinterpret_cast<uintptr_t>(dev) & 7)) return fail(CHQ_ERR_ARG, "z slabs: buffer must be 8-byte aligned");
  HaloArgs a;
  long words = 0;
  if (int rc = halo_spans(m, what, buf, side, pack, a, words)) return rc;
  // the packed buffer holds the spans back to back
  unsigned long long *b = static_cast<unsigned long long *>(dev);
  long maxw = 0;
  for (int q = 0; q < a.nspan; ++q) {
    if (pack) {
      a.src[q] = a.dst[q];
      a.dst[q] = b;
    } else {
      a.src[q] = b;
    }
    b += a.words[q];
    maxw = std::max(maxw, a.words[q]);
  }
  const dim3 grid((unsigned)std::max(1L, std::min(64L, (maxw + 255) / 256)), (unsigned)a.nspan);
  m->nlaunch += 1;
  halo_copy_kernel<<<grid, 256, 0, s>>>(a);
  CHQ_CUDA(cudaGetLastError());
  return CHQ_OK;
}

}  // namespace

extern "C" {

int chq_slab_info(const chq_mesh *m, int info[5]) {
  if (!m || !info) return fail(CHQ_ERR_ARG, "null argument");
  // info[2], info[3]: the side borders another slab (periodic wrap included)
  info[0] = m->slab_rank;
  info[1] = m->slab_count;
  info[2] = m->zpeer[0];
  info[3] = m->zpeer[1];
  info[4] = m->g.koff;
  return CHQ_OK;
}

int chq_slab_halo_bytes(chq_mesh *m, int what, int side, long long *bytes) {
  if (!m || !bytes || (side != 0 && side != 1)) return fail(CHQ_ERR_ARG, "bad argument");
  HaloArgs a;
  long words = 0;
  if (int rc = halo_spans(m, what, 0, side, true, a, words)) return rc;
  *bytes = (long long)words * 8;
  return CHQ_OK;
}

int chq_slab_pack(chq_mesh *m, int what, int buf, int side, void *dev, void *stream) {
  if (int rc = slab_check(m)) return rc;
  return halo_copy(m, what, buf, side, true, dev, S(m, stream));
}

int chq_slab_unpack(chq_mesh *m, int what, int buf, int side, const void *dev, void *stream) {
  if (int rc = slab_check(m)) return rc;
  return halo_copy(m, what, buf, side, false, const_cast<void *>(dev), S(m, stream));
}

int chq_slab_ctl(chq_mesh *m, int **nbad, unsigned long long **mdt_bits, unsigned long long **rho_bits) {
  if (!m) return fail(CHQ_ERR_ARG, "null mesh");
  if (nbad) *nbad = &m->ctl->nbad;
  if (mdt_bits) *mdt_bits = &m->ctl->mdt_bits;
  if (rho_bits) *rho_bits = &m->ctl->rho_bits;
  return CHQ_OK;
}

int chq_slab_prime(chq_mesh *m, double t, int part, void *stream) {
  if (int rc = slab_check(m)) return rc;
  cudaStream_t s = S(m, stream);
  int rc = CHQ_OK;
  if (part == 0) {
    ctl_prime_kernel<<<1, 1, 0, s>>>(m->ctl, t);
    CHQ_CUDA(cudaGetLastError());
    m->nlaunch += 1;
    return do_bc(m, 0, nullptr, s);
  }
  if (part == 1) {
    if ((rc = DISPATCH_P(m, do_c2p)(m, 0, 1, &m->ctl->mdt_bits, m->ctl, nullptr, s))) return rc;
    if (m->diff && (rc = DISPATCH_P(m, do_rho_min)(m, nullptr, s))) return rc;
    return CHQ_OK;
  }
  if (part == 2) {
    ctl_take_dt_kernel<<<1, 1, 0, s>>>(m->ctl);
    CHQ_CUDA(cudaGetLastError());
    m->nlaunch += 1;
    return CHQ_OK;
  }
  return fail(CHQ_ERR_ARG, "z slabs: prime part must be 0, 1 or 2");
}

int chq_slab_begin(chq_mesh *m, void *stream) {
  if (int rc = slab_check(m)) return rc;
  cudaStream_t s = S(m, stream);
  ctl_begin_kernel<<<1, 1, 0, s>>>(m->ctl, 0);
  CHQ_CUDA(cudaGetLastError());
  m->nlaunch += 1;
  return CHQ_OK;
}

int chq_slab_stage(chq_mesh *m, int stage, int part, void *stream) {
  if (int rc = slab_check(m)) return rc;
  if (stage < 1 || stage > m->nstage) return fail(CHQ_ERR_ARG, "z slabs: stage out of range");
  cudaStream_t s = S(m, stream);
  double g0, g1, beta;
  int cur, out;
  stage_table(m->nstage, stage, g0, g1, beta, cur, out);
  const int *done = &m->ctl->done;
  const double *bdt = &m->ctl->beta_dt[stage - 1];
  if (part == 0) return run_stage_a(m, cur, out, g0, g1, 0.0, bdt, done, s);
  if (part == 1) return run_stage_b(m, cur, out, g0, g1, 0.0, bdt, done, s);
  if (part == 2) {
    const bool last = (stage == m->nstage);
    int rc = last ? DISPATCH_P(m, do_c2p_end)(m, done, s)
                  : DISPATCH_P(m, do_c2p)(m, out, 0, &m->ctl->mdt_bits, m->ctl, done, s);
    if (!rc && last && m->diff) rc = DISPATCH_P(m, do_rho_min)(m, done, s);
    return rc;
  }
  return fail(CHQ_ERR_ARG, "z slabs: stage part must be 0, 1 or 2");
}

int chq_slab_end(chq_mesh *m, void *stream) {
  if (int rc = slab_check(m)) return rc;
  cudaStream_t s = S(m, stream);
  ctl_end_kernel<<<1, 1, 0, s>>>(m->ctl);
  CHQ_CUDA(cudaGetLastError());
  m->nlaunch += 1;
  return CHQ_OK;
}

}  // extern "C"
