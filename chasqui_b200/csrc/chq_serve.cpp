// chasqui_b200 — continuous-batching simulation server, host C++ above the C ABI.
//
// Jobs (a mesh configuration, a device problem generator and its parameters, an end time or
// cycle limit) are submitted at any time. Each scheduling step
//   1. reads every running class's member clocks and retires finished jobs (their history
//      sums are kept, their device memory is freed),
//   2. admits queued jobs in submission order while they fit the HBM budget and the slot
//      limit (a job that does not fit does not block smaller ones behind it),
//   3. rebuilds the batch of every lane whose membership changed, and
//   4. launches `cycles_per_step` batched cycles of every lane. A class (jobs that share a
//      kernel instantiation) is spread over up to `lanes` batches, a new job joining the lane
//      with the fewest cells; each lane has its own stream and replays a CUDA graph, so the
//      flux kernel of one lane overlaps the memory-bound kernels of another. Batching alone
//      serialises every job through the same kernel sequence.
// Jobs of 2^21 cells or more (chq_server_set_solo_cells raises the threshold) are not
// batched: each runs "solo" on its own mesh stream (replaying a CUDA graph of one cycle, except with RKL2) and the
// server polls an event behind its chunk instead of waiting for it, so a large job never holds
// up the lanes (or another large job). At most `solo_slots` solo jobs run at once (default 1,
// chq_server_set_solo_slots): each fills the device alone, and two of them at once share it
// less efficiently (the 40 solo-sized jobs of the 256-job ensemble draw: 15.4 s with two at
// once, 13.2 s with one, as fast as running them one after another); the others wait in the
// queue while smaller jobs behind them are admitted into the lanes. No chunk is queued past a
// job's end where that is known (cycles_left), and a finished solo job's events and pinned
// clock slots go to the next one. Diffusion (explicit or RKL2), cooling and gravity
// batch with jobs that have the same terms switched on.
// Each job keeps its own dt and clock on the device, so its result is the same alone and in
// any mix. Times are seconds on the server's steady clock.
#include <chrono>
#include <cmath>
#include <cstring>
#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <utility>
#include <vector>
#include <cuda_runtime.h>
#include "chq.h"

namespace chq {
void set_last_error(const std::string &msg);
cudaStream_t mesh_stream(chq_mesh *m);
size_t clock_bytes();
int clock_enqueue(chq_mesh *m, void *pinned);
void clock_decode(const void *pinned, double *t, int *cycle);
}

namespace {

struct Job {
  long long id = 0;
  chq_config cfg{};
  int problem = 0;
  double prm[12] = {};
  int nprm = 0;
  int state = CHQ_JOB_QUEUED;
  chq_mesh *mesh = nullptr;
  long long bytes = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
  double t = 0;
  int cycle = 0;
  long long cells = 0;
  double hist[10] = {};
  // solo jobs (large meshes) run on their own stream with graph-replayed cycles, two chunks
  // queued; behind each chunk a copy of the clock lands in pinned memory and an event is
  // recorded, which the server polls, so a solo job never waits for the rest of the server
  bool solo = false;
  int head = 0, nfly = 0;             // oldest chunk in flight, chunks in flight
  long long queued = 0;               // cycles queued since the job was primed
  cudaEvent_t ev[2] = {nullptr, nullptr};
  void *clk[2] = {nullptr, nullptr};  // pinned clock copies
};

void free_solo(Job *j) {
  for (int q = 0; q < 2; ++q) {
    if (j->ev[q]) cudaEventDestroy(j->ev[q]);
    if (j->clk[q]) cudaFreeHost(j->clk[q]);
    j->ev[q] = nullptr;
    j->clk[q] = nullptr;
  }
}

// (precision, reconstruction, Riemann solver, characteristic, integrator, FOFC, limiter,
//  diffusion | cooling << 1 | gravity << 2 | RKL2 << 3, lane)
using ClassKey = std::tuple<int, int, int, int, int, int, int, int, int>;

bool has_diffusion(const chq_config &c) { return c.nu > 0 || c.kappa > 0 || c.eta > 0; }

int features(const chq_config &c) {
  return (has_diffusion(c) ? 1 : 0) | (c.cooling ? 2 : 0) | ((c.gravity_uniform || c.gravity_point) ? 4 : 0) |
         ((has_diffusion(c) && c.sts) ? 8 : 0);
}

ClassKey key_of(const chq_config &c, int lane) {
  return ClassKey{c.precision, c.recon, c.rsolver, c.characteristic, c.integrator, c.fofc, c.flux_limiter,
                  features(c), lane};
}

struct Group {
  std::vector<Job *> members;
  chq_batch *batch = nullptr;
  bool dirty = false;
  long long cells = 0;
  std::vector<chq_mesh *> retired;   // finished members' meshes, freed after their batch is dropped
  // launch settings of the lane, timed by chq_batch_autotune when the lane is first built and
  // given to the members of every later rebuild (no timing then)
  bool tuned = false;
  int seglen = 0, xvar = 0;
};

int err(int code, const std::string &m) {
  chq::set_last_error(m);
  return code;
}

// Cycles a job still needs beyond its first `from` cycles, or -1 when that is not known yet.
// A cycle limit (time.nlim) gives the exact count. An end time gives an estimate from the
// job's clock: the mean step so far carries it to tlim, with 5 % and one cycle to spare for
// a shrinking step. Cycles queued past a job's end return at once on the device, but each
// still launches every kernel of a cycle over the job's whole grid: this count keeps the
// server from queueing them.
long long cycles_left(const Job *j, long long from) {
  long long need = (j->cfg.nlim >= 0) ? (long long)j->cfg.nlim : -1;
  if (j->cycle > 0 && j->t > 0 && j->t < j->cfg.tlim) {
    const double mean = j->t / j->cycle;
    const double more = std::ceil(1.05 * (j->cfg.tlim - j->t) / mean) + 1.0;
    const long long est = j->cycle + (long long)std::min(more, 1e9);
    need = (need < 0) ? est : std::min(need, est);
  }
  return (need < 0) ? -1 : need - from;
}

}  // namespace

struct chq_server {
  long long budget = 0, used = 0;
  int max_active = 0, cycles_per_step = 1, lanes = 8;
  long long solo_cells = 0;   // jobs of at least this many cells run unbatched
  int solo_slots = 1;         // solo jobs running at once
  int autotune = 0;           // tune each new lane's batch (chq_batch_autotune); off by default
  long long next_id = 1;
  std::map<long long, Job *> jobs;
  std::vector<Job *> queue;
  std::map<ClassKey, Group> groups;
  std::vector<Job *> solo;   // running solo jobs
  // events and pinned clock copies of finished solo jobs, handed to the next solo jobs:
  // freeing pinned memory synchronises the device, and pinning it costs milliseconds
  std::vector<std::pair<cudaEvent_t, void *>> spare;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  long long zone_updates = 0;
  double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

namespace {

int retire_finished(chq_server *S) {
  for (auto &kv : S->groups) {
    Group &g = kv.second;
    if (!g.batch || g.members.empty()) continue;
    const size_t n = g.members.size();
    std::vector<double> t(n);
    std::vector<int> cyc(n), done(n);
    int rc = chq_batch_status(g.batch, t.data(), cyc.data(), done.data());
    if (rc) return rc;
    const double now = S->now();
    std::vector<Job *> keep;
    for (size_t q = 0; q < n; ++q) {
      Job *j = g.members[q];
      S->zone_updates += (long long)(cyc[q] - j->cycle) * j->cells;
      j->t = t[q];
      j->cycle = cyc[q];
      if (!done[q]) {
        keep.push_back(j);
        continue;
      }
      rc = chq_history(j->mesh, j->hist, nullptr);
      if (rc) return rc;
      bool finite = true;
      for (double v : j->hist) finite = finite && (v == v) && (v - v == 0.0);
      g.retired.push_back(j->mesh);   // freed below, after the batch that lists it
      j->mesh = nullptr;
      S->used -= j->bytes;
      // a state that went non-finite is quarantined: its neighbours in the batch never
      // read it (every kernel indexes its own job only)
      j->state = finite ? CHQ_JOB_DONE : CHQ_JOB_FAILED;
      j->t_done = now;
      g.cells -= j->cells;
      g.dirty = true;
    }
    g.members.swap(keep);
    if (!g.retired.empty()) {
      // the batch lists the finished meshes: drop it (the rebuild makes a new one) before
      // their memory is freed
      if (g.batch) chq_batch_destroy(g.batch);
      g.batch = nullptr;
      for (chq_mesh *m : g.retired) chq_mesh_destroy(m);
      g.retired.clear();
    }
  }
  return CHQ_OK;
}

// Jobs of at least this many cells run solo: one mesh stream each, cycles replayed as a CUDA
// graph; such a job fills the device by itself. chq_server_set_solo_cells can raise the
// threshold, not lower it.
const long long kSoloCells = 1LL << 21;   // default and minimum of chq_server::solo_cells

// finished solo chunks: progress and retirement; with `block`, wait for a chunk when none
// has finished
int retire_solo(chq_server *S, bool block) {
  bool any = false;
  Job *oldest = nullptr;
  auto finish = [&](Job *j) -> int {
    // the chunk behind the final one (if queued) returns at once on the device; history
    // runs after it on the mesh stream
    int rc = chq_history(j->mesh, j->hist, nullptr);
    if (rc) return rc;
    bool finite = true;
    for (double v : j->hist) finite = finite && (v == v) && (v - v == 0.0);
    chq_mesh_destroy(j->mesh);
    j->mesh = nullptr;
    // every chunk of the job has finished (chq_history waited for its stream)
    for (int q = 0; q < 2; ++q) {
      if (j->ev[q] && j->clk[q]) {
        S->spare.emplace_back(j->ev[q], j->clk[q]);
        j->ev[q] = nullptr;
        j->clk[q] = nullptr;
      }
    }
    free_solo(j);   // a half-made slot, if any
    j->nfly = 0;
    S->used -= j->bytes;
    j->state = finite ? CHQ_JOB_DONE : CHQ_JOB_FAILED;
    j->t_done = S->now();
    return CHQ_OK;
  };
  auto poll = [&]() -> int {
    for (Job *j : S->solo) {
      while (j->state == CHQ_JOB_RUNNING && j->nfly > 0) {
        const cudaError_t q = cudaEventQuery(j->ev[j->head]);
        if (q == cudaErrorNotReady) {
          if (!oldest) oldest = j;
          break;
        }
        if (q != cudaSuccess) return err(CHQ_ERR_CUDA, std::string("solo job: ") + cudaGetErrorString(q));
        double t = 0;
        int cyc = 0;
        chq::clock_decode(j->clk[j->head], &t, &cyc);
        j->head ^= 1;
        --j->nfly;
        any = true;
        S->zone_updates += (long long)(cyc - j->cycle) * j->cells;
        j->t = t;
        j->cycle = cyc;
        if (!(t < j->cfg.tlim) || (j->cfg.nlim >= 0 && cyc >= j->cfg.nlim)) {
          const int rc = finish(j);
          if (rc) return rc;
        }
      }
    }
    return CHQ_OK;
  };
  int rc = poll();
  if (rc) return rc;
  if (block && !any && oldest) {
    // no wait-for-any on events: wait for the first queued chunk, then take every chunk
    // that has finished by then
    const cudaError_t e = cudaEventSynchronize(oldest->ev[oldest->head]);
    if (e != cudaSuccess) return err(CHQ_ERR_CUDA, std::string("solo job: ") + cudaGetErrorString(e));
    if ((rc = poll())) return rc;
  }
  std::vector<Job *> keep;
  for (Job *j : S->solo)
    if (j->state == CHQ_JOB_RUNNING) keep.push_back(j);
  S->solo.swap(keep);
  return CHQ_OK;
}

// keep two chunks of cycles_per_step cycles queued on every solo job's stream, none past the
// job's end where that is known (the last chunk is shortened to it)
int launch_solo(chq_server *S) {
  for (Job *j : S->solo) {
    while (j->nfly < 2) {
      long long n = S->cycles_per_step;
      const long long left = cycles_left(j, j->queued);
      if (left >= 0) {
        if (left <= 0 && j->nfly > 0) break;
        // an end-time estimate fell short with nothing in flight: a short chunk more
        n = std::min(n, std::max(left, 2LL));
      }
      const int slot = (j->head + j->nfly) & 1;
      if (!j->ev[slot] && !S->spare.empty()) {
        j->ev[slot] = S->spare.back().first;
        j->clk[slot] = S->spare.back().second;
        S->spare.pop_back();
      }
      if (!j->ev[slot]) {
        cudaError_t e = cudaEventCreateWithFlags(&j->ev[slot], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaHostAlloc(&j->clk[slot], chq::clock_bytes(), cudaHostAllocDefault);
        if (e != cudaSuccess) return err(CHQ_ERR_CUDA, std::string("solo job: ") + cudaGetErrorString(e));
      }
      int rc = chq_cycles(j->mesh, (int)n, nullptr);
      if (!rc) rc = chq::clock_enqueue(j->mesh, j->clk[slot]);
      if (rc) return rc;
      j->queued += n;
      const cudaError_t e = cudaEventRecord(j->ev[slot], chq::mesh_stream(j->mesh));
      if (e != cudaSuccess) return err(CHQ_ERR_CUDA, std::string("solo job: ") + cudaGetErrorString(e));
      ++j->nfly;
    }
  }
  return CHQ_OK;
}

void admit(chq_server *S) {
  std::vector<Job *> still;
  int active = (int)S->solo.size();
  for (auto &kv : S->groups) active += (int)kv.second.members.size();
  int solo_running = (int)S->solo.size();
  for (Job *j : S->queue) {
    if (active >= S->max_active || S->used + j->bytes > S->budget ||
        (j->cells >= S->solo_cells && solo_running >= S->solo_slots)) {
      still.push_back(j);
      continue;
    }
    chq_mesh *m = nullptr;
    if (chq_mesh_create(&j->cfg, &m) != CHQ_OK) {
      still.push_back(j);   // e.g. the device is fuller than the budget says: retry later
      continue;
    }
    if (chq_init_problem(m, j->problem, j->prm, j->nprm, nullptr) != CHQ_OK || chq_prime(m, 0.0, nullptr) != CHQ_OK) {
      chq_mesh_destroy(m);
      j->state = CHQ_JOB_FAILED;
      j->t_done = S->now();
      continue;
    }
    j->mesh = m;
    j->bytes = chq_mesh_bytes(m);
    S->used += j->bytes;
    j->state = CHQ_JOB_RUNNING;
    j->t_start = S->now();
    if (j->cells >= S->solo_cells) {
      j->solo = true;
      S->solo.push_back(j);
      ++active;
      ++solo_running;
      continue;
    }
    int lane = 0;
    long long least = -1;
    for (int q = 0; q < S->lanes; ++q) {
      const auto it = S->groups.find(key_of(j->cfg, q));
      const long long c = (it == S->groups.end()) ? 0 : it->second.cells;
      if (least < 0 || c < least) {
        least = c;
        lane = q;
      }
    }
    Group &g = S->groups[key_of(j->cfg, lane)];
    g.members.push_back(j);
    g.cells += j->cells;
    g.dirty = true;
    ++active;
  }
  S->queue.swap(still);
}

int rebuild(chq_server *S) {
  for (auto &kv : S->groups) {
    Group &g = kv.second;
    if (!g.dirty) continue;
    if (g.batch) {
      chq_batch_destroy(g.batch);
      g.batch = nullptr;
    }
    for (chq_mesh *m : g.retired) chq_mesh_destroy(m);
    g.retired.clear();
    g.dirty = false;
    if (g.members.empty()) continue;
    std::vector<chq_mesh *> ms;
    int rc = CHQ_OK;
    for (Job *j : g.members) {
      ms.push_back(j->mesh);
      if (S->autotune && g.tuned) {
        if ((rc = chq_set_seglen(j->mesh, g.seglen)) || (rc = chq_set_xvariant(j->mesh, g.xvar))) return rc;
      }
    }
    rc = chq_batch_create(ms.data(), (int)ms.size(), &g.batch);
    if (rc) return rc;
    if (S->autotune && !g.tuned) {
      rc = chq_batch_autotune(g.batch, &g.seglen, &g.xvar, nullptr, nullptr);
      if (rc) return rc;
      g.tuned = true;
    }
    chq_batch_set_graph(g.batch, 1);
  }
  return CHQ_OK;
}

}  // namespace

extern "C" {

int chq_server_create(long long hbm_budget_bytes, int max_active, int cycles_per_step, chq_server **out) {
  if (!out || hbm_budget_bytes <= 0 || max_active < 1 || cycles_per_step < 1) return err(CHQ_ERR_ARG, "bad argument");
  chq_server *S = new chq_server;
  S->budget = hbm_budget_bytes;
  S->max_active = max_active;
  S->cycles_per_step = cycles_per_step;
  S->solo_cells = kSoloCells;
  *out = S;
  return CHQ_OK;
}

int chq_server_submit(chq_server *S, const chq_config *cfg, int problem, const double *params, int nparams,
                      long long *id) {
  if (!S || !cfg || nparams < 0 || nparams > 12 || (nparams && !params)) return err(CHQ_ERR_ARG, "bad argument");
  const long long bytes = chq_config_bytes(cfg);
  if (bytes <= 0) return err(CHQ_ERR_ARG, "invalid job configuration");
  if (bytes > S->budget) return err(CHQ_ERR_ARG, "job larger than the server's HBM budget");
  Job *j = new Job;
  j->id = S->next_id++;
  j->cfg = *cfg;
  j->problem = problem;
  j->nprm = nparams;
  for (int q = 0; q < nparams; ++q) j->prm[q] = params[q];
  j->bytes = bytes;
  j->cells = (long long)cfg->nx1 * cfg->nx2 * cfg->nx3;
  j->t_submit = S->now();
  S->jobs[j->id] = j;
  S->queue.push_back(j);
  if (id) *id = j->id;
  return CHQ_OK;
}

int chq_server_step(chq_server *S) {
  if (!S) return err(CHQ_ERR_ARG, "null server");
  bool lanes_busy = false;
  for (auto &kv : S->groups) lanes_busy = lanes_busy || (kv.second.batch && !kv.second.members.empty());
  // solo jobs first without waiting (block only when nothing else would make progress)
  int rc = retire_solo(S, !lanes_busy);
  if (rc) return rc;
  rc = retire_finished(S);
  if (rc) return rc;
  admit(S);
  rc = rebuild(S);
  if (rc) return rc;
  // Balanced chunks: the next step waits for every lane, so each lane gets about the same
  // work per step. The lane with the most cells runs cycles_per_step cycles, a lighter lane
  // proportionally more (at most 4x); cycles past a job's end return at once on the device.
  long long heaviest = 0;
  for (auto &kv : S->groups)
    if (kv.second.batch) heaviest = std::max(heaviest, kv.second.cells);
  rc = launch_solo(S);
  if (rc) return rc;
  int active = (int)S->solo.size();
  for (auto &kv : S->groups) {
    Group &g = kv.second;
    if (!g.batch) continue;
    long long n = S->cycles_per_step;
    if (g.cells > 0) n = std::min<long long>(4LL * S->cycles_per_step, (S->cycles_per_step * heaviest + g.cells - 1) / g.cells);
    // no cycles past the last member's end where every member's end is known (the members'
    // clocks were read at this step: the lane has nothing in flight)
    long long most = 0;
    for (const Job *j : g.members) {
      const long long left = cycles_left(j, j->cycle);
      most = (left < 0 || most < 0) ? -1 : std::max(most, left);
    }
    if (most >= 0) n = std::min(n, std::max(most, 1LL));
    rc = chq_batch_cycles(g.batch, (int)std::max(1LL, n), nullptr);
    if (rc) return rc;
    active += (int)g.members.size();
  }
  return active + (int)S->queue.size();
}

int chq_server_status(chq_server *S, long long id, chq_job_status *st) {
  if (!S || !st) return err(CHQ_ERR_ARG, "bad argument");
  auto it = S->jobs.find(id);
  if (it == S->jobs.end()) return err(CHQ_ERR_ARG, "unknown job id");
  const Job *j = it->second;
  std::memset(st, 0, sizeof(*st));
  st->state = j->state;
  st->cycle = j->cycle;
  st->t = j->t;
  st->t_submit = j->t_submit;
  st->t_start = j->t_start;
  st->t_done = j->t_done;
  st->zone_updates = (long long)j->cycle * j->cells;
  st->bytes = j->bytes;
  std::memcpy(st->history, j->hist, sizeof(j->hist));
  return CHQ_OK;
}

chq_mesh *chq_server_job_mesh(chq_server *S, long long id) {
  if (!S) return nullptr;
  auto it = S->jobs.find(id);
  return (it == S->jobs.end() || it->second->state != CHQ_JOB_RUNNING) ? nullptr : it->second->mesh;
}

int chq_server_stats(chq_server *S, long long *used_bytes, int *active, int *queued, long long *zone_updates,
                     double *clock) {
  if (!S) return err(CHQ_ERR_ARG, "null server");
  int a = (int)S->solo.size();
  for (auto &kv : S->groups) a += (int)kv.second.members.size();
  if (used_bytes) *used_bytes = S->used;
  if (active) *active = a;
  if (queued) *queued = (int)S->queue.size();
  if (zone_updates) *zone_updates = S->zone_updates;
  if (clock) *clock = S->now();
  return CHQ_OK;
}

int chq_server_set_lanes(chq_server *S, int lanes) {
  if (!S || lanes < 1 || lanes > 64) return err(CHQ_ERR_ARG, "lanes must be in [1, 64]");
  S->lanes = lanes;
  return CHQ_OK;
}

int chq_server_set_solo_cells(chq_server *S, long long cells) {
  if (!S || cells < 0) return err(CHQ_ERR_ARG, "bad argument");
  // lower thresholds (many more solo jobs) are not offered: a serving run with the threshold
  // at 2^15 cells ended in a device fault whose cause is not known
  if (cells < kSoloCells) return err(CHQ_ERR_ARG, "the solo threshold must be at least 2^21 cells");
  S->solo_cells = cells;
  return CHQ_OK;
}

int chq_server_set_solo_slots(chq_server *S, int slots) {
  if (!S || slots < 1 || slots > 1024) return err(CHQ_ERR_ARG, "solo slots must be in [1, 1024]");
  S->solo_slots = slots;
  return CHQ_OK;
}

int chq_server_set_autotune(chq_server *S, int enable) {
  if (!S) return err(CHQ_ERR_ARG, "null server");
  S->autotune = (enable != 0);
  return CHQ_OK;
}

int chq_server_destroy(chq_server *S) {
  if (!S) return CHQ_OK;
  for (auto &kv : S->groups) {
    if (kv.second.batch) chq_batch_destroy(kv.second.batch);
    for (chq_mesh *m : kv.second.retired) chq_mesh_destroy(m);
  }
  for (auto &kv : S->jobs) {
    if (kv.second->mesh) chq_mesh_destroy(kv.second->mesh);   // synchronises its stream first
    free_solo(kv.second);
    delete kv.second;
  }
  for (auto &sp : S->spare) {
    cudaEventDestroy(sp.first);
    if (sp.second) cudaFreeHost(sp.second);
  }
  delete S;
  return CHQ_OK;
}

}  // extern "C"
