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
// Each job keeps its own dt and clock on the device, so its result is the same alone and in
// any mix. Times are seconds on the server's steady clock.
#include <chrono>
#include <cstring>
#include <algorithm>
#include <map>
#include <string>
#include <tuple>
#include <vector>
#include "chq.h"

namespace chq {
void set_last_error(const std::string &msg);
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
};

// (precision, reconstruction, Riemann solver, characteristic, integrator, FOFC, limiter, lane)
using ClassKey = std::tuple<int, int, int, int, int, int, int, int>;

ClassKey key_of(const chq_config &c, int lane) {
  return ClassKey{c.precision, c.recon, c.rsolver, c.characteristic, c.integrator, c.fofc, c.flux_limiter, lane};
}

struct Group {
  std::vector<Job *> members;
  chq_batch *batch = nullptr;
  bool dirty = false;
  long long cells = 0;
  std::vector<chq_mesh *> retired;   // finished members' meshes, freed after their batch is dropped
};

int err(int code, const std::string &m) {
  chq::set_last_error(m);
  return code;
}

}  // namespace

struct chq_server {
  long long budget = 0, used = 0;
  int max_active = 0, cycles_per_step = 1, lanes = 8;
  long long next_id = 1;
  std::map<long long, Job *> jobs;
  std::vector<Job *> queue;
  std::map<ClassKey, Group> groups;
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

void admit(chq_server *S) {
  std::vector<Job *> still;
  int active = 0;
  for (auto &kv : S->groups) active += (int)kv.second.members.size();
  for (Job *j : S->queue) {
    if (active >= S->max_active || S->used + j->bytes > S->budget) {
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
    for (Job *j : g.members) ms.push_back(j->mesh);
    const int rc = chq_batch_create(ms.data(), (int)ms.size(), &g.batch);
    if (rc) return rc;
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
  *out = S;
  return CHQ_OK;
}

int chq_server_submit(chq_server *S, const chq_config *cfg, int problem, const double *params, int nparams,
                      long long *id) {
  if (!S || !cfg || nparams < 0 || nparams > 12 || (nparams && !params)) return err(CHQ_ERR_ARG, "bad argument");
  const long long bytes = chq_config_bytes(cfg);
  if (bytes <= 0) return err(CHQ_ERR_ARG, "invalid job configuration");
  if (bytes > S->budget) return err(CHQ_ERR_ARG, "job larger than the server's HBM budget");
  if (cfg->nu > 0 || cfg->kappa > 0 || cfg->eta > 0 || cfg->cooling || cfg->gravity_uniform || cfg->gravity_point)
    return err(CHQ_ERR_ARG, "the server batches ideal-MHD jobs; run jobs with diffusion or source terms on their "
                            "own mesh");
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
  int rc = retire_finished(S);
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
  int active = 0;
  for (auto &kv : S->groups) {
    Group &g = kv.second;
    if (!g.batch) continue;
    long long n = S->cycles_per_step;
    if (g.cells > 0) n = std::min<long long>(4LL * S->cycles_per_step, (S->cycles_per_step * heaviest + g.cells - 1) / g.cells);
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
  int a = 0;
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

int chq_server_destroy(chq_server *S) {
  if (!S) return CHQ_OK;
  for (auto &kv : S->groups) {
    if (kv.second.batch) chq_batch_destroy(kv.second.batch);
    for (chq_mesh *m : kv.second.retired) chq_mesh_destroy(m);
  }
  for (auto &kv : S->jobs) {
    if (kv.second->mesh) chq_mesh_destroy(kv.second->mesh);
    delete kv.second;
  }
  delete S;
  return CHQ_OK;
}

}  // extern "C"
