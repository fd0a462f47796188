// C entry points over the reference's OWN kernels (compiled in place from the reference's
// src/ headers against oracle/kokkos_shim), so that tests and the CPU baseline can drive the
// reference stage by stage, kernel by kernel, or point function by point function.
//
// Test infrastructure only: the product never links or loads this library. The reference
// driver (src/main.cpp) is included with its `main` renamed so that its own `Stage()`
// (src/main.cpp:46-93) and `Physics` are the ones exercised; the configuration reading and
// the cycle below restate src/main.cpp:113-201 and src/main.cpp:246-297 for a library caller.
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#define main chasqui_reference_main
#include "main.cpp"
#undef main

namespace {

struct RefSim {
  Params pin;
  Physics ph;
  Mesh m;
  Real t = 0, tlim = 1, min_dt = 0;
  int cycle = 0, nlim = -1;
};

void Configure(RefSim &s) {
  // src/main.cpp:113-163 (same keys, same defaults)
  Params &pin = s.pin;
  Physics &ph = s.ph;
  Config &cfg = ph.cfg;
  const std::string r = pin.GetOrAddString("mhd", "reconstruct", "ppm");
  if (r == "dc") cfg.recon = Recon::dc;
  else if (r == "plm") cfg.recon = Recon::plm;
  else if (r == "ppm") cfg.recon = Recon::ppm;
  else if (r == "ppmx") cfg.recon = Recon::ppmx;
  else if (r == "wenoz") cfg.recon = Recon::wenoz;
  else throw std::runtime_error("unknown reconstruct: " + r);
  const std::string rs = pin.GetOrAddString("mhd", "rsolver", "hlld");
  if (rs == "hlld") cfg.rsolver = RSolver::hlld;
  else if (rs == "lhlld") cfg.rsolver = RSolver::lhlld;
  else if (rs == "hlle") cfg.rsolver = RSolver::hlle;
  else throw std::runtime_error("unknown rsolver: " + rs);
  cfg.characteristic = pin.GetOrAddBool("mhd", "characteristic", false);
  cfg.lhlld_phi = pin.GetOrAddReal("mhd", "lhlld_phi", -1.0);
  cfg.eos.dual_energy = pin.GetOrAddBool("mhd", "dual_energy", false);
  cfg.eos.de_eta = pin.GetOrAddReal("mhd", "de_eta", 1.0e-3);
  const std::string t = pin.GetOrAddString("time", "integrator", "rk3");
  if (t == "rk1") cfg.integ = Integrator::rk1;
  else if (t == "rk2") cfg.integ = Integrator::rk2;
  else if (t == "rk3") cfg.integ = Integrator::rk3;
  else if (t == "rk4" || t == "ssprk43") cfg.integ = Integrator::rk4;
  else throw std::runtime_error("unknown integrator: " + t);
  cfg.low_mach = pin.GetOrAddBool("mhd", "low_mach", false);
  cfg.flatten = pin.GetOrAddBool("mhd", "flatten", true);
  cfg.cfl = pin.GetOrAddReal("time", "cfl", 0.3);
  cfg.eos.gamma = pin.GetOrAddReal("mhd", "gamma", 5.0 / 3.0);
  cfg.eos.gm1 = cfg.eos.gamma - 1.0;
  cfg.eos.dfloor = pin.GetOrAddReal("mhd", "dfloor", 1.0e-10);
  cfg.eos.pfloor = pin.GetOrAddReal("mhd", "pfloor", 1.0e-12);
  cfg.bc1 = ParseBC(pin.GetOrAddString("mesh", "bc_x1", "periodic"));
  cfg.bc2 = ParseBC(pin.GetOrAddString("mesh", "bc_x2", "periodic"));
  cfg.bc3 = ParseBC(pin.GetOrAddString("mesh", "bc_x3", "periodic"));
  ph.fofc = pin.GetOrAddBool("mhd", "fofc", true);
  ph.flux_limiter = pin.GetOrAddBool("mhd", "flux_limiter", false);
  ph.sts = pin.GetOrAddBool("diffusion", "sts", false);
  ph.diff.nu = pin.GetOrAddReal("diffusion", "nu", 0.0);
  ph.diff.kappa = pin.GetOrAddReal("diffusion", "kappa", 0.0);
  ph.diff.eta = pin.GetOrAddReal("diffusion", "eta", 0.0);
  // gravity and cooling: src/main.cpp:147-162
  ph.grav.uniform = pin.GetOrAddBool("gravity", "uniform", false);
  ph.grav.g1 = pin.GetOrAddReal("gravity", "g1", 0.0);
  ph.grav.g2 = pin.GetOrAddReal("gravity", "g2", 0.0);
  ph.grav.g3 = pin.GetOrAddReal("gravity", "g3", 0.0);
  ph.grav.point = pin.GetOrAddBool("gravity", "point_mass", false);
  ph.grav.gm = pin.GetOrAddReal("gravity", "gm", 0.0);
  ph.grav.x0 = pin.GetOrAddReal("gravity", "x0", 0.0);
  ph.grav.y0 = pin.GetOrAddReal("gravity", "y0", 0.0);
  ph.grav.z0 = pin.GetOrAddReal("gravity", "z0", 0.0);
  ph.grav.rsoft = pin.GetOrAddReal("gravity", "rsoft", 0.0);
  ph.cool.enabled = pin.GetOrAddBool("cooling", "enabled", false);
  ph.cool.lambda0 = pin.GetOrAddReal("cooling", "lambda0", 0.0);
  ph.cool.alpha = pin.GetOrAddReal("cooling", "alpha", 1.0);
  ph.cool.tfloor = pin.GetOrAddReal("cooling", "tfloor", 0.0);
  // src/main.cpp:165-178
  Mesh &m = s.m;
  m.nx1 = pin.GetInt("mesh", "nx1");
  m.nx2 = pin.GetOrAddInt("mesh", "nx2", 1);
  m.nx3 = pin.GetOrAddInt("mesh", "nx3", 1);
  const bool wide = (cfg.recon == Recon::ppm || cfg.recon == Recon::ppmx || cfg.recon == Recon::wenoz);
  const int ng_min = wide ? 3 : 2;
  m.ng = pin.GetOrAddInt("mesh", "nghost", ng_min);
  if (m.ng < ng_min) throw std::runtime_error("nghost too small for the reconstruction method");
  m.x1min = pin.GetOrAddReal("mesh", "x1min", 0.0); m.x1max = pin.GetOrAddReal("mesh", "x1max", 1.0);
  m.x2min = pin.GetOrAddReal("mesh", "x2min", 0.0); m.x2max = pin.GetOrAddReal("mesh", "x2max", 1.0);
  m.x3min = pin.GetOrAddReal("mesh", "x3min", 0.0); m.x3max = pin.GetOrAddReal("mesh", "x3max", 1.0);
  m.Allocate();
  s.tlim = pin.GetOrAddReal("time", "tlim", 1.0);
  s.nlim = pin.GetOrAddInt("time", "nlim", -1);
}

// src/main.cpp:200-202: ghost fill + primitives + first time step on the u0 / b?f0 state
void Prime(RefSim &s) {
  Mesh &m = s.m;
  kernels::Boundaries(m, s.ph.cfg, m.u0, m.b1f0, m.b2f0, m.b3f0);
  s.min_dt = kernels::ConsToPrim(m, s.ph.cfg, m.u0, m.b1f0, m.b2f0, m.b3f0, true);
  if (!s.ph.sts) s.min_dt = fmin(s.min_dt, diffusion::TimeStep(m, s.ph.cfg, s.ph.diff));
}

// (g0, g1, beta, cur, out) of stage s: src/main.cpp:250-268
void StageCoeffs(int nstage, int st, Real &g0, Real &g1, Real &beta, bool &cur_u1, bool &out_u1) {
  if (nstage == 1) { g0 = 1; g1 = 0; beta = 1; cur_u1 = false; out_u1 = false; }
  else if (nstage == 2) {
    if (st == 1) { g0 = 1; g1 = 0; beta = 1; cur_u1 = false; out_u1 = true; }
    else { g0 = 0.5; g1 = 0.5; beta = 0.5; cur_u1 = true; out_u1 = false; }
  } else if (nstage == 3) {
    if (st == 1) { g0 = 1; g1 = 0; beta = 1; cur_u1 = false; out_u1 = true; }
    else if (st == 2) { g0 = 0.75; g1 = 0.25; beta = 0.25; cur_u1 = true; out_u1 = true; }
    else { g0 = 1.0 / 3.0; g1 = 2.0 / 3.0; beta = 2.0 / 3.0; cur_u1 = true; out_u1 = false; }
  } else {
    if (st == 1) { g0 = 1; g1 = 0; beta = 0.5; cur_u1 = false; out_u1 = true; }
    else if (st == 2) { g0 = 0; g1 = 1; beta = 0.5; cur_u1 = true; out_u1 = true; }
    else if (st == 3) { g0 = 2.0 / 3.0; g1 = 1.0 / 3.0; beta = 1.0 / 6.0; cur_u1 = true; out_u1 = true; }
    else { g0 = 0; g1 = 1; beta = 0.5; cur_u1 = true; out_u1 = false; }
  }
}

// one cycle of src/main.cpp:246-297 without outputs; returns false when tlim was reached
bool Cycle(RefSim &s) {
  Mesh &m = s.m;
  Physics &ph = s.ph;
  const Config &cfg = ph.cfg;
  if (!(s.t < s.tlim)) return false;
  Real dt = cfg.cfl * s.min_dt;
  if (s.t + dt > s.tlim) dt = s.tlim - s.t;
  const int nstage = static_cast<int>(cfg.integ);
  for (int st = 1; st <= nstage; ++st) {
    Real g0, g1, beta;
    bool cur_u1, out_u1;
    StageCoeffs(nstage, st, g0, g1, beta, cur_u1, out_u1);
    const bool last = (st == nstage);
    Stage(m, ph, cur_u1, out_u1, g0, g1, beta * dt);
    Arr4 uo = out_u1 ? m.u1 : m.u0;
    Arr3 b1o = out_u1 ? m.b1f1 : m.b1f0, b2o = out_u1 ? m.b2f1 : m.b2f0, b3o = out_u1 ? m.b3f1 : m.b3f0;
    const bool split_ops = last && (ph.sts || ph.cool.enabled);
    const Real mdt = kernels::ConsToPrim(m, cfg, uo, b1o, b2o, b3o, last && !split_ops);
    if (last && !split_ops) s.min_dt = fmin(mdt, diffusion::TimeStep(m, cfg, ph.diff));
  }
  // operator-split pieces on the end-of-step state: src/main.cpp:281-290
  if (ph.sts) {
    ph.sts_stages += sts::Advance(m, cfg, ph.diff, ph.sts_work, dt, diffusion::TimeStep(m, cfg, ph.diff));
    kernels::Boundaries(m, cfg, m.u0, m.b1f0, m.b2f0, m.b3f0);
  }
  if (ph.cool.enabled) {
    kernels::ConsToPrim(m, cfg, m.u0, m.b1f0, m.b2f0, m.b3f0, false);
    srcterms::ApplyCooling(m, cfg.eos, ph.cool, m.u0, dt);
    kernels::Boundaries(m, cfg, m.u0, m.b1f0, m.b2f0, m.b3f0);
  }
  if (ph.sts || ph.cool.enabled) {
    s.min_dt = kernels::ConsToPrim(m, cfg, m.u0, m.b1f0, m.b2f0, m.b3f0, true);
    if (!ph.sts) s.min_dt = fmin(s.min_dt, diffusion::TimeStep(m, cfg, ph.diff));
  }
  s.t += dt;
  ++s.cycle;
  return true;
}

Arr4 *Arr4By(Mesh &m, const char *n) {
  if (!std::strcmp(n, "u0")) return &m.u0;
  if (!std::strcmp(n, "u1")) return &m.u1;
  if (!std::strcmp(n, "w")) return &m.w;
  if (!std::strcmp(n, "bcc")) return &m.bcc;
  if (!std::strcmp(n, "ecc")) return &m.ecc;
  if (!std::strcmp(n, "f1")) return &m.f1;
  if (!std::strcmp(n, "f2")) return &m.f2;
  if (!std::strcmp(n, "f3")) return &m.f3;
  return nullptr;
}
Arr3 *Arr3By(Mesh &m, const char *n) {
  static const char *names[] = {"b1f0", "b2f0", "b3f0", "b1f1", "b2f1", "b3f1", "e2x1", "e3x1", "e1x2",
                                "e3x2", "e1x3", "e2x3", "e1",   "e2",   "e3"};
  Arr3 *arrs[] = {&m.b1f0, &m.b2f0, &m.b3f0, &m.b1f1, &m.b2f1, &m.b3f1, &m.e2x1, &m.e3x1,
                  &m.e1x2, &m.e3x2, &m.e1x3, &m.e2x3, &m.e1,   &m.e2,   &m.e3};
  for (int q = 0; q < 15; ++q)
    if (!std::strcmp(n, names[q])) return arrs[q];
  return nullptr;
}

thread_local std::string g_err;

template <class F>
int Guard(F f) {
  try {
    return f();
  } catch (const std::exception &e) {
    g_err = e.what();
    return -1;
  }
}

}  // namespace

extern "C" {

const char *chqref_last_error() { return g_err.c_str(); }

void chqref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}
int chqref_get_threads() { return omp_get_max_threads(); }

// infile: a reference input file; over: "block.key=value" overrides; rstfile: optional restart
// (the reference's own binary format) to start from instead of the problem generator.
void *chqref_open(const char *infile, int nover, const char **over, const char *rstfile) {
  RefSim *s = new RefSim;
  const int rc = Guard([&] {
    s->pin.ReadFile(infile);
    for (int q = 0; q < nover; ++q) s->pin.Override(over[q]);
    Configure(*s);
    if (rstfile && rstfile[0]) {
      restart::Read(s->m, rstfile, s->t, s->cycle);
    } else {
      pgen::Initialize(s->pin.GetString("problem", "name"), s->pin, s->m, s->ph.cfg);
    }
    Prime(*s);
    return 0;
  });
  if (rc != 0) { delete s; return nullptr; }
  return s;
}

void chqref_close(void *h) { delete static_cast<RefSim *>(h); }

int chqref_dims(void *h, int out[10]) {
  Mesh &m = static_cast<RefSim *>(h)->m;
  const int v[10] = {m.nx1, m.nx2, m.nx3, m.ng, m.ni, m.nj, m.nk, static_cast<int>(static_cast<RefSim *>(h)->ph.cfg.integ),
                     m.two_d ? 1 : 0, m.three_d ? 1 : 0};
  std::memcpy(out, v, sizeof(v));
  return 0;
}

double chqref_time(void *h) { return static_cast<RefSim *>(h)->t; }
int chqref_cycle(void *h) { return static_cast<RefSim *>(h)->cycle; }
double chqref_min_dt(void *h) { return static_cast<RefSim *>(h)->min_dt; }
long chqref_fofc_count(void *h) { return static_cast<RefSim *>(h)->ph.fofc_count; }
long chqref_limiter_count(void *h) { return static_cast<RefSim *>(h)->ph.limiter_count; }
long chqref_sts_stages(void *h) { return static_cast<RefSim *>(h)->ph.sts_stages; }
void chqref_set_time(void *h, double t, double tlim) {
  RefSim *s = static_cast<RefSim *>(h);
  s->t = t;
  s->tlim = tlim;
}

// copy a named mesh array out (get) or in (set), in the reference's layout including ghosts.
// "flag" is the FOFC int array converted to doubles.
long chqref_array_size(void *h, const char *name) {
  Mesh &m = static_cast<RefSim *>(h)->m;
  if (Arr4 *a = Arr4By(m, name)) return static_cast<long>(a->size());
  if (Arr3 *a = Arr3By(m, name)) return static_cast<long>(a->size());
  if (!std::strcmp(name, "flag")) return static_cast<long>(m.flag.size());
  return -1;
}
int chqref_get(void *h, const char *name, double *out, long n) {
  Mesh &m = static_cast<RefSim *>(h)->m;
  if (chqref_array_size(h, name) != n) return -1;
  if (Arr4 *a = Arr4By(m, name)) { std::memcpy(out, a->data(), n * sizeof(double)); return 0; }
  if (Arr3 *a = Arr3By(m, name)) { std::memcpy(out, a->data(), n * sizeof(double)); return 0; }
  for (long q = 0; q < n; ++q) out[q] = m.flag.data()[q];
  return 0;
}
int chqref_set(void *h, const char *name, const double *in, long n) {
  Mesh &m = static_cast<RefSim *>(h)->m;
  if (chqref_array_size(h, name) != n) return -1;
  if (Arr4 *a = Arr4By(m, name)) { std::memcpy(a->data(), in, n * sizeof(double)); return 0; }
  if (Arr3 *a = Arr3By(m, name)) { std::memcpy(a->data(), in, n * sizeof(double)); return 0; }
  for (long q = 0; q < n; ++q) m.flag.data()[q] = static_cast<int>(in[q]);
  return 0;
}

// ghost fill + primitives + dt of the u0/b?f0 state (after chqref_set of a new state)
int chqref_prime(void *h) { return Guard([&] { Prime(*static_cast<RefSim *>(h)); return 0; }); }

// up to n cycles; returns the number done (fewer when tlim is reached)
int chqref_cycles(void *h, int n) {
  RefSim *s = static_cast<RefSim *>(h);
  int done = 0;
  Guard([&] {
    while (done < n && Cycle(*s)) ++done;
    return 0;
  });
  return done;
}

// ---- kernel-level entry points (buffer selectors: 0 = u0/b?f0, 1 = u1/b?f1) ----
int chqref_stage(void *h, int cur_u1, int out_u1, double g0, double g1, double beta_dt) {
  RefSim *s = static_cast<RefSim *>(h);
  Stage(s->m, s->ph, cur_u1 != 0, out_u1 != 0, g0, g1, beta_dt);
  return 0;
}
double chqref_cons_to_prim(void *h, int buf, int compute_dt) {
  RefSim *s = static_cast<RefSim *>(h);
  Mesh &m = s->m;
  if (buf) return kernels::ConsToPrim(m, s->ph.cfg, m.u1, m.b1f1, m.b2f1, m.b3f1, compute_dt != 0);
  return kernels::ConsToPrim(m, s->ph.cfg, m.u0, m.b1f0, m.b2f0, m.b3f0, compute_dt != 0);
}
int chqref_boundaries(void *h, int buf) {
  RefSim *s = static_cast<RefSim *>(h);
  Mesh &m = s->m;
  if (buf) kernels::Boundaries(m, s->ph.cfg, m.u1, m.b1f1, m.b2f1, m.b3f1);
  else kernels::Boundaries(m, s->ph.cfg, m.u0, m.b1f0, m.b2f0, m.b3f0);
  return 0;
}
int chqref_fluxes(void *h, int dir, int cur_u1) {
  RefSim *s = static_cast<RefSim *>(h);
  Mesh &m = s->m;
  if (dir == 0) kernels::FluxesDispatch<0>(m, s->ph.cfg, cur_u1 ? m.b1f1 : m.b1f0);
  else if (dir == 1) kernels::FluxesDispatch<1>(m, s->ph.cfg, cur_u1 ? m.b2f1 : m.b2f0);
  else kernels::FluxesDispatch<2>(m, s->ph.cfg, cur_u1 ? m.b3f1 : m.b3f0);
  return 0;
}
int chqref_corner_emf(void *h) {
  kernels::CornerEMF(static_cast<RefSim *>(h)->m);
  return 0;
}
int chqref_update(void *h, int out_u1, double g0, double g1, double beta_dt) {
  Mesh &m = static_cast<RefSim *>(h)->m;
  kernels::StageArrays s;
  s.ua = m.u0; s.ub = m.u1; s.uout = out_u1 ? m.u1 : m.u0;
  s.b1a = m.b1f0; s.b2a = m.b2f0; s.b3a = m.b3f0;
  s.b1b = m.b1f1; s.b2b = m.b2f1; s.b3b = m.b3f1;
  s.b1out = out_u1 ? m.b1f1 : m.b1f0;
  s.b2out = out_u1 ? m.b2f1 : m.b2f0;
  s.b3out = out_u1 ? m.b3f1 : m.b3f0;
  kernels::Update(m, s, g0, g1, beta_dt);
  return 0;
}
int chqref_fofc_flag(void *h, int buf) {
  RefSim *s = static_cast<RefSim *>(h);
  Mesh &m = s->m;
  if (buf) return fofc::FlagBadCells(m, s->ph.cfg, m.u1, m.b1f1, m.b2f1, m.b3f1);
  return fofc::FlagBadCells(m, s->ph.cfg, m.u0, m.b1f0, m.b2f0, m.b3f0);
}
int chqref_fofc_repair(void *h, int dir, int cur_u1) {
  RefSim *s = static_cast<RefSim *>(h);
  Mesh &m = s->m;
  Arr3 b1 = cur_u1 ? m.b1f1 : m.b1f0, b2 = cur_u1 ? m.b2f1 : m.b2f0, b3 = cur_u1 ? m.b3f1 : m.b3f0;
  const diffusion::Coeffs dc = s->ph.sts ? diffusion::Coeffs{} : s->ph.diff;
  if (dir == 0) fofc::RepairFluxes<0>(m, s->ph.cfg, dc, b1, b2, b3);
  else if (dir == 1) fofc::RepairFluxes<1>(m, s->ph.cfg, dc, b1, b2, b3);
  else fofc::RepairFluxes<2>(m, s->ph.cfg, dc, b1, b2, b3);
  return 0;
}
long chqref_limit_fluxes(void *h, int dir, double beta_dt) {
  RefSim *s = static_cast<RefSim *>(h);
  Mesh &m = s->m;
  long cnt = 0;
  if (dir == 0) positivity::LimitFluxes<0>(m, s->ph.cfg, beta_dt, m.b1f0, &cnt);
  else if (dir == 1) positivity::LimitFluxes<1>(m, s->ph.cfg, beta_dt, m.b2f0, &cnt);
  else positivity::LimitFluxes<2>(m, s->ph.cfg, beta_dt, m.b3f0, &cnt);
  return cnt;
}
int chqref_history(void *h, double out[10]) {
  Mesh &m = static_cast<RefSim *>(h)->m;
  auto d = output::History(m, m.u0, m.b1f0, m.b2f0, m.b3f0);
  const double v[10] = {d.mass, d.mom1, d.mom2, d.mom3, d.etot, d.ekin, d.emag, d.eint, d.divb_max, d.divb_l1};
  std::memcpy(out, v, sizeof(v));
  return 0;
}
int chqref_write_vtk(void *h, const char *fname) {
  RefSim *s = static_cast<RefSim *>(h);
  return Guard([&] { output::WriteVTK(s->m, fname, s->t, s->cycle); return 0; });
}
int chqref_write_restart(void *h, const char *fname) {
  RefSim *s = static_cast<RefSim *>(h);
  return Guard([&] { restart::Write(s->m, fname, s->t, s->cycle); return 0; });
}

// ---- point functions (src/recon.hpp, src/riemann.hpp, src/eigen_mhd.hpp) ----
// scheme: 0 dc, 1 plm, 2 ppm, 3 wenoz, 4 ppmx (the reference's Recon enum values)
int chqref_recon(int scheme, const double *q, long n, double *ql, double *qr) {
  for (long s = 0; s < n; ++s) {
    const Real *qq = q + 6 * s;
    switch (scheme) {
      case 0: recon::Face<Recon::dc>(qq, ql[s], qr[s]); break;
      case 1: recon::Face<Recon::plm>(qq, ql[s], qr[s]); break;
      case 2: recon::Face<Recon::ppm>(qq, ql[s], qr[s]); break;
      case 3: recon::Face<Recon::wenoz>(qq, ql[s], qr[s]); break;
      case 4: recon::Face<Recon::ppmx>(qq, ql[s], qr[s]); break;
      default: return -1;
    }
  }
  return 0;
}
// p[5], u_{j-1}, u_{j+1} per sample
int chqref_flattening(const double *p5, const double *um1, const double *up1, long n, double *out) {
  for (long s = 0; s < n; ++s) out[s] = recon::Flattening(p5 + 5 * s, um1[s], up1[s]);
  return 0;
}
// solver: 0 hlle, 1 hlld, 2 hlld with explicit (theta, phi) and LHLLD speeds.
// states: 7 per sample (d, u, v, w, p, by, bz); f: 7 per sample
int chqref_riemann(int solver, const double *L, const double *R, const double *bn, long n, double gamma,
                   const double *theta, const double *phi, double *f) {
  EOS eos{gamma, gamma - 1.0, 1e-10, 1e-12};
  for (long s = 0; s < n; ++s) {
    const double *a = L + 7 * s, *b = R + 7 * s;
    State sl{a[0], a[1], a[2], a[3], a[4], a[5], a[6]};
    State sr{b[0], b[1], b[2], b[3], b[4], b[5], b[6]};
    if (solver == 0) HLLE(sl, sr, bn[s], eos, f + 7 * s);
    else if (solver == 1) HLLD(sl, sr, bn[s], eos, f + 7 * s);
    else HLLD(sl, sr, bn[s], eos, f + 7 * s, theta[s], phi[s], true);
  }
  return 0;
}
// w: (d,u,v,w,p,by,bz,bx) per sample -> L[49], R[49] row-major per sample
int chqref_eigen(const double *w, long n, double gamma, double *Lout, double *Rout) {
  for (long s = 0; s < n; ++s) {
    const double *q = w + 8 * s;
    Real Lm[7][7], Rm[7][7];
    eigen_mhd::Eigensystem(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], gamma, Lm, Rm);
    std::memcpy(Lout + 49 * s, Lm, sizeof(Lm));
    std::memcpy(Rout + 49 * s, Rm, sizeof(Rm));
  }
  return 0;
}

}  // extern "C"
