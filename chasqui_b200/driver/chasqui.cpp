// chasqui_b200 — command-line driver, a drop-in for the reference's `chasqui` binary:
//
//   chasqui -i input.in [-r restart.rst] [block.key=value ...]
//
// Same input keys and defaults, problem generators, outputs (.vtk, .hst, .rst, _errors.dat)
// and end-of-run lines as the reference driver (src/main.cpp:95-329); the time loop runs on
// the device through the C ABI (include/chq.h): whole cycles are queued with chq_cycles and
// dt, the FOFC and limiter counts stay on the device. The host reads the clock once per
// cycle only while outputs are scheduled, otherwise once per `time.ndiag` cycles (at most 256).
// Gravity and cooling source terms (src/srcterms.hpp) run on the device as well.
// `mhd.precision = mixed` selects the mixed FP32/FP64 form. `--write-ic FILE`
// writes the problem generator's initial state as a restart file and exits without a GPU.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "chq.h"
#include "outputs.hpp"
#include "params.hpp"
#include "problems.hpp"

namespace {

void check(int rc, const char *what) {
  if (rc != CHQ_OK) throw std::runtime_error(std::string(what) + ": " + chq_last_error());
}

int parse_bc(const std::string &s) {
  if (s == "periodic") return CHQ_BC_PERIODIC;
  if (s == "outflow") return CHQ_BC_OUTFLOW;
  if (s == "reflect") return CHQ_BC_REFLECT;
  throw std::runtime_error("unknown boundary condition: " + s);
}

std::vector<double> download(chq_mesh *m, const char *name) {
  std::vector<double> v((size_t)chq_array_size(m, name));
  check(chq_download(m, name, v.data(), (long)v.size(), nullptr), name);
  return v;
}

void upload(chq_mesh *m, const char *name, const std::vector<double> &v) {
  check(chq_upload(m, name, v.data(), (long)v.size(), nullptr), name);
}

int run(int argc, char **argv) {
  chqd::Params pin;
  std::string input, rstfile, icfile;
  for (int a = 1; a < argc; ++a) {
    if (!std::strcmp(argv[a], "-i") && a + 1 < argc) input = argv[++a];
    else if (!std::strcmp(argv[a], "-r") && a + 1 < argc) rstfile = argv[++a];
    else if (!std::strcmp(argv[a], "--write-ic") && a + 1 < argc) icfile = argv[++a];
  }
  if (input.empty()) {
    std::cerr << "usage: chasqui -i input.in [-r restart.rst] [block.key=value ...]\n";
    return 1;
  }
  pin.read_file(input);
  for (int a = 1; a < argc; ++a) {
    if (!std::strcmp(argv[a], "-i") || !std::strcmp(argv[a], "-r") || !std::strcmp(argv[a], "--write-ic")) {
      ++a;
      continue;
    }
    if (std::strchr(argv[a], '=')) pin.override_with(argv[a]);
  }

  // ---- configuration (keys and defaults of src/main.cpp:113-185) ----
  chq_config cfg;
  chq_config_defaults(&cfg);
  const std::string r = pin.str("mhd", "reconstruct", "ppm");
  cfg.recon = (r == "dc") ? CHQ_RECON_DC : (r == "plm") ? CHQ_RECON_PLM : (r == "ppm") ? CHQ_RECON_PPM
            : (r == "ppmx") ? CHQ_RECON_PPMX : (r == "wenoz") ? CHQ_RECON_WENOZ : -1;
  if (cfg.recon < 0) throw std::runtime_error("unknown reconstruct: " + r);
  const std::string rs = pin.str("mhd", "rsolver", "hlld");
  cfg.rsolver = (rs == "hlld") ? CHQ_RS_HLLD : (rs == "lhlld") ? CHQ_RS_LHLLD : (rs == "hlle") ? CHQ_RS_HLLE : -1;
  if (cfg.rsolver < 0) throw std::runtime_error("unknown rsolver: " + rs);
  cfg.characteristic = pin.boolean("mhd", "characteristic", false);
  cfg.lhlld_phi = pin.real("mhd", "lhlld_phi", -1.0);
  cfg.dual_energy = pin.boolean("mhd", "dual_energy", false);
  cfg.de_eta = pin.real("mhd", "de_eta", 1.0e-3);
  const std::string ti = pin.str("time", "integrator", "rk3");
  cfg.integrator = (ti == "rk1") ? 1 : (ti == "rk2") ? 2 : (ti == "rk3") ? 3 : (ti == "rk4" || ti == "ssprk43") ? 4 : -1;
  if (cfg.integrator < 0) throw std::runtime_error("unknown integrator: " + ti);
  cfg.low_mach = pin.boolean("mhd", "low_mach", false);
  cfg.flatten = pin.boolean("mhd", "flatten", true);
  cfg.cfl = pin.real("time", "cfl", 0.3);
  cfg.gamma = pin.real("mhd", "gamma", 5.0 / 3.0);
  cfg.dfloor = pin.real("mhd", "dfloor", 1.0e-10);
  cfg.pfloor = pin.real("mhd", "pfloor", 1.0e-12);
  cfg.bc1 = parse_bc(pin.str("mesh", "bc_x1", "periodic"));
  cfg.bc2 = parse_bc(pin.str("mesh", "bc_x2", "periodic"));
  cfg.bc3 = parse_bc(pin.str("mesh", "bc_x3", "periodic"));
  cfg.fofc = pin.boolean("mhd", "fofc", true);
  cfg.flux_limiter = pin.boolean("mhd", "flux_limiter", false);
  cfg.sts = pin.boolean("diffusion", "sts", false);
  cfg.nu = pin.real("diffusion", "nu", 0.0);
  cfg.kappa = pin.real("diffusion", "kappa", 0.0);
  cfg.eta = pin.real("diffusion", "eta", 0.0);
  cfg.gravity_uniform = pin.boolean("gravity", "uniform", false);
  cfg.g1 = pin.real("gravity", "g1", 0.0);
  cfg.g2 = pin.real("gravity", "g2", 0.0);
  cfg.g3 = pin.real("gravity", "g3", 0.0);
  cfg.gravity_point = pin.boolean("gravity", "point_mass", false);
  cfg.gm = pin.real("gravity", "gm", 0.0);
  cfg.gx0 = pin.real("gravity", "x0", 0.0);
  cfg.gy0 = pin.real("gravity", "y0", 0.0);
  cfg.gz0 = pin.real("gravity", "z0", 0.0);
  cfg.rsoft = pin.real("gravity", "rsoft", 0.0);
  cfg.cooling = pin.boolean("cooling", "enabled", false);
  cfg.lambda0 = pin.real("cooling", "lambda0", 0.0);
  cfg.cool_alpha = pin.real("cooling", "alpha", 1.0);
  cfg.tfloor = pin.real("cooling", "tfloor", 0.0);
  const std::string prec = pin.str("mhd", "precision", "fp64");
  cfg.precision = (prec == "fp64") ? CHQ_FP64 : (prec == "mixed") ? CHQ_MIXED : -1;
  if (cfg.precision < 0) throw std::runtime_error("unknown precision: " + prec + " (fp64 or mixed)");

  chqd::Grid g{};
  g.nx1 = pin.integer("mesh", "nx1");
  g.nx2 = pin.integer("mesh", "nx2", 1);
  g.nx3 = pin.integer("mesh", "nx3", 1);
  const bool wide = cfg.recon == CHQ_RECON_PPM || cfg.recon == CHQ_RECON_PPMX || cfg.recon == CHQ_RECON_WENOZ;
  const int ng_min = wide ? 3 : 2;
  g.ng = pin.integer("mesh", "nghost", ng_min);
  if (g.ng < ng_min) throw std::runtime_error("nghost too small for the reconstruction method");
  g.x1min = pin.real("mesh", "x1min", 0.0); g.x1max = pin.real("mesh", "x1max", 1.0);
  g.x2min = pin.real("mesh", "x2min", 0.0); g.x2max = pin.real("mesh", "x2max", 1.0);
  g.x3min = pin.real("mesh", "x3min", 0.0); g.x3max = pin.real("mesh", "x3max", 1.0);
  g.setup();
  cfg.nx1 = g.nx1; cfg.nx2 = g.nx2; cfg.nx3 = g.nx3; cfg.nghost = g.ng;
  cfg.x1min = g.x1min; cfg.x1max = g.x1max; cfg.x2min = g.x2min; cfg.x2max = g.x2max;
  cfg.x3min = g.x3min; cfg.x3max = g.x3max;

  const double tlim = pin.real("time", "tlim", 1.0);
  const int nlim = pin.integer("time", "nlim", -1);
  const int ndiag = pin.integer("time", "ndiag", 100);
  const std::string problem = pin.str("problem", "name");
  const std::string basename = pin.str("output", "basename", problem);
  const double dt_vtk = pin.real("output", "vtk_dt", -1.0);
  const double dt_hst = pin.real("output", "hst_dt", -1.0);
  const double dt_rst = pin.real("output", "rst_dt", -1.0);
  const bool compute_error = pin.boolean("output", "compute_error", false);
  cfg.tlim = tlim;
  cfg.nlim = nlim;

  std::cout << "# Chasqui MHD\n";
  pin.print(std::cout);
  std::cout << "# execution space: CUDA sm_100a (chasqui_b200 device stage path, "
            << (cfg.precision == CHQ_MIXED ? "mixed FP32/FP64" : "FP64") << ")\n";

  // ---- initial conditions or restart ----
  double t = 0.0;
  int cycle = 0;
  chqd::HostState h(g);
  if (rstfile.empty()) {
    chqd::initialize(problem, pin, g, cfg.gamma, h);
  } else {
    chqd::read_restart(g, rstfile, t, cycle, h.u, h.b1, h.b2, h.b3);
    std::cout << "# restarted from " << rstfile << " at t = " << t << ", cycle = " << cycle << "\n";
  }
  if (!icfile.empty()) {
    chqd::write_restart(g, icfile, t, cycle, h.u, h.b1, h.b2, h.b3);
    std::cout << "# initial state written to " << icfile << "\n";
    return 0;
  }

  chq_mesh *m = nullptr;
  check(chq_mesh_create(&cfg, &m), "mesh");
  struct Guard {
    chq_mesh *m;
    ~Guard() { chq_mesh_destroy(m); }
  } guard{m};
  upload(m, "u0", h.u);
  upload(m, "b1f0", h.b1);
  upload(m, "b2f0", h.b2);
  upload(m, "b3f0", h.b3);
  check(chq_prime(m, t, nullptr), "prime");   // boundaries, con2prim and the first dt

  std::vector<double> u_init, bcc_init;
  if (compute_error) {
    u_init = download(m, "u0");
    bcc_init = download(m, "bcc");
  }

  // ---- outputs ----
  int nvtk = 0, nrst = 0;
  double next_vtk = t, next_hst = t, next_rst = t + dt_rst;
  std::ofstream hst;
  if (dt_hst > 0) {
    hst.open(basename + ".hst", rstfile.empty() ? std::ios::out : std::ios::app);
    if (rstfile.empty()) hst << "# time dt mass mom1 mom2 mom3 etot ekin emag eint divB_max divB_L1\n";
  }
  // VTK and restart dumps go through chq_snapshot: the state is copied on the device behind
  // the queued work and downloaded while the next cycle runs; the files are written from the
  // page-locked buffers once the copy has landed (flush), overlapping the device.
  struct Pinned {
    double *p = nullptr;
    long n = 0;
    ~Pinned() { if (p) chq_host_free(p); }
  };
  // "vtk": the dump's cell data as the device builds it (big-endian float32 planes)
  const char *snap_names[5] = {"vtk", "u0", "b1f0", "b2f0", "b3f0"};
  Pinned snap_buf[5];
  std::vector<std::function<void()>> pending;
  auto buf = [&](int q) -> Pinned & {
    Pinned &b = snap_buf[q];
    if (!b.p) {
      b.n = chq_array_size(m, snap_names[q]);
      void *p = nullptr;
      check(chq_host_alloc(b.n * (long long)sizeof(double), &p), "host buffer");
      b.p = static_cast<double *>(p);
    }
    return b;
  };
  auto as_vec = [](const Pinned &b) { return std::vector<double>(b.p, b.p + b.n); };
  auto flush = [&]() {
    if (pending.empty()) return;
    check(chq_snapshot_wait(m), "snapshot");
    for (auto &w : pending) w();
    pending.clear();
  };
  bool hst_on_device = false;
  auto do_outputs = [&](double dt, bool force, bool final_dump) {
    const double eps = 1e-10 * (tlim > 0 ? tlim : 1.0);
    const bool vtk_now = dt_vtk > 0 && (t >= next_vtk - eps || force);
    const bool rst_now = dt_rst > 0 && (t >= next_rst - eps || final_dump);
    if (vtk_now || rst_now) {
      flush();
      std::vector<int> fields;
      if (vtk_now) fields.push_back(0);
      if (rst_now) fields.insert(fields.end(), {1, 2, 3, 4});
      std::vector<const char *> names;
      std::vector<double *> ptrs;
      std::vector<long> sizes;
      for (int q : fields) {
        Pinned &b = buf(q);
        names.push_back(snap_names[q]);
        ptrs.push_back(b.p);
        sizes.push_back(b.n);
      }
      check(chq_snapshot(m, (int)fields.size(), names.data(), ptrs.data(), sizes.data()), "snapshot");
      const double tw = t;
      const int cw = cycle;
      if (vtk_now) {
        char fn[512];
        std::snprintf(fn, sizeof(fn), "%s.%04d.vtk", basename.c_str(), nvtk++);
        const std::string f = fn;
        pending.push_back([&, f, tw, cw]() {
          chqd::write_vtk(g, reinterpret_cast<const char *>(snap_buf[0].p), f, tw, cw);
        });
        next_vtk += dt_vtk;
      }
      if (rst_now) {
        char fn[512];
        std::snprintf(fn, sizeof(fn), "%s.%04d.rst", basename.c_str(), nrst++);
        const std::string f = fn;
        pending.push_back([&, f, tw, cw]() {
          chqd::write_restart(g, f, tw, cw, as_vec(snap_buf[1]), as_vec(snap_buf[2]), as_vec(snap_buf[3]),
                              as_vec(snap_buf[4]));
        });
        next_rst += dt_rst;
      }
    }
    // with device recording on, the cycles' rows come from chq_history_drain instead
    if (dt_hst > 0 && (force || (!hst_on_device && t >= next_hst - eps))) {
      double hv[10];
      check(chq_history(m, hv, nullptr), "history");
      hst << std::setprecision(12) << t << " " << dt;
      for (double v : hv) hst << " " << v;
      hst << "\n";
      hst.flush();
      next_hst += dt_hst;
    }
  };
  if (rstfile.empty()) do_outputs(0.0, true, false);
  flush();

  // ---- time loop on the device ----
  const bool outputs_on = dt_vtk > 0 || dt_hst > 0 || dt_rst > 0;
  // .hst rows are recorded on the device (the history sums ride on the con2prim of each
  // output cycle), so history alone does not stop the queue after every cycle; VTK and
  // restart dumps still do, since their snapshot is queued from the host
  const bool dumps_on = dt_vtk > 0 || dt_rst > 0;
  const int kHstRing = 256;
  if (dt_hst > 0) {
    const double eps = 1e-10 * (tlim > 0 ? tlim : 1.0);
    check(chq_history_record(m, dt_hst, next_hst, eps, kHstRing), "history record");
    hst_on_device = true;
  }
  std::vector<double> hrows(12 * (size_t)kHstRing);
  auto drain_hst = [&]() {
    if (!hst_on_device) return;
    int nrow = 0, nlost = 0;
    check(chq_history_drain(m, hrows.data(), kHstRing, &nrow, &nlost, &next_hst), "history drain");
    if (nlost > 0) throw std::runtime_error("history ring overflow");
    for (int r = 0; r < nrow; ++r) {
      const double *row = &hrows[12 * (size_t)r];
      hst << std::setprecision(12) << row[0] << " " << row[1];
      for (int q = 2; q < 12; ++q) hst << " " << row[q];
      hst << "\n";
    }
    if (nrow) hst.flush();
  };
  const int cycle0 = cycle;
  {
    double tt, dd, mm;
    int cc;
    check(chq_clock(m, &tt, &cc, &dd, &mm), "clock");   // the device is idle when the clock starts
  }
  auto t0 = std::chrono::steady_clock::now();
  while (true) {
    int chunk = 1;
    if (!dumps_on) {
      chunk = hst_on_device ? kHstRing : 256;
      if (ndiag > 0) chunk = std::min(chunk, ndiag - (cycle % ndiag));
    }
    check(chq_cycles(m, chunk, nullptr), "cycles");
    flush();   // files of the previous output, written while these cycles run
    double tdev = 0.0, dt = 0.0, mdt = 0.0;
    int cdev = 0;
    check(chq_clock(m, &tdev, &cdev, &dt, &mdt), "clock");
    const int advanced = cycle0 + cdev - cycle;
    t = tdev;
    cycle = cycle0 + cdev;
    drain_hst();
    if (advanced == 0) break;
    if (ndiag > 0 && cycle % ndiag == 0)
      std::cout << "cycle=" << cycle << " time=" << std::setprecision(8) << t << " dt=" << dt << "\n";
    do_outputs(dt, false, false);
    if (advanced < chunk) break;
  }
  flush();
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (hst_on_device) {
    check(chq_history_record(m, 0.0, 0.0, 0.0, 0), "history record");
    hst_on_device = false;
  }
  if (outputs_on) do_outputs(0.0, true, true);
  flush();

  const double zones = (double)g.nx1 * g.nx2 * g.nx3;
  const int ncyc = cycle - cycle0;
  std::cout << "# cycles = " << ncyc << ", time = " << t << ", wall = " << wall << " s\n";
  std::cout << "# zone-cycles/second = " << std::scientific << zones * ncyc / wall << "\n";
  long long nfofc = 0, nlimit = 0;
  check(chq_counters(m, &nfofc, &nlimit), "counters");
  if (cfg.fofc) std::cout << "# first-order flux corrections applied: " << nfofc << "\n";
  if (cfg.flux_limiter) std::cout << "# positivity flux limiter activations: " << nlimit << "\n";
  if (cfg.sts) std::cout << "# super-time-stepping stages (total): " << chq_sts_stages(m) << "\n";

  if (compute_error) {
    const std::vector<double> u = download(m, "u0"), b = download(m, "bcc");
    const size_t nc = g.cells();
    double err[9] = {0}, tot = 0;
    for (int k = g.ks; k <= g.ke; ++k)
      for (int j = g.js; j <= g.je; ++j)
        for (int i = g.is; i <= g.ie; ++i) {
          const size_t l = g.c(k, j, i);
          for (int n = 0; n < 6; ++n) err[n] += std::fabs(u[n * nc + l] - u_init[n * nc + l]);
          for (int n = 0; n < 3; ++n) err[6 + n] += std::fabs(b[n * nc + l] - bcc_init[n * nc + l]);
        }
    std::cout << "# L1 errors vs initial state (rho m1 m2 m3 E rho*s B1 B2 B3 | total):\n# ";
    for (double &e : err) {
      e /= zones;
      tot += e;
      std::cout << e << " ";
    }
    std::cout << "| " << tot << "\n";
    std::ofstream ef(basename + "_errors.dat", std::ios::app);
    ef << g.nx1 << " " << g.nx2 << " " << g.nx3 << " " << std::scientific << std::setprecision(8);
    for (double e : err) ef << e << " ";
    ef << tot << "\n";
  }
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  try {
    return run(argc, argv);
  } catch (const std::exception &e) {
    std::cerr << "chasqui: " << e.what() << "\n";
    return 1;
  }
}
