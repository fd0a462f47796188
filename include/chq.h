/* chasqui_b200 — C ABI of the B200-native per-Runge-Kutta-stage ideal-MHD path.
 *
 * This is the drop-in boundary for Chasqui's stage seam: every function below replaces one
 * call inside the reference's Stage() / time loop (src/main.cpp:46-93, 200-201, 246-297),
 * keeps its argument meaning, and runs hand-written sm_100a CUDA kernels. The mesh keeps the
 * reference's state model: conserved u0/u1 and face fields b?f0/b?f1 as RK double buffers,
 * primitives w, centred B bcc, cell EMF ecc, fluxes f1..f3, face EMFs e<c>x<d>, edge EMFs
 * e1..e3 and the FOFC flag array (src/mesh.hpp:13-63).
 *
 * Conventions
 *   - Every call returns CHQ_OK (0) or a negative CHQ_ERR_* code and never throws; the
 *     message of the last failure on the calling thread is chq_last_error().
 *   - `stream` is a cudaStream_t (NULL = the mesh's own stream). Calls are asynchronous on
 *     that stream unless they return a host value (documented per call).
 *   - Buffer selectors: 0 = u0 / b?f0, 1 = u1 / b?f1 (the reference's cur_is_u1/out_is_u1).
 *   - Host arrays use the reference's packed LayoutRight shapes including ghost zones:
 *     cells (ncomp, nk, nj, ni), faces and edges (ncomp, nk+1, nj+1, ni+1).
 *   - Plain pointers and sizes only; no framework types cross this boundary.
 */
#ifndef CHQ_H_
#define CHQ_H_

#if defined(__GNUC__)
#define CHQ_API __attribute__((visibility("default")))
#else
#define CHQ_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define CHQ_OK 0
#define CHQ_ERR_ARG (-1)     /* invalid argument or configuration */
#define CHQ_ERR_CUDA (-2)    /* CUDA runtime error */
#define CHQ_ERR_NOMEM (-3)   /* device allocation failed */
#define CHQ_ERR_STATE (-4)   /* operation not valid in the mesh's current state */

/* enum values are the reference's (src/defs.hpp:35-37, src/physics.hpp:20) */
enum { CHQ_RECON_DC = 0, CHQ_RECON_PLM = 1, CHQ_RECON_PPM = 2, CHQ_RECON_WENOZ = 3, CHQ_RECON_PPMX = 4 };
enum { CHQ_RS_HLLE = 0, CHQ_RS_HLLD = 1, CHQ_RS_LHLLD = 2 };
enum { CHQ_BC_PERIODIC = 0, CHQ_BC_OUTFLOW = 1, CHQ_BC_REFLECT = 2 };
/* FP64: everything in double. MIXED: primitives, reconstruction, Riemann fluxes and EMFs in
 * float; RK accumulation of u, the face-B CT update, con2prim's pressure recovery and the
 * dt / history reductions stay double. */
enum { CHQ_FP64 = 0, CHQ_MIXED = 1 };

typedef struct chq_config {
  int nx1, nx2, nx3;      /* active cells; nx2 = 1 (1D) and nx3 = 1 (1D/2D) collapse axes */
  int nghost;             /* <= 0: the reference default (3 for ppm/ppmx/wenoz, else 2) */
  double x1min, x1max, x2min, x2max, x3min, x3max;
  int recon, rsolver;
  int integrator;         /* 1 rk1, 2 rk2, 3 rk3 (SSP), 4 SSPRK(4,3) (src/main.cpp:250-268) */
  int bc1, bc2, bc3;
  double gamma, dfloor, pfloor, cfl, de_eta, lhlld_phi;
  int dual_energy, low_mach, flatten, characteristic, fofc, flux_limiter;
  double nu, kappa, eta;  /* explicit diffusion coefficients (0 = off) */
  int sts;                /* RKL2 super-time-stepping of the diffusive terms */
  int precision;          /* CHQ_FP64 or CHQ_MIXED */
  double tlim;            /* end time used by chq_cycles */
  int nlim;               /* < 0: no cycle limit; else stop after nlim cycles (time.nlim) */
  /* gravity source (src/srcterms.hpp:10-41): uniform (g1, g2, g3) and/or a softened point
   * mass gm at (gx0, gy0, gz0), applied after every Update with the stage's beta*dt */
  int gravity_uniform, gravity_point;
  double g1, g2, g3, gm, gx0, gy0, gz0, rsoft;
  /* optically thin cooling Lambda = lambda0 T^alpha, integrated exactly over each step after
   * the hyperbolic update (src/srcterms.hpp:43-71); cool_alpha defaults to 1 */
  int cooling;
  double lambda0, cool_alpha, tfloor;
} chq_config;

typedef struct chq_mesh chq_mesh;

/* ---- configuration and lifetime -------------------------------------------------------- */
/* Fill the reference's defaults (src/main.cpp:116-178): ppm, hlld, rk3, cfl 0.3,
 * gamma 5/3, dfloor 1e-10, pfloor 1e-12, flatten and fofc on, periodic boundaries. */
CHQ_API void chq_config_defaults(chq_config *cfg);
/* Allocate a device mesh with all fields zero (Mesh::Allocate, src/mesh.hpp:37-63). */
CHQ_API int chq_mesh_create(const chq_config *cfg, chq_mesh **out);
CHQ_API int chq_mesh_destroy(chq_mesh *m);
/* dims[0..9] = nx1, nx2, nx3, ng, ni, nj, nk, nstage, two_d, three_d */
CHQ_API int chq_mesh_dims(const chq_mesh *m, int dims[10]);
/* device bytes held by the mesh, and what chq_mesh_create would allocate for a config */
CHQ_API long long chq_mesh_bytes(const chq_mesh *m);
CHQ_API long long chq_config_bytes(const chq_config *cfg);
CHQ_API const char *chq_last_error(void);

/* ---- state transfer in the reference layout ---------------------------------------------
 * name: u0 u1 w bcc ecc b1f0 b2f0 b3f0 b1f1 b2f1 b3f1 f1 f2 f3 e2x1 e3x1 e1x2 e3x2 e1x3
 *       e2x3 e1 e2 e3 flag. n must equal chq_array_size(). Mixed-form float fields are
 *       converted on the host. Both calls synchronise the stream before returning. */
CHQ_API long chq_array_size(const chq_mesh *m, const char *name);
CHQ_API int chq_upload(chq_mesh *m, const char *name, const double *host, long n, void *stream);
CHQ_API int chq_download(chq_mesh *m, const char *name, double *host, long n, void *stream);
/* Output snapshot that does not stall the stepping (no reference counterpart: the reference
 * writes outputs between cycles with a synchronous copy, src/output.hpp, src/restart.hpp).
 * Packs the named fields (any chq_download name) on the device into a snapshot area in the
 * reference layout behind the work queued on the mesh stream, then downloads them on a
 * separate stream into
 * host[q] (n[q] doubles each, the reference layout) while later cycles run. Host buffers
 * from chq_host_alloc make the download asynchronous; pageable ones work but may block.
 * The host buffers must stay untouched until chq_snapshot_wait returns. One snapshot per
 * mesh is in flight; a new one waits for the previous. The snapshot area is allocated on
 * first use and kept with the mesh.
 * The name "vtk" (snapshot only) is the cell data of the reference's VTK dump
 * (src/output.hpp:71-84) built on the device: rho, prs, vx1, vx2, vx3, Bx1, Bx2, Bx3 over the
 * active cells, i fastest, each rounded to float and stored big-endian, 32 bytes per cell
 * (chq_array_size(m, "vtk") = 4 nx1 nx2 nx3 doubles of storage); a file writer emits the
 * bytes unchanged after each SCALARS header. */
CHQ_API int chq_snapshot(chq_mesh *m, int nfields, const char *const *names, double *const *host, const long *n);
CHQ_API int chq_snapshot_wait(chq_mesh *m);

/* ---- stage seam (replaces src/main.cpp:46-93 call by call) ------------------------------ */
/* kernels::FluxesDispatch<dir> (src/physics.hpp:505-514): fluxes and face EMFs of one
 * direction from the primitives and the face field of buffer cur. */
CHQ_API int chq_fluxes(chq_mesh *m, int dir, int cur, void *stream);
/* all active directions in one launch (the fused K1) */
CHQ_API int chq_fluxes_all(chq_mesh *m, int cur, void *stream);
/* kernels::CornerEMF (src/physics.hpp:242-297) */
CHQ_API int chq_corner_emf(chq_mesh *m, void *stream);
/* kernels::Update (src/physics.hpp:307-348): out = g0*(u0,b?f0) + g1*(u1,b?f1) - beta_dt*L */
/* kernels::Update, followed by srcterms::ApplyGravity when gravity is configured (the
 * reference always applies it right after Update, src/main.cpp:75-76) */
CHQ_API int chq_update(chq_mesh *m, int out, double g0, double g1, double beta_dt, void *stream);
/* kernels::Boundaries (src/physics.hpp:354-432) on buffer buf */
CHQ_API int chq_boundaries(chq_mesh *m, int buf, void *stream);
/* kernels::ConsToPrim (src/physics.hpp:437-494) on buffer buf. With compute_dt and a
 * non-NULL min_dt the call synchronises and returns min dx/(|v|+c_f) in *min_dt. */
CHQ_API int chq_cons_to_prim(chq_mesh *m, int buf, int compute_dt, double *min_dt, void *stream);
/* fofc::FlagBadCells (src/fofc.hpp:17-43) on buffer buf; synchronises, count in *nbad */
CHQ_API int chq_fofc_flag(chq_mesh *m, int buf, int *nbad, void *stream);
/* fofc::RepairFluxes<dir> (src/fofc.hpp:46-95) using the flags of the last chq_fofc_flag */
CHQ_API int chq_fofc_repair(chq_mesh *m, int dir, int cur, void *stream);
/* positivity::LimitFluxes<dir> (src/positivity.hpp:25-88); synchronises, adds to *count */
CHQ_API int chq_limit_fluxes(chq_mesh *m, int dir, double beta_dt, long *count, void *stream);
/* one whole RK stage: Stage() of src/main.cpp:46-93 (FOFC decision on the device) */
CHQ_API int chq_stage(chq_mesh *m, int cur, int out, double g0, double g1, double beta_dt, void *stream);

/* ---- problem generators on the device (src/pgen.hpp:269-307 for these problems) ---------
 * Write the initial u0 / b?f0 of every cell and face (ghosts included); call chq_prime next.
 *   CHQ_PGEN_ORSZAG_TANG  params {beta}: pressure beta*B0^2/2, beta <= 0: the reference's
 *                         5/(12 pi) (src/pgen.hpp:94-111)
 *   CHQ_PGEN_CPAW         params {m1, m2, m3, dens, pres, b_par, amp}: circularly polarised
 *                         Alfven wave along 2 pi (m1/L1, m2/L2, m3/L3) of the mesh box
 *   CHQ_PGEN_BLAST        params {pres_in, pres_out, radius, b0, angle_deg, noise_amp, seed}:
 *                         src/pgen.hpp:114-135 with rho = 1 + amp (2U - 1), U from a
 *                         splitmix64 stream of (seed, active-cell index in C order) */
enum { CHQ_PGEN_ORSZAG_TANG = 0, CHQ_PGEN_CPAW = 1, CHQ_PGEN_BLAST = 2 };
CHQ_API int chq_init_problem(chq_mesh *m, int problem, const double *params, int nparams, void *stream);

/* ---- whole cycles with the time step on the device (src/main.cpp:200-201, 246-297) ----- */
/* Boundaries + ConsToPrim(dt) of u0/b?f0 and reset of the clock to t. */
CHQ_API int chq_prime(chq_mesh *m, double t, void *stream);
/* Up to n cycles, stopping at cfg.tlim; no host synchronisation between cycles. */
CHQ_API int chq_cycles(chq_mesh *m, int n, void *stream);
/* Synchronises; returns time, cycle count, last dt and the next cycle's min_dt. */
CHQ_API int chq_clock(chq_mesh *m, double *t, int *cycle, double *dt, double *min_dt);
/* Synchronises; FOFC corrections and limiter activations so far. */
CHQ_API int chq_counters(chq_mesh *m, long long *fofc, long long *limiter);
/* Total RKL2 super-time-stepping stages taken so far (the reference's "super-time-stepping
 * stages (total)" line, src/main.cpp:303); 0 unless diffusion.sts is on. */
CHQ_API long long chq_sts_stages(const chq_mesh *m);
/* output::History (src/output.hpp:91-119) of u0/b?f0: mass mom1 mom2 mom3 etot ekin emag
 * eint divB_max divB_L1 (volume-weighted like the reference). Synchronises. */
CHQ_API int chq_history(chq_mesh *m, double out[10], void *stream);
/* .hst rows recorded on the device, so that history output does not stop the queue of cycles
 * (the reference computes output::History on the host side after each cycle whose time
 * reaches the next output time, src/main.cpp:212-223, src/output.hpp:91-119). With recording
 * on, every cycle of chq_cycles tests on the device whether its end time t satisfies
 * t >= next - eps; if so, the con2prim of the cycle's final state also reduces the history
 * sums (fixed-order, deterministic), the row {t, dt, the ten chq_history values} is appended
 * to a device ring of `capacity` rows, and next advances by dt_hst. capacity 0 turns recording
 * off. Synchronises the mesh stream; drops the captured cycle graph. */
CHQ_API int chq_history_record(chq_mesh *m, double dt_hst, double next, double eps, int capacity);
/* Synchronises the mesh stream and moves up to max_rows recorded rows (12 doubles each, oldest
 * first) into rows; rows that do not fit stay in the ring for the next drain. *n: rows copied;
 * *lost: rows dropped on a full ring since the last drain; *next: the next output time. Any
 * of the three pointers may be null. CHQ_ERR_ARG if recording is off. */
CHQ_API int chq_history_drain(chq_mesh *m, double *rows, int max_rows, int *n, int *lost, double *next);

/* ---- host-buffer job entry point (end-to-end path) ---------------------------------------
 * Upload a reference-layout state (u: 6 x cells, b1/b2/b3: faces), prime it, run n cycles
 * and download the result state into the same host arrays. Returns the cycles done. */
CHQ_API int chq_run_host(chq_mesh *m, double *u, double *b1, double *b2, double *b3, int ncycles, double t0,
                 void *stream);
/* The same job queued without waiting: returns once the upload, priming, cycles and download
 * are queued. The host arrays must be page-locked (chq_host_alloc) and stay untouched until
 * the chq_run_host_wait() that returns this job. Up to two host jobs per mesh are in flight:
 * the result leaves through the snapshot area (chq_snapshot), so the next job's upload
 * overlaps the previous job's download, and jobs on two meshes overlap one job's copies with
 * the other's cycles. */
CHQ_API int chq_run_host_async(chq_mesh *m, double *u, double *b1, double *b2, double *b3, int ncycles, double t0);
/* Waits for the mesh's oldest host job; *cycles (may be NULL) = its cycle count. */
CHQ_API int chq_run_host_wait(chq_mesh *m, int *cycles);

/* ---- device, host memory and timing utilities (no reference counterpart) ----------------- */
/* Make `device` current for this host thread's subsequent chq calls and meshes. */
CHQ_API int chq_set_device(int device);
CHQ_API int chq_device_count(int *count);
/* Page-locked host memory for fast, asynchronous transfers. */
CHQ_API int chq_host_alloc(long long bytes, void **ptr);
CHQ_API int chq_host_free(void *ptr);
/* Record CUDA event `slot` (0..7) on the mesh stream; elapsed device time between two slots
 * (synchronises on the later one). */
CHQ_API int chq_event_record(chq_mesh *m, int slot);
CHQ_API int chq_event_elapsed(chq_mesh *m, int from_slot, int to_slot, float *ms);
/* elapsed device time from slot a of mesh ma to slot b of mesh mb (events of two streams) */
CHQ_API int chq_event_elapsed_between(chq_mesh *ma, int a, chq_mesh *mb, int b, float *ms);
/* Per-kernel CUDA-event timing inside the stage sequence (off by default). Kinds:
 * 0 fluxes (K1), 1 corner EMF (K2), 2 update (K3), 3 FOFC flag, 4 FOFC repair + re-run,
 * 5 boundaries (K4), 6 con2prim + dt (K5), 7 positivity limiter, 8 step control,
 * 9 explicit diffusion (diffusive fluxes, resistive EMF, density minimum), 10 RKL2 super-step. */
#define CHQ_NPROF 11
/* Number of CUDA kernels this mesh has launched so far (including early-exit launches). */
CHQ_API long long chq_kernel_launches(const chq_mesh *m);
CHQ_API int chq_profile(chq_mesh *m, int enable);

/* ---- flux-kernel autotuning (no reference counterpart: the reference has one fixed
 * Kokkos range policy) ---------------------------------------------------------------------
 * Two knobs of the face-flux launch, neither of which changes any result bit:
 *  - march length = faces each thread of the y/z sweeps carries its cell states across
 *    (CHQ_TUNE_LENGTHS). The default is the longest of 16, 8, 4 that keeps a full device of
 *    y/z threads busy (16 from about 128^3 up, 4 for small meshes);
 *  - x-sweep variant = the register cap the x-sweep kernel is compiled for (0: 5 resident
 *    128-thread blocks per SM in FP64 / 10 in FP32; 1: 6 / 12, more resident warps, fewer
 *    registers). Default 0. The tuner varies it in the FP64 form only: there both builds
 *    compute the same bits, while in the mixed form the compiler may contract the FP32
 *    arithmetic of the two builds differently (chq_set_xvariant still selects it there).
 * chq_autotune2 times the flux launch of this mesh's scheme on its current state (call it
 * after chq_prime): every march length with variant 0, then every variant at the best length;
 * it keeps the fastest pair on the mesh and returns it with the ms per launch of each
 * candidate (the arrays may be NULL). The choice is cached for the process per (precision,
 * reconstruction, Riemann solver, characteristic flag, nx1, nx2, nx3); a later mesh with the
 * same key takes it without timing (the arrays then hold -1). Synchronises the mesh stream.
 * chq_autotune is the same search reporting the march length only.
 * chq_batch_autotune does the same for a batch: it times the batched flux launch over all its
 * members (their march lengths and the batch's x variant change together; the batch's tables
 * are rebuilt for each candidate) and caches per (precision, scheme, log2 of the batch's
 * cells, log2 of its member count); a batch of 2^23 cells or more fills the device with its
 * members' own settings and is returned untimed (the arrays hold -1). A batch starts with its
 * members' march lengths and its first member's x variant. */
#define CHQ_TUNE_NLEN 5
#define CHQ_TUNE_LENGTHS {4, 8, 16, 32, 64}
#define CHQ_TUNE_NXVAR 2
CHQ_API int chq_autotune(chq_mesh *m, int *seglen, double ms[CHQ_TUNE_NLEN]);
CHQ_API int chq_autotune2(chq_mesh *m, int *seglen, int *xvar, double ms_len[CHQ_TUNE_NLEN],
                          double ms_xvar[CHQ_TUNE_NXVAR]);
CHQ_API int chq_set_seglen(chq_mesh *m, int seglen);
CHQ_API int chq_get_seglen(const chq_mesh *m);
CHQ_API int chq_set_xvariant(chq_mesh *m, int xvar);
CHQ_API int chq_get_xvariant(const chq_mesh *m);
/* y/z staging of the FP64 streaming-PPM march (2-D and 3-D meshes, PPM without characteristic
 * projection): 0 (default) copies each thread's next stencil values with cp.async, 1 lets one
 * lane per warp fetch the next cell's 32-cell rows with bulk tensor copies (TMA) over the
 * mesh's own arrays. Same results bit for bit. chq_autotune_yz times both on the mesh's state
 * (call after chq_prime and chq_autotune2) and keeps the faster (ms[v] = ms per flux launch
 * of variant v; -1 where the variant does not apply). No counterpart in the reference. */
CHQ_API int chq_set_yzvariant(chq_mesh *m, int yzvar);
CHQ_API int chq_get_yzvariant(const chq_mesh *m);
CHQ_API int chq_autotune_yz(chq_mesh *m, int *yzvar, double ms[2]);
/* Synchronises; totals in ms and launch counts per kind since the last reset. */
CHQ_API int chq_profile_read(chq_mesh *m, double ms[CHQ_NPROF], long long launches[CHQ_NPROF], int reset);

/* ---- batched stepping of many meshes (no reference counterpart: the reference steps one
 * mesh at a time) ---------------------------------------------------------------------------
 * A batch groups primed meshes of one class (same precision, reconstruction, Riemann solver,
 * characteristic flag, integrator, FOFC and limiter switches, and diffusion, RKL2
 * super-time-stepping, cooling and gravity either on in every member or off in every
 * member; coefficients may differ) of any sizes and dimensions and advances all of them with
 * one launch per kernel kind per stage, the blocks of every member in the same grid. Each
 * member keeps its own dt (the parabolic limit included), clock, boundaries and FOFC
 * decisions, and stops at its own tlim, so its results are identical to stepping it alone.
 * With RKL2 the stage count of every member is a host decision each cycle: the batch
 * synchronises once per cycle, then runs super-time-stepping stage j of all members in one
 * launch per kernel kind, members past their own count skipping (no graph replay for such
 * batches).
 * Membership is fixed at creation; meshes must outlive the batch. */
typedef struct chq_batch chq_batch;
CHQ_API int chq_batch_create(chq_mesh *const *meshes, int n, chq_batch **out);
CHQ_API int chq_batch_destroy(chq_batch *b);
/* n cycles of every member (asynchronous on `stream`, NULL = the batch's stream). */
CHQ_API int chq_batch_cycles(chq_batch *b, int n, void *stream);
/* enable: capture one whole cycle as a CUDA graph on first use and replay it. */
CHQ_API int chq_batch_set_graph(chq_batch *b, int enable);
/* Synchronises; per member time, cycle count and done flag (arrays of length n, any NULL). */
CHQ_API int chq_batch_status(chq_batch *b, double *t, int *cycle, int *done);
/* see "flux-kernel autotuning" above; call after the members are primed */
CHQ_API int chq_batch_autotune(chq_batch *b, int *seglen, int *xvar, double ms_len[CHQ_TUNE_NLEN],
                               double ms_xvar[CHQ_TUNE_NXVAR]);
CHQ_API long long chq_batch_kernel_launches(const chq_batch *b);
/* the batch's own stream (cudaStream_t) */
CHQ_API void *chq_batch_stream(chq_batch *b);

/* ---- continuous-batching server (no reference counterpart) -------------------------------
 * Jobs = a mesh configuration (tlim / nlim bound the run), a device problem generator and
 * its parameters. chq_server_step() retires finished jobs (keeping their history sums and
 * freeing their memory), admits queued jobs in submission order while they fit the HBM
 * budget and the slot limit, rebuilds the batch of every class whose membership changed and
 * launches cycles_per_step batched cycles of every class. Each class is split into up to
 * `lanes` batches (default 8) of balanced cell counts, each on its own stream as a replayed
 * CUDA graph, so that the memory-bound kernels of one lane overlap the flux kernel of another.
 * Jobs of 2^21 cells or more run solo on their own mesh stream; the server polls an event
 * behind each solo chunk instead of waiting for it. Jobs with diffusion (explicit or RKL2),
 * cooling or gravity batch with jobs that have the same terms.
 * A job whose final state is not finite is reported FAILED; kernels index only their own
 * job, so it never disturbs the others. Times are seconds on the server clock. */
enum { CHQ_JOB_QUEUED = 0, CHQ_JOB_RUNNING = 1, CHQ_JOB_DONE = 2, CHQ_JOB_FAILED = 3 };
typedef struct chq_job_status {
  int state, cycle;
  double t, t_submit, t_start, t_done;
  long long zone_updates, bytes;
  double history[10];    /* chq_history() of the final state (DONE jobs) */
} chq_job_status;
typedef struct chq_server chq_server;
CHQ_API int chq_server_create(long long hbm_budget_bytes, int max_active, int cycles_per_step, chq_server **out);
CHQ_API int chq_server_submit(chq_server *s, const chq_config *cfg, int problem, const double *params, int nparams,
                              long long *job_id);
/* One scheduling round; returns the number of running + queued jobs (0: idle) or < 0. */
CHQ_API int chq_server_step(chq_server *s);
CHQ_API int chq_server_status(chq_server *s, long long job_id, chq_job_status *st);
/* The device mesh of a RUNNING job (NULL otherwise), e.g. to download its state. */
CHQ_API chq_mesh *chq_server_job_mesh(chq_server *s, long long job_id);
CHQ_API int chq_server_stats(chq_server *s, long long *used_bytes, int *active, int *queued, long long *zone_updates,
                             double *clock);
CHQ_API int chq_server_destroy(chq_server *s);
/* concurrent batches (streams) per class, 1..64; takes effect for newly admitted jobs */
CHQ_API int chq_server_set_lanes(chq_server *s, int lanes);
/* jobs of at least `cells` cells run unbatched on their own streams (default and minimum
 * 2^21; smaller values return CHQ_ERR_ARG); takes effect for newly admitted jobs */
CHQ_API int chq_server_set_solo_cells(chq_server *s, long long cells);
/* solo jobs (those above the solo threshold) running at once, default 1: each fills the
 * device alone; the others wait in the queue while smaller jobs are admitted into the lanes */
CHQ_API int chq_server_set_solo_slots(chq_server *s, int slots);
/* tune every new lane's batch with chq_batch_autotune (1) or keep the members' default launch
 * settings (0, the default: on the ensemble and serving mixes the timing of the candidates
 * cost more than the tuned settings gained); takes effect for batches built afterwards. A lane
 * is timed once, when it is first built; its later rebuilds (members admitted or finished)
 * give the new members the lane's tuned march length and x variant without timing. */
CHQ_API int chq_server_set_autotune(chq_server *s, int enable);

/* ---- z slabs: one mesh decomposed over several GPUs ------------------------------------------
 * No counterpart in the reference, whose mesh is one block on one device (src/mesh.hpp;
 * README.md:163 and :175 list domain decomposition as future work). A mesh of nx3 planes is
 * cut into nslab slabs of nx3 / nslab planes along z, one per rank and device; each slab
 * runs the same stage kernels on its own planes with the whole mesh's cell widths and
 * coordinates, and its z ghost planes on a side that borders another slab come from that
 * slab (periodic z: every side). The results are bitwise those of the whole mesh.
 * chq_slab_create: slab `rank` of `nslab` of the mesh cfg describes (3-D, nx3 a multiple of
 * nslab, at least nghost planes per slab, no RKL2 or cooling). A slab steps only through
 * the calls below: chq_prime, chq_stage, chq_cycles and batches reject it. Its FOFC repair
 * scans every face (it reads the neighbouring slabs' flags, which its cell list lacks).
 * Order of one cycle on every slab, `x` marking where the caller moves data between slabs:
 *   chq_slab_begin
 *   for stage s = 1..nstage:
 *     chq_slab_stage(s, 0)   fluxes .. update, FOFC flags
 *     x  nbad = sum over slabs of nbad; FOFC message (what 1) of the stage's output buffer
 *        out (1 for stages before the last, 0 for the last): pack(1, out, side) -> the
 *        neighbour's unpack(1, out, other side). It carries the boundary plane's flags and
 *        face fields (the repair of a face next to another slab reads both) and crosses
 *        internal slab boundaries only (at the periodic wrap, between the last and the
 *        first slab, the whole mesh's repair sees ghost cells: there pack and unpack of
 *        what 1 do nothing and the message need not be sent)
 *     chq_slab_stage(s, 1)   FOFC repair and re-runs, x/y ghosts, physical z sides
 *     x  state planes of buffer out (what 0) exchanged the same way
 *     chq_slab_stage(s, 2)   con2prim (dt and density minima at the last stage)
 *   x  mdt_bits (and rho_bits with explicit diffusion) = minimum over slabs
 *   chq_slab_end
 * and to prime: chq_slab_prime(t, 0); x state planes of buffer 0; chq_slab_prime(t, 1);
 * x minima; chq_slab_prime(t, 2). The step-control words live in device memory
 * (chq_slab_ctl: int nbad; mdt_bits and rho_bits, non-negative doubles as 64-bit integers,
 * so an integer minimum is the double minimum). A message for `side` packs the planes the
 * neighbour on that side needs; chq_slab_halo_bytes gives its size (8-byte aligned device
 * buffers). info = rank, nslab, lower side is a slab, upper side is a slab, first plane. */
CHQ_API int chq_slab_create(const chq_config *cfg, int nslab, int rank, chq_mesh **out);
CHQ_API int chq_slab_info(const chq_mesh *m, int info[5]);
CHQ_API int chq_slab_halo_bytes(chq_mesh *m, int what, int side, long long *bytes);
CHQ_API int chq_slab_pack(chq_mesh *m, int what, int buf, int side, void *dev, void *stream);
CHQ_API int chq_slab_unpack(chq_mesh *m, int what, int buf, int side, const void *dev, void *stream);
CHQ_API int chq_slab_ctl(chq_mesh *m, int **nbad, unsigned long long **mdt_bits, unsigned long long **rho_bits);
CHQ_API int chq_slab_prime(chq_mesh *m, double t, int part, void *stream);
CHQ_API int chq_slab_begin(chq_mesh *m, void *stream);
CHQ_API int chq_slab_stage(chq_mesh *m, int stage, int part, void *stream);
CHQ_API int chq_slab_end(chq_mesh *m, void *stream);

/* ---- history sums without any device allocation --------------------------------------------
 * No counterpart in the reference. For callers that cannot allocate device memory: an
 * application whose memory belongs to its own pool or framework allocator (for example a
 * Kokkos code that keeps its fields in its own Views), code that must not trigger the
 * implicit device synchronisation of cudaMalloc/cudaFree inside a latency-critical loop,
 * or a monitoring hook that only holds pointers to someone else's state. Same ten values as
 * chq_history() (mass mom1 mom2 mom3 etot ekin emag eint divB_max divB_L1), computed from
 * caller-owned DEVICE arrays in the reference layout: u (6, nk, nj, ni) conserved state and
 * b1/b2/b3 (nk+1, nj+1, ni+1) face fields; the ten results are written to the HOST array
 * `out` and the call synchronises `stream`. Velocities come from u as m / rho, so rho must
 * be positive. Nothing is allocated: block partials live in one fixed static device array
 * of 8192 x 10 doubles (about 640 KiB, held by every device that loads the library until
 * the process exits), which limits meshes to nx3 * ceil(nx2 / 128) <= 8192 (e.g. 1024^3);
 * larger ones return CHQ_ERR_ARG. Every call looks up the array's device address in the
 * current context (no allocation; still right after a cudaDeviceReset or in another context
 * on the same device); the first call on each device also loads the library's device code
 * there (a one-time set-up), so make that first call before any stream capture. All calls
 * share the array: calls that overlap on the GPU (other streams or threads on the same
 * device) race and must be serialised by the caller. One thread block reduces each k-plane x
 * 128-row slab, so a 1-D mesh, or a large 2-D mesh with few rows, runs on few blocks and is
 * slower than chq_history(), with the same results. */
CHQ_API int chq_history_noalloc(int nx1, int nx2, int nx3, int ng, double dx1, double dx2, double dx3,
                                const double *u, const double *b1, const double *b2, const double *b3,
                                double out[10], void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CHQ_H_ */
