/* Oracle (test infrastructure): a plain-C restatement of Chasqui's per-RK-stage MHD path
 * (ideal MHD, explicit diffusion, RKL2, gravity, cooling), written per face like the
 * published algorithm, on the reference's packed
 * LayoutRight arrays (cells (ncomp,nk,nj,ni), faces/edges (ncomp,nk+1,nj+1,ni+1)).
 * Every function cites the reference file:line it restates. It is pinned against the
 * reference's own kernels (oracle/_ref) by tests/test_oracle_port.py. The product never
 * links it. Build: make -C oracle (-> oracle/_port/libchqport.so), -ffp-contract=off. */
#ifndef CHQ_ORACLE_PORT_H_
#define CHQ_ORACLE_PORT_H_

typedef struct port_cfg {
  int nx1, nx2, nx3, ng;
  double x1min, x1max, x2min, x2max, x3min, x3max;
  int recon, rsolver, nstage;  /* reference enum values; nstage 1..4 */
  int bc[3];
  double gamma, dfloor, pfloor, cfl, de_eta, lhlld_phi, tlim;
  int dual_energy, low_mach, flatten, characteristic, fofc, flux_limiter;
  /* explicit diffusion / RKL2 (src/diffusion.hpp, src/sts.hpp) and source terms
   * (src/srcterms.hpp); zero = off */
  double nu, kappa, eta;
  int sts;
  int grav_uniform, grav_point;
  double g1, g2, g3, gm, gx0, gy0, gz0, rsoft;
  int cooling;
  double lambda0, cool_alpha, tfloor;
} port_cfg;

typedef struct port_mesh port_mesh;

port_mesh *port_create(const port_cfg *c);
void port_destroy(port_mesh *m);
/* named array in the reference layout (u0 u1 w bcc ecc b1f0.. b3f1 f1 f2 f3 e2x1 e3x1 e1x2 e3x2
 * e1x3 e2x3 e1 e2 e3 flag); flag is returned as doubles through port_get/port_set */
long port_size(port_mesh *m, const char *name);
int port_get(port_mesh *m, const char *name, double *out, long n);
int port_set(port_mesh *m, const char *name, const double *in, long n);

void port_fluxes(port_mesh *m, int dir, int cur);
void port_corner_emf(port_mesh *m);
void port_update(port_mesh *m, int out, double g0, double g1, double beta_dt);
void port_boundaries(port_mesh *m, int buf);
double port_cons_to_prim(port_mesh *m, int buf, int compute_dt);
int port_fofc_flag(port_mesh *m, int buf);
void port_fofc_repair(port_mesh *m, int dir, int cur);
long port_limit_fluxes(port_mesh *m, int dir, double beta_dt);
void port_stage(port_mesh *m, int cur, int out, double g0, double g1, double beta_dt);
void port_prime(port_mesh *m, double t);
int port_cycles(port_mesh *m, int n);
void port_clock(port_mesh *m, double *t, int *cycle, double *min_dt, long *fofc_count);
void port_history(port_mesh *m, double out[10]);
long port_sts_stages(port_mesh *m);   /* RKL2 stages taken so far */

/* point functions */
void port_recon(int scheme, const double q[6], double *ql, double *qr);
double port_flattening(const double p[5], double um1, double up1);
void port_riemann(int solver, const double L[7], const double R[7], double bn, double gamma, double theta,
                  double phi, double f[7]);
void port_eigen(const double w8[8], double gamma, double Lm[49], double Rm[49]);
void port_set_threads(int n);

#endif
