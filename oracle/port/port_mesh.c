/* Oracle (test infrastructure): the stage kernels of Chasqui's ideal-MHD path restated in C
 * over the reference's packed arrays, with OpenMP loops. Each routine cites the reference
 * lines it restates; operation order matches them exactly. */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>
#include "port.h"
#include "port_internal.h"

enum { IDN = 0, IM1 = 1, IM2 = 2, IM3 = 3, IEN = 4, IENT = 5, NVAR = 6 };

struct port_mesh {
  port_cfg c;
  int nx1, nx2, nx3, ng, ni, nj, nk, is, ie, js, je, ks, ke, two_d, three_d;
  double dx1, dx2, dx3, gm1;
  long ncell, nface;
  double *u[2], *w, *bcc, *ecc, *b[2][3], *f[3], *et2[3], *et1[3], *e[3];
  int *flag;
  double t, min_dt;
  int cycle;
  long fofc_count, limiter_count;
};

/* cell (n,k,j,i) and face/edge (n,k,j,i) linear indices of the packed layouts */
#define CI(m, n, k, j, i) ((((long)(n) * (m)->nk + (k)) * (m)->nj + (j)) * (m)->ni + (i))
#define FI(m, n, k, j, i) ((((long)(n) * ((m)->nk + 1) + (k)) * ((m)->nj + 1) + (j)) * ((m)->ni + 1) + (i))

void port_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}

/* src/mesh.hpp:37-63 */
port_mesh *port_create(const port_cfg *c) {
  port_mesh *m = (port_mesh *)calloc(1, sizeof(port_mesh));
  int q;
  m->c = *c;
  m->nx1 = c->nx1; m->nx2 = c->nx2; m->nx3 = c->nx3; m->ng = c->ng;
  m->ni = c->nx1 + 2 * c->ng;
  m->nj = (c->nx2 > 1) ? c->nx2 + 2 * c->ng : 1;
  m->nk = (c->nx3 > 1) ? c->nx3 + 2 * c->ng : 1;
  m->is = c->ng; m->ie = c->ng + c->nx1 - 1;
  m->js = (c->nx2 > 1) ? c->ng : 0; m->je = (c->nx2 > 1) ? c->ng + c->nx2 - 1 : 0;
  m->ks = (c->nx3 > 1) ? c->ng : 0; m->ke = (c->nx3 > 1) ? c->ng + c->nx3 - 1 : 0;
  m->two_d = c->nx2 > 1; m->three_d = c->nx3 > 1;
  m->dx1 = (c->x1max - c->x1min) / c->nx1;
  m->dx2 = (c->x2max - c->x2min) / c->nx2;
  m->dx3 = (c->x3max - c->x3min) / c->nx3;
  m->gm1 = c->gamma - 1.0;
  m->ncell = (long)m->nk * m->nj * m->ni;
  m->nface = (long)(m->nk + 1) * (m->nj + 1) * (m->ni + 1);
  m->u[0] = calloc(NVAR * m->ncell, 8); m->u[1] = calloc(NVAR * m->ncell, 8);
  m->w = calloc(NVAR * m->ncell, 8); m->bcc = calloc(3 * m->ncell, 8); m->ecc = calloc(3 * m->ncell, 8);
  for (q = 0; q < 3; ++q) {
    m->b[0][q] = calloc(m->nface, 8); m->b[1][q] = calloc(m->nface, 8);
    m->f[q] = calloc(NVAR * m->nface, 8);
    m->et2[q] = calloc(m->nface, 8); m->et1[q] = calloc(m->nface, 8); m->e[q] = calloc(m->nface, 8);
  }
  m->flag = calloc(m->ncell, sizeof(int));
  return m;
}

void port_destroy(port_mesh *m) {
  int q;
  if (!m) return;
  free(m->u[0]); free(m->u[1]); free(m->w); free(m->bcc); free(m->ecc); free(m->flag);
  for (q = 0; q < 3; ++q) {
    free(m->b[0][q]); free(m->b[1][q]); free(m->f[q]); free(m->et2[q]); free(m->et1[q]); free(m->e[q]);
  }
  free(m);
}

static double *lookup(port_mesh *m, const char *n, long *size) {
  struct { const char *name; double *p; long sz; } tab[] = {
      {"u0", m->u[0], NVAR * m->ncell}, {"u1", m->u[1], NVAR * m->ncell}, {"w", m->w, NVAR * m->ncell},
      {"bcc", m->bcc, 3 * m->ncell}, {"ecc", m->ecc, 3 * m->ncell}, {"b1f0", m->b[0][0], m->nface},
      {"b2f0", m->b[0][1], m->nface}, {"b3f0", m->b[0][2], m->nface}, {"b1f1", m->b[1][0], m->nface},
      {"b2f1", m->b[1][1], m->nface}, {"b3f1", m->b[1][2], m->nface}, {"f1", m->f[0], NVAR * m->nface},
      {"f2", m->f[1], NVAR * m->nface}, {"f3", m->f[2], NVAR * m->nface}, {"e2x1", m->et1[0], m->nface},
      {"e3x1", m->et2[0], m->nface}, {"e1x2", m->et2[1], m->nface}, {"e3x2", m->et1[1], m->nface},
      {"e1x3", m->et1[2], m->nface}, {"e2x3", m->et2[2], m->nface}, {"e1", m->e[0], m->nface},
      {"e2", m->e[1], m->nface}, {"e3", m->e[2], m->nface}};
  unsigned q;
  for (q = 0; q < sizeof(tab) / sizeof(tab[0]); ++q)
    if (!strcmp(tab[q].name, n)) { *size = tab[q].sz; return tab[q].p; }
  *size = strcmp(n, "flag") == 0 ? m->ncell : -1;
  return NULL;
}

long port_size(port_mesh *m, const char *name) {
  long sz;
  lookup(m, name, &sz);
  return sz;
}

int port_get(port_mesh *m, const char *name, double *out, long n) {
  long sz, q;
  double *p = lookup(m, name, &sz);
  if (sz != n) return -1;
  if (p) memcpy(out, p, n * sizeof(double));
  else for (q = 0; q < n; ++q) out[q] = m->flag[q];
  return 0;
}

int port_set(port_mesh *m, const char *name, const double *in, long n) {
  long sz, q;
  double *p = lookup(m, name, &sz);
  if (sz != n) return -1;
  if (p) memcpy(p, in, n * sizeof(double));
  else for (q = 0; q < n; ++q) m->flag[q] = (int)in[q];
  return 0;
}

/* ---- face range of the fluxes of direction d (src/physics.hpp:85-88) ---- */
static void flux_range(const port_mesh *m, int d, int lo[3], int hi[3]) {
  int il = m->is, iu = m->ie, jl = m->js, ju = m->je, kl = m->ks, ku = m->ke;
  if (d == 0) iu = m->ie + 1; else if (m->nx1 > 1) { il = m->is - 1; iu = m->ie + 1; }
  if (d == 1) ju = m->je + 1; else if (m->two_d) { jl = m->js - 1; ju = m->je + 1; }
  if (d == 2) ku = m->ke + 1; else if (m->three_d) { kl = m->ks - 1; ku = m->ke + 1; }
  lo[0] = kl; lo[1] = jl; lo[2] = il;
  hi[0] = ku; hi[1] = ju; hi[2] = iu;
}

/* stencil of cells (k,j,i) + s*(dk,dj,di), s = -3..2, of component n of a cell array
 * (src/physics.hpp:40-57; DC/PLM read s = -2..1 and copy the ends) */
static void stencil(const port_mesh *m, const double *a, int n, int k, int j, int i, int dk, int dj, int di, int wide,
                    double q[6]) {
  int s;
  if (!wide) {
    for (s = 1; s <= 4; ++s) q[s] = a[CI(m, n, k + (s - 3) * dk, j + (s - 3) * dj, i + (s - 3) * di)];
    q[0] = q[1];
    q[5] = q[4];
  } else {
    for (s = 0; s < 6; ++s) q[s] = a[CI(m, n, k + (s - 3) * dk, j + (s - 3) * dj, i + (s - 3) * di)];
  }
}

/* Fluxes<DIR,R,S> (src/physics.hpp:66-226) */
void port_fluxes(port_mesh *m, int dir, int cur) {
  const port_cfg *c = &m->c;
  const int R = c->recon, S = c->rsolver;
  const int di = (dir == 0), dj = (dir == 1), dk = (dir == 2);
  const int IVU = 1 + dir, IVV = 1 + (dir + 1) % 3, IVW = 1 + (dir + 2) % 3;
  const int IBT1 = (dir + 1) % 3, IBT2 = (dir + 2) % 3;
  const int t1 = (dir + 1) % 3, t2 = (dir + 2) % 3;
  const int di1 = (t1 == 0), dj1 = (t1 == 1), dk1 = (t1 == 2), di2 = (t2 == 0), dj2 = (t2 == 1), dk2 = (t2 == 2);
  const int has_t1 = (t1 == 0) || (t1 == 1 && m->two_d) || (t1 == 2 && m->three_d);
  const int has_t2 = (t2 == 0) || (t2 == 1 && m->two_d) || (t2 == 2 && m->three_d);
  const int wide = (R == 2 || R == 3 || R == 4);
  const int flatten = c->flatten && wide;
  const int charac = c->characteristic && R != 0;
  const double *bn = m->b[cur][dir];
  double *flx = m->f[dir], *et2 = m->et2[dir], *et1 = m->et1[dir];
  int lo[3], hi[3], k;
  flux_range(m, dir, lo, hi);
#pragma omp parallel for collapse(2) schedule(static)
  for (k = lo[0]; k <= hi[0]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[2]; i <= hi[2]; ++i) {
        double qs[7][6], wl[7], wr[7], q[6], sl, sr, sld, srd, L[7], Rr[7], f[7];
        const double *src[7] = {m->w, m->w, m->w, m->w, m->w, m->bcc, m->bcc};
        const int comp[7] = {IDN, IVU, IVV, IVW, 4, IBT1, IBT2};
        int n, kk, st;
        const int kL = k - dk, jL = j - dj, iL = i - di;
        for (n = 0; n < 7; ++n) stencil(m, src[n], comp[n], k, j, i, dk, dj, di, wide, qs[n]);
        if (!charac) {
          for (n = 0; n < 7; ++n) port_recon(R, qs[n], &wl[n], &wr[n]);
        } else {
          /* characteristic projection on each side's cell (src/physics.hpp:108-150) */
          double w8[8], Lm[49], Rm[49], cc[6], cl, cr, ch[7], acc;
          int side;
          for (side = 0; side < 2; ++side) {
            const int col = side ? 3 : 2;
            for (n = 0; n < 7; ++n) w8[n] = qs[n][col];
            w8[7] = side ? m->bcc[CI(m, dir, k, j, i)] : m->bcc[CI(m, dir, kL, jL, iL)];
            port_eigen(w8, c->gamma, Lm, Rm);
            for (kk = 0; kk < 7; ++kk) {
              for (st = 0; st < 6; ++st) {
                acc = 0.0;
                for (n = 0; n < 7; ++n) acc += Lm[kk * 7 + n] * qs[n][st];
                cc[st] = acc;
              }
              port_recon(R, cc, &cl, &cr);
              ch[kk] = side ? cr : cl;
            }
            for (n = 0; n < 7; ++n) {
              acc = 0.0;
              for (kk = 0; kk < 7; ++kk) acc += Rm[n * 7 + kk] * ch[kk];
              if (side) wr[n] = acc; else wl[n] = acc;
            }
          }
        }
        stencil(m, m->w, IENT, k, j, i, dk, dj, di, wide, q);
        port_recon(R, q, &sl, &sr);
        sld = q[2];
        srd = q[3];
        if (flatten) {
          const double fL = port_flattening(&qs[4][0], qs[1][1], qs[1][3]);
          const double fR = port_flattening(&qs[4][1], qs[1][2], qs[1][4]);
          if (fL > 0.0) { for (n = 0; n < 7; ++n) wl[n] += fL * (qs[n][2] - wl[n]); sl += fL * (sld - sl); }
          if (fR > 0.0) { for (n = 0; n < 7; ++n) wr[n] += fR * (qs[n][3] - wr[n]); sr += fR * (srd - sr); }
        }
        if (wl[0] <= c->dfloor || wl[4] <= c->pfloor) { for (n = 0; n < 7; ++n) wl[n] = qs[n][2]; sl = sld; }
        if (wr[0] <= c->dfloor || wr[4] <= c->pfloor) { for (n = 0; n < 7; ++n) wr[n] = qs[n][3]; sr = srd; }
        memcpy(L, wl, sizeof(L));
        memcpy(Rr, wr, sizeof(Rr));
        {
          const long lf = FI(m, 0, k, j, i);
          const double b_n = bn[lf];
          if (c->low_mach) {
            const double cl = port_cfast(L, b_n, c->gamma), cr = port_cfast(Rr, b_n, c->gamma);
            const double z = fmin(1.0, fmax(fabs(L[1]) / cl, fabs(Rr[1]) / cr));
            const double um = 0.5 * (L[1] + Rr[1]), ud = 0.5 * (z * (L[1] - Rr[1]));
            L[1] = um + ud;
            Rr[1] = um - ud;
          }
          if (S == 1) {
            port_riemann(1, L, Rr, b_n, c->gamma, 1.0, 1.0, f);
          } else if (S == 2) {
            const double *w = m->w;
            const double cfmax = fmax(port_cfast(L, b_n, c->gamma), port_cfast(Rr, b_n, c->gamma));
            const double du = w[CI(m, IVU, k, j, i)] - w[CI(m, IVU, kL, jL, iL)];
            double dvw = 0.0, ratio, r2, theta, chi, phi;
            if (has_t1) {
              const double d1 = fmin(fmin(w[CI(m, IVV, kL, jL, iL)] - w[CI(m, IVV, kL - dk1, jL - dj1, iL - di1)],
                                          w[CI(m, IVV, kL + dk1, jL + dj1, iL + di1)] - w[CI(m, IVV, kL, jL, iL)]),
                                     fmin(w[CI(m, IVV, k, j, i)] - w[CI(m, IVV, k - dk1, j - dj1, i - di1)],
                                          w[CI(m, IVV, k + dk1, j + dj1, i + di1)] - w[CI(m, IVV, k, j, i)]));
              dvw = fmin(dvw, d1);
            }
            if (has_t2) {
              const double d2 = fmin(fmin(w[CI(m, IVW, kL, jL, iL)] - w[CI(m, IVW, kL - dk2, jL - dj2, iL - di2)],
                                          w[CI(m, IVW, kL + dk2, jL + dj2, iL + di2)] - w[CI(m, IVW, kL, jL, iL)]),
                                     fmin(w[CI(m, IVW, k, j, i)] - w[CI(m, IVW, k - dk2, j - dj2, i - di2)],
                                          w[CI(m, IVW, k + dk2, j + dj2, i + di2)] - w[CI(m, IVW, k, j, i)]));
              dvw = fmin(dvw, d2);
            }
            ratio = fmin(1.0, (-fmin(du, 0.0) + cfmax) / (-dvw + cfmax));
            r2 = ratio * ratio;
            theta = r2 * r2;
            chi = fmin(1.0, fmax(port_cflow(L, b_n), port_cflow(Rr, b_n)) / cfmax);
            phi = (c->lhlld_phi >= 0.0) ? c->lhlld_phi : chi * (2.0 - chi);
            port_riemann(2, L, Rr, b_n, c->gamma, theta, phi, f);
          } else {
            port_riemann(0, L, Rr, b_n, c->gamma, 1.0, 1.0, f);
          }
          flx[FI(m, IDN, k, j, i)] = f[0];
          flx[FI(m, IVU, k, j, i)] = f[1];
          flx[FI(m, IVV, k, j, i)] = f[2];
          flx[FI(m, IVW, k, j, i)] = f[3];
          flx[FI(m, IEN, k, j, i)] = f[4];
          flx[FI(m, IENT, k, j, i)] = (f[0] > 0.0) ? f[0] * sl : (f[0] < 0.0) ? f[0] * sr : 0.5 * (f[0] * (sl + sr));
          et2[lf] = -f[5];
          et1[lf] = f[6];
        }
      }
}

/* src/physics.hpp:233-236 */
static double upwind(double flux, double l, double r) {
  const double tol = 1e-14;
  return (flux > tol) ? l : (flux < -tol) ? r : 0.5 * (l + r);
}

/* CornerEMF (src/physics.hpp:242-297) */
void port_corner_emf(port_mesh *m) {
  double *e1 = m->e[0], *e2 = m->e[1], *e3 = m->e[2];
  const double *e2x1 = m->et1[0], *e3x1 = m->et2[0], *e1x2 = m->et2[1], *e3x2 = m->et1[1], *e1x3 = m->et1[2],
               *e2x3 = m->et2[2], *f1 = m->f[0], *f2 = m->f[1], *f3 = m->f[2], *ecc = m->ecc;
  int k;
#define F(a, k, j, i) (a)[FI(m, 0, k, j, i)]
#define EC(n, k, j, i) ecc[CI(m, n, k, j, i)]
  if (!m->three_d) {
    const int k0 = m->ks;
#pragma omp parallel for schedule(static)
    for (int j = m->js; j <= m->je + 1; ++j)
      for (int i = m->is; i <= m->ie + 1; ++i) {
        F(e1, k0, j, i) = F(e1x2, k0, j, i); F(e1, k0 + 1, j, i) = F(e1x2, k0, j, i);
        F(e2, k0, j, i) = F(e2x1, k0, j, i); F(e2, k0 + 1, j, i) = F(e2x1, k0, j, i);
      }
    if (!m->two_d) {
      for (int i = m->is; i <= m->ie + 1; ++i) { F(e3, k0, m->js, i) = F(e3x1, k0, m->js, i); F(e3, k0, m->js + 1, i) = F(e3x1, k0, m->js, i); }
      return;
    }
  } else {
#pragma omp parallel for collapse(2) schedule(static)
    for (k = m->ks; k <= m->ke + 1; ++k)
      for (int j = m->js; j <= m->je + 1; ++j)
        for (int i = m->is; i <= m->ie; ++i) {
          double l3 = upwind(F(f2, k - 1, j, i), F(e1x3, k, j - 1, i) - EC(0, k - 1, j - 1, i), F(e1x3, k, j, i) - EC(0, k - 1, j, i));
          double r3 = upwind(F(f2, k, j, i), F(e1x3, k, j - 1, i) - EC(0, k, j - 1, i), F(e1x3, k, j, i) - EC(0, k, j, i));
          double l2 = upwind(F(f3, k, j - 1, i), F(e1x2, k - 1, j, i) - EC(0, k - 1, j - 1, i), F(e1x2, k, j, i) - EC(0, k, j - 1, i));
          double r2 = upwind(F(f3, k, j, i), F(e1x2, k - 1, j, i) - EC(0, k - 1, j, i), F(e1x2, k, j, i) - EC(0, k, j, i));
          F(e1, k, j, i) = 0.25 * (((l3 + r3) + (l2 + r2)) + ((F(e1x2, k - 1, j, i) + F(e1x2, k, j, i)) + (F(e1x3, k, j - 1, i) + F(e1x3, k, j, i))));
        }
#pragma omp parallel for collapse(2) schedule(static)
    for (k = m->ks; k <= m->ke + 1; ++k)
      for (int j = m->js; j <= m->je; ++j)
        for (int i = m->is; i <= m->ie + 1; ++i) {
          double l3 = upwind(F(f1, k - 1, j, i), F(e2x3, k, j, i - 1) - EC(1, k - 1, j, i - 1), F(e2x3, k, j, i) - EC(1, k - 1, j, i));
          double r3 = upwind(F(f1, k, j, i), F(e2x3, k, j, i - 1) - EC(1, k, j, i - 1), F(e2x3, k, j, i) - EC(1, k, j, i));
          double l1 = upwind(F(f3, k, j, i - 1), F(e2x1, k - 1, j, i) - EC(1, k - 1, j, i - 1), F(e2x1, k, j, i) - EC(1, k, j, i - 1));
          double r1 = upwind(F(f3, k, j, i), F(e2x1, k - 1, j, i) - EC(1, k - 1, j, i), F(e2x1, k, j, i) - EC(1, k, j, i));
          F(e2, k, j, i) = 0.25 * (((l3 + r3) + (l1 + r1)) + ((F(e2x3, k, j, i - 1) + F(e2x3, k, j, i)) + (F(e2x1, k - 1, j, i) + F(e2x1, k, j, i))));
        }
  }
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= m->ke; ++k)
    for (int j = m->js; j <= m->je + 1; ++j)
      for (int i = m->is; i <= m->ie + 1; ++i) {
        double l2 = upwind(F(f1, k, j - 1, i), F(e3x2, k, j, i - 1) - EC(2, k, j - 1, i - 1), F(e3x2, k, j, i) - EC(2, k, j - 1, i));
        double r2 = upwind(F(f1, k, j, i), F(e3x2, k, j, i - 1) - EC(2, k, j, i - 1), F(e3x2, k, j, i) - EC(2, k, j, i));
        double l1 = upwind(F(f2, k, j, i - 1), F(e3x1, k, j - 1, i) - EC(2, k, j - 1, i - 1), F(e3x1, k, j, i) - EC(2, k, j, i - 1));
        double r1 = upwind(F(f2, k, j, i), F(e3x1, k, j - 1, i) - EC(2, k, j - 1, i), F(e3x1, k, j, i) - EC(2, k, j, i));
        F(e3, k, j, i) = 0.25 * (((l2 + r2) + (l1 + r1)) + ((F(e3x2, k, j, i - 1) + F(e3x2, k, j, i)) + (F(e3x1, k, j - 1, i) + F(e3x1, k, j, i))));
      }
#undef F
#undef EC
}

/* Update (src/physics.hpp:307-348) */
void port_update(port_mesh *m, int out, double g0, double g1, double bdt) {
  const double idx1 = 1.0 / m->dx1, idx2 = 1.0 / m->dx2, idx3 = 1.0 / m->dx3;
  const double *ua = m->u[0], *ub = m->u[1];
  double *uo = m->u[out];
  const double *b1a = m->b[0][0], *b2a = m->b[0][1], *b3a = m->b[0][2], *b1b = m->b[1][0], *b2b = m->b[1][1], *b3b = m->b[1][2];
  double *b1o = m->b[out][0], *b2o = m->b[out][1], *b3o = m->b[out][2];
  const double *e1 = m->e[0], *e2 = m->e[1], *e3 = m->e[2];
  int k;
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= m->ke; ++k)
    for (int j = m->js; j <= m->je; ++j)
      for (int i = m->is; i <= m->ie; ++i)
        for (int n = 0; n < NVAR; ++n) {
          double divf = (m->f[0][FI(m, n, k, j, i + 1)] - m->f[0][FI(m, n, k, j, i)]) * idx1;
          if (m->two_d) divf += (m->f[1][FI(m, n, k, j + 1, i)] - m->f[1][FI(m, n, k, j, i)]) * idx2;
          if (m->three_d) divf += (m->f[2][FI(m, n, k + 1, j, i)] - m->f[2][FI(m, n, k, j, i)]) * idx3;
          uo[CI(m, n, k, j, i)] = g0 * ua[CI(m, n, k, j, i)] + g1 * ub[CI(m, n, k, j, i)] - bdt * divf;
        }
#define F(a, k, j, i) (a)[FI(m, 0, k, j, i)]
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= m->ke + 1; ++k)
    for (int j = m->js; j <= m->je + 1; ++j)
      for (int i = m->is; i <= m->ie + 1; ++i) {
        if (j <= m->je && k <= m->ke) {
          double curl = 0.0;
          if (m->two_d) curl += (F(e3, k, j + 1, i) - F(e3, k, j, i)) * idx2;
          if (m->three_d) curl -= (F(e2, k + 1, j, i) - F(e2, k, j, i)) * idx3;
          F(b1o, k, j, i) = g0 * F(b1a, k, j, i) + g1 * F(b1b, k, j, i) - bdt * curl;
        }
        if (i <= m->ie && k <= m->ke && (m->two_d || j == m->js)) {
          double curl = -(F(e3, k, j, i + 1) - F(e3, k, j, i)) * idx1;
          if (m->three_d) curl += (F(e1, k + 1, j, i) - F(e1, k, j, i)) * idx3;
          F(b2o, k, j, i) = g0 * F(b2a, k, j, i) + g1 * F(b2b, k, j, i) - bdt * curl;
          if (!m->two_d) F(b2o, k, j + 1, i) = F(b2o, k, j, i);
        }
        if (i <= m->ie && j <= m->je && (m->three_d || k == m->ks)) {
          double curl = (F(e2, k, j, i + 1) - F(e2, k, j, i)) * idx1;
          if (m->two_d) curl -= (F(e1, k, j + 1, i) - F(e1, k, j, i)) * idx2;
          F(b3o, k, j, i) = g0 * F(b3a, k, j, i) + g1 * F(b3b, k, j, i) - bdt * curl;
          if (!m->three_d) F(b3o, k + 1, j, i) = F(b3o, k, j, i);
        }
      }
#undef F
}

/* Boundaries (src/physics.hpp:354-432); the three directions in order */
void port_boundaries(port_mesh *m, int buf) {
  double *u = m->u[buf], *b1 = m->b[buf][0], *b2 = m->b[buf][1], *b3 = m->b[buf][2];
  const int ng = m->ng;
  int k;
#define F(a, k, j, i) (a)[FI(m, 0, k, j, i)]
  {
    const int bc = m->c.bc[0];
    const double sgn = (bc == 2) ? -1.0 : 1.0;
#pragma omp parallel for collapse(2) schedule(static)
    for (k = 0; k <= m->nk; ++k)
      for (int j = 0; j <= m->nj; ++j)
        for (int g = 0; g < ng; ++g) {
          const int il = g, ir = m->ie + 1 + g;
          const int sl = (bc == 0) ? il + m->nx1 : (bc == 1) ? m->is : 2 * m->is - 1 - il;
          const int sr = (bc == 0) ? ir - m->nx1 : (bc == 1) ? m->ie : 2 * m->ie + 1 - ir;
          const int fl = g, fr = m->ie + 2 + g;
          if (k < m->nk && j < m->nj) {
            for (int n = 0; n < NVAR; ++n) {
              const double f = (n == IM1) ? sgn : 1.0;
              u[CI(m, n, k, j, il)] = f * u[CI(m, n, k, j, sl)];
              u[CI(m, n, k, j, ir)] = f * u[CI(m, n, k, j, sr)];
            }
            F(b2, k, j, il) = F(b2, k, j, sl); F(b2, k, j, ir) = F(b2, k, j, sr);
            F(b3, k, j, il) = F(b3, k, j, sl); F(b3, k, j, ir) = F(b3, k, j, sr);
          }
          if (bc == 0) { F(b1, k, j, fl) = F(b1, k, j, fl + m->nx1); F(b1, k, j, fr) = F(b1, k, j, fr - m->nx1); }
          else if (bc == 1) { F(b1, k, j, fl) = F(b1, k, j, m->is); F(b1, k, j, fr) = F(b1, k, j, m->ie + 1); }
          else { F(b1, k, j, fl) = -F(b1, k, j, 2 * m->is - fl); F(b1, k, j, fr) = -F(b1, k, j, 2 * (m->ie + 1) - fr); }
          if (bc == 0 && g == 0) F(b1, k, j, m->ie + 1) = F(b1, k, j, m->is);
        }
  }
  if (m->two_d) {
    const int bc = m->c.bc[1];
    const double sgn = (bc == 2) ? -1.0 : 1.0;
#pragma omp parallel for collapse(2) schedule(static)
    for (k = 0; k <= m->nk; ++k)
      for (int g = 0; g < ng; ++g)
        for (int i = 0; i <= m->ni; ++i) {
          const int jl = g, jr = m->je + 1 + g;
          const int sl = (bc == 0) ? jl + m->nx2 : (bc == 1) ? m->js : 2 * m->js - 1 - jl;
          const int sr = (bc == 0) ? jr - m->nx2 : (bc == 1) ? m->je : 2 * m->je + 1 - jr;
          const int fl = g, fr = m->je + 2 + g;
          if (k < m->nk && i < m->ni) {
            for (int n = 0; n < NVAR; ++n) {
              const double f = (n == IM2) ? sgn : 1.0;
              u[CI(m, n, k, jl, i)] = f * u[CI(m, n, k, sl, i)];
              u[CI(m, n, k, jr, i)] = f * u[CI(m, n, k, sr, i)];
            }
            F(b3, k, jl, i) = F(b3, k, sl, i); F(b3, k, jr, i) = F(b3, k, sr, i);
          }
          if (k < m->nk) { F(b1, k, jl, i) = F(b1, k, sl, i); F(b1, k, jr, i) = F(b1, k, sr, i); }
          if (bc == 0) { F(b2, k, fl, i) = F(b2, k, fl + m->nx2, i); F(b2, k, fr, i) = F(b2, k, fr - m->nx2, i); }
          else if (bc == 1) { F(b2, k, fl, i) = F(b2, k, m->js, i); F(b2, k, fr, i) = F(b2, k, m->je + 1, i); }
          else { F(b2, k, fl, i) = -F(b2, k, 2 * m->js - fl, i); F(b2, k, fr, i) = -F(b2, k, 2 * (m->je + 1) - fr, i); }
          if (bc == 0 && g == 0) F(b2, k, m->je + 1, i) = F(b2, k, m->js, i);
        }
  }
  if (m->three_d) {
    const int bc = m->c.bc[2];
    const double sgn = (bc == 2) ? -1.0 : 1.0;
    int g;
#pragma omp parallel for collapse(2) schedule(static)
    for (g = 0; g < ng; ++g)
      for (int j = 0; j <= m->nj; ++j)
        for (int i = 0; i <= m->ni; ++i) {
          const int kl = g, kr = m->ke + 1 + g;
          const int sl = (bc == 0) ? kl + m->nx3 : (bc == 1) ? m->ks : 2 * m->ks - 1 - kl;
          const int sr = (bc == 0) ? kr - m->nx3 : (bc == 1) ? m->ke : 2 * m->ke + 1 - kr;
          const int fl = g, fr = m->ke + 2 + g;
          if (j < m->nj && i < m->ni) {
            for (int n = 0; n < NVAR; ++n) {
              const double f = (n == IM3) ? sgn : 1.0;
              u[CI(m, n, kl, j, i)] = f * u[CI(m, n, sl, j, i)];
              u[CI(m, n, kr, j, i)] = f * u[CI(m, n, sr, j, i)];
            }
          }
          F(b1, kl, j, i) = F(b1, sl, j, i); F(b1, kr, j, i) = F(b1, sr, j, i);
          F(b2, kl, j, i) = F(b2, sl, j, i); F(b2, kr, j, i) = F(b2, sr, j, i);
          if (bc == 0) { F(b3, fl, j, i) = F(b3, fl + m->nx3, j, i); F(b3, fr, j, i) = F(b3, fr - m->nx3, j, i); }
          else if (bc == 1) { F(b3, fl, j, i) = F(b3, m->ks, j, i); F(b3, fr, j, i) = F(b3, m->ke + 1, j, i); }
          else { F(b3, fl, j, i) = -F(b3, 2 * m->ks - fl, j, i); F(b3, fr, j, i) = -F(b3, 2 * (m->ke + 1) - fr, j, i); }
          if (bc == 0 && g == 0) F(b3, m->ke + 1, j, i) = F(b3, m->ks, j, i);
        }
  }
#undef F
}

/* ConsToPrim (src/physics.hpp:437-494); returns min dt over active cells (huge if none) */
double port_cons_to_prim(port_mesh *m, int buf, int compute_dt) {
  double *u = m->u[buf];
  const double *b1 = m->b[buf][0], *b2 = m->b[buf][1], *b3 = m->b[buf][2];
  const port_cfg *c = &m->c;
  double mdt = 1.79769313486231570815e+308;
  int k;
#pragma omp parallel for collapse(2) schedule(static) reduction(min : mdt)
  for (k = 0; k < m->nk; ++k)
    for (int j = 0; j < m->nj; ++j)
      for (int i = 0; i < m->ni; ++i) {
        const long f0 = FI(m, 0, k, j, i);
        const double bx = 0.5 * (b1[f0] + b1[f0 + 1]);
        const double by = m->two_d ? 0.5 * (b2[f0] + b2[FI(m, 0, k, j + 1, i)]) : b2[f0];
        const double bz = m->three_d ? 0.5 * (b3[f0] + b3[FI(m, 0, k + 1, j, i)]) : b3[f0];
        const double d = fmax(u[CI(m, IDN, k, j, i)], c->dfloor), id = 1.0 / d;
        const double vx = u[CI(m, IM1, k, j, i)] * id, vy = u[CI(m, IM2, k, j, i)] * id, vz = u[CI(m, IM3, k, j, i)] * id;
        const double bsq = bx * bx + by * by + bz * bz;
        const double ke = 0.5 * d * (vx * vx + vy * vy + vz * vz);
        const double et = u[CI(m, IEN, k, j, i)], ei = et - ke - 0.5 * bsq;
        double p = m->gm1 * ei, s = u[CI(m, IENT, k, j, i)] * id;
        if (c->dual_energy && ei < c->de_eta * fabs(et)) {
          p = s * pow(d, c->gamma);
          p = fmax(p, c->pfloor);
          u[CI(m, IEN, k, j, i)] = ke + 0.5 * bsq + p / m->gm1;
        } else {
          p = fmax(p, c->pfloor);
          s = p / pow(d, c->gamma);
          u[CI(m, IENT, k, j, i)] = d * s;
        }
        m->w[CI(m, IDN, k, j, i)] = d; m->w[CI(m, 1, k, j, i)] = vx; m->w[CI(m, 2, k, j, i)] = vy;
        m->w[CI(m, 3, k, j, i)] = vz; m->w[CI(m, 4, k, j, i)] = p; m->w[CI(m, IENT, k, j, i)] = s;
        m->bcc[CI(m, 0, k, j, i)] = bx; m->bcc[CI(m, 1, k, j, i)] = by; m->bcc[CI(m, 2, k, j, i)] = bz;
        m->ecc[CI(m, 0, k, j, i)] = vz * by - vy * bz;
        m->ecc[CI(m, 1, k, j, i)] = vx * bz - vz * bx;
        m->ecc[CI(m, 2, k, j, i)] = vy * bx - vx * by;
        if (compute_dt && i >= m->is && i <= m->ie && j >= m->js && j <= m->je && k >= m->ks && k <= m->ke) {
          const double gp = c->gamma * p, a = (gp + bsq) * id;
          double bns[3] = {bx, by, bz}, cf[3], dt;
          for (int q = 0; q < 3; ++q) {
            const double disc = a * a - 4.0 * gp * bns[q] * bns[q] * id * id;
            cf[q] = sqrt(0.5 * (a + sqrt(fmax(disc, 0.0))));
          }
          dt = m->dx1 / (fabs(vx) + cf[0]);
          if (m->two_d) dt = fmin(dt, m->dx2 / (fabs(vy) + cf[1]));
          if (m->three_d) dt = fmin(dt, m->dx3 / (fabs(vz) + cf[2]));
          mdt = fmin(mdt, dt);
        }
      }
  return mdt;
}

/* FlagBadCells (src/fofc.hpp:17-43) */
int port_fofc_flag(port_mesh *m, int buf) {
  const double *u = m->u[buf], *b1 = m->b[buf][0], *b2 = m->b[buf][1], *b3 = m->b[buf][2];
  const port_cfg *c = &m->c;
  int nbad = 0, k;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : nbad)
  for (k = m->ks; k <= m->ke; ++k)
    for (int j = m->js; j <= m->je; ++j)
      for (int i = m->is; i <= m->ie; ++i) {
        const long f0 = FI(m, 0, k, j, i);
        const double bx = 0.5 * (b1[f0] + b1[f0 + 1]);
        const double by = m->two_d ? 0.5 * (b2[f0] + b2[FI(m, 0, k, j + 1, i)]) : b2[f0];
        const double bz = m->three_d ? 0.5 * (b3[f0] + b3[FI(m, 0, k + 1, j, i)]) : b3[f0];
        const double d = u[CI(m, IDN, k, j, i)];
        int bad = (d <= c->dfloor);
        if (!bad) {
          const double m1 = u[CI(m, IM1, k, j, i)], m2 = u[CI(m, IM2, k, j, i)], m3 = u[CI(m, IM3, k, j, i)];
          const double ke = 0.5 * (m1 * m1 + m2 * m2 + m3 * m3) / d;
          const double ei = u[CI(m, IEN, k, j, i)] - ke - 0.5 * (bx * bx + by * by + bz * bz);
          double p = m->gm1 * ei;
          if (c->dual_energy && ei < c->de_eta * fabs(u[CI(m, IEN, k, j, i)]))
            p = (u[CI(m, IENT, k, j, i)] / d) * pow(d, c->gamma);
          bad = (p <= c->pfloor);
        }
        m->flag[CI(m, 0, k, j, i)] = bad;
        nbad += bad;
      }
  return nbad;
}

/* RepairFluxes<DIR> without diffusion (src/fofc.hpp:46-95) */
void port_fofc_repair(port_mesh *m, int dir, int cur) {
  const int di = (dir == 0), dj = (dir == 1), dk = (dir == 2);
  const int IVU = 1 + dir, IVV = 1 + (dir + 1) % 3, IVW = 1 + (dir + 2) % 3, IBT1 = (dir + 1) % 3, IBT2 = (dir + 2) % 3;
  const double *bn = m->b[cur][dir];
  int lo[3], hi[3], k;
  flux_range(m, dir, lo, hi);
#pragma omp parallel for collapse(2) schedule(static)
  for (k = lo[0]; k <= hi[0]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[2]; i <= hi[2]; ++i) {
        const int kL = k - dk, jL = j - dj, iL = i - di;
#define INSIDE(kk, jj, ii) ((ii) >= m->is && (ii) <= m->ie && (jj) >= m->js && (jj) <= m->je && (kk) >= m->ks && (kk) <= m->ke)
        const int fr = INSIDE(k, j, i) && m->flag[CI(m, 0, k, j, i)];
        const int fl = INSIDE(kL, jL, iL) && m->flag[CI(m, 0, kL, jL, iL)];
#undef INSIDE
        double L[7], R[7], f[7];
        const long lf = FI(m, 0, k, j, i);
        if (!(fl || fr)) continue;
        L[0] = m->w[CI(m, IDN, kL, jL, iL)]; L[1] = m->w[CI(m, IVU, kL, jL, iL)]; L[2] = m->w[CI(m, IVV, kL, jL, iL)];
        L[3] = m->w[CI(m, IVW, kL, jL, iL)]; L[4] = m->w[CI(m, 4, kL, jL, iL)];
        L[5] = m->bcc[CI(m, IBT1, kL, jL, iL)]; L[6] = m->bcc[CI(m, IBT2, kL, jL, iL)];
        R[0] = m->w[CI(m, IDN, k, j, i)]; R[1] = m->w[CI(m, IVU, k, j, i)]; R[2] = m->w[CI(m, IVV, k, j, i)];
        R[3] = m->w[CI(m, IVW, k, j, i)]; R[4] = m->w[CI(m, 4, k, j, i)];
        R[5] = m->bcc[CI(m, IBT1, k, j, i)]; R[6] = m->bcc[CI(m, IBT2, k, j, i)];
        port_riemann(0, L, R, bn[lf], m->c.gamma, 1.0, 1.0, f);
        m->f[dir][FI(m, IDN, k, j, i)] = f[0];
        m->f[dir][FI(m, IVU, k, j, i)] = f[1];
        m->f[dir][FI(m, IVV, k, j, i)] = f[2];
        m->f[dir][FI(m, IVW, k, j, i)] = f[3];
        m->f[dir][FI(m, IEN, k, j, i)] = f[4];
        {
          const double sL = m->w[CI(m, IENT, kL, jL, iL)], sR = m->w[CI(m, IENT, k, j, i)];
          m->f[dir][FI(m, IENT, k, j, i)] = (f[0] > 0.0) ? f[0] * sL : (f[0] < 0.0) ? f[0] * sR : 0.5 * (f[0] * (sL + sR));
        }
        m->et2[dir][lf] = -f[5];
        m->et1[dir][lf] = f[6];
      }
}

/* LimitFluxes<DIR> (src/positivity.hpp:25-88) */
static void cell_flux(const double *s, double bn, double sent, double gm1, double gamma, double fc[6], double uc[6],
                      double *cf) {
  double f[7], e, pt;
  port_pflux(s, bn, gm1, &e, &pt, f);
  fc[0] = f[0]; fc[1] = f[1]; fc[2] = f[2]; fc[3] = f[3]; fc[4] = f[4]; fc[5] = f[0] * sent;
  uc[0] = s[0]; uc[1] = s[0] * s[1]; uc[2] = s[0] * s[2]; uc[3] = s[0] * s[3]; uc[4] = e; uc[5] = s[0] * sent;
  *cf = port_cfast(s, bn, gamma);
}

typedef struct { const double *fho, *flf, *uL, *uR, *fL, *fR; double lam2, emL, emR; const port_cfg *c; double gm1; } lim_ctx;

static int lim_ok(const lim_ctx *x, double th) {
  double f[6], a[5], b[5], ea, eb, pa, pb;
  int n;
  for (n = 0; n < 6; ++n) f[n] = x->flf[n] + th * (x->fho[n] - x->flf[n]);
  for (n = 0; n < 5; ++n) { a[n] = x->uL[n] - x->lam2 * (f[n] - x->fL[n]); b[n] = x->uR[n] + x->lam2 * (f[n] - x->fR[n]); }
  if (a[0] < x->c->dfloor || b[0] < x->c->dfloor) return 0;
  ea = a[4] - 0.5 * (a[1] * a[1] + a[2] * a[2] + a[3] * a[3]) / a[0] - x->emL;
  eb = b[4] - 0.5 * (b[1] * b[1] + b[2] * b[2] + b[3] * b[3]) / b[0] - x->emR;
  pa = x->gm1 * ea;
  pb = x->gm1 * eb;
  if (x->c->dual_energy) {
    const double sa = (x->uL[5] - x->lam2 * (f[5] - x->fL[5])) / a[0], sb = (x->uR[5] + x->lam2 * (f[5] - x->fR[5])) / b[0];
    if (ea < x->c->de_eta * fabs(a[4])) pa = sa * pow(a[0], x->c->gamma);
    if (eb < x->c->de_eta * fabs(b[4])) pb = sb * pow(b[0], x->c->gamma);
  }
  return (pa >= x->c->pfloor && pb >= x->c->pfloor);
}

long port_limit_fluxes(port_mesh *m, int dir, double bdt) {
  const int di = (dir == 0), dj = (dir == 1), dk = (dir == 2);
  const int IVU = 1 + dir, IVV = 1 + (dir + 1) % 3, IVW = 1 + (dir + 2) % 3, IBT1 = (dir + 1) % 3, IBT2 = (dir + 2) % 3;
  const int iu = (dir == 0) ? m->ie + 1 : m->ie, ju = (dir == 1) ? m->je + 1 : m->je, ku = (dir == 2) ? m->ke + 1 : m->ke;
  const int ndim = 1 + m->two_d + m->three_d;
  const double dx = (dir == 0) ? m->dx1 : (dir == 1) ? m->dx2 : m->dx3;
  const double lam2 = 2.0 * ndim * bdt / dx;
  const int nv[6] = {IDN, IVU, IVV, IVW, IEN, IENT};
  long cnt = 0;
  int k;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : cnt)
  for (k = m->ks; k <= ku; ++k)
    for (int j = m->js; j <= ju; ++j)
      for (int i = m->is; i <= iu; ++i) {
        const int kL = k - dk, jL = j - dj, iL = i - di;
        double L[7], R[7], fL[6], fR[6], uL[6], uR[6], cfL, cfR, alpha, fho[6], flf[6], bnL, bnR, lo, hi, th;
        lim_ctx x;
        int n, it;
        L[0] = m->w[CI(m, IDN, kL, jL, iL)]; L[1] = m->w[CI(m, IVU, kL, jL, iL)]; L[2] = m->w[CI(m, IVV, kL, jL, iL)];
        L[3] = m->w[CI(m, IVW, kL, jL, iL)]; L[4] = m->w[CI(m, 4, kL, jL, iL)];
        L[5] = m->bcc[CI(m, IBT1, kL, jL, iL)]; L[6] = m->bcc[CI(m, IBT2, kL, jL, iL)];
        R[0] = m->w[CI(m, IDN, k, j, i)]; R[1] = m->w[CI(m, IVU, k, j, i)]; R[2] = m->w[CI(m, IVV, k, j, i)];
        R[3] = m->w[CI(m, IVW, k, j, i)]; R[4] = m->w[CI(m, 4, k, j, i)];
        R[5] = m->bcc[CI(m, IBT1, k, j, i)]; R[6] = m->bcc[CI(m, IBT2, k, j, i)];
        bnL = m->bcc[CI(m, dir, kL, jL, iL)];
        bnR = m->bcc[CI(m, dir, k, j, i)];
        cell_flux(L, bnL, m->w[CI(m, IENT, kL, jL, iL)], m->gm1, m->c.gamma, fL, uL, &cfL);
        cell_flux(R, bnR, m->w[CI(m, IENT, k, j, i)], m->gm1, m->c.gamma, fR, uR, &cfR);
        alpha = fmax(fabs(L[1]) + cfL, fabs(R[1]) + cfR);
        for (n = 0; n < 6; ++n) {
          fho[n] = m->f[dir][FI(m, nv[n], k, j, i)];
          flf[n] = 0.5 * (fL[n] + fR[n]) - 0.5 * (alpha * (uR[n] - uL[n]));
        }
        x.fho = fho; x.flf = flf; x.uL = uL; x.uR = uR; x.fL = fL; x.fR = fR; x.lam2 = lam2;
        x.emL = 0.5 * (bnL * bnL + L[5] * L[5] + L[6] * L[6]);
        x.emR = 0.5 * (bnR * bnR + R[5] * R[5] + R[6] * R[6]);
        x.c = &m->c;
        x.gm1 = m->gm1;
        if (lim_ok(&x, 1.0)) continue;
        lo = 0.0;
        hi = 1.0;
        for (it = 0; it < 12; ++it) {
          const double mid = 0.5 * (lo + hi);
          if (lim_ok(&x, mid)) lo = mid; else hi = mid;
        }
        th = lo;
        for (n = 0; n < 6; ++n) m->f[dir][FI(m, nv[n], k, j, i)] = flf[n] + th * (fho[n] - flf[n]);
        ++cnt;
      }
  m->limiter_count += cnt;
  return cnt;
}

/* Stage (src/main.cpp:46-93) without diffusion and source terms */
void port_stage(port_mesh *m, int cur, int out, double g0, double g1, double bdt) {
  const int nd = 1 + m->two_d + m->three_d;
  int d;
  for (d = 0; d < nd; ++d) port_fluxes(m, d, cur);
  if (m->c.flux_limiter)
    for (d = 0; d < nd; ++d) port_limit_fluxes(m, d, bdt);
  port_corner_emf(m);
  port_update(m, out, g0, g1, bdt);
  if (m->c.fofc) {
    const int nbad = port_fofc_flag(m, out);
    if (nbad > 0) {
      m->fofc_count += nbad;
      for (d = 0; d < nd; ++d) port_fofc_repair(m, d, cur);
      port_corner_emf(m);
      port_update(m, out, g0, g1, bdt);
    }
  }
  port_boundaries(m, out);
}

/* src/main.cpp:200-201 */
void port_prime(port_mesh *m, double t) {
  port_boundaries(m, 0);
  m->min_dt = port_cons_to_prim(m, 0, 1);
  m->t = t;
  m->cycle = 0;
}

/* (g0, g1, beta, cur, out) of stage s (src/main.cpp:250-268) */
static void table(int ns, int s, double *g0, double *g1, double *beta, int *cur, int *out) {
  static const double T3[3][3] = {{1, 0, 1}, {0.75, 0.25, 0.25}, {1.0 / 3.0, 2.0 / 3.0, 2.0 / 3.0}};
  static const double T4[4][3] = {{1, 0, 0.5}, {0, 1, 0.5}, {2.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0}, {0, 1, 0.5}};
  if (ns == 1) { *g0 = 1; *g1 = 0; *beta = 1; *cur = 0; *out = 0; return; }
  if (ns == 2) {
    if (s == 1) { *g0 = 1; *g1 = 0; *beta = 1; *cur = 0; *out = 1; }
    else { *g0 = 0.5; *g1 = 0.5; *beta = 0.5; *cur = 1; *out = 0; }
    return;
  }
  if (ns == 3) { *g0 = T3[s - 1][0]; *g1 = T3[s - 1][1]; *beta = T3[s - 1][2]; }
  else { *g0 = T4[s - 1][0]; *g1 = T4[s - 1][1]; *beta = T4[s - 1][2]; }
  *cur = (s == 1) ? 0 : 1;
  *out = (s == ns) ? 0 : 1;
}

/* src/main.cpp:246-297 (no outputs, no operator-split terms) */
int port_cycles(port_mesh *m, int n) {
  int c, done = 0;
  for (c = 0; c < n; ++c) {
    double dt;
    int s;
    if (!(m->t < m->c.tlim)) break;
    dt = m->c.cfl * m->min_dt;
    if (m->t + dt > m->c.tlim) dt = m->c.tlim - m->t;
    for (s = 1; s <= m->c.nstage; ++s) {
      double g0, g1, beta;
      int cur, out;
      table(m->c.nstage, s, &g0, &g1, &beta, &cur, &out);
      port_stage(m, cur, out, g0, g1, beta * dt);
      {
        const double mdt = port_cons_to_prim(m, out, s == m->c.nstage);
        if (s == m->c.nstage) m->min_dt = mdt;
      }
    }
    m->t += dt;
    ++m->cycle;
    ++done;
  }
  return done;
}

void port_clock(port_mesh *m, double *t, int *cycle, double *min_dt, long *fofc_count) {
  if (t) *t = m->t;
  if (cycle) *cycle = m->cycle;
  if (min_dt) *min_dt = m->min_dt;
  if (fofc_count) *fofc_count = m->fofc_count;
}

/* History (src/output.hpp:91-119) of u0 / b?f0 with the current primitives */
void port_history(port_mesh *m, double out[10]) {
  const double idx1 = 1.0 / m->dx1, idx2 = 1.0 / m->dx2, idx3 = 1.0 / m->dx3;
  const double *u = m->u[0], *b1 = m->b[0][0], *b2 = m->b[0][1], *b3 = m->b[0][2];
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0, s6 = 0, s7 = 0, dbm = 0, dbs = 0, vol;
  int k;
#pragma omp parallel for collapse(2) schedule(static) reduction(+ : s0, s1, s2, s3, s4, s5, s6, s7, dbs) reduction(max : dbm)
  for (k = m->ks; k <= m->ke; ++k)
    for (int j = m->js; j <= m->je; ++j)
      for (int i = m->is; i <= m->ie; ++i) {
        const double d = m->w[CI(m, 0, k, j, i)];
        const double v2 = m->w[CI(m, 1, k, j, i)] * m->w[CI(m, 1, k, j, i)] + m->w[CI(m, 2, k, j, i)] * m->w[CI(m, 2, k, j, i)] +
                          m->w[CI(m, 3, k, j, i)] * m->w[CI(m, 3, k, j, i)];
        const double b2c = m->bcc[CI(m, 0, k, j, i)] * m->bcc[CI(m, 0, k, j, i)] + m->bcc[CI(m, 1, k, j, i)] * m->bcc[CI(m, 1, k, j, i)] +
                           m->bcc[CI(m, 2, k, j, i)] * m->bcc[CI(m, 2, k, j, i)];
        double db;
        s0 += u[CI(m, 0, k, j, i)]; s1 += u[CI(m, 1, k, j, i)]; s2 += u[CI(m, 2, k, j, i)]; s3 += u[CI(m, 3, k, j, i)];
        s4 += u[CI(m, 4, k, j, i)];
        s5 += 0.5 * d * v2;
        s6 += 0.5 * b2c;
        s7 += u[CI(m, 4, k, j, i)] - 0.5 * d * v2 - 0.5 * b2c;
        db = (b1[FI(m, 0, k, j, i + 1)] - b1[FI(m, 0, k, j, i)]) * idx1;
        if (m->two_d) db += (b2[FI(m, 0, k, j + 1, i)] - b2[FI(m, 0, k, j, i)]) * idx2;
        if (m->three_d) db += (b3[FI(m, 0, k + 1, j, i)] - b3[FI(m, 0, k, j, i)]) * idx3;
        dbm = fmax(dbm, fabs(db));
        dbs += fabs(db);
      }
  vol = m->dx1 * (m->two_d ? m->dx2 : 1.0) * (m->three_d ? m->dx3 : 1.0);
  out[0] = s0 * vol; out[1] = s1 * vol; out[2] = s2 * vol; out[3] = s3 * vol; out[4] = s4 * vol;
  out[5] = s5 * vol; out[6] = s6 * vol; out[7] = s7 * vol; out[8] = dbm;
  out[9] = dbs / ((double)m->nx1 * m->nx2 * m->nx3);
}
