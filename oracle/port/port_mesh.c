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
  long fofc_count, limiter_count, sts_stages;
  /* RKL2 scratch (src/sts.hpp:16-31), allocated on first use: three states, two operator
   * values, each with three face fields */
  double *sy[3], *sm[2], *syb[3][3], *smb[2][3];
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
    free(m->sy[q]);
    for (int r = 0; r < 3; ++r) free(m->syb[q][r]);
  }
  for (q = 0; q < 2; ++q) {
    free(m->sm[q]);
    for (int r = 0; r < 3; ++r) free(m->smb[q][r]);
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

/* Boundaries (src/physics.hpp:354-432) of any state; the three directions in order */
static void bc_on(port_mesh *m, double *u, double *b1, double *b2, double *b3) {
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

void port_boundaries(port_mesh *m, int buf) { bc_on(m, m->u[buf], m->b[buf][0], m->b[buf][1], m->b[buf][2]); }

/* ConsToPrim (src/physics.hpp:437-494) of any state; returns min dt over active cells (huge
 * if none) */
static double c2p_on(port_mesh *m, double *u, const double *b1, const double *b2, const double *b3, int compute_dt) {
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

double port_cons_to_prim(port_mesh *m, int buf, int compute_dt) {
  return c2p_on(m, m->u[buf], m->b[buf][0], m->b[buf][1], m->b[buf][2], compute_dt);
}

/* ---- explicit diffusion (src/diffusion.hpp) ----------------------------------------- */
static int diff_any(const port_mesh *m) { return m->c.nu > 0 || m->c.kappa > 0 || m->c.eta > 0; }

/* edge current density from face fields (src/diffusion.hpp:24-44): J1 at (k-1/2, j-1/2, i),
 * J2 at (k-1/2, j, i-1/2), J3 at (k, j-1/2, i-1/2) */
typedef struct { const double *b1, *b2, *b3; double idx1, idx2, idx3; } curl_ctx;
#define FB(a, k, j, i) (a)[FI(m, 0, k, j, i)]
static double cur1(const port_mesh *m, const curl_ctx *J, int k, int j, int i) {
  double r = 0.0;
  if (m->two_d) r += (FB(J->b3, k, j, i) - FB(J->b3, k, j - 1, i)) * J->idx2;
  if (m->three_d) r -= (FB(J->b2, k, j, i) - FB(J->b2, k - 1, j, i)) * J->idx3;
  return r;
}
static double cur2(const port_mesh *m, const curl_ctx *J, int k, int j, int i) {
  double r = -(FB(J->b3, k, j, i) - FB(J->b3, k, j, i - 1)) * J->idx1;
  if (m->three_d) r += (FB(J->b1, k, j, i) - FB(J->b1, k - 1, j, i)) * J->idx3;
  return r;
}
static double cur3(const port_mesh *m, const curl_ctx *J, int k, int j, int i) {
  double r = (FB(J->b2, k, j, i) - FB(J->b2, k, j, i - 1)) * J->idx1;
  if (m->two_d) r -= (FB(J->b1, k, j, i) - FB(J->b1, k, j - 1, i)) * J->idx2;
  return r;
}
static curl_ctx curl_of(const port_mesh *m, const double *b1, const double *b2, const double *b3) {
  curl_ctx J;
  J.b1 = b1; J.b2 = b2; J.b3 = b3;
  J.idx1 = 1.0 / m->dx1; J.idx2 = 1.0 / m->dx2; J.idx3 = 1.0 / m->dx3;
  return J;
}

/* viscous, conductive and resistive-Poynting fluxes added to face (k, j, i) of direction dir
 * (FaceCtx::Add, src/diffusion.hpp:74-136) */
static void diff_face(port_mesh *m, int dir, const curl_ctx *J, int k, int j, int i) {
  const int t1 = (dir + 1) % 3, t2 = (dir + 2) % 3;
  const int has[3] = {1, m->two_d, m->three_d};
  const int has1 = has[t1], has2 = has[t2];
  const double idx[3] = {1.0 / m->dx1, 1.0 / m->dx2, 1.0 / m->dx3};
  const double idn = idx[dir], idt1 = idx[t1], idt2 = idx[t2];
  const int dk = (dir == 2), dj = (dir == 1), di = (dir == 0);
  const int dk1 = (t1 == 2), dj1 = (t1 == 1), di1 = (t1 == 0), dk2 = (t2 == 2), dj2 = (t2 == 1), di2 = (t2 == 0);
  const int IVU = 1 + dir, IVV = 1 + t1, IVW = 1 + t2;
  const int kL = k - dk, jL = j - dj, iL = i - di;
  const double *w = m->w;
  double *flx = m->f[dir];
#define W(n, kk, jj, ii) w[CI(m, n, kk, jj, ii)]
  if (m->c.nu > 0) {
    const double mu = m->c.nu * 0.5 * (W(IDN, kL, jL, iL) + W(IDN, k, j, i));
    const double dun = (W(IVU, k, j, i) - W(IVU, kL, jL, iL)) * idn;
    const double dvn = (W(IVV, k, j, i) - W(IVV, kL, jL, iL)) * idn;
    const double dwn = (W(IVW, k, j, i) - W(IVW, kL, jL, iL)) * idn;
    double dut1 = 0, dvt1 = 0, dut2 = 0, dwt2 = 0;
    if (has1) {
      dut1 = 0.25 * idt1 * ((W(IVU, k + dk1, j + dj1, i + di1) - W(IVU, k - dk1, j - dj1, i - di1)) +
                            (W(IVU, kL + dk1, jL + dj1, iL + di1) - W(IVU, kL - dk1, jL - dj1, iL - di1)));
      dvt1 = 0.25 * idt1 * ((W(IVV, k + dk1, j + dj1, i + di1) - W(IVV, k - dk1, j - dj1, i - di1)) +
                            (W(IVV, kL + dk1, jL + dj1, iL + di1) - W(IVV, kL - dk1, jL - dj1, iL - di1)));
    }
    if (has2) {
      dut2 = 0.25 * idt2 * ((W(IVU, k + dk2, j + dj2, i + di2) - W(IVU, k - dk2, j - dj2, i - di2)) +
                            (W(IVU, kL + dk2, jL + dj2, iL + di2) - W(IVU, kL - dk2, jL - dj2, iL - di2)));
      dwt2 = 0.25 * idt2 * ((W(IVW, k + dk2, j + dj2, i + di2) - W(IVW, k - dk2, j - dj2, i - di2)) +
                            (W(IVW, kL + dk2, jL + dj2, iL + di2) - W(IVW, kL - dk2, jL - dj2, iL - di2)));
    }
    {
      const double divv = dun + dvt1 + dwt2;
      const double tnn = mu * (2.0 * dun - (2.0 / 3.0) * divv);
      const double tnt1 = mu * (dvn + dut1), tnt2 = mu * (dwn + dut2);
      const double uf = 0.5 * (W(IVU, kL, jL, iL) + W(IVU, k, j, i));
      const double vf = 0.5 * (W(IVV, kL, jL, iL) + W(IVV, k, j, i));
      const double wf = 0.5 * (W(IVW, kL, jL, iL) + W(IVW, k, j, i));
      flx[FI(m, IVU, k, j, i)] -= tnn;
      flx[FI(m, IVV, k, j, i)] -= tnt1;
      flx[FI(m, IVW, k, j, i)] -= tnt2;
      flx[FI(m, IEN, k, j, i)] -= tnn * uf + tnt1 * vf + tnt2 * wf;
    }
  }
  if (m->c.kappa > 0) {
    const double tL = W(4, kL, jL, iL) / W(IDN, kL, jL, iL), tR = W(4, k, j, i) / W(IDN, k, j, i);
    flx[FI(m, IEN, k, j, i)] -= m->c.kappa * (tR - tL) * idn;
  }
  if (m->c.eta > 0) {
    const double eta = m->c.eta;
    double et1, et2;
    if (dir == 0) {
      et1 = eta * 0.5 * (cur2(m, J, k, j, i) + (has2 ? cur2(m, J, k + 1, j, i) : cur2(m, J, k, j, i)));
      et2 = eta * 0.5 * (cur3(m, J, k, j, i) + (has1 ? cur3(m, J, k, j + 1, i) : cur3(m, J, k, j, i)));
    } else if (dir == 1) {
      et1 = eta * 0.5 * (cur3(m, J, k, j, i) + cur3(m, J, k, j, i + 1));
      et2 = eta * 0.5 * (cur1(m, J, k, j, i) + (has1 ? cur1(m, J, k + 1, j, i) : cur1(m, J, k, j, i)));
    } else {
      et1 = eta * 0.5 * (cur1(m, J, k, j, i) + cur1(m, J, k, j + 1, i));
      et2 = eta * 0.5 * (cur2(m, J, k, j, i) + cur2(m, J, k, j, i + 1));
    }
    {
      const double bt1 = 0.5 * (m->bcc[CI(m, t1, kL, jL, iL)] + m->bcc[CI(m, t1, k, j, i)]);
      const double bt2 = 0.5 * (m->bcc[CI(m, t2, kL, jL, iL)] + m->bcc[CI(m, t2, k, j, i)]);
      flx[FI(m, IEN, k, j, i)] += et1 * bt2 - et2 * bt1;
    }
  }
#undef W
}

/* diffusive fluxes on the faces of the active cells of one direction (src/diffusion.hpp:139-146) */
static void diff_fluxes(port_mesh *m, int dir, const double *b1, const double *b2, const double *b3) {
  const curl_ctx J = curl_of(m, b1, b2, b3);
  const int iu = (dir == 0) ? m->ie + 1 : m->ie, ju = (dir == 1) ? m->je + 1 : m->je, ku = (dir == 2) ? m->ke + 1 : m->ke;
  int k;
  if (!diff_any(m)) return;
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= ku; ++k)
    for (int j = m->js; j <= ju; ++j)
      for (int i = m->is; i <= iu; ++i) diff_face(m, dir, &J, k, j, i);
}

/* eta J added to the edge EMFs (src/diffusion.hpp:149-161) */
static void res_emf(port_mesh *m, const double *b1, const double *b2, const double *b3) {
  const curl_ctx J = curl_of(m, b1, b2, b3);
  const int ku = m->three_d ? m->ke + 1 : m->ks + 1, ju = m->two_d ? m->je + 1 : m->js + 1;
  const double eta = m->c.eta;
  int k;
  if (!(eta > 0)) return;
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= ku; ++k)
    for (int j = m->js; j <= ju; ++j)
      for (int i = m->is; i <= m->ie + 1; ++i) {
        if (i <= m->ie) FB(m->e[0], k, j, i) += eta * cur1(m, &J, k, j, i);
        if (j <= m->je || !m->two_d) FB(m->e[1], k, j, i) += eta * cur2(m, &J, k, j, i);
        if (k <= m->ke || !m->three_d) FB(m->e[2], k, j, i) += eta * cur3(m, &J, k, j, i);
      }
}

/* parabolic time-step limit over the active cells (src/diffusion.hpp:164-174) */
static double parabolic_dt(port_mesh *m) {
  const int ndim = 1 + m->two_d + m->three_d;
  double dxmin = m->dx1, rho_min = 1e300, chi, dmax;
  int k;
  if (!diff_any(m)) return 1e300;
  if (m->two_d) dxmin = fmin(dxmin, m->dx2);
  if (m->three_d) dxmin = fmin(dxmin, m->dx3);
#pragma omp parallel for collapse(2) schedule(static) reduction(min : rho_min)
  for (k = m->ks; k <= m->ke; ++k)
    for (int j = m->js; j <= m->je; ++j)
      for (int i = m->is; i <= m->ie; ++i) rho_min = fmin(rho_min, m->w[CI(m, IDN, k, j, i)]);
  chi = (m->c.kappa > 0) ? m->c.kappa * m->gm1 / rho_min : 0.0;
  dmax = fmax(fmax(m->c.nu, m->c.eta), chi);
  return dxmin * dxmin / (2.0 * ndim * dmax);
}

/* ---- source terms (src/srcterms.hpp) ------------------------------------------------- */
/* gravity on the stage output with the stage primitives and beta*dt (srcterms.hpp:20-41) */
static void gravity(port_mesh *m, double *uo, double bdt) {
  const port_cfg *c = &m->c;
  int k;
  if (!(c->grav_uniform || c->grav_point)) return;
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= m->ke; ++k)
    for (int j = m->js; j <= m->je; ++j)
      for (int i = m->is; i <= m->ie; ++i) {
        double a1 = c->g1, a2 = c->g2, a3 = c->g3, d;
        if (c->grav_point) {
          const double dx = (c->x1min + (i - m->is + 0.5) * m->dx1) - c->gx0;
          const double dy = m->two_d ? (c->x2min + (j - m->js + 0.5) * m->dx2) - c->gy0 : 0.0;
          const double dz = m->three_d ? (c->x3min + (k - m->ks + 0.5) * m->dx3) - c->gz0 : 0.0;
          const double r2 = dx * dx + dy * dy + dz * dz + c->rsoft * c->rsoft;
          const double f = -c->gm / (r2 * sqrt(r2));
          a1 += f * dx; a2 += f * dy; a3 += f * dz;
        }
        d = m->w[CI(m, IDN, k, j, i)];
        uo[CI(m, IM1, k, j, i)] += bdt * d * a1;
        uo[CI(m, IM2, k, j, i)] += bdt * d * a2;
        uo[CI(m, IM3, k, j, i)] += bdt * d * a3;
        uo[CI(m, IEN, k, j, i)] += bdt * d * (m->w[CI(m, 1, k, j, i)] * a1 + m->w[CI(m, 2, k, j, i)] * a2 +
                                               m->w[CI(m, 3, k, j, i)] * a3);
      }
}

/* exact power-law cooling of u over dt with the current primitives (srcterms.hpp:51-70) */
static void cooling(port_mesh *m, double *u, double dt) {
  const port_cfg *c = &m->c;
  int k;
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= m->ke; ++k)
    for (int j = m->js; j <= m->je; ++j)
      for (int i = m->is; i <= m->ie; ++i) {
        const double d = m->w[CI(m, IDN, k, j, i)], p = m->w[CI(m, 4, k, j, i)];
        const double t0 = p / d, cc = m->gm1 * d * c->lambda0;
        double t1;
        if (fabs(c->cool_alpha - 1.0) < 1e-12) {
          t1 = t0 * exp(-cc * dt);
        } else {
          const double e = 1.0 - c->cool_alpha;
          const double base = pow(t0, e) + (c->cool_alpha - 1.0) * cc * dt;
          t1 = (base > 0.0) ? pow(base, 1.0 / e) : c->tfloor;
        }
        t1 = fmax(t1, c->tfloor);
        u[CI(m, IEN, k, j, i)] += d * (t1 - t0) / m->gm1;
      }
}

/* ---- RKL2 super-time-stepping (src/sts.hpp) ------------------------------------------ */
static int sts_count(double tau, double dt_par) {   /* Stages, sts.hpp:35-39 */
  const double r = tau / dt_par;
  const int s = (int)ceil(0.5 * (-1.0 + sqrt(9.0 + 16.0 * r)));
  return (s < 2) ? 2 : s;
}
static double sts_bj(int j) { return (j <= 2) ? 1.0 / 3.0 : ((double)j * j + j - 2.0) / (2.0 * j * (j + 1.0)); }

/* M(U, B) = -div F_diff, -curl(eta J) of the state whose primitives are in m->w, face fields
 * b (Operator, sts.hpp:43-96) */
static void sts_op(port_mesh *m, double *const b[3], double *mu, double *const mb[3]) {
  const double idx1 = 1.0 / m->dx1, idx2 = 1.0 / m->dx2, idx3 = 1.0 / m->dx3;
  int q, k;
  for (q = 0; q < 3; ++q) {
    memset(m->f[q], 0, NVAR * m->nface * sizeof(double));
    memset(m->e[q], 0, m->nface * sizeof(double));
  }
  diff_fluxes(m, 0, b[0], b[1], b[2]);
  if (m->two_d) diff_fluxes(m, 1, b[0], b[1], b[2]);
  if (m->three_d) diff_fluxes(m, 2, b[0], b[1], b[2]);
  res_emf(m, b[0], b[1], b[2]);
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= m->ke + 1; ++k)
    for (int j = m->js; j <= m->je + 1; ++j)
      for (int i = m->is; i <= m->ie + 1; ++i) {
        const double *e1 = m->e[0], *e2 = m->e[1], *e3 = m->e[2];
        if (i <= m->ie && j <= m->je && k <= m->ke)
          for (int n = 0; n < NVAR; ++n) {
            double d = (m->f[0][FI(m, n, k, j, i + 1)] - m->f[0][FI(m, n, k, j, i)]) * idx1;
            if (m->two_d) d += (m->f[1][FI(m, n, k, j + 1, i)] - m->f[1][FI(m, n, k, j, i)]) * idx2;
            if (m->three_d) d += (m->f[2][FI(m, n, k + 1, j, i)] - m->f[2][FI(m, n, k, j, i)]) * idx3;
            mu[CI(m, n, k, j, i)] = -d;
          }
        if (j <= m->je && k <= m->ke) {
          double c = 0.0;
          if (m->two_d) c += (FB(e3, k, j + 1, i) - FB(e3, k, j, i)) * idx2;
          if (m->three_d) c -= (FB(e2, k + 1, j, i) - FB(e2, k, j, i)) * idx3;
          FB(mb[0], k, j, i) = -c;
        }
        if (i <= m->ie && k <= m->ke && (m->two_d || j == m->js)) {
          double c = -(FB(e3, k, j, i + 1) - FB(e3, k, j, i)) * idx1;
          if (m->three_d) c += (FB(e1, k + 1, j, i) - FB(e1, k, j, i)) * idx3;
          FB(mb[1], k, j, i) = -c;
          if (!m->two_d) FB(mb[1], k, j + 1, i) = -c;
        }
        if (i <= m->ie && j <= m->je && (m->three_d || k == m->ks)) {
          double c = (FB(e2, k, j, i + 1) - FB(e2, k, j, i)) * idx1;
          if (m->two_d) c -= (FB(e1, k, j + 1, i) - FB(e1, k, j, i)) * idx2;
          FB(mb[2], k, j, i) = -c;
          if (!m->three_d) FB(mb[2], k + 1, j, i) = -c;
        }
      }
}

/* out = ((a x + b y) + c z) + (d p + e q) on the active cells and the update-range faces
 * (Combine / CombineB, sts.hpp:99-114) */
static void sts_comb(port_mesh *m, double *out, double *const ob[3], double a, const double *x, double *const xb[3],
                     double b, const double *y, double *const yb[3], double c, const double *z, double *const zb[3],
                     double d, const double *p, double *const pb[3], double e, const double *q, double *const qb[3]) {
  int k;
#pragma omp parallel for collapse(2) schedule(static)
  for (k = m->ks; k <= m->ke; ++k)
    for (int j = m->js; j <= m->je; ++j)
      for (int i = m->is; i <= m->ie; ++i)
        for (int n = 0; n < NVAR; ++n) {
          const long l = CI(m, n, k, j, i);
          out[l] = ((a * x[l] + b * y[l]) + c * z[l]) + (d * p[l] + e * q[l]);
        }
  for (int f = 0; f < 3; ++f) {
#pragma omp parallel for collapse(2) schedule(static)
    for (k = m->ks; k <= m->ke + 1; ++k)
      for (int j = m->js; j <= m->je + 1; ++j)
        for (int i = m->is; i <= m->ie + 1; ++i) {
          const long l = FI(m, 0, k, j, i);
          ob[f][l] = ((a * xb[f][l] + b * yb[f][l]) + c * zb[f][l]) + (d * pb[f][l] + e * qb[f][l]);
        }
  }
}

/* advance the diffusive terms of (u0, b?f0) over tau (Advance, sts.hpp:118-156); the stage
 * states rotate through three scratch states and u1 / b?f1 as in the reference */
static int sts_advance(port_mesh *m, double tau, double dt_par) {
  const int s = sts_count(tau, dt_par);
  const double w1 = 4.0 / ((double)s * s + s - 2.0);
  const long cb = NVAR * m->ncell * sizeof(double), fb = m->nface * sizeof(double);
  double *y[4], *yb[4][3];
  int a = 0, b = 1, cn = 2, j, q;
  if (!m->sy[0])
    for (q = 0; q < 3; ++q) {
      m->sy[q] = calloc(NVAR * m->ncell, 8);
      for (int r = 0; r < 3; ++r) m->syb[q][r] = calloc(m->nface, 8);
      if (q < 2) {
        m->sm[q] = calloc(NVAR * m->ncell, 8);
        for (int r = 0; r < 3; ++r) m->smb[q][r] = calloc(m->nface, 8);
      }
    }
  for (q = 0; q < 3; ++q) {
    y[q] = m->sy[q];
    for (int r = 0; r < 3; ++r) yb[q][r] = m->syb[q][r];
  }
  y[3] = m->u[1];
  for (q = 0; q < 3; ++q) yb[3][q] = m->b[1][q];
  /* Y0 = (u0, b?f0); M0 = M(Y0) */
  memcpy(y[0], m->u[0], cb);
  for (q = 0; q < 3; ++q) memcpy(yb[0][q], m->b[0][q], fb);
  c2p_on(m, y[0], yb[0][0], yb[0][1], yb[0][2], 0);
  sts_op(m, yb[0], m->sm[0], m->smb[0]);
  {
    const double mt1 = (sts_bj(1) * w1) * tau;
    sts_comb(m, y[1], yb[1], 1.0, y[0], yb[0], 0.0, y[0], yb[0], 0.0, y[0], yb[0], mt1, m->sm[0], m->smb[0], 0.0,
             m->sm[0], m->smb[0]);
  }
  bc_on(m, y[1], yb[1][0], yb[1][1], yb[1][2]);
  /* a = Y_{j-2}, b = Y_{j-1}, cn = Y_j (indices into y); the reference's spare is u1 */
  for (j = 2; j <= s; ++j) {
    const double b_j = sts_bj(j), b_jm1 = sts_bj(j - 1), b_jm2 = sts_bj(j - 2);
    const double mu = (2.0 * j - 1.0) / j * b_j / b_jm1;
    const double nu = -(j - 1.0) / j * b_j / b_jm2;
    const double mut = mu * w1;
    const double gt = -(1.0 - b_jm1) * mut;
    int freed;
    c2p_on(m, y[b], yb[b][0], yb[b][1], yb[b][2], 0);
    sts_op(m, yb[b], m->sm[1], m->smb[1]);
    sts_comb(m, y[cn], yb[cn], mu, y[b], yb[b], nu, y[a], yb[a], 1.0 - mu - nu, y[0], yb[0], mut * tau, m->sm[1],
             m->smb[1], gt * tau, m->sm[0], m->smb[0]);
    bc_on(m, y[cn], yb[cn][0], yb[cn][1], yb[cn][2]);
    freed = (j == 2) ? 3 : a;
    a = b;
    b = cn;
    cn = freed;
  }
  memcpy(m->u[0], y[b], cb);
  for (q = 0; q < 3; ++q) memcpy(m->b[0][q], yb[b][q], fb);
  return s;
}
#undef FB

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

/* RepairFluxes<DIR> (src/fofc.hpp:46-95); the diffusive fluxes are re-added on the repaired
 * faces of active cells when diffusion runs inside the stage (no RKL2) */
void port_fofc_repair(port_mesh *m, int dir, int cur) {
  const int di = (dir == 0), dj = (dir == 1), dk = (dir == 2);
  const int dcr = !m->c.sts && diff_any(m);
  const curl_ctx J = curl_of(m, m->b[cur][0], m->b[cur][1], m->b[cur][2]);
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
        if (dcr) {
          const int af = (dir == 0)   ? (i >= m->is && i <= m->ie + 1 && j >= m->js && j <= m->je && k >= m->ks && k <= m->ke)
                         : (dir == 1) ? (j >= m->js && j <= m->je + 1 && i >= m->is && i <= m->ie && k >= m->ks && k <= m->ke)
                                      : (k >= m->ks && k <= m->ke + 1 && i >= m->is && i <= m->ie && j >= m->js && j <= m->je);
          if (af) diff_face(m, dir, &J, k, j, i);
        }
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

/* Stage (src/main.cpp:46-93): hyperbolic fluxes, in-stage diffusive fluxes (no RKL2), the
 * positivity limiter, corner EMFs plus eta J, the update and gravity, then the FOFC pass */
void port_stage(port_mesh *m, int cur, int out, double g0, double g1, double bdt) {
  const int nd = 1 + m->two_d + m->three_d;
  double *b1c = m->b[cur][0], *b2c = m->b[cur][1], *b3c = m->b[cur][2];
  int d;
  for (d = 0; d < nd; ++d) port_fluxes(m, d, cur);
  if (!m->c.sts)
    for (d = 0; d < nd; ++d) diff_fluxes(m, d, b1c, b2c, b3c);
  if (m->c.flux_limiter)
    for (d = 0; d < nd; ++d) port_limit_fluxes(m, d, bdt);
  port_corner_emf(m);
  if (!m->c.sts) res_emf(m, b1c, b2c, b3c);
  port_update(m, out, g0, g1, bdt);
  gravity(m, m->u[out], bdt);
  if (m->c.fofc) {
    const int nbad = port_fofc_flag(m, out);
    if (nbad > 0) {
      m->fofc_count += nbad;
      for (d = 0; d < nd; ++d) port_fofc_repair(m, d, cur);
      port_corner_emf(m);
      if (!m->c.sts) res_emf(m, b1c, b2c, b3c);
      port_update(m, out, g0, g1, bdt);
      gravity(m, m->u[out], bdt);
    }
  }
  port_boundaries(m, out);
}

/* src/main.cpp:200-202 */
void port_prime(port_mesh *m, double t) {
  port_boundaries(m, 0);
  m->min_dt = port_cons_to_prim(m, 0, 1);
  if (!m->c.sts) m->min_dt = fmin(m->min_dt, parabolic_dt(m));
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

/* src/main.cpp:246-297 without the outputs: the stages, then RKL2 and cooling split after
 * the last stage on (u0, b?f0) */
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
        const int last = (s == m->c.nstage), split = last && (m->c.sts || m->c.cooling);
        const double mdt = port_cons_to_prim(m, out, last && !split);
        if (last && !split) m->min_dt = fmin(mdt, parabolic_dt(m));
      }
    }
    if (m->c.sts) {
      m->sts_stages += sts_advance(m, dt, parabolic_dt(m));
      port_boundaries(m, 0);
    }
    if (m->c.cooling) {
      port_cons_to_prim(m, 0, 0);
      cooling(m, m->u[0], dt);
      port_boundaries(m, 0);
    }
    if (m->c.sts || m->c.cooling) {
      m->min_dt = port_cons_to_prim(m, 0, 1);
      if (!m->c.sts) m->min_dt = fmin(m->min_dt, parabolic_dt(m));
    }
    m->t += dt;
    ++m->cycle;
    ++done;
  }
  return done;
}

long port_sts_stages(port_mesh *m) { return m->sts_stages; }

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
