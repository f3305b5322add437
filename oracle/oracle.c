/*
 * CPU oracle: a plain-C restatement of sputniPIC's particle mover and
 * particle-to-grid deposition, written from the reference's behaviour.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library. Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it.
 *
 * Parity pin: tests/test_oracle_golden.py checks this restatement against
 * fixtures produced by the reference's own sources (tests/golden/, made by
 * tests/golden/make_golden.py through oracle/_ref). In the float build the
 * particle outputs must be bit-identical to the reference; moments too, since
 * both accumulate serially in the same particle order.
 *
 * Build: -DORACLE_FP64 gives the FP64 oracle (every FP type double), as if the
 * reference's include/PrecisionTypes.h:6-10 typedefs were double. Compiled
 * with -ffp-contract=off, as the baseline x86-64 reference build has no FMA.
 *
 * Arithmetic follows the C promotion rules of the reference expressions:
 * where the reference mixes a float with a double member or literal the
 * operation happens in double and is rounded on assignment.
 */
#include "oracle_api.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifdef ORACLE_FP64
typedef double fpp; /* FPpart   */
typedef double fpf; /* FPfield  */
typedef double fpi; /* FPinterp */
#else
typedef float fpp;
typedef float fpf;
typedef float fpi;
#endif

/* Grid geometry, as setGrid computes it (src/Grid.cpp:5-62). The node
 * coordinate arrays XN/YN/ZN only depend on their own axis index, so the
 * oracle keeps one 1D array per axis. */
typedef struct og_grid {
  int nxc, nyc, nzc; /* guard cells included */
  int nxn, nyn, nzn;
  double dx, dy, dz;
  fpf invdx, invdy, invdz, invVOL;
  double xStart, yStart, zStart;
  double Lx, Ly, Lz;
  fpf *xn, *yn, *zn;
} og_grid;

static int og_make_grid(const orc_setup *s, og_grid *g) {
  /* src/Grid.cpp:9-15: two guard cells, one extra node */
  g->nxc = s->nxc + 2;
  g->nyc = s->nyc + 2;
  g->nzc = s->nzc + 2;
  g->nxn = g->nxc + 1;
  g->nyn = g->nyc + 1;
  g->nzn = g->nzc + 1;
  /* src/Grid.cpp:19-27: spacing in double; inverses rounded to FPfield */
  g->dx = s->Lx / s->nxc;
  g->dy = s->Ly / s->nyc;
  g->dz = s->Lz / s->nzc;
  g->invVOL = (fpf)((fpf)1.0 / (g->dx * g->dy * g->dz));
  g->invdx = (fpf)((fpf)1.0 / g->dx);
  g->invdy = (fpf)((fpf)1.0 / g->dy);
  g->invdz = (fpf)((fpf)1.0 / g->dz);
  /* src/Grid.cpp:30-41 */
  g->xStart = 0.0;
  g->yStart = 0.0;
  g->zStart = 0.0;
  g->Lx = s->Lx;
  g->Ly = s->Ly;
  g->Lz = s->Lz;
  g->xn = (fpf *)malloc(sizeof(fpf) * g->nxn);
  g->yn = (fpf *)malloc(sizeof(fpf) * g->nyn);
  g->zn = (fpf *)malloc(sizeof(fpf) * g->nzn);
  if (!g->xn || !g->yn || !g->zn) return -1;
  /* src/Grid.cpp:53-61: node i sits at (i-1)*dx */
  for (int i = 0; i < g->nxn; i++) g->xn[i] = (fpf)(g->xStart + (i - 1) * g->dx);
  for (int j = 0; j < g->nyn; j++) g->yn[j] = (fpf)(g->yStart + (j - 1) * g->dy);
  for (int k = 0; k < g->nzn; k++) g->zn[k] = (fpf)(g->zStart + (k - 1) * g->dz);
  return 0;
}

static void og_free_grid(og_grid *g) {
  free(g->xn);
  free(g->yn);
  free(g->zn);
}

static inline long og_node(const og_grid *g, int i, int j, int k) {
  return ((long)i * g->nyn + j) * g->nzn + k;
}

/* Time-step constants of mover_PC (src/Mover.cpp:11-12). dt_sub_cycling is
 * the float dt divided in double by n_sub_cycles, then rounded. */
typedef struct og_push {
  fpp dt_sub_cycling, dto2, qomdt2;
} og_push;

static og_push og_push_consts(const orc_setup *s, double qom_in) {
  og_push p;
  fpp qom = (fpp)qom_in; /* part->qom = (FPpart)param->qom[is], src/Particles.cpp:25 */
  p.dt_sub_cycling = (fpp)((double)(fpp)s->dt / ((double)s->n_sub_cycles));
  p.dto2 = (fpp)(.5 * p.dt_sub_cycling);
  p.qomdt2 = (fpp)((fpp)(qom * p.dto2) / s->c);
  return p;
}

/* One particle of mover_PC, src/Mover.cpp:33-157. The order of every sum
 * and product is the reference's. */
static void og_move_one(const og_grid *g, const orc_setup *s, const og_push *pc,
                        const fpf *const *F, fpp *x, fpp *y, fpp *z, fpp *u,
                        fpp *v, fpp *w, int bc_v) {
  const fpp qomdt2 = pc->qomdt2;
  fpp xptilde = *x, yptilde = *y, zptilde = *z;
  fpp uptilde = 0, vptilde = 0, wptilde = 0;
  for (int it = 0; it < s->niter; it++) {
    /* cell index: truncation of a double product (:39-41) */
    int ix = 2 + (int)(((double)*x - g->xStart) * (double)g->invdx);
    int iy = 2 + (int)(((double)*y - g->yStart) * (double)g->invdy);
    int iz = 2 + (int)(((double)*z - g->zStart) * (double)g->invdz);
    fpf xi[2], eta[2], zeta[2], wgt[2][2][2];
    xi[0] = *x - g->xn[ix - 1];
    eta[0] = *y - g->yn[iy - 1];
    zeta[0] = *z - g->zn[iz - 1];
    xi[1] = g->xn[ix] - *x;
    eta[1] = g->yn[iy] - *y;
    zeta[1] = g->zn[iz] - *z;
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++)
        for (int c = 0; c < 2; c++) wgt[a][b][c] = xi[a] * eta[b] * zeta[c] * g->invVOL;
    fpf El[6] = {0, 0, 0, 0, 0, 0};
    for (int a = 0; a < 2; a++)
      for (int b = 0; b < 2; b++)
        for (int c = 0; c < 2; c++) {
          long n = og_node(g, ix - a, iy - b, iz - c);
          for (int f = 0; f < 6; f++) El[f] += wgt[a][b][c] * F[f][n];
        }
    const fpf Exl = El[0], Eyl = El[1], Ezl = El[2];
    const fpf Bxl = El[3], Byl = El[4], Bzl = El[5];
    /* implicit velocity solve (:70-83); denom is computed in double */
    fpp omdtsq = qomdt2 * qomdt2 * (Bxl * Bxl + Byl * Byl + Bzl * Bzl);
    fpp denom = (fpp)(1.0 / (1.0 + (double)omdtsq));
    fpp ut = *u + qomdt2 * Exl;
    fpp vt = *v + qomdt2 * Eyl;
    fpp wt = *w + qomdt2 * Ezl;
    fpp udotb = ut * Bxl + vt * Byl + wt * Bzl;
    uptilde = (ut + qomdt2 * (vt * Bzl - wt * Byl + qomdt2 * udotb * Bxl)) * denom;
    vptilde = (vt + qomdt2 * (wt * Bxl - ut * Bzl + qomdt2 * udotb * Byl)) * denom;
    wptilde = (wt + qomdt2 * (ut * Byl - vt * Bxl + qomdt2 * udotb * Bzl)) * denom;
    /* half-step position (:85-87) */
    *x = xptilde + uptilde * pc->dto2;
    *y = yptilde + vptilde * pc->dto2;
    *z = zptilde + wptilde * pc->dto2;
  }
  /* final velocity in double, position in FPpart (:91-96) */
  *u = (fpp)(2.0 * (double)uptilde - (double)*u);
  *v = (fpp)(2.0 * (double)vptilde - (double)*v);
  *w = (fpp)(2.0 * (double)wptilde - (double)*w);
  *x = xptilde + uptilde * pc->dt_sub_cycling;
  *y = yptilde + vptilde * pc->dt_sub_cycling;
  *z = zptilde + wptilde * pc->dt_sub_cycling;

  /* particle BC per axis (:103-157): an "above L" test, then a separate
   * "below 0" test; the field periodicity flags choose periodic or mirror */
  fpp *pos[3] = {x, y, z};
  fpp *vel[3] = {u, v, w};
  const double L[3] = {g->Lx, g->Ly, g->Lz};
  if (bc_v) {
    /* mover_PC_V (src/Mover.cpp:296-379): per axis, periodic shifts; else the
     * position is mirrored first, then the velocity is flipped only where
     * the mirrored position is still outside [0, L] */
    for (int d = 0; d < 3; d++) {
      if (s->periodic[d]) {
        if ((double)*pos[d] > L[d]) *pos[d] = (fpp)((double)*pos[d] - L[d]);
        if (*pos[d] < 0) *pos[d] = (fpp)((double)*pos[d] + L[d]);
      } else {
        if ((double)*pos[d] > L[d]) *pos[d] = (fpp)(2 * L[d] - (double)*pos[d]);
        if (*pos[d] < 0) *pos[d] = -*pos[d];
        if ((double)*pos[d] > L[d]) *vel[d] = -*vel[d];
        if (*pos[d] < 0) *vel[d] = -*vel[d];
      }
    }
    return;
  }
  for (int d = 0; d < 3; d++) {
    if ((double)*pos[d] > L[d]) {
      if (s->periodic[d]) {
        *pos[d] = (fpp)((double)*pos[d] - L[d]);
      } else {
        *vel[d] = -*vel[d];
        *pos[d] = (fpp)(2 * L[d] - (double)*pos[d]);
      }
    }
    if (*pos[d] < 0) {
      if (s->periodic[d]) {
        *pos[d] = (fpp)((double)*pos[d] + L[d]);
      } else {
        *vel[d] = -*vel[d];
        *pos[d] = -*pos[d];
      }
    }
  }
}

/* Deposit of one particle, interpP2G's loop body (src/Mover.cpp:399-570). */
static void og_deposit_one(const og_grid *g, fpp x, fpp y, fpp z, fpp u, fpp v,
                           fpp w, fpi q, fpi *const *mom) {
  /* cell index: floor of a double product (:399-401) */
  int ix = 2 + (int)floor(((double)x - g->xStart) * (double)g->invdx);
  int iy = 2 + (int)floor(((double)y - g->yStart) * (double)g->invdy);
  int iz = 2 + (int)floor(((double)z - g->zStart) * (double)g->invdz);
  fpp xi[2], eta[2], zeta[2], wgt[2][2][2];
  xi[0] = x - g->xn[ix - 1];
  eta[0] = y - g->yn[iy - 1];
  zeta[0] = z - g->zn[iz - 1];
  xi[1] = g->xn[ix] - x;
  eta[1] = g->yn[iy] - y;
  zeta[1] = g->zn[iz] - z;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) wgt[a][b][c] = q * xi[a] * eta[b] * zeta[c] * g->invVOL;
  /* moment factors: 1, u, v, w, uu, uv, uw, vv, vw, ww (:469-570) */
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 2; b++)
      for (int c = 0; c < 2; c++) {
        const long n = og_node(g, ix - a, iy - b, iz - c);
        const fpp wv = wgt[a][b][c];
        mom[0][n] += wv * g->invVOL;
        mom[1][n] += (fpp)(u * wv) * g->invVOL;
        mom[2][n] += (fpp)(v * wv) * g->invVOL;
        mom[3][n] += (fpp)(w * wv) * g->invVOL;
        mom[4][n] += (fpp)(u * u * wv) * g->invVOL;
        mom[5][n] += (fpp)(u * v * wv) * g->invVOL;
        mom[6][n] += (fpp)(u * w * wv) * g->invVOL;
        mom[7][n] += (fpp)(v * v * wv) * g->invVOL;
        mom[8][n] += (fpp)(v * w * wv) * g->invVOL;
        mom[9][n] += (fpp)(w * w * wv) * g->invVOL;
      }
}

/* The reference adds the ten moments one moment at a time over the eight
 * nodes (src/Mover.cpp:466-570). Each node receives exactly one add per
 * moment per particle, so the per-node summation order of
 * og_deposit_one (node-major) equals the reference's (moment-major). */

static int og_mover(const orc_setup *s, const void *const fld[6], void *x, void *y,
                    void *z, void *u, void *v, void *w, long nop, double qom, int bc_v) {
  og_grid g;
  if (og_make_grid(s, &g)) return -1;
  og_push pc = og_push_consts(s, qom);
  const fpf *F[6];
  for (int f = 0; f < 6; f++) F[f] = (const fpf *)fld[f];
  fpp *X = (fpp *)x, *Y = (fpp *)y, *Z = (fpp *)z;
  fpp *U = (fpp *)u, *V = (fpp *)v, *W = (fpp *)w;
#pragma omp parallel for schedule(static)
  for (long i = 0; i < nop; i++)
    og_move_one(&g, s, &pc, F, &X[i], &Y[i], &Z[i], &U[i], &V[i], &W[i], bc_v);
  og_free_grid(&g);
  return 0;
}

int orc_mover_pc(const orc_setup *s, const void *const fld[6], void *x, void *y,
                 void *z, void *u, void *v, void *w, long nop, double qom) {
  return og_mover(s, fld, x, y, z, u, v, w, nop, qom, 0);
}

int orc_mover_pc_v(const orc_setup *s, const void *const fld[6], void *x, void *y,
                   void *z, void *u, void *v, void *w, long nop, double qom) {
  return og_mover(s, fld, x, y, z, u, v, w, nop, qom, 1);
}

void orc_interp_p2g(const orc_setup *s, const void *x, const void *y,
                    const void *z, const void *u, const void *v, const void *w,
                    const void *q, long nop, void *const mom[10]) {
  og_grid g;
  if (og_make_grid(s, &g)) return;
  const fpp *X = (const fpp *)x, *Y = (const fpp *)y, *Z = (const fpp *)z;
  const fpp *U = (const fpp *)u, *V = (const fpp *)v, *W = (const fpp *)w;
  const fpi *Q = (const fpi *)q;
  fpi *M[10];
  for (int m = 0; m < 10; m++) M[m] = (fpi *)mom[m];
  for (long i = 0; i < nop; i++) og_deposit_one(&g, X[i], Y[i], Z[i], U[i], V[i], W[i], Q[i], M);
  og_free_grid(&g);
}

/* applyBCids (src/BC.cpp:362-615): periodic axes fold the last active node
 * onto the first (node1 += node[n-2]; node[n-2] = node1) in the order X, Y,
 * Z; then non-periodic axes double both boundary planes, again X, Y, Z. */
static void og_apply_bc(const og_grid *g, const orc_setup *s, fpi *const *mom) {
  const int nxn = g->nxn, nyn = g->nyn, nzn = g->nzn;
  for (int m = 0; m < 10; m++) {
    fpi *a = mom[m];
#define N3(i, j, k) a[((long)(i) * nyn + (j)) * nzn + (k)]
    if (s->periodic[0])
      for (int j = 1; j < nyn - 1; j++)
        for (int k = 1; k < nzn - 1; k++) {
          N3(1, j, k) += N3(nxn - 2, j, k);
          N3(nxn - 2, j, k) = N3(1, j, k);
        }
    if (s->periodic[1])
      for (int i = 1; i < nxn - 1; i++)
        for (int k = 1; k < nzn - 1; k++) {
          N3(i, 1, k) += N3(i, nyn - 2, k);
          N3(i, nyn - 2, k) = N3(i, 1, k);
        }
    if (s->periodic[2])
      for (int i = 1; i < nxn - 1; i++)
        for (int j = 1; j < nyn - 1; j++) {
          N3(i, j, 1) += N3(i, j, nzn - 2);
          N3(i, j, nzn - 2) = N3(i, j, 1);
        }
    if (!s->periodic[0])
      for (int j = 1; j < nyn - 1; j++)
        for (int k = 1; k < nzn - 1; k++) {
          N3(1, j, k) *= 2;
          N3(nxn - 2, j, k) *= 2;
        }
    if (!s->periodic[1])
      for (int i = 1; i < nxn - 1; i++)
        for (int k = 1; k < nzn - 1; k++) {
          N3(i, 1, k) *= 2;
          N3(i, nyn - 2, k) *= 2;
        }
    if (!s->periodic[2])
      for (int i = 1; i < nxn - 1; i++)
        for (int j = 1; j < nyn - 1; j++) {
          N3(i, j, 1) *= 2;
          N3(i, j, nzn - 2) *= 2;
        }
#undef N3
  }
}

void orc_apply_bc_ids(const orc_setup *s, void *const mom[10]) {
  og_grid g;
  if (og_make_grid(s, &g)) return;
  fpi *M[10];
  for (int m = 0; m < 10; m++) M[m] = (fpi *)mom[m];
  og_apply_bc(&g, s, M);
  og_free_grid(&g);
}

int orc_mover_interp(const orc_setup *s, const void *const fld[6], void *x,
                     void *y, void *z, void *u, void *v, void *w, const void *q,
                     long nop, double qom, void *const mom[10]) {
  og_grid g;
  if (og_make_grid(s, &g)) return -1;
  og_push pc = og_push_consts(s, qom);
  const fpf *F[6];
  for (int f = 0; f < 6; f++) F[f] = (const fpf *)fld[f];
  fpp *X = (fpp *)x, *Y = (fpp *)y, *Z = (fpp *)z;
  fpp *U = (fpp *)u, *V = (fpp *)v, *W = (fpp *)w;
  const fpi *Q = (const fpi *)q;
  fpi *M[10];
  for (int m = 0; m < 10; m++) M[m] = (fpi *)mom[m];
  for (long i = 0; i < nop; i++) {
    og_move_one(&g, s, &pc, F, &X[i], &Y[i], &Z[i], &U[i], &V[i], &W[i], 0);
    og_deposit_one(&g, X[i], Y[i], Z[i], U[i], V[i], W[i], Q[i], M);
  }
  og_free_grid(&g);
  return 0;
}

#ifdef _OPENMP
static double og_now(void) { return omp_get_wtime(); }
#else
#include <time.h>
static double og_now(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + 1e-9 * t.tv_nsec;
}
#endif

int orc_cycle(const orc_setup *s, const void *const fld[6], int ns,
              void *const *x, void *const *y, void *const *z, void *const *u,
              void *const *v, void *const *w, void *const *q, const long *nop,
              const double *qom, void *const *mom, double *t_mover,
              double *t_interp) {
  og_grid g;
  if (og_make_grid(s, &g)) return -1;
  const fpf *F[6];
  for (int f = 0; f < 6; f++) F[f] = (const fpf *)fld[f];
  const long nodes = (long)g.nxn * g.nyn * g.nzn;
  double t0 = og_now();
  for (int is = 0; is < ns; is++) {
    og_push pc = og_push_consts(s, qom[is]);
    fpp *X = (fpp *)x[is], *Y = (fpp *)y[is], *Z = (fpp *)z[is];
    fpp *U = (fpp *)u[is], *V = (fpp *)v[is], *W = (fpp *)w[is];
#pragma omp parallel for schedule(static)
    for (long i = 0; i < nop[is]; i++)
      og_move_one(&g, s, &pc, F, &X[i], &Y[i], &Z[i], &U[i], &V[i], &W[i], 0);
  }
  double t1 = og_now();
  for (int a = 0; a < ns * 10; a++) memset(mom[a], 0, sizeof(fpi) * nodes);
#pragma omp parallel for schedule(static, 1)
  for (int is = 0; is < ns; is++) {
    fpi *M[10];
    for (int m = 0; m < 10; m++) M[m] = (fpi *)mom[is * 10 + m];
    const fpp *X = (const fpp *)x[is], *Y = (const fpp *)y[is], *Z = (const fpp *)z[is];
    const fpp *U = (const fpp *)u[is], *V = (const fpp *)v[is], *W = (const fpp *)w[is];
    const fpi *Q = (const fpi *)q[is];
    for (long i = 0; i < nop[is]; i++) og_deposit_one(&g, X[i], Y[i], Z[i], U[i], V[i], W[i], Q[i], M);
    og_apply_bc(&g, s, M);
  }
  double t2 = og_now();
  if (t_mover) *t_mover = t1 - t0;
  if (t_interp) *t_interp = t2 - t1;
  og_free_grid(&g);
  return 0;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int orc_fp_bytes(void) { return (int)sizeof(fpp); }

/* particle_sort, binned branch (src/Particles.cpp:153-233): bin counts from the
 * grid's cell counts with guard cells (grd->nxc), bin width L / (FPpart)n_bin
 * rounded to FPpart, bin floor(x / width) in FPpart arithmetic, index
 * z + y*nbz + x*nbz*nby (src/Particles.cpp:67-69), particles outside every bin
 * in a last bin; a bin keeps the particles' original order. */
int orc_particle_sort(const orc_setup *s, int sort_cps, void *xv, void *yv, void *zv, void *uv,
                      void *vv, void *wv, void *qv, long n) {
  if (n <= 0) return 0;
  if (sort_cps < 1) return -1;
  const long ncx = s->nxc + 2, ncy = s->nyc + 2, ncz = s->nzc + 2;   /* grd->nxc */
  const long nbx = 1 + ((ncx - 1) / sort_cps);
  const long nby = 1 + ((ncy - 1) / sort_cps);
  const long nbz = 1 + ((ncz - 1) / sort_cps);
  const fpp dx = (fpp)(s->Lx / (fpp)nbx), dy = (fpp)(s->Ly / (fpp)nby),
            dz = (fpp)(s->Lz / (fpp)nbz);
  const long bins = nbx * nby * nbz + 1;
  fpp *arr[6] = {(fpp *)xv, (fpp *)yv, (fpp *)zv, (fpp *)uv, (fpp *)vv, (fpp *)wv};
  fpi *q = (fpi *)qv;
  long *key = (long *)malloc(sizeof(long) * n);
  long *start = (long *)calloc(bins + 1, sizeof(long));
  fpp *tmp = (fpp *)malloc(sizeof(fpp) * n);
  fpi *tmpq = (fpi *)malloc(sizeof(fpi) * n);
  long *dst = (long *)malloc(sizeof(long) * n);
  if (!key || !start || !tmp || !tmpq || !dst) {
    free(key); free(start); free(tmp); free(tmpq); free(dst);
    return -1;
  }
  for (long i = 0; i < n; i++) {
    const fpp fx = (fpp)floor(arr[0][i] / dx), fy = (fpp)floor(arr[1][i] / dy),
              fz = (fpp)floor(arr[2][i] / dz);
    const int in = fx >= 0 && fx < (fpp)nbx && fy >= 0 && fy < (fpp)nby && fz >= 0 &&
                   fz < (fpp)nbz;
    key[i] = in ? (long)fz + (long)fy * nbz + (long)fx * nbz * nby : bins - 1;
    start[key[i] + 1]++;
  }
  for (long b = 0; b < bins; b++) start[b + 1] += start[b];
  for (long i = 0; i < n; i++) dst[i] = start[key[i]]++;   /* in index order: stable */
  for (int a = 0; a < 6; a++) {
    for (long i = 0; i < n; i++) tmp[dst[i]] = arr[a][i];
    memcpy(arr[a], tmp, sizeof(fpp) * n);
  }
  for (long i = 0; i < n; i++) tmpq[dst[i]] = q[i];
  memcpy(q, tmpq, sizeof(fpi) * n);
  free(key); free(start); free(tmp); free(tmpq); free(dst);
  return 0;
}

/* ------------------------------------------------------------------------
 * calculateHatDensities (src/MaxwellSolver.cpp:465-603): the implicit
 * sources J-hat (nodes) and rho-hat (cell centres) from the species moments.
 * ---------------------------------------------------------------------- */

/* Guard-cell fill of one scalar array of n0 x n1 x n2 points
 * (applyBCscalarDensC, src/BC.cpp:623-727, and applyBCscalarDensN,
 * src/BC.cpp:11-121). Phases in the reference order: periodic faces X, Y, Z;
 * edges along X, Y, Z; corners; then non-periodic faces X, Y, Z, which copy
 * the neighbouring plane. A periodic face copies from index n-1-s to 0 and
 * from s to n-1, with s = 1 on centres and 2 on nodes. yhi is the end of the
 * Y-edge loop (the centre version runs it to nyn - 1 = n1). */
static void og_bc_scalar(fpi *a, int n0, int n1, int n2, const int per[3], int s, int yhi) {
#define A3(i, j, k) a[((long)(i) * n1 + (j)) * n2 + (k)]
  const int e0 = n0 - 1, e1 = n1 - 1, e2 = n2 - 1;      /* last index */
  const int f0 = n0 - 1 - s, f1 = n1 - 1 - s, f2 = n2 - 1 - s;  /* periodic source */
  if (per[0])
    for (int j = 1; j < e1; j++)
      for (int k = 1; k < e2; k++) {
        A3(0, j, k) = A3(f0, j, k);
        A3(e0, j, k) = A3(s, j, k);
      }
  if (per[1])
    for (int i = 1; i < e0; i++)
      for (int k = 1; k < e2; k++) {
        A3(i, 0, k) = A3(i, f1, k);
        A3(i, e1, k) = A3(i, s, k);
      }
  if (per[2])
    for (int i = 1; i < e0; i++)
      for (int j = 1; j < e1; j++) {
        A3(i, j, 0) = A3(i, j, f2);
        A3(i, j, e2) = A3(i, j, s);
      }
  if (per[1] || per[2])
    for (int i = 1; i < e0; i++) {
      A3(i, e1, e2) = A3(i, s, s);
      A3(i, 0, 0) = A3(i, f1, f2);
      A3(i, 0, e2) = A3(i, f1, s);
      A3(i, e1, 0) = A3(i, s, f2);
    }
  if (per[0] || per[2])
    for (int j = 1; j < yhi; j++) {
      A3(e0, j, e2) = A3(s, j, s);
      A3(0, j, 0) = A3(f0, j, f2);
      A3(0, j, e2) = A3(f0, j, s);
      A3(e0, j, 0) = A3(s, j, f2);
    }
  if (per[0] || per[1])
    for (int k = 1; k < e2; k++) {
      A3(e0, e1, k) = A3(s, s, k);
      A3(0, 0, k) = A3(f0, f1, k);
      A3(e0, 0, k) = A3(s, f1, k);
      A3(0, e1, k) = A3(f0, s, k);
    }
  if (per[0] || per[1] || per[2]) {
    A3(e0, e1, e2) = A3(s, s, s);
    A3(0, e1, e2) = A3(f0, s, s);
    A3(e0, 0, e2) = A3(s, f1, s);
    A3(0, 0, e2) = A3(f0, f1, s);
    A3(e0, e1, 0) = A3(s, s, f2);
    A3(0, e1, 0) = A3(f0, s, f2);
    A3(e0, 0, 0) = A3(s, f1, f2);
    A3(0, 0, 0) = A3(f0, f1, f2);
  }
  if (!per[0])
    for (int j = 0; j < n1; j++)
      for (int k = 0; k < n2; k++) {
        A3(0, j, k) = A3(1, j, k);
        A3(e0, j, k) = A3(e0 - 1, j, k);
      }
  if (!per[1])
    for (int i = 0; i < n0; i++)
      for (int k = 0; k < n2; k++) {
        A3(i, 0, k) = A3(i, 1, k);
        A3(i, e1, k) = A3(i, e1 - 1, k);
      }
  if (!per[2])
    for (int i = 0; i < n0; i++)
      for (int j = 0; j < n1; j++) {
        A3(i, j, 0) = A3(i, j, 1);
        A3(i, j, e2) = A3(i, j, e2 - 1);
      }
#undef A3
}

/* Centre-difference stencil of a node array at cell (i, j, k) along `axis`:
 * the four node differences across the cell's faces, each times .25 and the
 * inverse spacing, summed in double in the reference order (src/Grid.cpp:
 * 267-319 divN2C, 322-396 divSymmTensorN2C). The caller rounds. */
static double og_d4(const og_grid *g, const fpi *a, int i, int j, int k, int axis, fpi inv) {
  /* the two indices that run across the face, in the order the reference
   * lists the four terms: x (j, k) with k fastest; y (i, k) with k fastest;
   * z (i, j) with i fastest */
  double sum = 0.0;
  for (int t = 0; t < 4; t++) {
    int i0 = i, j0 = j, k0 = k;
    int hi = t >> 1, lo = t & 1;
    if (axis == 0) { j0 += hi; k0 += lo; }
    else if (axis == 1) { i0 += hi; k0 += lo; }
    else { j0 += hi; i0 += lo; }
    const long n0 = og_node(g, i0, j0, k0);
    const long n1 = og_node(g, i0 + (axis == 0), j0 + (axis == 1), k0 + (axis == 2));
    const double term = .25 * (fpi)(a[n1] - a[n0]) * inv;
    sum = t ? sum + term : term;
  }
  return sum;
}

int orc_hat_densities(const orc_setup *s, double th, int ns, const double *qom,
                      const void *const *mom, const void *const fld[6], const void *rhoc_v,
                      void *jxh_v, void *jyh_v, void *jzh_v, void *rhoh_v) {
  og_grid g;
  if (og_make_grid(s, &g)) return -1;
  const int nxc = g.nxc, nyc = g.nyc, nzc = g.nzc;
  const int nxn = g.nxn, nyn = g.nyn, nzn = g.nzn;
  const long nc = (long)nxc * nyc * nzc, nn = (long)nxn * nyn * nzn;
  fpi *tc[3], *tn[3];
  for (int a = 0; a < 3; a++) {
    tc[a] = (fpi *)calloc(nc, sizeof(fpi));
    tn[a] = (fpi *)calloc(nn, sizeof(fpi));
  }
  fpi *jh[3] = {(fpi *)jxh_v, (fpi *)jyh_v, (fpi *)jzh_v};
  fpi *rhoh = (fpi *)rhoh_v;
  const fpi *rhoc = (const fpi *)rhoc_v;
  const fpf *Bn[3] = {(const fpf *)fld[3], (const fpf *)fld[4], (const fpf *)fld[5]};
  const fpi inv[3] = {(fpi)g.invdx, (fpi)g.invdy, (fpi)g.invdz};
#define CI(i, j, k) (((long)(i) * nyc + (j)) * nzc + (k))
  for (long n = 0; n < nn; n++) jh[0][n] = jh[1][n] = jh[2][n] = 0;
  for (long c = 0; c < nc; c++) rhoh[c] = 0;
  const fpf alfa = (fpf)(-s->dt / 2.0);
  for (int is = 0; is < ns; is++) {
    const fpi *const *M = (const fpi *const *)mom + 10 * is;
    /* divSymmTensorN2C: row r of the symmetric tensor, columns x, y, z
     * (pxx pxy pxz / pxy pyy pyz / pxz pyz pzz), then scaled by -dt/2 */
    const fpi *T[3][3] = {{M[4], M[5], M[6]}, {M[5], M[7], M[8]}, {M[6], M[8], M[9]}};
    for (int i = 1; i < nxc - 1; i++)
      for (int j = 1; j < nyc - 1; j++)
        for (int k = 1; k < nzc - 1; k++) {
          fpi comp[3][3]; /* [row][axis] */
          for (int r = 0; r < 3; r++)
            for (int ax = 0; ax < 3; ax++)
              comp[r][ax] = (fpi)og_d4(&g, T[ax][r], i, j, k, ax, inv[ax]);
          for (int r = 0; r < 3; r++) tc[r][CI(i, j, k)] = comp[r][0] + comp[r][1] + comp[r][2];
        }
    for (int r = 0; r < 3; r++) {
      for (long c = 0; c < nc; c++) tc[r][c] *= alfa;
      og_bc_scalar(tc[r], nxc, nyc, nzc, s->periodic, 1, nyn - 1);
    }
    /* interpC2Ninterp on the inner nodes, then + J (src/Grid.cpp:122-139) */
    for (int r = 0; r < 3; r++) {
      const fpi *C = tc[r];
      for (int i = 1; i < nxn - 1; i++)
        for (int j = 1; j < nyn - 1; j++)
          for (int k = 1; k < nzn - 1; k++) {
            fpi sum8 = C[CI(i, j, k)] + C[CI(i - 1, j, k)];
            sum8 = sum8 + C[CI(i, j - 1, k)];
            sum8 = sum8 + C[CI(i, j, k - 1)];
            sum8 = sum8 + C[CI(i - 1, j - 1, k)];
            sum8 = sum8 + C[CI(i - 1, j, k - 1)];
            sum8 = sum8 + C[CI(i, j - 1, k - 1)];
            sum8 = sum8 + C[CI(i - 1, j - 1, k - 1)];
            tn[r][og_node(&g, i, j, k)] = (fpi)(.125 * sum8);
          }
      const fpi *J = M[1 + r];
      for (long n = 0; n < nn; n++) tn[r][n] += J[n];
    }
    /* PIdot: rotate with the species' omega_c dt / 2 and accumulate */
    const fpf beta = (fpf)(.5 * qom[is] * s->dt / s->c);
    for (long n = 0; n < nn; n++) {
      const fpf ox = beta * Bn[0][n], oy = beta * Bn[1][n], oz = beta * Bn[2][n];
      const fpi X = tn[0][n], Y = tn[1][n], Z = tn[2][n];
      const fpf edotb = X * ox + Y * oy + Z * oz;
      const fpf denom = (fpf)(1 / (1.0 + ox * ox + oy * oy + oz * oz));
      jh[0][n] += (X + (Y * oz - Z * oy + edotb * ox)) * denom;
      jh[1][n] += (Y + (Z * ox - X * oz + edotb * oy)) * denom;
      jh[2][n] += (Z + (X * oy - Y * ox + edotb * oz)) * denom;
    }
  }
  for (int r = 0; r < 3; r++) og_bc_scalar(jh[r], nxn, nyn, nzn, s->periodic, 2, nyn - 1);
  /* rho hat = rho_c - dt theta div(J hat) (divN2C on the inner cells) */
  fpi *dv = tc[0];
  for (long c = 0; c < nc; c++) dv[c] = 0;
  for (int i = 1; i < nxc - 1; i++)
    for (int j = 1; j < nyc - 1; j++)
      for (int k = 1; k < nzc - 1; k++) {
        const fpf cx = (fpf)og_d4(&g, jh[0], i, j, k, 0, inv[0]);
        const fpf cy = (fpf)og_d4(&g, jh[1], i, j, k, 1, inv[1]);
        const fpf cz = (fpf)og_d4(&g, jh[2], i, j, k, 2, inv[2]);
        dv[CI(i, j, k)] = cx + cy + cz;
      }
  for (long c = 0; c < nc; c++) rhoh[c] = (fpi)(rhoc[c] - s->dt * th * dv[c]);
  og_bc_scalar(rhoh, nxc, nyc, nzc, s->periodic, 1, nyn - 1);
#undef CI
  for (int a = 0; a < 3; a++) {
    free(tc[a]);
    free(tn[a]);
  }
  og_free_grid(&g);
  return 0;
}
