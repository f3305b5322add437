/*
 * Flat C wrapper around the REFERENCE's own mover_PC / interpP2G /
 * mover_interp / applyBCids, so the tests can run sputniPIC's code on the
 * same arrays as the restatement (oracle.c) and the CUDA library.
 *
 * TEST INFRASTRUCTURE ONLY. Built by oracle/Makefile against the reference's
 * sources where they lie (src/Mover.cpp, src/Grid.cpp, src/BC.cpp,
 * src/EMfield.cpp, src/InterpDensSpecies.cpp, src/InterpDensNet.cpp,
 * src/Particles.cpp, src/MaxwellSolver.cpp with src/Basic.cpp and
 * src/Solvers.cpp it links against) into oracle/_ref/, which is never
 * committed.
 *
 * Each call builds the reference structs the way the CPU driver does
 * (src/sputniPIC_CPU.cpp:105-135: setGrid, field_allocate,
 * interp_dens_species_allocate) and points `particles` at the caller's
 * arrays, so mover_PC updates them in place.
 */
#include <omp.h>

#include <cstring>
#include <vector>

#include "BC.h"
#include "InterpDensNet.h"
#include "MaxwellSolver.h"
#include "Mover.h"
#include "Particles.h"
#include "oracle_api.h"

namespace {

struct RefWorld {
  parameters param;
  grid grd;
  EMfield field;
  bool has_field = false;

  explicit RefWorld(const orc_setup *s) : param() {
    param.c = s->c;
    param.dt = s->dt;
    param.NiterMover = s->niter;
    param.n_sub_cycles = s->n_sub_cycles;
    param.Lx = s->Lx;
    param.Ly = s->Ly;
    param.Lz = s->Lz;
    param.nxc = s->nxc;
    param.nyc = s->nyc;
    param.nzc = s->nzc;
    param.PERIODICX = s->periodic[0] != 0;
    param.PERIODICY = s->periodic[1] != 0;
    param.PERIODICZ = s->periodic[2] != 0;
    param.PERIODICX_P = param.PERIODICX;
    param.PERIODICY_P = param.PERIODICY;
    param.PERIODICZ_P = param.PERIODICZ;
    param.ns = 1;
    setGrid(&param, &grd);
  }
  ~RefWorld() {
    if (has_field) field_deallocate(&grd, &field);
    grid_deallocate(&grd);
  }
  long nodes() const { return (long)grd.nxn * grd.nyn * grd.nzn; }

  void load_field(const void *const fld[6]) {
    field_allocate(&grd, &field);
    has_field = true;
    FPfield *dst[6] = {field.Ex_flat, field.Ey_flat, field.Ez_flat,
                       field.Bxn_flat, field.Byn_flat, field.Bzn_flat};
    for (int f = 0; f < 6; f++) std::memcpy(dst[f], fld[f], sizeof(FPfield) * nodes());
  }
};

void wrap_particles(particles *p, const orc_setup *s, void *x, void *y, void *z,
                    void *u, void *v, void *w, const void *q, long nop, double qom) {
  std::memset(p, 0, sizeof(*p));
  p->species_ID = 0;
  p->nop = nop;
  p->npmax = nop;
  p->NiterMover = s->niter;
  p->n_sub_cycles = s->n_sub_cycles;
  p->qom = (FPpart)qom; /* src/Particles.cpp:25 */
  p->x = (FPpart *)x;
  p->y = (FPpart *)y;
  p->z = (FPpart *)z;
  p->u = (FPpart *)u;
  p->v = (FPpart *)v;
  p->w = (FPpart *)w;
  p->q = (FPinterp *)q;
}

FPinterp *const *moment_slots(interpDensSpecies *ids, FPinterp *out[10]) {
  out[0] = ids->rhon_flat;
  out[1] = ids->Jx_flat;
  out[2] = ids->Jy_flat;
  out[3] = ids->Jz_flat;
  out[4] = ids->pxx_flat;
  out[5] = ids->pxy_flat;
  out[6] = ids->pxz_flat;
  out[7] = ids->pyy_flat;
  out[8] = ids->pyz_flat;
  out[9] = ids->pzz_flat;
  return out;
}

}  // namespace

extern "C" {

int orc_mover_pc(const orc_setup *s, const void *const fld[6], void *x, void *y,
                 void *z, void *u, void *v, void *w, long nop, double qom) {
  RefWorld W(s);
  W.load_field(fld);
  particles p;
  wrap_particles(&p, s, x, y, z, u, v, w, nullptr, nop, qom);
  return mover_PC(&p, &W.field, &W.grd, &W.param);
}

int orc_mover_pc_v(const orc_setup *s, const void *const fld[6], void *x, void *y,
                   void *z, void *u, void *v, void *w, long nop, double qom) {
  RefWorld W(s);
  W.load_field(fld);
  particles p;
  wrap_particles(&p, s, x, y, z, u, v, w, nullptr, nop, qom);
  return mover_PC_V(&p, &W.field, &W.grd, &W.param);
}

void orc_interp_p2g(const orc_setup *s, const void *x, const void *y,
                    const void *z, const void *u, const void *v, const void *w,
                    const void *q, long nop, void *const mom[10]) {
  RefWorld W(s);
  particles p;
  wrap_particles(&p, s, (void *)x, (void *)y, (void *)z, (void *)u, (void *)v,
                 (void *)w, q, nop, 1.0);
  interpDensSpecies ids;
  interp_dens_species_allocate(&W.grd, &ids, 0);
  FPinterp *slot[10];
  moment_slots(&ids, slot);
  for (int m = 0; m < 10; m++) std::memcpy(slot[m], mom[m], sizeof(FPinterp) * W.nodes());
  interpP2G(&p, &ids, &W.grd);
  for (int m = 0; m < 10; m++) std::memcpy(mom[m], slot[m], sizeof(FPinterp) * W.nodes());
  interp_dens_species_deallocate(&W.grd, &ids);
}

void orc_apply_bc_ids(const orc_setup *s, void *const mom[10]) {
  RefWorld W(s);
  interpDensSpecies ids;
  interp_dens_species_allocate(&W.grd, &ids, 0);
  FPinterp *slot[10];
  moment_slots(&ids, slot);
  for (int m = 0; m < 10; m++) std::memcpy(slot[m], mom[m], sizeof(FPinterp) * W.nodes());
  applyBCids(&ids, &W.grd, &W.param);
  for (int m = 0; m < 10; m++) std::memcpy(mom[m], slot[m], sizeof(FPinterp) * W.nodes());
  interp_dens_species_deallocate(&W.grd, &ids);
}

int orc_mover_interp(const orc_setup *s, const void *const fld[6], void *x,
                     void *y, void *z, void *u, void *v, void *w, const void *q,
                     long nop, double qom, void *const mom[10]) {
  RefWorld W(s);
  W.load_field(fld);
  particles p;
  wrap_particles(&p, s, x, y, z, u, v, w, q, nop, qom);
  interpDensSpecies ids;
  interp_dens_species_allocate(&W.grd, &ids, 0);
  FPinterp *slot[10];
  moment_slots(&ids, slot);
  for (int m = 0; m < 10; m++) std::memcpy(slot[m], mom[m], sizeof(FPinterp) * W.nodes());
  int rc = mover_interp(&p, &W.field, &ids, &W.grd, &W.param);
  for (int m = 0; m < 10; m++) std::memcpy(mom[m], slot[m], sizeof(FPinterp) * W.nodes());
  interp_dens_species_deallocate(&W.grd, &ids);
  return rc;
}

/* The driver's hot section, src/sputniPIC_CPU.cpp:232-256, with the same
 * calls in the same order and the same OpenMP team over species. */
int orc_cycle(const orc_setup *s, const void *const fld[6], int ns,
              void *const *x, void *const *y, void *const *z, void *const *u,
              void *const *v, void *const *w, void *const *q, const long *nop,
              const double *qom, void *const *mom, double *t_mover,
              double *t_interp) {
  RefWorld W(s);
  W.param.ns = ns;
  W.load_field(fld);
  std::vector<particles> part(ns);
  for (int is = 0; is < ns; is++) {
    wrap_particles(&part[is], s, x[is], y[is], z[is], u[is], v[is], w[is], q[is],
                   nop[is], qom[is]);
    part[is].species_ID = is;
  }
  std::vector<interpDensSpecies> ids(ns);
  for (int is = 0; is < ns; is++) interp_dens_species_allocate(&W.grd, &ids[is], is);
  interpDensNet idn;
  interp_dens_net_allocate(&W.grd, &idn);

  double t0 = omp_get_wtime();
  for (int is = 0; is < ns; is++) mover_PC(&part[is], &W.field, &W.grd, &W.param);
  double t1 = omp_get_wtime();
  setZeroDensities(&idn, ids.data(), &W.grd, ns);
#pragma omp parallel for
  for (int is = 0; is < ns; is++) {
    interpP2G(&part[is], &ids[is], &W.grd);
    applyBCids(&ids[is], &W.grd, &W.param);
  }
  double t2 = omp_get_wtime();
  if (t_mover) *t_mover = t1 - t0;
  if (t_interp) *t_interp = t2 - t1;

  for (int is = 0; is < ns; is++) {
    FPinterp *slot[10];
    moment_slots(&ids[is], slot);
    for (int m = 0; m < 10; m++)
      std::memcpy(mom[is * 10 + m], slot[m], sizeof(FPinterp) * W.nodes());
    interp_dens_species_deallocate(&W.grd, &ids[is]);
  }
  interp_dens_net_deallocate(&W.grd, &idn);
  return 0;
}

int orc_num_threads(void) { return omp_get_max_threads(); }

int orc_fp_bytes(void) { return (int)sizeof(FPpart); }

int orc_particle_sort(const orc_setup *s, int sort_cps, void *x, void *y, void *z, void *u,
                      void *v, void *w, void *q, long n) {
  if (n <= 0) return 0;
  if (sort_cps < 1) return -1;
  RefWorld W(s);
  W.param.sort_cps = sort_cps;
  particles p;
  wrap_particles(&p, s, x, y, z, u, v, w, q, n, 0.0);
  particle_sort(&W.param, &p, &W.grd);   // src/Particles.cpp:72-234
  return 0;
}

/* calculateHatDensities (src/MaxwellSolver.cpp:465-603) on the caller's
 * arrays: the structs are built as the CPU driver builds them
 * (src/sputniPIC_CPU.cpp:105-135), the moments and rhoc copied in, the hat
 * densities copied out. */
int orc_hat_densities(const orc_setup *s, double th, int ns, const double *qom,
                      const void *const *mom, const void *const fld[6], const void *rhoc,
                      void *jxh, void *jyh, void *jzh, void *rhoh) {
  if (ns < 1 || ns > NS_MAX) return -1;
  RefWorld W(s);
  W.param.ns = ns;
  W.param.th = th;
  for (int is = 0; is < ns; is++) W.param.qom[is] = qom[is];
  W.load_field(fld);
  std::vector<interpDensSpecies> ids(ns);
  for (int is = 0; is < ns; is++) {
    interp_dens_species_allocate(&W.grd, &ids[is], is);
    FPinterp *slot[10];
    moment_slots(&ids[is], slot);
    for (int m = 0; m < 10; m++)
      std::memcpy(slot[m], ((const void *const *)mom)[10 * is + m], sizeof(FPinterp) * W.nodes());
  }
  interpDensNet idn;
  interp_dens_net_allocate(&W.grd, &idn);
  const long cells = (long)W.grd.nxc * W.grd.nyc * W.grd.nzc;
  std::memcpy(idn.rhoc_flat, rhoc, sizeof(FPinterp) * cells);
  interpDens_aux aux;
  interp_dens_aux_allocate(&W.grd, &aux);
  calculateHatDensities(&aux, &idn, ids.data(), &W.field, &W.grd, &W.param);
  std::memcpy(jxh, &aux.Jxh[0][0][0], sizeof(FPinterp) * W.nodes());
  std::memcpy(jyh, &aux.Jyh[0][0][0], sizeof(FPinterp) * W.nodes());
  std::memcpy(jzh, &aux.Jzh[0][0][0], sizeof(FPinterp) * W.nodes());
  std::memcpy(rhoh, &aux.rhoh[0][0][0], sizeof(FPinterp) * cells);
  interp_dens_aux_deallocate(&W.grd, &aux);
  interp_dens_net_deallocate(&W.grd, &idn);
  for (int is = 0; is < ns; is++) interp_dens_species_deallocate(&W.grd, &ids[is]);
  return 0;
}

}  // extern "C"
