/*
 * Flat C interface shared by the two CPU oracles of the particle mover and
 * the particle-to-grid (P2G) moment deposition.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the shipped library links, loads or
 * calls these functions. Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py use them, as the checker.
 *
 * Two libraries implement this header:
 *   - oracle/liboracle_{fp32,fp64}.so: oracle.c, a plain-C restatement of
 *     sputniPIC's src/Mover.cpp, src/Grid.cpp:5-62 and src/BC.cpp:362-615,
 *     src/Particles.cpp:72-234 (particle_sort) and
 *     src/MaxwellSolver.cpp:465-603 (calculateHatDensities) with the Grid.cpp
 *     stencils and BC.cpp guard-cell fills it calls.
 *   - oracle/_ref/libref_{fp32,fp64}.so: ref_shim.cpp linked against the
 *     reference's own sources, compiled where they lie.
 * ORC_FP is float in the *_fp32 builds (the reference's PrecisionTypes.h)
 * and double in the *_fp64 builds.
 *
 * Field arrays follow the reference node layout: flat [nxn][nyn][nzn],
 * index (i*nyn + j)*nzn + k, nxn = nxc + 3 (include/Alloc.h:111-124,
 * src/Grid.cpp:9-15). Moment order (src/Mover.cpp:466-570):
 *   0 rhon, 1 Jx, 2 Jy, 3 Jz, 4 pxx, 5 pxy, 6 pxz, 7 pyy, 8 pyz, 9 pzz.
 * Field order: 0 Ex, 1 Ey, 2 Ez, 3 Bxn, 4 Byn, 5 Bzn (include/EMfield.h).
 */
#ifndef SPUTNIPIC_ORACLE_API_H
#define SPUTNIPIC_ORACLE_API_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_setup {
  int nxc, nyc, nzc;    /* active cells per axis, guard cells excluded */
  double Lx, Ly, Lz;    /* domain lengths */
  int periodic[3];      /* field periodicity flags; the mover's particle BC reads these */
  double dt;            /* time step */
  double c;             /* light speed */
  int niter;            /* NiterMover */
  int n_sub_cycles;     /* n_sub_cycles (mover_PC only divides dt by it) */
} orc_setup;

/* Every function is compiled twice: ORC_FP = float and ORC_FP = double. The
 * prototypes use void pointers so one header serves both builds. */

/* mover_PC on one species (src/Mover.cpp:4-162). Returns 0. */
int orc_mover_pc(const orc_setup *s, const void *const fld[6], void *x, void *y,
                 void *z, void *u, void *v, void *w, long nop, double qom);

/* mover_PC_V on one species (src/Mover.cpp:166-382): the same push; the
 * reflecting BC mirrors the position first and flips the velocity only if the
 * mirrored position is still outside the box. Returns 0. */
int orc_mover_pc_v(const orc_setup *s, const void *const fld[6], void *x, void *y,
                   void *z, void *u, void *v, void *w, long nop, double qom);

/* interpP2G on one species (src/Mover.cpp:385-572): ADDS into mom[10]. */
void orc_interp_p2g(const orc_setup *s, const void *x, const void *y,
                    const void *z, const void *u, const void *v, const void *w,
                    const void *q, long nop, void *const mom[10]);

/* applyBCids on one species' moments (src/BC.cpp:362-615). */
void orc_apply_bc_ids(const orc_setup *s, void *const mom[10]);
/* particle_sort (src/Particles.cpp:72-234, the binned branch) over n
 * particles: bins of sort_cps cells per axis, stable within a bin, particles
 * outside the bins last. Returns 0, or -1 when out of memory. */
int orc_particle_sort(const orc_setup *s, int sort_cps, void *x, void *y, void *z, void *u,
                      void *v, void *w, void *q, long n);

/* mover_interp (src/Mover.cpp:575-862): mover then deposit, per particle. */
int orc_mover_interp(const orc_setup *s, const void *const fld[6], void *x,
                     void *y, void *z, void *u, void *v, void *w, const void *q,
                     long nop, double qom, void *const mom[10]);

/* One cycle of the CPU driver's hot section for ns species
 * (src/sputniPIC_CPU.cpp:232-256): mover_PC per species, zero the moments,
 * then in an OpenMP team over species interpP2G + applyBCids. mom holds
 * ns*10 arrays (species-major) and is overwritten. Wall times in seconds. */
int orc_cycle(const orc_setup *s, const void *const fld[6], int ns,
              void *const *x, void *const *y, void *const *z, void *const *u,
              void *const *v, void *const *w, void *const *q, const long *nop,
              const double *qom, void *const *mom, double *t_mover,
              double *t_interp);

/* calculateHatDensities (src/MaxwellSolver.cpp:465-603) for ns species
 * (ns <= 6, the reference's NS_MAX): mom holds ns*10 node arrays
 * (species-major, interpP2G order; Jx..Jz and pxx..pzz are read), fld the
 * six field node arrays (Bxn..Bzn are read), rhoc the net charge density on
 * the cell centres, flat [nxc+2][nyc+2][nzc+2]; qom[ns] the species'
 * charge-to-mass ratios, th the implicitness parameter theta. Writes the node
 * arrays jxh, jyh, jzh and the centre array rhoh. Returns 0, -1 when out of
 * memory. */
int orc_hat_densities(const orc_setup *s, double th, int ns, const double *qom,
                      const void *const *mom, const void *const fld[6], const void *rhoc,
                      void *jxh, void *jyh, void *jzh, void *rhoh);

/* Number of OpenMP threads the library will use. */
int orc_num_threads(void);

/* sizeof(ORC_FP) of the loaded library: 4 (FP32 variant) or 8 (FP64 variant). */
int orc_fp_bytes(void);

#ifdef __cplusplus
}
#endif
#endif
