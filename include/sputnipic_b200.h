/*
 * libsputnipic_b200: B200 (sm_100a) particle mover and particle-to-grid (P2G)
 * moment deposition for sputniPIC, behind the reference's own entry points.
 *
 * Boundary. The reference exposes the hot path as C-style free functions over
 * plain structs (include/Mover.h:11-26):
 *
 *   int  mover_PC(struct particles*, struct EMfield*, struct grid*, struct parameters*);
 *   int  mover_PC_V(struct particles*, struct EMfield*, struct grid*, struct parameters*);
 *   void interpP2G(struct particles*, struct interpDensSpecies*, struct grid*);
 *   int  mover_interp(struct particles*, struct EMfield*, struct interpDensSpecies*,
 *                     struct grid*, struct parameters*);
 *
 * The library exports those four symbols with C++ linkage (the reference is
 * compiled as C++), so the unchanged driver links against this library in
 * place of src/Mover.cpp, and an extern "C" twin of each (spb_*) for FFI.
 * Struct layouts: include/sputnipic_ref_layout.h (or the reference's own
 * headers). Every other entry point below uses plain pointers and sizes.
 *
 * Errors. The reference exits the process on a CUDA error
 * (include/gpu/cuda_helper.h:14-21). Here every call returns a status
 * (0 = SPB_OK); interpP2G, which returns void, leaves its status in
 * spb_last_error(). Nothing in the library exits, aborts or traps.
 *
 * Threading. The reference driver calls interpP2G from an OpenMP team over
 * species (src/sputniPIC_CPU.cpp:250-256). All entry points are thread-safe;
 * calls on different species run on their own CUDA streams.
 */
#ifndef SPUTNIPIC_B200_H
#define SPUTNIPIC_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

struct particles;
struct EMfield;
struct grid;
struct interpDensSpecies;
struct parameters;

/* ---------------------------------------------------------------------------
 * Status codes
 * ------------------------------------------------------------------------- */
enum spb_status {
  SPB_OK = 0,
  SPB_ERR_CUDA = 1,          /* a CUDA runtime call failed */
  SPB_ERR_INVALID = 2,       /* bad argument (null pointer, size, layout) */
  SPB_ERR_OUT_OF_GRID = 3,   /* a particle's cell index left the node array;
                                the reference reads out of bounds there */
  SPB_ERR_NO_DEVICE = 4,     /* no CUDA device */
  SPB_ERR_ALLOC = 5,         /* device or pinned allocation failed */
  SPB_ERR_UNSUPPORTED = 6,   /* configuration outside what the kernels cover */
  SPB_ERR_TIMEOUT = 7,       /* a bounded device wait gave up */
  SPB_ERR_CAPACITY = 8       /* a request exceeds a fixed capacity */
};

/* Status of the calling thread's most recent failing call (sticky until
 * spb_clear_error), with a one-line message. */
int spb_last_error(void);
const char *spb_last_error_message(void);
void spb_clear_error(void);
const char *spb_error_string(int status);

/* Library version string and the sm architecture it was built for. */
const char *spb_version(void);

/* Number of kernels this library has launched in this process. */
long spb_launch_count(void);

/* How the plain interpP2G / mover_interp deposits (process-wide):
 * SPB_DEPOSIT_ACCUMULATOR (default) adds into a node-interleaved buffer of
 * 48 bytes per node from the device's stream-ordered pool, then into the
 * ten moment arrays (fewer L2 transactions); SPB_DEPOSIT_DIRECT adds straight
 * into the ten arrays and needs no memory. The accumulator form falls back to
 * the direct one when its buffer cannot be allocated. Returns the previous
 * mode, or SPB_ERR_INVALID for an unknown mode. */
enum { SPB_DEPOSIT_ACCUMULATOR = 0, SPB_DEPOSIT_DIRECT = 1 };
int spb_set_plain_deposit_mode(int mode);

/* JSON object: "struct.member": offset for every member of the boundary
 * structs as this library lays them out (see sputnipic_ref_layout.h). */
const char *spb_abi_layout_json(void);

/* Select the CUDA device used by the drop-in entry points (default 0). */
int spb_set_device(int device);

/* ---------------------------------------------------------------------------
 * Drop-in entry points, extern "C" twins of the reference functions.
 * Replace: include/Mover.h:11 (mover_PC), :16 (mover_PC_V), :20 (interpP2G),
 * :24 (mover_interp); bodies src/Mover.cpp:4-162, :166-382, :385-572, :575-862.
 *
 * Semantics match the reference's CPU functions: mover_PC updates
 * part->x..w in place (NiterMover predictor-corrector iterations, one pass,
 * particle BC from param->PERIODICX/Y/Z); interpP2G ADDS the ten moments of
 * every particle into ids->rhon..pzz (the caller zeroes them and applies
 * applyBCids afterwards); mover_interp does both per particle.
 * Arithmetic: float with the reference's double promotions, no FMA
 * contraction, so particle outputs are bit-identical to the reference CPU
 * code. Moments are FP32 sums in a different order (within tolerance).
 * ------------------------------------------------------------------------- */
int spb_mover_PC(struct particles *part, struct EMfield *field, struct grid *grd,
                 struct parameters *param);
int spb_mover_PC_V(struct particles *part, struct EMfield *field,
                   struct grid *grd, struct parameters *param);
void spb_interpP2G(struct particles *part, struct interpDensSpecies *ids,
                   struct grid *grd);
int spb_mover_interp(struct particles *part, struct EMfield *field,
                     struct interpDensSpecies *ids, struct grid *grd,
                     struct parameters *param);

/* The reference driver's moment section in one call (no single reference
 * function: it replaces src/sputniPIC_CPU.cpp:247-259): setZeroDensities
 * (src/InterpDensNet.cpp:113-117), interpP2G of species 0..param->ns-1 into
 * zeroed device moments, applyBCids per species (src/BC.cpp:362-615) and
 * sumOverSpecies (src/InterpDensNet.cpp:120-146) on the device; the species'
 * and net host arrays are written once (rhoc of both zeroed, as
 * setZeroDensities does). applyBCids and sumOverSpecies are bit-identical to
 * the reference on the same deposit; the deposit is interpP2G's. */
struct interpDensNet;
int spb_interp_all_species(struct particles *part, struct interpDensSpecies *ids,
                           struct interpDensNet *idn, struct grid *grd,
                           struct parameters *param);

/* particle_sort (src/Particles.cpp:72-234; declared in include/Particles.h)
 * on the device: particles ordered by bin of param->sort_cps cells per axis,
 * stably, particles outside every bin last, over all part->npmax entries, with
 * the reference's float arithmetic for the bins (bit-identical order). Named
 * spb_particle_sort, not particle_sort, because src/Particles.cpp, which the
 * driver keeps, defines that symbol. */
int spb_particle_sort(struct parameters *param, struct particles *part, struct grid *grd);

/* calculateHatDensities (src/MaxwellSolver.cpp:465-603; declared in
 * include/MaxwellSolver.h:37-40), the field solver's first consumer of the
 * moments: J hat on the nodes (the divergence of each species' pressure tensor
 * scaled by -dt/2 and interpolated to the nodes, plus its J, rotated with the
 * species' qom dt B / 2c and summed over species; node guards filled as
 * applyBCscalarDensN) and rho hat = rho_c - dt theta div(J hat) on the cell
 * centres (guards filled as applyBCscalarDensC). Bit-identical to the
 * reference's FP32 build (and, with double arrays, its FP64 build).
 *
 * spb_calculateHatDensities is the drop-in over the reference's host structs
 * (reads ids[0..param->ns-1] J and pressures, field->B*n, idn->rhoc; writes
 * id_aux->Jxh/Jyh/Jzh/rhoh); the C++-linkage calculateHatDensities below
 * has the reference's signature. The spb_hat_densities_* entry points work
 * on device arrays: mom holds ns*10 device pointers (species-major, the
 * interpP2G moment order; entries 1..9 are read), B the three magnetic
 * field node arrays, rhoc the centre array [nxc][nyc][nzc] (guards
 * included); outputs as the drop-in's. Asynchronous on `stream`. */
struct interpDens_aux;
#define SPB_HAT_MAX_SPECIES 16
typedef struct spb_hat_desc {
  int nxc, nyc, nzc;           /* cells per axis, guard cells included (grid.nxc) */
  double invdx, invdy, invdz;  /* the grid's inverse spacings (grid.invdx) */
  int periodic[3];             /* param.PERIODICX/Y/Z */
  double dt, c, th;            /* param.dt, param.c, param.th */
  int ns;                      /* species, 1..SPB_HAT_MAX_SPECIES */
  double qom[SPB_HAT_MAX_SPECIES];
} spb_hat_desc;
int spb_calculateHatDensities(struct interpDens_aux *id_aux, struct interpDensNet *idn,
                              struct interpDensSpecies *ids, struct EMfield *field,
                              struct grid *grd, struct parameters *param);
int spb_hat_densities_f32(const spb_hat_desc *d, const float *const *mom,
                          const float *const B[3], const float *rhoc, float *jxh, float *jyh,
                          float *jzh, float *rhoh, void *stream);
int spb_hat_densities_f64(const spb_hat_desc *d, const double *const *mom,
                          const double *const B[3], const double *rhoc, double *jxh,
                          double *jyh, double *jzh, double *rhoh, void *stream);

/* Host coherence of the drop-in. COPY (default): particles are uploaded and
 * downloaded on every call, so the host arrays are always current. DEVICE:
 * particles stay in HBM between calls; the host arrays are refreshed only by
 * spb_sync_particles_to_host (call it before particle_sort or particle IO),
 * and spb_invalidate_particles must follow any host-side change. */
enum spb_residency { SPB_RESIDENCY_COPY = 0, SPB_RESIDENCY_DEVICE = 1 };
int spb_set_residency(int mode);
int spb_sync_particles_to_host(struct particles *part);
int spb_invalidate_particles(struct particles *part);
/* Free every device mirror and stream the drop-in holds. */
int spb_release_all(void);

/* ---------------------------------------------------------------------------
 * Device-pointer API of the plain form (reference precision types, arrays in
 * HBM). A grid context holds the grid geometry, the node coordinates and
 * the packed E/B fields on one device.
 * Replaces the reference GPU build's per-batch staging path
 * (src/gpu/Particles_gpu.cu:221-287, batch_update_particles) and its kernel
 * move_and_interpolate (src/gpu/Particles_gpu.cu:291-577).
 * `stream` is a cudaStream_t (NULL = legacy default stream).
 * ------------------------------------------------------------------------- */
typedef struct spb_grid_ctx spb_grid_ctx;

/* Time-step parameters of one species' push. */
typedef struct spb_push {
  double dt;          /* param->dt */
  double c;           /* param->c */
  float qom;          /* part->qom */
  int niter;          /* part->NiterMover (>= 1) */
  int n_sub_cycles;   /* part->n_sub_cycles (>= 1; divides dt only) */
  int periodic[3];    /* param->PERIODICX/Y/Z */
} spb_push;

/* Build a context from a host `struct grid` (setGrid output). The node
 * coordinate arrays must be separable (XN depends on i only, and so on),
 * which setGrid guarantees (src/Grid.cpp:53-61). */
int spb_grid_create(const struct grid *grd, spb_grid_ctx **out);
/* Same, from scalars: active cells and lengths, as setGrid computes them. */
int spb_grid_create_uniform(int nxc, int nyc, int nzc, double Lx, double Ly,
                            double Lz, spb_grid_ctx **out);
void spb_grid_destroy(spb_grid_ctx *ctx);
/* Number of nodes nxn*nyn*nzn. */
long spb_grid_nodes(const spb_grid_ctx *ctx);
/* Upload and pack the six node fields (Ex, Ey, Ez, Bxn, Byn, Bzn; each
 * nodes floats). `on_device` != 0: the pointers are device pointers. */
int spb_grid_set_fields(spb_grid_ctx *ctx, const float *const fields[6],
                        int on_device, void *stream);
/* mover_PC over n particles in device memory. */
int spb_grid_mover(spb_grid_ctx *ctx, const spb_push *push, float *x, float *y,
                   float *z, float *u, float *v, float *w, long n, void *stream);
/* interpP2G over n particles: ADDS into mom[0..9] (device, nodes floats each,
 * anywhere in memory; order rhon, Jx, Jy, Jz, pxx, pxy, pxz, pyy, pyz, pzz).
 * The deposit accumulates into a node-interleaved buffer (48 bytes per node,
 * from the device's stream-ordered pool on `stream`), which a second kernel
 * adds into the ten arrays. */
int spb_grid_p2g(spb_grid_ctx *ctx, const float *x, const float *y,
                 const float *z, const float *u, const float *v, const float *w,
                 const float *q, long n, float *const mom[10], void *stream);
/* mover_interp: move then deposit, one kernel (plus the accumulator fold, as
 * spb_grid_p2g). */
int spb_grid_mover_interp(spb_grid_ctx *ctx, const spb_push *push, float *x,
                          float *y, float *z, float *u, float *v, float *w,
                          const float *q, long n, float *const mom[10],
                          void *stream);
/* applyBCids (src/BC.cpp:362-615) on device moments, for callers that keep
 * the moments in HBM. periodic = param->PERIODICX/Y/Z. */
int spb_grid_apply_bc_ids(spb_grid_ctx *ctx, const int periodic[3],
                          float *const mom[10], void *stream);
/* Synchronise `stream` and report SPB_ERR_OUT_OF_GRID if any kernel of this
 * context saw a cell index outside the node array since the last check
 * (such particles are clamped to the edge cell instead of reading out of
 * bounds). Clears the flag. */
int spb_grid_check(spb_grid_ctx *ctx, void *stream);
/* Kernel launches issued by this context since creation. */
long spb_grid_launches(const spb_grid_ctx *ctx);

/* ---------------------------------------------------------------------------
 * Precision form (device-resident simulation). Replaces, for callers that
 * keep particles in HBM across cycles, the per-cycle section of the CPU
 * driver that calls mover_PC and interpP2G for every species
 * (src/sputniPIC_CPU.cpp:232-256; src/Mover.cpp:4-162 and :385-572).
 *
 * Particles live in HBM bucketed by cell: every cell owns a fixed number of
 * record slots (two float4 per particle: FP32 in-cell offsets, charge,
 * velocities; the cell is implicit), cells numbered tile-major; particles that
 * find their cell's bucket full go to a per-species overflow list. A cycle is
 * two kernels: the push runs the NiterMover predictor-corrector (FP32, E/B
 * gathered from a TMA-staged tile of nodes) and writes every particle into
 * the bucket of its new cell in a second buffer set, so the particles stay
 * grouped by cell with no sort; the deposit sums each cell's bucket in
 * registers (FP32) and adds the node sums into FP64 global moments.
 * Moments are the raw interpP2G sums (zeroed at the start of every cycle, no
 * applyBCids), FP64, [10][nxn*nyn*nzn] per species in the reference order.
 * ------------------------------------------------------------------------- */
typedef struct spb_sim spb_sim;

#define SPB_SIM_MAX_SPECIES 8

typedef struct spb_sim_desc {
  int nxc, nyc, nzc;        /* active cells; multiples of the tile shape */
  double Lx, Ly, Lz;
  double dt, c;             /* param->dt (divided by part->n_sub_cycles when
                               the species sub-cycle: mover_PC's time step,
                               src/Mover.cpp:11), param->c */
  int niter;                /* NiterMover (param->NiterMover, which
                               particle_allocate gives every species) */
  int periodic[3];          /* param->PERIODICX/Y/Z */
  int ns;                   /* species, 1..8 */
  double qom[SPB_SIM_MAX_SPECIES];
  long capacity[SPB_SIM_MAX_SPECIES]; /* optional: particles a species' buffers
                               are sized for at its first load (at least the
                               loaded count), so that reloading it with up to
                               that many particles reallocates nothing */
  int tile[3];              /* cells per tile (0,0,0: default 8x4x4) */
  int resort_every;         /* cycles between overflow checks (>= 1): a species
                               whose overflow list holds more than 1/256 of
                               its particles (at least 256, at most a quarter
                               of the list) is re-laid out */
  int ctas;                 /* persistent CTAs of the push (0: per variant) */
  int variant;              /* push kernel residency: 0 three CTAs per SM (up
                               to 80 registers, 2 KB record-ring halves),
                               1 two (up to 128, 4 KB halves), 2 four (up to
                               64, 2 KB halves) */
  int bucket_slots;         /* record slots of every cell's bucket (0: each
                               cell's count at the last layout + max(16,
                               count/2), rounded up to 4) */
  int graph;                /* 1: each cycle's launches (zeroing, push,
                               deposit) replay as a CUDA graph captured per
                               buffer-parity pattern; not while timing */
  int deterministic;        /* 1: bitwise reproducible moments. Every deposit
                               term is rounded down to a power-of-two grid
                               (2^-38 of the species' largest possible term of
                               that moment at load: |q|max for rhon, |q|max x
                               4 |v|max for J, |q|max x 16 |v|max^2 for the
                               pressures, |v|max the largest velocity
                               component at load but at least c/8, so that a
                               species loaded at rest keeps room for the
                               velocities it gains; the rounding's average loss,
                               half a grid step per term, is added back) and
                               summed exactly
                               in FP64, so the moments do not depend on the
                               particles' order in their buckets or on the
                               order of the atomics; the push gives every
                               particle the same result on every path. Two
                               runs from the same inputs give identical
                               moments and the same particles. One thread per
                               cell with 80 FP64 sums: slower than the default
                               deposit. spb_sim_check reports SPB_ERR_CAPACITY
                               if a sum ever left its exact range. */
  int fused;                /* 1: each cycle is one persistent cooperative
                               launch (the batching form): every CTA pushes a
                               tile, then deposits the tile it pushed
                               ceil(R/G) steps earlier once the 27 tiles around
                               it are pushed, so the deposit overlaps the
                               push; overflow entries are pushed and deposited
                               after two grid barriers. Not with
                               deterministic. */
  int overflow_per_mille;   /* overflow list entries per 1000 particles of a
                               species, at least 65536 entries (0: about one
                               per 32 particles; a fixed bucket_slots makes
                               it one per particle). A species is re-laid out
                               once its list passes 1/256 of its particles,
                               so the default leaves 8x that for the cycles
                               until the check that sees it */
} spb_sim_desc;

/* Whether a tile shape has an instantiated kernel. */
int spb_sim_tile_supported(int tx, int ty, int tz);
int spb_sim_create(const spb_sim_desc *desc, spb_sim **out);
void spb_sim_destroy(spb_sim *sim);
long spb_sim_nodes(const spb_sim *sim);
long spb_sim_count(const spb_sim *sim, int species);
/* Kernel launches issued by this simulation. */
long spb_sim_launches(const spb_sim *sim);
/* Six node fields (Ex, Ey, Ez, Bxn, Byn, Bzn), nodes floats each. */
int spb_sim_set_fields(spb_sim *sim, const float *const fields[6], int on_device,
                       void *stream);
/* Load one species from reference-style float arrays (positions in domain
 * units, inside [0, L]); converts to cell + offset and lays the particles out
 * in buckets (synchronises `stream`). */
int spb_sim_load_species(spb_sim *sim, int species, const float *x, const float *y,
                         const float *z, const float *u, const float *v,
                         const float *w, const float *q, long n, int on_device,
                         void *stream);
/* ncycles of mover + deposit for all species (the last cycle's moments
 * remain). Every desc.resort_every cycles the overflow lists are checked
 * (a synchronisation) and species whose list is past its threshold are
 * re-laid out, which resizes every cell's bucket to its current count plus
 * slack. Overflow entries are pushed and deposited exactly in the meantime. */
int spb_sim_cycle(spb_sim *sim, int ncycles, void *stream);
/* Re-lay out every species now: buckets sized from the current counts, the
 * buckets and the overflow list copied into them (queued on `stream`; the
 * buffer sets sized at the load hold any layout of the species). */
int spb_sim_resort(spb_sim *sim, void *stream);
/* Record slots of a species' bucket layout, summed over the cells (-1: bad
 * arguments; synchronises the device the first time after a load or
 * re-layout). */
long spb_sim_bucket_slots(spb_sim *sim, int species);
/* Entries in a species' overflow list (synchronises `stream`; -1 on error). */
long spb_sim_overflow(spb_sim *sim, int species, void *stream);
/* FP64 moments of a species: 10*nodes doubles. */
int spb_sim_moments(spb_sim *sim, int species, double *out, int on_device,
                    void *stream);
/* applyBCids (src/BC.cpp:362-615) on a species' FP64 moments, in place. */
int spb_sim_apply_bc_ids(spb_sim *sim, int species, void *stream);
/* Device address of a species' FP64 moments ([10][nodes], reference order),
 * valid until spb_sim_destroy; NULL on a bad argument. The caller may read
 * or update them in place between cycles, as the reference's
 * mpi_reduce_densities (src/mpi_comm.cpp:58-117) sums the ranks' moments
 * into ids[is] after interpP2G (src/sputniPIC_CPU.cpp:262-265); the next
 * cycle zeroes them. */
double *spb_sim_moments_device(spb_sim *sim, int species);
/* Positions x = (cell + offset) * dx, velocities and (if q is not NULL)
 * charges, as floats: cells in tile-major order, each cell's particles in
 * bucket order, then the overflow list. */
int spb_sim_particles(spb_sim *sim, int species, float *x, float *y, float *z,
                      float *u, float *v, float *w, float *q, int on_device,
                      void *stream);
/* Synchronise; SPB_ERR_OUT_OF_GRID / SPB_ERR_TIMEOUT from the kernels. */
int spb_sim_check(spb_sim *sim, void *stream);
/* CUDA-event timing of the cycle kernels (push + deposit) and of the
 * re-layouts, recorded on the launching stream while enabled. The queries
 * synchronise, return the summed milliseconds and counts since the last
 * query, and clear them. */
int spb_sim_set_timing(spb_sim *sim, int on);
int spb_sim_timing(spb_sim *sim, double *cycle_ms, int *ncycle, double *sort_ms,
                   int *nsort);
int spb_sim_kernel_timing(spb_sim *sim, double *push_ms, double *deposit_ms,
                          int *ncycles, double *relayout_ms, int *nrelayouts);

/* ---------------------------------------------------------------------------
 * Serving form: a stream of independent frozen-field test-particle jobs (the
 * reference's particle tracking use, src/Tracking.cpp), each with its own
 * grid, fields, species and cycle count. No counterpart in the reference's
 * hot path, which runs one simulation.
 *
 * Jobs wait in a queue until their estimated HBM footprint fits the engine's
 * budget, are then admitted (fields and particles uploaded into device-
 * resident precision-form state), and run together: every spb_serve_step runs
 * one cycle of every admitted job in one launch each of zeroing, push and
 * deposit (the jobs' tiles concatenated), so jobs that arrive while others run
 * join the next step. A job finishes after its cycle count; its results stay
 * on the device until fetched and released. One host thread drives an engine;
 * calls must not overlap. All jobs of an engine use its tile shape, so their
 * cells per axis must be multiples of it.
 * ------------------------------------------------------------------------- */
typedef struct spb_serve spb_serve;

/* Returns the device memory that the library's allocation pool holds but no
 * simulation uses (after a device synchronisation). Simulations keep freed
 * memory in the pool, so that creating and destroying them maps nothing. */
int spb_release_cached_memory(void);

typedef struct spb_serve_desc {
  int tile[3];              /* tile shape of every job (0,0,0: 4x4x4) */
  long long hbm_budget;     /* bytes the admitted jobs may hold (0: 90% of the
                               device memory free at creation, counting what
                               the device's memory pool holds unused) */
  int max_jobs;             /* jobs per launch (0 or above 64: 64) */
  int check_every;          /* a job's cycles between checks of its overflow
                               lists (0: 4); a job gets further cycles in a
                               step only while its last evaluated check is
                               less than 2 x check_every cycles old */
  long long reserve_bytes;  /* device memory the library's pool maps up front
                               (0: none), so that admitting jobs maps nothing;
                               spb_release_cached_memory gives it back */
  double extra_budget;      /* after a step's launch of every admitted job,
                               up to 7 further launches: each gives one more
                               cycle to every job with cycles left whose cost
                               still fits (cost of a cycle: particles + 4 x
                               cells; cheapest jobs first), while the added
                               cost stays within this multiple of the first
                               launch's. Once the largest job no longer fits,
                               the smaller ones keep getting cycles, so they
                               are not paced by it. 0: 1.0; negative: one
                               cycle per job and step */
} spb_serve_desc;

typedef struct spb_job_desc {
  int nxc, nyc, nzc;        /* active cells */
  double Lx, Ly, Lz;
  double dt, c;             /* param->dt, param->c */
  int niter;                /* NiterMover */
  int periodic[3];          /* param->PERIODICX/Y/Z */
  int ns;                   /* species, 1..8 */
  double qom[SPB_SIM_MAX_SPECIES];
  int ncycles;              /* cycles to run (>= 1) */
} spb_job_desc;

enum { SPB_JOB_PENDING = 0, SPB_JOB_ACTIVE = 1, SPB_JOB_DONE = 2, SPB_JOB_FAILED = 3 };

int spb_serve_create(const spb_serve_desc *desc, spb_serve **out);
void spb_serve_destroy(spb_serve *srv);
/* Queues a job. fields: Ex, Ey, Ez, Bxn, Byn, Bzn (nodes floats each);
 * parts: ns x 7 arrays x, y, z, u, v, w, q (positions in [0, L]); counts[ns].
 * The arrays stay the caller's and must stay valid until the job leaves the
 * queue (status not PENDING). Returns the job id (>= 0) or -status. */
long spb_serve_submit(spb_serve *srv, const spb_job_desc *job, const float *const fields[6],
                      const float *const *parts, const long *counts, int on_device);
/* Launches one cycle of every admitted job (and more for the cheap ones, see
 * extra_budget) and, while they run, admits the queued jobs that fit (in
 * order of arrival; they upload on a stream of their own and join the next
 * step). It waits for the previous step's launches, not its own, so the host
 * prepares the next step while the device runs this one; a job whose last
 * cycle is launched finishes (DONE, or FAILED with its error) once its work
 * has completed, seen at a later step, or at this one when nothing else is
 * left to run. Returns the number of jobs admitted and not yet finished, or
 * -status. */
int spb_serve_step(spb_serve *srv);
/* Ids of the jobs that finished (DONE or FAILED) since the last call, at
 * most max of them, oldest first; returns how many (or -status). */
int spb_serve_finished(spb_serve *srv, long *ids, int max);
/* SPB_JOB_*, or -1 for an unknown id. */
int spb_serve_status(const spb_serve *srv, long id);
/* Status code of a failed job (why it failed). */
int spb_serve_error(const spb_serve *srv, long id);
/* Results of a finished job: particles of one species (as spb_sim_particles,
 * any pointer may be NULL) and its raw FP64 moments of the last cycle
 * (10 x nodes, NULL to skip). Synchronises. */
int spb_serve_result(spb_serve *srv, long id, int species, float *x, float *y, float *z,
                     float *u, float *v, float *w, float *q, double *moments,
                     int on_device);
/* Seconds since the engine's creation at which the job was submitted,
 * admitted and finished (negative where not yet). */
int spb_serve_times(const spb_serve *srv, long id, double t[3]);
/* Frees a finished or failed job. */
int spb_serve_release(spb_serve *srv, long id);
/* Steps run, then host seconds spent in admitting jobs, overflow checks,
 * the launches and their completion, and retiring jobs (5 values). */
int spb_serve_stats(const spb_serve *srv, double out[5]);
/* Jobs queued, admitted and finished (not yet released); bytes held by the
 * admitted and finished jobs, and the budget. */
int spb_serve_counts(const spb_serve *srv, int *pending, int *active, int *done,
                     long long *bytes_held, long long *budget);

/* ---------------------------------------------------------------------------
 * Particle load + cell sort that allocates nothing. No counterpart in the
 * reference: it is the conversion and counting sort behind
 * spb_sim_load_species, for callers that cannot call cudaMalloc where they
 * sort (codes that hand all device memory to their own pool allocator at
 * start-up, or loops that cannot afford an allocation's implicit
 * synchronisation). The caller passes inputs (reference-layout positions in
 * [0, L], velocities, charges; device pointers) and outputs (precision-form
 * arrays of n elements, cell_start of nxc*nyc*nzc + 1 ints); only desc's
 * grid and tile fields are read. Scratch is a fixed __device__ array for at
 * most SPB_NOALLOC_MAX_CELLS cells (about 8 MB per device, held until the
 * process exits); larger grids return SPB_ERR_CAPACITY. All calls share that
 * array: calls that overlap on the GPU race. The first call on a device
 * looks up the array's device address, so make it before any stream capture.
 * The call synchronises `stream` before returning.
 * ------------------------------------------------------------------------- */
#define SPB_NOALLOC_MAX_CELLS (1L << 20)
int spb_sort_particles_noalloc(const spb_sim_desc *desc, const float *x,
                               const float *y, const float *z, const float *u,
                               const float *v, const float *w, const float *q,
                               long n, uint32_t *cell, float *ox, float *oy,
                               float *oz, float *u_out, float *v_out,
                               float *w_out, float *q_out, int *cell_start,
                               void *stream);

/* ---------------------------------------------------------------------------
 * Seeded synthetic GEM (Harris current sheet) inputs, generated on the device.
 * No counterpart in the reference's hot path: the reference builds its inputs
 * on the host with initGEM (src/IC.cpp:7-188). Same hash and formulas as
 * sputnipic_b200/workload.py.
 * ------------------------------------------------------------------------- */
typedef struct spb_gem_desc {
  int nxc, nyc, nzc;        /* active cells */
  double Lx, Ly, Lz;
  double B0, delta, pert;   /* Harris sheet amplitude, width, flux perturbation */
  double E_amp;             /* E ~ U(-E_amp, E_amp) per node and axis */
  int lattice;              /* 0: uniform in the cell; m: m^3 jittered sub-lattice */
  unsigned long long seed;
} spb_gem_desc;

typedef struct spb_gem_species {
  double qom, rho0, vth, w0, ppc;
  int sheet;                /* 1: sech^2 current sheet density, 0: uniform */
} spb_gem_species;

/* Particles of one species in the whole grid: floor(cells * ppc). */
long spb_gem_species_count(const spb_gem_desc *d, const spb_gem_species *sp);
/* Fields on all nodes: six device arrays of nxn*nyn*nzn floats. */
int spb_gen_gem_fields(const spb_gem_desc *d, float *const fields[6], void *stream);
/* Particles [first, first+count) of species `species` (cells in x-major
 * order) into device arrays; `cell` (optional) receives the active-cell
 * index of each particle. */
int spb_gen_gem_particles(const spb_gem_desc *d, const spb_gem_species *sp,
                          int species, long first, long count, float *x, float *y,
                          float *z, float *u, float *v, float *w, float *q,
                          int *cell, void *stream);

#ifdef __cplusplus
} /* extern "C" */

/* C++-linkage drop-ins with the reference's exact signatures, so objects
 * compiled against the reference's include/Mover.h link to this library. */
int mover_PC(struct particles *part, struct EMfield *field, struct grid *grd,
             struct parameters *param);
int mover_PC_V(struct particles *part, struct EMfield *field, struct grid *grd,
               struct parameters *param);
void interpP2G(struct particles *part, struct interpDensSpecies *ids,
               struct grid *grd);
int mover_interp(struct particles *part, struct EMfield *field,
                 struct interpDensSpecies *ids, struct grid *grd,
                 struct parameters *param);
void calculateHatDensities(struct interpDens_aux *id_aux, struct interpDensNet *idn,
                           struct interpDensSpecies *ids, struct EMfield *field,
                           struct grid *grd, struct parameters *param);
#endif

#endif /* SPUTNIPIC_B200_H */
