// Launchers of the kernels, one declaration per kernel family.
#pragma once

#include "common.h"

namespace spb {

// plain_kernels.cu
int launch_pack_fields(const float *const f[6], float4 *eb4, float2 *eb2, long nodes,
                       cudaStream_t s);
int launch_plain_mover(const GeomDev &g, const PushDev &p, const PackedFields &F, float *x,
                       float *y, float *z, float *u, float *v, float *w, long n, int *err,
                       cudaStream_t s, int bc_variant = 0);
// particle_sort.cu: particle_sort's bins (src/Particles.cpp:158-163).
struct SortBins {
  int nb[3];       // bins per axis
  float dist[3];   // bin widths, rounded to float as the reference does
};
size_t particle_sort_scratch_bytes(long n);
// Sorts arr[0..6] (x, y, z, u, v, w, q; n each) by bin, stably; tmp: seven
// arrays of n floats; scratch: particle_sort_scratch_bytes(n). Queued on st in
// stream order (the caller synchronises before it frees tmp or scratch).
int device_particle_sort(float *const arr[7], float *const tmp[7], long n, const SortBins &B,
                         void *scratch, cudaStream_t st);

// net[m*nodes + i] = sum over species s (in order) of bases[s][m*nodes + i].
int launch_sum_species(const float *const *bases, int ns, long nodes, float *net,
                       cudaStream_t s);
// Scratch from the device's stream-ordered pool on stream s (which keeps freed
// memory for reuse), or nullptr when it cannot be had; pool_free returns it in
// stream order.
void *pool_alloc(size_t bytes, cudaStream_t s);
void pool_free(void *p, cudaStream_t s);
// The plain deposit's accumulator: a zeroed node-interleaved buffer (the ten
// moments of a node side by side, 48 bytes per node) from the device's
// stream-ordered pool on stream s, or nullptr when it cannot be had (the
// deposits then add straight into the moment arrays).
float *plain_acc_alloc(const GeomDev &g, cudaStream_t s);
// Adds the accumulator into mom[0..9] and returns it to the pool (nothing
// for nullptr).
int plain_acc_fold(float *acc, const GeomDev &g, float *const mom[10], cudaStream_t s);
// interpP2G / mover_interp deposits into acc (mom when acc is nullptr).
int launch_plain_p2g_into(const GeomDev &g, const float *x, const float *y, const float *z,
                          const float *u, const float *v, const float *w, const float *q, long n,
                          float *acc, float *const mom[10], int *err, cudaStream_t s);
int launch_plain_mover_interp_into(const GeomDev &g, const PushDev &p, const PackedFields &F,
                                   float *x, float *y, float *z, float *u, float *v, float *w,
                                   const float *q, long n, float *acc, float *const mom[10],
                                   int *err, cudaStream_t s);
// The same with their own accumulator: allocate, deposit, fold.
int launch_plain_p2g(const GeomDev &g, const float *x, const float *y, const float *z,
                     const float *u, const float *v, const float *w, const float *q, long n,
                     float *const mom[10], int *err, cudaStream_t s);
int launch_plain_mover_interp(const GeomDev &g, const PushDev &p, const PackedFields &F,
                              float *x, float *y, float *z, float *u, float *v, float *w,
                              const float *q, long n, float *const mom[10], int *err,
                              cudaStream_t s);
int launch_apply_bc_ids(int nxn, int nyn, int nzn, const int periodic[3],
                        float *const mom[10], cudaStream_t s, long *launches);

// The reference's time-step constants (src/Mover.cpp:11-12) for one species.
PushDev make_push(const spb_push &p);

}  // namespace spb
