// Precision form: device data layout and the fused mover + deposit kernel.
//
// Particles (per species, HBM-resident SoA, cell-sorted):
//   cell  uint32  packed active-cell coordinates cz | cy << 11 | cx << 21
//   ox, oy, oz    float in-cell offsets in cell units, [0, 1]
//   u, v, w       float velocities
//   q             float charge x statistical weight
// Fields: one 32-byte record per node (Ex, Ey, Ez, Bx, By, Bz, 0, 0), the
// reference node layout [nxn][nyn][nzn] (include/Alloc.h:111-124).
// Moments: FP64 [10][nxn*nyn*nzn] per species, the reference order
// rhon, Jx, Jy, Jz, pxx, pxy, pxz, pyy, pyz, pzz (src/Mover.cpp:466-570).
//
// The kernel: persistent CTAs walk tiles of TX x TY x TZ cells. For each tile
// one thread stages the tile's E/B nodes plus a one-cell halo into shared
// memory with a TMA tensor copy; then, species by species, the warps walk the
// tile's cells (particles are sorted tile-major, so every cell is one
// contiguous segment) and push 4 consecutive particles per lane, read and
// written with 128-bit accesses. The NiterMover predictor-corrector
// iterations gather from the staged tile (or from L2 past the halo). The
// deposit of particles that end in their segment's cell accumulates in
// registers and is summed over the warp by recursive halving; particles that
// changed cell go through a per-warp queue and shared-memory atomics. The
// FP32 shared-memory partials of the tile are added to the FP64 global
// moments with double atomics.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "common.h"

namespace spb {

constexpr int SIM_MAX_SPECIES = 8;

__host__ __device__ __forceinline__ uint32_t pack_cell(int cx, int cy, int cz) {
  return (uint32_t)cz | ((uint32_t)cy << 11) | ((uint32_t)cx << 21);
}
__host__ __device__ __forceinline__ int cell_x(uint32_t c) { return (int)(c >> 21); }
__host__ __device__ __forceinline__ int cell_y(uint32_t c) { return (int)((c >> 11) & 1023u); }
__host__ __device__ __forceinline__ int cell_z(uint32_t c) { return (int)(c & 2047u); }

struct SpeciesDev {
  uint32_t *cell;
  float *ox, *oy, *oz, *u, *v, *w, *q;
  const int *cell_start;  // [ncells + 1] tile-major segment starts
  double *mom;            // [10][nodes]
  long n;
  float qomdt2;
  float fix;              // fixed-point scale of the tile partials: 2^40 / max|q| (power of 2)
  double unfix;           // invVOL / fix, applied when the partials are flushed
};

struct CycleParams {
  int nxc, nyc, nzc;          // active cells
  int nxn, nyn, nzn;          // nodes
  int ntx, nty, ntz;          // tiles per axis
  int niter;
  int periodic[3];
  float hdt[3];               // (dt/2)/d per axis: half-step displacement per unit velocity
  float fdt[3];               // dt/d per axis
  double scale;               // invVOL in double, applied when the partials are flushed
  const float *fields8;       // packed node fields in HBM (gathers past the halo)
  int *err;
  int ns;
  SpeciesDev sp[SIM_MAX_SPECIES];
};

// Sort key: tile-major cell order.
template <int TX, int TY, int TZ>
__host__ __device__ __forceinline__ int tile_key(int cx, int cy, int cz, int nty, int ntz) {
  const int tx = cx / TX, ty = cy / TY, tz = cz / TZ;
  const int lx = cx % TX, ly = cy % TY, lz = cz % TZ;
  return ((tx * nty + ty) * ntz + tz) * (TX * TY * TZ) + (lx * TY + ly) * TZ + lz;
}

}  // namespace spb
