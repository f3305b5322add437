// Precision form: device data layout of the mover + deposit.
//
// Particles (per species, HBM-resident, bucketed by cell):
//   cell k owns the record slots [base[k], base[k+1]); a record is two float4,
//   (ox, oy, oz, q) and (u, v, w, 0): in-cell offsets in cell units, charge x
//   statistical weight, velocities. A cell's particles are the first
//   min(count, capacity) slots of its bucket; the capacity is the cell's count
//   at the last layout plus slack, so memory stays ~1.25x the particles
//   however they cluster. Particles that find their cell's bucket full are
//   kept in a per-species overflow list (records + cell keys). Buckets are
//   double-buffered with one shared layout: a cycle reads one set and writes
//   every pushed particle straight into its new cell's bucket of the other,
//   so particles stay grouped by cell without a sort.
// Cells are numbered tile-major (tile_key): the cells of a TX x TY x TZ tile
// are consecutive, so a tile's buckets are one contiguous range.
// Fields: one 32-byte record per node (Ex, Ey, Ez, Bx, By, Bz, 0, 0), the
// reference node layout [nxn][nyn][nzn] (include/Alloc.h:111-124).
// Moments: FP64 [10][nxn*nyn*nzn] per species, the reference order
// rhon, Jx, Jy, Jz, pxx, pxy, pxz, pyy, pyz, pzz (src/Mover.cpp:466-570).
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "common.h"

namespace spb {

constexpr int SIM_MAX_SPECIES = 8;
constexpr int SERVE_MAX_JOBS = 64;   // jobs per multi-job launch

__host__ __device__ __forceinline__ uint32_t pack_cell(int cx, int cy, int cz) {
  return (uint32_t)cz | ((uint32_t)cy << 11) | ((uint32_t)cx << 21);
}
__host__ __device__ __forceinline__ int cell_x(uint32_t c) { return (int)(c >> 21); }
__host__ __device__ __forceinline__ int cell_y(uint32_t c) { return (int)((c >> 11) & 1023u); }
__host__ __device__ __forceinline__ int cell_z(uint32_t c) { return (int)(c & 2047u); }

struct SpeciesDev {
  const float4 *rin;   // buckets read this cycle, [slots][2]
  float4 *rout;        // buckets written this cycle (same layout)
  const long long *base;   // [ncells + 1] first slot of each cell's bucket
  const int *cin;      // per-cell fill counters of rin (may exceed the capacity: clamp)
  int *cout;           // per-cell fill counters of rout (zero at the start of the cycle)
  const float4 *oin;   // overflow records read this cycle, [ocap][2]
  const int *okin;     // their cell keys
  const int *ocin;     // overflow entries of oin (may exceed ocap: clamp)
  float4 *oout;        // overflow written this cycle
  int *okout;
  int *ocout;
  double *mom;         // [10][nodes]
  int ocap;
  float qomdt2;        // qom * (dt/2) / c
  double quantum[3];   // deterministic deposit: the grid every term of rhon,
                       // of Jx..Jz and of pxx..pzz is rounded down to (powers
                       // of two; see exact_terms)
};

struct CycleParams {
  int nxc, nyc, nzc;          // active cells
  int nxn, nyn, nzn;          // nodes
  int ntx, nty, ntz;          // tiles per axis
  int niter;
  int periodic[3];
  float hdt[3];               // (dt/2)/d per axis: half-step displacement per unit velocity
  float fdt[3];               // dt/d per axis
  double scale;               // invVOL in double, applied when cell sums reach the moments
  const float *fields8;       // packed node fields in HBM (gathers past the staged tile)
  int *err;
  int ns;
  SpeciesDev sp[SIM_MAX_SPECIES];
};

// Cell key: tile-major cell order. Tile extents are powers of two.
template <int TX, int TY, int TZ>
__host__ __device__ __forceinline__ int tile_key(int cx, int cy, int cz, int nty, int ntz) {
  const unsigned x = (unsigned)cx, y = (unsigned)cy, z = (unsigned)cz;
  const int tx = (int)(x / TX), ty = (int)(y / TY), tz = (int)(z / TZ);
  const int lx = (int)(x % TX), ly = (int)(y % TY), lz = (int)(z % TZ);
  return ((tx * nty + ty) * ntz + tz) * (TX * TY * TZ) + (lx * TY + ly) * TZ + lz;
}

template <int TX, int TY, int TZ>
__host__ __device__ __forceinline__ void key_cell(int key, int nty, int ntz, int &cx, int &cy,
                                                  int &cz) {
  constexpr int TC = TX * TY * TZ;
  const int t = key / TC, lc = key % TC;
  const int tz = t % ntz, ty = (t / ntz) % nty, tx = t / (ntz * nty);
  cx = tx * TX + lc / (TY * TZ);
  cy = ty * TY + (lc / TZ) % TY;
  cz = tz * TZ + lc % TZ;
}

}  // namespace spb
