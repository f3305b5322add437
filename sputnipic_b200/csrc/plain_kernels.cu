// Plain-form kernels: the reference's mover_PC / interpP2G / mover_interp /
// applyBCids on device-resident SoA particles with the reference's precision
// types (float particles, fields and moments).
//
// Bit-exactness. The mover reproduces src/Mover.cpp:31-157 operation by
// operation: float arithmetic in the reference's evaluation order, the double
// promotions where the reference mixes float with double (cell index,
// denominator, final velocity, boundary tests), truncating (mover) and
// flooring (P2G) double-to-int conversions. This file is compiled with
// -fmad=false so no multiply-add pair is contracted into an FMA, matching a
// baseline x86-64 build of the reference. Particle outputs are therefore
// bit-identical to the reference CPU code; moments differ only by the order
// of the FP32 additions.
//
// Launch shape. One thread per particle, 256 threads per block: the particle
// SoA streams through once (coalesced 4-byte loads per array per warp), the
// 8-node gathers hit the packed fields, which stay L2-resident (14 MB at
// 128x64x64 cells).
#include "grid_ctx.h"
#include "warp_sum.cuh"

#include <atomic>

namespace spb {

namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int TPB = 256;

struct Moments10 {
  float *m[10];
};

// The double product (x - start) * inv, limited to [-8, n + 8] so that the
// int conversion below never overflows (NaN maps to -8). Exact for every
// position inside the grid, where the limit does not bite.
__device__ __forceinline__ double cell_coord(float p, double start, float inv, int n) {
  const double d = ((double)p - start) * (double)inv;
  return fmin(fmax(d, -8.0), (double)n + 8.0);
}

// Reference cell index of the mover: 2 + int((x - xStart) * invdx), the
// product in double, truncated toward zero (src/Mover.cpp:39-41).
__device__ __forceinline__ int cell_trunc(float p, double start, float inv, int n) {
  return 2 + __double2int_rz(cell_coord(p, start, inv, n));
}

// Reference cell index of the deposit: 2 + int(floor(...)) (src/Mover.cpp:399-401).
__device__ __forceinline__ int cell_floor(float p, double start, float inv, int n) {
  return 2 + __double2int_rd(cell_coord(p, start, inv, n));
}

// Keeps the node pair (i-1, i) inside [0, n-1]. The reference reads out of
// bounds for such particles; here they are flagged and clamped.
__device__ __forceinline__ int clamp_cell(int i, int n, int &bad) {
  if (i < 1) { bad = 1; return 1; }
  if (i > n - 1) { bad = 1; return n - 1; }
  return i;
}

// x * y on a pair of floats, each half rounded to nearest on its own, as a
// scalar float multiply rounds it. The mover adds the two halves with scalar
// adds: a packed product that feeds a packed add came out rounded once with
// its sum, which the reference's float code does not do.
__device__ __forceinline__ float2 mul2_rn(float2 x, float2 y) {
  float2 d;
  asm("{\n\t.reg .b64 a, b, c;\n\t"
      "mov.b64 a, {%2, %3};\n\t"
      "mov.b64 b, {%4, %5};\n\t"
      "mul.rn.f32x2 c, a, b;\n\t"
      "mov.b64 {%0, %1}, c;\n\t}"
      : "=f"(d.x), "=f"(d.y)
      : "f"(x.x), "f"(x.y), "f"(y.x), "f"(y.y));
  return d;
}

// Particle boundary condition on one axis (src/Mover.cpp:103-157): an
// "above L" test in double, then a separate "below 0" test in float.
__device__ __forceinline__ void bc_axis(float &pos, float &vel, double L, int periodic) {
  if ((double)pos > L) {
    if (periodic) {
      pos = (float)((double)pos - L);
    } else {
      vel = -vel;
      pos = (float)(2.0 * L - (double)pos);
    }
  }
  if (pos < 0.0f) {
    if (periodic) {
      pos = (float)((double)pos + L);
    } else {
      vel = -vel;
      pos = -pos;
    }
  }
}

// Particle boundary condition of mover_PC_V (src/Mover.cpp:296-379): the
// periodic branch is mover_PC's; the reflecting branch first mirrors the
// position, then flips the velocity only if the MIRRORED position is still
// outside [0, L].
__device__ __forceinline__ void bc_axis_v(float &pos, float &vel, double L, int periodic) {
  if (periodic) {
    if ((double)pos > L) pos = (float)((double)pos - L);
    if (pos < 0.0f) pos = (float)((double)pos + L);
  } else {
    if ((double)pos > L) pos = (float)(2.0 * L - (double)pos);
    if (pos < 0.0f) pos = -pos;
    if ((double)pos > L) vel = -vel;
    if (pos < 0.0f) vel = -vel;
  }
}

// One particle of mover_PC (src/Mover.cpp:33-157); BCV = 1 gives mover_PC_V's
// boundary handling instead.
template <int BCV>
__device__ __forceinline__ void move_one(const GeomDev &g, const PushDev &p,
                                         const PackedFields &F, float &x, float &y,
                                         float &z, float &u, float &v, float &w,
                                         int &bad) {
  const float xpt = x, ypt = y, zpt = z;
  const float qomdt2 = p.qomdt2;
  float upt = 0.0f, vpt = 0.0f, wpt = 0.0f;
  float xc = x, yc = y, zc = z;
  const int sx = g.nyn * g.nzn, sy = g.nzn;   // nodes < 2^31 (spb_grid_create)
  for (int it = 0; it < p.niter; ++it) {
    const int ix = clamp_cell(cell_trunc(xc, g.xStart, g.invdx, g.nxn), g.nxn, bad);
    const int iy = clamp_cell(cell_trunc(yc, g.yStart, g.invdy, g.nyn), g.nyn, bad);
    const int iz = clamp_cell(cell_trunc(zc, g.zStart, g.invdz, g.nzn), g.nzn, bad);
    const float xi[2] = {xc - __ldg(g.xn + ix - 1), __ldg(g.xn + ix) - xc};
    const float eta[2] = {yc - __ldg(g.yn + iy - 1), __ldg(g.yn + iy) - yc};
    const float zeta[2] = {zc - __ldg(g.zn + iz - 1), __ldg(g.zn + iz) - zc};
    float Ex = 0.0f, Ey = 0.0f, Ez = 0.0f, Bx = 0.0f, By = 0.0f, Bz = 0.0f;
    const int base = ix * sx + iy * sy + iz;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const float wgt = xi[a] * eta[b] * zeta[c] * g.invVOL;
          const int n = base - a * sx - b * sy - c;
          const float4 f4 = __ldg(F.eb4 + n);
          const float2 f2 = __ldg(F.eb2 + n);
          // the six products as three packed multiplies, summed one by one
          const float2 w2 = make_float2(wgt, wgt);
          const float2 pxy = mul2_rn(w2, make_float2(f4.x, f4.y));
          const float2 pzx = mul2_rn(w2, make_float2(f4.z, f4.w));
          const float2 pyz = mul2_rn(w2, f2);
          Ex += pxy.x;
          Ey += pxy.y;
          Ez += pzx.x;
          Bx += pzx.y;
          By += pyz.x;
          Bz += pyz.y;
        }
    const float omdtsq = qomdt2 * qomdt2 * (Bx * Bx + By * By + Bz * Bz);
    const float denom = (float)(1.0 / (1.0 + (double)omdtsq));
    const float ut = u + qomdt2 * Ex;
    const float vt = v + qomdt2 * Ey;
    const float wt = w + qomdt2 * Ez;
    const float udotb = ut * Bx + vt * By + wt * Bz;
    upt = (ut + qomdt2 * (vt * Bz - wt * By + qomdt2 * udotb * Bx)) * denom;
    vpt = (vt + qomdt2 * (wt * Bx - ut * Bz + qomdt2 * udotb * By)) * denom;
    wpt = (wt + qomdt2 * (ut * By - vt * Bx + qomdt2 * udotb * Bz)) * denom;
    xc = xpt + upt * p.dto2;
    yc = ypt + vpt * p.dto2;
    zc = zpt + wpt * p.dto2;
  }
  u = (float)(2.0 * (double)upt - (double)u);
  v = (float)(2.0 * (double)vpt - (double)v);
  w = (float)(2.0 * (double)wpt - (double)w);
  x = xpt + upt * p.dt_sub;
  y = ypt + vpt * p.dt_sub;
  z = zpt + wpt * p.dt_sub;
  if (BCV == 0) {
    bc_axis(x, u, g.Lx, p.periodic[0]);
    bc_axis(y, v, g.Ly, p.periodic[1]);
    bc_axis(z, w, g.Lz, p.periodic[2]);
  } else {
    bc_axis_v(x, u, g.Lx, p.periodic[0]);
    bc_axis_v(y, v, g.Ly, p.periodic[1]);
    bc_axis_v(z, w, g.Lz, p.periodic[2]);
  }
}

// The 40 summands of one x half of a particle (src/Mover.cpp:399-570), each
// computed as the reference does (weight = q * xi * eta * zeta * invVOL,
// then e.g. (u * weight) * invVOL, no FMA), in the packed, lane-permuted
// layout of warp_sum80: t[(b * 2 + c) * 5 + k] = (moment k, moment k + 5) of
// node slot (a, b, c), slot a = `a` given, with physical node (a ^ bit4(lane),
// b ^ bit3(lane), c ^ bit2(lane)); the physical node (a, b, c) is (ix - a,
// iy - b, iz - c). ADD: added to t (else stored).
template <bool ADD>
__device__ __forceinline__ void half_terms(const GeomDev &g, float x, float y, float z, float u,
                                           float v, float w, float q, float2 (&t)[20], int lane,
                                           int a) {
  int ignored = 0;   // the range flag was raised when the cell key was formed
  const int ix = clamp_cell(cell_floor(x, g.xStart, g.invdx, g.nxn), g.nxn, ignored);
  const int iy = clamp_cell(cell_floor(y, g.yStart, g.invdy, g.nyn), g.nyn, ignored);
  const int iz = clamp_cell(cell_floor(z, g.zStart, g.invdz, g.nzn), g.nzn, ignored);
  const float xi0 = x - __ldg(g.xn + ix - 1), xi1 = __ldg(g.xn + ix) - x;
  const float eta0 = y - __ldg(g.yn + iy - 1), eta1 = __ldg(g.yn + iy) - y;
  const float zeta0 = z - __ldg(g.zn + iz - 1), zeta1 = __ldg(g.zn + iz) - z;
  const bool pb = lane & 8, pc = lane & 4;
  const float xia = (a ^ ((lane >> 4) & 1)) ? xi1 : xi0;
  const float eta[2] = {pb ? eta1 : eta0, pb ? eta0 : eta1};
  const float zeta[2] = {pc ? zeta1 : zeta0, pc ? zeta0 : zeta1};
  const float uu = u * u, uv = u * v, uw = u * w, vv = v * v, vw = v * w, ww = w * w;
  const float inv = g.invVOL;
#pragma unroll
  for (int b = 0; b < 2; ++b)
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const float wgt = q * xia * eta[b] * zeta[c] * inv;
      float2 *o = t + (b * 2 + c) * 5;
      const float2 n[5] = {make_float2(wgt * inv, (uv * wgt) * inv),
                           make_float2((u * wgt) * inv, (uw * wgt) * inv),
                           make_float2((v * wgt) * inv, (vv * wgt) * inv),
                           make_float2((w * wgt) * inv, (vw * wgt) * inv),
                           make_float2((uu * wgt) * inv, (ww * wgt) * inv)};
#pragma unroll
      for (int k = 0; k < 5; ++k) o[k] = ADD ? __fadd2_rn(o[k], n[k]) : n[k];
    }
}

struct Particle {
  float x, y, z, u, v, w, q;
};

// One 16-byte add to global memory (p 16-byte aligned): one L2 atomic
// operation for four floats.
__device__ __forceinline__ void red_v4(float *p, float a, float b, float c, float d) {
  asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a), "f"(b),
               "f"(c), "f"(d)
               : "memory");
}

// The plain deposit's accumulator: the ten moments of node n side by side,
// acc[n * ACC_STRIDE + m] (m = rhon, Jx, Jy, Jz, pxx, pxy, pxz, pyy, pyz, pzz;
// two pad floats keep every node's record on a 16-byte boundary). A
// particle's 80 terms then land in about a dozen 32-byte sectors instead of
// the forty that ten separate arrays take; k_fold_acc adds it into the ten
// arrays afterwards.
constexpr int ACC_STRIDE = 12;

// Where a plain deposit adds: the accumulator (ACC) or, when none could be
// allocated, the ten moment arrays themselves.
struct DepTarget {
  float *acc;
  Moments10 mom;
};

// Adds v to moment m of node n.
template <bool ACC>
__device__ __forceinline__ void dep_add(const DepTarget &T, long n, int m, float v) {
  if (ACC)
    atomicAdd(T.acc + n * ACC_STRIDE + m, v);
  else
    atomicAdd(T.mom.m[m] + n, v);
}

// Adds v0..v3 to moments 4 grp .. 4 grp + 3 of node n (moments below 10).
template <bool ACC>
__device__ __forceinline__ void dep_add4(const DepTarget &T, long n, int grp, float v0, float v1,
                                         float v2, float v3) {
  if (ACC) {
    red_v4(T.acc + n * ACC_STRIDE + 4 * grp, v0, v1, v2, v3);
  } else {
    const float v[4] = {v0, v1, v2, v3};
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (4 * grp + i < 10) atomicAdd(T.mom.m[4 * grp + i] + n, v[i]);
  }
}

// Adds one warp's deposits to the accumulator. For each of up to four
// distinct cells among the warp's particles (cell-ordered particles give one
// or two), the members compute their terms and the warp sums them (the steps
// of warp_sum80, one x half of the terms at a time) and adds the 80 totals;
// each lone particle of a further cell (a particle that moved, unordered
// input) is spread over 24 lanes, four moments of one node each, added with
// one 16-byte add per lane. Terms are recomputed per round rather than kept,
// which keeps the registers down. All 32 lanes call.
template <bool ACC>
__device__ __forceinline__ void deposit_warp(const GeomDev &g, const DepTarget &T, bool valid,
                                             const Particle &p, int &bad) {
  const int lane = threadIdx.x & 31;
  const int sx = g.nyn * g.nzn, sy = g.nzn;   // nodes < 2^31 (spb_grid_create)
  int key = 0;
  if (valid) {
    const int ix = clamp_cell(cell_floor(p.x, g.xStart, g.invdx, g.nxn), g.nxn, bad);
    const int iy = clamp_cell(cell_floor(p.y, g.yStart, g.invdy, g.nyn), g.nyn, bad);
    const int iz = clamp_cell(cell_floor(p.z, g.zStart, g.invdz, g.nzn), g.nzn, bad);
    key = (ix * g.nyn + iy) * g.nzn + iz;
  }
  // this lane's totals after warp_sum80: physical node (bit4, bit3, bit2),
  // moments mbase + [lo, hi)
  const int na = (lane >> 4) & 1, nb = (lane >> 3) & 1, nc = (lane >> 2) & 1;
  const int mbase = 5 * ((lane >> 1) & 1);
  const int lo = (lane & 1) ? 3 : 0, hi = (lane & 1) ? 5 : 3;
  unsigned remaining = __ballot_sync(FULL, valid);
#pragma unroll 1
  for (int round = 0; round < 4 && remaining; ++round) {
    const int leader = __ffs(remaining) - 1;
    const int k = __shfl_sync(FULL, key, leader);
    const bool member = valid && key == k;
    const unsigned members = __ballot_sync(FULL, member);
    remaining &= ~members;
    if (__popc(members) < 2 && round > 0) continue;   // lone particle: direct atomics below
    // warp_sum80 in halves: the slot a = 1 terms go to lane ^ 16, whose slot
    // a = 0 holds the same physical x node, and each lane adds its own slot
    // a = 0 terms to what it received (40 live values instead of 80)
    float2 t[20];
    if (member) {
      half_terms<false>(g, p.x, p.y, p.z, p.u, p.v, p.w, p.q, t, lane, 1);
    } else {
#pragma unroll
      for (int j = 0; j < 20; ++j) t[j] = make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int j = 0; j < 20; ++j) t[j] = shfl_xor2(t[j], 16);
    if (member) half_terms<true>(g, p.x, p.y, p.z, p.u, p.v, p.w, p.q, t, lane, 0);
    float r[5];
    warp_sum80_tail(t, r, lane);
    const int node = k - na * sx - nb * sy - nc;
#pragma unroll
    for (int i = 0; i < 5; ++i)
      if (i >= lo && i < hi) dep_add<ACC>(T, node, mbase + i, r[i]);
    if (member) valid = false;   // done
  }
  // lone particles of further cells, one at a time: lane j < 24 takes node
  // j / 3 and moments 4 (j % 3) .. 4 (j % 3) + 3 of the particle, each term
  // computed as half_terms does, and adds them with one 16-byte add
  unsigned lone = __ballot_sync(FULL, valid);
  if (lone) {
    const int ix = (int)(key / sx), iy = (int)((key / sy) % g.nyn), iz = (int)(key % sy);
    float d[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};   // xi0, xi1, eta0, eta1, zeta0, zeta1
    if (valid) {
      d[0] = p.x - __ldg(g.xn + ix - 1);
      d[1] = __ldg(g.xn + ix) - p.x;
      d[2] = p.y - __ldg(g.yn + iy - 1);
      d[3] = __ldg(g.yn + iy) - p.y;
      d[4] = p.z - __ldg(g.zn + iz - 1);
      d[5] = __ldg(g.zn + iz) - p.z;
    }
    const float inv = g.invVOL;
    while (lone) {
      const int L = __ffs(lone) - 1;
      lone &= lone - 1;
      float e[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) e[j] = __shfl_sync(FULL, d[j], L);
      const float q = __shfl_sync(FULL, p.q, L), u = __shfl_sync(FULL, p.u, L);
      const float v = __shfl_sync(FULL, p.v, L), w = __shfl_sync(FULL, p.w, L);
      const int k = __shfl_sync(FULL, key, L);
      if (lane < 24) {
        const int node = lane / 3, grp = lane % 3;
        const int a = node >> 2, b = (node >> 1) & 1, c = node & 1;
        const float wgt = q * (a ? e[1] : e[0]) * (b ? e[3] : e[2]) * (c ? e[5] : e[4]) * inv;
        // moment factors of the group: (1, u, v, w), (uu, uv, uw, vv) or
        // (vw, ww, 0, 0) (rhon's (1 * wgt) * inv is the reference's wgt * inv
        // exactly; the pad slots add zeros)
        const float f0 = grp == 0 ? 1.0f : (grp == 1 ? u * u : v * w);
        const float f1 = grp == 0 ? u : (grp == 1 ? u * v : w * w);
        const float f2 = grp == 0 ? v : (grp == 1 ? u * w : 0.0f);
        const float f3 = grp == 0 ? w : (grp == 1 ? v * v : 0.0f);
        dep_add4<ACC>(T, k - a * sx - b * sy - c, grp, (f0 * wgt) * inv, (f1 * wgt) * inv,
                      (f2 * wgt) * inv, (f3 * wgt) * inv);
      }
    }
  }
}

// One lone particle (its cell's only member in a group) of a warp's
// deposit: lane j < 24 takes node j / 3 and moments 4 (j % 3) .. 4 (j % 3) + 3,
// each term computed as half_terms does, added with one 16-byte add. Every
// lane passes the same particle and key. All 32 lanes call.
template <bool ACC>
__device__ __forceinline__ void deposit_lone(const GeomDev &g, const DepTarget &T,
                                             const Particle &p, int key) {
  const int lane = threadIdx.x & 31;
  const int sx = g.nyn * g.nzn, sy = g.nzn;
  if (lane >= 24) return;
  const int ix = key / sx, iy = (key / sy) % g.nyn, iz = key % sy;
  const float e[6] = {p.x - __ldg(g.xn + ix - 1), __ldg(g.xn + ix) - p.x,
                      p.y - __ldg(g.yn + iy - 1), __ldg(g.yn + iy) - p.y,
                      p.z - __ldg(g.zn + iz - 1), __ldg(g.zn + iz) - p.z};
  const float inv = g.invVOL, u = p.u, v = p.v, w = p.w;
  const int node = lane / 3, grp = lane % 3;
  const int a = node >> 2, b = (node >> 1) & 1, c = node & 1;
  const float wgt = p.q * (a ? e[1] : e[0]) * (b ? e[3] : e[2]) * (c ? e[5] : e[4]) * inv;
  const float f0 = grp == 0 ? 1.0f : (grp == 1 ? u * u : v * w);
  const float f1 = grp == 0 ? u : (grp == 1 ? u * v : w * w);
  const float f2 = grp == 0 ? v : (grp == 1 ? u * w : 0.0f);
  const float f3 = grp == 0 ? w : (grp == 1 ? v * v : 0.0f);
  dep_add4<ACC>(T, key - a * sx - b * sy - c, grp, (f0 * wgt) * inv, (f1 * wgt) * inv,
                (f2 * wgt) * inv, (f3 * wgt) * inv);
}

// The grouped plain deposit. A CTA takes a chunk of GP_CHUNK consecutive
// particles into shared memory and groups them by cell (a shared-memory hash
// table of GP_SLOTS cells; each warp inserts each of its distinct cells once),
// then every group is deposited by one warp: its lanes take the group's
// particles in turn and accumulate their terms in the packed layout of
// warp_sum80 (one x half of the terms at a time), and one warp reduction and
// 80 adds serve the whole group instead of one per 32 particles. Groups of up
// to three particles deposit particle by particle (deposit_lone). A chunk
// with more distinct cells than the table holds (unordered input) falls back
// to the per-warp deposit of k_plain_p2g.
constexpr int GP_TPB = 256;
constexpr int GP_PER_THREAD = 4;
constexpr int GP_CHUNK = GP_TPB * GP_PER_THREAD;
constexpr int GP_SLOTS = 256;
static_assert(GP_SLOTS == GP_TPB, "one table slot per thread in the scans");

struct GroupSmem {
  float p[7][GP_CHUNK];                 // x, y, z, u, v, w, q
  int key[GP_CHUNK];                    // node-space cell of each particle
  short slot[GP_CHUNK];                 // its table slot
  unsigned short order[GP_CHUNK];       // chunk indices grouped by slot
  int hkey[GP_SLOTS], hcnt[GP_SLOTS], hstart[GP_SLOTS], hcur[GP_SLOTS];
  int wsum[GP_TPB / 32];
  int full;
};

__device__ __forceinline__ Particle smem_particle(const GroupSmem &S, int j) {
  return Particle{S.p[0][j], S.p[1][j], S.p[2][j], S.p[3][j], S.p[4][j], S.p[5][j], S.p[6][j]};
}

// (Particles in the arrays' own order; cell-ordered input goes through
// k_plain_p2g_runs instead.)
template <bool ACC>
__global__ void __launch_bounds__(GP_TPB) k_plain_p2g_grouped(
    GeomDev g, const float *__restrict__ x, const float *__restrict__ y,
    const float *__restrict__ z, const float *__restrict__ u, const float *__restrict__ v,
    const float *__restrict__ w, const float *__restrict__ q, long n,
    const __grid_constant__ DepTarget T, int *__restrict__ err) {
  __shared__ GroupSmem S;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long base = (long)blockIdx.x * GP_CHUNK;
  const int cnt = (int)min((long)GP_CHUNK, n - base);
  S.hkey[tid] = -1;
  S.hcnt[tid] = 0;
  if (tid == 0) S.full = 0;
  __syncthreads();
  int bad = 0;
  const float *const src[7] = {x, y, z, u, v, w, q};
#pragma unroll
  for (int r = 0; r < GP_PER_THREAD; ++r) {
    const int j = tid + r * GP_TPB;
    const bool valid = j < cnt;
    int key = -1;
    if (valid) {
      const long i = base + j;
#pragma unroll
      for (int a = 0; a < 7; ++a) S.p[a][j] = src[a][i];
      const int ix = clamp_cell(cell_floor(S.p[0][j], g.xStart, g.invdx, g.nxn), g.nxn, bad);
      const int iy = clamp_cell(cell_floor(S.p[1][j], g.yStart, g.invdy, g.nyn), g.nyn, bad);
      const int iz = clamp_cell(cell_floor(S.p[2][j], g.zStart, g.invdz, g.nzn), g.nzn, bad);
      key = (ix * g.nyn + iy) * g.nzn + iz;
      S.key[j] = key;
    }
    // one insertion per distinct cell of the warp (linear probing)
    const unsigned peers = __match_any_sync(FULL, key);
    const int leader = __ffs(peers) - 1;
    int slot = -1;
    if (valid && lane == leader) {
      unsigned h = ((unsigned)key * 2654435761u) >> 24;
      for (int t = 0; t < GP_SLOTS; ++t) {
        const int prev = atomicCAS(&S.hkey[h], -1, key);
        if (prev == -1 || prev == key) {
          slot = (int)h;
          break;
        }
        h = (h + 1) & (GP_SLOTS - 1);
      }
      if (slot < 0)
        S.full = 1;
      else
        atomicAdd(&S.hcnt[slot], __popc(peers));
    }
    slot = __shfl_sync(FULL, slot, leader);
    if (valid) S.slot[j] = (short)slot;
  }
  __syncthreads();
  if (S.full) {
    // more distinct cells than table slots: the per-warp deposit, in order
#pragma unroll 1
    for (int r = 0; r < GP_PER_THREAD; ++r) {
      const int j = tid + r * GP_TPB;
      const bool valid = j < cnt;
      Particle p{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      if (valid) p = smem_particle(S, j);
      deposit_warp<ACC>(g, T, valid, p, bad);
    }
    if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
    return;
  }
  // group starts: exclusive scan of the slot counts
  {
    const int c = S.hcnt[tid];
    int xs = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, xs, o);
      if (lane >= o) xs += t;
    }
    if (lane == 31) S.wsum[warp] = xs;
    __syncthreads();
    int pre = 0;
    for (int k = 0; k < warp; ++k) pre += S.wsum[k];
    S.hstart[tid] = pre + xs - c;
    S.hcur[tid] = pre + xs - c;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < GP_PER_THREAD; ++r) {
    const int j = tid + r * GP_TPB;
    const bool valid = j < cnt;
    const int slot = valid ? S.slot[j] : -1;
    const unsigned peers = __match_any_sync(FULL, slot);
    const int leader = __ffs(peers) - 1;
    int first = 0;
    if (valid && lane == leader) first = atomicAdd(&S.hcur[slot], __popc(peers));
    first = __shfl_sync(FULL, first, leader);
    if (valid) S.order[first + __popc(peers & ((1u << lane) - 1u))] = (unsigned short)j;
  }
  __syncthreads();
  const int sx = g.nyn * g.nzn, sy = g.nzn;
  const int na = (lane >> 4) & 1, nb = (lane >> 3) & 1, nc = (lane >> 2) & 1;
  const int mbase = 5 * ((lane >> 1) & 1);
  const int lo = (lane & 1) ? 3 : 0, hi = (lane & 1) ? 5 : 3;
#pragma unroll 1
  for (int s = warp; s < GP_SLOTS; s += GP_TPB / 32) {
    const int c = S.hcnt[s];
    if (c == 0) continue;
    const int st = S.hstart[s], key = S.hkey[s];
    if (c <= 3) {
      for (int m = 0; m < c; ++m) deposit_lone<ACC>(g, T, smem_particle(S, S.order[st + m]), key);
      continue;
    }
    float2 t[20];
#pragma unroll
    for (int i = 0; i < 20; ++i) t[i] = make_float2(0.0f, 0.0f);
    for (int m = lane; m < c; m += 32) {
      const Particle p = smem_particle(S, S.order[st + m]);
      half_terms<true>(g, p.x, p.y, p.z, p.u, p.v, p.w, p.q, t, lane, 1);
    }
#pragma unroll
    for (int i = 0; i < 20; ++i) t[i] = shfl_xor2(t[i], 16);
    for (int m = lane; m < c; m += 32) {
      const Particle p = smem_particle(S, S.order[st + m]);
      half_terms<true>(g, p.x, p.y, p.z, p.u, p.v, p.w, p.q, t, lane, 0);
    }
    float r[5];
    warp_sum80_tail(t, r, lane);
    const int node = key - na * sx - nb * sy - nc;
#pragma unroll
    for (int i = 0; i < 5; ++i)
      if (i >= lo && i < hi) dep_add<ACC>(T, node, mbase + i, r[i]);
  }
  if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
}

// The plain deposit over particles in cell order (a permutation from the cell
// sort below). A CTA takes a chunk of RUN_CHUNK consecutive positions of the
// permutation; while loading them it computes each particle's deposit cell
// and its six node distances (xi0 = x - xn[ix-1], xi1 = xn[ix] - x, and so
// on, src/Mover.cpp:399-410) once, into shared memory with u, v, w, q. Each
// warp then takes an equal slice of the chunk: in the slice the particles of
// one cell form runs, and a run of four or more is deposited as one group
// (run_terms for both x halves, one warp reduction, 80 adds), shorter runs
// particle by particle. A run that a slice or chunk boundary cuts is
// deposited in parts.
constexpr int RUN_TPB = 256;
constexpr int RUN_PER_THREAD = 4;
constexpr int RUN_CHUNK = RUN_TPB * RUN_PER_THREAD;
static_assert(RUN_CHUNK == GP_CHUNK, "one grid size for both deposit kernels");

struct RunSmem {
  float d[10][RUN_CHUNK];   // xi0, xi1, eta0, eta1, zeta0, zeta1, u, v, w, q
  int key[RUN_CHUNK];       // node-space cell
};

// half_terms from the stored node distances of particle j: the same 40
// summands, each product in the reference's order (pairs of independent
// products issued as one packed FP32x2 multiply). With ADD, a term's last
// multiply may be fused into the packed sum that follows it (one rounding
// instead of two); the moments are a reordered FP32 sum either way.
template <bool ADD>
__device__ __forceinline__ void run_terms(const GeomDev &g, const RunSmem &S, int j,
                                          float2 (&t)[20], int lane, int a) {
  const bool pb = lane & 8, pc = lane & 4;
  const float xi0 = S.d[0][j], xi1 = S.d[1][j], eta0 = S.d[2][j], eta1 = S.d[3][j];
  const float zeta0 = S.d[4][j], zeta1 = S.d[5][j];
  const float u = S.d[6][j], v = S.d[7][j], w = S.d[8][j], q = S.d[9][j];
  const float xia = (a ^ ((lane >> 4) & 1)) ? xi1 : xi0;
  const float eta[2] = {pb ? eta1 : eta0, pb ? eta0 : eta1};
  const float2 zeta = pc ? make_float2(zeta1, zeta0) : make_float2(zeta0, zeta1);
  const float2 uu_vv = __fmul2_rn(make_float2(u, v), make_float2(u, v));
  const float2 uv_vw = __fmul2_rn(make_float2(u, v), make_float2(v, w));
  const float2 uw_ww = __fmul2_rn(make_float2(u, w), make_float2(w, w));
  // factor pairs (moment k, moment k + 5); rhon's (1 * wgt) * inv is the
  // reference's wgt * inv exactly
  const float2 f[5] = {make_float2(1.0f, uv_vw.x), make_float2(u, uw_ww.x),
                       make_float2(v, uu_vv.y), make_float2(w, uv_vw.y),
                       make_float2(uu_vv.x, uw_ww.y)};
  const float2 inv = make_float2(g.invVOL, g.invVOL);
  const float qx = q * xia;
#pragma unroll
  for (int b = 0; b < 2; ++b) {
    const float qxe = qx * eta[b];
    // ((q * xi * eta) * zeta) * invVOL for both z nodes
    const float2 wgt = __fmul2_rn(__fmul2_rn(make_float2(qxe, qxe), zeta), inv);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const float wc = c ? wgt.y : wgt.x;
      const float2 w2 = make_float2(wc, wc);
      float2 *o = t + (b * 2 + c) * 5;
#pragma unroll
      for (int k = 0; k < 5; ++k) {
        const float2 n = __fmul2_rn(__fmul2_rn(f[k], w2), inv);
        o[k] = ADD ? __fadd2_rn(o[k], n) : n;
      }
    }
  }
}

// deposit_lone from the stored node distances of particle j (all 32 lanes
// call with the same j and key).
template <bool ACC>
__device__ __forceinline__ void run_lone(const GeomDev &g, const DepTarget &T, const RunSmem &S,
                                         int j, int key) {
  const int lane = threadIdx.x & 31;
  const int sx = g.nyn * g.nzn, sy = g.nzn;
  if (lane >= 24) return;
  const int node = lane / 3, grp = lane % 3;
  const int a = node >> 2, b = (node >> 1) & 1, c = node & 1;
  const float inv = g.invVOL, u = S.d[6][j], v = S.d[7][j], w = S.d[8][j];
  const float wgt = S.d[9][j] * S.d[a][j] * S.d[2 + b][j] * S.d[4 + c][j] * inv;
  const float f0 = grp == 0 ? 1.0f : (grp == 1 ? u * u : v * w);
  const float f1 = grp == 0 ? u : (grp == 1 ? u * v : w * w);
  const float f2 = grp == 0 ? v : (grp == 1 ? u * w : 0.0f);
  const float f3 = grp == 0 ? w : (grp == 1 ? v * v : 0.0f);
  dep_add4<ACC>(T, key - a * sx - b * sy - c, grp, (f0 * wgt) * inv, (f1 * wgt) * inv,
                (f2 * wgt) * inv, (f3 * wgt) * inv);
}

template <bool ACC>
__global__ void __launch_bounds__(RUN_TPB, 3) k_plain_p2g_runs(
    GeomDev g, const float *__restrict__ x, const float *__restrict__ y,
    const float *__restrict__ z, const float *__restrict__ u, const float *__restrict__ v,
    const float *__restrict__ w, const float *__restrict__ q, long n,
    const unsigned *__restrict__ perm, const __grid_constant__ DepTarget T,
    int *__restrict__ err) {
  __shared__ RunSmem S;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long base = (long)blockIdx.x * RUN_CHUNK;
  const int cnt = (int)min((long)RUN_CHUNK, n - base);
  int bad = 0;
#pragma unroll
  for (int r = 0; r < RUN_PER_THREAD; ++r) {
    const int j = tid + r * RUN_TPB;
    if (j < cnt) {
      const long i = perm[base + j];
      const float px = x[i], py = y[i], pz = z[i];
      const int ix = clamp_cell(cell_floor(px, g.xStart, g.invdx, g.nxn), g.nxn, bad);
      const int iy = clamp_cell(cell_floor(py, g.yStart, g.invdy, g.nyn), g.nyn, bad);
      const int iz = clamp_cell(cell_floor(pz, g.zStart, g.invdz, g.nzn), g.nzn, bad);
      S.key[j] = (ix * g.nyn + iy) * g.nzn + iz;
      S.d[0][j] = px - __ldg(g.xn + ix - 1);
      S.d[1][j] = __ldg(g.xn + ix) - px;
      S.d[2][j] = py - __ldg(g.yn + iy - 1);
      S.d[3][j] = __ldg(g.yn + iy) - py;
      S.d[4][j] = pz - __ldg(g.zn + iz - 1);
      S.d[5][j] = __ldg(g.zn + iz) - pz;
      S.d[6][j] = u[i];
      S.d[7][j] = v[i];
      S.d[8][j] = w[i];
      S.d[9][j] = q[i];
    }
  }
  __syncthreads();
  const int sx = g.nyn * g.nzn, sy = g.nzn;
  const int na = (lane >> 4) & 1, nb = (lane >> 3) & 1, nc = (lane >> 2) & 1;
  const int mbase = 5 * ((lane >> 1) & 1);
  const int lo = (lane & 1) ? 3 : 0, hi = (lane & 1) ? 5 : 3;
  constexpr int PW = RUN_CHUNK / (RUN_TPB / 32);   // positions per warp
  const int jend = min((warp + 1) * PW, cnt);
#pragma unroll 1
  for (int j = warp * PW; j < jend;) {
    // the run of key S.key[j]: up to the first position with another key
    const int key = S.key[j];
    int e = jend;
#pragma unroll 1
    for (int b = j + 1; b < jend; b += 32) {
      const int t = b + lane;
      const unsigned m = __ballot_sync(FULL, t < jend && S.key[t] != key);
      if (m) {
        e = b + __ffs(m) - 1;
        break;
      }
    }
    const int c = e - j;
    if (c <= 3) {
      for (int m = 0; m < c; ++m) run_lone<ACC>(g, T, S, j + m, key);
    } else {
      float2 t[20];
#pragma unroll
      for (int i = 0; i < 20; ++i) t[i] = make_float2(0.0f, 0.0f);
      for (int m = lane; m < c; m += 32) run_terms<true>(g, S, j + m, t, lane, 1);
#pragma unroll
      for (int i = 0; i < 20; ++i) t[i] = shfl_xor2(t[i], 16);
      for (int m = lane; m < c; m += 32) run_terms<true>(g, S, j + m, t, lane, 0);
      float r[5];
      warp_sum80_tail(t, r, lane);
      const int node = key - na * sx - nb * sy - nc;
#pragma unroll
      for (int i = 0; i < 5; ++i)
        if (i >= lo && i < hi) dep_add<ACC>(T, node, mbase + i, r[i]);
    }
    j = e;
  }
  if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
}

// The plain deposit's cell sort: a counting sort of (cell, index) pairs by
// the deposit's own cell (the node-space floor cell of src/Mover.cpp:399-401).
// Keys and per-cell counts (one atomic per distinct cell of a warp) ...
__global__ void __launch_bounds__(TPB) k_p2g_keys(GeomDev g, const float *__restrict__ x,
                                                  const float *__restrict__ y,
                                                  const float *__restrict__ z, long n,
                                                  unsigned *__restrict__ key,
                                                  unsigned *__restrict__ count) {
  const int lane = threadIdx.x & 31;
  int ignored = 0;   // the deposit flags cells off the node array
  for (long base = (long)blockIdx.x * TPB; base < n; base += (long)gridDim.x * TPB) {
    const long i = base + threadIdx.x;
    const bool valid = i < n;
    unsigned k = 0xffffffffu;
    if (valid) {
      const int ix = clamp_cell(cell_floor(x[i], g.xStart, g.invdx, g.nxn), g.nxn, ignored);
      const int iy = clamp_cell(cell_floor(y[i], g.yStart, g.invdy, g.nyn), g.nyn, ignored);
      const int iz = clamp_cell(cell_floor(z[i], g.zStart, g.invdz, g.nzn), g.nzn, ignored);
      k = (unsigned)((ix * g.nyn + iy) * g.nzn + iz);
      key[i] = k;
    }
    const unsigned peers = __match_any_sync(FULL, k);
    if (valid && lane == __ffs(peers) - 1) atomicAdd(count + k, (unsigned)__popc(peers));
  }
}

// ... an exclusive scan of the counts into the cells' first positions (three
// passes over blocks of P2S_B) ...
constexpr int P2S_B = 1024;
__device__ __forceinline__ unsigned p2s_block_scan(unsigned v, unsigned *ws, unsigned &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned xs = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(FULL, xs, o);
    if (lane >= o) xs += t;
  }
  if (lane == 31) ws[warp] = xs;
  __syncthreads();
  if (warp == 0) {
    unsigned s = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(FULL, s, o);
      if (lane >= o) s += t;
    }
    ws[lane] = s;
  }
  __syncthreads();
  const unsigned pre = warp ? ws[warp - 1] : 0u;
  total = ws[31];
  __syncthreads();
  return pre + xs - v;
}

__global__ void __launch_bounds__(P2S_B) k_p2s_scan_blocks(const unsigned *in, long m,
                                                           unsigned *out, unsigned *bsum) {
  __shared__ unsigned ws[32];
  const long i = blockIdx.x * (long)P2S_B + threadIdx.x;
  unsigned total;
  const unsigned ex = p2s_block_scan(i < m ? in[i] : 0u, ws, total);
  if (i < m) out[i] = ex;
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(P2S_B) k_p2s_scan_sums(unsigned *bsum, int nb) {
  __shared__ unsigned ws[32];
  unsigned carry = 0;
  for (int b = 0; b < nb; b += P2S_B) {
    const int i = b + threadIdx.x;
    unsigned total;
    const unsigned ex = p2s_block_scan(i < nb ? bsum[i] : 0u, ws, total);
    if (i < nb) bsum[i] = ex + carry;
    carry += total;
  }
}

__global__ void __launch_bounds__(P2S_B) k_p2s_scan_add(unsigned *out, long m,
                                                        const unsigned *bsum) {
  const long i = blockIdx.x * (long)P2S_B + threadIdx.x;
  if (i < m) out[i] += bsum[blockIdx.x];
}

// ... and every index at its cell's next free position (cursor: the first
// positions, advanced; the order inside a cell is the atomics').
__global__ void __launch_bounds__(TPB) k_p2g_scatter(const unsigned *__restrict__ key, long n,
                                                     unsigned *__restrict__ cursor,
                                                     unsigned *__restrict__ perm) {
  const int lane = threadIdx.x & 31;
  for (long base = (long)blockIdx.x * TPB; base < n; base += (long)gridDim.x * TPB) {
    const long i = base + threadIdx.x;
    const bool valid = i < n;
    const unsigned k = valid ? key[i] : 0xffffffffu;
    const unsigned peers = __match_any_sync(FULL, k);
    const int leader = __ffs(peers) - 1;
    unsigned first = 0;
    if (valid && lane == leader) first = atomicAdd(cursor + k, (unsigned)__popc(peers));
    first = __shfl_sync(FULL, first, leader);
    if (valid) perm[first + __popc(peers & ((1u << lane) - 1u))] = (unsigned)i;
  }
}

__global__ void __launch_bounds__(TPB) k_pack_fields(const float *__restrict__ ex,
                                                     const float *__restrict__ ey,
                                                     const float *__restrict__ ez,
                                                     const float *__restrict__ bx,
                                                     const float *__restrict__ by,
                                                     const float *__restrict__ bz,
                                                     float4 *__restrict__ eb4,
                                                     float2 *__restrict__ eb2, long nodes) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nodes;
       i += (long)gridDim.x * blockDim.x) {
    eb4[i] = make_float4(ex[i], ey[i], ez[i], bx[i]);
    eb2[i] = make_float2(by[i], bz[i]);
  }
}

template <int BCV>
__global__ void __launch_bounds__(TPB) k_plain_mover(GeomDev g, PushDev p, PackedFields F,
                                                     float *__restrict__ x, float *__restrict__ y,
                                                     float *__restrict__ z, float *__restrict__ u,
                                                     float *__restrict__ v, float *__restrict__ w,
                                                     long n, int *__restrict__ err) {
  const long i = blockIdx.x * (long)TPB + threadIdx.x;
  if (i >= n) return;
  float px = x[i], py = y[i], pz = z[i], pu = u[i], pv = v[i], pw = w[i];
  int bad = 0;
  move_one<BCV>(g, p, F, px, py, pz, pu, pv, pw, bad);
  x[i] = px;
  y[i] = py;
  z[i] = pz;
  u[i] = pu;
  v[i] = pv;
  w[i] = pw;
  if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
}

template <bool ACC>
__global__ void __launch_bounds__(TPB) k_plain_p2g(GeomDev g, const float *__restrict__ x,
                                                   const float *__restrict__ y,
                                                   const float *__restrict__ z,
                                                   const float *__restrict__ u,
                                                   const float *__restrict__ v,
                                                   const float *__restrict__ w,
                                                   const float *__restrict__ q, long n,
                                                   const __grid_constant__ DepTarget T,
                                                   int *__restrict__ err) {
  const long i = blockIdx.x * (long)TPB + threadIdx.x;
  const bool valid = i < n;
  Particle p{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (valid) p = Particle{x[i], y[i], z[i], u[i], v[i], w[i], q[i]};
  int bad = 0;
  deposit_warp<ACC>(g, T, valid, p, bad);
  if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
}

template <bool ACC>
__global__ void __launch_bounds__(TPB) k_plain_mover_interp(
    GeomDev g, PushDev p, PackedFields F, float *__restrict__ x, float *__restrict__ y,
    float *__restrict__ z, float *__restrict__ u, float *__restrict__ v,
    float *__restrict__ w, const float *__restrict__ q, long n,
    const __grid_constant__ DepTarget T, int *__restrict__ err) {
  const long i = blockIdx.x * (long)TPB + threadIdx.x;
  const bool valid = i < n;
  Particle pt{0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  int bad = 0;
  if (valid) {
    float px = x[i], py = y[i], pz = z[i], pu = u[i], pv = v[i], pw = w[i];
    move_one<0>(g, p, F, px, py, pz, pu, pv, pw, bad);
    x[i] = px;
    y[i] = py;
    z[i] = pz;
    u[i] = pu;
    v[i] = pv;
    w[i] = pw;
    pt = Particle{px, py, pz, pu, pv, pw, q[i]};
  }
  deposit_warp<ACC>(g, T, valid, pt, bad);
  if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
}

// applyBCids (src/BC.cpp:362-615), one launch per step so the axis order of
// the reference holds: periodic folds X, Y, Z, then non-periodic doubling X,
// Y, Z. Thread t handles one (row, col) pair of the boundary planes of all
// ten moments.
// sumOverSpecies (src/InterpDensNet.cpp:120-146) on the device: net moment m
// of node i = the species' values added in species order, from zero, as the
// reference's loop does (so the float sums are bit-identical).
constexpr int SUM_MAX_SPECIES = 32;
struct SpeciesBases {
  const float *b[SUM_MAX_SPECIES];   // [10][nodes] moments of each species
};

__global__ void __launch_bounds__(TPB) k_sum_species(SpeciesBases S, int ns, long nodes,
                                                     float *__restrict__ net) {
  const long total = 10 * nodes;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    float acc = 0.0f;
    for (int s = 0; s < ns; ++s) acc += S.b[s][i];
    net[i] = acc;
  }
}

// mom[m][n] += acc[n * ACC_STRIDE + m] for the non-zero entries (atomically:
// the pipeline streams of the drop-in fold into the same arrays).
__global__ void __launch_bounds__(TPB) k_fold_acc(const float4 *__restrict__ acc, long nodes,
                                                  Moments10 M) {
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < nodes;
       n += (long)gridDim.x * blockDim.x) {
    const float4 a = acc[3 * n], b = acc[3 * n + 1], c = acc[3 * n + 2];
    const float v[10] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y};
#pragma unroll
    for (int m = 0; m < 10; ++m)
      if (v[m] != 0.0f) atomicAdd(M.m[m] + n, v[m]);
  }
}

__global__ void __launch_bounds__(TPB) k_bc_fold(Moments10 M, int nxn, int nyn, int nzn,
                                                 int axis, int periodic) {
  int n1, n2;
  if (axis == 0) {
    n1 = nyn - 2;
    n2 = nzn - 2;
  } else if (axis == 1) {
    n1 = nxn - 2;
    n2 = nzn - 2;
  } else {
    n1 = nxn - 2;
    n2 = nyn - 2;
  }
  const long t = blockIdx.x * (long)TPB + threadIdx.x;
  if (t >= (long)n1 * n2) return;
  const int r = 1 + (int)(t / n2), s = 1 + (int)(t % n2);
  long lo, hi;
  if (axis == 0) {
    lo = ((long)1 * nyn + r) * nzn + s;
    hi = ((long)(nxn - 2) * nyn + r) * nzn + s;
  } else if (axis == 1) {
    lo = ((long)r * nyn + 1) * nzn + s;
    hi = ((long)r * nyn + (nyn - 2)) * nzn + s;
  } else {
    lo = ((long)r * nyn + s) * nzn + 1;
    hi = ((long)r * nyn + s) * nzn + (nzn - 2);
  }
#pragma unroll
  for (int m = 0; m < 10; ++m) {
    float *a = M.m[m];
    if (periodic) {
      const float sum = a[lo] + a[hi];
      a[lo] = sum;
      a[hi] = sum;
    } else {
      a[lo] *= 2.0f;
      a[hi] *= 2.0f;
    }
  }
}

inline unsigned blocks_for(long n) { return (unsigned)ceil_div(n, TPB); }

// Deposits of at least this many particles sort them by cell first.
constexpr long P2S_MIN = 65536;

}  // namespace

int launch_pack_fields(const float *const f[6], float4 *eb4, float2 *eb2, long nodes,
                       cudaStream_t s) {
  const unsigned blocks = (unsigned)std::min<long>(ceil_div(nodes, TPB), 4096);
  k_pack_fields<<<blocks, TPB, 0, s>>>(f[0], f[1], f[2], f[3], f[4], f[5], eb4, eb2, nodes);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  return SPB_OK;
}

int launch_plain_mover(const GeomDev &g, const PushDev &p, const PackedFields &F, float *x,
                       float *y, float *z, float *u, float *v, float *w, long n, int *err,
                       cudaStream_t s, int bc_variant) {
  if (n <= 0) return SPB_OK;
  if (bc_variant == 0)
    k_plain_mover<0><<<blocks_for(n), TPB, 0, s>>>(g, p, F, x, y, z, u, v, w, n, err);
  else
    k_plain_mover<1><<<blocks_for(n), TPB, 0, s>>>(g, p, F, x, y, z, u, v, w, n, err);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  return SPB_OK;
}

int launch_sum_species(const float *const *bases, int ns, long nodes, float *net,
                       cudaStream_t s) {
  if (ns < 1 || ns > SUM_MAX_SPECIES) return fail(SPB_ERR_UNSUPPORTED, "1..32 species");
  SpeciesBases S{};
  for (int i = 0; i < ns; ++i) S.b[i] = bases[i];
  k_sum_species<<<(unsigned)std::min<long>(ceil_div(10 * nodes, TPB), 4096), TPB, 0, s>>>(
      S, ns, nodes, net);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  return SPB_OK;
}

namespace {
// The device's stream-ordered pool keeps freed memory for reuse (once per
// device), so the per-deposit accumulators map nothing after the first.
void keep_pool_memory() {
  static std::atomic<unsigned long long> done{0};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev >= 64 || ((done.load() >> dev) & 1ull)) {
    cudaGetLastError();
    return;
  }
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    unsigned long long keep = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  done |= 1ull << dev;
}

}  // namespace

namespace {
std::atomic<int> g_deposit_mode{SPB_DEPOSIT_ACCUMULATOR};
}  // namespace

void *pool_alloc(size_t bytes, cudaStream_t s) {
  keep_pool_memory();
  void *p = nullptr;
  if (cudaMallocAsync(&p, std::max<size_t>(bytes, 1), s) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return p;
}

void pool_free(void *p, cudaStream_t s) {
  if (p) cudaFreeAsync(p, s);
}

float *plain_acc_alloc(const GeomDev &g, cudaStream_t s) {
  if (g_deposit_mode.load() == SPB_DEPOSIT_DIRECT) return nullptr;
  keep_pool_memory();
  const size_t bytes = (size_t)g.nxn * g.nyn * g.nzn * ACC_STRIDE * sizeof(float);
  float *acc = nullptr;
  if (cudaMallocAsync(reinterpret_cast<void **>(&acc), bytes, s) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  // the 16-byte adds need the alignment (pool allocations have it)
  if ((reinterpret_cast<uintptr_t>(acc) & 15u) || cudaMemsetAsync(acc, 0, bytes, s) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeAsync(acc, s);
    cudaGetLastError();
    return nullptr;
  }
  return acc;
}

int plain_acc_fold(float *acc, const GeomDev &g, float *const mom[10], cudaStream_t s) {
  if (!acc) return SPB_OK;
  const long nodes = (long)g.nxn * g.nyn * g.nzn;
  Moments10 M;
  for (int m = 0; m < 10; ++m) M.m[m] = mom[m];
  k_fold_acc<<<(unsigned)std::min<long>(ceil_div(nodes, TPB), 4096), TPB, 0, s>>>(
      reinterpret_cast<const float4 *>(acc), nodes, M);
  const cudaError_t e = cudaGetLastError();
  cudaFreeAsync(acc, s);
  if (e != cudaSuccess) return fail_cuda(e, "k_fold_acc");
  g_launches++;
  return SPB_OK;
}

namespace {
DepTarget target(float *acc, float *const mom[10]) {
  DepTarget T;
  T.acc = acc;
  for (int m = 0; m < 10; ++m) T.mom.m[m] = mom[m];
  return T;
}
}  // namespace

int launch_plain_p2g_into(const GeomDev &g, const float *x, const float *y, const float *z,
                          const float *u, const float *v, const float *w, const float *q, long n,
                          float *acc, float *const mom[10], int *err, cudaStream_t s) {
  if (n <= 0) return SPB_OK;
  const DepTarget T = target(acc, mom);
  const unsigned chunks = (unsigned)ceil_div(n, GP_CHUNK);
  // the particles in cell order first (above P2S_MIN; scratch from the
  // device's pool, skipped if it cannot be had)
  unsigned *scratch = nullptr, *perm = nullptr;
  const long nodes = (long)g.nxn * g.nyn * g.nzn;
  if (n >= P2S_MIN) {
    const long nb = ceil_div(nodes, P2S_B);
    keep_pool_memory();
    const size_t words = (size_t)2 * n + 2 * nodes + nb;
    if (cudaMallocAsync(reinterpret_cast<void **>(&scratch), words * sizeof(unsigned), s) !=
        cudaSuccess) {
      cudaGetLastError();
      scratch = nullptr;
    }
    if (scratch) {
      unsigned *key = scratch, *pm = scratch + n, *count = pm + n, *first = count + nodes;
      unsigned *bsum = first + nodes;
      SPB_CUDA(cudaMemsetAsync(count, 0, nodes * sizeof(unsigned), s));
      const unsigned blocks = (unsigned)std::min<long>(ceil_div(n, TPB), 148L * 16);
      k_p2g_keys<<<blocks, TPB, 0, s>>>(g, x, y, z, n, key, count);
      k_p2s_scan_blocks<<<(unsigned)nb, P2S_B, 0, s>>>(count, nodes, first, bsum);
      k_p2s_scan_sums<<<1, P2S_B, 0, s>>>(bsum, (int)nb);
      k_p2s_scan_add<<<(unsigned)nb, P2S_B, 0, s>>>(first, nodes, bsum);
      k_p2g_scatter<<<blocks, TPB, 0, s>>>(key, n, first, pm);
      SPB_CUDA(cudaGetLastError());
      g_launches += 5;
      perm = pm;
    }
  }
  if (perm && acc)
    k_plain_p2g_runs<true><<<chunks, RUN_TPB, 0, s>>>(g, x, y, z, u, v, w, q, n, perm, T, err);
  else if (perm)
    k_plain_p2g_runs<false><<<chunks, RUN_TPB, 0, s>>>(g, x, y, z, u, v, w, q, n, perm, T, err);
  else if (acc)
    k_plain_p2g_grouped<true><<<chunks, GP_TPB, 0, s>>>(g, x, y, z, u, v, w, q, n, T, err);
  else
    k_plain_p2g_grouped<false><<<chunks, GP_TPB, 0, s>>>(g, x, y, z, u, v, w, q, n, T, err);
  if (scratch) cudaFreeAsync(scratch, s);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  return SPB_OK;
}

int launch_plain_mover_interp_into(const GeomDev &g, const PushDev &p, const PackedFields &F,
                                   float *x, float *y, float *z, float *u, float *v, float *w,
                                   const float *q, long n, float *acc, float *const mom[10],
                                   int *err, cudaStream_t s) {
  if (n <= 0) return SPB_OK;
  const DepTarget T = target(acc, mom);
  if (acc)
    k_plain_mover_interp<true><<<blocks_for(n), TPB, 0, s>>>(g, p, F, x, y, z, u, v, w, q, n, T,
                                                             err);
  else
    k_plain_mover_interp<false><<<blocks_for(n), TPB, 0, s>>>(g, p, F, x, y, z, u, v, w, q, n,
                                                              T, err);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  return SPB_OK;
}

int launch_plain_p2g(const GeomDev &g, const float *x, const float *y, const float *z,
                     const float *u, const float *v, const float *w, const float *q, long n,
                     float *const mom[10], int *err, cudaStream_t s) {
  if (n <= 0) return SPB_OK;
  float *acc = plain_acc_alloc(g, s);
  const int rc = launch_plain_p2g_into(g, x, y, z, u, v, w, q, n, acc, mom, err, s);
  if (rc) {
    if (acc) cudaFreeAsync(acc, s);
    return rc;
  }
  return plain_acc_fold(acc, g, mom, s);
}

int launch_plain_mover_interp(const GeomDev &g, const PushDev &p, const PackedFields &F,
                              float *x, float *y, float *z, float *u, float *v, float *w,
                              const float *q, long n, float *const mom[10], int *err,
                              cudaStream_t s) {
  if (n <= 0) return SPB_OK;
  float *acc = plain_acc_alloc(g, s);
  const int rc = launch_plain_mover_interp_into(g, p, F, x, y, z, u, v, w, q, n, acc, mom, err, s);
  if (rc) {
    if (acc) cudaFreeAsync(acc, s);
    return rc;
  }
  return plain_acc_fold(acc, g, mom, s);
}

int launch_apply_bc_ids(int nxn, int nyn, int nzn, const int periodic[3],
                        float *const mom[10], cudaStream_t s, long *launches) {
  Moments10 M;
  for (int m = 0; m < 10; ++m) M.m[m] = mom[m];
  const long plane[3] = {(long)(nyn - 2) * (nzn - 2), (long)(nxn - 2) * (nzn - 2),
                         (long)(nxn - 2) * (nyn - 2)};
  // periodic folds in axis order, then the doubling of non-periodic axes
  for (int pass = 0; pass < 2; ++pass)
    for (int axis = 0; axis < 3; ++axis) {
      const bool fold = periodic[axis] != 0;
      if (fold != (pass == 0)) continue;
      k_bc_fold<<<blocks_for(plane[axis]), TPB, 0, s>>>(M, nxn, nyn, nzn, axis, fold ? 1 : 0);
      SPB_CUDA(cudaGetLastError());
      g_launches++;
      if (launches) ++*launches;
    }
  return SPB_OK;
}

}  // namespace spb

extern "C" int spb_set_plain_deposit_mode(int mode) {
  if (mode != SPB_DEPOSIT_ACCUMULATOR && mode != SPB_DEPOSIT_DIRECT)
    return spb::fail(SPB_ERR_INVALID, "spb_set_plain_deposit_mode: unknown mode");
  return spb::g_deposit_mode.exchange(mode);
}
