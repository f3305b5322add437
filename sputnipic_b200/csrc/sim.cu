// Precision form of the mover + deposit (spb_sim_*): HBM-resident particles
// bucketed by cell, int32 cell (implicit in the bucket) + FP32 in-cell
// offsets, FP32 push and gather, FP32 per-cell deposit sums added into FP64
// global moments.
//
// The arithmetic is the reference's mover_PC / interpP2G (src/Mover.cpp:4-162,
// :385-572) restated in cell units: a position is (cell c, offset o) with
// x = (c + o) * dx, the predictor-corrector displacement is u * (dt/2)/dx,
// the trilinear weights are o and 1 - o, and the moments carry one factor of
// invVOL, as the reference's weight * invVOL does once the weight's own
// xi*eta*zeta*invVOL is normalised. Reference behaviours kept:
//   - the mover's cell index truncates toward zero (src/Mover.cpp:39-41), so
//     a predicted position in (-dx, 0) gathers from cell 0 with a negative
//     offset (extrapolation), not from the guard cell;
//   - the particle BC tests "x > L" and then "x < 0" (src/Mover.cpp:103-157);
//   - the deposit uses the post-BC position and velocity, floor cell.
//
// A cycle is two kernels: k_push moves every particle and writes it into the
// bucket of its new cell (second buffer set), k_deposit sums each cell's
// bucket in registers and adds the node sums into the moments.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <type_traits>
#include <vector>

#include "grid_ctx.h"
#include "kernels.h"
#include "sim_host.h"
#include "sim_kernels.cuh"
#include "warp_sum.cuh"

namespace spb {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int SIM_TPB = 256;                 // 8 warps per CTA
constexpr int SIM_NW = SIM_TPB / 32;
constexpr long long WAIT_CYCLES = 200000000; // bounded mbarrier wait (~0.1 s)

// ---------------------------------------------------------------------------
// PTX helpers: mbarrier + TMA tensor copy (no cluster, one CTA)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// Raises the barrier's expected transaction bytes without arriving: several
// copies can be armed one by one and the phase closed by one mbar_arrive.
__device__ __forceinline__ void mbar_expect_tx_only(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}

// Waits for the phase with a cycle budget; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned phase) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, phase))
    if (clock64() - t0 > WAIT_CYCLES) return false;
  return true;
}

// 4D tiled TMA load of one box into shared memory, completion on `bar`.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, int c3, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3),
      "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Untiled bulk copy global -> this CTA's shared memory (no multicast),
// completion on `bar`. Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, unsigned bytes,
                                          uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// ---------------------------------------------------------------------------
// push in cell units
// ---------------------------------------------------------------------------

// floor(p) for |p| < 2^22 as a float (s) and an int, from one add rounded
// toward -infinity against 1.5 * 2^23 (whose neighbours are the integers):
// full-rate adds instead of a rounding instruction and a conversion. For
// |p| >= 2^22, infinities and NaN the int is at least 2^22 away from 0 (the
// float bit patterns are ordered), so a particle that far out lands outside
// any grid, where the range check flags it.
__device__ __forceinline__ int floor_split(float p, float &s) {
  constexpr float M = 12582912.0f;   // 1.5 * 2^23
  const float t = __fadd_rd(p, M);
  s = __fsub_rn(t, M);
  return __float_as_int(t) - __float_as_int(M);
}

// Gather cell and fraction of a predicted position p (cells, relative to the
// particle's cell c), rounding down. Cells outside [-1, N] are left to the
// gather's bounds handling.
__device__ __forceinline__ void locate(float p, int c, int &g, float &f) {
  float s;
  g = c + floor_split(p, s);
  f = __fsub_rn(p, s);
}

// Below the domain the reference's int() truncates toward zero
// (src/Mover.cpp:39-41): the cell rounds up and the fraction goes negative.
__device__ __forceinline__ void truncate_below(int &g, float &f) {
  const bool trunc = (g < 0) & (f != 0.0f);
  g = trunc ? g + 1 : g;
  f = trunc ? f - 1.0f : f;
}

// Particle BC on one axis in cell units: "x > L" first, then "x < 0"
// (src/Mover.cpp:103-157). On entry o is in [0, 1). Branch-free.
__device__ __forceinline__ void bc_cell(int &c, float &o, float &vel, int N, int periodic) {
  {
    const bool over = (c > N) | ((c == N) & (o > 0.0f));
    const bool pos = o > 0.0f;
    const int cr = pos ? 2 * N - c - 1 : 2 * N - c;     // mirror of x about L
    const float orf = pos ? 1.0f - o : o;
    c = over ? (periodic ? c - N : cr) : c;
    o = (over & !periodic) ? orf : o;
    vel = (over & !periodic) ? -vel : vel;
  }
  {
    const bool under = c < 0;
    const bool pos = o > 0.0f;
    const int cr = pos ? -c - 1 : -c;                    // mirror of x about 0
    const float orf = pos ? 1.0f - o : o;
    c = under ? (periodic ? c + N : cr) : c;
    o = (under & !periodic) ? orf : o;
    vel = (under & !periodic) ? -vel : vel;
  }
  const bool top = (c == N) & (o == 0.0f);   // x == L exactly: top face of the last cell
  c = top ? N - 1 : c;
  o = top ? 1.0f : o;
}

// Final position update on one axis: p = o + displacement, new cell and offset.
__device__ __forceinline__ void advance(int &c, float &o, float disp) {
  const float p = __fadd_rn(o, disp);
  float s;
  c += floor_split(p, s);
  o = __fsub_rn(p, s);
  const bool wrap = o >= 1.0f;
  c = wrap ? c + 1 : c;
  o = wrap ? 0.0f : o;
}

// E and B as three packed pairs (Ex,Ey), (Ez,Bx), (By,Bz): the node record in
// shared memory is (Ex,Ey,Ez,Bx | By,Bz,0,0), so every pair is a register
// pair and one packed FP32x2 FMA updates two components.
struct Field6 {
  float2 exy, ezbx, byz;
};

__device__ __forceinline__ Field6 first_node(float w, float4 a, float2 b) {
  const float2 w2 = make_float2(w, w);
  return {__fmul2_rn(w2, make_float2(a.x, a.y)), __fmul2_rn(w2, make_float2(a.z, a.w)),
          __fmul2_rn(w2, b)};
}

__device__ __forceinline__ void acc_node(Field6 &F, float w, float4 a, float2 b) {
  const float2 w2 = make_float2(w, w);
  F.exy = __ffma2_rn(w2, make_float2(a.x, a.y), F.exy);
  F.ezbx = __ffma2_rn(w2, make_float2(a.z, a.w), F.ezbx);
  F.byz = __ffma2_rn(w2, b, F.byz);
}

template <int TX, int TY, int TZ>
struct Tile {
  static constexpr int BX = TX + 3, BY = TY + 3, BZ = TZ + 3;
  static constexpr int BN = BX * BY * BZ;    // staged nodes
  static constexpr int TC = TX * TY * TZ;    // cells per tile
  // floats per field stage, padded so every stage starts on the 128-byte
  // boundary a TMA tensor copy's shared-memory destination needs
  static constexpr int SF = ((8 * BN + 31) / 32) * 32;
  static_assert((SF * 4) % 128 == 0, "field stages must stay 128-byte aligned");
};

// Trilinear gather of E and B from the node array in HBM/L2, for a particle
// whose nodes lie outside the staged tile (rare: kept out of line, so the
// staged gather's registers and code stay those of the common case). The
// same operations in the same order as the staged gather below, so a
// particle's push does not depend on which of the two paths served it.
__device__ __noinline__ Field6 gather_global(const float *__restrict__ fields8, int nxc, int nyc,
                                             int nzc, int nyn, int nzn, int gx, int gy, int gz,
                                             float fx, float fy, float fz) {
  const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
  const long sy = nzn, sx = (long)nyn * nzn;
  const int hx = min(max(gx, -1), nxc), hy = min(max(gy, -1), nyc), hz = min(max(gz, -1), nzc);
  const long n0 = (long)(hx + 1) * sx + (long)(hy + 1) * sy + (hz + 1);
  Field6 F[2];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wab = __fmul_rn(wx[a], wy[b]);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const long n = n0 + a * sx + b * sy + c;
        const float4 A = __ldg(reinterpret_cast<const float4 *>(fields8 + 8 * n));
        const float2 B = __ldg(reinterpret_cast<const float2 *>(fields8 + 8 * n + 4));
        if (b == 0 && c == 0)
          F[a] = first_node(__fmul_rn(wab, wz[c]), A, B);
        else
          acc_node(F[a], __fmul_rn(wab, wz[c]), A, B);
      }
    }
  return {__fadd2_rn(F[0].exy, F[1].exy), __fadd2_rn(F[0].ezbx, F[1].ezbx),
          __fadd2_rn(F[0].byz, F[1].byz)};
}

// Trilinear gather of E and B at fraction f per axis from the staged tile,
// node n0 the lower corner of the particle's cell (tile node index). The two
// x layers accumulate separately (shorter dependency chains).
template <int TX, int TY, int TZ>
__device__ __forceinline__ Field6 gather(const float *__restrict__ sF, int n0, float fx, float fy,
                                         float fz) {
  using T = Tile<TX, TY, TZ>;
  const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
  Field6 F[2];
#pragma unroll
  for (int a = 0; a < 2; ++a) {
#pragma unroll
    for (int b = 0; b < 2; ++b) {
      const float wab = __fmul_rn(wx[a], wy[b]);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int n = n0 + (a * T::BY + b) * T::BZ + c;
        const float4 A = *reinterpret_cast<const float4 *>(sF + 8 * n);
        const float2 B = *reinterpret_cast<const float2 *>(sF + 8 * n + 4);
        if (b == 0 && c == 0)   // each layer's sum starts from its first product
          F[a] = first_node(__fmul_rn(wab, wz[c]), A, B);
        else
          acc_node(F[a], __fmul_rn(wab, wz[c]), A, B);
      }
    }
  }
  return {__fadd2_rn(F[0].exy, F[1].exy), __fadd2_rn(F[0].ezbx, F[1].ezbx),
          __fadd2_rn(F[0].byz, F[1].byz)};
}

// Tile node index of the lower corner of cell g (tile origin c0), and whether
// all 8 nodes of the cell are staged; 0 (a valid node) when they are not.
template <int TX, int TY, int TZ>
__device__ __forceinline__ int tile_node(int c0x, int c0y, int c0z, int gx, int gy, int gz,
                                         bool &inbox) {
  using T = Tile<TX, TY, TZ>;
  const int bx = gx + 1 - c0x, by = gy + 1 - c0y, bz = gz + 1 - c0z;
  inbox = ((unsigned)bx <= (unsigned)(TX + 1)) & ((unsigned)by <= (unsigned)(TY + 1)) &
          ((unsigned)bz <= (unsigned)(TZ + 1));
  return inbox ? (bx * T::BY + by) * T::BZ + bz : 0;
}

// One NiterMover step from the field F at the predicted position: the
// implicit velocity solve (src/Mover.cpp:60-89), giving u-tilde and the
// half-step displacement in cells.
__device__ __forceinline__ void boris(const CycleParams &P, const Field6 &F, float qomdt2,
                                      float u, float v, float w, float &up, float &vp, float &wp,
                                      float &dx, float &dy, float &dz) {
  // every operation spelled out (no contraction left to the compiler), so
  // each inlined copy of the push rounds alike
  const float ex = F.exy.x, ey = F.exy.y, ez = F.ezbx.x;
  const float bx = F.ezbx.y, by = F.byz.x, bz = F.byz.y;
  const float b2 = __fmaf_rn(bz, bz, __fmaf_rn(by, by, __fmul_rn(bx, bx)));
  const float omdtsq = __fmul_rn(__fmul_rn(qomdt2, qomdt2), b2);
  const float denom = __fdividef(1.0f, __fadd_rn(1.0f, omdtsq));
  const float ut = __fmaf_rn(qomdt2, ex, u);
  const float vt = __fmaf_rn(qomdt2, ey, v);
  const float wt = __fmaf_rn(qomdt2, ez, w);
  const float qud = __fmul_rn(qomdt2, __fmaf_rn(wt, bz, __fmaf_rn(vt, by, __fmul_rn(ut, bx))));
  up = __fmul_rn(__fmaf_rn(qomdt2, __fmaf_rn(qud, bx, __fmaf_rn(-wt, by, __fmul_rn(vt, bz))), ut),
                 denom);
  vp = __fmul_rn(__fmaf_rn(qomdt2, __fmaf_rn(qud, by, __fmaf_rn(-ut, bz, __fmul_rn(wt, bx))), vt),
                 denom);
  wp = __fmul_rn(__fmaf_rn(qomdt2, __fmaf_rn(qud, bz, __fmaf_rn(-vt, bx, __fmul_rn(ut, by))), wt),
                 denom);
  dx = __fmul_rn(up, P.hdt[0]);
  dy = __fmul_rn(vp, P.hdt[1]);
  dz = __fmul_rn(wp, P.hdt[2]);
}

// Field at (cell g, fraction f): from the staged tile at node n0 when the
// cell's nodes are staged (inbox), from HBM/L2 for the lanes whose are not.
// All 32 lanes call.
template <int TX, int TY, int TZ>
__device__ __forceinline__ Field6 field_at(const CycleParams &P, const float *__restrict__ sF,
                                           int n0, bool inbox, int gx, int gy, int gz, float fx,
                                           float fy, float fz) {
  Field6 F = gather<TX, TY, TZ>(sF, n0, fx, fy, fz);
  if (__any_sync(0xffffffffu, !inbox)) {
    if (!inbox)
      F = gather_global(P.fields8, P.nxc, P.nyc, P.nzc, P.nyn, P.nzn, gx, gy, gz, fx, fy, fz);
  }
  return F;
}

// mover_PC for one particle in cell units (src/Mover.cpp:33-157). n0c is the
// tile node of the particle's start cell (the first gather is there, at the
// stored offsets), or -1 when the start cell is not known to be staged. All
// 32 lanes of the warp must call (the gathers vote: lanes whose cell lies
// past the staged halo re-gather from HBM/L2). P.niter >= 1.
template <int TX, int TY, int TZ>
__device__ __forceinline__ void push(const CycleParams &P, const float *__restrict__ sF, int c0x,
                                     int c0y, int c0z, int n0c, float qomdt2, int &cx, int &cy,
                                     int &cz, float &ox, float &oy, float &oz, float &u, float &v,
                                     float &w, int &bad) {
  float dx, dy, dz;   // predicted displacement in cells
  float up, vp, wp;
  {
    // the first iteration gathers at the stored position, in the start cell
    bool inbox = true;
    int n0 = n0c;
    if (n0c < 0) n0 = tile_node<TX, TY, TZ>(c0x, c0y, c0z, cx, cy, cz, inbox);
    const Field6 F = field_at<TX, TY, TZ>(P, sF, n0, inbox, cx, cy, cz, ox, oy, oz);
    boris(P, F, qomdt2, u, v, w, up, vp, wp, dx, dy, dz);
  }
#pragma unroll 1
  for (int it = 1; it < P.niter; ++it) {
    int gx, gy, gz;
    float fx, fy, fz;
    locate(__fadd_rn(ox, dx), cx, gx, fx);
    locate(__fadd_rn(oy, dy), cy, gy, fy);
    locate(__fadd_rn(oz, dz), cz, gz, fz);
    if (__any_sync(0xffffffffu, (gx | gy | gz) < 0)) {   // some lane is below the domain
      truncate_below(gx, fx);
      truncate_below(gy, fy);
      truncate_below(gz, fz);
    }
    bool inbox;
    const int n0 = tile_node<TX, TY, TZ>(c0x, c0y, c0z, gx, gy, gz, inbox);
    const Field6 F = field_at<TX, TY, TZ>(P, sF, n0, inbox, gx, gy, gz, fx, fy, fz);
    boris(P, F, qomdt2, u, v, w, up, vp, wp, dx, dy, dz);
  }
  u = __fmaf_rn(2.0f, up, -u);
  v = __fmaf_rn(2.0f, vp, -v);
  w = __fmaf_rn(2.0f, wp, -w);
  advance(cx, ox, __fmul_rn(up, P.fdt[0]));
  advance(cy, oy, __fmul_rn(vp, P.fdt[1]));
  advance(cz, oz, __fmul_rn(wp, P.fdt[2]));
  // the particle BC, the range flag and the clamps change nothing for a
  // particle whose new cell is inside the domain: skipped unless some lane
  // needs them
  const bool inside = ((unsigned)cx < (unsigned)P.nxc) & ((unsigned)cy < (unsigned)P.nyc) &
                      ((unsigned)cz < (unsigned)P.nzc);
  if (!__all_sync(0xffffffffu, inside)) {
    bc_cell(cx, ox, u, P.nxc, P.periodic[0]);
    bc_cell(cy, oy, v, P.nyc, P.periodic[1]);
    bc_cell(cz, oz, w, P.nzc, P.periodic[2]);
    bad |= (cx < 0) | (cx >= P.nxc) | (cy < 0) | (cy >= P.nyc) | (cz < 0) | (cz >= P.nzc);
    cx = min(max(cx, 0), P.nxc - 1);
    cy = min(max(cy, 0), P.nyc - 1);
    cz = min(max(cz, 0), P.nzc - 1);
  }
}

// Deposit terms of one particle added to 40 packed accumulators:
// acc[node*5 + k] += W_node * (mf[k], mf[k+5]) with the moment factors
// mf = 1, u, v, w, uu | uv, uw, vv, vw, ww, i.e. the pairs (1,uv) (u,uw)
// (v,vv) (w,vw) (uu,ww), in the reference order rhon, Jx, Jy, Jz, pxx | pxy,
// pxz, pyy, pyz, pzz (src/Mover.cpp:466-570); node = a*4 + b*2 + c with
// a/b/c = 1 the upper node on that axis, XOR-permuted by bits 4/3/2 of
// `perm` (the lane for warp_sum80, 0 for the plain order). q is folded into
// the x weights; q = 0 adds nothing.
__device__ __forceinline__ void add_terms(float2 (&acc)[40], float q, float ox, float oy, float oz,
                                          float u, float v, float w, int perm) {
  const bool px = perm & 16, py = perm & 8, pz = perm & 4;
  const float lox = 1.0f - ox, loy = 1.0f - oy, loz = 1.0f - oz;
  const float wx0 = q * (px ? ox : lox), wx1 = q * (px ? lox : ox);
  const float wy0 = py ? oy : loy, wy1 = py ? loy : oy;
  const float wz0 = pz ? oz : loz, wz1 = pz ? loz : oz;
  const float2 mf[5] = {make_float2(1.0f, u * v), make_float2(u, u * w), make_float2(v, v * v),
                        make_float2(w, v * w), make_float2(u * u, w * w)};
  const float wxy[4] = {wx0 * wy0, wx0 * wy1, wx1 * wy0, wx1 * wy1};
#pragma unroll
  for (int ab = 0; ab < 4; ++ab) {
    const float W0 = wxy[ab] * wz0, W1 = wxy[ab] * wz1;
    const float2 W02 = make_float2(W0, W0), W12 = make_float2(W1, W1);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
      acc[(ab * 2 + 0) * 5 + k] = __ffma2_rn(W02, mf[k], acc[(ab * 2 + 0) * 5 + k]);
      acc[(ab * 2 + 1) * 5 + k] = __ffma2_rn(W12, mf[k], acc[(ab * 2 + 1) * 5 + k]);
    }
  }
}

// One 32-byte record store (one 256-bit access; p 32-byte aligned).
__device__ __forceinline__ void st_rec(float4 *p, float4 a, float4 b) {
  asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(a.x),
               "f"(a.y), "f"(a.z), "f"(a.w), "f"(b.x), "f"(b.y), "f"(b.z), "f"(b.w)
               : "memory");
}

// Stores one pushed record in slot `slot` of the bucket [dbase, dend) of cell
// `key`, or appends it to the overflow list when the bucket is full. Returns
// 1 if the overflow list was full too (the particle is lost; reported).

__device__ __forceinline__ int put_at(const SpeciesDev &S, int key, long long dbase,
                                      long long dend, int slot, float4 a, float4 b) {
  if (dbase + slot < dend) {
    st_rec(S.rout + 2 * (dbase + slot), a, b);
    return 0;
  }
  const int o = atomicAdd(S.ocout, 1);
  if (o >= S.ocap) return 1;
  st_rec(S.oout + 2 * (long)o, a, b);
  S.okout[o] = key;
  return 0;
}

// A pushed slot of 32 particles whose stores wait for their counter updates:
// the updates are issued right after the push and consumed one slot later,
// so their round trip overlaps the next slot's push. The lanes are grouped by
// destination cell; each group's lowest lane reserves the group's slots with
// one atomic. The records wait in a per-warp shared-memory staging area (two
// float4 per lane).
struct Pending {
  long long dbase, dend;  // destination bucket
  int key;                // destination cell
  int slot0;              // group leader: first slot reserved for its group
  int leader, rank;       // this lane's group leader and rank in the group
  bool valid;
};

// Completes a pending slot. All 32 lanes call.
__device__ __forceinline__ void flush(const SpeciesDev &S, const Pending &p, const float4 *stage,
                                      int lane, int &lost) {
  const int s0 = __shfl_sync(FULL, p.slot0, p.leader);
  if (p.valid)
    lost |= put_at(S, p.key, p.dbase, p.dend, s0 + p.rank, stage[lane], stage[32 + lane]);
}

// Issues the counter updates of a pushed slot and stages its records. All 32
// lanes call, after the previous slot's flush.
// `far`: the particle goes to the overflow list whatever its bucket's room
// (the fused cycle's particles that left their tile's neighbourhood; every
// lane of a destination group has the same value).
__device__ __forceinline__ void issue_slot(const SpeciesDev &S, Pending &p, float4 *stage,
                                          int nkey, bool valid, float4 a, float4 b, int lane,
                                          bool far = false) {
  const unsigned peers = __match_any_sync(FULL, valid ? nkey : -1);
  p.leader = __ffs(peers) - 1;
  p.rank = __popc(peers & ((1u << lane) - 1u));
  p.slot0 = 0;
  const bool place = valid && !far;
  if (place && lane == p.leader) p.slot0 = atomicAdd(S.cout + nkey, __popc(peers));
  p.key = nkey;
  p.valid = valid;
  p.dbase = place ? __ldg(S.base + nkey) : 0;
  p.dend = place ? __ldg(S.base + nkey + 1) : 0;
  stage[lane] = a;
  stage[32 + lane] = b;
}

// Records per half of a warp's record ring: 4 KB at two resident CTAs per SM,
// 2 KB at three or more (so that three CTAs fit in shared memory).
template <int MINB>
__host__ __device__ constexpr int ring_half() {
  return MINB >= 3 ? 64 : 128;
}

// Independent jobs (own grid, fields, species and buckets; one tile shape)
// processed by one launch: the launch walks the concatenation of the jobs'
// tiles, and a CTA reads a tile's job from the prefix table.
struct JobTable {
  int njobs, total_tiles;
  const int *tile_base;          // [njobs + 1] first launch-wide tile of each job
  const CycleParams *params;     // [njobs]
};

// The jobs' field maps travel as a kernel parameter, like the single job's.
struct JobMaps {
  CUtensorMap m[SERVE_MAX_JOBS];
};
struct NoMaps {
  int unused;
};
template <bool MULTI>
using MapsOf = typename std::conditional<MULTI, JobMaps, NoMaps>::type;

// The job of launch-wide tile t: the largest j with tile_base[j] <= t.
__device__ __forceinline__ int job_of(const JobTable &J, int t) {
  int lo = 0, hi = J.njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (J.tile_base[mid] <= t)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Copies one job's parameters into shared memory (all threads of the CTA call).
__device__ __forceinline__ void load_params(CycleParams *dst, const CycleParams *src) {
  static_assert(sizeof(CycleParams) % 8 == 0, "copied in 8-byte words");
  const unsigned long long *s = reinterpret_cast<const unsigned long long *>(src);
  unsigned long long *d = reinterpret_cast<unsigned long long *>(dst);
  for (int i = threadIdx.x; i < (int)(sizeof(CycleParams) / 8); i += blockDim.x) d[i] = s[i];
  __syncthreads();
}

// Per-warp state of the push that lives across tiles and jobs.
struct PushWarp {
  float4 *wrec;        // staged records of the pending slot
  float4 *ring;        // record ring: two halves of RH records
  uint64_t *cbar;      // the halves' barriers
  unsigned phase = 0, inflight = 0;   // per half: next parity, copies armed
  bool dead = false;   // a bounded wait for records ran out
  int bad = 0, lost = 0;
};

// All species of one tile (tile-local index `tile` of the job P) on the
// staged fields sF. All threads call.
//
// Each warp owns NC cells of the tile (tile-local warp + j * NW) and pushes
// their records as one stream: slot k holds the stream's records 32k..32k+31
// whatever their cells, so slots stay full however the counts fall. Lane 0
// copies the cells' records into a two-half ring (bulk copies, one per cell
// piece; a half's barrier closes after its last piece is armed); a half is
// refilled as soon as its last slot has been read.
// Whether a destination tile coordinate d tiles away on an axis of n tiles
// (periodic or not) lies outside the source tile's neighbourhood.
__device__ __forceinline__ bool far_axis(int d, int n, int periodic) {
  if (periodic && n > 2) d = d == n - 1 ? -1 : (d == 1 - n ? 1 : d);
  return d < -1 || d > 1;
}

template <int TX, int TY, int TZ, int RH, bool FUSED = false>
__device__ __forceinline__ void push_tile(const CycleParams &P, int tile, const float *sF,
                                          PushWarp &W) {
  using T = Tile<TX, TY, TZ>;
  constexpr int NC = T::TC / SIM_NW;   // cells per warp and tile
  static_assert(RH % 32 == 0, "slots must not straddle ring halves");
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tz = tile % P.ntz, ty = (tile / P.ntz) % P.nty, tx = tile / (P.ntz * P.nty);
  const int c0x = tx * TX, c0y = ty * TY, c0z = tz * TZ;
  for (int s = 0; s < P.ns; ++s) {
    const SpeciesDev &S = P.sp[s];
    // lane j < NC: bucket start and particle count of the warp's j-th cell,
    // and cp = the cell's first index in the warp's stream
    long long cb = 0;
    int cc = 0;
    if (lane < NC) {
      const int key = tile * T::TC + warp + lane * SIM_NW;
      cb = S.base[key];
      cc = min(S.cin[key], (int)(S.base[key + 1] - cb));
    }
    int cp = cc;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(FULL, cp, o);
      if (lane >= o) cp += t;
    }
    const int total = __shfl_sync(FULL, cp, 31);
    cp -= cc;
    if (total == 0 || W.dead) continue;

    int pj = 0, poff = 0, pv = 0;   // next record to copy: cell, offset, stream index
    // Copies the next records (at most RH) into half h; all lanes call.
    auto fill = [&](int h) {
      const int end = min(pv + RH, total);
      if (lane == 0) fence_proxy_async();   // the half's previous reads come first
      while (pv < end) {
        int cnt = __shfl_sync(FULL, cc, pj);
        while (poff >= cnt && pj < NC - 1) {
          ++pj;
          poff = 0;
          cnt = __shfl_sync(FULL, cc, pj);
        }
        const int n = min(cnt - poff, end - pv);
        if (n <= 0) break;   // unreachable: the counts sum to total
        const long long b0 = __shfl_sync(FULL, cb, pj);
        if (lane == 0) {
          mbar_expect_tx_only(W.cbar + h, (unsigned)n * 32u);
          bulk_load(W.ring + 2 * (pv % (2 * RH)), S.rin + 2 * (b0 + poff), (unsigned)n * 32u,
                    W.cbar + h);
        }
        pv += n;
        poff += n;
      }
      if (lane == 0) mbar_arrive(W.cbar + h);
      W.inflight |= 1u << h;
    };
    fill(0);
    if (pv < total) fill(1);

    Pending pend;
    pend.valid = false;
    pend.slot0 = pend.leader = pend.rank = 0;
#pragma unroll 1
    for (int rv = 0; rv < total; rv += 32) {
      const int h = (rv / RH) & 1;
      if (rv % RH == 0) {   // first slot of half h: wait for its copies
        const bool ok = mbar_wait_bounded(W.cbar + h, (W.phase >> h) & 1u);
        if (!__all_sync(FULL, ok)) {
          W.dead = true;
          break;
        }
        W.phase ^= 1u << h;
        W.inflight &= ~(1u << h);
      }
      const int i = rv + lane;
      const bool valid = i < total;
      // idle lanes of the last slot push a copy of the stream's last particle
      // (results discarded): one instruction stream per warp
      const int ii = valid ? i : total - 1;
      const float4 *rp = W.ring + 2 * (ii % (2 * RH));
      const float4 a = rp[0], b = rp[1];
      // the lane's cell: the last j with cp_j <= ii
      int j = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1) {
        const int cand = j + st;
        const int pc = __shfl_sync(FULL, cp, cand & 31);
        if (cand < NC && pc <= ii) j = cand;
      }
      const int lc = warp + j * SIM_NW;
      const int lx = lc / (TY * TZ), ly = (lc / TZ) % TY, lz = lc % TZ;
      const int n0c = ((lx + 1) * T::BY + (ly + 1)) * T::BZ + (lz + 1);
      int cx = c0x + lx, cy = c0y + ly, cz = c0z + lz;
      float ox = a.x, oy = a.y, oz = a.z, u = b.x, v = b.y, w = b.z;
      int pbad = 0;
      push<TX, TY, TZ>(P, sF, c0x, c0y, c0z, n0c, S.qomdt2, cx, cy, cz, ox, oy, oz, u, v, w,
                       pbad);
      W.bad |= valid ? pbad : 0;
      const int nkey = tile_key<TX, TY, TZ>(cx, cy, cz, P.nty, P.ntz);
      bool far = false;
      if constexpr (FUSED)
        far = far_axis(cx / TX - tx, P.ntx, P.periodic[0]) |
              far_axis(cy / TY - ty, P.nty, P.periodic[1]) |
              far_axis(cz / TZ - tz, P.ntz, P.periodic[2]);
      flush(S, pend, W.wrec, lane, W.lost);   // the previous slot's counters are back
      __syncwarp();
      issue_slot(S, pend, W.wrec, nkey, valid, make_float4(ox, oy, oz, a.w),
                 make_float4(u, v, w, 0.f), lane, far);
      // last slot of half h read by every lane: refill it
      if ((rv + 32) % RH == 0 && pv < total) {
        __syncwarp();
        fill(h);
      }
    }
    flush(S, pend, W.wrec, lane, W.lost);
    __syncwarp();
  }
}

// The overflow entries of every species of job P: pushed with gathers from
// L2 (the staged-tile origin is placed out of reach, so every gather takes
// the global path). sF is any valid staged buffer. All threads call.
// TO_LIST: every pushed entry goes to the new overflow list (the fused cycle
// has deposited the buckets already).
template <int TX, int TY, int TZ, bool TO_LIST = false>
__device__ __forceinline__ void push_overflow(const CycleParams &P, const float *sF, PushWarp &W) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int s = 0; s < P.ns; ++s) {
    const SpeciesDev &S = P.sp[s];
    const int on = min(*S.ocin, S.ocap);
    for (long base = ((long)blockIdx.x * SIM_NW + warp) * 32; base < on;
         base += (long)gridDim.x * SIM_TPB) {
      const int i = (int)base + lane;
      const bool valid = i < on;
      const int ii = valid ? i : on - 1;
      const int key = S.okin[ii];
      const float4 a = S.oin[2 * (long)ii], b = S.oin[2 * (long)ii + 1];
      int cx, cy, cz;
      key_cell<TX, TY, TZ>(key, P.nty, P.ntz, cx, cy, cz);
      float ox = a.x, oy = a.y, oz = a.z, u = b.x, v = b.y, w = b.z;
      int pbad = 0;
      constexpr int FAR = -(1 << 20);
      push<TX, TY, TZ>(P, sF, FAR, FAR, FAR, -1, S.qomdt2, cx, cy, cz, ox, oy, oz, u, v, w,
                       pbad);
      W.bad |= valid ? pbad : 0;
      const int nkey = tile_key<TX, TY, TZ>(cx, cy, cz, P.nty, P.ntz);
      if (valid) {
        if (TO_LIST) {
          W.lost |= put_at(S, nkey, 0, 0, 0, make_float4(ox, oy, oz, a.w),
                           make_float4(u, v, w, 0.f));
        } else {
          const int slot = atomicAdd(S.cout + nkey, 1);
          W.lost |= put_at(S, nkey, S.base[nkey], S.base[nkey + 1], slot,
                           make_float4(ox, oy, oz, a.w), make_float4(u, v, w, 0.f));
        }
      }
    }
  }
}

// Reports and clears a warp state's flags into job P's error word.
__device__ __forceinline__ void report(const CycleParams &P, PushWarp &W) {
  if (W.bad) atomicOr(P.err, ERRBIT_OUT_OF_GRID);
  if (W.lost) atomicOr(P.err, ERRBIT_LOST);
  W.bad = W.lost = 0;
}

// The mover (mover_PC, src/Mover.cpp:4-162) for every species. Persistent
// CTAs walk tiles of TX x TY x TZ cells; one thread stages the tile's E/B
// nodes plus a one-cell halo into shared memory with a TMA tensor copy (two
// stages: the next tile's copy overlaps this tile's work). Warps walk the
// tile's cells, one particle per lane, with the cells' records streamed
// through two shared-memory chunk buffers per warp by bulk copies; the
// gathers of the NiterMover iterations read the staged tile (or L2 past the
// halo), and every pushed particle is written into the bucket of its new
// cell. Afterwards the CTAs push the overflow entries (gathers from L2).
// MULTI = false: one job, parameters P1 and field map fmap. MULTI = true: the
// jobs of table J, each tile's job parameters staged in shared memory.
template <int TX, int TY, int TZ, int MINB, bool MULTI>
__global__ void __launch_bounds__(SIM_TPB, MINB)
    k_push(const __grid_constant__ CUtensorMap fmap, const __grid_constant__ CycleParams P1,
           const __grid_constant__ JobTable J, const __grid_constant__ MapsOf<MULTI> M) {
  using T = Tile<TX, TY, TZ>;
  constexpr int RH = ring_half<MINB>();
  static_assert(T::TC % SIM_NW == 0 && T::TC / SIM_NW <= 32,
                "cells per warp must fit a warp's lanes");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *sF0 = reinterpret_cast<float *>(smem_raw);                 // 2 stages x SF
  float4 *sRec = reinterpret_cast<float4 *>(sF0 + 2 * T::SF);       // NW x 64 staged records
  float4 *sBuf = sRec + SIM_NW * 64;                                // NW x 2 x RH records
  CycleParams *sP = reinterpret_cast<CycleParams *>(sBuf + SIM_NW * 2 * RH * 2);  // MULTI
  uint64_t *bar = reinterpret_cast<uint64_t *>(sP + (MULTI ? 1 : 0));   // 2 + 2 NW

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  PushWarp W;
  W.wrec = sRec + warp * 64;
  W.ring = sBuf + warp * 2 * RH * 2;
  W.cbar = bar + 2 + warp * 2;
  int *const err0 = MULTI ? J.params[0].err : P1.err;
  if (smem_addr(sF0) & 127u) {   // TMA destinations need 128-byte alignment
    if (tid == 0) atomicOr(err0, ERRBIT_SMEM_ALIGN);
    return;
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
  }
  if (lane == 0) {
    mbar_init(W.cbar, 1);
    mbar_init(W.cbar + 1, 1);
  }
  __syncthreads();

  const int ntiles = MULTI ? J.total_tiles : P1.ntx * P1.nty * P1.ntz;
  auto locate_tile = [&](int t, int &job, int &local) {
    if constexpr (MULTI) {
      job = job_of(J, t);
      local = t - J.tile_base[job];
    } else {
      job = 0;
      local = t;
    }
  };
  const unsigned box_bytes = (unsigned)(T::BN * 8 * sizeof(float));
  auto issue = [&](int t, int stage) {   // thread 0
    int job, local;
    locate_tile(t, job, local);
    const int nty = MULTI ? J.params[job].nty : P1.nty;
    const int ntz = MULTI ? J.params[job].ntz : P1.ntz;
    const CUtensorMap *map;
    if constexpr (MULTI)
      map = &M.m[job];
    else
      map = &fmap;
    const int z = local % ntz, y = (local / ntz) % nty, x = local / (ntz * nty);
    fence_proxy_async();
    mbar_expect_tx(bar + stage, box_bytes);
    // box origin: node c0 on every axis (the lower node of halo cell c0-1)
    tma_load_4d(sF0 + stage * T::SF, map, 0, z * TZ, y * TY, x * TX, bar + stage);
  };
  if (tid == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);
  int it = 0, cur_job = -1;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const int stage = it & 1;
    // prefetch the next tile's fields into the other stage (read by the
    // previous tile, which every thread finished before the last barrier)
    if (tid == 0 && tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x, stage ^ 1);
    const bool arrived = mbar_wait_bounded(bar + stage, (it >> 1) & 1);
    if (__syncthreads_or(!arrived)) {
      // the staged fields never arrived (for some thread): the whole CTA
      // reports, waits once more for its copies in flight, and gives up
      if (tid == 0) atomicOr(err0, ERRBIT_TIMEOUT);
      mbar_wait_bounded(bar + stage, (it >> 1) & 1);
      mbar_wait_bounded(bar + (stage ^ 1), ((it + 1) >> 1) & 1);
      return;
    }
    const float *sF = sF0 + stage * T::SF;
    int job, local;
    locate_tile(tile, job, local);
    if constexpr (MULTI) {
      if (job != cur_job) {
        load_params(sP, J.params + job);
        cur_job = job;
      }
      push_tile<TX, TY, TZ, RH>(*sP, local, sF, W);
      report(*sP, W);
    } else {
      push_tile<TX, TY, TZ, RH>(P1, local, sF, W);
    }
    // every warp is done with this field stage (and the staged parameters)
    // before they are refilled
    if (__syncthreads_or(W.dead)) {
      // a record chunk never arrived: report, wait (bounded) for this warp's
      // copies still in flight and for the prefetched field stage, give up
      if (tid == 0) atomicOr(err0, ERRBIT_TIMEOUT);
      for (int b = 0; b < 2; ++b)
        if (W.inflight & (1u << b)) mbar_wait_bounded(W.cbar + b, (W.phase >> b) & 1u);
      if (tile + (int)gridDim.x < ntiles)
        mbar_wait_bounded(bar + (stage ^ 1), ((it + 1) >> 1) & 1);
      return;
    }
  }
  if constexpr (MULTI) {
    for (int job = 0; job < J.njobs; ++job) {
      load_params(sP, J.params + job);
      push_overflow<TX, TY, TZ>(*sP, sF0, W);
      report(*sP, W);
      __syncthreads();   // before the next job's parameters overwrite these
    }
  } else {
    push_overflow<TX, TY, TZ>(P1, sF0, W);
    report(P1, W);
  }
}

// Deposit of one particle with FP64 global atomics (overflow entries; a rare
// path, kept rolled so that it does not raise the kernel's register count).
__device__ __noinline__ void deposit_global(const CycleParams &P, const SpeciesDev &S, int cx,
                                            int cy, int cz, float4 a, float4 b) {
  const long nodes = (long)P.nxn * P.nyn * P.nzn;
  const float u = b.x, v = b.y, w = b.z;
  const float mf[10] = {1.0f, u, v, w, u * u, u * v, u * w, v * v, v * w, w * w};
  const long sy = P.nzn, sx = (long)P.nyn * P.nzn;
  const long n0 = (long)(cx + 1) * sx + (long)(cy + 1) * sy + (cz + 1);
#pragma unroll 1
  for (int node = 0; node < 8; ++node) {
    const int i = node >> 2, j = (node >> 1) & 1, k = node & 1;
    const float wx = a.w * (i ? a.x : 1.0f - a.x);
    const float wy = j ? a.y : 1.0f - a.y, wz = k ? a.z : 1.0f - a.z;
    const double W = (double)(wx * wy * wz) * P.scale;
    const long n = n0 + i * sx + j * sy + k;
#pragma unroll
    for (int m = 0; m < 10; ++m) atomicAdd(S.mom + m * nodes + n, W * (double)mf[m]);
  }
}

// The deterministic deposit. Every one of a particle's 80 terms W_node x mf
// (W = q x the trilinear weight in FP32, mf = 1, u, v, w, uu, uv, uw, vv, vw,
// ww in FP32) is formed exactly in FP64 (a product of two floats) and rounded
// down to a multiple of its moment's quantum Q, a power of two: a fused
// multiply-add rounding toward -infinity into an accumulator that holds
// M + S with M = 1.5 x 2^52 x Q, whose unit in the last place is exactly Q
// while |S| < 2^51 Q. Every partial sum is then a multiple of Q below 2^53 Q,
// so every later FP64 addition (across lanes, cells, tiles and the global
// atomics) is exact and the moments do not depend on the order of the
// particles in their buckets or of the atomics. Q = 2^(ceil(log2 T) - 38)
// with T the species' largest possible term of that moment at load: max|q|
// for rhon, max|q| x 4 vmax for Jx..Jz, max|q| x 16 vmax^2 for pxx..pzz
// (vmax the largest velocity component, at least c/8): 2^-38 T resolution, 2^13 T headroom
// per cell and 2^15 T per node. Rounding down loses Q/2 per term on average,
// which over a node's N terms would be N Q/2, comparable to a cancelling sum
// (~sqrt(N) of its terms, each far below T): every term's Q/2 is added back
// (a cell's count x Q/2 with its exact sum, or Q/2 with an overflow entry's
// term), so the sums stay on an exact Q/2 grid, unbiased, and still depend
// only on the particles, not on their order. The moments are the sums times
// invVOL, applied once at the end.
__device__ __forceinline__ double exact_quantum(const SpeciesDev &S, int m) {
  return S.quantum[m == 0 ? 0 : (m < 4 ? 1 : 2)];
}
__device__ __forceinline__ double exact_offset(double quantum) {
  return 6755399441055744.0 * quantum;   // 1.5 * 2^52 * Q
}

// The 8 node weights (q folded in; node = a*4 + b*2 + c, a/b/c = 1 the upper
// node on x/y/z) and the 10 moment factors of one record, in FP32 with every
// operation spelled out (both exact deposit paths must form them alike).
__device__ __forceinline__ void exact_terms(float4 a, float4 b, float (&W)[8], float (&mf)[10]) {
  const float q = a.w, ox = a.x, oy = a.y, oz = a.z, u = b.x, v = b.y, w = b.z;
  const float wx[2] = {__fmul_rn(q, __fsub_rn(1.0f, ox)), __fmul_rn(q, ox)};
  const float wy[2] = {__fsub_rn(1.0f, oy), oy}, wz[2] = {__fsub_rn(1.0f, oz), oz};
#pragma unroll
  for (int n = 0; n < 8; ++n)
    W[n] = __fmul_rn(__fmul_rn(wx[n >> 2], wy[(n >> 1) & 1]), wz[n & 1]);
  mf[0] = 1.0f;
  mf[1] = u;
  mf[2] = v;
  mf[3] = w;
  mf[4] = __fmul_rn(u, u);
  mf[5] = __fmul_rn(u, v);
  mf[6] = __fmul_rn(u, w);
  mf[7] = __fmul_rn(v, v);
  mf[8] = __fmul_rn(v, w);
  mf[9] = __fmul_rn(w, w);
}

// One overflow entry of the deterministic deposit: its 80 terms rounded down
// to the species' grid, added with FP64 atomics (exact).
__device__ __noinline__ void deposit_global_exact(const CycleParams &P, const SpeciesDev &S,
                                                  int cx, int cy, int cz, float4 a, float4 b) {
  const long nodes = (long)P.nxn * P.nyn * P.nzn;
  const long sy = P.nzn, sx = (long)P.nyn * P.nzn;
  const long n0 = (long)(cx + 1) * sx + (long)(cy + 1) * sy + (cz + 1);
  float W[8], mf[10];
  exact_terms(a, b, W, mf);
#pragma unroll 1
  for (int node = 0; node < 8; ++node) {
    const long n = n0 + (node >> 2) * sx + ((node >> 1) & 1) * sy + (node & 1);
    const double Wd = (double)W[node];
#pragma unroll
    for (int m = 0; m < 10; ++m) {
      const double Q = exact_quantum(S, m), M = exact_offset(Q);
      atomicAdd(S.mom + m * nodes + n, (__fma_rd(Wd, (double)mf[m], M) - M) + 0.5 * Q);
    }
  }
}

// Threads of a deposit CTA: one per cell of the tile, in whole warps.
template <int TX, int TY, int TZ>
__host__ __device__ constexpr int dep_tpb() {
  return ((TX * TY * TZ + 31) / 32) * 32;
}

// Read-only 32-byte load of one particle record (one 256-bit access) that asks
// L2 to fetch the surrounding 256 bytes: a lane walking its cell's bucket then
// finds the next records in L2.
__device__ __forceinline__ void ld_rec(const float4 *p, float4 &a, float4 &b) {
  asm("ld.global.nc.L2::256B.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

// The same through L2 only (coherent with records written by other CTAs of
// the same launch, which the fused cycle deposits).
__device__ __forceinline__ void ld_rec_cg(const float4 *p, float4 &a, float4 &b) {
  asm("ld.global.cg.L2::256B.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
      : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
      : "l"(p));
}

template <bool COH>
__device__ __forceinline__ void ld_record(const float4 *p, float4 &a, float4 &b) {
  if constexpr (COH)
    ld_rec_cg(p, a, b);
  else
    ld_rec(p, a, b);
}

// Per-warp quota of the deposit (all 32 lanes call with their cell's count):
// lanes sum at most Q particles of their own cell, one particle per lane per
// step; the excess of the cells above Q is summed by the whole warp, 32
// particles per step plus one warp reduction per cell. Q minimises the
// estimated issue slots, 60 per lane step and 65 per warp step + 160 per
// excess cell, over the candidates Q = one of the lanes' counts; a warp whose
// largest count is at most 1.25 x its mean keeps Q = its largest count.
__device__ __forceinline__ int deposit_quota(int cnt) {
  const int mx = __reduce_max_sync(FULL, cnt);
  if (mx > (1 << 24)) return mx;   // keeps the cost sums below 2^32
  const int sum = __reduce_add_sync(FULL, cnt);
  if ((long long)mx * 32 * 4 <= (long long)sum * 5) return mx;   // max <= 1.25 x mean
  unsigned cost = 60u * (unsigned)cnt;
#pragma unroll 4
  for (int i = 0; i < 32; ++i) {
    const int c = __shfl_sync(FULL, cnt, i);
    if (c > cnt) cost += 65u * (unsigned)((c - cnt + 31) >> 5) + 160u;
  }
  const unsigned lane = threadIdx.x & 31;
  const unsigned best = __reduce_min_sync(FULL, (min(cost, (1u << 26) - 1) << 5) | lane);
  return __shfl_sync(FULL, cnt, (int)(best & 31u));
}

// All species of one tile (tile-local index `tile` of job P). Thread t owns
// cell t of the tile: it walks the cell's bucket, accumulating the 80 terms
// of every particle in packed FP32 registers (no cross-lane reduction), and
// stores the cell's totals in shared memory, term-major (sCell[j * TC + t]).
// Each node of the tile then adds up the totals of its (up to 8) cells in the
// tile and one FP64 atomic per node and moment adds the sum into the moments.
// All threads call.
// NT: the CTA's threads (at least one per cell); COH: coherent loads of the
// counters and records (the fused cycle, where other CTAs of the launch wrote
// them).
template <int TX, int TY, int TZ, int NT = dep_tpb<TX, TY, TZ>(), bool COH = false>
__device__ __forceinline__ void deposit_tile(const CycleParams &P, int tile, float *sCell) {
  using T = Tile<TX, TY, TZ>;
  constexpr int NX = TX + 1, NY = TY + 1, NZ = TZ + 1, NB = NX * NY * NZ;
  constexpr int TC = T::TC;
  static_assert(NT >= TC && NT % 32 == 0, "one thread per cell, whole warps");
  const int tid = threadIdx.x;
  const bool own = tid < TC;
  const long nodes = (long)P.nxn * P.nyn * P.nzn;
  const int tz = tile % P.ntz, ty = (tile / P.ntz) % P.nty, tx = tile / (P.ntz * P.nty);
  const int c0x = tx * TX, c0y = ty * TY, c0z = tz * TZ;
  for (int s = 0; s < P.ns; ++s) {
    const SpeciesDev &S = P.sp[s];
    const float4 *rec = S.rout;
    int cnt = 0;
    if (own) {
      const int key = tile * TC + tid;
      const long long b0 = S.base[key];
      cnt = (int)min((long long)(COH ? __ldcg(S.cout + key) : S.cout[key]), S.base[key + 1] - b0);
      rec += 2 * b0;
    }
    // quota: each lane sums at most Q particles of its own cell; the rest of
    // the few cells above Q is summed by the whole warp afterwards
    const int Q = deposit_quota(cnt);
    const int n1 = min(cnt, Q);
    const int trips = __reduce_max_sync(FULL, n1);
    float2 acc[40];
#pragma unroll
    for (int i = 0; i < 40; ++i) acc[i] = make_float2(0.f, 0.f);
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, a1 = a, b1 = a;
    if (n1 > 0) ld_record<COH>(rec, a, b);
    if (n1 > 1) ld_record<COH>(rec + 2, a1, b1);
#pragma unroll 1
    for (int k = 0; k < trips; ++k) {
      // two records in flight while this one is summed; lanes past their
      // count add zero terms
      float4 na = a1, nb = b1;
      if (k + 2 < n1) ld_record<COH>(rec + 2 * (k + 2), na, nb);
      add_terms(acc, k < n1 ? a.w : 0.0f, a.x, a.y, a.z, b.x, b.y, b.z, 0);
      a = a1;
      b = b1;
      a1 = na;
      b1 = nb;
    }
    if (own) {
#pragma unroll
      for (int i = 0; i < 40; ++i) {
        const int node = i / 5, k = i % 5;
        sCell[(node * 10 + k) * TC + tid] = acc[i].x;
        sCell[(node * 10 + k + 5) * TC + tid] = acc[i].y;
      }
    }
    // the cells above the quota: particles Q.. of each, one per lane, summed
    // by the warp (warp_sum80) and added to the cell's totals
    unsigned heavy = __ballot_sync(FULL, cnt > Q);
    if (heavy) {
      __syncwarp();
      const int lane = tid & 31, wbase = tid & ~31;
      const int corner = (lane >> 2) & 7, mbase = 5 * ((lane >> 1) & 1);
      const int lo = (lane & 1) ? 3 : 0, hi = (lane & 1) ? 5 : 3;
      while (heavy) {
        const int hl = __ffs(heavy) - 1;
        heavy &= heavy - 1;
        const int hc = __shfl_sync(FULL, cnt, hl);
        const float4 *hrec = reinterpret_cast<const float4 *>(
            __shfl_sync(FULL, reinterpret_cast<unsigned long long>(rec), hl));
#pragma unroll
        for (int i = 0; i < 40; ++i) acc[i] = make_float2(0.f, 0.f);
#pragma unroll 1
        for (int o = Q; o < hc; o += 32) {
          const int i = o + lane;
          float4 ha = make_float4(0.f, 0.f, 0.f, 0.f), hb = ha;
          if (i < hc) ld_record<COH>(hrec + 2 * i, ha, hb);
          add_terms(acc, i < hc ? ha.w : 0.0f, ha.x, ha.y, ha.z, hb.x, hb.y, hb.z, lane);
        }
        float r[5];
        warp_sum80(acc, r, lane);
        float *dst = sCell + (corner * 10 + mbase) * TC + wbase + hl;
#pragma unroll
        for (int k = 0; k < 5; ++k)
          if (k >= lo && k < hi) dst[k * TC] += r[k];
      }
    }
    __syncthreads();
    for (int idx = tid; idx < 10 * NB; idx += NT) {
      const int m = idx / NB, nb = idx % NB;
      const int bz = nb % NZ, by = (nb / NZ) % NY, bx = nb / (NZ * NY);
      float sum = 0.0f;
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const int lx = bx - a, ly = by - b, lz = bz - c;
            if (lx >= 0 && lx < TX && ly >= 0 && ly < TY && lz >= 0 && lz < TZ)
              sum += sCell[((a * 4 + b * 2 + c) * 10 + m) * TC + (lx * TY + ly) * TZ + lz];
          }
      if (sum != 0.0f) {
        const long g = ((long)(c0x + bx + 1) * P.nyn + (c0y + by + 1)) * P.nzn + (c0z + bz + 1);
        atomicAdd(S.mom + m * nodes + g, (double)sum * P.scale);
      }
    }
    __syncthreads();
  }
}

// The deterministic deposit of one tile (see exact_terms): thread t walks
// cell t's whole bucket (no quota: a clumped cell keeps its thread longer),
// rounding every term down to the species' grid into 80 FP64 accumulators;
// the cells' exact sums go to shared memory and each node of the tile adds
// its (up to 8) cells' sums and issues one FP64 atomic per moment, all exact.
// The moments stay unscaled until k_scale_moments. All threads call.
template <int TX, int TY, int TZ>
__device__ __forceinline__ void deposit_tile_exact(const CycleParams &P, int tile, double *sCell,
                                                   int &inexact) {
  using T = Tile<TX, TY, TZ>;
  constexpr int NX = TX + 1, NY = TY + 1, NZ = TZ + 1, NB = NX * NY * NZ;
  constexpr int TC = T::TC, NT = dep_tpb<TX, TY, TZ>();
  const int tid = threadIdx.x;
  const bool own = tid < TC;
  const long nodes = (long)P.nxn * P.nyn * P.nzn;
  const int tz = tile % P.ntz, ty = (tile / P.ntz) % P.nty, tx = tile / (P.ntz * P.nty);
  const int c0x = tx * TX, c0y = ty * TY, c0z = tz * TZ;
  for (int s = 0; s < P.ns; ++s) {
    const SpeciesDev &S = P.sp[s];
    const double M[3] = {exact_offset(S.quantum[0]), exact_offset(S.quantum[1]),
                         exact_offset(S.quantum[2])};
    const float4 *rec = S.rout;
    int cnt = 0;
    if (own) {
      const int key = tile * TC + tid;
      const long long b0 = S.base[key];
      cnt = (int)min((long long)S.cout[key], S.base[key + 1] - b0);
      rec += 2 * b0;
    }
    double acc[80];
#pragma unroll
    for (int i = 0; i < 80; ++i) acc[i] = M[(i % 10) == 0 ? 0 : ((i % 10) < 4 ? 1 : 2)];
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, a1 = a, b1 = a;
    if (cnt > 0) ld_rec(rec, a, b);
    if (cnt > 1) ld_rec(rec + 2, a1, b1);
#pragma unroll 1
    for (int k = 0; k < cnt; ++k) {
      float4 na = a1, nb = b1;
      if (k + 2 < cnt) ld_rec(rec + 2 * (k + 2), na, nb);
      float W[8], mf[10];
      exact_terms(a, b, W, mf);
#pragma unroll
      for (int node = 0; node < 8; ++node) {
        const double Wd = (double)W[node];
#pragma unroll
        for (int m = 0; m < 10; ++m) acc[node * 10 + m] = __fma_rd(Wd, (double)mf[m], acc[node * 10 + m]);
      }
      a = a1;
      b = b1;
      a1 = na;
      b1 = nb;
    }
    if (own) {
#pragma unroll
      for (int i = 0; i < 80; ++i) {
        const int k = (i % 10) == 0 ? 0 : ((i % 10) < 4 ? 1 : 2);
        const double lo = 4503599627370496.0 * S.quantum[k];   // 2^52 Q; 2^53 Q above
        inexact |= (acc[i] < lo) | (acc[i] >= 2.0 * lo);
        sCell[i * TC + tid] = (acc[i] - M[k]) + (double)cnt * 0.5 * S.quantum[k];
      }
    }
    __syncthreads();
    for (int idx = tid; idx < 10 * NB; idx += NT) {
      const int m = idx / NB, nb = idx % NB;
      const int bz = nb % NZ, by = (nb / NZ) % NY, bx = nb / (NZ * NY);
      double sum = 0.0;
#pragma unroll
      for (int a2 = 0; a2 < 2; ++a2)
#pragma unroll
        for (int b2 = 0; b2 < 2; ++b2)
#pragma unroll
          for (int c2 = 0; c2 < 2; ++c2) {
            const int lx = bx - a2, ly = by - b2, lz = bz - c2;
            if (lx >= 0 && lx < TX && ly >= 0 && ly < TY && lz >= 0 && lz < TZ)
              sum += sCell[((a2 * 4 + b2 * 2 + c2) * 10 + m) * TC + (lx * TY + ly) * TZ + lz];
          }
      if (sum != 0.0) {
        const long g = ((long)(c0x + bx + 1) * P.nyn + (c0y + by + 1)) * P.nzn + (c0z + bz + 1);
        atomicAdd(S.mom + m * nodes + g, sum);
      }
    }
    __syncthreads();
  }
}

// Overflow entries of every species of job P. Each warp takes 32 consecutive
// entries; the push appends the particles of one slot that overflow the same
// full bucket next to each other, so most entries of a warp share their cell.
// Up to four groups of at least two entries with one cell are summed by the
// warp in FP32 (warp_sum80) and added with one FP64 atomic per node and
// moment; the remaining entries deposit one by one (deposit_global). Called
// by whole warps.
template <int TX, int TY, int TZ, bool EXACT, bool COH = false>
__device__ __forceinline__ void deposit_overflow(const CycleParams &P) {
  const int lane = threadIdx.x & 31;
  const long nwarps = (long)gridDim.x * (blockDim.x >> 5);
  const long gwarp = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const long nodes = (long)P.nxn * P.nyn * P.nzn;
  const long sy = P.nzn, sx = (long)P.nyn * P.nzn;
  // this lane's totals after warp_sum80: node corner (bit4, bit3, bit2),
  // moments mbase + [lo, hi)
  const int ca = (lane >> 4) & 1, cb = (lane >> 3) & 1, cc = (lane >> 2) & 1;
  const int mbase = 5 * ((lane >> 1) & 1);
  const int lo = (lane & 1) ? 3 : 0, hi = (lane & 1) ? 5 : 3;
  for (int s = 0; s < P.ns; ++s) {
    const SpeciesDev &S = P.sp[s];
    const long on = min(COH ? __ldcg(S.ocout) : *S.ocout, S.ocap);
    for (long base = gwarp * 32; base < on; base += nwarps * 32) {
      const long i = base + lane;
      bool valid = i < on;
      int key = -1;
      float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a;
      if (valid) {
        key = COH ? __ldcg(S.okout + i) : S.okout[i];
        a = COH ? __ldcg(S.oout + 2 * i) : S.oout[2 * i];
        b = COH ? __ldcg(S.oout + 2 * i + 1) : S.oout[2 * i + 1];
      }
      if constexpr (EXACT) {   // every entry on its own, exactly
        if (valid) {
          int cx, cy, cz;
          key_cell<TX, TY, TZ>(key, P.nty, P.ntz, cx, cy, cz);
          deposit_global_exact(P, S, cx, cy, cz, a, b);
        }
        continue;
      }
      unsigned remaining = __ballot_sync(FULL, valid);
      int groups = 0;
#pragma unroll 1
      while (remaining && groups < 4) {
        const int leader = __ffs(remaining) - 1;
        const int k = __shfl_sync(FULL, key, leader);
        const bool member = valid && key == k;
        const unsigned members = __ballot_sync(FULL, member);
        remaining &= ~members;
        if (__popc(members) < 2) continue;   // a lone entry: deposited below
        ++groups;
        float2 acc[40];
#pragma unroll
        for (int j = 0; j < 40; ++j) acc[j] = make_float2(0.f, 0.f);
        add_terms(acc, member ? a.w : 0.0f, a.x, a.y, a.z, b.x, b.y, b.z, lane);
        float r[5];
        warp_sum80(acc, r, lane);
        int cx, cy, cz;
        key_cell<TX, TY, TZ>(k, P.nty, P.ntz, cx, cy, cz);
        const long n = (long)(cx + 1 + ca) * sx + (long)(cy + 1 + cb) * sy + (cz + 1 + cc);
#pragma unroll
        for (int m = 0; m < 5; ++m)
          if (m >= lo && m < hi)
            atomicAdd(S.mom + (mbase + m) * nodes + n, (double)r[m] * P.scale);
        if (member) valid = false;
      }
      if (valid) {
        int cx, cy, cz;
        key_cell<TX, TY, TZ>(key, P.nty, P.ntz, cx, cy, cz);
        deposit_global(P, S, cx, cy, cz, a, b);
      }
    }
  }
}

// The deposit (interpP2G, src/Mover.cpp:385-572) for every species, from the
// buckets the push wrote: persistent CTAs walk the tiles, one thread per cell
// (deposit_tile); then the overflow entries (deposit_overflow).
// MULTI as for k_push.
template <int TX, int TY, int TZ, bool MULTI, bool EXACT>
__global__ void __launch_bounds__(dep_tpb<TX, TY, TZ>(),
                                  EXACT ? (256 / dep_tpb<TX, TY, TZ>() > 0
                                               ? 256 / dep_tpb<TX, TY, TZ>() : 1)
                                        : 512 / dep_tpb<TX, TY, TZ>())
    k_deposit(const __grid_constant__ CycleParams P1, const __grid_constant__ JobTable J) {
  using T = Tile<TX, TY, TZ>;
  static_assert(!(MULTI && EXACT), "the deterministic deposit runs one simulation");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *sCell = reinterpret_cast<float *>(smem_raw);   // 80 x TC (float, or double if EXACT)
  CycleParams *sP =
      reinterpret_cast<CycleParams *>(smem_raw + (size_t)T::TC * 80 * (EXACT ? 8 : 4));   // MULTI
  const int ntiles = MULTI ? J.total_tiles : P1.ntx * P1.nty * P1.ntz;
  int cur_job = -1;
  if constexpr (EXACT) {
    int inexact = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x)
      deposit_tile_exact<TX, TY, TZ>(P1, tile, reinterpret_cast<double *>(smem_raw), inexact);
    if (inexact) atomicOr(P1.err, ERRBIT_INEXACT);
    deposit_overflow<TX, TY, TZ, true>(P1);
  } else {
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
      if constexpr (MULTI) {
        const int job = job_of(J, tile);
        if (job != cur_job) {
          __syncthreads();   // every thread is done with the staged parameters
          load_params(sP, J.params + job);
          cur_job = job;
        }
        deposit_tile<TX, TY, TZ>(*sP, tile - J.tile_base[job], sCell);
      } else {
        deposit_tile<TX, TY, TZ>(P1, tile, sCell);
      }
    }
    if constexpr (MULTI) {
      for (int job = 0; job < J.njobs; ++job) {
        __syncthreads();   // every thread is done with the staged parameters
        load_params(sP, J.params + job);
        deposit_overflow<TX, TY, TZ, false>(*sP);
      }
    } else {
      deposit_overflow<TX, TY, TZ, false>(P1);
    }
  }
}

// ---------------------------------------------------------------------------
// the fused cycle: push and deposit in one persistent cooperative launch
// ---------------------------------------------------------------------------

// Per-cycle device state of the fused cycle (zeroed before every cycle).
struct FusedAux {
  int *done;        // [ntiles] 1 once a tile's particles are pushed
  unsigned *bar;    // [2] arrivals at the two grid barriers
  int lag;          // waves between a tile's push and its deposit
};

constexpr long long GRID_WAIT_CYCLES = 4000000000LL;   // ~2 s: bounded waits

__device__ __forceinline__ int ld_acquire(const int *p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned ld_acquire_u(const unsigned *p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier of a cooperative launch (all CTAs resident): thread 0 of
// each CTA arrives and waits, bounded; false for every thread if it gave up.
__device__ __forceinline__ bool grid_barrier(unsigned *count) {
  __threadfence();
  __syncthreads();
  int ok = 1;
  if (threadIdx.x == 0) {
    atomicAdd(count, 1u);
    const long long t0 = clock64();
    while (ld_acquire_u(count) < gridDim.x) {
      if (clock64() - t0 > GRID_WAIT_CYCLES) {
        ok = 0;
        break;
      }
      __nanosleep(128);
    }
  }
  ok = __syncthreads_and(ok);
  __threadfence();
  return ok != 0;
}

// Launch order of the tiles: on a periodic axis of n > 2 tiles the order
// folds (0, n-1, 1, n-2, ...) so that a tile's wrap-around neighbour comes
// next to it; every neighbour is then at most 2 positions away per axis.
__host__ __device__ __forceinline__ int unfold_pos(int f, int n, int periodic) {
  if (!periodic || n <= 2) return f;
  return (f & 1) ? n - 1 - (f >> 1) : (f >> 1);
}
__device__ __forceinline__ int tile_of_order(const CycleParams &P, int o) {
  const int fz = o % P.ntz, fy = (o / P.ntz) % P.nty, fx = o / (P.ntz * P.nty);
  return (unfold_pos(fx, P.ntx, P.periodic[0]) * P.nty + unfold_pos(fy, P.nty, P.periodic[1])) *
             P.ntz +
         unfold_pos(fz, P.ntz, P.periodic[2]);
}

// Shared memory of the fused cycle: the push's field stages, then its record
// staging and ring or the deposit's per-cell sums (whichever is larger; the
// two are used at different times), then the barriers.
template <int TX, int TY, int TZ, int MINB>
__host__ __device__ constexpr size_t fused_rec_bytes() {
  return (size_t)(SIM_NW * 64 + SIM_NW * 2 * ring_half<MINB>() * 2) * 16 >
                 (size_t)Tile<TX, TY, TZ>::TC * 80 * 4
             ? (size_t)(SIM_NW * 64 + SIM_NW * 2 * ring_half<MINB>() * 2) * 16
             : (size_t)Tile<TX, TY, TZ>::TC * 80 * 4;
}
template <int TX, int TY, int TZ, int MINB>
__host__ __device__ constexpr size_t fused_smem() {
  return 2 * (size_t)Tile<TX, TY, TZ>::SF * 4 + fused_rec_bytes<TX, TY, TZ, MINB>() +
         (2 + 2 * SIM_NW) * sizeof(uint64_t);
}

// Thread 0 waits (bounded) until every neighbour of `tile` (itself included,
// wrapping on periodic axes) is pushed; false for every thread if it gave up.
__device__ __forceinline__ bool wait_neighbours(const CycleParams &P, const int *done, int tile) {
  int ok = 1;
  if (threadIdx.x == 0) {
    const int tz = tile % P.ntz, ty = (tile / P.ntz) % P.nty, tx = tile / (P.ntz * P.nty);
    const long long t0 = clock64();
    for (int dx = -1; dx <= 1 && ok; ++dx)
      for (int dy = -1; dy <= 1 && ok; ++dy)
        for (int dz = -1; dz <= 1 && ok; ++dz) {
          int n[3] = {tx + dx, ty + dy, tz + dz};
          const int N[3] = {P.ntx, P.nty, P.ntz};
          bool skip = false;
          for (int a = 0; a < 3; ++a) {
            if (n[a] >= 0 && n[a] < N[a]) continue;
            if (!P.periodic[a]) skip = true;
            n[a] = (n[a] + N[a]) % N[a];
          }
          if (skip) continue;
          const int *f = done + (n[0] * P.nty + n[1]) * P.ntz + n[2];
          while (ld_acquire(f) == 0) {
            if (clock64() - t0 > GRID_WAIT_CYCLES) {
              ok = 0;
              break;
            }
            __nanosleep(64);
          }
        }
  }
  ok = __syncthreads_and(ok);
  __threadfence();
  return ok != 0;
}

// The fused cycle (the batching form's one launch per cycle), all species.
// Persistent CTAs, all resident (cooperative launch), take the tiles in the
// launch order above: at step k a CTA pushes its k-th tile (as k_push does:
// TMA-staged fields, record ring, particles written into their new cells'
// buckets) and publishes it, then deposits its tile from lag steps earlier
// (as k_deposit does, with coherent loads) once the 27 tiles around it are
// published, whose pushes are the only ones that write into its buckets. The
// push keeps the SM's shared-memory pipe busy and the deposit its arithmetic
// and load units, so the two phases overlap across the CTAs of an SM. A
// pushed particle that left its tile's neighbourhood goes to the overflow
// list. Then, after a grid barrier, the entries of the previous overflow list
// are pushed into the new overflow list, and after a second barrier every
// entry of the new list is deposited. lag = ceil(R / G) with R the largest
// launch-order distance between neighbouring tiles and G the CTAs, so that a
// CTA only ever waits for pushes of steps up to its own: no cycle of waits.
// Every wait is bounded (an error bit, then the CTA stops).
template <int TX, int TY, int TZ, int MINB>
__global__ void __launch_bounds__(SIM_TPB, MINB)
    k_cycle(const __grid_constant__ CUtensorMap fmap, const __grid_constant__ CycleParams P,
            const __grid_constant__ FusedAux X) {
  using T = Tile<TX, TY, TZ>;
  constexpr int RH = ring_half<MINB>();
  static_assert(T::TC % SIM_NW == 0 && T::TC / SIM_NW <= 32,
                "cells per warp must fit a warp's lanes");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *sF0 = reinterpret_cast<float *>(smem_raw);                 // 2 stages x SF
  float4 *sRec = reinterpret_cast<float4 *>(sF0 + 2 * T::SF);       // NW x 64 staged records
  float4 *sBuf = sRec + SIM_NW * 64;                                // NW x 2 x RH records
  uint64_t *bar = reinterpret_cast<uint64_t *>(reinterpret_cast<unsigned char *>(sRec) +
                                               fused_rec_bytes<TX, TY, TZ, MINB>());   // 2 + 2 NW
  // the deposit's per-cell sums reuse the record staging and ring (idle
  // between two tiles' pushes; the field stages stay untouched)
  float *sCell = reinterpret_cast<float *>(sRec);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  PushWarp W;
  W.wrec = sRec + warp * 64;
  W.ring = sBuf + warp * 2 * RH * 2;
  W.cbar = bar + 2 + warp * 2;
  if (smem_addr(sF0) & 127u) {
    if (tid == 0) atomicOr(P.err, ERRBIT_SMEM_ALIGN);
    return;
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
  }
  if (lane == 0) {
    mbar_init(W.cbar, 1);
    mbar_init(W.cbar + 1, 1);
  }
  __syncthreads();

  const int ntiles = P.ntx * P.nty * P.ntz;
  const int G = gridDim.x;
  const unsigned box_bytes = (unsigned)(T::BN * 8 * sizeof(float));
  auto issue = [&](int tile, int stage) {   // thread 0
    const int z = tile % P.ntz, y = (tile / P.ntz) % P.nty, x = tile / (P.ntz * P.nty);
    fence_proxy_async();
    mbar_expect_tx(bar + stage, box_bytes);
    tma_load_4d(sF0 + stage * T::SF, &fmap, 0, z * TZ, y * TY, x * TX, bar + stage);
  };
  const int first = blockIdx.x;
  if (tid == 0 && first < ntiles) issue(tile_of_order(P, first), 0);
  int it = 0;   // tiles pushed by this CTA
  for (int k = 0;; ++k) {
    const int o = first + k * G;                // order index pushed at this step
    const int od = first + (k - X.lag) * G;     // order index deposited at this step
    if (o >= ntiles && od >= ntiles) break;
    if (o < ntiles) {
      const int stage = it & 1;
      if (tid == 0 && o + G < ntiles) issue(tile_of_order(P, o + G), stage ^ 1);
      const bool arrived = mbar_wait_bounded(bar + stage, (it >> 1) & 1);
      if (__syncthreads_or(!arrived)) {
        if (tid == 0) atomicOr(P.err, ERRBIT_TIMEOUT);
        mbar_wait_bounded(bar + stage, (it >> 1) & 1);
        mbar_wait_bounded(bar + (stage ^ 1), ((it + 1) >> 1) & 1);
        return;
      }
      const int tile = tile_of_order(P, o);
      push_tile<TX, TY, TZ, RH, true>(P, tile, sF0 + stage * T::SF, W);
      if (__syncthreads_or(W.dead)) {
        if (tid == 0) atomicOr(P.err, ERRBIT_TIMEOUT);
        for (int b = 0; b < 2; ++b)
          if (W.inflight & (1u << b)) mbar_wait_bounded(W.cbar + b, (W.phase >> b) & 1u);
        if (o + G < ntiles) mbar_wait_bounded(bar + (stage ^ 1), ((it + 1) >> 1) & 1);
        return;
      }
      // publish: every thread's stores, then the flag
      __threadfence();
      __syncthreads();
      if (tid == 0) st_release(X.done + tile, 1);
      ++it;
    }
    if (od >= 0 && od < ntiles) {
      const int tile = tile_of_order(P, od);
      if (!wait_neighbours(P, X.done, tile)) {
        if (tid == 0) atomicOr(P.err, ERRBIT_TIMEOUT);
        if (o + G < ntiles) mbar_wait_bounded(bar + (it & 1), (it >> 1) & 1);
        return;
      }
      deposit_tile<TX, TY, TZ, SIM_TPB, true>(P, tile, sCell);
      // the next tile's bulk copies overwrite the sums written here
      fence_proxy_async();
      __syncthreads();
    }
  }
  report(P, W);
  if (!grid_barrier(X.bar)) {
    if (tid == 0) atomicOr(P.err, ERRBIT_TIMEOUT);
    return;
  }
  push_overflow<TX, TY, TZ, true>(P, sF0, W);
  report(P, W);
  if (!grid_barrier(X.bar + 1)) {
    if (tid == 0) atomicOr(P.err, ERRBIT_TIMEOUT);
    return;
  }
  deposit_overflow<TX, TY, TZ, false, true>(P);
}

// The deterministic deposit's moments are unscaled sums: times invVOL, once.
__global__ void k_scale_moments(const __grid_constant__ CycleParams P) {
  const long n = 10L * P.nxn * P.nyn * P.nzn;
  for (int s = 0; s < P.ns; ++s)
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
      P.sp[s].mom[i] *= P.scale;
}

// Largest |q| and largest velocity component of a species being loaded, as
// the bit patterns of non-negative floats (ordered like the values).
__global__ void k_species_bounds(const float *__restrict__ q, const float *__restrict__ u,
                                 const float *__restrict__ v, const float *__restrict__ w, long n,
                                 unsigned *out) {
  float mq = 0.0f, mv = 0.0f;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    mq = fmaxf(mq, fabsf(q[i]));
    mv = fmaxf(mv, fmaxf(fabsf(u[i]), fmaxf(fabsf(v[i]), fabsf(w[i]))));
  }
  const unsigned bq = __reduce_max_sync(0xffffffffu, __float_as_uint(mq));
  const unsigned bv = __reduce_max_sync(0xffffffffu, __float_as_uint(mv));
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, bq);
    atomicMax(out + 1, bv);
  }
}

// Zeroes every job's write-side fill counters and overflow counter and its
// moments before a multi-job cycle (one launch instead of three memsets per
// job and species).
__global__ void k_zero_jobs(const __grid_constant__ JobTable J) {
  const long stride = (long)gridDim.x * blockDim.x;
  const long t0 = blockIdx.x * (long)blockDim.x + threadIdx.x;
  for (int j = 0; j < J.njobs; ++j) {
    const CycleParams &P = J.params[j];
    const long ncells = (long)P.nxc * P.nyc * P.nzc, nodes = (long)P.nxn * P.nyn * P.nzn;
    for (int s = 0; s < P.ns; ++s) {
      const SpeciesDev &S = P.sp[s];
      for (long i = t0; i < ncells; i += stride) S.cout[i] = 0;
      if (t0 == 0) *S.ocout = 0;
      for (long i = t0; i < 10 * nodes; i += stride) S.mom[i] = 0.0;
    }
  }
}

// ---------------------------------------------------------------------------
// layout (load, re-layout), readback, field packing, boundary fold
// ---------------------------------------------------------------------------
struct GridScalars {
  int nxc, nyc, nzc;
  double invdx, invdy, invdz, dx, dy, dz;
};

// Position (float, domain units) -> cell + offset; exact double arithmetic.
__device__ __forceinline__ void to_cell(float x, double inv, int N, int &c, float &o, int &bad) {
  const double X = (double)x * inv;
  double f = floor(X);
  if (!(X >= 0.0) || X > (double)N) {
    bad = 1;
    f = X > (double)N ? (double)(N - 1) : 0.0;
    c = (int)f;
    o = X > (double)N ? 1.0f : 0.0f;
    return;
  }
  c = (int)f;
  o = (float)(X - f);
  if (o >= 1.0f) {
    c += 1;
    o = 0.0f;
  }
  if (c == N) {
    c = N - 1;
    o = 1.0f;
  }
}

// Particles per cell of reference-layout positions.
template <int TX, int TY, int TZ>
__global__ void k_count_keys(GridScalars g, int nty, int ntz, const float *__restrict__ x,
                             const float *__restrict__ y, const float *__restrict__ z, long n,
                             int *__restrict__ count, int *err) {
  const int lane = threadIdx.x & 31;
  int bad = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    int cx, cy, cz;
    float o;
    to_cell(x[i], g.invdx, g.nxc, cx, o, bad);
    to_cell(y[i], g.invdy, g.nyc, cy, o, bad);
    to_cell(z[i], g.invdz, g.nzc, cz, o, bad);
    const int key = tile_key<TX, TY, TZ>(cx, cy, cz, nty, ntz);
    const unsigned peers = __match_any_sync(__activemask(), key);
    if (lane == __ffs(peers) - 1) atomicAdd(count + key, __popc(peers));
  }
  if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
}

// Particles per cell of the buckets (clamped counters) ...
__global__ void k_count_buckets(const long long *__restrict__ base, const int *__restrict__ cnt,
                                long ncells, int *__restrict__ count) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < ncells;
       k += (long)gridDim.x * blockDim.x)
    count[k] = (int)min((long long)cnt[k], base[k + 1] - base[k]);
}

// ... plus the overflow list (a separate launch: it adds to those counts).
__global__ void k_count_overflow(const int *__restrict__ okey, const int *__restrict__ ocnt,
                                 int ocap, int *__restrict__ count) {
  const int on = min(*ocnt, ocap);
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < on;
       j += (long)gridDim.x * blockDim.x)
    atomicAdd(count + okey[j], 1);
}

// Bucket capacity of each cell from its particle count: fixed (`fixed` > 0)
// or the count plus max(16, count/2) slots, rounded up to a multiple of 4
// (128-byte aligned buckets).
__global__ void k_capacity(const int *__restrict__ count, long ncells, int fixed,
                           long long *__restrict__ cap) {
  for (long k = blockIdx.x * (long)blockDim.x + threadIdx.x; k < ncells;
       k += (long)gridDim.x * blockDim.x) {
    const long long c = count[k];
    cap[k] = fixed > 0 ? fixed : ((c + max(16LL, c / 2) + 3) / 4) * 4;
  }
}

// Reference-layout particles into the buckets S.rout (counters S.cout and the
// overflow list zeroed beforehand).
template <int TX, int TY, int TZ>
__global__ void k_fill(GridScalars g, int nty, int ntz, const float *__restrict__ x,
                       const float *__restrict__ y, const float *__restrict__ z,
                       const float *__restrict__ u, const float *__restrict__ v,
                       const float *__restrict__ w, const float *__restrict__ q, long n,
                       SpeciesDev S, int *err) {
  int bad = 0, lost = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    int cx, cy, cz;
    float ox, oy, oz;
    to_cell(x[i], g.invdx, g.nxc, cx, ox, bad);
    to_cell(y[i], g.invdy, g.nyc, cy, oy, bad);
    to_cell(z[i], g.invdz, g.nzc, cz, oz, bad);
    const int key = tile_key<TX, TY, TZ>(cx, cy, cz, nty, ntz);
    const int slot = atomicAdd(S.cout + key, 1);
    lost |= put_at(S, key, S.base[key], S.base[key + 1], slot, make_float4(ox, oy, oz, q[i]),
                   make_float4(u[i], v[i], w[i], 0.f));
  }
  if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
  if (lost) atomicOr(err, ERRBIT_LOST);
}

// Re-layout: buckets (old layout, buffer set `in`) and overflow list into
// the buckets of the new layout S.base / S.rout (counters zeroed beforehand).
// One warp per cell copies its bucket; then the overflow entries are placed.
// Every cell's new capacity covers its particles, so nothing overflows unless
// the capacities were fixed by the caller.
__global__ void k_relayout(const long long *__restrict__ obase, const float4 *__restrict__ rin,
                           const int *__restrict__ cin, long ncells,
                           const float4 *__restrict__ oin, const int *__restrict__ okin,
                           const int *__restrict__ ocin, int ocap_in, SpeciesDev S, int *err) {
  const int lane = threadIdx.x & 31;
  const long warps = (long)gridDim.x * (blockDim.x >> 5);
  int lost = 0;
  for (long key = blockIdx.x * (long)(blockDim.x >> 5) + (threadIdx.x >> 5); key < ncells;
       key += warps) {
    const long long ob = obase[key];
    const int c = (int)min((long long)cin[key], obase[key + 1] - ob);
    if (c <= 0) continue;
    int first = 0;
    if (lane == 0) first = atomicAdd(S.cout + key, c);
    first = __shfl_sync(FULL, first, 0);
    const long long nb = S.base[key], ne = S.base[key + 1];
    for (int j = lane; j < c; j += 32)
      lost |= put_at(S, (int)key, nb, ne, first + j, rin[2 * (ob + j)], rin[2 * (ob + j) + 1]);
  }
  const int on = min(*ocin, ocap_in);
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < on;
       j += (long)gridDim.x * blockDim.x) {
    const int key = okin[j];
    const int slot = atomicAdd(S.cout + key, 1);
    lost |= put_at(S, key, S.base[key], S.base[key + 1], slot, oin[2 * j], oin[2 * j + 1]);
  }
  if (lost) atomicOr(err, ERRBIT_LOST);
}

__global__ void k_clamp_counts(const long long *__restrict__ base, const int *__restrict__ cnt,
                               long k, long long *__restrict__ out) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < k;
       i += (long)gridDim.x * blockDim.x)
    out[i] = min((long long)cnt[i], base[i + 1] - base[i]);
}

struct Unload {
  float *x, *y, *z, *u, *v, *w, *q;   // q may be null
  long n;                             // output length
};

__device__ __forceinline__ void unload_one(const GridScalars &g, const Unload &o, long at, int cx,
                                           int cy, int cz, float4 a, float4 b) {
  if (at >= o.n) return;   // only if the counters were corrupted
  o.x[at] = (float)(((double)cx + (double)a.x) * g.dx);
  o.y[at] = (float)(((double)cy + (double)a.y) * g.dy);
  o.z[at] = (float)(((double)cz + (double)a.z) * g.dz);
  o.u[at] = b.x;
  o.v[at] = b.y;
  o.w[at] = b.z;
  if (o.q) o.q[at] = a.w;
}

// Buckets (cell order, tile-major) then overflow entries into flat
// reference-layout arrays; offset[] is the exclusive scan of the clamped
// counts, offset[ncells] their total.
template <int TX, int TY, int TZ>
__global__ void k_unload(GridScalars g, int nty, int ntz, long ncells, const float4 *__restrict__ rec,
                         const long long *__restrict__ base, const int *__restrict__ cnt,
                         const long long *__restrict__ offset, const float4 *__restrict__ orec,
                         const int *__restrict__ okey, const int *__restrict__ ocnt, int ocap,
                         Unload o) {
  const int lane = threadIdx.x & 31;
  const long warps = (long)gridDim.x * (blockDim.x >> 5);
  for (long key = blockIdx.x * (long)(blockDim.x >> 5) + (threadIdx.x >> 5); key < ncells;
       key += warps) {
    const long long b0 = base[key];
    const int c = (int)min((long long)cnt[key], base[key + 1] - b0);
    if (c <= 0) continue;
    int cx, cy, cz;
    key_cell<TX, TY, TZ>((int)key, nty, ntz, cx, cy, cz);
    const long off = offset[key];
    for (int j = lane; j < c; j += 32)
      unload_one(g, o, off + j, cx, cy, cz, rec[2 * (b0 + j)], rec[2 * (b0 + j) + 1]);
  }
  const int on = min(*ocnt, ocap);
  const long ob = offset[ncells];
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < on;
       j += (long)gridDim.x * blockDim.x) {
    int cx, cy, cz;
    key_cell<TX, TY, TZ>(okey[j], nty, ntz, cx, cy, cz);
    unload_one(g, o, ob + j, cx, cy, cz, orec[2 * j], orec[2 * j + 1]);
  }
}

// Exclusive scan of k 64-bit entries into out[0..k]; three passes.
constexpr int SCAN_B = 1024;
__device__ __forceinline__ long long block_exclusive_scan(long long v, long long *warp_sums,
                                                          long long &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  long long x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    long long s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(FULL, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  const long long pre = warp ? warp_sums[warp - 1] : 0;
  total = warp_sums[nw - 1];
  __syncthreads();
  return pre + x - v;
}

__global__ void __launch_bounds__(SCAN_B) k_scan_blocks(const long long *in, long k,
                                                        long long *out, long long *block_sums) {
  __shared__ long long ws[32];
  const long i = blockIdx.x * (long)SCAN_B + threadIdx.x;
  const long long v = i < k ? in[i] : 0;
  long long total;
  const long long ex = block_exclusive_scan(v, ws, total);
  if (i < k) out[i] = ex;
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_B) k_scan_sums(long long *block_sums, int nb,
                                                      long long *grand) {
  __shared__ long long ws[32];
  long long carry = 0;
  for (int base = 0; base < nb; base += SCAN_B) {
    const int i = base + threadIdx.x;
    const long long v = i < nb ? block_sums[i] : 0;
    long long total;
    const long long ex = block_exclusive_scan(v, ws, total);
    if (i < nb) block_sums[i] = ex + carry;
    carry += total;
  }
  if (threadIdx.x == 0) *grand = carry;
}

__global__ void __launch_bounds__(SCAN_B) k_scan_add(long long *out, long k,
                                                     const long long *block_sums) {
  const long i = blockIdx.x * (long)SCAN_B + threadIdx.x;
  if (i < k) out[i] += block_sums[blockIdx.x];
}

__global__ void k_pack_fields8(const float *__restrict__ ex, const float *__restrict__ ey,
                               const float *__restrict__ ez, const float *__restrict__ bx,
                               const float *__restrict__ by, const float *__restrict__ bz,
                               float *__restrict__ f8, long nodes) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < nodes;
       i += (long)gridDim.x * blockDim.x) {
    reinterpret_cast<float4 *>(f8)[2 * i] = make_float4(ex[i], ey[i], ez[i], bx[i]);
    reinterpret_cast<float4 *>(f8)[2 * i + 1] = make_float4(by[i], bz[i], 0.f, 0.f);
  }
}

// applyBCids (src/BC.cpp:362-615) on FP64 moments: periodic folds X, Y, Z,
// then the doubling of non-periodic axes; one launch per step.
__global__ void k_bc_fold64(double *mom, int nxn, int nyn, int nzn, int axis, int periodic) {
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
  const long nodes = (long)nxn * nyn * nzn;
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
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
  for (int m = 0; m < 10; ++m) {
    double *a = mom + m * nodes;
    if (periodic) {
      const double sum = a[lo] + a[hi];
      a[lo] = sum;
      a[hi] = sum;
    } else {
      a[lo] *= 2.0;
      a[hi] *= 2.0;
    }
  }
}

int blocks_for(long n, int tpb) {
  return (int)std::max<long>(1, std::min<long>(ceil_div(n, tpb), 148L * 32));
}

}  // namespace
}  // namespace spb

using namespace spb;

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

// Device memory of the precision form comes from the device's stream-ordered
// pool (cudaMallocAsync), which keeps freed memory for reuse: creating and
// destroying simulations (one per serving job) then maps and unmaps nothing.
// dmalloc returns memory usable by every stream; dfree hands it back at once,
// so its callers make sure no queued work still reads it.
cudaStream_t pool_stream() {
  static std::mutex mu;
  static std::map<int, cudaStream_t> streams;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(mu);
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t st = nullptr;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    st = nullptr;
  }
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    unsigned long long keep = ~0ull;   // keep freed memory in the pool
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
  streams[dev] = st;
  return st;
}

template <typename T>
cudaError_t dmalloc(T **p, size_t bytes) {
  cudaStream_t st = pool_stream();
  cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(p), std::max<size_t>(bytes, 1), st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  // the kernels move records with 32-byte accesses and bulk copies: every
  // array must start on (at least) a 256-byte boundary, as device
  // allocations do
  if (e == cudaSuccess && (reinterpret_cast<uintptr_t>(*p) & 255u)) {
    cudaFreeAsync(*p, st);
    e = cudaErrorMisalignedAddress;
  }
  if (e != cudaSuccess) *p = nullptr;
  return e;
}

void dfree(void *p) {
  if (p) cudaFreeAsync(p, pool_stream());
}

cudaEvent_t record_event(spb_sim *s, cudaStream_t st) {
  cudaEvent_t e = nullptr;
  if (s->timing && cudaEventCreate(&e) == cudaSuccess) cudaEventRecord(e, st);
  return e;
}

int encode_field_map(spb_sim *s) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return fail(SPB_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is not available");
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  // dims innermost first: 8 channels, z nodes, y nodes, x nodes
  const cuuint64_t dims[4] = {8, (cuuint64_t)s->nzn, (cuuint64_t)s->nyn, (cuuint64_t)s->nxn};
  const cuuint64_t strides[3] = {32, 32ull * s->nzn, 32ull * s->nzn * s->nyn};
  const cuuint32_t box[4] = {8, (cuuint32_t)(s->tile[2] + 3), (cuuint32_t)(s->tile[1] + 3),
                             (cuuint32_t)(s->tile[0] + 3)};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = encode(&s->fmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, s->fields8, dims, strides,
                      box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(SPB_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  return SPB_OK;
}

// Dynamic shared memory of the kernels; the multi-job kernels also stage one
// job's parameters.
template <int TX, int TY, int TZ, int MINB>
size_t push_smem(bool multi = false) {
  return 2 * (size_t)Tile<TX, TY, TZ>::SF * 4 + (size_t)SIM_NW * 64 * sizeof(float4) +
         (size_t)SIM_NW * 2 * ring_half<MINB>() * 2 * sizeof(float4) +
         (multi ? sizeof(CycleParams) : 0) +
         (2 + 2 * SIM_NW) * sizeof(uint64_t);
}
template <int TX, int TY, int TZ>
size_t deposit_smem(bool multi = false, bool exact = false) {
  return (size_t)Tile<TX, TY, TZ>::TC * 80 * (exact ? sizeof(double) : sizeof(float)) +
         (multi ? sizeof(CycleParams) : 0);
}

}  // namespace

namespace spb {
// Kernel parameters for a cycle that reads buffer set `cur` and writes the other.
CycleParams make_params(spb_sim *s) {
  CycleParams P{};
  P.nxc = s->N[0];
  P.nyc = s->N[1];
  P.nzc = s->N[2];
  P.nxn = s->nxn;
  P.nyn = s->nyn;
  P.nzn = s->nzn;
  P.ntx = s->nt[0];
  P.nty = s->nt[1];
  P.ntz = s->nt[2];
  P.niter = s->d.niter;
  for (int a = 0; a < 3; ++a) {
    P.periodic[a] = s->d.periodic[a] ? 1 : 0;
    P.hdt[a] = (float)(0.5 * s->d.dt / s->dxyz[a]);
    P.fdt[a] = (float)(s->d.dt / s->dxyz[a]);
  }
  P.scale = 1.0 / (s->dxyz[0] * s->dxyz[1] * s->dxyz[2]);
  P.fields8 = s->fields8;
  P.err = s->d_err;
  P.ns = (int)s->sp.size();
  for (int i = 0; i < P.ns; ++i) {
    SimSpecies &q = s->sp[i];
    SpeciesDev &D = P.sp[i];
    const int c = q.cur, x = 1 - q.cur;
    D.rin = q.rec[c];
    D.rout = q.rec[x];
    D.base = q.base;
    D.cin = q.cnt[c];
    D.cout = q.cnt[x];
    D.oin = q.orec[c];
    D.okin = q.okey[c];
    D.ocin = q.ocnt + c;
    D.oout = q.orec[x];
    D.okout = q.okey[x];
    D.ocout = q.ocnt + x;
    D.mom = q.mom;
    D.ocap = q.ocap;
    D.qomdt2 = (float)(q.qom * (0.5 * s->d.dt) / s->d.c);
    for (int k = 0; k < 3; ++k) D.quantum[k] = q.quantum[k];
  }
  return P;
}
}  // namespace spb

namespace {

// One cycle: zero the moments and the write-side counters, push, deposit.
template <int TX, int TY, int TZ, int MINB>
int launch_cycle_v(spb_sim *s, cudaStream_t st) {
  for (auto &q : s->sp) {
    if (!q.rec[0]) return fail(SPB_ERR_INVALID, "spb_sim_cycle: a species was never loaded");
    SPB_CUDA(cudaMemsetAsync(q.mom, 0, 10 * s->nodes * sizeof(double), st));
    SPB_CUDA(cudaMemsetAsync(q.cnt[1 - q.cur], 0, s->ncells * sizeof(int), st));
    SPB_CUDA(cudaMemsetAsync(q.ocnt + (1 - q.cur), 0, sizeof(int), st));
  }
  const bool exact = s->d.deterministic != 0;
  const size_t psm = push_smem<TX, TY, TZ, MINB>(), dsm = deposit_smem<TX, TY, TZ>(false, exact);
  auto *const kdep = exact ? k_deposit<TX, TY, TZ, false, true> : k_deposit<TX, TY, TZ, false, false>;
  static bool attr = false;
  if (!attr) {
    SPB_CUDA(cudaFuncSetAttribute(k_push<TX, TY, TZ, MINB, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
    SPB_CUDA(cudaFuncSetAttribute(k_deposit<TX, TY, TZ, false, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)deposit_smem<TX, TY, TZ>(false, false)));
    SPB_CUDA(cudaFuncSetAttribute(k_deposit<TX, TY, TZ, false, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)deposit_smem<TX, TY, TZ>(false, true)));
    attr = true;
  }
  const CycleParams P = make_params(s);
  const int ntiles = s->nt[0] * s->nt[1] * s->nt[2];
  static int pocc = 0, docc[2] = {0, 0};   // resident CTAs per SM
  if (!pocc) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pocc, k_push<TX, TY, TZ, MINB, false>,
                                                      SIM_TPB, psm) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &docc[0], k_deposit<TX, TY, TZ, false, false>, dep_tpb<TX, TY, TZ>(),
            deposit_smem<TX, TY, TZ>(false, false)) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &docc[1], k_deposit<TX, TY, TZ, false, true>, dep_tpb<TX, TY, TZ>(),
            deposit_smem<TX, TY, TZ>(false, true)) != cudaSuccess) {
      cudaGetLastError();
      pocc = MINB;
      docc[0] = docc[1] = 1;
    }
    pocc = std::max(pocc, 1);
    docc[0] = std::max(docc[0], 1);
    docc[1] = std::max(docc[1], 1);
  }
  const int pctas = std::min(ntiles, s->d.ctas > 0 ? s->d.ctas : pocc * num_sms());
  const int dctas = std::min(ntiles, docc[exact ? 1 : 0] * num_sms());
  EvCycle ev{record_event(s, st), nullptr, nullptr};
  k_push<TX, TY, TZ, MINB, false><<<pctas, SIM_TPB, psm, st>>>(s->fmap, P, JobTable{},
                                                                      NoMaps{});
  SPB_CUDA(cudaGetLastError());
  ev.m = record_event(s, st);
  kdep<<<dctas, dep_tpb<TX, TY, TZ>(), dsm, st>>>(P, JobTable{});
  SPB_CUDA(cudaGetLastError());
  if (exact) {
    k_scale_moments<<<2 * num_sms(), 256, 0, st>>>(P);
    SPB_CUDA(cudaGetLastError());
    g_launches++;
    s->launches++;
  }
  ev.e = record_event(s, st);
  if (ev.b && ev.m && ev.e) s->ev_cycle.push_back(ev);
  g_launches += 2;
  s->launches += 2;
  for (auto &q : s->sp) q.cur = 1 - q.cur;
  return SPB_OK;
}

// The fused cycle: zeroing (moments, write-side counters, the tiles' flags
// and the barrier counters), then k_cycle as one cooperative launch of every
// CTA that fits on the device at once.
template <int TX, int TY, int TZ>
int launch_cycle_fused(spb_sim *s, cudaStream_t st) {
  constexpr int MINB = 2;
  for (auto &q : s->sp) {
    if (!q.rec[0]) return fail(SPB_ERR_INVALID, "spb_sim_cycle: a species was never loaded");
    SPB_CUDA(cudaMemsetAsync(q.mom, 0, 10 * s->nodes * sizeof(double), st));
    SPB_CUDA(cudaMemsetAsync(q.cnt[1 - q.cur], 0, s->ncells * sizeof(int), st));
    SPB_CUDA(cudaMemsetAsync(q.ocnt + (1 - q.cur), 0, sizeof(int), st));
  }
  const int ntiles = s->nt[0] * s->nt[1] * s->nt[2];
  SPB_CUDA(cudaMemsetAsync(s->fused_done, 0, (ntiles + 2) * sizeof(int), st));
  const size_t sm = fused_smem<TX, TY, TZ, MINB>();
  static int occ = -1;
  if (occ < 0) {
    SPB_CUDA(cudaFuncSetAttribute(k_cycle<TX, TY, TZ, MINB>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    SPB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cycle<TX, TY, TZ, MINB>,
                                                           SIM_TPB, sm));
  }
  if (occ < 1) return fail(SPB_ERR_UNSUPPORTED, "fused cycle: the kernel does not fit an SM");
  const int G = occ * num_sms();
  // largest launch-order distance between neighbouring tiles (folded
  // periodic axes: 2 positions)
  int step[3];
  for (int a = 0; a < 3; ++a) step[a] = (s->d.periodic[a] && s->nt[a] > 2) ? 2 : 1;
  const long R = (long)step[0] * s->nt[1] * s->nt[2] + (long)step[1] * s->nt[2] + step[2];
  const FusedAux X{s->fused_done, reinterpret_cast<unsigned *>(s->fused_done + ntiles),
                   (int)std::max<long>(1, ceil_div(R, G))};
  const CycleParams P = make_params(s);
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)G);
  cfg.blockDim = dim3(SIM_TPB);
  cfg.dynamicSmemBytes = sm;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  EvCycle ev{record_event(s, st), nullptr, nullptr};
  SPB_CUDA(cudaLaunchKernelEx(&cfg, k_cycle<TX, TY, TZ, MINB>, s->fmap, P, X));
  ev.m = record_event(s, st);
  ev.e = record_event(s, st);
  if (ev.b && ev.m && ev.e) s->ev_cycle.push_back(ev);
  g_launches += 1;
  s->launches += 1;
  for (auto &q : s->sp) q.cur = 1 - q.cur;
  return SPB_OK;
}

template <int TX, int TY, int TZ>
int launch_cycle(spb_sim *s, cudaStream_t st) {
  if (s->d.fused) return launch_cycle_fused<TX, TY, TZ>(s, st);
  switch (s->d.variant) {
    case 1: return launch_cycle_v<TX, TY, TZ, 2>(s, st);
    case 2: return launch_cycle_v<TX, TY, TZ, 4>(s, st);
    default: return launch_cycle_v<TX, TY, TZ, 3>(s, st);
  }
}

GridScalars scalars(const spb_sim *s) {
  GridScalars g;
  g.nxc = s->N[0];
  g.nyc = s->N[1];
  g.nzc = s->N[2];
  g.dx = s->dxyz[0];
  g.dy = s->dxyz[1];
  g.dz = s->dxyz[2];
  g.invdx = 1.0 / g.dx;
  g.invdy = 1.0 / g.dy;
  g.invdz = 1.0 / g.dz;
  return g;
}

void free_set(SimSpecies &q, int b) {
  dfree(q.rec[b]);
  q.rec[b] = nullptr;
  q.slots[b] = 0;
}

void free_buckets(SimSpecies &q) {
  for (int b = 0; b < 2; ++b) {
    free_set(q, b);
    dfree(q.cnt[b]);
    dfree(q.orec[b]);
    dfree(q.okey[b]);
    q.orec[b] = nullptr;
    q.cnt[b] = q.okey[b] = nullptr;
  }
  dfree(q.ocnt);
  dfree(q.base);
  dfree(q.base2);
  q.ocnt = nullptr;
  q.base = q.base2 = nullptr;
  q.ocap = 0;
  q.total = 0;
}

// Per-species arrays whose size does not depend on the layout.
int alloc_fixed(spb_sim *s, SimSpecies &q, int ocap) {
  if (q.base && q.ocap == ocap) return SPB_OK;
  if (q.base) SPB_CUDA(cudaDeviceSynchronize());   // queued work may still read the old arrays
  free_buckets(q);
  bool ok = dmalloc(&q.ocnt, 2 * sizeof(int)) == cudaSuccess &&
            dmalloc(&q.base, (s->ncells + 1) * sizeof(long long)) == cudaSuccess &&
            dmalloc(&q.base2, (s->ncells + 1) * sizeof(long long)) == cudaSuccess;
  for (int b = 0; b < 2 && ok; ++b)
    ok = dmalloc(&q.cnt[b], s->ncells * sizeof(int)) == cudaSuccess &&
         dmalloc(&q.orec[b], (size_t)ocap * 2 * sizeof(float4)) == cudaSuccess &&
         dmalloc(&q.okey[b], (size_t)ocap * sizeof(int)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    free_buckets(q);
    return fail(SPB_ERR_ALLOC, "overflow list / counter allocation failed");
  }
  q.ocap = ocap;
  return SPB_OK;
}

// Makes buffer set b hold at least `slots` records (1/16 headroom when it
// grows); waits for `st` only when it replaces a set queued work may read.
int ensure_set(SimSpecies &q, int b, long long slots, cudaStream_t st) {
  if (q.slots[b] >= slots && q.rec[b]) return SPB_OK;
  if (q.rec[b]) SPB_CUDA(cudaStreamSynchronize(st));
  free_set(q, b);
  const long long want = std::max<long long>(slots + slots / 16, 32);
  if (dmalloc(&q.rec[b], (size_t)want * 2 * sizeof(float4)) != cudaSuccess) {
    cudaGetLastError();
    return fail(SPB_ERR_ALLOC, "bucket allocation failed (64 bytes per record slot)");
  }
  q.slots[b] = want;
  return SPB_OK;
}

// Record slots any layout of n particles can need: every cell's capacity is
// at most count + count/2 + 16 rounded up to 4 (k_capacity), or the fixed
// bucket size. Buffer sets of this size are allocated before the layout is
// counted, so no load or re-layout waits for its counts on the host.
long long slots_bound(const spb_sim *s, long n) {
  const long long K = s->ncells;
  return s->d.bucket_slots > 0 ? (long long)s->d.bucket_slots * K : (3LL * n) / 2 + 19 * K;
}

// base[0..ncells] = exclusive scan of v[0..ncells); with `total`, returns
// base[ncells] (synchronises the stream).
int scan_layout(spb_sim *s, const long long *v, long long *out, long long *total,
                cudaStream_t st) {
  const long K = s->ncells;
  const int nb = (int)ceil_div(K, SCAN_B);
  k_scan_blocks<<<nb, SCAN_B, 0, st>>>(v, K, out, s->scan_tmp);
  k_scan_sums<<<1, SCAN_B, 0, st>>>(s->scan_tmp, nb, out + K);
  k_scan_add<<<nb, SCAN_B, 0, st>>>(out, K, s->scan_tmp);
  SPB_CUDA(cudaGetLastError());
  g_launches += 3;
  s->launches += 3;
  if (total) {
    SPB_CUDA(cudaMemcpyAsync(total, out + K, sizeof(long long), cudaMemcpyDeviceToHost, st));
    SPB_CUDA(cudaStreamSynchronize(st));
  }
  return SPB_OK;
}

SpeciesDev write_side(SimSpecies &q, int b, const long long *base) {
  SpeciesDev D{};
  D.rout = q.rec[b];
  D.base = base;
  D.cout = q.cnt[b];
  D.oout = q.orec[b];
  D.okout = q.okey[b];
  D.ocout = q.ocnt + b;
  D.ocap = q.ocap;
  return D;
}

// Lays out n reference-layout particles (device arrays) in fresh buckets:
// counts per cell, bucket capacities (count + slack, or desc.bucket_slots),
// fills buffer set 0.
template <int TX, int TY, int TZ>
int build(spb_sim *s, SimSpecies &q, const float *const src[7], long n, cudaStream_t st) {
  const GridScalars g = scalars(s);
  // the buffers hold max(n, the species' reserved capacity) particles
  const long sidx = (long)(&q - s->sp.data());
  const long nres = std::max<long>(n, sidx < SPB_SIM_MAX_SPECIES ? s->d.capacity[sidx] : 0);
  const long per = s->d.bucket_slots > 0      ? 1000
                   : s->d.overflow_per_mille > 0 ? s->d.overflow_per_mille
                                                 : 0;
  const long ocap =
      std::max<long>(65536, per > 0 ? (long)((double)nres * per / 1000.0) : nres / 32);
  if (ocap > (1L << 31) - 1) return fail(SPB_ERR_CAPACITY, "overflow list too large");
  if (int rc = alloc_fixed(s, q, (int)ocap)) return rc;
  if (int rc = ensure_set(q, 0, slots_bound(s, nres), st)) return rc;
  if (int rc = ensure_set(q, 1, slots_bound(s, nres), st)) return rc;
  SPB_CUDA(cudaMemsetAsync(s->counts, 0, s->ncells * sizeof(int), st));
  if (n > 0) {
    k_count_keys<TX, TY, TZ><<<blocks_for(n, 256), 256, 0, st>>>(g, s->nt[1], s->nt[2], src[0],
                                                                  src[1], src[2], n, s->counts,
                                                                  s->d_err);
    SPB_CUDA(cudaGetLastError());
  }
  k_capacity<<<blocks_for(s->ncells, 256), 256, 0, st>>>(s->counts, s->ncells,
                                                         s->d.bucket_slots, s->lcap);
  SPB_CUDA(cudaGetLastError());
  g_launches += 2;
  s->launches += 2;
  if (int rc = scan_layout(s, s->lcap, q.base, nullptr, st)) return rc;
  SPB_CUDA(cudaMemsetAsync(q.cnt[0], 0, s->ncells * sizeof(int), st));
  SPB_CUDA(cudaMemsetAsync(q.ocnt, 0, 2 * sizeof(int), st));
  if (n > 0) {
    k_fill<TX, TY, TZ><<<blocks_for(n, 256), 256, 0, st>>>(g, s->nt[1], s->nt[2], src[0], src[1],
                                                           src[2], src[3], src[4], src[5], src[6],
                                                           n, write_side(q, 0, q.base), s->d_err);
    SPB_CUDA(cudaGetLastError());
    g_launches++;
    s->launches++;
  }
  q.total = -1;   // read back when asked for (spb_sim_bucket_slots)
  q.n = n;
  q.cur = 0;
  // the deterministic deposit's grids: Q = 2^(ceil(log2 T) - 38) with T the
  // largest term of rhon, Jx..Jz, pxx..pzz (see exact_terms)
  q.quantum[0] = q.quantum[1] = q.quantum[2] = 1.0;
  if (n > 0 && s->d.deterministic) {
    unsigned *bounds = reinterpret_cast<unsigned *>(s->scan_tmp);   // free until the next scan
    unsigned h[2] = {0, 0};
    SPB_CUDA(cudaMemsetAsync(bounds, 0, 2 * sizeof(unsigned), st));
    k_species_bounds<<<blocks_for(n, 256), 256, 0, st>>>(src[6], src[3], src[4], src[5], n,
                                                         bounds);
    SPB_CUDA(cudaGetLastError());
    SPB_CUDA(cudaMemcpyAsync(h, bounds, sizeof(h), cudaMemcpyDeviceToHost, st));
    SPB_CUDA(cudaStreamSynchronize(st));
    g_launches++;
    s->launches++;
    float qmax, vmax;
    std::memcpy(&qmax, &h[0], sizeof(float));
    std::memcpy(&vmax, &h[1], sizeof(float));
    // |v|max at least c/8, so that a species loaded at rest keeps room for
    // the velocities it gains: a cell's sums have 2^13 T of room, so with 128
    // particles in a cell its pressure terms may grow to 64 T (velocities to
    // 8 x the bound) before a sum leaves its exact range
    const double qm = std::max((double)qmax, 1e-300);
    const double vm = std::max((double)vmax, std::max(s->d.c / 8.0, 1e-30));
    const double T[3] = {qm, qm * 4.0 * vm, qm * 16.0 * vm * vm};
    for (int k = 0; k < 3; ++k)
      q.quantum[k] = std::ldexp(1.0, (int)std::ceil(std::log2(T[k])) - 38);
  }
  return SPB_OK;
}

// Re-layout in place of the buffer sets: bucket capacities from the current
// counts (buckets + overflow list), then one copy from buffer set `cur` into
// the other. 64 bytes per particle plus the per-cell passes.
int relayout(spb_sim *s, SimSpecies &q, cudaStream_t st) {
  if (!q.base) return SPB_OK;
  const long K = s->ncells;
  const int c = q.cur, x = 1 - q.cur;
  k_count_buckets<<<blocks_for(K, 256), 256, 0, st>>>(q.base, q.cnt[c], K, s->counts);
  k_count_overflow<<<blocks_for(q.ocap, 256), 256, 0, st>>>(q.okey[c], q.ocnt + c, q.ocap,
                                                            s->counts);
  k_capacity<<<blocks_for(K, 256), 256, 0, st>>>(s->counts, K, s->d.bucket_slots, s->lcap);
  SPB_CUDA(cudaGetLastError());
  g_launches += 3;
  s->launches += 3;
  if (int rc = scan_layout(s, s->lcap, q.base2, nullptr, st)) return rc;
  // the counts sum to the species' particles: the sets sized at the load hold it
  if (int rc = ensure_set(q, x, slots_bound(s, q.n), st)) return rc;
  SPB_CUDA(cudaMemsetAsync(q.cnt[x], 0, K * sizeof(int), st));
  SPB_CUDA(cudaMemsetAsync(q.ocnt + x, 0, sizeof(int), st));
  k_relayout<<<blocks_for(K * 32, 256), 256, 0, st>>>(q.base, q.rec[c], q.cnt[c], K, q.orec[c],
                                                       q.okey[c], q.ocnt + c, q.ocap,
                                                       write_side(q, x, q.base2), s->d_err);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  s->launches++;
  std::swap(q.base, q.base2);
  q.total = -1;
  q.cur = x;
  // the other set is written by the next cycle: it must hold the new layout too
  return ensure_set(q, c, slots_bound(s, q.n), st);
}

// Particles of buffer set `cur` into flat device arrays (dst[6], q, may be null).
template <int TX, int TY, int TZ>
int unload(spb_sim *s, SimSpecies &q, float *const dst[7], cudaStream_t st) {
  const long K = s->ncells;
  k_clamp_counts<<<blocks_for(K, 256), 256, 0, st>>>(q.base, q.cnt[q.cur], K, s->lcap);
  SPB_CUDA(cudaGetLastError());
  if (int rc = scan_layout(s, s->lcap, s->offset, nullptr, st)) return rc;
  Unload o{dst[0], dst[1], dst[2], dst[3], dst[4], dst[5], dst[6], q.n};
  k_unload<TX, TY, TZ><<<blocks_for(K * 32, 256), 256, 0, st>>>(
      scalars(s), s->nt[1], s->nt[2], K, q.rec[q.cur], q.base, q.cnt[q.cur], s->offset,
      q.orec[q.cur], q.okey[q.cur], q.ocnt + q.cur, q.ocap, o);
  SPB_CUDA(cudaGetLastError());
  g_launches += 2;
  s->launches += 2;
  return SPB_OK;
}

}  // namespace

namespace spb {

JobBuffers::~JobBuffers() {
  if (ready) cudaEventDestroy(ready);
  cudaFree(d_tile_base);
  cudaFree(d_params);
  cudaFreeHost(h_tile_base);
  cudaFreeHost(h_params);
}

}  // namespace spb

namespace {

int ensure_job_buffers(JobBuffers &B, int n) {
  if (!B.ready) SPB_CUDA(cudaEventCreateWithFlags(&B.ready, cudaEventDisableTiming));
  // the pinned mirrors may still be read by the previous launch's copies
  SPB_CUDA(cudaEventSynchronize(B.ready));
  if (n <= B.cap) return SPB_OK;
  const int cap = std::max(n, 2 * B.cap);
  cudaFree(B.d_tile_base);
  cudaFree(B.d_params);
  cudaFreeHost(B.h_tile_base);
  cudaFreeHost(B.h_params);
  B.d_tile_base = B.h_tile_base = nullptr;
  B.d_params = B.h_params = nullptr;
  B.cap = 0;
  if (cudaMalloc(&B.d_tile_base, (cap + 1) * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&B.d_params, cap * sizeof(CycleParams)) != cudaSuccess ||
      cudaMallocHost(&B.h_tile_base, (cap + 1) * sizeof(int)) != cudaSuccess ||
      cudaMallocHost(&B.h_params, cap * sizeof(CycleParams)) != cudaSuccess) {
    cudaGetLastError();
    return fail(SPB_ERR_ALLOC, "job table allocation failed");
  }
  B.cap = cap;
  return SPB_OK;
}

template <int TX, int TY, int TZ>
int launch_jobs_t(spb_sim *const *sims, int n, JobBuffers &B, cudaStream_t st) {
  constexpr int MINB = 3;
  const size_t psm = push_smem<TX, TY, TZ, MINB>(true), dsm = deposit_smem<TX, TY, TZ>(true);
  static int pocc = 0, docc = 0;
  if (!pocc) {
    SPB_CUDA(cudaFuncSetAttribute(k_push<TX, TY, TZ, MINB, true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
    SPB_CUDA(cudaFuncSetAttribute(k_deposit<TX, TY, TZ, true, false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dsm));
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pocc, k_push<TX, TY, TZ, MINB, true>,
                                                      SIM_TPB, psm) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&docc, k_deposit<TX, TY, TZ, true, false>,
                                                      dep_tpb<TX, TY, TZ>(), dsm) != cudaSuccess) {
      cudaGetLastError();
      pocc = MINB;
      docc = 1;
    }
    pocc = std::max(pocc, 1);
    docc = std::max(docc, 1);
  }
  if (n > SERVE_MAX_JOBS) return fail(SPB_ERR_CAPACITY, "at most 64 jobs per launch");
  if (int rc = ensure_job_buffers(B, n)) return rc;
  static JobMaps maps;   // 8 KB, passed by value as a kernel parameter
  int total = 0;
  for (int j = 0; j < n; ++j) {
    spb_sim *s = sims[j];
    B.h_tile_base[j] = total;
    total += s->nt[0] * s->nt[1] * s->nt[2];
    B.h_params[j] = make_params(s);
    maps.m[j] = s->fmap;
  }
  B.h_tile_base[n] = total;
  SPB_CUDA(cudaMemcpyAsync(B.d_tile_base, B.h_tile_base, (n + 1) * sizeof(int),
                           cudaMemcpyHostToDevice, st));
  SPB_CUDA(cudaMemcpyAsync(B.d_params, B.h_params, n * sizeof(CycleParams),
                           cudaMemcpyHostToDevice, st));
  SPB_CUDA(cudaEventRecord(B.ready, st));
  const JobTable J{n, total, B.d_tile_base, B.d_params};
  k_zero_jobs<<<2 * num_sms(), 256, 0, st>>>(J);
  SPB_CUDA(cudaGetLastError());
  const int pctas = std::min(total, pocc * num_sms());
  const int dctas = std::min(total, docc * num_sms());
  k_push<TX, TY, TZ, MINB, true><<<pctas, SIM_TPB, psm, st>>>(CUtensorMap{}, CycleParams{}, J,
                                                              maps);
  SPB_CUDA(cudaGetLastError());
  k_deposit<TX, TY, TZ, true, false><<<dctas, dep_tpb<TX, TY, TZ>(), dsm, st>>>(CycleParams{}, J);
  SPB_CUDA(cudaGetLastError());
  g_launches += 3;
  for (int j = 0; j < n; ++j) {
    sims[j]->launches += 2;
    for (auto &q : sims[j]->sp) q.cur = 1 - q.cur;
  }
  return SPB_OK;
}

}  // namespace

namespace {

// Tile shapes the kernels are instantiated for.
struct TileImpl {
  int t[3];
  int (*cycle)(spb_sim *, cudaStream_t);
  int (*jobs)(spb_sim *const *, int, JobBuffers &, cudaStream_t);
  int (*build)(spb_sim *, SimSpecies &, const float *const *, long, cudaStream_t);
  int (*unload)(spb_sim *, SimSpecies &, float *const *, cudaStream_t);
};

#define SPB_TILE(X, Y, Z) \
  TileImpl {                                                                   \
    {X, Y, Z}, launch_cycle<X, Y, Z>, launch_jobs_t<X, Y, Z>, build<X, Y, Z>, unload<X, Y, Z> \
  }
const TileImpl kTiles[] = {SPB_TILE(8, 4, 4), SPB_TILE(4, 4, 4), SPB_TILE(2, 2, 2),
                           SPB_TILE(8, 8, 4)};
#undef SPB_TILE

const TileImpl *find_tile(const int t[3]) {
  for (const TileImpl &ti : kTiles)
    if (ti.t[0] == t[0] && ti.t[1] == t[1] && ti.t[2] == t[2]) return &ti;
  return nullptr;
}

}  // namespace

namespace spb {

int launch_jobs(spb_sim *const *sims, int n, JobBuffers &buf, cudaStream_t st) {
  if (n <= 0) return SPB_OK;
  for (int j = 0; j < n; ++j) {
    const spb_sim *s = sims[j];
    if (!s || !s->fields_set) return fail(SPB_ERR_INVALID, "launch_jobs: job without fields");
    for (int a = 0; a < 3; ++a)
      if (s->tile[a] != sims[0]->tile[a])
        return fail(SPB_ERR_INVALID, "launch_jobs: jobs of one launch share the tile shape");
    for (const auto &q : s->sp)
      if (!q.rec[0]) return fail(SPB_ERR_INVALID, "launch_jobs: a species was never loaded");
  }
  return find_tile(sims[0]->tile)->jobs(sims, n, buf, st);
}

}  // namespace spb

namespace {

// Temporary flat reference-layout arrays (7 x n floats).
struct Flat {
  float *buf = nullptr;
  float *p[7] = {};
  int alloc(long n) {
    if (dmalloc(&buf, 7 * std::max<long>(n, 1) * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return fail(SPB_ERR_ALLOC, "temporary particle arrays: allocation failed");
    }
    for (int a = 0; a < 7; ++a) p[a] = buf + a * n;
    return SPB_OK;
  }
  void release(cudaStream_t st) {
    if (buf) {
      cudaStreamSynchronize(st);
      dfree(buf);
      buf = nullptr;
    }
  }
};

}  // namespace

extern "C" int spb_sim_tile_supported(int tx, int ty, int tz) {
  const int t[3] = {tx, ty, tz};
  return find_tile(t) != nullptr;
}

extern "C" int spb_sim_create(const spb_sim_desc *d, spb_sim **out) {
  if (!d || !out) return fail(SPB_ERR_INVALID, "spb_sim_create: null argument");
  *out = nullptr;
  if (d->ns < 1 || d->ns > SIM_MAX_SPECIES)
    return fail(SPB_ERR_INVALID, "spb_sim_create: 1..8 species");
  if (d->nxc < 1 || d->nyc < 1 || d->nzc < 1 || d->nxc > 2047 || d->nyc > 1023 || d->nzc > 2047)
    return fail(SPB_ERR_UNSUPPORTED, "spb_sim_create: cells per axis must be in [1,2047]x[1,1023]x[1,2047]");
  if ((long)d->nxc * d->nyc * d->nzc >= (1L << 31))
    return fail(SPB_ERR_UNSUPPORTED, "spb_sim_create: at most 2^31 - 1 cells");
  if (d->niter < 1 || !(d->dt > 0) || !(d->c != 0))
    return fail(SPB_ERR_INVALID, "spb_sim_create: bad NiterMover, dt or c");
  if (d->bucket_slots < 0) return fail(SPB_ERR_INVALID, "spb_sim_create: bucket_slots < 0");
  if (d->fused && d->deterministic)
    return fail(SPB_ERR_UNSUPPORTED,
                "spb_sim_create: the fused cycle has no deterministic deposit (use one of them)");
  int tile[3] = {d->tile[0], d->tile[1], d->tile[2]};
  if (!tile[0] || !tile[1] || !tile[2]) {
    tile[0] = 8;
    tile[1] = 4;
    tile[2] = 4;
  }
  const TileImpl *ti = find_tile(tile);
  if (!ti) return fail(SPB_ERR_UNSUPPORTED, "spb_sim_create: tile shape not instantiated");
  if (d->nxc % tile[0] || d->nyc % tile[1] || d->nzc % tile[2])
    return fail(SPB_ERR_UNSUPPORTED, "spb_sim_create: cells per axis must be multiples of the tile");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(SPB_ERR_NO_DEVICE, "no CUDA device");
  }
  auto *s = new spb_sim();
  s->d = *d;
  SPB_CUDA(cudaGetDevice(&s->device));
  s->N[0] = d->nxc;
  s->N[1] = d->nyc;
  s->N[2] = d->nzc;
  for (int a = 0; a < 3; ++a) {
    s->tile[a] = tile[a];
    s->nt[a] = s->N[a] / tile[a];
  }
  s->dxyz[0] = d->Lx / d->nxc;
  s->dxyz[1] = d->Ly / d->nyc;
  s->dxyz[2] = d->Lz / d->nzc;
  s->nxn = d->nxc + 3;
  s->nyn = d->nyc + 3;
  s->nzn = d->nzc + 3;
  s->nodes = (long)s->nxn * s->nyn * s->nzn;
  s->ncells = (long)d->nxc * d->nyc * d->nzc;
  auto bail = [&](int rc) {
    spb_sim_destroy(s);
    return rc;
  };
  const long nb = ceil_div(s->ncells, SCAN_B);
  if (dmalloc(&s->fields8, s->nodes * 8 * sizeof(float)) != cudaSuccess ||
      dmalloc(&s->d_err, sizeof(int)) != cudaSuccess ||
      dmalloc(&s->scan_tmp, (nb + 1) * sizeof(long long)) != cudaSuccess ||
      dmalloc(&s->counts, s->ncells * sizeof(int)) != cudaSuccess ||
      dmalloc(&s->lcap, s->ncells * sizeof(long long)) != cudaSuccess ||
      dmalloc(&s->offset, (s->ncells + 1) * sizeof(long long)) != cudaSuccess) {
    cudaGetLastError();
    return bail(fail(SPB_ERR_ALLOC, "spb_sim_create: device allocation failed"));
  }
  if (d->fused && dmalloc(&s->fused_done, (s->nt[0] * s->nt[1] * s->nt[2] + 2) * sizeof(int)) !=
                      cudaSuccess) {
    cudaGetLastError();
    return bail(fail(SPB_ERR_ALLOC, "spb_sim_create: device allocation failed"));
  }
  if (cudaMemset(s->d_err, 0, sizeof(int)) != cudaSuccess ||
      cudaMemset(s->fields8, 0, s->nodes * 8 * sizeof(float)) != cudaSuccess)
    return bail(fail(SPB_ERR_CUDA, "spb_sim_create: memset failed"));
  if (int rc = encode_field_map(s)) return bail(rc);
  s->sp.resize(d->ns);
  for (int i = 0; i < d->ns; ++i) {
    SimSpecies &q = s->sp[i];
    q.qom = d->qom[i];
    if (dmalloc(&q.mom, 10 * s->nodes * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return bail(fail(SPB_ERR_ALLOC, "spb_sim_create: device allocation failed"));
    }
    if (cudaMemset(q.mom, 0, 10 * s->nodes * sizeof(double)) != cudaSuccess)
      return bail(fail(SPB_ERR_CUDA, "spb_sim_create: memset failed"));
  }
  *out = s;
  return SPB_OK;
}

namespace {
float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float t = 0;
  if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&t, a, b) != cudaSuccess)
    return 0.0f;
  return t;
}

void drain(spb_sim *s, double *push_ms, double *dep_ms, int *ncycles, double *relayout_ms,
           int *nrelayouts) {
  double p = 0, d = 0, r = 0;
  for (auto &e : s->ev_cycle) {
    p += elapsed(e.b, e.m);
    d += elapsed(e.m, e.e);
    cudaEventDestroy(e.b);
    cudaEventDestroy(e.m);
    cudaEventDestroy(e.e);
  }
  for (auto &e : s->ev_relayout) {
    r += elapsed(e.first, e.second);
    cudaEventDestroy(e.first);
    cudaEventDestroy(e.second);
  }
  if (push_ms) *push_ms = p;
  if (dep_ms) *dep_ms = d;
  if (relayout_ms) *relayout_ms = r;
  if (ncycles) *ncycles = (int)s->ev_cycle.size();
  if (nrelayouts) *nrelayouts = (int)s->ev_relayout.size();
  s->ev_cycle.clear();
  s->ev_relayout.clear();
}
}  // namespace

extern "C" int spb_sim_set_timing(spb_sim *s, int on) {
  if (!s) return fail(SPB_ERR_INVALID, "spb_sim_set_timing: null simulation");
  s->timing = on != 0;
  return SPB_OK;
}

extern "C" int spb_sim_timing(spb_sim *s, double *cycle_ms, int *ncycle, double *sort_ms,
                              int *nsort) {
  if (!s) return fail(SPB_ERR_INVALID, "spb_sim_timing: null simulation");
  double p = 0, d = 0;
  drain(s, &p, &d, ncycle, sort_ms, nsort);
  if (cycle_ms) *cycle_ms = p + d;
  return SPB_OK;
}

extern "C" int spb_sim_kernel_timing(spb_sim *s, double *push_ms, double *deposit_ms,
                                     int *ncycles, double *relayout_ms, int *nrelayouts) {
  if (!s) return fail(SPB_ERR_INVALID, "spb_sim_kernel_timing: null simulation");
  drain(s, push_ms, deposit_ms, ncycles, relayout_ms, nrelayouts);
  return SPB_OK;
}

namespace {

void drop_graphs(spb_sim *s) {
  for (auto &g : s->graphs) cudaGraphExecDestroy(g.second);
  s->graphs.clear();
}

unsigned parity_key(const spb_sim *s) {
  unsigned k = 0;
  for (size_t i = 0; i < s->sp.size(); ++i) k |= (unsigned)s->sp[i].cur << i;
  return k;
}

// One cycle. With desc.graph (and timing off) the cycle's launches (zeroing,
// push, deposit) are captured once per buffer-parity pattern of the species
// as a CUDA graph and replayed; the first cycle of a simulation runs directly
// (it sets the kernels' attributes). Any capture failure falls back to
// direct launches for the rest of the simulation's life.
int run_cycle(spb_sim *s, const TileImpl *ti, cudaStream_t st) {
  const bool use_graph = s->d.graph && !s->timing && !s->graph_failed && s->cycles_run > 0;
  s->cycles_run++;
  if (!use_graph) return ti->cycle(s, st);
  if (!s->gstream) {
    if (cudaStreamCreateWithFlags(&s->gstream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->gev[0], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->gev[1], cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      s->graph_failed = true;
      return ti->cycle(s, st);
    }
  }
  SPB_CUDA(cudaEventRecord(s->gev[0], st));
  SPB_CUDA(cudaStreamWaitEvent(s->gstream, s->gev[0], 0));
  const unsigned key = parity_key(s);
  auto it = s->graphs.find(key);
  if (it != s->graphs.end()) {
    SPB_CUDA(cudaGraphLaunch(it->second, s->gstream));
    for (auto &q : s->sp) q.cur = 1 - q.cur;
    g_launches += 2;
    s->launches += 2;
  } else {
    // capture (the captured call flips the buffer sets, as a direct launch does)
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    SPB_CUDA(cudaStreamBeginCapture(s->gstream, cudaStreamCaptureModeThreadLocal));
    const int rc = ti->cycle(s, s->gstream);
    const cudaError_t e1 = cudaStreamEndCapture(s->gstream, &g);
    const cudaError_t e2 = (rc == SPB_OK && e1 == cudaSuccess)
                               ? cudaGraphInstantiate(&ex, g, 0)
                               : cudaErrorStreamCaptureInvalidated;
    if (g) cudaGraphDestroy(g);
    if (rc != SPB_OK || e1 != cudaSuccess || e2 != cudaSuccess) {
      // undo the flip of the captured (never executed) call, then run directly
      cudaGetLastError();
      if (rc == SPB_OK)
        for (auto &q : s->sp) q.cur = 1 - q.cur;
      s->graph_failed = true;
      return ti->cycle(s, st);
    }
    s->graphs[key] = ex;
    SPB_CUDA(cudaGraphLaunch(ex, s->gstream));
  }
  SPB_CUDA(cudaEventRecord(s->gev[1], s->gstream));
  SPB_CUDA(cudaStreamWaitEvent(st, s->gev[1], 0));
  return SPB_OK;
}

}  // namespace

namespace spb {
// Frees a simulation. sync: wait for the whole device first (queued work may
// still read the memory returned); the serving engine passes false for jobs
// whose work it knows to be complete.
void sim_free(spb_sim *s, bool sync);
}  // namespace spb

extern "C" void spb_sim_destroy(spb_sim *s) { spb::sim_free(s, true); }

void spb::sim_free(spb_sim *s, bool sync) {
  if (!s) return;
  drop_graphs(s);
  if (s->gstream) cudaStreamDestroy(s->gstream);
  for (cudaEvent_t e : s->gev)
    if (e) cudaEventDestroy(e);
  drain(s, nullptr, nullptr, nullptr, nullptr, nullptr);
  if (sync) cudaDeviceSynchronize();   // no queued work may still read the memory returned below
  for (auto &q : s->sp) {
    free_buckets(q);
    dfree(q.mom);
  }
  dfree(s->fields8);
  dfree(s->stage);
  dfree(s->d_err);
  dfree(s->scan_tmp);
  dfree(s->counts);
  dfree(s->lcap);
  dfree(s->offset);
  dfree(s->fused_done);
  delete s;
}

extern "C" long spb_sim_nodes(const spb_sim *s) { return s ? s->nodes : 0; }
extern "C" long spb_sim_count(const spb_sim *s, int species) {
  if (!s || species < 0 || species >= (int)s->sp.size()) return -1;
  return s->sp[species].n;
}
extern "C" long spb_sim_launches(const spb_sim *s) { return s ? s->launches : 0; }

extern "C" long spb_sim_bucket_slots(spb_sim *s, int species) {
  if (!s || species < 0 || species >= (int)s->sp.size()) return -1;
  SimSpecies &q = s->sp[species];
  if (q.total < 0 && q.base) {
    long long t = 0;
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(&t, q.base + s->ncells, sizeof(t), cudaMemcpyDeviceToHost) != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
    q.total = t;
  }
  return (long)std::max<long long>(q.total, 0);
}

extern "C" long spb_sim_overflow(spb_sim *s, int species, void *stream) {
  if (!s || species < 0 || species >= (int)s->sp.size()) return -1;
  SimSpecies &q = s->sp[species];
  if (!q.ocnt) return 0;
  int h = 0;
  if (cudaMemcpyAsync(&h, q.ocnt + q.cur, sizeof(int), cudaMemcpyDeviceToHost,
                      (cudaStream_t)stream) != cudaSuccess ||
      cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  return h;
}

extern "C" int spb_sim_set_fields(spb_sim *s, const float *const fields[6], int on_device,
                                  void *stream) {
  if (!s || !fields) return fail(SPB_ERR_INVALID, "spb_sim_set_fields: null argument");
  for (int f = 0; f < 6; ++f)
    if (!fields[f]) return fail(SPB_ERR_INVALID, "spb_sim_set_fields: null field array");
  cudaStream_t st = (cudaStream_t)stream;
  const float *src[6];
  if (on_device) {
    for (int f = 0; f < 6; ++f) src[f] = fields[f];
  } else {
    if (!s->stage && dmalloc(&s->stage, 6 * s->nodes * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return fail(SPB_ERR_ALLOC, "spb_sim_set_fields: staging allocation failed");
    }
    for (int f = 0; f < 6; ++f) {
      SPB_CUDA(cudaMemcpyAsync(s->stage + f * s->nodes, fields[f], s->nodes * sizeof(float),
                               cudaMemcpyHostToDevice, st));
      src[f] = s->stage + f * s->nodes;
    }
  }
  k_pack_fields8<<<blocks_for(s->nodes, 256), 256, 0, st>>>(src[0], src[1], src[2], src[3],
                                                            src[4], src[5], s->fields8, s->nodes);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  s->launches++;
  s->fields_set = true;
  return SPB_OK;
}

extern "C" int spb_sim_load_species(spb_sim *s, int species, const float *x, const float *y,
                                    const float *z, const float *u, const float *v, const float *w,
                                    const float *q, long n, int on_device, void *stream) {
  if (!s || species < 0 || species >= (int)s->sp.size())
    return fail(SPB_ERR_INVALID, "spb_sim_load_species: bad species");
  if (n < 0 || (n > 0 && (!x || !y || !z || !u || !v || !w || !q)))
    return fail(SPB_ERR_INVALID, "spb_sim_load_species: bad particle arrays");
  if (n >= (1L << 31) - 256)
    return fail(SPB_ERR_UNSUPPORTED, "spb_sim_load_species: at most 2^31 - 256 particles");
  cudaStream_t st = (cudaStream_t)stream;
  const float *src[7] = {x, y, z, u, v, w, q};
  Flat f;
  if (!on_device && n > 0) {
    if (int rc = f.alloc(n)) return rc;
    for (int a = 0; a < 7; ++a) {
      SPB_CUDA(cudaMemcpyAsync(f.p[a], src[a], n * sizeof(float), cudaMemcpyHostToDevice, st));
      src[a] = f.p[a];
    }
  }
  const TileImpl *ti = find_tile(s->tile);
  drop_graphs(s);   // the new layout's pointers differ from the captured ones
  const int rc = ti->build(s, s->sp[species], src, n, st);
  f.release(st);
  s->cycles_since_check = 0;
  return rc;
}

extern "C" int spb_sim_resort(spb_sim *s, void *stream) {
  if (!s) return fail(SPB_ERR_INVALID, "spb_sim_resort: null simulation");
  cudaStream_t st = (cudaStream_t)stream;
  const cudaEvent_t b = record_event(s, st);
  drop_graphs(s);
  for (auto &q : s->sp)
    if (int rc = relayout(s, q, st)) return rc;
  const cudaEvent_t e = record_event(s, st);
  if (b && e) s->ev_relayout.push_back({b, e});
  s->cycles_since_check = 0;
  return SPB_OK;
}

namespace spb {
// Maps up to `bytes` of device memory into the pool (chunks allocated and
// freed again; the pool keeps them). Stops quietly at the first chunk that
// does not fit.
void pool_reserve(long long bytes) {
  cudaStream_t st = pool_stream();
  std::vector<void *> chunks;
  const long long chunk = 1LL << 30;
  for (long long got = 0; got < bytes; got += chunk) {
    void *p = nullptr;
    if (cudaMallocAsync(&p, (size_t)std::min(chunk, bytes - got), st) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    chunks.push_back(p);
  }
  for (void *p : chunks) cudaFreeAsync(p, st);
  cudaStreamSynchronize(st);
}

// Overflow entries at which a species is re-laid out: 1/256 of its particles
// (at least 256), at most a quarter of the overflow list, so that the list
// keeps room for the cycles until the next check.
long relayout_threshold(const SimSpecies &q) {
  return std::min<long>(q.ocap / 4, std::max<long>(256, q.n / 256));
}
}  // namespace spb

extern "C" int spb_release_cached_memory(void) {
  SPB_CUDA(cudaDeviceSynchronize());
  int dev = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  SPB_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  SPB_CUDA(cudaMemPoolTrimTo(pool, 0));
  return SPB_OK;
}

extern "C" int spb_sim_cycle(spb_sim *s, int ncycles, void *stream) {
  if (!s || ncycles < 0) return fail(SPB_ERR_INVALID, "spb_sim_cycle: bad arguments");
  if (!s->fields_set) return fail(SPB_ERR_INVALID, "spb_sim_cycle: fields not set");
  cudaStream_t st = (cudaStream_t)stream;
  const TileImpl *ti = find_tile(s->tile);
  const int k = std::max(1, s->d.resort_every);
  for (int c = 0; c < ncycles; ++c) {
    if (s->cycles_since_check >= k) {
      // re-lay out the species whose overflow list has grown past its
      // threshold (the entries below it are pushed and deposited exactly,
      // only more slowly)
      const cudaEvent_t b = record_event(s, st);
      bool any = false;
      for (int i = 0; i < (int)s->sp.size(); ++i) {
        const long o = spb_sim_overflow(s, i, stream);
        if (o < 0) return fail(SPB_ERR_CUDA, "spb_sim_cycle: overflow counter read failed");
        if (o > relayout_threshold(s->sp[i])) {
          drop_graphs(s);
          if (int rc = relayout(s, s->sp[i], st)) return rc;
          any = true;
        }
      }
      const cudaEvent_t e = record_event(s, st);
      if (b && e && any) {
        s->ev_relayout.push_back({b, e});
      } else {
        if (b) cudaEventDestroy(b);
        if (e) cudaEventDestroy(e);
      }
      s->cycles_since_check = 0;
    }
    if (int rc = run_cycle(s, ti, st)) return rc;
    s->cycles_since_check++;
  }
  return SPB_OK;
}

extern "C" int spb_sim_moments(spb_sim *s, int species, double *out, int on_device,
                               void *stream) {
  if (!s || !out || species < 0 || species >= (int)s->sp.size())
    return fail(SPB_ERR_INVALID, "spb_sim_moments: bad arguments");
  SPB_CUDA(cudaMemcpyAsync(out, s->sp[species].mom, 10 * s->nodes * sizeof(double),
                           on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           (cudaStream_t)stream));
  return SPB_OK;
}

extern "C" double *spb_sim_moments_device(spb_sim *s, int species) {
  if (!s || species < 0 || species >= (int)s->sp.size()) {
    fail(SPB_ERR_INVALID, "spb_sim_moments_device: bad arguments");
    return nullptr;
  }
  return s->sp[species].mom;
}

extern "C" int spb_sim_apply_bc_ids(spb_sim *s, int species, void *stream) {
  if (!s || species < 0 || species >= (int)s->sp.size())
    return fail(SPB_ERR_INVALID, "spb_sim_apply_bc_ids: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const long plane[3] = {(long)(s->nyn - 2) * (s->nzn - 2), (long)(s->nxn - 2) * (s->nzn - 2),
                         (long)(s->nxn - 2) * (s->nyn - 2)};
  for (int pass = 0; pass < 2; ++pass)
    for (int axis = 0; axis < 3; ++axis) {
      const bool fold = s->d.periodic[axis] != 0;
      if (fold != (pass == 0)) continue;
      k_bc_fold64<<<(unsigned)ceil_div(plane[axis], 256), 256, 0, st>>>(
          s->sp[species].mom, s->nxn, s->nyn, s->nzn, axis, fold ? 1 : 0);
      SPB_CUDA(cudaGetLastError());
      g_launches++;
      s->launches++;
    }
  return SPB_OK;
}

extern "C" int spb_sim_particles(spb_sim *s, int species, float *x, float *y, float *z, float *u,
                                 float *v, float *w, float *q, int on_device, void *stream) {
  if (!s || species < 0 || species >= (int)s->sp.size())
    return fail(SPB_ERR_INVALID, "spb_sim_particles: bad arguments");
  SimSpecies &S = s->sp[species];
  if (S.n == 0 || !S.rec[0]) return SPB_OK;
  if (!x || !y || !z || !u || !v || !w)
    return fail(SPB_ERR_INVALID, "spb_sim_particles: null output array");
  cudaStream_t st = (cudaStream_t)stream;
  const TileImpl *ti = find_tile(s->tile);
  float *dst[7] = {x, y, z, u, v, w, q};
  if (on_device) return ti->unload(s, S, dst, st);
  Flat f;
  if (int rc = f.alloc(S.n)) return rc;
  float *tmp[7];
  for (int a = 0; a < 7; ++a) tmp[a] = dst[a] ? f.p[a] : nullptr;
  int rc = ti->unload(s, S, tmp, st);
  for (int a = 0; a < 7 && !rc; ++a)
    if (dst[a] && cudaMemcpyAsync(dst[a], tmp[a], S.n * sizeof(float), cudaMemcpyDeviceToHost,
                                  st) != cudaSuccess)
      rc = fail_cuda(cudaGetLastError(), "spb_sim_particles: copy to host");
  f.release(st);
  return rc;
}

namespace spb {
// The status of a simulation's error word (0: SPB_OK).
int sim_status(int h) {
  if (h) {
    if (h & ERRBIT_TIMEOUT) return fail(SPB_ERR_TIMEOUT, "a staged field tile never arrived (bounded wait)");
    if (h & ERRBIT_SMEM_ALIGN) return fail(SPB_ERR_UNSUPPORTED, "shared memory not 128-byte aligned for TMA");
    if (h & ERRBIT_INEXACT)
      return fail(SPB_ERR_CAPACITY,
                  "a deterministic deposit sum left its exact range (the moments are accurate "
                  "but not guaranteed bitwise reproducible)");
    if (h & ERRBIT_LOST)
      return fail(SPB_ERR_CAPACITY, "a cell's bucket and the overflow list were both full: particles lost");
    return fail(SPB_ERR_OUT_OF_GRID, "a particle left the node array and was clamped");
  }
  return SPB_OK;
}
}  // namespace spb

extern "C" int spb_sim_check(spb_sim *s, void *stream) {
  if (!s) return fail(SPB_ERR_INVALID, "spb_sim_check: null simulation");
  SPB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  int h = 0;
  SPB_CUDA(cudaMemcpy(&h, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) SPB_CUDA(cudaMemset(s->d_err, 0, sizeof(int)));
  return spb::sim_status(h);
}
