// Precision form of the mover + deposit (spb_sim_*): HBM-resident, cell-sorted
// particles with int32 cell + FP32 in-cell offsets, FP32 push and gather,
// FP32 shared-memory deposit partials flushed into FP64 global moments.
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
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "grid_ctx.h"
#include "kernels.h"
#include "sim_kernels.cuh"

namespace spb {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int SIM_TPB = 256;                 // 8 warps per CTA
constexpr int SIM_NW = SIM_TPB / 32;
constexpr int QCAP = 64;                     // mover queue entries per warp
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

// ---------------------------------------------------------------------------
// push in cell units
// ---------------------------------------------------------------------------

// Gather cell and fraction of a predicted position p (cells, relative to the
// particle's cell c). Below the domain the reference's int() truncates toward
// zero, so the cell rounds up and the fraction goes negative. Branch-free;
// cells outside [-1, N] are left to the gather's bounds handling.
__device__ __forceinline__ void locate(float p, int c, int N, int &g, float &f) {
  const float lim = (float)(N + 8);
  const float s = fminf(fmaxf(floorf(p), -lim), lim);
  int gg = c + __float2int_rz(s);
  float ff = p - s;
  const bool trunc = (gg < 0) & (ff != 0.0f);
  g = trunc ? gg + 1 : gg;
  f = trunc ? ff - 1.0f : ff;
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
__device__ __forceinline__ void advance(int &c, float &o, float disp, int N) {
  const float lim = (float)(N + 8);
  const float p = o + disp;
  const float s = fminf(fmaxf(floorf(p), -lim), lim);
  c += __float2int_rz(s);
  o = p - s;
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

// Trilinear gather of E and B at (cell g, fraction f) per axis from the staged
// tile. Every lane reads the tile (indices clamped into it); lanes whose 8
// nodes lie outside the tile then re-gather from HBM/L2, a warp-uniform branch
// that is skipped when no lane needs it. All 32 lanes must call.
template <int TX, int TY, int TZ>
__device__ __forceinline__ Field6 gather(const CycleParams &P, const float *__restrict__ sF,
                                         int c0x, int c0y, int c0z, int gx, int gy, int gz,
                                         float fx, float fy, float fz) {
  using T = Tile<TX, TY, TZ>;
  const float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
  Field6 F = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  const int bx = gx + 1 - c0x, by = gy + 1 - c0y, bz = gz + 1 - c0z;
  const bool inbox = ((unsigned)bx <= (unsigned)(TX + 1)) & ((unsigned)by <= (unsigned)(TY + 1)) &
                     ((unsigned)bz <= (unsigned)(TZ + 1));
  {
    const int n0 = (min(max(bx, 0), TX + 1) * T::BY + min(max(by, 0), TY + 1)) * T::BZ +
                   min(max(bz, 0), TZ + 1);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b) {
        const float wab = wx[a] * wy[b];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int n = n0 + (a * T::BY + b) * T::BZ + c;
          const float4 A = *reinterpret_cast<const float4 *>(sF + 8 * n);
          const float2 B = *reinterpret_cast<const float2 *>(sF + 8 * n + 4);
          acc_node(F, wab * wz[c], A, B);
        }
      }
  }
  if (__any_sync(0xffffffffu, !inbox)) {
    if (!inbox) {
      F = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
      const long sy = P.nzn, sx = (long)P.nyn * P.nzn;
      const int hx = min(max(gx, -1), P.nxc), hy = min(max(gy, -1), P.nyc),
                hz = min(max(gz, -1), P.nzc);
      const long n0 = (long)(hx + 1) * sx + (long)(hy + 1) * sy + (hz + 1);
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          const float wab = wx[a] * wy[b];
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const long n = n0 + a * sx + b * sy + c;
            const float4 A = __ldg(reinterpret_cast<const float4 *>(P.fields8 + 8 * n));
            const float2 B = __ldg(reinterpret_cast<const float2 *>(P.fields8 + 8 * n + 4));
            acc_node(F, wab * wz[c], A, B);
          }
        }
    }
  }
  return F;
}

// mover_PC for one particle in cell units (src/Mover.cpp:33-157). All 32 lanes
// of the warp must call (the gather votes).
template <int TX, int TY, int TZ>
__device__ __forceinline__ void push(const CycleParams &P, const float *__restrict__ sF, int c0x,
                                     int c0y, int c0z, float qomdt2, int &cx, int &cy, int &cz,
                                     float &ox, float &oy, float &oz, float &u, float &v, float &w,
                                     int &bad) {
  float dx = 0.f, dy = 0.f, dz = 0.f;   // predicted displacement in cells
  float up = 0.f, vp = 0.f, wp = 0.f;
#pragma unroll 1
  for (int it = 0; it < P.niter; ++it) {
    int gx = cx, gy = cy, gz = cz;
    float fx = ox, fy = oy, fz = oz;
    if (it > 0) {   // the first gather is at the start position: (c, o) as stored
      locate(ox + dx, cx, P.nxc, gx, fx);
      locate(oy + dy, cy, P.nyc, gy, fy);
      locate(oz + dz, cz, P.nzc, gz, fz);
    }
    const Field6 F = gather<TX, TY, TZ>(P, sF, c0x, c0y, c0z, gx, gy, gz, fx, fy, fz);
    const float ex = F.exy.x, ey = F.exy.y, ez = F.ezbx.x;
    const float bx = F.ezbx.y, by = F.byz.x, bz = F.byz.y;
    const float omdtsq = qomdt2 * qomdt2 * (bx * bx + by * by + bz * bz);
    const float denom = __fdividef(1.0f, 1.0f + omdtsq);
    const float ut = fmaf(qomdt2, ex, u);
    const float vt = fmaf(qomdt2, ey, v);
    const float wt = fmaf(qomdt2, ez, w);
    const float qud = qomdt2 * (ut * bx + vt * by + wt * bz);
    up = fmaf(qomdt2, vt * bz - wt * by + qud * bx, ut) * denom;
    vp = fmaf(qomdt2, wt * bx - ut * bz + qud * by, vt) * denom;
    wp = fmaf(qomdt2, ut * by - vt * bx + qud * bz, wt) * denom;
    dx = up * P.hdt[0];
    dy = vp * P.hdt[1];
    dz = wp * P.hdt[2];
  }
  u = 2.0f * up - u;
  v = 2.0f * vp - v;
  w = 2.0f * wp - w;
  advance(cx, ox, up * P.fdt[0], P.nxc);
  advance(cy, oy, vp * P.fdt[1], P.nyc);
  advance(cz, oz, wp * P.fdt[2], P.nzc);
  bc_cell(cx, ox, u, P.nxc, P.periodic[0]);
  bc_cell(cy, oy, v, P.nyc, P.periodic[1]);
  bc_cell(cz, oz, w, P.nzc, P.periodic[2]);
  bad |= (cx < 0) | (cx >= P.nxc) | (cy < 0) | (cy >= P.nyc) | (cz < 0) | (cz >= P.nzc);
  cx = min(max(cx, 0), P.nxc - 1);
  cy = min(max(cy, 0), P.nyc - 1);
  cz = min(max(cz, 0), P.nzc - 1);
}

// Deposit terms of one particle added to 40 packed accumulators:
// acc[node*5 + k] += W_node * (mf[k], mf[k+5]) with the moment factors
// mf = 1, u, v, w, uu | uv, uw, vv, vw, ww, i.e. the pairs (1,uv) (u,uw)
// (v,vv) (w,vw) (uu,ww). node = a*4 + b*2 + c, a/b/c = 1 the upper node on
// that axis, XOR-permuted by lane bits 4/3/2 (see warp_sum80). q is folded
// into the x weights; q = 0 adds nothing.
__device__ __forceinline__ void add_terms(float2 (&acc)[40], float q, float ox, float oy, float oz,
                                          float u, float v, float w, int lane) {
  const bool px = lane & 16, py = lane & 8, pz = lane & 4;
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

__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
  return make_float2(__shfl_xor_sync(FULL, v.x, m), __shfl_xor_sync(FULL, v.y, m));
}

// Sums the packed accumulators over the warp. Lanes hold their terms with
// the x/y/z node halves swapped by lane bits 4/3/2, so the first three
// halving steps need no selects: every lane keeps its lower half and
// receives its partner's upper half. Afterwards lane l holds in r[0..4] the
// totals of node (a, b, c) = (bit4, bit3, bit2) of l, moments
// 5*bit1(l) .. 5*bit1(l)+4 (reference order).
__device__ __forceinline__ void warp_sum80(float2 (&acc)[40], float (&r)[5], int lane) {
#pragma unroll
  for (int i = 0; i < 20; ++i) acc[i] = __fadd2_rn(acc[i], shfl_xor2(acc[i + 20], 16));
#pragma unroll
  for (int i = 0; i < 10; ++i) acc[i] = __fadd2_rn(acc[i], shfl_xor2(acc[i + 10], 8));
#pragma unroll
  for (int i = 0; i < 5; ++i) acc[i] = __fadd2_rn(acc[i], shfl_xor2(acc[i + 5], 4));
  const bool h = lane & 2;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const float send = h ? acc[k].x : acc[k].y;
    const float keep = h ? acc[k].y : acc[k].x;
    r[k] = keep + __shfl_xor_sync(FULL, send, 2);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) r[k] += __shfl_xor_sync(FULL, r[k], 1);
}

struct MoverEntry {  // one queued deposit: final cell and state
  uint32_t cell;
  float ox, oy, oz, q, u, v, w;
};

// Tile partials are 64-bit fixed point: a term t is added as
// round(t * fix), fix = 2^40 / max|q| (a power of two, so the scaling is
// exact). Integer shared-memory atomics are native and do not retry under
// contention, unlike float ones; the sums are exact, so their order does not
// matter. |t * fix| beyond 2^62 (|velocity| in the thousands) is flagged.
__device__ __forceinline__ void add_fixed(unsigned long long *a, float t, float fix, int &bad) {
  const float x = t * fix;
  bad |= !(fabsf(x) < 4.0e18f);
  atomicAdd(a, (unsigned long long)__float2ll_rn(fminf(fmaxf(x, -4.0e18f), 4.0e18f)));
}

// Deposit of one queued particle per lane with shared-memory atomics (inside
// the staged box) or FP64 global atomics (outside it; a warp-uniform branch
// skipped when no lane needs it). All 32 lanes call; `active` lanes deposit.
template <int TX, int TY, int TZ>
__device__ __forceinline__ void deposit_scatter(const CycleParams &P, const SpeciesDev &S,
                                                unsigned long long *__restrict__ sAcc, int c0x,
                                                int c0y, int c0z, const MoverEntry &e,
                                                bool active, int &bad) {
  using T = Tile<TX, TY, TZ>;
  const int cx = cell_x(e.cell), cy = cell_y(e.cell), cz = cell_z(e.cell);
  const float wx[2] = {e.q * (1.0f - e.ox), e.q * e.ox};
  const float wy[2] = {1.0f - e.oy, e.oy}, wz[2] = {1.0f - e.oz, e.oz};
  const float mf[10] = {1.0f,      e.u,       e.v,       e.w,       e.u * e.u,
                        e.u * e.v, e.u * e.w, e.v * e.v, e.v * e.w, e.w * e.w};
  const int bx = cx + 1 - c0x, by = cy + 1 - c0y, bz = cz + 1 - c0z;
  const bool inbox = ((unsigned)bx <= (unsigned)(TX + 1)) & ((unsigned)by <= (unsigned)(TY + 1)) &
                     ((unsigned)bz <= (unsigned)(TZ + 1));
  if (active & inbox) {
    const int n0 = (bx * T::BY + by) * T::BZ + bz;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const float W = wx[a] * wy[b] * wz[c];
          const int n = n0 + (a * T::BY + b) * T::BZ + c;
#pragma unroll
          for (int m = 0; m < 10; ++m) add_fixed(sAcc + m * T::BN + n, W * mf[m], S.fix, bad);
        }
  }
  if (__any_sync(0xffffffffu, active & !inbox)) {
    if (active & !inbox) {
      const long nodes = (long)P.nxn * P.nyn * P.nzn;
      const long sy = P.nzn, sx = (long)P.nyn * P.nzn;
      const long n0 = (long)(cx + 1) * sx + (long)(cy + 1) * sy + (cz + 1);
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const double W = (double)(wx[a] * wy[b] * wz[c]) * P.scale;
            const long n = n0 + a * sx + b * sy + c;
#pragma unroll
            for (int m = 0; m < 10; ++m) atomicAdd(S.mom + m * nodes + n, W * (double)mf[m]);
          }
    }
  }
}

// Adds the warp totals of the segment cell's 8 nodes into the tile partials.
template <int TX, int TY, int TZ>
__device__ __forceinline__ void flush_cell(float2 (&acc)[40], unsigned long long *__restrict__ sAcc,
                                           int lx, int ly, int lz, int lane, float fix, int &bad) {
  using T = Tile<TX, TY, TZ>;
  float r[5];
  warp_sum80(acc, r, lane);
  const int a = (lane >> 4) & 1, bb = (lane >> 3) & 1, c = (lane >> 2) & 1;
  const int mbase = 5 * ((lane >> 1) & 1);
  const int n = ((lx + 1 + a) * T::BY + (ly + 1 + bb)) * T::BZ + (lz + 1 + c);
  const int lo = (lane & 1) ? 3 : 0, hi = (lane & 1) ? 5 : 3;
#pragma unroll
  for (int k = 0; k < 5; ++k)
    if (k >= lo && k < hi) add_fixed(sAcc + (mbase + k) * T::BN + n, r[k], fix, bad);
}

// ACC = true: each lane accumulates the terms of all its particles of a cell
// in registers and the warp sums once per cell. ACC = false: the warp sums
// after every 32 particles (fewer live registers, more occupancy).
template <int TX, int TY, int TZ, bool ACC>
__global__ void __launch_bounds__(SIM_TPB, ACC ? 1 : 2)
    k_cycle(const __grid_constant__ CUtensorMap fmap, const __grid_constant__ CycleParams P) {
  using T = Tile<TX, TY, TZ>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float *sF0 = reinterpret_cast<float *>(smem_raw);                 // 2 stages x SF
  unsigned long long *sAcc =
      reinterpret_cast<unsigned long long *>(sF0 + 2 * T::SF);      // 10 * BN fixed point
  MoverEntry *sQ = reinterpret_cast<MoverEntry *>(sAcc + 10 * T::BN);  // NW * QCAP
  uint64_t *bar = reinterpret_cast<uint64_t *>(sQ + SIM_NW * QCAP);   // 2 barriers

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  MoverEntry *myQ = sQ + warp * QCAP;
  if (smem_addr(sF0) & 127u) {   // TMA destinations need 128-byte alignment
    if (tid == 0) atomicOr(P.err, 8);
    return;
  }
  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_init(bar + 1, 1);
  }
  for (int i = tid; i < 10 * T::BN; i += SIM_TPB) sAcc[i] = 0ull;
  __syncthreads();

  const int ntiles = P.ntx * P.nty * P.ntz;
  const long nodes = (long)P.nxn * P.nyn * P.nzn;
  const unsigned box_bytes = (unsigned)(T::BN * 8 * sizeof(float));
  auto issue = [&](int t, int stage) {
    const int z = t % P.ntz, y = (t / P.ntz) % P.nty, x = t / (P.ntz * P.nty);
    fence_proxy_async();
    mbar_expect_tx(bar + stage, box_bytes);
    // box origin: node c0 on every axis (the lower node of halo cell c0-1)
    tma_load_4d(sF0 + stage * T::SF, &fmap, 0, z * TZ, y * TY, x * TX, bar + stage);
  };
  if (tid == 0 && blockIdx.x < ntiles) issue(blockIdx.x, 0);
  int bad = 0, it = 0;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
    const int stage = it & 1;
    // prefetch the next tile's fields into the other stage (read by the
    // previous tile, which every thread finished before the last barrier)
    if (tid == 0 && tile + (int)gridDim.x < ntiles) issue(tile + gridDim.x, stage ^ 1);
    if (!mbar_wait_bounded(bar + stage, (it >> 1) & 1)) {
      // the staged fields never arrived: report, wait once more, give up
      if (tid == 0) atomicOr(P.err, 2);
      mbar_wait_bounded(bar + stage, (it >> 1) & 1);
      mbar_wait_bounded(bar + (stage ^ 1), ((it + 1) >> 1) & 1);
      return;
    }
    const float *sF = sF0 + stage * T::SF;
    const int tz = tile % P.ntz, ty = (tile / P.ntz) % P.nty, tx = tile / (P.ntz * P.nty);
    const int c0x = tx * TX, c0y = ty * TY, c0z = tz * TZ;

    for (int s = 0; s < P.ns; ++s) {
      const SpeciesDev S = P.sp[s];
      const float qomdt2 = S.qomdt2;
      int qcount = 0;
      for (int lc = warp; lc < T::TC; lc += SIM_NW) {
        const long key = (long)tile * T::TC + lc;
        const int b = (int)min((long)S.cell_start[key], S.n);
        const int e = (int)min((long)S.cell_start[key + 1], S.n);
        if (b >= e) continue;
        const int lx = lc / (TY * TZ), ly = (lc / TZ) % TY, lz = lc % TZ;
        const uint32_t seg = pack_cell(c0x + lx, c0y + ly, c0z + lz);
        float2 acc[40];
        if (ACC) {
#pragma unroll
          for (int i = 0; i < 40; ++i) acc[i] = make_float2(0.f, 0.f);
        }
#pragma unroll 1
        for (int base = b; base < e; base += 32) {
          const int i = base + lane;
          const bool valid = i < e;
          // idle lanes of the last slot push a copy of the cell's last particle
          // (results discarded), so the whole warp runs one instruction stream
          const int ii = valid ? i : e - 1;
          uint32_t cell = S.cell[ii];
          float ox = S.ox[ii], oy = S.oy[ii], oz = S.oz[ii];
          float u = S.u[ii], v = S.v[ii], w = S.w[ii];
          const float q = valid ? S.q[ii] : 0.0f;
          {
            int cx = cell_x(cell), cy = cell_y(cell), cz = cell_z(cell);
            int pbad = 0;
            push<TX, TY, TZ>(P, sF, c0x, c0y, c0z, qomdt2, cx, cy, cz, ox, oy, oz, u, v, w, pbad);
            bad |= valid ? pbad : 0;
            cell = pack_cell(cx, cy, cz);
          }
          __syncwarp();
          if (valid) {
            S.cell[i] = cell;
            S.ox[i] = ox;
            S.oy[i] = oy;
            S.oz[i] = oz;
            S.u[i] = u;
            S.v[i] = v;
            S.w[i] = w;
          }
          const bool mover = valid & (cell != seg);
          // particles that stay in the segment cell: register terms
          if (!ACC) {
#pragma unroll
            for (int k = 0; k < 40; ++k) acc[k] = make_float2(0.f, 0.f);
          }
          add_terms(acc, mover ? 0.0f : q, ox, oy, oz, u, v, w, lane);
          if (!ACC) flush_cell<TX, TY, TZ>(acc, sAcc, lx, ly, lz, lane, S.fix, bad);
          // particles that changed cell: per-warp queue, shared atomics
          const unsigned mb = __ballot_sync(FULL, mover);
          if (mb) {
            if (mover) {
              const int slot = qcount + __popc(mb & ((1u << lane) - 1u));
              myQ[slot] = MoverEntry{cell, ox, oy, oz, q, u, v, w};
            }
            qcount += __popc(mb);
            __syncwarp();
            if (qcount >= 32) {
              deposit_scatter<TX, TY, TZ>(P, S, sAcc, c0x, c0y, c0z, myQ[lane], true, bad);
              __syncwarp();
              if (lane < qcount - 32) myQ[lane] = myQ[32 + lane];
              qcount -= 32;
              __syncwarp();
            }
          }
        }
        if (ACC) flush_cell<TX, TY, TZ>(acc, sAcc, lx, ly, lz, lane, S.fix, bad);
      }
      // remaining queued movers of this warp
      if (qcount > 0)
        deposit_scatter<TX, TY, TZ>(P, S, sAcc, c0x, c0y, c0z, myQ[lane], lane < qcount, bad);
      __syncthreads();
      // flush the tile's partials into the FP64 moments, and clear them
      for (int i = tid; i < 10 * T::BN; i += SIM_TPB) {
        const long long val = (long long)sAcc[i];
        if (val != 0) {
          const int m = i / T::BN, n = i % T::BN;
          const int bz = n % T::BZ, by = (n / T::BZ) % T::BY, bx = n / (T::BZ * T::BY);
          const long g = ((long)(c0x + bx) * P.nyn + (c0y + by)) * P.nzn + (c0z + bz);
          atomicAdd(S.mom + m * nodes + g, (double)val * S.unfix);
          sAcc[i] = 0ull;
        }
      }
      __syncthreads();
    }
  }
  if (bad) atomicOr(P.err, ERRBIT_OUT_OF_GRID);
}

// ---------------------------------------------------------------------------
// conversion, sort, field packing, readback
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

__global__ void k_load(GridScalars g, const float *__restrict__ x, const float *__restrict__ y,
                       const float *__restrict__ z, const float *__restrict__ u,
                       const float *__restrict__ v, const float *__restrict__ w,
                       const float *__restrict__ q, long n, uint32_t *cell, float *ox, float *oy,
                       float *oz, float *uo, float *vo, float *wo, float *qo, int *err) {
  int bad = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    int cx, cy, cz;
    float a, b, c;
    to_cell(x[i], g.invdx, g.nxc, cx, a, bad);
    to_cell(y[i], g.invdy, g.nyc, cy, b, bad);
    to_cell(z[i], g.invdz, g.nzc, cz, c, bad);
    cell[i] = pack_cell(cx, cy, cz);
    ox[i] = a;
    oy[i] = b;
    oz[i] = c;
    uo[i] = u[i];
    vo[i] = v[i];
    wo[i] = w[i];
    qo[i] = q[i];
  }
  if (bad) atomicOr(err, ERRBIT_OUT_OF_GRID);
}

// max |q| as the bit pattern of a non-negative float (ordered like an int)
__global__ void k_absmax(const float *__restrict__ q, long n, unsigned *__restrict__ out) {
  float m = 0.0f;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x)
    m = fmaxf(m, fabsf(q[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(FULL, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

__global__ void k_unload(GridScalars g, const uint32_t *__restrict__ cell,
                         const float *__restrict__ ox, const float *__restrict__ oy,
                         const float *__restrict__ oz, const float *__restrict__ u,
                         const float *__restrict__ v, const float *__restrict__ w,
                         const float *__restrict__ q, long n, float *x, float *y, float *z,
                         float *uo, float *vo, float *wo, float *qo) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const uint32_t c = cell[i];
    x[i] = (float)(((double)cell_x(c) + (double)ox[i]) * g.dx);
    y[i] = (float)(((double)cell_y(c) + (double)oy[i]) * g.dy);
    z[i] = (float)(((double)cell_z(c) + (double)oz[i]) * g.dz);
    uo[i] = u[i];
    vo[i] = v[i];
    wo[i] = w[i];
    if (qo) qo[i] = q[i];
  }
}

template <int TX, int TY, int TZ>
__global__ void k_sort_count(const uint32_t *__restrict__ cell, long n, int nty, int ntz,
                             int *__restrict__ count) {
  const int lane = threadIdx.x & 31;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const uint32_t c = cell[i];
    const int key = tile_key<TX, TY, TZ>(cell_x(c), cell_y(c), cell_z(c), nty, ntz);
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, key);
    if (lane == __ffs(peers) - 1) atomicAdd(count + key, __popc(peers));
  }
}

template <int TX, int TY, int TZ>
__global__ void k_sort_scatter(const uint32_t *__restrict__ cell, const float *__restrict__ ox,
                               const float *__restrict__ oy, const float *__restrict__ oz,
                               const float *__restrict__ u, const float *__restrict__ v,
                               const float *__restrict__ w, const float *__restrict__ q, long n,
                               int nty, int ntz, int *__restrict__ cursor, uint32_t *cell2,
                               float *ox2, float *oy2, float *oz2, float *u2, float *v2, float *w2,
                               float *q2, int *err) {
  const int lane = threadIdx.x & 31;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const uint32_t c = cell[i];
    const int key = tile_key<TX, TY, TZ>(cell_x(c), cell_y(c), cell_z(c), nty, ntz);
    const unsigned active = __activemask();
    const unsigned peers = __match_any_sync(active, key);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(cursor + key, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    const long d = base + __popc(peers & ((1u << lane) - 1u));
    if (d < 0 || d >= n) {   // only reachable if the counts were corrupted
      atomicOr(err, 4);
      continue;
    }
    cell2[d] = c;
    ox2[d] = ox[i];
    oy2[d] = oy[i];
    oz2[d] = oz[i];
    u2[d] = u[i];
    v2[d] = v[i];
    w2[d] = w[i];
    q2[d] = q[i];
  }
}

// Exclusive scan of `count` (k entries) into out[0..k]; three passes.
constexpr int SCAN_B = 1024;
__device__ __forceinline__ int block_exclusive_scan(int v, int *warp_sums, int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(FULL, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) warp_sums[lane] = s;
  }
  __syncthreads();
  const int pre = warp ? warp_sums[warp - 1] : 0;
  total = warp_sums[nw - 1];
  __syncthreads();
  return pre + x - v;
}

__global__ void __launch_bounds__(SCAN_B) k_scan_blocks(const int *in, long k, int *out,
                                                        int *block_sums) {
  __shared__ int ws[32];
  const long i = blockIdx.x * (long)SCAN_B + threadIdx.x;
  const int v = i < k ? in[i] : 0;
  int total;
  const int ex = block_exclusive_scan(v, ws, total);
  if (i < k) out[i] = ex;
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(SCAN_B) k_scan_sums(int *block_sums, int nb, int *grand) {
  __shared__ int ws[32];
  int carry = 0;
  for (int base = 0; base < nb; base += SCAN_B) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? block_sums[i] : 0;
    int total;
    const int ex = block_exclusive_scan(v, ws, total);
    if (i < nb) block_sums[i] = ex + carry;
    carry += total;
  }
  if (threadIdx.x == 0) *grand = carry;
}

__global__ void __launch_bounds__(SCAN_B) k_scan_add(int *out, long k, const int *block_sums) {
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

struct SimSpecies {
  long n = 0, cap = 0;
  double qom = 0;
  float fix = 1.0f;     // fixed-point scale of the tile partials (2^40 / max|q|)
  uint32_t *cell[2] = {};
  float *f[2][7] = {};   // ox oy oz u v w q, double-buffered for the sort
  int cur = 0;
  int *cell_start = nullptr;   // [ncells + 1]
  double *mom = nullptr;       // [10][nodes]
  bool sorted = false;
};

using LaunchFn = int (*)(spb_sim *, cudaStream_t);

}  // namespace

struct spb_sim {
  spb_sim_desc d{};
  int device = 0;
  int N[3] = {0, 0, 0};
  int tile[3] = {8, 4, 4};
  int nt[3] = {0, 0, 0};
  long ncells = 0, nodes = 0;
  int nxn = 0, nyn = 0, nzn = 0;
  double dxyz[3] = {0, 0, 0};
  float *fields8 = nullptr;
  float *stage = nullptr;       // 6*nodes for host field uploads
  int *d_err = nullptr;
  int *scan_tmp = nullptr;      // block sums + grand total
  int *counts = nullptr;        // [ncells]
  int *cursor = nullptr;        // [ncells + 1]
  CUtensorMap fmap{};
  bool fields_set = false;
  int cycles_since_sort = 0;
  int grid_ctas = 0;
  std::vector<SimSpecies> sp;
  long launches = 0;
  std::mutex mu;
  // optional CUDA-event timing of the cycle kernel and of the sorts
  bool timing = false;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev_cycle, ev_sort;
};

namespace {

// Records an event pair around a launch when timing is on.
struct Timed {
  spb_sim *s;
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> *v;
  cudaStream_t st;
  cudaEvent_t b = nullptr;
  Timed(spb_sim *s_, std::vector<std::pair<cudaEvent_t, cudaEvent_t>> *v_, cudaStream_t st_)
      : s(s_), v(v_), st(st_) {
    if (s->timing && cudaEventCreate(&b) == cudaSuccess) cudaEventRecord(b, st);
  }
  ~Timed() {
    cudaEvent_t e = nullptr;
    if (b && cudaEventCreate(&e) == cudaSuccess) {
      cudaEventRecord(e, st);
      v->push_back({b, e});
    }
  }
};

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

template <int TX, int TY, int TZ>
size_t cycle_smem() {
  using T = Tile<TX, TY, TZ>;
  return 2 * (size_t)T::SF * 4 + (size_t)T::BN * 10 * 8 +
         (size_t)SIM_NW * QCAP * sizeof(MoverEntry) + 16;
}

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
    D.cell = q.cell[q.cur];
    D.ox = q.f[q.cur][0];
    D.oy = q.f[q.cur][1];
    D.oz = q.f[q.cur][2];
    D.u = q.f[q.cur][3];
    D.v = q.f[q.cur][4];
    D.w = q.f[q.cur][5];
    D.q = q.f[q.cur][6];
    D.cell_start = q.cell_start;
    D.mom = q.mom;
    D.n = q.n;
    D.qomdt2 = (float)(q.qom * (0.5 * s->d.dt) / s->d.c);
    D.fix = q.fix;
    D.unfix = P.scale / (double)q.fix;
  }
  return P;
}

template <int TX, int TY, int TZ, bool ACC>
int launch_cycle_v(spb_sim *s, cudaStream_t st) {
  const size_t smem = cycle_smem<TX, TY, TZ>();
  static bool attr = false;
  if (!attr) {
    SPB_CUDA(cudaFuncSetAttribute(k_cycle<TX, TY, TZ, ACC>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  const CycleParams P = make_params(s);
  const int ntiles = s->nt[0] * s->nt[1] * s->nt[2];
  const int per_sm = ACC ? 1 : 2;
  const int ctas = std::min(ntiles, s->grid_ctas > 0 ? s->grid_ctas : per_sm * num_sms());
  Timed tm(s, &s->ev_cycle, st);
  k_cycle<TX, TY, TZ, ACC><<<ctas, SIM_TPB, smem, st>>>(s->fmap, P);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  s->launches++;
  return SPB_OK;
}

template <int TX, int TY, int TZ>
int launch_cycle(spb_sim *s, cudaStream_t st) {
  return s->d.variant == 1 ? launch_cycle_v<TX, TY, TZ, false>(s, st)
                           : launch_cycle_v<TX, TY, TZ, true>(s, st);
}

template <int TX, int TY, int TZ>
int launch_sort(spb_sim *s, SimSpecies &q, cudaStream_t st) {
  const long K = s->ncells;
  Timed tm(s, &s->ev_sort, st);
  SPB_CUDA(cudaMemsetAsync(s->counts, 0, K * sizeof(int), st));
  const int tpb = 256;
  k_sort_count<TX, TY, TZ><<<blocks_for(q.n, tpb), tpb, 0, st>>>(q.cell[q.cur], q.n, s->nt[1],
                                                                 s->nt[2], s->counts);
  SPB_CUDA(cudaGetLastError());
  const int nb = (int)ceil_div(K, SCAN_B);
  k_scan_blocks<<<nb, SCAN_B, 0, st>>>(s->counts, K, q.cell_start, s->scan_tmp);
  k_scan_sums<<<1, SCAN_B, 0, st>>>(s->scan_tmp, nb, q.cell_start + K);
  k_scan_add<<<nb, SCAN_B, 0, st>>>(q.cell_start, K, s->scan_tmp);
  SPB_CUDA(cudaGetLastError());
  SPB_CUDA(cudaMemcpyAsync(s->cursor, q.cell_start, (K + 1) * sizeof(int),
                           cudaMemcpyDeviceToDevice, st));
  const int src = q.cur, dst = 1 - q.cur;
  k_sort_scatter<TX, TY, TZ><<<blocks_for(q.n, tpb), tpb, 0, st>>>(
      q.cell[src], q.f[src][0], q.f[src][1], q.f[src][2], q.f[src][3], q.f[src][4], q.f[src][5],
      q.f[src][6], q.n, s->nt[1], s->nt[2], s->cursor, q.cell[dst], q.f[dst][0], q.f[dst][1],
      q.f[dst][2], q.f[dst][3], q.f[dst][4], q.f[dst][5], q.f[dst][6], s->d_err);
  SPB_CUDA(cudaGetLastError());
  g_launches += 5;
  s->launches += 5;
  q.cur = dst;
  q.sorted = true;
  return SPB_OK;
}

// Tile shapes the kernels are instantiated for.
struct TileImpl {
  int t[3];
  int (*cycle)(spb_sim *, cudaStream_t);
  int (*sort)(spb_sim *, SimSpecies &, cudaStream_t);
  size_t (*smem)();
};

#define SPB_TILE(X, Y, Z) \
  TileImpl { {X, Y, Z}, launch_cycle<X, Y, Z>, launch_sort<X, Y, Z>, cycle_smem<X, Y, Z> }
const TileImpl kTiles[] = {SPB_TILE(8, 4, 4), SPB_TILE(4, 4, 4), SPB_TILE(2, 2, 2),
                           SPB_TILE(8, 8, 4)};
#undef SPB_TILE

const TileImpl *find_tile(const int t[3]) {
  for (const TileImpl &ti : kTiles)
    if (ti.t[0] == t[0] && ti.t[1] == t[1] && ti.t[2] == t[2]) return &ti;
  return nullptr;
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

void free_species(SimSpecies &q) {
  for (int b = 0; b < 2; ++b) {
    cudaFree(q.cell[b]);
    q.cell[b] = nullptr;
    for (float *&p : q.f[b]) {
      cudaFree(p);
      p = nullptr;
    }
  }
  cudaFree(q.cell_start);
  cudaFree(q.mom);
  q.cell_start = nullptr;
  q.mom = nullptr;
}

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
  if (d->niter < 1 || !(d->dt > 0) || !(d->c != 0))
    return fail(SPB_ERR_INVALID, "spb_sim_create: bad NiterMover, dt or c");
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
  s->grid_ctas = d->ctas;
  auto bail = [&](int rc) {
    spb_sim_destroy(s);
    return rc;
  };
  const long nb = ceil_div(s->ncells, SCAN_B);
  if (cudaMalloc(&s->fields8, s->nodes * 8 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&s->d_err, sizeof(int)) != cudaSuccess ||
      cudaMalloc(&s->scan_tmp, (nb + 1) * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&s->counts, s->ncells * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&s->cursor, (s->ncells + 1) * sizeof(int)) != cudaSuccess) {
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
    if (cudaMalloc(&q.cell_start, (s->ncells + 1) * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&q.mom, 10 * s->nodes * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return bail(fail(SPB_ERR_ALLOC, "spb_sim_create: device allocation failed"));
    }
    if (cudaMemset(q.mom, 0, 10 * s->nodes * sizeof(double)) != cudaSuccess ||
        cudaMemset(q.cell_start, 0, (s->ncells + 1) * sizeof(int)) != cudaSuccess)
      return bail(fail(SPB_ERR_CUDA, "spb_sim_create: memset failed"));
    if (d->capacity[i] > 0) {
      // reserve now so that later loads allocate nothing
      q.cap = 0;
    }
  }
  *out = s;
  return SPB_OK;
}

namespace {
double drain(std::vector<std::pair<cudaEvent_t, cudaEvent_t>> &v, int *count) {
  double ms = 0;
  for (auto &p : v) {
    float t = 0;
    if (cudaEventSynchronize(p.second) == cudaSuccess &&
        cudaEventElapsedTime(&t, p.first, p.second) == cudaSuccess)
      ms += t;
    cudaEventDestroy(p.first);
    cudaEventDestroy(p.second);
  }
  if (count) *count = (int)v.size();
  v.clear();
  return ms;
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
  const double c = drain(s->ev_cycle, ncycle), o = drain(s->ev_sort, nsort);
  if (cycle_ms) *cycle_ms = c;
  if (sort_ms) *sort_ms = o;
  return SPB_OK;
}

extern "C" void spb_sim_destroy(spb_sim *s) {
  if (!s) return;
  drain(s->ev_cycle, nullptr);
  drain(s->ev_sort, nullptr);
  for (auto &q : s->sp) free_species(q);
  cudaFree(s->fields8);
  cudaFree(s->stage);
  cudaFree(s->d_err);
  cudaFree(s->scan_tmp);
  cudaFree(s->counts);
  cudaFree(s->cursor);
  delete s;
}

extern "C" long spb_sim_nodes(const spb_sim *s) { return s ? s->nodes : 0; }
extern "C" long spb_sim_count(const spb_sim *s, int species) {
  if (!s || species < 0 || species >= (int)s->sp.size()) return -1;
  return s->sp[species].n;
}
extern "C" long spb_sim_launches(const spb_sim *s) { return s ? s->launches : 0; }

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
    if (!s->stage && cudaMalloc(&s->stage, 6 * s->nodes * sizeof(float)) != cudaSuccess) {
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
  SimSpecies &S = s->sp[species];
  // capacity: padded to whole 128-particle chunks plus one spare chunk, so the
  // 128-bit reads of a cell's last chunk stay inside the allocation
  const long cap = (ceil_div(std::max<long>(n, 1), 128) + 1) * 128;
  if (cap > S.cap) {
    for (int b = 0; b < 2; ++b) {
      cudaFree(S.cell[b]);
      S.cell[b] = nullptr;
      for (float *&p : S.f[b]) {
        cudaFree(p);
        p = nullptr;
      }
    }
    S.cap = 0;
    for (int b = 0; b < 2; ++b) {
      if (cudaMalloc(&S.cell[b], cap * sizeof(uint32_t)) != cudaSuccess) {
        cudaGetLastError();
        return fail(SPB_ERR_ALLOC, "spb_sim_load_species: allocation failed");
      }
      SPB_CUDA(cudaMemsetAsync(S.cell[b], 0, cap * sizeof(uint32_t), st));
      for (float *&p : S.f[b]) {
        if (cudaMalloc(&p, cap * sizeof(float)) != cudaSuccess) {
          cudaGetLastError();
          return fail(SPB_ERR_ALLOC, "spb_sim_load_species: allocation failed");
        }
        SPB_CUDA(cudaMemsetAsync(p, 0, cap * sizeof(float), st));
      }
    }
    S.cap = cap;
  }
  S.n = n;
  S.cur = 0;
  const float *src[7] = {x, y, z, u, v, w, q};
  float *tmp = nullptr;
  if (!on_device && n > 0) {
    // stage through the second buffer set
    for (int a = 0; a < 7; ++a) {
      SPB_CUDA(cudaMemcpyAsync(S.f[1][a], src[a], n * sizeof(float), cudaMemcpyHostToDevice, st));
      src[a] = S.f[1][a];
    }
  }
  (void)tmp;
  if (n > 0) {
    k_load<<<blocks_for(n, 256), 256, 0, st>>>(scalars(s), src[0], src[1], src[2], src[3], src[4],
                                               src[5], src[6], n, S.cell[0], S.f[0][0], S.f[0][1],
                                               S.f[0][2], S.f[0][3], S.f[0][4], S.f[0][5],
                                               S.f[0][6], s->d_err);
    SPB_CUDA(cudaGetLastError());
    g_launches++;
    s->launches++;
  }
  // fixed-point scale of the tile partials from max |q| (q never changes)
  S.fix = 1.0f;
  if (n > 0) {
    unsigned *d_max = reinterpret_cast<unsigned *>(s->scan_tmp);
    SPB_CUDA(cudaMemsetAsync(d_max, 0, sizeof(unsigned), st));
    k_absmax<<<blocks_for(n, 256), 256, 0, st>>>(S.f[0][6], n, d_max);
    SPB_CUDA(cudaGetLastError());
    g_launches++;
    s->launches++;
    unsigned h = 0;
    SPB_CUDA(cudaMemcpyAsync(&h, d_max, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    SPB_CUDA(cudaStreamSynchronize(st));
    float qmax;
    std::memcpy(&qmax, &h, sizeof(float));
    if (qmax > 0.0f && std::isfinite(qmax)) {
      int e;
      std::frexp(qmax, &e);                   // qmax < 2^e
      S.fix = std::ldexp(1.0f, 40 - e);      // |q| * fix < 2^40
    }
  }
  const TileImpl *ti = find_tile(s->tile);
  if (int rc = ti->sort(s, S, st)) return rc;
  s->cycles_since_sort = 0;
  return SPB_OK;
}

extern "C" int spb_sim_resort(spb_sim *s, void *stream) {
  if (!s) return fail(SPB_ERR_INVALID, "spb_sim_resort: null simulation");
  const TileImpl *ti = find_tile(s->tile);
  for (auto &q : s->sp)
    if (q.n > 0)
      if (int rc = ti->sort(s, q, (cudaStream_t)stream)) return rc;
  s->cycles_since_sort = 0;
  return SPB_OK;
}

extern "C" int spb_sim_cycle(spb_sim *s, int ncycles, void *stream) {
  if (!s || ncycles < 0) return fail(SPB_ERR_INVALID, "spb_sim_cycle: bad arguments");
  if (!s->fields_set) return fail(SPB_ERR_INVALID, "spb_sim_cycle: fields not set");
  cudaStream_t st = (cudaStream_t)stream;
  const TileImpl *ti = find_tile(s->tile);
  const int k = std::max(1, s->d.resort_every);
  for (int c = 0; c < ncycles; ++c) {
    if (s->cycles_since_sort >= k)
      if (int rc = spb_sim_resort(s, stream)) return rc;
    for (auto &q : s->sp) SPB_CUDA(cudaMemsetAsync(q.mom, 0, 10 * s->nodes * sizeof(double), st));
    if (int rc = ti->cycle(s, st)) return rc;
    s->cycles_since_sort++;
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
  if (S.n == 0) return SPB_OK;
  if (!x || !y || !z || !u || !v || !w)
    return fail(SPB_ERR_INVALID, "spb_sim_particles: null output array");
  cudaStream_t st = (cudaStream_t)stream;
  float *dst[7] = {x, y, z, u, v, w, q};
  float *tmp[7];
  const int spare = 1 - S.cur;
  for (int a = 0; a < 7; ++a) tmp[a] = on_device ? dst[a] : (dst[a] ? S.f[spare][a] : nullptr);
  k_unload<<<blocks_for(S.n, 256), 256, 0, st>>>(
      scalars(s), S.cell[S.cur], S.f[S.cur][0], S.f[S.cur][1], S.f[S.cur][2], S.f[S.cur][3],
      S.f[S.cur][4], S.f[S.cur][5], S.f[S.cur][6], S.n, tmp[0], tmp[1], tmp[2], tmp[3], tmp[4],
      tmp[5], tmp[6]);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  s->launches++;
  if (!on_device)
    for (int a = 0; a < 7; ++a)
      if (dst[a])
        SPB_CUDA(cudaMemcpyAsync(dst[a], tmp[a], S.n * sizeof(float), cudaMemcpyDeviceToHost, st));
  return SPB_OK;
}

extern "C" int spb_sim_check(spb_sim *s, void *stream) {
  if (!s) return fail(SPB_ERR_INVALID, "spb_sim_check: null simulation");
  SPB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  int h = 0;
  SPB_CUDA(cudaMemcpy(&h, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    SPB_CUDA(cudaMemset(s->d_err, 0, sizeof(int)));
    if (h & 2) return fail(SPB_ERR_TIMEOUT, "a staged field tile never arrived (bounded wait)");
    if (h & 4) return fail(SPB_ERR_CUDA, "the counting sort produced an out-of-range slot");
    if (h & 8) return fail(SPB_ERR_UNSUPPORTED, "shared memory not 128-byte aligned for TMA");
    return fail(SPB_ERR_OUT_OF_GRID, "a particle left the node array and was clamped");
  }
  return SPB_OK;
}
