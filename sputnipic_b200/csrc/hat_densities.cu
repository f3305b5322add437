// calculateHatDensities (src/MaxwellSolver.cpp:465-603) on the device: the
// implicit sources of the field solver, J hat on the nodes and rho hat on the
// cell centres, from the species moments, in the reference's arithmetic.
//
// Six launches for all species: the divergence of every species' pressure
// tensor on the inner cells (divSymmTensorN2C, src/Grid.cpp:322-396) scaled by
// -dt/2; the centre guard cells of all 3 ns temporaries (applyBCscalarDensC,
// src/BC.cpp:623-727); one node pass that, species by species, interpolates
// the centres to the inner nodes (interpC2Ninterp, src/Grid.cpp:122-139),
// adds the species' J, rotates with its omega_c dt/2 and accumulates J hat
// in registers (the PIdot loop, MaxwellSolver.cpp:535-566); the node guards
// of J hat (applyBCscalarDensN, src/BC.cpp:11-121); one cell pass for
// rho hat = rho_c - dt theta div(J hat) (divN2C, src/Grid.cpp:267-319); the
// centre guards of rho hat.
//
// Arithmetic. This file is compiled with -fmad=false and follows the C
// promotions of the reference expressions: the stencils' .25 * (a - b) * inv
// terms and the .125 interpolation scale are double, rounded to the array
// type on assignment; PIdot's denominator is double, the rest of PIdot is in
// the array type. The float instantiation reproduces the reference's FP32
// build bit for bit, the double one its FP64 build.
//
// Guard values. The reference leaves its temporaries' guard entries
// uninitialised; the guard-cell fills overwrite every one of them before it
// is read, each with the value its phase-by-phase fill would leave there
// (fill_source).
#include <algorithm>
#include <cstring>

#include "../../include/sputnipic_ref_layout.h"
#include "common.h"
#include "grid_ctx.h"

namespace spb {
namespace {

struct HatGeom {
  int nxc, nyc, nzc;   // cells, guard cells included
  int nxn, nyn, nzn;   // nodes
  double inv[3];       // the grid's inverse spacings
};

__device__ __forceinline__ long nidx(const HatGeom &g, int i, int j, int k) {
  return ((long)i * g.nyn + j) * g.nzn + k;
}
__device__ __forceinline__ long cidx(const HatGeom &g, int i, int j, int k) {
  return ((long)i * g.nyc + j) * g.nzc + k;
}

// The four node differences across cell (i, j, k) along `axis`, each times
// .25 and the inverse spacing, summed in double in the reference's order:
// x runs over (j, k), y over (i, k), both with k fastest; z over (i, j) with
// i fastest.
template <typename T>
__device__ __forceinline__ double d4(const HatGeom &g, const T *__restrict__ a, int i, int j,
                                     int k, int axis) {
  double sum = 0.0;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int hi = t >> 1, lo = t & 1;
    int i0 = i, j0 = j, k0 = k;
    if (axis == 0) {
      j0 += hi;
      k0 += lo;
    } else if (axis == 1) {
      i0 += hi;
      k0 += lo;
    } else {
      j0 += hi;
      i0 += lo;
    }
    const T a0 = a[nidx(g, i0, j0, k0)];
    const T a1 = a[nidx(g, i0 + (axis == 0), j0 + (axis == 1), k0 + (axis == 2))];
    const T diff = a1 - a0;
    const double term = 0.25 * (double)diff * g.inv[axis];
    sum = t ? sum + term : term;
  }
  return sum;
}

constexpr int HAT_MAXS = SPB_HAT_MAX_SPECIES;

// Every species' inputs: pressure tensors (pxx, pxy, pxz, pyy, pyz, pzz), J,
// the centre temporaries (three per species) and beta = qom dt / 2c.
template <typename T>
struct Species6 {
  const T *p[HAT_MAXS][6];
  const T *j[HAT_MAXS][3];
  T *tc[HAT_MAXS][3];
  T beta[HAT_MAXS];
};

// Pressure-tensor rows (pxx pxy pxz / pxy pyy pyz / pxz pyz pzz): divergence
// of each row on the inner cells, times alfa = (T)(-dt/2); species blockIdx.y.
// Five CTAs per SM (at most 51 registers; a few bytes spill): the pass is
// bound by the latency of its FP64 stencil loads, so residency pays.
template <typename T>
__global__ void __launch_bounds__(256, 5) k_hat_div_tensor(HatGeom g, const __grid_constant__ Species6<T> S, T alfa) {
  const int is = blockIdx.y;
  const int mx = g.nxc - 2, my = g.nyc - 2, mz = g.nzc - 2;
  const long inner = (long)mx * my * mz;
  // row r, column ax -> tensor component
  const int comp[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < inner;
       t += (long)gridDim.x * blockDim.x) {
    const int k = 1 + (int)(t % mz), j = 1 + (int)((t / mz) % my), i = 1 + (int)(t / ((long)mz * my));
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const T c0 = (T)d4(g, S.p[is][comp[r][0]], i, j, k, 0);
      const T c1 = (T)d4(g, S.p[is][comp[r][1]], i, j, k, 1);
      const T c2 = (T)d4(g, S.p[is][comp[r][2]], i, j, k, 2);
      const T div = c0 + c1 + c2;
      S.tc[is][r][cidx(g, i, j, k)] = div * alfa;
    }
  }
}

// Guard-cell fill of n0 x n1 x n2 scalar arrays (applyBCscalarDensC with
// s = 1, applyBCscalarDensN with s = 2). The reference's phases: periodic
// faces X, Y, Z; edges along X, Y, Z; corners; non-periodic faces X, Y, Z. A
// periodic face copies from n-1-s to 0 and from s to n-1; yhi ends the
// Y-edge loop (nyn - 1 in both reference functions). Every guard cell gets
// the value of one cell of the array before the fill (fill_source), so the
// fill runs as one gather of all guard values and one scatter.
struct Fill {
  int n0, n1, n2, s, yhi;
  int per[3];
};

template <typename T>
struct Arrays {
  T *a[3 * HAT_MAXS];
};

// The guard cells of an n0 x n1 x n2 array, numbered face by face: the two x
// faces (every j, k), the two y faces (inner i, every k), the two z faces
// (inner i, j).
__host__ __device__ __forceinline__ long guard_count(const Fill &f) {
  return 2L * f.n1 * f.n2 + 2L * (f.n0 - 2) * f.n2 + 2L * (f.n0 - 2) * (f.n1 - 2);
}

__device__ __forceinline__ void guard_cell(const Fill &f, long g, int &i, int &j, int &k) {
  const long fx = (long)f.n1 * f.n2, fy = (long)(f.n0 - 2) * f.n2;
  if (g < 2 * fx) {
    i = g < fx ? 0 : f.n0 - 1;
    const long r = g % fx;
    j = (int)(r / f.n2);
    k = (int)(r % f.n2);
  } else if ((g -= 2 * fx) < 2 * fy) {
    j = g < fy ? 0 : f.n1 - 1;
    const long r = g % fy;
    i = 1 + (int)(r / f.n2);
    k = (int)(r % f.n2);
  } else {
    g -= 2 * fy;
    const long fz = (long)(f.n0 - 2) * (f.n1 - 2);
    k = g < fz ? 0 : f.n2 - 1;
    const long r = g % fz;
    i = 1 + (int)(r / (f.n1 - 2));
    j = 1 + (int)(r % (f.n1 - 2));
  }
}

// Periodic source along one axis: the guard at e copies from s, the guard
// at 0 from e - s.
__device__ __forceinline__ int per_src(int x, int e, int s) {
  return x == e ? s : (x == 0 ? e - s : x);
}

// The cell whose value before the fill ends up in cell (i, j, k) after it
// (every phase of the reference's fill copies one cell into another and
// never writes what it reads). The phases in the reference order are:
// periodic faces X, Y, Z; edges along X, Y (j < yhi only), Z; corners;
// non-periodic faces X, Y, Z. Walking them backwards, each phase that writes
// the current cell replaces it by that phase's source.
__device__ __forceinline__ void fill_source(const Fill &f, int &i, int &j, int &k) {
  const int e0 = f.n0 - 1, e1 = f.n1 - 1, e2 = f.n2 - 1, s = f.s;
  const bool p0 = f.per[0], p1 = f.per[1], p2 = f.per[2];
  auto guard = [](int x, int e) { return x == 0 || x == e; };
  auto inner = [](int x, int e) { return x >= 1 && x <= e - 1; };
  if (!p2 && guard(k, e2)) k = k == 0 ? 1 : e2 - 1;   // non-periodic Z faces
  if (!p1 && guard(j, e1)) j = j == 0 ? 1 : e1 - 1;   // non-periodic Y faces
  if (!p0 && guard(i, e0)) i = i == 0 ? 1 : e0 - 1;   // non-periodic X faces
  if ((p0 || p1 || p2) && guard(i, e0) && guard(j, e1) && guard(k, e2)) {   // corners
    i = per_src(i, e0, s);
    j = per_src(j, e1, s);
    k = per_src(k, e2, s);
  }
  if ((p0 || p1) && inner(k, e2) && guard(i, e0) && guard(j, e1)) {   // edges along Z
    i = per_src(i, e0, s);
    j = per_src(j, e1, s);
  }
  if ((p0 || p2) && j >= 1 && j <= f.yhi - 1 && guard(i, e0) && guard(k, e2)) {   // along Y
    i = per_src(i, e0, s);
    k = per_src(k, e2, s);
  }
  if ((p1 || p2) && inner(i, e0) && guard(j, e1) && guard(k, e2)) {   // edges along X
    j = per_src(j, e1, s);
    k = per_src(k, e2, s);
  }
  if (p2 && inner(i, e0) && inner(j, e1) && guard(k, e2)) k = per_src(k, e2, s);   // Z faces
  if (p1 && inner(i, e0) && inner(k, e2) && guard(j, e1)) j = per_src(j, e1, s);   // Y faces
  if (p0 && inner(j, e1) && inner(k, e2) && guard(i, e0)) i = per_src(i, e0, s);   // X faces
}

// Guard-cell fill of narr arrays, first pass: every guard cell's final value
// (from its fill_source, before any guard cell changes) into tmp.
template <typename T>
__global__ void k_hat_guard_gather(Fill f, const __grid_constant__ Arrays<T> A, int narr,
                                   T *__restrict__ tmp) {
  const long G = guard_count(f), total = narr * G;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    int i, j, k;
    guard_cell(f, t % G, i, j, k);
    fill_source(f, i, j, k);
    tmp[t] = A.a[t / G][((long)i * f.n1 + j) * f.n2 + k];
  }
}

// Second pass: the values into the guard cells.
template <typename T>
__global__ void k_hat_guard_scatter(Fill f, const __grid_constant__ Arrays<T> A, int narr,
                                    const T *__restrict__ tmp) {
  const long G = guard_count(f), total = narr * G;
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    int i, j, k;
    guard_cell(f, t % G, i, j, k);
    A.a[t / G][((long)i * f.n1 + j) * f.n2 + k] = tmp[t];
  }
}

template <typename T>
struct Vec3 {
  const T *v[3];
};
template <typename T>
struct Out3 {
  T *v[3];
};

// Every node: per species in order, the interpolated divergence (inner
// nodes) plus J, rotated by the species' beta B and added into J hat, which
// starts at 0 (the reference's per-species accumulation, in registers).
// Four CTAs per SM (at most 64 registers), for the same reason.
template <typename T>
__global__ void __launch_bounds__(256, 4) k_hat_pidot(HatGeom g, const __grid_constant__ Species6<T> S, int ns, Vec3<T> B,
                            Out3<T> JH) {
  const long nodes = (long)g.nxn * g.nyn * g.nzn;
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < nodes;
       n += (long)gridDim.x * blockDim.x) {
    const int k = (int)(n % g.nzn), j = (int)((n / g.nzn) % g.nyn), i = (int)(n / ((long)g.nzn * g.nyn));
    const bool inner = i >= 1 && i < g.nxn - 1 && j >= 1 && j < g.nyn - 1 && k >= 1 && k < g.nzn - 1;
    const T bx = B.v[0][n], by = B.v[1][n], bz = B.v[2][n];
    T jh[3] = {(T)0, (T)0, (T)0};
    for (int is = 0; is < ns; ++is) {
      T tn[3];
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        T v = (T)0;
        if (inner) {
          const T *c = S.tc[is][r];
          T s8 = c[cidx(g, i, j, k)] + c[cidx(g, i - 1, j, k)];
          s8 = s8 + c[cidx(g, i, j - 1, k)];
          s8 = s8 + c[cidx(g, i, j, k - 1)];
          s8 = s8 + c[cidx(g, i - 1, j - 1, k)];
          s8 = s8 + c[cidx(g, i - 1, j, k - 1)];
          s8 = s8 + c[cidx(g, i, j - 1, k - 1)];
          s8 = s8 + c[cidx(g, i - 1, j - 1, k - 1)];
          v = (T)(0.125 * (double)s8);
        }
        tn[r] = v + S.j[is][r][n];
      }
      const T beta = S.beta[is];
      const T ox = beta * bx, oy = beta * by, oz = beta * bz;
      const T X = tn[0], Y = tn[1], Z = tn[2];
      const T edotb = X * ox + Y * oy + Z * oz;
      const T oxx = ox * ox, oyy = oy * oy, ozz = oz * oz;
      const T denom = (T)(1 / (1.0 + (double)oxx + (double)oyy + (double)ozz));
      jh[0] = jh[0] + (X + (Y * oz - Z * oy + edotb * ox)) * denom;
      jh[1] = jh[1] + (Y + (Z * ox - X * oz + edotb * oy)) * denom;
      jh[2] = jh[2] + (Z + (X * oy - Y * ox + edotb * oz)) * denom;
    }
    JH.v[0][n] = jh[0];
    JH.v[1][n] = jh[1];
    JH.v[2][n] = jh[2];
  }
}

// rho hat = rho_c - dt theta div(J hat) on every cell (the divergence is 0 on
// the guard cells, whose values the final fill replaces).
template <typename T>
__global__ void k_hat_rho(HatGeom g, Vec3<T> JH, const T *__restrict__ rhoc, double dt_th,
                          T *__restrict__ rhoh) {
  const long cells = (long)g.nxc * g.nyc * g.nzc;
  for (long c = blockIdx.x * (long)blockDim.x + threadIdx.x; c < cells;
       c += (long)gridDim.x * blockDim.x) {
    const int k = (int)(c % g.nzc), j = (int)((c / g.nzc) % g.nyc), i = (int)(c / ((long)g.nzc * g.nyc));
    T dv = (T)0;
    if (i >= 1 && i < g.nxc - 1 && j >= 1 && j < g.nyc - 1 && k >= 1 && k < g.nzc - 1) {
      const T cx = (T)d4(g, JH.v[0], i, j, k, 0);
      const T cy = (T)d4(g, JH.v[1], i, j, k, 1);
      const T cz = (T)d4(g, JH.v[2], i, j, k, 2);
      dv = cx + cy + cz;
    }
    rhoh[c] = (T)((double)rhoc[c] - dt_th * (double)dv);
  }
}

int blocks_for(long n, int tpb) {
  return (int)std::max<long>(1, std::min<long>((n + tpb - 1) / tpb, 148L * 16));
}

template <typename T>
int hat_densities(const spb_hat_desc *d, const T *const *mom, const T *const B[3], const T *rhoc,
                  T *jxh, T *jyh, T *jzh, T *rhoh, cudaStream_t st) {
  if (!d || !mom || !B || !rhoc || !jxh || !jyh || !jzh || !rhoh)
    return fail(SPB_ERR_INVALID, "spb_hat_densities: null argument");
  if (d->ns < 1 || d->ns > SPB_HAT_MAX_SPECIES)
    return fail(SPB_ERR_INVALID, "spb_hat_densities: ns out of range");
  if (d->nxc < 3 || d->nyc < 3 || d->nzc < 3)
    return fail(SPB_ERR_INVALID, "spb_hat_densities: at least 3 cells per axis (guards included)");
  HatGeom g;
  g.nxc = d->nxc;
  g.nyc = d->nyc;
  g.nzc = d->nzc;
  g.nxn = d->nxc + 1;
  g.nyn = d->nyc + 1;
  g.nzn = d->nzc + 1;
  g.inv[0] = d->invdx;
  g.inv[1] = d->invdy;
  g.inv[2] = d->invdz;
  const long cells = (long)g.nxc * g.nyc * g.nzc, nodes = (long)g.nxn * g.nyn * g.nzn;
  const int ns = d->ns;
  Fill fc{g.nxc, g.nyc, g.nzc, 1, g.nyn - 1, {d->periodic[0], d->periodic[1], d->periodic[2]}};
  Fill fn{g.nxn, g.nyn, g.nzn, 2, g.nyn - 1, {d->periodic[0], d->periodic[1], d->periodic[2]}};
  // three centre temporaries per species, then the guard fills' buffer
  const long gtmp = std::max(3 * ns * guard_count(fc), 3 * guard_count(fn));
  T *tc = nullptr;
  SPB_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&tc),
                           (3 * ns * cells + gtmp) * sizeof(T), st));
  T *const gbuf = tc + 3 * ns * cells;
  auto fill = [&](const Fill &f, const Arrays<T> &arr, int narr) {
    const unsigned blocks = (unsigned)std::min<long>(blocks_for(narr * guard_count(f), 256), 4096);
    k_hat_guard_gather<T><<<blocks, 256, 0, st>>>(f, arr, narr, gbuf);
    k_hat_guard_scatter<T><<<blocks, 256, 0, st>>>(f, arr, narr, gbuf);
  };
  Species6<T> S;   // kernel parameters (copied at launch)
  Arrays<T> A;
  std::memset(&S, 0, sizeof(S));
  std::memset(&A, 0, sizeof(A));
  for (int is = 0; is < ns; ++is) {
    const T *const *M = mom + 10 * is;
    for (int c = 0; c < 6; ++c) S.p[is][c] = M[4 + c];
    for (int r = 0; r < 3; ++r) {
      S.j[is][r] = M[1 + r];
      S.tc[is][r] = tc + (3 * is + r) * cells;
      A.a[3 * is + r] = S.tc[is][r];
    }
    S.beta[is] = (T)(.5 * d->qom[is] * d->dt / d->c);
  }
  const T alfa = (T)(-d->dt / 2.0);
  const long inner = (long)(g.nxc - 2) * (g.nyc - 2) * (g.nzc - 2);
  int rc = SPB_OK;
  const int gx = std::max(1, blocks_for(inner, 256) / ns);
  k_hat_div_tensor<T><<<dim3(gx, ns), 256, 0, st>>>(g, S, alfa);
  fill(fc, A, 3 * ns);
  k_hat_pidot<T><<<blocks_for(nodes, 256), 256, 0, st>>>(g, S, ns, Vec3<T>{{B[0], B[1], B[2]}},
                                                         Out3<T>{{jxh, jyh, jzh}});
  Arrays<T> J{};
  J.a[0] = jxh;
  J.a[1] = jyh;
  J.a[2] = jzh;
  fill(fn, J, 3);
  k_hat_rho<T><<<blocks_for(cells, 256), 256, 0, st>>>(g, Vec3<T>{{jxh, jyh, jzh}}, rhoc,
                                                       d->dt * d->th, rhoh);
  Arrays<T> R{};
  R.a[0] = rhoh;
  fill(fc, R, 1);
  if (cudaGetLastError() != cudaSuccess) rc = fail(SPB_ERR_CUDA, "spb_hat_densities: launch");
  g_launches += 9;
  cudaFreeAsync(tc, st);
  return rc;
}

spb_hat_desc desc_from(const struct grid *grd, const struct parameters *param) {
  spb_hat_desc d;
  std::memset(&d, 0, sizeof(d));
  d.nxc = grd->nxc;
  d.nyc = grd->nyc;
  d.nzc = grd->nzc;
  d.invdx = grd->invdx;
  d.invdy = grd->invdy;
  d.invdz = grd->invdz;
  d.periodic[0] = param->PERIODICX;
  d.periodic[1] = param->PERIODICY;
  d.periodic[2] = param->PERIODICZ;
  d.dt = param->dt;
  d.c = param->c;
  d.th = param->th;
  d.ns = param->ns;
  for (int is = 0; is < param->ns && is < SPB_HAT_MAX_SPECIES; ++is) d.qom[is] = param->qom[is];
  return d;
}

// The drop-in over host arrays: uploads what the computation reads, runs it
// on a library stream, downloads J hat and rho hat.
int hat_dropin(struct interpDens_aux *aux, struct interpDensNet *idn,
               struct interpDensSpecies *ids, struct EMfield *field, struct grid *grd,
               struct parameters *param) {
  if (!aux || !idn || !ids || !field || !grd || !param)
    return fail(SPB_ERR_INVALID, "calculateHatDensities: null argument");
  if (param->ns < 1 || param->ns > SPB_NS_MAX)
    return fail(SPB_ERR_INVALID, "calculateHatDensities: ns out of range");
  const spb_hat_desc d = desc_from(grd, param);
  const long cells = (long)grd->nxc * grd->nyc * grd->nzc;
  const long nodes = (long)grd->nxn * grd->nyn * grd->nzn;
  if (d.nxc < 3 || d.nyc < 3 || d.nzc < 3)
    return fail(SPB_ERR_INVALID, "calculateHatDensities: grid too small");
  typedef spb_FPinterp T;
  static_assert(sizeof(spb_FPinterp) == sizeof(spb_FPfield), "one array type");
  cudaStream_t st;
  SPB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  // node arrays: 9 per species (Jx..pzz), 3 fields, 3 outputs; centre arrays: rhoc, rhoh
  const int nin = 9 * d.ns + 3;
  T *buf = nullptr;
  const size_t bytes = ((size_t)(nin + 3) * nodes + 2 * (size_t)cells) * sizeof(T);
  int rc = SPB_OK;
  if (cudaMallocAsync(reinterpret_cast<void **>(&buf), bytes, st) != cudaSuccess) {
    cudaGetLastError();
    cudaStreamDestroy(st);
    return fail(SPB_ERR_ALLOC, "calculateHatDensities: device allocation failed");
  }
  const T *mom[10 * SPB_NS_MAX];
  T *p = buf;
  for (int is = 0; is < d.ns && rc == SPB_OK; ++is) {
    const struct interpDensSpecies &s = ids[is];
    const T *src[9] = {s.Jx_flat, s.Jy_flat, s.Jz_flat, s.pxx_flat, s.pxy_flat,
                       s.pxz_flat, s.pyy_flat, s.pyz_flat, s.pzz_flat};
    mom[10 * is] = nullptr;   // rhon: not read
    for (int m = 0; m < 9; ++m, p += nodes) {
      if (cudaMemcpyAsync(p, src[m], nodes * sizeof(T), cudaMemcpyHostToDevice, st) != cudaSuccess)
        rc = fail(SPB_ERR_CUDA, "calculateHatDensities: upload");
      mom[10 * is + 1 + m] = p;
    }
  }
  const T *fsrc[3] = {field->Bxn_flat, field->Byn_flat, field->Bzn_flat};
  const T *Bd[3];
  for (int a = 0; a < 3 && rc == SPB_OK; ++a, p += nodes) {
    if (cudaMemcpyAsync(p, fsrc[a], nodes * sizeof(T), cudaMemcpyHostToDevice, st) != cudaSuccess)
      rc = fail(SPB_ERR_CUDA, "calculateHatDensities: upload");
    Bd[a] = p;
  }
  T *jh[3] = {p, p + nodes, p + 2 * nodes};
  p += 3 * nodes;
  T *rhoc = p, *rhoh = p + cells;
  if (rc == SPB_OK &&
      cudaMemcpyAsync(rhoc, idn->rhoc_flat, cells * sizeof(T), cudaMemcpyHostToDevice, st) !=
          cudaSuccess)
    rc = fail(SPB_ERR_CUDA, "calculateHatDensities: upload");
  if (rc == SPB_OK) rc = hat_densities<T>(&d, mom, Bd, rhoc, jh[0], jh[1], jh[2], rhoh, st);
  T *dst[4] = {&aux->Jxh[0][0][0], &aux->Jyh[0][0][0], &aux->Jzh[0][0][0], &aux->rhoh[0][0][0]};
  const T *srcd[4] = {jh[0], jh[1], jh[2], rhoh};
  const long cnt[4] = {nodes, nodes, nodes, cells};
  for (int a = 0; a < 4 && rc == SPB_OK; ++a)
    if (cudaMemcpyAsync(dst[a], srcd[a], cnt[a] * sizeof(T), cudaMemcpyDeviceToHost, st) !=
        cudaSuccess)
      rc = fail(SPB_ERR_CUDA, "calculateHatDensities: download");
  cudaFreeAsync(buf, st);
  if (cudaStreamSynchronize(st) != cudaSuccess && rc == SPB_OK)
    rc = fail(SPB_ERR_CUDA, "calculateHatDensities: stream");
  cudaStreamDestroy(st);
  return rc;
}

}  // namespace
}  // namespace spb

extern "C" int spb_hat_densities_f32(const spb_hat_desc *d, const float *const *mom,
                                     const float *const B[3], const float *rhoc, float *jxh,
                                     float *jyh, float *jzh, float *rhoh, void *stream) {
  return spb::hat_densities<float>(d, mom, B, rhoc, jxh, jyh, jzh, rhoh, (cudaStream_t)stream);
}

extern "C" int spb_hat_densities_f64(const spb_hat_desc *d, const double *const *mom,
                                     const double *const B[3], const double *rhoc, double *jxh,
                                     double *jyh, double *jzh, double *rhoh, void *stream) {
  return spb::hat_densities<double>(d, mom, B, rhoc, jxh, jyh, jzh, rhoh, (cudaStream_t)stream);
}

extern "C" int spb_calculateHatDensities(struct interpDens_aux *id_aux, struct interpDensNet *idn,
                                         struct interpDensSpecies *ids, struct EMfield *field,
                                         struct grid *grd, struct parameters *param) {
  return spb::hat_dropin(id_aux, idn, ids, field, grd, param);
}

void calculateHatDensities(struct interpDens_aux *id_aux, struct interpDensNet *idn,
                           struct interpDensSpecies *ids, struct EMfield *field, struct grid *grd,
                           struct parameters *param) {
  spb::hat_dropin(id_aux, idn, ids, field, grd, param);
}
