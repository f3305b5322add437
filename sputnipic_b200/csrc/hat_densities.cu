// calculateHatDensities (src/MaxwellSolver.cpp:465-603) on the device: the
// implicit sources of the field solver, J hat on the nodes and rho hat on the
// cell centres, from the species moments, in the reference's arithmetic.
//
// Per species: the divergence of the pressure tensor on the inner cells
// (divSymmTensorN2C, src/Grid.cpp:322-396) scaled by -dt/2, the centre guard
// cells filled (applyBCscalarDensC, src/BC.cpp:623-727), then one node pass
// that interpolates the centres to the inner nodes (interpC2Ninterp,
// src/Grid.cpp:122-139), adds the species' J, rotates with the species'
// omega_c dt/2 and accumulates J hat (the PIdot loop, MaxwellSolver.cpp:
// 535-566). Afterwards the node guards of J hat (applyBCscalarDensN,
// src/BC.cpp:11-121), one cell pass for rho hat = rho_c - dt theta div(J hat)
// (divN2C, src/Grid.cpp:267-319) and the centre guards of rho hat.
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
// is read, in a fixed phase order that the fill kernel keeps (one CTA per
// array, phases separated by barriers).
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

// Pressure-tensor rows (pxx pxy pxz / pxy pyy pyz / pxz pyz pzz): divergence
// of each row on the inner cells, times alfa = (T)(-dt/2).
template <typename T>
struct Tensor6 {
  const T *p[6];   // pxx, pxy, pxz, pyy, pyz, pzz
};

template <typename T>
__global__ void k_hat_div_tensor(HatGeom g, Tensor6<T> P, T alfa, T *__restrict__ cx,
                                 T *__restrict__ cy, T *__restrict__ cz) {
  const int mx = g.nxc - 2, my = g.nyc - 2, mz = g.nzc - 2;
  const long inner = (long)mx * my * mz;
  // row r, column ax -> tensor component
  const int comp[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  T *out[3] = {cx, cy, cz};
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < inner;
       t += (long)gridDim.x * blockDim.x) {
    const int k = 1 + (int)(t % mz), j = 1 + (int)((t / mz) % my), i = 1 + (int)(t / ((long)mz * my));
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      const T c0 = (T)d4(g, P.p[comp[r][0]], i, j, k, 0);
      const T c1 = (T)d4(g, P.p[comp[r][1]], i, j, k, 1);
      const T c2 = (T)d4(g, P.p[comp[r][2]], i, j, k, 2);
      const T div = c0 + c1 + c2;
      out[r][cidx(g, i, j, k)] = div * alfa;
    }
  }
}

// Guard-cell fill of n0 x n1 x n2 scalar arrays, one CTA per array
// (applyBCscalarDensC with s = 1, applyBCscalarDensN with s = 2). Phases in
// the reference order: periodic faces X, Y, Z; edges along X, Y, Z; corners;
// non-periodic faces X, Y, Z. A periodic face copies from n-1-s to 0 and from
// s to n-1; yhi ends the Y-edge loop (nyn - 1 in both reference functions).
struct Fill {
  int n0, n1, n2, s, yhi;
  int per[3];
};

template <typename T>
__global__ void k_hat_fill(Fill f, T *a0, T *a1, T *a2) {
  T *a = blockIdx.x == 0 ? a0 : (blockIdx.x == 1 ? a1 : a2);
  if (!a) return;
  const int n1 = f.n1, n2 = f.n2, s = f.s;
  const int e0 = f.n0 - 1, e1 = n1 - 1, e2 = n2 - 1;
  const int f0 = e0 - s, f1 = e1 - s, f2 = e2 - s;
  auto at = [&](int i, int j, int k) -> T & { return a[((long)i * n1 + j) * n2 + k]; };
  const int tid = threadIdx.x, nt = blockDim.x;
  if (f.per[0])
    for (int t = tid; t < (e1 - 1) * (e2 - 1); t += nt) {
      const int j = 1 + t / (e2 - 1), k = 1 + t % (e2 - 1);
      at(0, j, k) = at(f0, j, k);
      at(e0, j, k) = at(s, j, k);
    }
  __syncthreads();
  if (f.per[1])
    for (int t = tid; t < (e0 - 1) * (e2 - 1); t += nt) {
      const int i = 1 + t / (e2 - 1), k = 1 + t % (e2 - 1);
      at(i, 0, k) = at(i, f1, k);
      at(i, e1, k) = at(i, s, k);
    }
  __syncthreads();
  if (f.per[2])
    for (int t = tid; t < (e0 - 1) * (e1 - 1); t += nt) {
      const int i = 1 + t / (e1 - 1), j = 1 + t % (e1 - 1);
      at(i, j, 0) = at(i, j, f2);
      at(i, j, e2) = at(i, j, s);
    }
  __syncthreads();
  if (f.per[1] || f.per[2])
    for (int i = 1 + tid; i < e0; i += nt) {
      at(i, e1, e2) = at(i, s, s);
      at(i, 0, 0) = at(i, f1, f2);
      at(i, 0, e2) = at(i, f1, s);
      at(i, e1, 0) = at(i, s, f2);
    }
  __syncthreads();
  if (f.per[0] || f.per[2])
    for (int j = 1 + tid; j < f.yhi; j += nt) {
      at(e0, j, e2) = at(s, j, s);
      at(0, j, 0) = at(f0, j, f2);
      at(0, j, e2) = at(f0, j, s);
      at(e0, j, 0) = at(s, j, f2);
    }
  __syncthreads();
  if (f.per[0] || f.per[1])
    for (int k = 1 + tid; k < e2; k += nt) {
      at(e0, e1, k) = at(s, s, k);
      at(0, 0, k) = at(f0, f1, k);
      at(e0, 0, k) = at(s, f1, k);
      at(0, e1, k) = at(f0, s, k);
    }
  __syncthreads();
  if ((f.per[0] || f.per[1] || f.per[2]) && tid == 0) {
    at(e0, e1, e2) = at(s, s, s);
    at(0, e1, e2) = at(f0, s, s);
    at(e0, 0, e2) = at(s, f1, s);
    at(0, 0, e2) = at(f0, f1, s);
    at(e0, e1, 0) = at(s, s, f2);
    at(0, e1, 0) = at(f0, s, f2);
    at(e0, 0, 0) = at(s, f1, f2);
    at(0, 0, 0) = at(f0, f1, f2);
  }
  __syncthreads();
  if (!f.per[0])
    for (int t = tid; t < n1 * n2; t += nt) {
      const int j = t / n2, k = t % n2;
      at(0, j, k) = at(1, j, k);
      at(e0, j, k) = at(e0 - 1, j, k);
    }
  __syncthreads();
  if (!f.per[1])
    for (int t = tid; t < f.n0 * n2; t += nt) {
      const int i = t / n2, k = t % n2;
      at(i, 0, k) = at(i, 1, k);
      at(i, e1, k) = at(i, e1 - 1, k);
    }
  __syncthreads();
  if (!f.per[2])
    for (int t = tid; t < f.n0 * n1; t += nt) {
      const int i = t / n1, j = t % n1;
      at(i, j, 0) = at(i, j, 1);
      at(i, j, e2) = at(i, j, e2 - 1);
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

// One species on every node: the interpolated divergence (inner nodes) plus
// J, rotated by the species' beta B and added into J hat (written fresh for
// the first species).
template <typename T>
__global__ void k_hat_pidot(HatGeom g, Vec3<T> C, Vec3<T> J, Vec3<T> B, T beta, int first,
                            Out3<T> JH) {
  const long nodes = (long)g.nxn * g.nyn * g.nzn;
  for (long n = blockIdx.x * (long)blockDim.x + threadIdx.x; n < nodes;
       n += (long)gridDim.x * blockDim.x) {
    const int k = (int)(n % g.nzn), j = (int)((n / g.nzn) % g.nyn), i = (int)(n / ((long)g.nzn * g.nyn));
    const bool inner = i >= 1 && i < g.nxn - 1 && j >= 1 && j < g.nyn - 1 && k >= 1 && k < g.nzn - 1;
    T tn[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      T v = (T)0;
      if (inner) {
        const T *c = C.v[r];
        T s8 = c[cidx(g, i, j, k)] + c[cidx(g, i - 1, j, k)];
        s8 = s8 + c[cidx(g, i, j - 1, k)];
        s8 = s8 + c[cidx(g, i, j, k - 1)];
        s8 = s8 + c[cidx(g, i - 1, j - 1, k)];
        s8 = s8 + c[cidx(g, i - 1, j, k - 1)];
        s8 = s8 + c[cidx(g, i, j - 1, k - 1)];
        s8 = s8 + c[cidx(g, i - 1, j - 1, k - 1)];
        v = (T)(0.125 * (double)s8);
      }
      tn[r] = v + J.v[r][n];
    }
    const T ox = beta * B.v[0][n], oy = beta * B.v[1][n], oz = beta * B.v[2][n];
    const T X = tn[0], Y = tn[1], Z = tn[2];
    const T edotb = X * ox + Y * oy + Z * oz;
    const T oxx = ox * ox, oyy = oy * oy, ozz = oz * oz;
    const T denom = (T)(1 / (1.0 + (double)oxx + (double)oyy + (double)ozz));
    const T rx = (X + (Y * oz - Z * oy + edotb * ox)) * denom;
    const T ry = (Y + (Z * ox - X * oz + edotb * oy)) * denom;
    const T rz = (Z + (X * oy - Y * ox + edotb * oz)) * denom;
    JH.v[0][n] = (first ? (T)0 : JH.v[0][n]) + rx;
    JH.v[1][n] = (first ? (T)0 : JH.v[1][n]) + ry;
    JH.v[2][n] = (first ? (T)0 : JH.v[2][n]) + rz;
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
  T *tc = nullptr;   // the three centre temporaries
  SPB_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&tc), 3 * cells * sizeof(T), st));
  Fill fc{g.nxc, g.nyc, g.nzc, 1, g.nyn - 1, {d->periodic[0], d->periodic[1], d->periodic[2]}};
  Fill fn{g.nxn, g.nyn, g.nzn, 2, g.nyn - 1, {d->periodic[0], d->periodic[1], d->periodic[2]}};
  const T alfa = (T)(-d->dt / 2.0);
  const long inner = (long)(g.nxc - 2) * (g.nyc - 2) * (g.nzc - 2);
  int rc = SPB_OK;
  for (int is = 0; is < d->ns && rc == SPB_OK; ++is) {
    const T *const *M = mom + 10 * is;
    Tensor6<T> P{{M[4], M[5], M[6], M[7], M[8], M[9]}};
    k_hat_div_tensor<T><<<blocks_for(inner, 256), 256, 0, st>>>(g, P, alfa, tc, tc + cells,
                                                                 tc + 2 * cells);
    k_hat_fill<T><<<3, 1024, 0, st>>>(fc, tc, tc + cells, tc + 2 * cells);
    const T beta = (T)(.5 * d->qom[is] * d->dt / d->c);
    k_hat_pidot<T><<<blocks_for(nodes, 256), 256, 0, st>>>(
        g, Vec3<T>{{tc, tc + cells, tc + 2 * cells}}, Vec3<T>{{M[1], M[2], M[3]}},
        Vec3<T>{{B[0], B[1], B[2]}}, beta, is == 0 ? 1 : 0, Out3<T>{{jxh, jyh, jzh}});
    if (cudaGetLastError() != cudaSuccess) rc = fail(SPB_ERR_CUDA, "spb_hat_densities: launch");
  }
  if (rc == SPB_OK) {
    k_hat_fill<T><<<3, 1024, 0, st>>>(fn, jxh, jyh, jzh);
    k_hat_rho<T><<<blocks_for(cells, 256), 256, 0, st>>>(g, Vec3<T>{{jxh, jyh, jzh}}, rhoc,
                                                         d->dt * d->th, rhoh);
    k_hat_fill<T><<<1, 1024, 0, st>>>(fc, rhoh, (T *)nullptr, (T *)nullptr);
    if (cudaGetLastError() != cudaSuccess) rc = fail(SPB_ERR_CUDA, "spb_hat_densities: launch");
    g_launches += 3 * d->ns + 3;
  }
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
