// Seeded synthetic GEM (Harris current sheet) inputs generated on the device:
// the same counter-based hash (splitmix64) and formulas as
// sputnipic_b200/workload.py, so a workload of hundreds of millions of
// particles is built in HBM in milliseconds. Positions are exactly rounded
// and agree bit for bit with the host generator; velocities, charges and
// fields use CUDA's double-precision tanh/cos/log and may differ from numpy's
// by a few double ulps before the final rounding to float.
#include <cmath>

#include "grid_ctx.h"

namespace spb {
namespace {

constexpr unsigned long long GOLD = 0x9E3779B97F4A7C15ull;

__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ unsigned long long stream_key(unsigned long long seed,
                                                                  unsigned stream) {
  const unsigned long long z = ((seed & 0xFFFFFFFFull) << 32) | (unsigned long long)stream;
  return mix64(z * GOLD + GOLD);
}

__device__ __forceinline__ double uniform01(unsigned long long key, unsigned long long idx) {
  const unsigned long long z = mix64((idx + 1ull) * GOLD + key);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

constexpr unsigned STREAM_PHASE = 1, STREAM_E = 2, STREAM_SPECIES = 16;
constexpr int TPB = 256;

struct GenGrid {
  int nxc, nyc, nzc;
  double Lx, Ly, Lz, dx, dy, dz;
  float invVOL;
};

__global__ void __launch_bounds__(TPB) k_gen_fields(GenGrid g, spb_gem_desc d, double phase,
                                                    unsigned long long kE0, unsigned long long kE1,
                                                    unsigned long long kE2, float *ex, float *ey,
                                                    float *ez, float *bx, float *by, float *bz) {
  const int nxn = g.nxc + 3, nyn = g.nyc + 3, nzn = g.nzc + 3;
  const long nodes = (long)nxn * nyn * nzn;
  const double kx = 2.0 * M_PI / g.Lx, ky = M_PI / g.Ly, amp = d.pert * d.B0;
  for (long n = blockIdx.x * (long)TPB + threadIdx.x; n < nodes; n += (long)gridDim.x * TPB) {
    const int i = (int)(n / ((long)nyn * nzn));
    const int j = (int)((n / nzn) % nyn);
    // node coordinates as setGrid stores them (float), used in double
    const double X = (double)(float)((i - 1.0) * g.dx);
    const double Y = (double)(float)((j - 1.0) * g.dy) - g.Ly / 2;
    bx[n] = (float)(d.B0 * tanh(Y / d.delta) - amp * cos(kx * X + phase) * sin(ky * Y));
    by[n] = (float)(amp * (kx / ky) * sin(kx * X + phase) * cos(ky * Y));
    bz[n] = 0.0f;
    if (d.E_amp != 0.0) {
      ex[n] = (float)(d.E_amp * (2.0 * uniform01(kE0, n) - 1.0));
      ey[n] = (float)(d.E_amp * (2.0 * uniform01(kE1, n) - 1.0));
      ez[n] = (float)(d.E_amp * (2.0 * uniform01(kE2, n) - 1.0));
    } else {
      ex[n] = ey[n] = ez[n] = 0.0f;
    }
  }
}

__device__ __forceinline__ long edge(long c, double ppc) {
  return (long)floor((double)c * ppc + 1e-9);
}

// Cell of the particle with species-global index p: edge(c) <= p < edge(c+1).
__device__ __forceinline__ long cell_of(long p, double ppc, long ncells) {
  long c = (long)floor(((double)p + 0.5) / ppc);
  if (c < 0) c = 0;
  if (c > ncells - 1) c = ncells - 1;
  while (c > 0 && edge(c, ppc) > p) --c;
  while (c < ncells - 1 && edge(c + 1, ppc) <= p) ++c;
  return c;
}

struct Keys {
  unsigned long long pos[3], vel[4];
};

__global__ void __launch_bounds__(TPB) k_gen_particles(GenGrid g, spb_gem_desc d,
                                                       spb_gem_species sp, Keys K, long p_lo,
                                                       long p_hi, float *x, float *y, float *z,
                                                       float *u, float *v, float *w, float *q,
                                                       int *cell_out) {
  const long ncells = (long)g.nxc * g.nyc * g.nzc;
  for (long p = p_lo + blockIdx.x * (long)TPB + threadIdx.x; p < p_hi;
       p += (long)gridDim.x * TPB) {
    const long c = cell_of(p, sp.ppc, ncells);
    const long k = p - edge(c, sp.ppc);
    const long cx = c / ((long)g.nyc * g.nzc), cy = (c / g.nzc) % g.nyc, cz = c % g.nzc;
    const unsigned long long idx = (unsigned long long)p;
    double o[3];
    for (int a = 0; a < 3; ++a) o[a] = uniform01(K.pos[a], idx);
    if (d.lattice > 0) {
      const long m = d.lattice;
      const long sub[3] = {k / (m * m), (k / m) % m, k % m};
      for (int a = 0; a < 3; ++a) o[a] = ((double)sub[a] + o[a]) / (double)m;
    }
    const long i = p - p_lo;
    x[i] = (float)(((double)cx + o[0]) * g.dx);
    y[i] = (float)(((double)cy + o[1]) * g.dy);
    z[i] = (float)(((double)cz + o[2]) * g.dz);
    const double u1 = uniform01(K.vel[0], idx), u2 = uniform01(K.vel[1], idx);
    const double u3 = uniform01(K.vel[2], idx), u4 = uniform01(K.vel[3], idx);
    const double r1 = sqrt(-2.0 * log(1.0 - u1)), r2 = sqrt(-2.0 * log(1.0 - u3));
    u[i] = (float)(sp.vth * (r1 * cos(2.0 * M_PI * u2)));
    v[i] = (float)(sp.vth * (r1 * sin(2.0 * M_PI * u2)));
    w[i] = (float)(sp.w0 + sp.vth * (r2 * cos(2.0 * M_PI * u4)));
    double rho = sp.rho0;
    if (sp.sheet) {
      const double yc = ((double)cy + 0.5) * g.dy - g.Ly / 2;
      const double ch = cosh(yc / d.delta);
      rho = sp.rho0 / (ch * ch);
    }
    q[i] = (float)(copysign(1.0, sp.qom) * rho / (4.0 * M_PI) / sp.ppc / (double)g.invVOL);
    if (cell_out) cell_out[i] = (int)c;
  }
}

GenGrid gen_grid(const spb_gem_desc &d) {
  GenGrid g;
  g.nxc = d.nxc;
  g.nyc = d.nyc;
  g.nzc = d.nzc;
  g.Lx = d.Lx;
  g.Ly = d.Ly;
  g.Lz = d.Lz;
  g.dx = d.Lx / d.nxc;
  g.dy = d.Ly / d.nyc;
  g.dz = d.Lz / d.nzc;
  g.invVOL = (float)(1.0 / (g.dx * g.dy * g.dz));
  return g;
}

int grid_blocks(long n) { return (int)std::min<long>(ceil_div(n, TPB), 148L * 64); }

}  // namespace
}  // namespace spb

using namespace spb;

extern "C" long spb_gem_species_count(const spb_gem_desc *d, const spb_gem_species *sp) {
  if (!d || !sp) return -1;
  const long ncells = (long)d->nxc * d->nyc * d->nzc;
  return (long)std::floor((double)ncells * sp->ppc + 1e-9);
}

extern "C" int spb_gen_gem_fields(const spb_gem_desc *d, float *const fields[6], void *stream) {
  if (!d || !fields) return fail(SPB_ERR_INVALID, "spb_gen_gem_fields: null argument");
  for (int f = 0; f < 6; ++f)
    if (!fields[f]) return fail(SPB_ERR_INVALID, "spb_gen_gem_fields: null field array");
  if (d->nxc < 1 || d->nyc < 1 || d->nzc < 1 || !(d->delta > 0))
    return fail(SPB_ERR_INVALID, "spb_gen_gem_fields: bad grid or sheet width");
  const GenGrid g = gen_grid(*d);
  // the phase draw of the host generator: uniform(seed, STREAM_PHASE, 0)
  const unsigned long long kp = stream_key(d->seed, STREAM_PHASE);
  const double phase =
      2.0 * M_PI * ((double)(mix64(1ull * GOLD + kp) >> 11) * (1.0 / 9007199254740992.0));
  const long nodes = (long)(d->nxc + 3) * (d->nyc + 3) * (d->nzc + 3);
  k_gen_fields<<<grid_blocks(nodes), TPB, 0, (cudaStream_t)stream>>>(
      g, *d, phase, stream_key(d->seed, STREAM_E), stream_key(d->seed, STREAM_E + 1),
      stream_key(d->seed, STREAM_E + 2), fields[0], fields[1], fields[2], fields[3], fields[4],
      fields[5]);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  return SPB_OK;
}

extern "C" int spb_gen_gem_particles(const spb_gem_desc *d, const spb_gem_species *sp,
                                     int species, long first, long count, float *x, float *y,
                                     float *z, float *u, float *v, float *w, float *q,
                                     int *cell, void *stream) {
  if (!d || !sp) return fail(SPB_ERR_INVALID, "spb_gen_gem_particles: null argument");
  const long total = spb_gem_species_count(d, sp);
  if (first < 0 || count < 0 || first + count > total)
    return fail(SPB_ERR_INVALID, "spb_gen_gem_particles: range outside the species");
  if (count == 0) return SPB_OK;
  if (!x || !y || !z || !u || !v || !w || !q)
    return fail(SPB_ERR_INVALID, "spb_gen_gem_particles: null particle array");
  Keys K;
  const unsigned st = STREAM_SPECIES + 16u * (unsigned)species;
  for (int a = 0; a < 3; ++a) K.pos[a] = stream_key(d->seed, st + a);
  for (int a = 0; a < 4; ++a) K.vel[a] = stream_key(d->seed, st + 3 + a);
  k_gen_particles<<<grid_blocks(count), TPB, 0, (cudaStream_t)stream>>>(
      gen_grid(*d), *d, *sp, K, first, first + count, x, y, z, u, v, w, q, cell);
  SPB_CUDA(cudaGetLastError());
  g_launches++;
  return SPB_OK;
}
