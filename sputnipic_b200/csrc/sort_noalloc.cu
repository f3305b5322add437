// Particle load + cell sort that allocates nothing.
//
// The same work as the load and counting sort behind spb_sim_load_species
// (positions -> int32 cell + FP32 offsets, then a counting sort by tile-major
// cell key), but the caller passes every input and output array and the
// scratch (per-cell counters, sort cursors, scan partial sums, an error word)
// lives in one file-scope __device__ array of fixed size. It exists for
// callers that cannot call cudaMalloc at the point where they sort: codes that
// give all device memory to their own pool allocator at start-up, or loops
// where the implicit synchronisation of an allocation is not acceptable.
//
// Limits and sharing: at most SPB_NOALLOC_MAX_CELLS active cells. Every call
// (on any stream) uses the same scratch array and leaves its contents behind;
// each call clears the counters it needs first, so calls that run one after
// another are fine, but calls that overlap on the GPU race on the scratch.
// The first call on a device looks the array's device address up with
// cudaGetSymbolAddress (a host-side name is not a device address) and keeps
// it for the life of the process; make that first call before any stream
// capture. The stream must belong to the current device. Every call waits for
// its stream before returning (it reads its error word back).
#include <mutex>

#include "grid_ctx.h"
#include "sim_kernels.cuh"

namespace spb {
namespace {

constexpr long NA_MAX_CELLS = SPB_NOALLOC_MAX_CELLS;
constexpr int NA_SCAN_B = 1024;
constexpr long NA_MAX_BLOCKS = NA_MAX_CELLS / NA_SCAN_B;
// counters [MAX_CELLS] | cursors [MAX_CELLS + 1] | block sums [MAX_BLOCKS + 1] | error word
constexpr long NA_COUNT_OFF = 0;
constexpr long NA_CURSOR_OFF = NA_MAX_CELLS;
constexpr long NA_BSUM_OFF = NA_CURSOR_OFF + NA_MAX_CELLS + 1;
constexpr long NA_ERR_OFF = NA_BSUM_OFF + NA_MAX_BLOCKS + 1;
constexpr long NA_SCRATCH_INTS = NA_ERR_OFF + 1;

static __device__ __align__(256) int g_noalloc_scratch[NA_SCRATCH_INTS];

constexpr unsigned NA_FULL = 0xffffffffu;

struct NaGrid {
  int nxc, nyc, nzc, nty, ntz;
  double invdx, invdy, invdz;
};

// Position -> cell + offset in cell units (exact double arithmetic); x = L
// maps to the top face of the last cell.
__device__ __forceinline__ void na_to_cell(float x, double inv, int N, int &c, float &o,
                                           int &bad) {
  const double X = (double)x * inv;
  if (!(X >= 0.0) || X > (double)N) {
    bad = 1;
    c = X > (double)N ? N - 1 : 0;
    o = X > (double)N ? 1.0f : 0.0f;
    return;
  }
  const double f = floor(X);
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

template <int TX, int TY, int TZ>
__global__ void k_na_count(NaGrid g, const float *__restrict__ x, const float *__restrict__ y,
                           const float *__restrict__ z, long n, int *__restrict__ counts,
                           int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  int bad = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    int cx, cy, cz;
    float o;
    na_to_cell(x[i], g.invdx, g.nxc, cx, o, bad);
    na_to_cell(y[i], g.invdy, g.nyc, cy, o, bad);
    na_to_cell(z[i], g.invdz, g.nzc, cz, o, bad);
    const int key = tile_key<TX, TY, TZ>(cx, cy, cz, g.nty, g.ntz);
    const unsigned peers = __match_any_sync(__activemask(), key);
    if (lane == __ffs(peers) - 1) atomicAdd(counts + key, __popc(peers));
  }
  if (bad) atomicOr(err, 1);
}

__device__ __forceinline__ int na_block_scan(int v, int *ws, int &total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(NA_FULL, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int s = lane < nw ? ws[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(NA_FULL, s, o);
      if (lane >= o) s += y;
    }
    if (lane < nw) ws[lane] = s;
  }
  __syncthreads();
  const int pre = warp ? ws[warp - 1] : 0;
  total = ws[nw - 1];
  __syncthreads();
  return pre + x - v;
}

__global__ void __launch_bounds__(NA_SCAN_B) k_na_scan_blocks(const int *in, long k, int *out,
                                                              int *bsum) {
  __shared__ int ws[32];
  const long i = blockIdx.x * (long)NA_SCAN_B + threadIdx.x;
  const int v = i < k ? in[i] : 0;
  int total;
  const int ex = na_block_scan(v, ws, total);
  if (i < k) out[i] = ex;
  if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(NA_SCAN_B) k_na_scan_sums(int *bsum, int nb, int *grand) {
  __shared__ int ws[32];
  int carry = 0;
  for (int base = 0; base < nb; base += NA_SCAN_B) {
    const int i = base + threadIdx.x;
    const int v = i < nb ? bsum[i] : 0;
    int total;
    const int ex = na_block_scan(v, ws, total);
    if (i < nb) bsum[i] = ex + carry;
    carry += total;
  }
  if (threadIdx.x == 0) *grand = carry;
}

__global__ void __launch_bounds__(NA_SCAN_B) k_na_scan_add(int *out, long k, const int *bsum,
                                                           int *cursor) {
  const long i = blockIdx.x * (long)NA_SCAN_B + threadIdx.x;
  if (i < k) {
    const int v = out[i] + bsum[blockIdx.x];
    out[i] = v;
    cursor[i] = v;
  }
}

template <int TX, int TY, int TZ>
__global__ void k_na_scatter(NaGrid g, const float *__restrict__ x, const float *__restrict__ y,
                             const float *__restrict__ z, const float *__restrict__ u,
                             const float *__restrict__ v, const float *__restrict__ w,
                             const float *__restrict__ q, long n, int *__restrict__ cursor,
                             uint32_t *cell_o, float *ox_o, float *oy_o, float *oz_o, float *u_o,
                             float *v_o, float *w_o, float *q_o, int *__restrict__ err) {
  const int lane = threadIdx.x & 31;
  int bad = 0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    int cx, cy, cz;
    float ox, oy, oz;
    na_to_cell(x[i], g.invdx, g.nxc, cx, ox, bad);
    na_to_cell(y[i], g.invdy, g.nyc, cy, oy, bad);
    na_to_cell(z[i], g.invdz, g.nzc, cz, oz, bad);
    const int key = tile_key<TX, TY, TZ>(cx, cy, cz, g.nty, g.ntz);
    const unsigned peers = __match_any_sync(__activemask(), key);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(cursor + key, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    const long d = base + __popc(peers & ((1u << lane) - 1u));
    if (d < 0 || d >= n) {
      bad = 2;
      continue;
    }
    cell_o[d] = pack_cell(cx, cy, cz);
    ox_o[d] = ox;
    oy_o[d] = oy;
    oz_o[d] = oz;
    u_o[d] = u[i];
    v_o[d] = v[i];
    w_o[d] = w[i];
    q_o[d] = q[i];
  }
  if (bad) atomicOr(err, bad);
}

// Device address of the scratch array on the current device, looked up once
// per device for the life of the process (a cudaDeviceReset invalidates it).
// The stream must belong to the current device: the address is that device's.
int scratch_address(cudaStream_t st, int **out) {
  static std::mutex mu;
  static int *addr[64] = {};
  int dev = 0;
  SPB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SPB_ERR_UNSUPPORTED, "device index above 63");
  if (st) {
    int sdev = -1;
    SPB_CUDA(cudaStreamGetDevice(st, &sdev));
    if (sdev != dev)
      return fail(SPB_ERR_INVALID,
                  "spb_sort_particles_noalloc: the stream belongs to another device than the "
                  "current one");
  }
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(scratch)");
    addr[dev] = static_cast<int *>(p);
  }
  *out = addr[dev];
  return SPB_OK;
}

template <int TX, int TY, int TZ>
int na_sort(const NaGrid &g, long ncells, const float *const in[7], long n, uint32_t *cell_o,
            float *const out[7], int *cell_start, int *scratch, cudaStream_t st) {
  int *counts = scratch + NA_COUNT_OFF, *cursor = scratch + NA_CURSOR_OFF;
  int *bsum = scratch + NA_BSUM_OFF, *err = scratch + NA_ERR_OFF;
  // the scratch keeps the previous call's contents: clear counters and error
  SPB_CUDA(cudaMemsetAsync(counts, 0, ncells * sizeof(int), st));
  SPB_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
  const int tpb = 256;
  const unsigned blocks = (unsigned)std::max<long>(1, std::min<long>(ceil_div(n, tpb), 148L * 32));
  if (n > 0) {
    k_na_count<TX, TY, TZ><<<blocks, tpb, 0, st>>>(g, in[0], in[1], in[2], n, counts, err);
    SPB_CUDA(cudaGetLastError());
  }
  const int nb = (int)ceil_div(ncells, NA_SCAN_B);
  k_na_scan_blocks<<<nb, NA_SCAN_B, 0, st>>>(counts, ncells, cell_start, bsum);
  k_na_scan_sums<<<1, NA_SCAN_B, 0, st>>>(bsum, nb, cell_start + ncells);
  k_na_scan_add<<<nb, NA_SCAN_B, 0, st>>>(cell_start, ncells, bsum, cursor);
  SPB_CUDA(cudaGetLastError());
  if (n > 0) {
    k_na_scatter<TX, TY, TZ><<<blocks, tpb, 0, st>>>(
        g, in[0], in[1], in[2], in[3], in[4], in[5], in[6], n, cursor, cell_o, out[0], out[1],
        out[2], out[3], out[4], out[5], out[6], err);
    SPB_CUDA(cudaGetLastError());
  }
  g_launches += n > 0 ? 5 : 3;
  int h = 0;
  SPB_CUDA(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  SPB_CUDA(cudaStreamSynchronize(st));
  if (h & 2) return fail(SPB_ERR_CUDA, "noalloc sort: a scatter slot fell outside the output");
  if (h & 1) return fail(SPB_ERR_OUT_OF_GRID, "noalloc sort: a position lies outside [0, L]");
  return SPB_OK;
}

}  // namespace
}  // namespace spb

using namespace spb;

extern "C" int spb_sort_particles_noalloc(const spb_sim_desc *d, const float *x, const float *y,
                                          const float *z, const float *u, const float *v,
                                          const float *w, const float *q, long n,
                                          uint32_t *cell, float *ox, float *oy, float *oz,
                                          float *u_out, float *v_out, float *w_out, float *q_out,
                                          int *cell_start, void *stream) {
  if (!d || !cell_start) return fail(SPB_ERR_INVALID, "spb_sort_particles_noalloc: null argument");
  if (d->nxc < 1 || d->nyc < 1 || d->nzc < 1 || d->nxc > 2047 || d->nyc > 1023 || d->nzc > 2047)
    return fail(SPB_ERR_UNSUPPORTED, "spb_sort_particles_noalloc: bad cell counts");
  const long ncells = (long)d->nxc * d->nyc * d->nzc;
  if (ncells > NA_MAX_CELLS)
    return fail(SPB_ERR_CAPACITY,
                "spb_sort_particles_noalloc: the grid has " + std::to_string(ncells) +
                    " cells; the fixed scratch holds at most " + std::to_string(NA_MAX_CELLS));
  if (n < 0 || n >= (1L << 31))
    return fail(SPB_ERR_CAPACITY, "spb_sort_particles_noalloc: 0 <= n < 2^31 particles");
  if (n > 0 && (!x || !y || !z || !u || !v || !w || !q || !cell || !ox || !oy || !oz || !u_out ||
                !v_out || !w_out || !q_out))
    return fail(SPB_ERR_INVALID, "spb_sort_particles_noalloc: null particle array");
  const int t[3] = {d->tile[0] ? d->tile[0] : 8, d->tile[1] ? d->tile[1] : 4,
                    d->tile[2] ? d->tile[2] : 4};
  if (d->nxc % t[0] || d->nyc % t[1] || d->nzc % t[2])
    return fail(SPB_ERR_UNSUPPORTED, "spb_sort_particles_noalloc: cells must be tile multiples");
  cudaStream_t st = (cudaStream_t)stream;
  int *scratch = nullptr;
  if (int rc = scratch_address(st, &scratch)) return rc;
  NaGrid g;
  g.nxc = d->nxc;
  g.nyc = d->nyc;
  g.nzc = d->nzc;
  g.nty = d->nyc / t[1];
  g.ntz = d->nzc / t[2];
  g.invdx = 1.0 / (d->Lx / d->nxc);
  g.invdy = 1.0 / (d->Ly / d->nyc);
  g.invdz = 1.0 / (d->Lz / d->nzc);
  const float *in[7] = {x, y, z, u, v, w, q};
  float *out[7] = {ox, oy, oz, u_out, v_out, w_out, q_out};
  if (t[0] == 8 && t[1] == 4 && t[2] == 4)
    return na_sort<8, 4, 4>(g, ncells, in, n, cell, out, cell_start, scratch, st);
  if (t[0] == 4 && t[1] == 4 && t[2] == 4)
    return na_sort<4, 4, 4>(g, ncells, in, n, cell, out, cell_start, scratch, st);
  if (t[0] == 2 && t[1] == 2 && t[2] == 2)
    return na_sort<2, 2, 2>(g, ncells, in, n, cell, out, cell_start, scratch, st);
  if (t[0] == 8 && t[1] == 8 && t[2] == 4)
    return na_sort<8, 8, 4>(g, ncells, in, n, cell, out, cell_start, scratch, st);
  return fail(SPB_ERR_UNSUPPORTED, "spb_sort_particles_noalloc: tile shape not instantiated");
}
