// particle_sort (src/Particles.cpp:72-234) on the device: particles ordered by
// bin, each bin keeping the particles' original order, out-of-range particles
// in a last bin, as the reference's default (binned) branch does.
//
// Bins. n_bin = 1 + (nc - 1) / sort_cps per axis with nc the grid's cell count
// including guard cells (grd->nxc), bin width dist = L / (float)n_bin rounded to
// float, bin of a position floor(x / dist) in float arithmetic, linear index
// z + y*nbz + x*nbz*nby (src/Particles.cpp:67-69).
//
// Sort. A stable LSD radix sort of (bin, original index) pairs with 8-bit
// digits: per pass, each CTA counts the digits of its chunk, a scan (per tile,
// over the tiles' totals, then the carries) turns the counts into digit-major
// offsets, and each CTA scatters its chunk in order
// (ranks within a warp from match_any, across warps through shared counters),
// which keeps every pass stable. A gather then permutes the seven arrays.
#include <algorithm>

#include "common.h"
#include "grid_ctx.h"
#include "kernels.h"

namespace spb {
namespace {

constexpr int RS_TPB = 256;                  // threads per CTA
constexpr int RS_WARPS = RS_TPB / 32;
constexpr int RS_CHUNK = RS_TPB * 16;        // elements per CTA and pass
constexpr unsigned FULLM = 0xffffffffu;

__global__ void k_bin_keys(const float *__restrict__ x, const float *__restrict__ y,
                           const float *__restrict__ z, long n, SortBins B,
                           unsigned *__restrict__ key, unsigned *__restrict__ idx) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
       i += (long)gridDim.x * blockDim.x) {
    const float fx = floorf(__fdiv_rn(x[i], B.dist[0]));
    const float fy = floorf(__fdiv_rn(y[i], B.dist[1]));
    const float fz = floorf(__fdiv_rn(z[i], B.dist[2]));
    // out of the bin zone (or not a number): the last bin
    const bool in = fx >= 0.0f && fx < (float)B.nb[0] && fy >= 0.0f && fy < (float)B.nb[1] &&
                    fz >= 0.0f && fz < (float)B.nb[2];
    const long k = in ? (long)fz + (long)fy * B.nb[2] + (long)fx * B.nb[2] * B.nb[1]
                      : (long)B.nb[0] * B.nb[1] * B.nb[2];
    key[i] = (unsigned)k;
    idx[i] = (unsigned)i;
  }
}

// Digit counts of one chunk: hist[digit * nchunks + chunk].
__global__ void __launch_bounds__(RS_TPB) k_digit_hist(const unsigned *__restrict__ key, long n,
                                                       int shift, unsigned *__restrict__ hist,
                                                       int nchunks) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const long first = (long)blockIdx.x * RS_CHUNK;
  const long last = first + RS_CHUNK < n ? first + RS_CHUNK : n;
  for (long i = first + threadIdx.x; i < last; i += RS_TPB)
    atomicAdd(&h[(key[i] >> shift) & 255u], 1u);
  __syncthreads();
  hist[(long)threadIdx.x * nchunks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one chunk: element i goes to offset[digit][chunk] plus the
// number of earlier elements of the chunk with the same digit.
__global__ void __launch_bounds__(RS_TPB) k_digit_scatter(const unsigned *__restrict__ key,
                                                          const unsigned *__restrict__ idx, long n,
                                                          int shift,
                                                          const unsigned *__restrict__ offset,
                                                          int nchunks, unsigned *__restrict__ key2,
                                                          unsigned *__restrict__ idx2) {
  __shared__ unsigned base[256];                 // next free slot per digit
  __shared__ unsigned wcnt[RS_WARPS][256];       // this round's digit counts per warp
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  base[threadIdx.x] = offset[(long)threadIdx.x * nchunks + blockIdx.x];
  const long first = (long)blockIdx.x * RS_CHUNK;
  const long last = first + RS_CHUNK < n ? first + RS_CHUNK : n;
  for (long r0 = first; r0 < last; r0 += RS_TPB) {   // rounds of RS_TPB elements, in order
    for (int w = 0; w < RS_WARPS; ++w) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const long i = r0 + threadIdx.x;
    const bool valid = i < last;
    const unsigned k = valid ? key[i] : 0u, v = valid ? idx[i] : 0u;
    const unsigned d = valid ? (k >> shift) & 255u : 256u;   // 256: no digit
    const unsigned peers = __match_any_sync(FULLM, d);
    const unsigned rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    // digit-wise prefix over the warps, in warp order; then advance the bases
    {
      const unsigned dd = threadIdx.x;
      unsigned run = 0;
      for (int w = 0; w < RS_WARPS; ++w) {
        const unsigned c = wcnt[w][dd];
        wcnt[w][dd] = run;
        run += c;
      }
      __syncthreads();
      if (valid) {
        const unsigned pos = base[d] + wcnt[warp][d] + rank;
        key2[pos] = k;
        idx2[pos] = v;
      }
      __syncthreads();
      base[dd] += run;
    }
    __syncthreads();
  }
}

constexpr int SCAN_TPB = 1024;

// Exclusive scan of one tile of SCAN_TPB elements of a, in place; the tile's
// total goes to tot[tile].
__global__ void __launch_bounds__(SCAN_TPB) k_scan_tiles(unsigned *a, long m, unsigned *tot) {
  __shared__ unsigned ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long i = (long)blockIdx.x * SCAN_TPB + threadIdx.x;
  const unsigned v = i < m ? a[i] : 0u;
  unsigned x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const unsigned t = __shfl_up_sync(FULLM, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    unsigned t = ws[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned u = __shfl_up_sync(FULLM, t, o);
      if (lane >= o) t += u;
    }
    ws[lane] = t;
  }
  __syncthreads();
  if (i < m) a[i] = (warp ? ws[warp - 1] : 0u) + x - v;
  if (threadIdx.x == 0) tot[blockIdx.x] = ws[31];
}

// Adds each tile's carry (the exclusive scan of the tiles' totals).
__global__ void __launch_bounds__(SCAN_TPB) k_scan_carry(unsigned *a, long m,
                                                         const unsigned *__restrict__ tot) {
  const long i = (long)blockIdx.x * SCAN_TPB + threadIdx.x;
  if (i < m) a[i] += tot[blockIdx.x];
}

// Exclusive scan of a (here small) array in one CTA: block sums carried.
__global__ void __launch_bounds__(SCAN_TPB) k_scan_one(unsigned *a, long m) {
  __shared__ unsigned ws[32];
  unsigned carry = 0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (long b = 0; b < m; b += SCAN_TPB) {
    const long i = b + threadIdx.x;
    const unsigned v = i < m ? a[i] : 0u;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned t = __shfl_up_sync(FULLM, x, o);
      if (lane >= o) x += t;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
      unsigned s = ws[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(FULLM, s, o);
        if (lane >= o) s += t;
      }
      ws[lane] = s;
    }
    __syncthreads();
    const unsigned pre = (warp ? ws[warp - 1] : 0u) + carry;
    if (i < m) a[i] = pre + x - v;
    carry += ws[31];
    __syncthreads();
  }
}

// The seven source and destination arrays of the gather, passed by value.
struct Arrays7 {
  const float *src[7];
  float *dst[7];
};

// dst[a][j] = src[a][idx[j]] for the seven arrays.
__global__ void k_gather7(const __grid_constant__ Arrays7 A, const unsigned *__restrict__ idx,
                          long n) {
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n;
       j += (long)gridDim.x * blockDim.x) {
    const unsigned i = idx[j];
    float v[7];
#pragma unroll
    for (int a = 0; a < 7; ++a) v[a] = __ldg(A.src[a] + i);
#pragma unroll
    for (int a = 0; a < 7; ++a) A.dst[a][j] = v[a];
  }
}

}  // namespace

size_t particle_sort_scratch_bytes(long n) {
  const long nchunks = std::max<long>(1, ceil_div(n, RS_CHUNK));
  const long ntiles = ceil_div(nchunks * 256, SCAN_TPB);
  return (size_t)n * 4 * 4 + (size_t)nchunks * 256 * 4 + (size_t)ntiles * 4 + 256;
}

int device_particle_sort(float *const arr[7], float *const tmp[7], long n, const SortBins &B,
                         void *scratch, cudaStream_t st) {
  if (n <= 0) return SPB_OK;
  if (n >= (1L << 32) - 1) return fail(SPB_ERR_UNSUPPORTED, "particle_sort: at most 2^32-2 particles");
  const long bins = (long)B.nb[0] * B.nb[1] * B.nb[2] + 1;   // with the lost bin
  if (bins >= (1L << 32)) return fail(SPB_ERR_UNSUPPORTED, "particle_sort: too many bins");
  const long nchunks = std::max<long>(1, ceil_div(n, RS_CHUNK));
  unsigned char *p = static_cast<unsigned char *>(scratch);
  unsigned *key = reinterpret_cast<unsigned *>(p);
  unsigned *idx = key + n;
  unsigned *key2 = idx + n;
  unsigned *idx2 = key2 + n;
  unsigned *hist = idx2 + n;
  const long nh = nchunks * 256, ntiles = ceil_div(nh, SCAN_TPB);
  unsigned *tot = hist + nh;
  const unsigned blocks = (unsigned)std::min<long>(ceil_div(n, 256), 148L * 32);
  k_bin_keys<<<blocks, 256, 0, st>>>(arr[0], arr[1], arr[2], n, B, key, idx);
  SPB_CUDA(cudaGetLastError());
  long launches = 1;
  int bits = 0;
  while (bits < 32 && ((unsigned long long)(bins - 1) >> bits) != 0) bits += 8;
  for (int shift = 0; shift < bits; shift += 8) {
    k_digit_hist<<<(unsigned)nchunks, RS_TPB, 0, st>>>(key, n, shift, hist, (int)nchunks);
    // digit-major offsets: tiles, the tiles' totals, the carries
    k_scan_tiles<<<(unsigned)ntiles, SCAN_TPB, 0, st>>>(hist, nh, tot);
    k_scan_one<<<1, SCAN_TPB, 0, st>>>(tot, ntiles);
    k_scan_carry<<<(unsigned)ntiles, SCAN_TPB, 0, st>>>(hist, nh, tot);
    k_digit_scatter<<<(unsigned)nchunks, RS_TPB, 0, st>>>(key, idx, n, shift, hist,
                                                          (int)nchunks, key2, idx2);
    SPB_CUDA(cudaGetLastError());
    launches += 5;
    std::swap(key, key2);
    std::swap(idx, idx2);
  }
  // permute the seven arrays: tmp = arr[idx], then copy back (in stream order;
  // the caller synchronises)
  Arrays7 A;
  for (int a = 0; a < 7; ++a) {
    A.src[a] = arr[a];
    A.dst[a] = tmp[a];
  }
  k_gather7<<<blocks, 256, 0, st>>>(A, idx, n);
  SPB_CUDA(cudaGetLastError());
  for (int a = 0; a < 7; ++a)
    SPB_CUDA(cudaMemcpyAsync(arr[a], tmp[a], n * sizeof(float), cudaMemcpyDeviceToDevice, st));
  g_launches += launches + 1;
  return SPB_OK;
}

}  // namespace spb
