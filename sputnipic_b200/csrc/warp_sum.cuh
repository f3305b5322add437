// Warp sum of the 80 deposit terms of a cell (8 nodes x 10 moments), shared by
// the plain and the precision deposits.
//
// Layout: each lane holds its terms as 40 packed pairs acc[node * 5 + k] =
// (moment k, moment k + 5) in the reference order rhon, Jx, Jy, Jz, pxx | pxy,
// pxz, pyy, pyz, pzz (src/Mover.cpp:466-570), with node = a*4 + b*2 + c. The
// lane's x/y/z node halves are swapped by lane bits 4/3/2: slot a holds the
// physical node a ^ bit4(lane), and likewise for b (bit 3) and c (bit 2).
#pragma once

namespace spb {

__device__ __forceinline__ float2 shfl_xor2(float2 v, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// Sums the packed accumulators over the warp. Thanks to the swapped halves
// the first three halving steps need no selects: every lane keeps its lower
// half and receives its partner's upper half. Afterwards lane l holds in
// r[0..4] the totals of physical node (a, b, c) = (bit4, bit3, bit2) of l,
// moments 5*bit1(l) .. 5*bit1(l)+4; both lanes of a pair (l, l^1) hold them.
//
// warp_sum80_tail runs the steps after the first (x) halving on the 20 pairs
// of the lane's x half (its slot a = 0 after that step).
__device__ __forceinline__ void warp_sum80_tail(float2 (&acc)[20], float (&r)[5], int lane) {
#pragma unroll
  for (int i = 0; i < 10; ++i) acc[i] = __fadd2_rn(acc[i], shfl_xor2(acc[i + 10], 8));
#pragma unroll
  for (int i = 0; i < 5; ++i) acc[i] = __fadd2_rn(acc[i], shfl_xor2(acc[i + 5], 4));
  const bool h = lane & 2;
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    const float send = h ? acc[k].x : acc[k].y;
    const float keep = h ? acc[k].y : acc[k].x;
    r[k] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) r[k] += __shfl_xor_sync(0xffffffffu, r[k], 1);
}

__device__ __forceinline__ void warp_sum80(float2 (&acc)[40], float (&r)[5], int lane) {
#pragma unroll
  for (int i = 0; i < 20; ++i) acc[i] = __fadd2_rn(acc[i], shfl_xor2(acc[i + 20], 16));
  warp_sum80_tail(*reinterpret_cast<float2(*)[20]>(&acc[0]), r, lane);
}

}  // namespace spb
