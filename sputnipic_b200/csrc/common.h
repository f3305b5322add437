// Internal definitions shared by the CUDA translation units of
// libsputnipic_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <string>

#include "../../include/sputnipic_b200.h"

namespace spb {

// Records an error for spb_last_error()/spb_last_error_message() and returns
// the code, so call sites read `return fail(SPB_ERR_..., "...")`.
int fail(int code, const std::string &msg);
int fail_cuda(cudaError_t e, const char *what);

#define SPB_CUDA(call)                                                  \
  do {                                                                  \
    cudaError_t e_ = (call);                                            \
    if (e_ != cudaSuccess) return ::spb::fail_cuda(e_, #call);          \
  } while (0)

// Grid geometry as the kernels see it: the scalars of `struct grid`
// (include/Grid.h:11-63) plus device copies of the 1D node coordinates.
struct GeomDev {
  int nxn, nyn, nzn;
  double xStart, yStart, zStart;
  float invdx, invdy, invdz, invVOL;
  double Lx, Ly, Lz;
  const float *xn, *yn, *zn;  // node coordinates per axis (device)
};

// Time-step constants of mover_PC (src/Mover.cpp:11-12), already rounded
// to FPpart exactly as the reference rounds them.
struct PushDev {
  float dt_sub, dto2, qomdt2;
  int niter;
  int periodic[3];
};

// Packed node fields: one float4 (Ex, Ey, Ez, Bx) and one float2 (By, Bz)
// per node, so a node's six components arrive in two loads.
struct PackedFields {
  const float4 *eb4;
  const float2 *eb2;
};

// Device error word bits.
enum : int {
  ERRBIT_OUT_OF_GRID = 1,   // a cell index fell outside the node array
  ERRBIT_TIMEOUT = 2,       // a bounded wait for a TMA copy ran out
  ERRBIT_SMEM_ALIGN = 8,    // dynamic shared memory not 128-byte aligned
  ERRBIT_LOST = 16,         // a bucket and the overflow list were both full
  ERRBIT_INEXACT = 32,      // a deterministic deposit sum left its exact range
};

inline long ceil_div(long a, long b) { return (a + b - 1) / b; }

int num_sms();

}  // namespace spb
