// The grid context behind the opaque spb_grid_ctx handle.
#pragma once

#include <atomic>
#include <mutex>

#include "common.h"

struct spb_grid_ctx {
  int device = 0;
  int nxn = 0, nyn = 0, nzn = 0;
  long nodes = 0;
  spb::GeomDev geom{};
  float *d_nodes = nullptr;      // xn | yn | zn
  float4 *d_eb4 = nullptr;       // packed fields (Ex, Ey, Ez, Bx)
  float2 *d_eb2 = nullptr;       // packed fields (By, Bz)
  float *d_stage = nullptr;      // 6*nodes staging for host field uploads
  float *d_net = nullptr;        // 10*nodes: net densities (sum over species)
  int *d_err = nullptr;
  bool fields_set = false;
  std::atomic<long> launches{0};
  std::mutex mu;                 // guards the packed field buffer
};

namespace spb {
// Library-wide count of kernel launches (every launcher adds to it).
extern std::atomic<long> g_launches;
}  // namespace spb
