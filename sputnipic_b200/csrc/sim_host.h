// Host-side state of the precision form (spb_sim), shared by sim.cu and the
// serving engine (serve.cu). Internal to the library.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <utility>
#include <vector>

#include "../../include/sputnipic_b200.h"
#include "sim_kernels.cuh"

namespace spb {

struct SimSpecies {
  long n = 0;
  double qom = 0;
  int ocap = 0;                 // overflow entries
  float4 *rec[2] = {};          // buckets, [slots[b]][2] each
  long long slots[2] = {0, 0};  // allocated record slots per buffer set
  int *cnt[2] = {};             // per-cell fill counters
  float4 *orec[2] = {};         // overflow records, [ocap][2]
  int *okey[2] = {};            // overflow cell keys
  int *ocnt = nullptr;          // [2] overflow entry counters
  long long *base = nullptr;    // [ncells + 1] bucket layout of both buffer sets
  long long *base2 = nullptr;   // [ncells + 1] the next layout (re-layout)
  long long total = 0;          // record slots of the layout (-1: not read back yet)
  int cur = 0;                  // the buffer set holding the particles
  double *mom = nullptr;        // [10][nodes]
  double quantum[3] = {1.0, 1.0, 1.0};   // deterministic deposit grids (set at load)
};

using EvPair = std::pair<cudaEvent_t, cudaEvent_t>;
struct EvCycle {
  cudaEvent_t b, m, e;          // before push, between push and deposit, after deposit
};

// Device and pinned host buffers of a launch over several simulations.
struct JobBuffers {
  int cap = 0;                    // simulations the buffers hold
  int *d_tile_base = nullptr;     // [cap + 1]
  CycleParams *d_params = nullptr;
  int *h_tile_base = nullptr;     // pinned mirrors
  CycleParams *h_params = nullptr;
  cudaEvent_t ready = nullptr;    // the mirrors' last copies are done
  JobBuffers() = default;
  JobBuffers(const JobBuffers &) = delete;
  JobBuffers &operator=(const JobBuffers &) = delete;
  ~JobBuffers();
};

}  // namespace spb

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
  long long *scan_tmp = nullptr;  // scan block sums + grand total
  int *counts = nullptr;          // [ncells] particles per cell
  long long *lcap = nullptr;      // [ncells] capacities / clamped counts
  long long *offset = nullptr;    // [ncells + 1] readback offsets
  int *fused_done = nullptr;      // fused cycle: [tiles] pushed flags + 2 barrier counters
  CUtensorMap fmap{};
  bool fields_set = false;
  int cycles_since_check = 0;
  // CUDA graphs of one cycle's launches, keyed by the species' buffer parities;
  // captured and replayed on gstream, ordered after the caller's stream
  std::map<unsigned, cudaGraphExec_t> graphs;
  cudaStream_t gstream = nullptr;
  cudaEvent_t gev[2] = {nullptr, nullptr};
  long cycles_run = 0;
  bool graph_failed = false;
  std::vector<spb::SimSpecies> sp;
  long launches = 0;
  // optional CUDA-event timing of the cycle kernels and of the relayouts
  bool timing = false;
  std::vector<spb::EvCycle> ev_cycle;
  std::vector<spb::EvPair> ev_relayout;
};


namespace spb {

// Kernel parameters of a simulation's next cycle (reads buffer set cur).
CycleParams make_params(spb_sim *s);
long relayout_threshold(const SimSpecies &q);
void pool_reserve(long long bytes);

// One cycle of n simulations (all with the same tile shape) in one launch
// each of zeroing, push and deposit; flips their buffer sets.
int launch_jobs(spb_sim *const *sims, int n, JobBuffers &buf, cudaStream_t st);

// Frees a simulation; sync = false when no queued work still uses it.
void sim_free(spb_sim *s, bool sync);
// The status (SPB_OK or SPB_ERR_*, recorded for spb_last_error) of a
// simulation's device error word.
int sim_status(int word);

}  // namespace spb
