// Drop-in entry points over the reference's structs: mover_PC, mover_PC_V,
// interpP2G, mover_interp (include/Mover.h:11-26), their extern "C" twins,
// and the residency controls.
//
// Device state. The library keeps, per species (keyed by the address of the
// caller's part->x array, which the reference never reallocates: particle_sort
// copies back into the same arrays, src/Particles.cpp:218-224), device
// copies of x, y, z, u, v, w, q, a moment buffer, an error word and a CUDA
// stream; and per grid (keyed by the struct grid address and its contents) a
// grid context with node coordinates and packed fields.
//
// Coherence. COPY residency uploads the particles at every call and
// downloads what the call changed before returning, so the caller's host
// arrays are always current (the reference GPU build does the same per batch,
// src/gpu/Particles_gpu.cu:242-284). DEVICE residency keeps particles in HBM
// between calls; the caller refreshes the host copy with
// spb_sync_particles_to_host and reports host-side edits with
// spb_invalidate_particles.
//
// Concurrency. interpP2G is called from an OpenMP team over species
// (src/sputniPIC_CPU.cpp:250-256): each species has its own lock, buffers and
// stream, so different species deposit concurrently. Field upload + mover
// launch hold the grid context's lock until the mover finishes, because the
// packed field buffer is shared.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/sputnipic_ref_layout.h"
#include "grid_ctx.h"
#include "kernels.h"

using namespace spb;

namespace {

// Streams the chunks of a pipelined COPY call rotate over. A stream runs its
// chunks in order, so with two streams the upload of chunk k + 2 would wait
// for the download of chunk k (and that for chunk k's kernel): four keep the
// upload engine busy while a chunk's kernel and download complete.
constexpr int NPIPE = 4;

struct Species {
  cudaStream_t stream = nullptr;
  cudaStream_t pipe[NPIPE] = {};  // COPY residency: streams the particle chunks rotate over
  cudaEvent_t ev_in = nullptr;    // fields / moments uploaded
  cudaEvent_t ev_done[NPIPE] = {};   // a pipe stream's chunks finished
  long cap = 0;
  float *d[7] = {};           // x y z u v w q
  float *d_mom = nullptr;     // 10 * mom_nodes
  long mom_nodes = 0;
  int *d_err = nullptr;
  bool dev_current = false;   // the device holds the newest particle data
  bool host_stale = false;    // the host arrays are older than the device copy
  bool q_current = false;
  bool host_q_stale = false;  // a device-side sort permuted q too
  long nop = 0;
  std::mutex mu;

  ~Species() {
    for (float *p : d) cudaFree(p);
    cudaFree(d_mom);
    cudaFree(d_err);
    if (stream) cudaStreamDestroy(stream);
    for (int j = 0; j < NPIPE; ++j) {
      if (pipe[j]) cudaStreamDestroy(pipe[j]);
      if (ev_done[j]) cudaEventDestroy(ev_done[j]);
    }
    if (ev_in) cudaEventDestroy(ev_in);
  }
};

struct GridEntry {
  const struct grid *key = nullptr;
  // contents that must match for the cached context to be reused
  int nxn = 0, nyn = 0, nzn = 0;
  const float *xn_flat = nullptr;
  double xStart = 0, yStart = 0, zStart = 0, Lx = 0, Ly = 0, Lz = 0;
  float invdx = 0, invdy = 0, invdz = 0, invVOL = 0;
  spb_grid_ctx *ctx = nullptr;
};

struct State {
  std::mutex mu;
  int device = 0;
  int residency = SPB_RESIDENCY_COPY;
  std::map<const float *, std::unique_ptr<Species>> species;
  std::vector<GridEntry> grids;
};

State &S() {
  static State *s = new State();  // never destroyed: avoids CUDA calls at exit
  return *s;
}

bool same_grid(const GridEntry &e, const struct grid *g) {
  return e.key == g && e.nxn == g->nxn && e.nyn == g->nyn && e.nzn == g->nzn &&
         e.xn_flat == g->XN_flat && e.xStart == g->xStart && e.yStart == g->yStart &&
         e.zStart == g->zStart && e.Lx == g->Lx && e.Ly == g->Ly && e.Lz == g->Lz &&
         e.invdx == g->invdx && e.invdy == g->invdy && e.invdz == g->invdz &&
         e.invVOL == g->invVOL;
}

// Returns the grid context for `grd`, creating it on first use.
int get_grid(const struct grid *grd, spb_grid_ctx **out) {
  State &st = S();
  std::lock_guard<std::mutex> lk(st.mu);
  for (auto &e : st.grids)
    if (same_grid(e, grd)) {
      *out = e.ctx;
      return SPB_OK;
    }
  // a changed grid at a known address replaces the old entry
  for (auto it = st.grids.begin(); it != st.grids.end(); ++it)
    if (it->key == grd) {
      spb_grid_destroy(it->ctx);
      st.grids.erase(it);
      break;
    }
  spb_grid_ctx *c = nullptr;
  if (int rc = spb_grid_create(grd, &c)) return rc;
  GridEntry e;
  e.key = grd;
  e.nxn = grd->nxn;
  e.nyn = grd->nyn;
  e.nzn = grd->nzn;
  e.xn_flat = grd->XN_flat;
  e.xStart = grd->xStart;
  e.yStart = grd->yStart;
  e.zStart = grd->zStart;
  e.Lx = grd->Lx;
  e.Ly = grd->Ly;
  e.Lz = grd->Lz;
  e.invdx = grd->invdx;
  e.invdy = grd->invdy;
  e.invdz = grd->invdz;
  e.invVOL = grd->invVOL;
  e.ctx = c;
  st.grids.push_back(e);
  *out = c;
  return SPB_OK;
}

int get_species(const struct particles *part, Species **out) {
  State &st = S();
  std::lock_guard<std::mutex> lk(st.mu);
  auto it = st.species.find(part->x);
  if (it == st.species.end()) {
    auto sp = std::make_unique<Species>();
    SPB_CUDA(cudaStreamCreateWithFlags(&sp->stream, cudaStreamNonBlocking));
    SPB_CUDA(cudaMalloc(&sp->d_err, sizeof(int)));
    SPB_CUDA(cudaMemset(sp->d_err, 0, sizeof(int)));
    it = st.species.emplace(part->x, std::move(sp)).first;
  }
  *out = it->second.get();
  return SPB_OK;
}

int use_device() {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(SPB_ERR_NO_DEVICE, "no CUDA device");
  }
  SPB_CUDA(cudaSetDevice(S().device));
  return SPB_OK;
}

int ensure_capacity(Species *sp, long n) {
  if (n <= sp->cap) return SPB_OK;
  for (float *&p : sp->d) {
    cudaFree(p);
    p = nullptr;
  }
  sp->cap = 0;
  sp->dev_current = sp->q_current = false;
  for (float *&p : sp->d)
    if (cudaMalloc(&p, n * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return fail(SPB_ERR_ALLOC, "particle mirror allocation failed");
    }
  sp->cap = n;
  return SPB_OK;
}

int ensure_moments(Species *sp, long nodes) {
  if (sp->d_mom && sp->mom_nodes == nodes) return SPB_OK;
  cudaFree(sp->d_mom);
  sp->d_mom = nullptr;
  if (cudaMalloc(&sp->d_mom, 10 * nodes * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    return fail(SPB_ERR_ALLOC, "moment mirror allocation failed");
  }
  sp->mom_nodes = nodes;
  return SPB_OK;
}

float *const *host_particle_arrays(const struct particles *p, float *out[7]) {
  out[0] = p->x;
  out[1] = p->y;
  out[2] = p->z;
  out[3] = p->u;
  out[4] = p->v;
  out[5] = p->w;
  out[6] = p->q;
  return out;
}

float *const *host_moment_arrays(const struct interpDensSpecies *ids, float *out[10]) {
  out[0] = ids->rhon_flat;
  out[1] = ids->Jx_flat;
  out[2] = ids->Jy_flat;
  out[3] = ids->Jz_flat;
  out[4] = ids->pxx_flat;
  out[5] = ids->pxy_flat;
  out[6] = ids->pxz_flat;
  out[7] = ids->pyy_flat;
  out[8] = ids->pyz_flat;
  out[9] = ids->pzz_flat;
  return out;
}

// Copies arrays [first, last) of x..q between host and device.
int copy_particles(Species *sp, const struct particles *p, int first, int last, bool to_device,
                   long count = -1) {
  float *h[7];
  host_particle_arrays(p, h);
  const size_t bytes = (size_t)(count < 0 ? p->nop : count) * sizeof(float);
  for (int a = first; a < last; ++a) {
    if (!h[a]) return fail(SPB_ERR_INVALID, "particle array is null");
    if (to_device)
      SPB_CUDA(cudaMemcpyAsync(sp->d[a], h[a], bytes, cudaMemcpyHostToDevice, sp->stream));
    else
      SPB_CUDA(cudaMemcpyAsync(h[a], sp->d[a], bytes, cudaMemcpyDeviceToHost, sp->stream));
  }
  return SPB_OK;
}

// Reads and clears the species' device error word (stream already synced).
int take_device_error(Species *sp) {
  int h = 0;
  SPB_CUDA(cudaMemcpyAsync(&h, sp->d_err, sizeof(int), cudaMemcpyDeviceToHost, sp->stream));
  SPB_CUDA(cudaStreamSynchronize(sp->stream));
  if (h) {
    SPB_CUDA(cudaMemsetAsync(sp->d_err, 0, sizeof(int), sp->stream));
    SPB_CUDA(cudaStreamSynchronize(sp->stream));
    return fail(SPB_ERR_OUT_OF_GRID,
                "a particle cell index left the node array (the reference reads out of bounds "
                "there); it was clamped to the edge cell");
  }
  return SPB_OK;
}

spb_push push_of(const struct particles *part, const struct parameters *param) {
  spb_push p;
  p.dt = param->dt;
  p.c = param->c;
  p.qom = part->qom;
  p.niter = part->NiterMover;
  p.n_sub_cycles = part->n_sub_cycles;
  // the particle BC reads the FIELD periodicity flags (src/Mover.cpp:104,123,142)
  p.periodic[0] = param->PERIODICX;
  p.periodic[1] = param->PERIODICY;
  p.periodic[2] = param->PERIODICZ;
  return p;
}

enum class Op { Mover, MoverV, Interp, Fused };

// COPY residency for large species: the particles go through PCIe in chunks
// of PIPE_CHUNK, rotating over NPIPE streams, so one chunk's upload, its
// kernel and the previous chunk's download run at the same time (with pinned
// host arrays; pageable arrays are copied synchronously by CUDA, which is
// still correct). The results are those of one launch over all particles: the
// mover is per particle and the deposit adds into the same moments.
constexpr long PIPE_CHUNK = 1L << 22;

// The moment buffer of a deposit: the host arrays' values uploaded (the
// drop-ins add into them), or zeros that stay on the device (dev_mom).
int upload_moments(Species *sp, struct interpDensSpecies *ids, long nodes, bool dev_mom,
                   float *hm[10], float *dm[10]) {
  if (int rc = ensure_moments(sp, nodes)) return rc;
  if (!dev_mom) host_moment_arrays(ids, hm);
  for (int m = 0; m < 10; ++m) {
    dm[m] = sp->d_mom + m * nodes;
    if (dev_mom) continue;
    if (!hm[m]) return fail(SPB_ERR_INVALID, "moment array is null");
    SPB_CUDA(cudaMemcpyAsync(dm[m], hm[m], nodes * sizeof(float), cudaMemcpyHostToDevice,
                             sp->stream));
  }
  if (dev_mom) SPB_CUDA(cudaMemsetAsync(sp->d_mom, 0, 10 * nodes * sizeof(float), sp->stream));
  return SPB_OK;
}

int ensure_pipe(Species *sp) {
  for (int j = 0; j < NPIPE; ++j) {
    if (!sp->pipe[j]) SPB_CUDA(cudaStreamCreateWithFlags(&sp->pipe[j], cudaStreamNonBlocking));
    if (!sp->ev_done[j])
      SPB_CUDA(cudaEventCreateWithFlags(&sp->ev_done[j], cudaEventDisableTiming));
  }
  if (!sp->ev_in) SPB_CUDA(cudaEventCreateWithFlags(&sp->ev_in, cudaEventDisableTiming));
  return SPB_OK;
}

int run_copy_pipelined(Op op, Species *sp, struct particles *part, struct EMfield *field,
                       struct interpDensSpecies *ids, spb_grid_ctx *ctx,
                       struct parameters *param, long n, bool dev_mom) {
  const bool moves = op != Op::Interp;
  const bool deposits = op == Op::Interp || op == Op::Fused;
  if (int rc = ensure_pipe(sp)) return rc;
  float *h[7];
  host_particle_arrays(part, h);
  const int nin = deposits ? 7 : 6;   // arrays uploaded: x..w, and q to deposit
  for (int a = 0; a < nin; ++a)
    if (!h[a]) return fail(SPB_ERR_INVALID, "particle array is null");
  const long nodes = spb_grid_nodes(ctx);
  float *hm[10] = {};
  float *dm[10] = {};
  // fields are shared by all species: upload, launches and completion of the
  // mover happen under the grid lock
  std::unique_lock<std::mutex> glk(ctx->mu, std::defer_lock);
  if (moves) {
    glk.lock();
    const float *f[6] = {field->Ex_flat, field->Ey_flat, field->Ez_flat,
                         field->Bxn_flat, field->Byn_flat, field->Bzn_flat};
    for (int a = 0; a < 6; ++a)
      if (!f[a]) return fail(SPB_ERR_INVALID, "field array is null");
    if (int rc = spb_grid_set_fields(ctx, f, 0, sp->stream)) return rc;
  }
  float *acc = nullptr;   // one accumulator for all chunks, folded once
  if (deposits) {
    if (int rc = upload_moments(sp, ids, nodes, dev_mom, hm, dm)) return rc;
    acc = plain_acc_alloc(ctx->geom, sp->stream);
  }
  SPB_CUDA(cudaEventRecord(sp->ev_in, sp->stream));
  for (int j = 0; j < NPIPE; ++j) SPB_CUDA(cudaStreamWaitEvent(sp->pipe[j], sp->ev_in, 0));
  const PushDev p = moves ? make_push(push_of(part, param)) : PushDev{};
  const PackedFields F{ctx->d_eb4, ctx->d_eb2};
  long k = 0;
  for (long off = 0; off < n; off += PIPE_CHUNK, ++k) {
    cudaStream_t s = sp->pipe[k % NPIPE];
    const long cnt = std::min(PIPE_CHUNK, n - off);
    const size_t bytes = (size_t)cnt * sizeof(float);
    float *d[7];
    for (int a = 0; a < 7; ++a) d[a] = sp->d[a] + off;
    for (int a = 0; a < nin; ++a)
      SPB_CUDA(cudaMemcpyAsync(d[a], h[a] + off, bytes, cudaMemcpyHostToDevice, s));
    int rc;
    if (op == Op::Fused)
      rc = launch_plain_mover_interp_into(ctx->geom, p, F, d[0], d[1], d[2], d[3], d[4], d[5],
                                          d[6], cnt, acc, dm, sp->d_err, s);
    else if (moves)
      rc = launch_plain_mover(ctx->geom, p, F, d[0], d[1], d[2], d[3], d[4], d[5], cnt,
                              sp->d_err, s, op == Op::MoverV ? 1 : 0);
    else
      rc = launch_plain_p2g_into(ctx->geom, d[0], d[1], d[2], d[3], d[4], d[5], d[6], cnt, acc,
                                 dm, sp->d_err, s);
    if (rc) {
      if (acc) {   // after the chunks already queued on the pipe streams
        for (int j = 0; j < NPIPE; ++j) cudaStreamSynchronize(sp->pipe[j]);
        cudaFreeAsync(acc, sp->stream);
      }
      return rc;
    }
    ctx->launches++;
    if (moves)
      for (int a = 0; a < 6; ++a)
        SPB_CUDA(cudaMemcpyAsync(h[a] + off, d[a], bytes, cudaMemcpyDeviceToHost, s));
  }
  for (int j = 0; j < NPIPE; ++j) {
    SPB_CUDA(cudaEventRecord(sp->ev_done[j], sp->pipe[j]));
    SPB_CUDA(cudaStreamWaitEvent(sp->stream, sp->ev_done[j], 0));
  }
  if (acc) {
    if (int rc = plain_acc_fold(acc, ctx->geom, dm, sp->stream)) return rc;
    ctx->launches++;
  }
  if (deposits && !dev_mom)
    for (int m = 0; m < 10; ++m)
      SPB_CUDA(cudaMemcpyAsync(hm[m], dm[m], nodes * sizeof(float), cudaMemcpyDeviceToHost,
                               sp->stream));
  SPB_CUDA(cudaStreamSynchronize(sp->stream));
  sp->dev_current = true;
  sp->nop = n;
  sp->q_current = deposits;
  sp->host_stale = false;
  return take_device_error(sp);
}

// The common body of the four drop-ins.
int run(Op op, struct particles *part, struct EMfield *field, struct interpDensSpecies *ids,
        struct grid *grd, struct parameters *param, bool dev_mom = false) {
  if (!part || !grd) return fail(SPB_ERR_INVALID, "null particles or grid");
  const bool moves = op != Op::Interp;
  const bool deposits = op == Op::Interp || op == Op::Fused;
  if (moves && (!field || !param)) return fail(SPB_ERR_INVALID, "null field or parameters");
  if (deposits && !ids) return fail(SPB_ERR_INVALID, "null interpDensSpecies");
  if (part->nop < 0) return fail(SPB_ERR_INVALID, "negative particle count");
  if (moves) {
    if (part->NiterMover < 1) return fail(SPB_ERR_INVALID, "NiterMover must be >= 1");
    if (part->n_sub_cycles < 1) return fail(SPB_ERR_INVALID, "n_sub_cycles must be >= 1");
  }
  if (int rc = use_device()) return rc;
  spb_grid_ctx *ctx = nullptr;
  if (int rc = get_grid(grd, &ctx)) return rc;
  if (part->nop == 0) return SPB_OK;
  if (!part->x) return fail(SPB_ERR_INVALID, "particle array is null");
  Species *sp = nullptr;
  if (int rc = get_species(part, &sp)) return rc;
  std::lock_guard<std::mutex> lk(sp->mu);
  const long n = part->nop;
  if (int rc = ensure_capacity(sp, n)) return rc;
  const bool device_mode = S().residency == SPB_RESIDENCY_DEVICE;
  if (!device_mode && n > PIPE_CHUNK)
    return run_copy_pipelined(op, sp, part, field, ids, ctx, param, n, dev_mom);
  // particles: upload unless the device copy is known to be current
  if (!device_mode || !sp->dev_current || sp->nop != n) {
    if (int rc = copy_particles(sp, part, 0, 6, true)) return rc;
    sp->dev_current = true;
    sp->nop = n;
    sp->q_current = false;
  }
  if (deposits && (!device_mode || !sp->q_current)) {
    if (int rc = copy_particles(sp, part, 6, 7, true)) return rc;
    sp->q_current = true;
  }
  const long nodes = spb_grid_nodes(ctx);
  float *hm[10] = {};
  float *dm[10] = {};
  if (deposits)
    if (int rc = upload_moments(sp, ids, nodes, dev_mom, hm, dm)) return rc;
  int rc = SPB_OK;
  if (moves) {
    // fields are shared by all species: upload, launch and completion of the
    // mover happen under the grid lock
    std::lock_guard<std::mutex> glk(ctx->mu);
    const float *f[6] = {field->Ex_flat, field->Ey_flat, field->Ez_flat,
                         field->Bxn_flat, field->Byn_flat, field->Bzn_flat};
    for (int a = 0; a < 6; ++a)
      if (!f[a]) return fail(SPB_ERR_INVALID, "field array is null");
    if ((rc = spb_grid_set_fields(ctx, f, 0, sp->stream))) return rc;
    const PushDev p = make_push(push_of(part, param));
    const PackedFields F{ctx->d_eb4, ctx->d_eb2};
    if (op == Op::Fused)
      rc = launch_plain_mover_interp(ctx->geom, p, F, sp->d[0], sp->d[1], sp->d[2], sp->d[3],
                                     sp->d[4], sp->d[5], sp->d[6], n, dm, sp->d_err, sp->stream);
    else
      rc = launch_plain_mover(ctx->geom, p, F, sp->d[0], sp->d[1], sp->d[2], sp->d[3], sp->d[4],
                              sp->d[5], n, sp->d_err, sp->stream, op == Op::MoverV ? 1 : 0);
    if (rc) return rc;
    ctx->launches += op == Op::Fused ? 2 : 1;
    SPB_CUDA(cudaStreamSynchronize(sp->stream));
  } else {
    rc = launch_plain_p2g(ctx->geom, sp->d[0], sp->d[1], sp->d[2], sp->d[3], sp->d[4], sp->d[5],
                          sp->d[6], n, dm, sp->d_err, sp->stream);
    if (rc) return rc;
    ctx->launches += 2;
  }
  // results back to the host
  if (deposits && !dev_mom)
    for (int m = 0; m < 10; ++m)
      SPB_CUDA(cudaMemcpyAsync(hm[m], dm[m], nodes * sizeof(float), cudaMemcpyDeviceToHost,
                               sp->stream));
  if (moves) {
    if (device_mode) {
      sp->host_stale = true;
    } else {
      if ((rc = copy_particles(sp, part, 0, 6, false))) return rc;
      sp->host_stale = false;
    }
  }
  SPB_CUDA(cudaStreamSynchronize(sp->stream));
  return take_device_error(sp);
}

}  // namespace

// ---------------------------------------------------------------------------
// exported entry points
// ---------------------------------------------------------------------------
extern "C" int spb_mover_PC(struct particles *part, struct EMfield *field, struct grid *grd,
                            struct parameters *param) {
  return run(Op::Mover, part, field, nullptr, grd, param);
}

extern "C" int spb_mover_PC_V(struct particles *part, struct EMfield *field, struct grid *grd,
                              struct parameters *param) {
  return run(Op::MoverV, part, field, nullptr, grd, param);
}

extern "C" void spb_interpP2G(struct particles *part, struct interpDensSpecies *ids,
                              struct grid *grd) {
  run(Op::Interp, part, nullptr, ids, grd, nullptr);
}

extern "C" int spb_mover_interp(struct particles *part, struct EMfield *field,
                                struct interpDensSpecies *ids, struct grid *grd,
                                struct parameters *param) {
  return run(Op::Fused, part, field, ids, grd, param);
}

// The driver's moment section (src/sputniPIC_CPU.cpp:247-259) in one call:
// setZeroDensities, interpP2G of every species into zeroed device moments,
// applyBCids per species and sumOverSpecies on the device, then the species'
// and net host arrays written once. Species run one after another (each on
// its own stream, as in the drop-in interpP2G); the epilogue runs on the
// first species' stream after all of them finished.
extern "C" int spb_interp_all_species(struct particles *part, struct interpDensSpecies *ids,
                                      struct interpDensNet *idn, struct grid *grd,
                                      struct parameters *param) {
  if (!part || !ids || !idn || !grd || !param)
    return fail(SPB_ERR_INVALID, "spb_interp_all_species: null argument");
  const int ns = param->ns;
  if (ns < 1 || ns > 32) return fail(SPB_ERR_UNSUPPORTED, "spb_interp_all_species: 1..32 species");
  if (int rc = use_device()) return rc;
  spb_grid_ctx *ctx = nullptr;
  if (int rc = get_grid(grd, &ctx)) return rc;
  const long nodes = spb_grid_nodes(ctx);
  std::vector<const float *> bases;
  std::vector<Species *> sps(ns, nullptr);
  for (int s = 0; s < ns; ++s) {
    if (part[s].nop <= 0) continue;   // no particles: zero moments
    if (int rc = run(Op::Interp, &part[s], nullptr, &ids[s], grd, param, true)) return rc;
    if (int rc = get_species(&part[s], &sps[s])) return rc;
    bases.push_back(sps[s]->d_mom);
  }
  cudaStream_t st = nullptr;
  for (Species *sp : sps)
    if (sp && !st) st = sp->stream;
  const int periodic[3] = {param->PERIODICX, param->PERIODICY, param->PERIODICZ};
  if (!ctx->d_net && cudaMalloc(&ctx->d_net, 10 * nodes * sizeof(float)) != cudaSuccess) {
    cudaGetLastError();
    ctx->d_net = nullptr;
    return fail(SPB_ERR_ALLOC, "net density allocation failed");
  }
  long launches = 0;
  for (Species *sp : sps) {
    if (!sp) continue;
    float *dm[10];
    for (int m = 0; m < 10; ++m) dm[m] = sp->d_mom + m * nodes;
    if (int rc = launch_apply_bc_ids(ctx->nxn, ctx->nyn, ctx->nzn, periodic, dm, st, &launches))
      return rc;
  }
  if (bases.empty()) {
    SPB_CUDA(cudaMemsetAsync(ctx->d_net, 0, 10 * nodes * sizeof(float), st));
  } else if (int rc = launch_sum_species(bases.data(), (int)bases.size(), nodes, ctx->d_net,
                                         st)) {
    return rc;
  }
  // host arrays: species moments, net moments, and the zeroed cell-centred rhoc
  const size_t nb = nodes * sizeof(float);
  const size_t cells = (size_t)grd->nxc * grd->nyc * grd->nzc;
  float *hn[10];
  const float *const hnet[10] = {idn->rhon_flat, idn->Jx_flat, idn->Jy_flat, idn->Jz_flat,
                                 idn->pxx_flat, idn->pxy_flat, idn->pxz_flat, idn->pyy_flat,
                                 idn->pyz_flat, idn->pzz_flat};
  for (int m = 0; m < 10; ++m) {
    hn[m] = const_cast<float *>(hnet[m]);
    if (!hn[m]) return fail(SPB_ERR_INVALID, "net moment array is null");
    SPB_CUDA(cudaMemcpyAsync(hn[m], ctx->d_net + m * nodes, nb, cudaMemcpyDeviceToHost, st));
  }
  for (int s = 0; s < ns; ++s) {
    float *hm[10];
    host_moment_arrays(&ids[s], hm);
    for (int m = 0; m < 10; ++m) {
      if (!hm[m]) return fail(SPB_ERR_INVALID, "moment array is null");
      if (sps[s])
        SPB_CUDA(cudaMemcpyAsync(hm[m], sps[s]->d_mom + m * nodes, nb, cudaMemcpyDeviceToHost,
                                 st));
      else
        std::memset(hm[m], 0, nb);
    }
    if (ids[s].rhoc_flat) std::memset(ids[s].rhoc_flat, 0, cells * sizeof(float));
  }
  if (idn->rhoc_flat) std::memset(idn->rhoc_flat, 0, cells * sizeof(float));
  if (st) SPB_CUDA(cudaStreamSynchronize(st));
  ctx->launches += launches;
  return SPB_OK;
}

// particle_sort (src/Particles.cpp:72-234) on the device, over all npmax
// entries like the reference. COPY: the host arrays are uploaded, sorted and
// downloaded. A device-resident species with npmax == nop is sorted where it
// lies and its host arrays stay stale; otherwise its host arrays are brought
// up to date first.
extern "C" int spb_particle_sort(struct parameters *param, struct particles *part,
                                 struct grid *grd) {
  if (!param || !part || !grd) return fail(SPB_ERR_INVALID, "spb_particle_sort: null argument");
  if (param->sort_cps < 1) return fail(SPB_ERR_INVALID, "spb_particle_sort: sort_cps < 1");
  const long n = part->npmax;
  if (n <= 0) return SPB_OK;
  if (!part->x) return fail(SPB_ERR_INVALID, "particle array is null");
  if (int rc = use_device()) return rc;
  SortBins B;
  const long nc[3] = {grd->nxc, grd->nyc, grd->nzc};
  const double L[3] = {grd->Lx, grd->Ly, grd->Lz};
  for (int a = 0; a < 3; ++a) {
    const long nb = 1 + ((nc[a] - 1) / param->sort_cps);
    B.nb[a] = (int)nb;
    B.dist[a] = (float)(L[a] / (double)(float)nb);   // FPpart dist = Lx / (FPpart)n_bin
  }
  Species *sp = nullptr;
  if (int rc = get_species(part, &sp)) return rc;
  std::lock_guard<std::mutex> lk(sp->mu);
  const bool in_place = S().residency == SPB_RESIDENCY_DEVICE && sp->host_stale &&
                        sp->q_current && part->nop == n && sp->nop == n;
  if (!in_place && sp->host_stale) {   // the device holds the newest particles
    float *h[7];
    host_particle_arrays(part, h);
    for (int a = 0; a < (sp->host_q_stale ? 7 : 6); ++a)
      SPB_CUDA(cudaMemcpyAsync(h[a], sp->d[a], sp->nop * sizeof(float), cudaMemcpyDeviceToHost,
                               sp->stream));
    SPB_CUDA(cudaStreamSynchronize(sp->stream));
    sp->host_stale = false;
    sp->host_q_stale = false;
  }
  if (int rc = ensure_capacity(sp, n)) return rc;
  // seven temporary arrays and the sort's scratch in one block from the
  // device's memory pool (kept there for the next sort)
  const size_t tmp_bytes = 7 * (size_t)n * sizeof(float);
  const size_t bytes = tmp_bytes + particle_sort_scratch_bytes(n) + 256;
  void *block = pool_alloc(bytes, sp->stream);
  if (!block) return fail(SPB_ERR_ALLOC, "spb_particle_sort: scratch allocation failed");
  float *tmp[7];
  for (int a = 0; a < 7; ++a) tmp[a] = static_cast<float *>(block) + a * n;
  void *scratch = static_cast<unsigned char *>(block) + ((tmp_bytes + 255) & ~size_t(255));
  int rc = SPB_OK;
  if (!in_place) rc = copy_particles(sp, part, 0, 7, true, n);
  if (!rc) rc = device_particle_sort(sp->d, tmp, n, B, scratch, sp->stream);
  if (!rc && !in_place) rc = copy_particles(sp, part, 0, 7, false, n);
  pool_free(block, sp->stream);
  if (!rc) SPB_CUDA(cudaStreamSynchronize(sp->stream));
  if (rc) return rc;
  // the device copy now equals the (sorted) host arrays, or is the newest copy
  sp->dev_current = true;
  sp->q_current = true;
  sp->nop = part->nop;
  if (in_place) sp->host_q_stale = true;
  return SPB_OK;
}

// C++-linkage drop-ins: the symbols an object compiled against the
// reference's include/Mover.h references.
int mover_PC(struct particles *part, struct EMfield *field, struct grid *grd,
             struct parameters *param) {
  return spb_mover_PC(part, field, grd, param);
}

int mover_PC_V(struct particles *part, struct EMfield *field, struct grid *grd,
               struct parameters *param) {
  return spb_mover_PC_V(part, field, grd, param);
}

void interpP2G(struct particles *part, struct interpDensSpecies *ids, struct grid *grd) {
  spb_interpP2G(part, ids, grd);
}

int mover_interp(struct particles *part, struct EMfield *field, struct interpDensSpecies *ids,
                 struct grid *grd, struct parameters *param) {
  return spb_mover_interp(part, field, ids, grd, param);
}

extern "C" int spb_set_device(int device) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(SPB_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= ndev) return fail(SPB_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lk(S().mu);
  if (!S().species.empty() || !S().grids.empty())
    return fail(SPB_ERR_INVALID, "spb_set_device: release the drop-in state first");
  S().device = device;
  return SPB_OK;
}

extern "C" int spb_set_residency(int mode) {
  if (mode != SPB_RESIDENCY_COPY && mode != SPB_RESIDENCY_DEVICE)
    return fail(SPB_ERR_INVALID, "unknown residency mode");
  std::lock_guard<std::mutex> lk(S().mu);
  if (mode == SPB_RESIDENCY_COPY)
    for (auto &kv : S().species)
      if (kv.second->host_stale)
        return fail(SPB_ERR_INVALID,
                    "spb_set_residency: sync device-resident particles to the host first");
  S().residency = mode;
  return SPB_OK;
}

namespace {
Species *find_species(const struct particles *part) {
  std::lock_guard<std::mutex> lk(S().mu);
  auto it = S().species.find(part->x);
  return it == S().species.end() ? nullptr : it->second.get();
}
}  // namespace

extern "C" int spb_sync_particles_to_host(struct particles *part) {
  if (!part) return fail(SPB_ERR_INVALID, "null particles");
  Species *sp = find_species(part);
  if (!sp) return SPB_OK;
  std::lock_guard<std::mutex> lk(sp->mu);
  if (!sp->host_stale) return SPB_OK;
  if (int rc = use_device()) return rc;
  if (part->nop != sp->nop)
    return fail(SPB_ERR_INVALID, "particle count changed while the device copy was newer");
  if (int rc = copy_particles(sp, part, 0, sp->host_q_stale ? 7 : 6, false)) return rc;
  SPB_CUDA(cudaStreamSynchronize(sp->stream));
  sp->host_stale = false;
  sp->host_q_stale = false;
  return SPB_OK;
}

extern "C" int spb_invalidate_particles(struct particles *part) {
  if (!part) return fail(SPB_ERR_INVALID, "null particles");
  Species *sp = find_species(part);
  if (!sp) return SPB_OK;
  std::lock_guard<std::mutex> lk(sp->mu);
  sp->dev_current = false;
  sp->q_current = false;
  sp->host_stale = false;
  sp->host_q_stale = false;
  return SPB_OK;
}

extern "C" int spb_release_all(void) {
  State &st = S();
  std::lock_guard<std::mutex> lk(st.mu);
  if (cudaSetDevice(st.device) != cudaSuccess) cudaGetLastError();
  st.species.clear();
  for (auto &e : st.grids) spb_grid_destroy(e.ctx);
  st.grids.clear();
  return SPB_OK;
}
