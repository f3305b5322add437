// Error state, version/ABI queries and the device-pointer API of the plain
// form (spb_grid_*).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/sputnipic_ref_layout.h"
#include "abi_layout_fields.h"
#include "grid_ctx.h"
#include "kernels.h"

// --------------------------------------------------------------------------
// error state
// --------------------------------------------------------------------------
namespace spb {

namespace {
thread_local int t_last_code = SPB_OK;
thread_local std::string t_last_msg;
}  // namespace

int fail(int code, const std::string &msg) {
  t_last_code = code;
  t_last_msg = msg;
  return code;
}

int fail_cuda(cudaError_t e, const char *what) {
  return fail(SPB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorName(e) + " (" +
                                cudaGetErrorString(e) + ")");
}

std::atomic<long> g_launches{0};

int num_sms() {
  static int n = [] {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return v;
  }();
  return n;
}

PushDev make_push(const spb_push &p) {
  // src/Mover.cpp:11-12: dt_sub_cycling = (FPpart)dt / (double)n_sub_cycles,
  // dto2 = .5 * dt_sub_cycling, qomdt2 = qom * dto2 / c (float product, then
  // a double division), each rounded to FPpart on assignment.
  PushDev d;
  d.dt_sub = (float)((double)(float)p.dt / (double)p.n_sub_cycles);
  d.dto2 = (float)(0.5 * (double)d.dt_sub);
  const float qd = p.qom * d.dto2;
  d.qomdt2 = (float)((double)qd / p.c);
  d.niter = p.niter;
  for (int a = 0; a < 3; ++a) d.periodic[a] = p.periodic[a] ? 1 : 0;
  return d;
}

}  // namespace spb

using namespace spb;

extern "C" int spb_last_error(void) { return t_last_code; }
extern "C" const char *spb_last_error_message(void) { return t_last_msg.c_str(); }
extern "C" void spb_clear_error(void) {
  t_last_code = SPB_OK;
  t_last_msg.clear();
}

extern "C" const char *spb_error_string(int s) {
  switch (s) {
    case SPB_OK: return "ok";
    case SPB_ERR_CUDA: return "CUDA runtime error";
    case SPB_ERR_INVALID: return "invalid argument";
    case SPB_ERR_OUT_OF_GRID: return "particle cell index outside the node array";
    case SPB_ERR_NO_DEVICE: return "no CUDA device";
    case SPB_ERR_ALLOC: return "allocation failed";
    case SPB_ERR_UNSUPPORTED: return "unsupported configuration";
    case SPB_ERR_TIMEOUT: return "bounded device wait timed out";
    case SPB_ERR_CAPACITY: return "request exceeds a fixed capacity";
    default: return "unknown status";
  }
}

extern "C" long spb_launch_count(void) { return g_launches.load(); }

extern "C" const char *spb_version(void) { return "sputnipic_b200 0.1 sm_100a"; }

extern "C" const char *spb_abi_layout_json(void) {
  static const std::string doc = [] {
    std::string out = "{\n";
    SPB_LAYOUT_ALL(SPB_LAYOUT_EMIT_MEMBER)
    SPB_LAYOUT_STRUCTS(SPB_LAYOUT_EMIT_SIZE)
    out += "\"end\": 0\n}\n";
    return out;
  }();
  return doc.c_str();
}

// --------------------------------------------------------------------------
// grid context
// --------------------------------------------------------------------------
namespace {

int create_from_coords(const std::vector<float> &xn, const std::vector<float> &yn,
                       const std::vector<float> &zn, double xStart, double yStart,
                       double zStart, float invdx, float invdy, float invdz, float invVOL,
                       double Lx, double Ly, double Lz, spb_grid_ctx **out) {
  if (!out) return fail(SPB_ERR_INVALID, "spb_grid_create: null output pointer");
  *out = nullptr;
  // the plain kernels index nodes with 32-bit integers
  if ((double)xn.size() * (double)yn.size() * (double)zn.size() >= 2147483648.0)
    return fail(SPB_ERR_UNSUPPORTED, "spb_grid_create: 2^31 nodes or more");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(SPB_ERR_NO_DEVICE, "spb_grid_create: no CUDA device");
  auto *c = new spb_grid_ctx();
  SPB_CUDA(cudaGetDevice(&c->device));
  c->nxn = (int)xn.size();
  c->nyn = (int)yn.size();
  c->nzn = (int)zn.size();
  c->nodes = (long)c->nxn * c->nyn * c->nzn;
  const size_t ncoord = xn.size() + yn.size() + zn.size();
  auto cleanup = [&](int rc) {
    spb_grid_destroy(c);
    return rc;
  };
  if (cudaMalloc(&c->d_nodes, ncoord * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&c->d_eb4, c->nodes * sizeof(float4)) != cudaSuccess ||
      cudaMalloc(&c->d_eb2, c->nodes * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return cleanup(fail(SPB_ERR_ALLOC, "spb_grid_create: device allocation failed"));
  }
  std::vector<float> all(xn);
  all.insert(all.end(), yn.begin(), yn.end());
  all.insert(all.end(), zn.begin(), zn.end());
  if (cudaMemcpy(c->d_nodes, all.data(), ncoord * sizeof(float), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemset(c->d_err, 0, sizeof(int)) != cudaSuccess)
    return cleanup(fail(SPB_ERR_CUDA, "spb_grid_create: upload failed"));
  GeomDev &g = c->geom;
  g.nxn = c->nxn;
  g.nyn = c->nyn;
  g.nzn = c->nzn;
  g.xStart = xStart;
  g.yStart = yStart;
  g.zStart = zStart;
  g.invdx = invdx;
  g.invdy = invdy;
  g.invdz = invdz;
  g.invVOL = invVOL;
  g.Lx = Lx;
  g.Ly = Ly;
  g.Lz = Lz;
  g.xn = c->d_nodes;
  g.yn = c->d_nodes + xn.size();
  g.zn = c->d_nodes + xn.size() + yn.size();
  *out = c;
  return SPB_OK;
}

}  // namespace

extern "C" int spb_grid_create(const struct grid *grd, spb_grid_ctx **out) {
  if (!grd || !grd->XN_flat || !grd->YN_flat || !grd->ZN_flat)
    return fail(SPB_ERR_INVALID, "spb_grid_create: grid or node arrays missing");
  const int nxn = grd->nxn, nyn = grd->nyn, nzn = grd->nzn;
  if (nxn < 3 || nyn < 3 || nzn < 3)
    return fail(SPB_ERR_INVALID, "spb_grid_create: fewer than 3 nodes on an axis");
  // XN[i][j][k] must not depend on j, k (and so on), as setGrid builds it
  // (src/Grid.cpp:53-61); the kernels keep one coordinate array per axis.
  std::vector<float> xn(nxn), yn(nyn), zn(nzn);
  for (int i = 0; i < nxn; ++i) xn[i] = grd->XN_flat[(long)i * nyn * nzn];
  for (int j = 0; j < nyn; ++j) yn[j] = grd->YN_flat[(long)j * nzn];
  for (int k = 0; k < nzn; ++k) zn[k] = grd->ZN_flat[k];
  for (long i = 0; i < nxn; ++i)
    for (long j = 0; j < nyn; ++j)
      for (long k = 0; k < nzn; ++k) {
        const long n = (i * nyn + j) * nzn + k;
        if (grd->XN_flat[n] != xn[i] || grd->YN_flat[n] != yn[j] || grd->ZN_flat[n] != zn[k])
          return fail(SPB_ERR_UNSUPPORTED,
                      "spb_grid_create: node coordinates are not separable per axis");
      }
  return create_from_coords(xn, yn, zn, grd->xStart, grd->yStart, grd->zStart, grd->invdx,
                            grd->invdy, grd->invdz, grd->invVOL, grd->Lx, grd->Ly, grd->Lz,
                            out);
}

extern "C" int spb_grid_create_uniform(int nxc, int nyc, int nzc, double Lx, double Ly,
                                       double Lz, spb_grid_ctx **out) {
  if (nxc < 1 || nyc < 1 || nzc < 1 || !(Lx > 0) || !(Ly > 0) || !(Lz > 0))
    return fail(SPB_ERR_INVALID, "spb_grid_create_uniform: bad sizes");
  // setGrid, src/Grid.cpp:9-58
  const double dx = Lx / nxc, dy = Ly / nyc, dz = Lz / nzc;
  const int nxn = nxc + 3, nyn = nyc + 3, nzn = nzc + 3;
  std::vector<float> xn(nxn), yn(nyn), zn(nzn);
  for (int i = 0; i < nxn; ++i) xn[i] = (float)(0.0 + (i - 1) * dx);
  for (int j = 0; j < nyn; ++j) yn[j] = (float)(0.0 + (j - 1) * dy);
  for (int k = 0; k < nzn; ++k) zn[k] = (float)(0.0 + (k - 1) * dz);
  const float invVOL = (float)((float)1.0 / (dx * dy * dz));
  return create_from_coords(xn, yn, zn, 0.0, 0.0, 0.0, (float)((float)1.0 / dx),
                            (float)((float)1.0 / dy), (float)((float)1.0 / dz), invVOL, Lx, Ly,
                            Lz, out);
}

extern "C" void spb_grid_destroy(spb_grid_ctx *c) {
  if (!c) return;
  cudaFree(c->d_nodes);
  cudaFree(c->d_eb4);
  cudaFree(c->d_eb2);
  cudaFree(c->d_stage);
  cudaFree(c->d_net);
  cudaFree(c->d_err);
  delete c;
}

extern "C" long spb_grid_nodes(const spb_grid_ctx *c) { return c ? c->nodes : 0; }

extern "C" long spb_grid_launches(const spb_grid_ctx *c) { return c ? c->launches.load() : 0; }

extern "C" int spb_grid_set_fields(spb_grid_ctx *c, const float *const fields[6], int on_device,
                                   void *stream) {
  if (!c || !fields) return fail(SPB_ERR_INVALID, "spb_grid_set_fields: null argument");
  for (int f = 0; f < 6; ++f)
    if (!fields[f]) return fail(SPB_ERR_INVALID, "spb_grid_set_fields: null field array");
  cudaStream_t s = (cudaStream_t)stream;
  const float *src[6];
  if (on_device) {
    for (int f = 0; f < 6; ++f) src[f] = fields[f];
  } else {
    if (!c->d_stage && cudaMalloc(&c->d_stage, 6 * c->nodes * sizeof(float)) != cudaSuccess) {
      cudaGetLastError();
      return fail(SPB_ERR_ALLOC, "spb_grid_set_fields: staging allocation failed");
    }
    for (int f = 0; f < 6; ++f) {
      SPB_CUDA(cudaMemcpyAsync(c->d_stage + f * c->nodes, fields[f], c->nodes * sizeof(float),
                               cudaMemcpyHostToDevice, s));
      src[f] = c->d_stage + f * c->nodes;
    }
  }
  int rc = launch_pack_fields(src, c->d_eb4, c->d_eb2, c->nodes, s);
  if (rc) return rc;
  c->launches++;
  c->fields_set = true;
  return SPB_OK;
}

namespace {
int check_push(const spb_push *p) {
  if (!p) return fail(SPB_ERR_INVALID, "push parameters missing");
  if (p->niter < 1) return fail(SPB_ERR_INVALID, "NiterMover must be >= 1");
  if (p->n_sub_cycles < 1) return fail(SPB_ERR_INVALID, "n_sub_cycles must be >= 1");
  if (!(p->c != 0.0)) return fail(SPB_ERR_INVALID, "light speed c must be non-zero");
  return SPB_OK;
}
}  // namespace

extern "C" int spb_grid_mover(spb_grid_ctx *c, const spb_push *push, float *x, float *y,
                              float *z, float *u, float *v, float *w, long n, void *stream) {
  if (!c) return fail(SPB_ERR_INVALID, "spb_grid_mover: null context");
  if (int rc = check_push(push)) return rc;
  if (!c->fields_set) return fail(SPB_ERR_INVALID, "spb_grid_mover: fields not set");
  if (n < 0 || (n > 0 && (!x || !y || !z || !u || !v || !w)))
    return fail(SPB_ERR_INVALID, "spb_grid_mover: bad particle arrays");
  const PushDev p = make_push(*push);
  int rc = launch_plain_mover(c->geom, p, PackedFields{c->d_eb4, c->d_eb2}, x, y, z, u, v, w, n,
                              c->d_err, (cudaStream_t)stream);
  if (!rc && n > 0) c->launches++;
  return rc;
}

extern "C" int spb_grid_p2g(spb_grid_ctx *c, const float *x, const float *y, const float *z,
                            const float *u, const float *v, const float *w, const float *q,
                            long n, float *const mom[10], void *stream) {
  if (!c || !mom) return fail(SPB_ERR_INVALID, "spb_grid_p2g: null argument");
  for (int m = 0; m < 10; ++m)
    if (!mom[m]) return fail(SPB_ERR_INVALID, "spb_grid_p2g: null moment array");
  if (n < 0 || (n > 0 && (!x || !y || !z || !u || !v || !w || !q)))
    return fail(SPB_ERR_INVALID, "spb_grid_p2g: bad particle arrays");
  cudaStream_t st = (cudaStream_t)stream;
  int rc = launch_plain_p2g(c->geom, x, y, z, u, v, w, q, n, mom, c->d_err, st);
  if (!rc && n > 0) c->launches += 2;
  return rc;
}

extern "C" int spb_grid_mover_interp(spb_grid_ctx *c, const spb_push *push, float *x, float *y,
                                     float *z, float *u, float *v, float *w, const float *q,
                                     long n, float *const mom[10], void *stream) {
  if (!c || !mom) return fail(SPB_ERR_INVALID, "spb_grid_mover_interp: null argument");
  if (int rc = check_push(push)) return rc;
  if (!c->fields_set) return fail(SPB_ERR_INVALID, "spb_grid_mover_interp: fields not set");
  for (int m = 0; m < 10; ++m)
    if (!mom[m]) return fail(SPB_ERR_INVALID, "spb_grid_mover_interp: null moment array");
  if (n < 0 || (n > 0 && (!x || !y || !z || !u || !v || !w || !q)))
    return fail(SPB_ERR_INVALID, "spb_grid_mover_interp: bad particle arrays");
  const PushDev p = make_push(*push);
  cudaStream_t st = (cudaStream_t)stream;
  int rc = launch_plain_mover_interp(c->geom, p, PackedFields{c->d_eb4, c->d_eb2}, x, y, z, u, v,
                                     w, q, n, mom, c->d_err, st);
  if (!rc && n > 0) c->launches += 2;
  return rc;
}

extern "C" int spb_grid_apply_bc_ids(spb_grid_ctx *c, const int periodic[3],
                                     float *const mom[10], void *stream) {
  if (!c || !periodic || !mom) return fail(SPB_ERR_INVALID, "spb_grid_apply_bc_ids: null argument");
  for (int m = 0; m < 10; ++m)
    if (!mom[m]) return fail(SPB_ERR_INVALID, "spb_grid_apply_bc_ids: null moment array");
  long l = 0;
  int rc = launch_apply_bc_ids(c->nxn, c->nyn, c->nzn, periodic, mom, (cudaStream_t)stream, &l);
  c->launches += l;
  return rc;
}

extern "C" int spb_grid_check(spb_grid_ctx *c, void *stream) {
  if (!c) return fail(SPB_ERR_INVALID, "spb_grid_check: null context");
  SPB_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  int h = 0;
  SPB_CUDA(cudaMemcpy(&h, c->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    SPB_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
    return fail(SPB_ERR_OUT_OF_GRID,
                "a particle cell index left the node array; the particle was clamped to the "
                "edge cell");
  }
  return SPB_OK;
}

