// Serving form (spb_serve_*): a stream of independent frozen-field test-
// particle jobs, each a precision-form simulation of its own grid, admitted by
// free HBM and stepped together in one launch per kernel (spb::launch_jobs).
//
// Scheduling. Jobs queue in order of arrival. A step launches one cycle of
// every admitted job, then further launches for the jobs with cycles left,
// cheapest first, within a cost budget relative to the first launch (so a
// small job is not paced by the largest one), all asynchronous; meanwhile it
// admits queued jobs while the next one's estimated footprint fits the budget
// and the launch has room (first come, first served: a large job at the head
// waits rather than being overtaken), uploading them on a stream of their own
// so that the upload overlaps the launches; it then waits for both and
// retires the jobs that reached their cycle count. A job that can never fit
// (larger than the whole budget) fails with SPB_ERR_CAPACITY instead of
// blocking.
#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <memory>
#include <vector>

#include "grid_ctx.h"
#include "sim_host.h"

using namespace spb;

namespace {

using Clock = std::chrono::steady_clock;

constexpr int SERVE_OVERFLOW_PER_MILLE = 125;   // jobs' overflow lists: n/8 entries

struct ServeJob {
  long id = 0;
  spb_job_desc d{};
  const float *fields[6] = {};
  std::vector<const float *> parts;   // ns x 7
  std::vector<long> counts;
  int on_device = 0;
  long long bytes = 0;                // estimated footprint, held while admitted
  spb_sim *sim = nullptr;
  int cycles = 0;                     // cycles launched
  int state = SPB_JOB_PENDING;
  int error = SPB_OK;
  double t[3] = {-1.0, -1.0, -1.0};   // submitted, admitted, finished
  cudaEvent_t done = nullptr;         // recorded after the job's last launch
  long ovf_step = -1;                 // step whose overflow counters were copied back
  int cycles_copied = 0;              // the job's cycles when they were copied
  int cycles_checked = 0;             // cycles its last evaluated check (or re-layout) covers
  ~ServeJob() {
    // a released job's work is complete (its event was seen, or it never ran)
    if (sim) spb::sim_free(sim, false);
    if (done) cudaEventDestroy(done);
  }
};

// Estimated device bytes of a job's simulation, from its grid and particle
// counts: two bucket sets of 32-byte records at count + slack, overflow lists,
// counters and layouts, FP64 moments, fields and scratch, and the temporary
// flat arrays of a host upload.
long long footprint(const spb_job_desc &d, const long *counts, int on_device) {
  const long long ncells = (long long)d.nxc * d.nyc * d.nzc;
  const long long nodes = (long long)(d.nxc + 3) * (d.nyc + 3) * (d.nzc + 3);
  long long b = nodes * 32 + nodes * 24 + ncells * 20 + (1 << 20);
  long long nmax = 0;
  for (int s = 0; s < d.ns; ++s) {
    const long long n = counts[s];
    nmax = std::max(nmax, n);
    const long long slots = (3 * n) / 2 + 19 * ncells;   // as the buckets are allocated
    const long long ocap = std::max<long long>(65536, n * SERVE_OVERFLOW_PER_MILLE / 1000);
    b += 2 * (slots + slots / 16) * 32 + 2 * ocap * 36 + 2 * ncells * 4 + 2 * (ncells + 1) * 8 +
         nodes * 80;
  }
  if (!on_device) b += nmax * 28;
  return b;
}

double seconds_since(Clock::time_point t0) {
  return std::chrono::duration<double>(Clock::now() - t0).count();
}

}  // namespace

constexpr int SERVE_LAUNCHES = 8;   // launches per step at most
constexpr int SERVE_ADMIT_MAX = 8;  // admissions per step at most
constexpr double SERVE_ADMIT_SECONDS = 0.004;   // host time per step for admissions
constexpr int SERVE_ERR_SLOTS = 4096;   // pinned error words of jobs finishing

struct spb_serve {
  spb_serve_desc d{};
  int device = 0;
  cudaStream_t st = nullptr;       // the jobs' cycles
  cudaStream_t adm = nullptr;      // admissions (uploads of new jobs)
  cudaEvent_t adm_done = nullptr;
  JobBuffers buf[SERVE_LAUNCHES];
  long long budget = 0, used = 0;
  long next_id = 0;
  long steps = 0;
  double phase_s[4] = {0, 0, 0, 0};   // admit, overflow checks, launch + wait, retire
  int *h_ovf = nullptr;   // pinned: overflow counters of the jobs' species (by id)
  Clock::time_point t0;
  std::deque<ServeJob *> pending;
  std::vector<ServeJob *> active;      // cycles left to launch
  std::vector<ServeJob *> finishing;   // every cycle launched, not yet seen complete
  std::vector<long> finished;          // ids done or failed since spb_serve_finished
  int *h_err = nullptr;                // pinned: finishing jobs' error words (by id)
  cudaEvent_t step_done[2] = {nullptr, nullptr};
  bool step_pending[2] = {false, false};
  std::map<long, std::unique_ptr<ServeJob>> jobs;   // every job not yet released
};

namespace {

ServeJob *find_job(const spb_serve *s, long id) {
  auto it = s->jobs.find(id);
  return it == s->jobs.end() ? nullptr : it->second.get();
}

void fail_job(spb_serve *s, ServeJob *j, int status) {
  if (j->sim) {
    spb_sim_destroy(j->sim);
    j->sim = nullptr;
  }
  if (j->state == SPB_JOB_ACTIVE) s->used -= j->bytes;
  j->state = SPB_JOB_FAILED;
  j->error = status;
  j->t[2] = seconds_since(s->t0);
  s->finished.push_back(j->id);
}

// Finishing jobs whose last launch has completed: done, or failed with their
// error word's status. wait: block until every one has completed.
int retire(spb_serve *s, bool wait) {
  std::vector<ServeJob *> still;
  for (ServeJob *j : s->finishing) {
    const cudaError_t e = wait ? cudaEventSynchronize(j->done) : cudaEventQuery(j->done);
    if (e == cudaErrorNotReady) {
      still.push_back(j);
      continue;
    }
    if (e != cudaSuccess) return fail_cuda(e, "serving: job completion");
    const int rc = spb::sim_status(s->h_err[j->id % SERVE_ERR_SLOTS]);
    if (rc) {
      fail_job(s, j, rc);
    } else {
      j->state = SPB_JOB_DONE;
      j->t[2] = seconds_since(s->t0);
      s->finished.push_back(j->id);
    }
  }
  s->finishing.swap(still);
  return SPB_OK;
}

// Creates the job's simulation and uploads its fields and particles.
int admit(spb_serve *s, ServeJob *j) {
  spb_sim_desc sd{};
  sd.nxc = j->d.nxc;
  sd.nyc = j->d.nyc;
  sd.nzc = j->d.nzc;
  sd.Lx = j->d.Lx;
  sd.Ly = j->d.Ly;
  sd.Lz = j->d.Lz;
  sd.dt = j->d.dt;
  sd.c = j->d.c;
  sd.niter = j->d.niter;
  for (int a = 0; a < 3; ++a) {
    sd.periodic[a] = j->d.periodic[a];
    sd.tile[a] = s->d.tile[a];
  }
  sd.ns = j->d.ns;
  for (int i = 0; i < j->d.ns; ++i) sd.qom[i] = j->d.qom[i];
  sd.resort_every = 1 << 30;   // the engine checks overflow lists itself
  // its checks come back a few steps late: lists of n/8 entries leave 32x
  // the re-layout threshold for the cycles in between
  sd.overflow_per_mille = SERVE_OVERFLOW_PER_MILLE;
  if (int rc = spb_sim_create(&sd, &j->sim)) return rc;
  if (int rc = spb_sim_set_fields(j->sim, j->fields, j->on_device, s->adm)) return rc;
  for (int i = 0; i < j->d.ns; ++i) {
    const float *const *p = j->parts.data() + 7 * i;
    if (int rc = spb_sim_load_species(j->sim, i, p[0], p[1], p[2], p[3], p[4], p[5], p[6],
                                      j->counts[i], j->on_device, s->adm))
      return rc;
  }
  return SPB_OK;
}

// Estimated cost of one cycle of a job (particles + 4 x cells).
double cycle_cost(const ServeJob *j) {
  double n = 0;
  for (long c : j->counts) n += (double)c;
  return n + 4.0 * (double)j->d.nxc * j->d.nyc * j->d.nzc;
}

}  // namespace

extern "C" int spb_serve_create(const spb_serve_desc *desc, spb_serve **out) {
  if (!out) return fail(SPB_ERR_INVALID, "spb_serve_create: null argument");
  *out = nullptr;
  spb_serve_desc d = desc ? *desc : spb_serve_desc{};
  if (!d.tile[0] || !d.tile[1] || !d.tile[2]) d.tile[0] = d.tile[1] = d.tile[2] = 4;
  if (!spb_sim_tile_supported(d.tile[0], d.tile[1], d.tile[2]))
    return fail(SPB_ERR_UNSUPPORTED, "spb_serve_create: tile shape not instantiated");
  if (d.max_jobs <= 0 || d.max_jobs > SERVE_MAX_JOBS) d.max_jobs = SERVE_MAX_JOBS;
  if (d.check_every <= 0) d.check_every = 4;
  if (d.hbm_budget < 0) return fail(SPB_ERR_INVALID, "spb_serve_create: negative budget");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(SPB_ERR_NO_DEVICE, "no CUDA device");
  }
  if (d.extra_budget == 0.0) d.extra_budget = 1.0;
  auto s = std::make_unique<spb_serve>();
  s->d = d;
  SPB_CUDA(cudaGetDevice(&s->device));
  SPB_CUDA(cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking));
  SPB_CUDA(cudaStreamCreateWithFlags(&s->adm, cudaStreamNonBlocking));
  SPB_CUDA(cudaEventCreateWithFlags(&s->adm_done, cudaEventDisableTiming));
  SPB_CUDA(cudaMallocHost(&s->h_ovf, (size_t)SERVE_ERR_SLOTS * SPB_SIM_MAX_SPECIES * sizeof(int)));
  SPB_CUDA(cudaMallocHost(&s->h_err, (size_t)SERVE_ERR_SLOTS * sizeof(int)));
  for (auto &e : s->step_done) SPB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  if (d.hbm_budget > 0) {
    s->budget = d.hbm_budget;
  } else {
    // free device memory plus what the device's pool holds unused (the
    // library's allocations come from it and keep freed memory there)
    size_t free_b = 0, total_b = 0;
    SPB_CUDA(cudaMemGetInfo(&free_b, &total_b));
    unsigned long long reserved = 0, used = 0;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess &&
        reserved > used)
      free_b += (size_t)(reserved - used);
    cudaGetLastError();
    s->budget = (long long)(0.9 * (double)free_b);
  }
  if (d.reserve_bytes < 0) return fail(SPB_ERR_INVALID, "spb_serve_create: negative reserve");
  if (d.reserve_bytes > 0) pool_reserve(std::min(d.reserve_bytes, s->budget));
  s->t0 = Clock::now();
  *out = s.release();
  return SPB_OK;
}

extern "C" void spb_serve_destroy(spb_serve *s) {
  if (!s) return;
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->adm) cudaStreamSynchronize(s->adm);
  s->jobs.clear();
  if (s->st) cudaStreamDestroy(s->st);
  if (s->adm) cudaStreamDestroy(s->adm);
  if (s->adm_done) cudaEventDestroy(s->adm_done);
  for (cudaEvent_t e : s->step_done)
    if (e) cudaEventDestroy(e);
  cudaFreeHost(s->h_ovf);
  cudaFreeHost(s->h_err);
  delete s;
}

extern "C" long spb_serve_submit(spb_serve *s, const spb_job_desc *job,
                                 const float *const fields[6], const float *const *parts,
                                 const long *counts, int on_device) {
  if (!s || !job || !fields || !parts || !counts)
    return -fail(SPB_ERR_INVALID, "spb_serve_submit: null argument");
  if (job->ns < 1 || job->ns > SPB_SIM_MAX_SPECIES || job->ncycles < 1)
    return -fail(SPB_ERR_INVALID, "spb_serve_submit: 1..8 species and >= 1 cycle");
  if (job->nxc % s->d.tile[0] || job->nyc % s->d.tile[1] || job->nzc % s->d.tile[2])
    return -fail(SPB_ERR_UNSUPPORTED, "spb_serve_submit: cells per axis must be multiples of "
                                      "the engine's tile shape");
  for (int f = 0; f < 6; ++f)
    if (!fields[f]) return -fail(SPB_ERR_INVALID, "spb_serve_submit: null field array");
  for (int i = 0; i < job->ns; ++i) {
    if (counts[i] < 0) return -fail(SPB_ERR_INVALID, "spb_serve_submit: negative count");
    for (int a = 0; a < 7; ++a)
      if (counts[i] > 0 && !parts[7 * i + a])
        return -fail(SPB_ERR_INVALID, "spb_serve_submit: null particle array");
  }
  auto j = std::make_unique<ServeJob>();
  j->id = s->next_id++;
  j->d = *job;
  for (int f = 0; f < 6; ++f) j->fields[f] = fields[f];
  j->parts.assign(parts, parts + 7 * job->ns);
  j->counts.assign(counts, counts + job->ns);
  j->on_device = on_device;
  j->bytes = footprint(*job, counts, on_device);
  j->t[0] = seconds_since(s->t0);
  ServeJob *raw = j.get();
  s->jobs.emplace(raw->id, std::move(j));
  s->pending.push_back(raw);
  return raw->id;
}

extern "C" int spb_serve_step(spb_serve *s) {
  if (!s) return -fail(SPB_ERR_INVALID, "spb_serve_step: null engine");
  SPB_CUDA(cudaSetDevice(s->device));
  Clock::time_point tp = Clock::now();
  auto lap = [&](int phase) {
    const Clock::time_point t = Clock::now();
    s->phase_s[phase] += std::chrono::duration<double>(t - tp).count();
    tp = t;
  };
  // admit in order of arrival while the head fits, uploading on the
  // admission stream; the engine's stream then waits for the uploads. At
  // most SERVE_ADMIT_MAX jobs or SERVE_ADMIT_SECONDS of host time per step
  // (at least one job): the rest are admitted in the next steps, so a burst
  // of arrivals does not hold the launches back while each job's memory is
  // allocated and its layout queued
  auto admit_pending = [&](std::vector<ServeJob *> &joined) -> int {
    const Clock::time_point t_adm = Clock::now();
    int admitted = 0;
    while (!s->pending.empty() && (int)(s->active.size() + joined.size()) < s->d.max_jobs &&
           (admitted == 0 ||
            (admitted < SERVE_ADMIT_MAX && seconds_since(t_adm) < SERVE_ADMIT_SECONDS))) {
      ServeJob *j = s->pending.front();
      if (j->bytes > s->budget) {   // can never fit: fail it rather than block the queue
        s->pending.pop_front();
        fail_job(s, j, fail(SPB_ERR_CAPACITY, "job larger than the engine's HBM budget"));
        continue;
      }
      if (s->used + j->bytes > s->budget) break;
      s->pending.pop_front();
      j->state = SPB_JOB_ACTIVE;
      s->used += j->bytes;
      j->t[1] = seconds_since(s->t0);
      if (int rc = admit(s, j)) {
        cudaStreamSynchronize(s->adm);   // nothing of the failed job may still run
        fail_job(s, j, rc);
        continue;
      }
      joined.push_back(j);
      ++admitted;
    }
    SPB_CUDA(cudaEventRecord(s->adm_done, s->adm));
    SPB_CUDA(cudaStreamWaitEvent(s->st, s->adm_done, 0));
    return SPB_OK;
  };
  if (int rc = retire(s, false)) return -rc;
  lap(3);
  std::vector<ServeJob *> joined;
  const bool idle = s->active.empty();
  if (idle) {   // nothing to launch: the new jobs run in this step
    if (int rc = admit_pending(joined)) return -rc;
    s->active.swap(joined);
    lap(0);
  }
  // overflow lists past their threshold (counters copied back after an
  // earlier check step, whose launches have completed by now): re-lay out
  // those jobs, in stream order
  for (ServeJob *j : s->active) {
    if (j->ovf_step < 0 || s->steps < j->ovf_step + 2) continue;
    const int *h = s->h_ovf + (j->id % SERVE_ERR_SLOTS) * SPB_SIM_MAX_SPECIES;
    bool over = false;
    for (size_t i = 0; i < j->sim->sp.size(); ++i)
      over |= h[i] > spb::relayout_threshold(j->sim->sp[i]);
    j->ovf_step = -1;
    j->cycles_checked = j->cycles_copied;
    if (over) {
      if (int rc = spb_sim_resort(j->sim, s->st)) return -rc;
      j->cycles_checked = j->cycles;   // the lists are empty again from here
    }
  }
  lap(1);
  // this step's launches (asynchronous): one cycle of every admitted job,
  // then further cycles for the jobs with cycles left, cheapest first, while
  // the added cost stays within extra_budget of the first launch's; a job
  // gets further cycles only while its overflow lists were checked within
  // the last 2 x check_every cycles (so that they cannot fill unseen)
  const std::vector<ServeJob *> ran = s->active;
  if (!ran.empty()) {
    std::vector<spb_sim *> sims;
    sims.reserve(ran.size());
    double first = 0.0;
    for (ServeJob *j : ran) {
      sims.push_back(j->sim);
      first += cycle_cost(j);
      j->cycles++;
    }
    if (int rc = launch_jobs(sims.data(), (int)sims.size(), s->buf[0], s->st)) return -rc;
    if (s->d.extra_budget > 0.0) {
      std::vector<std::pair<double, ServeJob *>> cand;
      for (ServeJob *j : ran) cand.emplace_back(cycle_cost(j), j);
      std::stable_sort(cand.begin(), cand.end(),
                       [](const std::pair<double, ServeJob *> &a,
                          const std::pair<double, ServeJob *> &b) { return a.first < b.first; });
      double budget = s->d.extra_budget * first;
      for (int L = 1; L < SERVE_LAUNCHES && budget > 0.0; ++L) {
        sims.clear();
        double spent = 0.0;
        for (auto &c : cand)
          if (c.second->cycles < c.second->d.ncycles && spent + c.first <= budget &&
              c.second->cycles - c.second->cycles_checked < 2 * s->d.check_every) {
            sims.push_back(c.second->sim);
            spent += c.first;
            c.second->cycles++;
          }
        if (sims.empty()) break;
        if (int rc = launch_jobs(sims.data(), (int)sims.size(), s->buf[L], s->st)) return -rc;
        budget -= spent;
      }
    }
    // the jobs whose last cycle is launched: their error words come back
    // and an event marks their completion; the others' overflow counters
    // come back every check_every of their cycles
    std::vector<ServeJob *> still;
    for (ServeJob *j : ran) {
      if (j->cycles < j->d.ncycles) {
        if (j->ovf_step < 0 && j->cycles - j->cycles_copied >= s->d.check_every) {
          int *h = s->h_ovf + (j->id % SERVE_ERR_SLOTS) * SPB_SIM_MAX_SPECIES;
          for (size_t i = 0; i < j->sim->sp.size(); ++i)
            SPB_CUDA(cudaMemcpyAsync(h + i, j->sim->sp[i].ocnt + j->sim->sp[i].cur, sizeof(int),
                                     cudaMemcpyDeviceToHost, s->st));
          j->ovf_step = s->steps;
          j->cycles_copied = j->cycles;
        }
        still.push_back(j);
        continue;
      }
      if (!j->done) SPB_CUDA(cudaEventCreateWithFlags(&j->done, cudaEventDisableTiming));
      SPB_CUDA(cudaMemcpyAsync(s->h_err + j->id % SERVE_ERR_SLOTS, j->sim->d_err, sizeof(int),
                               cudaMemcpyDeviceToHost, s->st));
      SPB_CUDA(cudaEventRecord(j->done, s->st));
      s->finishing.push_back(j);
    }
    s->active.swap(still);
    s->steps++;
  }
  lap(2);
  // while the launches run: admit what fits; those jobs join the next step
  if (!idle) {
    if (int rc = admit_pending(joined)) return -rc;
    s->active.insert(s->active.end(), joined.begin(), joined.end());
    lap(0);
  }
  // at most one step in flight beyond this one: wait for the previous step's
  // launches, not for this step's, so the host prepares the next step while
  // the GPU runs this one
  const int cur = (int)(s->steps & 1);
  if (!ran.empty()) {
    if (s->step_pending[cur ^ 1]) SPB_CUDA(cudaEventSynchronize(s->step_done[cur ^ 1]));
    SPB_CUDA(cudaEventRecord(s->step_done[cur], s->st));
    s->step_pending[cur ^ 1] = false;
    s->step_pending[cur] = true;
  } else {
    // nothing launched: wait for whatever is still finishing
    SPB_CUDA(cudaStreamSynchronize(s->st));
    s->step_pending[0] = s->step_pending[1] = false;
  }
  lap(2);
  // with nothing else to launch or admit, wait for the finishing jobs (there
  // is no next step to prepare meanwhile)
  if (int rc = retire(s, ran.empty() || (s->active.empty() && s->pending.empty()))) return -rc;
  lap(3);
  return (int)(s->active.size() + s->finishing.size());
}

extern "C" int spb_serve_finished(spb_serve *s, long *ids, int max) {
  if (!s || (max > 0 && !ids)) return -fail(SPB_ERR_INVALID, "spb_serve_finished: bad arguments");
  const int n = std::min<int>(max, (int)s->finished.size());
  for (int i = 0; i < n; ++i) ids[i] = s->finished[i];
  s->finished.erase(s->finished.begin(), s->finished.begin() + n);
  return n;
}

extern "C" int spb_serve_stats(const spb_serve *s, double out[5]) {
  if (!s || !out) return fail(SPB_ERR_INVALID, "spb_serve_stats: null argument");
  out[0] = (double)s->steps;
  for (int i = 0; i < 4; ++i) out[1 + i] = s->phase_s[i];
  return SPB_OK;
}

extern "C" int spb_serve_status(const spb_serve *s, long id) {
  const ServeJob *j = s ? find_job(s, id) : nullptr;
  return j ? j->state : -1;
}

extern "C" int spb_serve_error(const spb_serve *s, long id) {
  const ServeJob *j = s ? find_job(s, id) : nullptr;
  return j ? j->error : SPB_ERR_INVALID;
}

extern "C" int spb_serve_result(spb_serve *s, long id, int species, float *x, float *y, float *z,
                                float *u, float *v, float *w, float *q, double *moments,
                                int on_device) {
  ServeJob *j = s ? find_job(s, id) : nullptr;
  if (!j || j->state != SPB_JOB_DONE)
    return fail(SPB_ERR_INVALID, "spb_serve_result: no finished job with this id");
  if (species < 0 || species >= j->d.ns)
    return fail(SPB_ERR_INVALID, "spb_serve_result: bad species");
  if (x && y && z && u && v && w)
    if (int rc = spb_sim_particles(j->sim, species, x, y, z, u, v, w, q, on_device, s->st))
      return rc;
  if (moments)
    if (int rc = spb_sim_moments(j->sim, species, moments, on_device, s->st)) return rc;
  SPB_CUDA(cudaStreamSynchronize(s->st));
  return SPB_OK;
}

extern "C" int spb_serve_times(const spb_serve *s, long id, double t[3]) {
  const ServeJob *j = s ? find_job(s, id) : nullptr;
  if (!j || !t) return fail(SPB_ERR_INVALID, "spb_serve_times: unknown job");
  for (int i = 0; i < 3; ++i) t[i] = j->t[i];
  return SPB_OK;
}

extern "C" int spb_serve_release(spb_serve *s, long id) {
  ServeJob *j = s ? find_job(s, id) : nullptr;
  if (!j || (j->state != SPB_JOB_DONE && j->state != SPB_JOB_FAILED))
    return fail(SPB_ERR_INVALID, "spb_serve_release: no finished job with this id");
  if (j->state == SPB_JOB_DONE) s->used -= j->bytes;
  s->jobs.erase(id);
  return SPB_OK;
}

extern "C" int spb_serve_counts(const spb_serve *s, int *pending, int *active, int *done,
                                long long *bytes_held, long long *budget) {
  if (!s) return fail(SPB_ERR_INVALID, "spb_serve_counts: null engine");
  int nd = 0;
  for (const auto &kv : s->jobs)
    if (kv.second->state == SPB_JOB_DONE || kv.second->state == SPB_JOB_FAILED) ++nd;
  if (pending) *pending = (int)s->pending.size();
  if (active) *active = (int)s->active.size();
  if (done) *done = nd;
  if (bytes_held) *bytes_held = s->used;
  if (budget) *budget = s->budget;
  return SPB_OK;
}
