"""Serving form: a stream of independent frozen-field test-particle jobs of
different grids and particle counts (spb_serve_* of libsputnipic_b200.so).

A `Server` queues jobs as they arrive, admits them when their HBM footprint
fits, and advances every admitted job at least one cycle per `step()` (one
launch per kernel for all of them, and further launches that give cheap jobs
more cycles within the engine's extra budget). `run_stream` is the request
loop: it submits jobs at their arrival times (wall clock), steps while
anything is queued or running, and reports each job's latency (arrival to
finish) and the aggregate throughput.
See include/sputnipic_b200.h.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field

from . import _lib

PENDING, ACTIVE, DONE, FAILED = 0, 1, 2, 3


@dataclass
class Job:
    """One test-particle job: a workload's grid and species, its fields
    (six float32 tensors) and per-species particle dicts (x..q float32 tensors,
    all on the device or all on the host), and the cycles to run."""
    wl: object
    fields: list
    parts: list
    ncycles: int
    species: list = None   # workload species indices of `parts` (default 0..)
    tag: object = None

    def particles(self) -> int:
        return sum(p["x"].numel() for p in self.parts)


@dataclass
class Finished:
    id: int
    job: Job
    times: tuple            # (submitted, admitted, finished), engine seconds
    status: int
    results: dict = field(default_factory=dict)
    late: float = 0.0       # seconds between the job's arrival and its submission
    error: int = 0          # status code of a failed job

    @property
    def latency(self) -> float:
        """Arrival to finish: the engine's submission-to-finish time plus the
        time the job waited for the request loop to submit it."""
        return self.times[2] - self.times[0] + self.late


class Server:
    def __init__(self, tile=(4, 4, 4), hbm_budget=0, max_jobs=64, check_every=4,
                 reserve_bytes=0, extra_budget=0.0):
        self.lib = _lib.load()
        d = _lib.ServeDesc()
        for a in range(3):
            d.tile[a] = tile[a]
        d.hbm_budget, d.max_jobs, d.check_every = int(hbm_budget), max_jobs, check_every
        d.reserve_bytes = int(reserve_bytes)
        d.extra_budget = float(extra_budget)
        h = ctypes.c_void_p()
        _lib.check(self.lib.spb_serve_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h
        self._inputs = {}   # id -> (job, pointer arrays): kept alive until admitted
        self.release_s = 0.0   # host seconds spent releasing finished jobs

    def close(self):
        if self.h:
            self.lib.spb_serve_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, job: Job) -> int:
        wl = job.wl
        species = job.species or list(range(len(job.parts)))
        d = _lib.JobDesc()
        d.nxc, d.nyc, d.nzc = wl.nxc, wl.nyc, wl.nzc
        d.Lx, d.Ly, d.Lz = wl.Lx, wl.Ly, wl.Lz
        d.dt, d.c, d.niter = wl.dt, wl.c, wl.niter
        for a in range(3):
            d.periodic[a] = 1 if wl.periodic[a] else 0
        d.ns = len(job.parts)
        for i, s in enumerate(species):
            d.qom[i] = wl.species[s].qom
        d.ncycles = job.ncycles
        on_dev = int(job.fields[0].is_cuda)
        f = (ctypes.c_void_p * 6)(*[t.data_ptr() for t in job.fields])
        ptrs = [p[k].data_ptr() for p in job.parts for k in "xyzuvwq"]
        pa = (ctypes.c_void_p * len(ptrs))(*ptrs)
        counts = (ctypes.c_long * d.ns)(*[p["x"].numel() for p in job.parts])
        jid = self.lib.spb_serve_submit(self.h, ctypes.byref(d), f, pa, counts, on_dev)
        if jid < 0:
            _lib.check(-jid)
        self._inputs[jid] = (job, f, pa, counts)
        return jid

    def step(self) -> int:
        n = self.lib.spb_serve_step(self.h)
        if n < 0:
            _lib.check(-n)
        self._steps = getattr(self, "_steps", 0) + 1
        if self._steps % 8 == 0 or n == 0:
            # admitted (or failed) jobs' inputs are no longer read
            for jid in [j for j in self._inputs if self.status(j) != PENDING]:
                del self._inputs[jid]
        return n

    def finished(self) -> list:
        """Ids of the jobs that finished (done or failed) since the last call."""
        out = []
        buf = (ctypes.c_long * 256)()
        while True:
            k = self.lib.spb_serve_finished(self.h, buf, 256)
            if k < 0:
                _lib.check(-k)
            out.extend(buf[:k])
            if k < 256:
                return out

    def status(self, jid: int) -> int:
        return self.lib.spb_serve_status(self.h, jid)

    def error(self, jid: int) -> int:
        """Status code of a failed job (why it failed)."""
        return self.lib.spb_serve_error(self.h, jid)

    def times(self, jid: int) -> tuple:
        t = (ctypes.c_double * 3)()
        _lib.check(self.lib.spb_serve_times(self.h, jid, t))
        return tuple(t)

    def counts(self) -> dict:
        p, a, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        held, budget = ctypes.c_longlong(), ctypes.c_longlong()
        _lib.check(self.lib.spb_serve_counts(self.h, ctypes.byref(p), ctypes.byref(a),
                                             ctypes.byref(d), ctypes.byref(held),
                                             ctypes.byref(budget)))
        return {"pending": p.value, "active": a.value, "done": d.value, "bytes": held.value,
                "budget": budget.value}

    def result(self, jid: int, species: int, nparticles: int, nodes: int,
               particles=True) -> dict:
        """Particles (float32 CUDA tensors x..q) and raw FP64 moments (10, nodes)
        of one species of a finished job."""
        import torch
        mom = torch.empty(10, nodes, dtype=torch.float64, device="cuda")
        out = {}
        ptr = [None] * 7
        if particles:
            out = {k: torch.empty(nparticles, dtype=torch.float32, device="cuda")
                   for k in "xyzuvwq"}
            ptr = [out[k].data_ptr() for k in "xyzuvwq"]
        _lib.check(self.lib.spb_serve_result(self.h, jid, species, *ptr, mom.data_ptr(), 1))
        out["moments"] = mom
        return out

    def release(self, jid: int):
        t = time.perf_counter()
        _lib.check(self.lib.spb_serve_release(self.h, jid))
        self.release_s += time.perf_counter() - t

    def stats(self) -> dict:
        """Steps run and host seconds per phase of the steps."""
        t = (ctypes.c_double * 5)()
        _lib.check(self.lib.spb_serve_stats(self.h, t))
        return {"steps": int(t[0]), "admit_s": t[1], "check_s": t[2], "run_s": t[3],
                "retire_s": t[4]}


def release_cached_memory():
    """Hands the device memory the library's pool keeps for reuse back
    (spb_release_cached_memory)."""
    _lib.check(_lib.load().spb_release_cached_memory())


def run_stream(server: Server, jobs, arrivals, keep=None, idle_sleep=1e-4):
    """The request loop. jobs[i] arrives `arrivals[i]` seconds after the start
    (sorted) and is submitted at the loop's first pass after that. Returns the
    finished jobs (with results for the indices in `keep`; latencies count
    from the arrival) and the wall time of the whole stream."""
    keep = set(keep or ())
    t0 = time.perf_counter()
    i, live, done, late = 0, {}, [], {}
    while i < len(jobs) or live:
        now = time.perf_counter() - t0
        while i < len(jobs) and arrivals[i] <= now:
            jid = server.submit(jobs[i])
            live[jid] = i
            late[jid] = max(0.0, time.perf_counter() - t0 - arrivals[i])
            i += 1
        if not live:
            time.sleep(min(idle_sleep, max(0.0, arrivals[i] - now)))
            continue
        server.step()
        for jid in server.finished():
            idx = live[jid]
            st = server.status(jid)
            job = jobs[idx]
            res = {}
            if st == DONE and idx in keep:
                wl = job.wl
                res = {s: server.result(jid, s, p["x"].numel(), wl.nodes)
                       for s, p in enumerate(job.parts)}
            done.append(Finished(jid, job, server.times(jid), st, res, late.pop(jid),
                                 server.error(jid) if st == FAILED else 0))
            server.release(jid)
            del live[jid]
    return done, time.perf_counter() - t0


SERVING_GRIDS = ((16, 8, 8), (32, 16, 16), (64, 32, 32), (128, 64, 64))
SERVING_GRID_WEIGHTS = (0.4, 0.3, 0.2, 0.1)
SERVING_PPC = (8, 27, 64, 125)


def job_mix(n_configs=12, seed=0, max_particles_per_species=5_000_000, max_cycles=50,
            uniform=False):
    """Seeded mix of job configurations: grid, particles per cell, 2 or 4
    species, 1..max_cycles cycles. Grids weighted SERVING_GRID_WEIGHTS and
    particles per cell lowered where a species would exceed the cap, or, with
    `uniform`, grids drawn uniformly and no cap. Returns (workload, ncycles,
    species) tuples."""
    import numpy as np

    from . import workload as W
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_configs):
        g = SERVING_GRIDS[rng.choice(len(SERVING_GRIDS), p=None if uniform else SERVING_GRID_WEIGHTS)]
        cells = g[0] * g[1] * g[2]
        cap = None if uniform else max_particles_per_species
        ppcs = [p for p in SERVING_PPC if cap is None or p * cells <= cap] or [1]
        ppc = int(rng.choice(ppcs))
        ns = int(rng.choice((2, 4)))
        wl = W.small_gem(nxc=g[0], nyc=g[1], nzc=g[2], E_amp=1e-3, seed=int(rng.integers(1 << 30)),
                         species=W.gem_species((ppc,) * 4))
        out.append((wl, int(rng.integers(1, max_cycles + 1)), list(range(ns))))
    return out


def device_jobs(configs):
    """Jobs with inputs generated on the device (one set per configuration;
    jobs of the same configuration share them: the engine copies inputs at
    admission)."""
    from .device import gen_fields, gen_particles
    jobs = []
    for wl, nc, species in configs:
        fields = gen_fields(wl)
        parts = [gen_particles(wl, s) for s in species]
        jobs.append(Job(wl=wl, fields=fields, parts=parts, ncycles=nc, species=list(species)))
    return jobs


def plain_job_seconds(job) -> float:
    """Wall seconds of one job run alone through the plain path (the
    reference's precision types on device arrays, spb_grid_*): grid context,
    fields, a copy of the particles, then per cycle mover_PC for every species,
    zeroed moments and interpP2G for every species, as the reference's CPU
    driver steps them (src/sputniPIC_CPU.cpp:232-256), synchronised at the end."""
    import torch

    from .device import GridContext, push_params
    wl = job.wl
    species = job.species or list(range(len(job.parts)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ctx = GridContext(wl)
    ctx.set_fields(job.fields)
    parts = [{k: p[k].clone() for k in "xyzuvwq"} for p in job.parts]
    pushes = [push_params(wl, s) for s in species]
    mom = torch.zeros(len(parts), 10, wl.nodes, device="cuda")
    for _ in range(job.ncycles):
        for p, push in zip(parts, pushes):
            ctx.mover(p, push)
        mom.zero_()
        for i, p in enumerate(parts):
            ctx.p2g(p, mom[i])
    rc = ctx.check()
    t = time.perf_counter() - t0
    ctx.close()
    if rc:
        raise RuntimeError(f"plain job status {rc}")
    return t


def fifo_latencies(arrivals, service):
    """Latencies of jobs served one at a time in order of arrival (a single
    server, no overlap): each starts when it has arrived and the previous one
    has finished. Returns (latencies, finish time of the last job)."""
    t, lat = 0.0, []
    for a, d in zip(arrivals, service):
        t = max(t, a) + d
        lat.append(t - a)
    return lat, t


def measure_stream(rate=10.0, njobs=100, n_configs=12, seed=0, tile=(4, 4, 4), rates=None,
                   extra_budget=0.0, uniform=False, reserve_fraction=0.6):
    """Poisson streams of `njobs` jobs drawn from a seeded mix of
    configurations, at `rate` jobs/s or at each of `rates`. Every
    configuration is also run alone, three times (its single-job latency is
    the median of the three). Returns per
    rate the latency percentiles, slowdowns against running alone and the
    aggregate throughput in particle-cycles per second (the first rate's also
    at the top level). The engines of the burst, the single-job runs and the
    streams map `reserve_fraction` of their budget into the memory pool when
    they are created (spb_serve_desc.reserve_bytes), so that admissions during
    a stream do not wait for the pool to grow."""
    import numpy as np
    configs = job_mix(n_configs, seed, uniform=uniform)
    pool = device_jobs(configs)
    # warm-up: the engine's kernels for this tile shape loaded and configured
    # once, outside the single-job latencies
    srv = Server(tile=tile, extra_budget=extra_budget)
    run_stream(srv, [pool[0]], [0.0])
    srv.close()
    # the baseline: every configuration alone through the plain path (warm;
    # before the engine's pool grows, as its copies come from torch)
    plain_job_seconds(pool[0])
    plain = [plain_job_seconds(job) for job in pool]
    probe = Server(tile=tile)
    reserve = int(reserve_fraction * probe.counts()["budget"])
    probe.close()
    # warm-up burst of a full launch's worth of jobs (every configuration,
    # repeated), so the device memory pool has grown to a saturated engine's
    # footprint before the single-job runs and the timed streams
    srv = Server(tile=tile, extra_budget=extra_budget, reserve_bytes=reserve)
    burst = [pool[i % len(pool)] for i in range(max(len(pool), 64))]
    run_stream(srv, burst, [0.0] * len(burst))
    srv.close()
    # each configuration's single-job latency: the median of three runs alone
    # (one run that meets a host-side stall does not set it)
    alone = []
    for job in pool:
        runs = []
        for _ in range(3):
            srv = Server(tile=tile, extra_budget=extra_budget, reserve_bytes=reserve)
            done, _ = run_stream(srv, [job], [0.0])
            srv.close()
            assert done[0].status == DONE
            runs.append(done[0].latency)
        alone.append(float(np.median(runs)))
    index = {id(j): k for k, j in enumerate(pool)}
    sweep = []
    for r in (rates or [rate]):
        rng = np.random.default_rng(seed + 1)
        pick = rng.integers(0, len(pool), size=njobs)
        arrivals = np.cumsum(rng.exponential(1.0 / r, size=njobs))
        arrivals -= arrivals[0]
        jobs = [pool[i] for i in pick]
        srv = Server(tile=tile, extra_budget=extra_budget, reserve_bytes=reserve)
        done, wall = run_stream(srv, jobs, list(arrivals))
        stats = srv.stats()
        stats["release_s"] = srv.release_s
        srv.close()
        ok = [d for d in done if d.status == DONE]
        failed = len(done) - len(ok)
        lat = np.array([d.latency for d in ok])
        slow = np.array([d.latency / alone[index[id(d.job)]] for d in ok])
        work = sum(d.job.particles() * d.job.ncycles for d in ok)
        plat, pend = fifo_latencies(list(arrivals), [plain[i] for i in pick])
        sweep.append({
            "rate_jobs_per_s": r, "jobs": njobs, "completed": len(ok), "failed": failed,
            "failure_codes": sorted({d.error for d in done if d.status != DONE}),
            "failed_jobs": [{"config": index[id(d.job)], "code": d.error} for d in done
                            if d.status != DONE],
            "latency_ms": {"p50": 1e3 * float(np.percentile(lat, 50)),
                           "p99": 1e3 * float(np.percentile(lat, 99))},
            "slowdown_vs_alone": {"p50": float(np.percentile(slow, 50)),
                                  "p99": float(np.percentile(slow, 99))},
            "throughput_particle_cycles_per_s": work / wall, "wall_s": wall, "engine": stats,
            "plain_one_at_a_time": {
                "latency_ms": {"p50": 1e3 * float(np.percentile(plat, 50)),
                               "p99": 1e3 * float(np.percentile(plat, 99))},
                "throughput_particle_cycles_per_s":
                    sum(jobs[k].particles() * jobs[k].ncycles for k in range(njobs)) / pend}})
    release_cached_memory()
    out = dict(sweep[0])
    out.update({
        "single_job_latency_ms": {"p50": 1e3 * float(np.percentile(alone, 50)),
                                  "p99": 1e3 * float(np.percentile(alone, 99))},
        "p99_over_single_job_p99": sweep[0]["latency_ms"]["p99"] / (1e3 * float(np.percentile(alone, 99))),
        "extra_budget": extra_budget or 1.0,
        "plain_alone_ms": {"p50": 1e3 * float(np.percentile(plain, 50)),
                           "p99": 1e3 * float(np.percentile(plain, 99))},
        "baseline": ("plain_one_at_a_time: the same stream served one job at a time through the "
                     "plain path (each configuration's wall time alone, measured; FIFO queue "
                     "over the same arrivals)"),
        "mix": (f"{n_configs} configurations: grids {list(SERVING_GRIDS)} drawn uniformly, ppc "
                f"from {list(SERVING_PPC)}, 2 or 4 species, 1-50 cycles, frozen GEM fields; "
                "Poisson arrivals" if uniform else
                f"{n_configs} configurations: grids {list(SERVING_GRIDS)} "
                f"(weights {list(SERVING_GRID_WEIGHTS)}), ppc from {list(SERVING_PPC)} "
                "(capped at 5M particles per species), 2 or 4 species, 1-50 cycles, "
                "frozen GEM fields; Poisson arrivals")})
    if rates:
        out["sweep"] = [{k: v for k, v in e.items() if k != "engine"} for e in sweep]
        for e in out["sweep"]:
            e["p99_over_single_job_p99"] = e["latency_ms"]["p99"] / out["single_job_latency_ms"]["p99"]
    return out
