"""Serving form: a stream of independent frozen-field test-particle jobs of
different grids and particle counts (spb_serve_* of libsputnipic_b200.so).

A `Server` queues jobs as they arrive, admits them when their HBM footprint
fits, and steps every admitted job one cycle per `step()` in one launch per
kernel. `run_stream` is the request loop: it submits jobs at their arrival
times (wall clock), steps while anything is queued or running, and reports
each job's latency (submission to finish) and the aggregate throughput.
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

    @property
    def latency(self) -> float:
        return self.times[2] - self.times[0]


class Server:
    def __init__(self, tile=(4, 4, 4), hbm_budget=0, max_jobs=64, check_every=4):
        self.lib = _lib.load()
        d = _lib.ServeDesc()
        for a in range(3):
            d.tile[a] = tile[a]
        d.hbm_budget, d.max_jobs, d.check_every = int(hbm_budget), max_jobs, check_every
        h = ctypes.c_void_p()
        _lib.check(self.lib.spb_serve_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h
        self._inputs = {}   # id -> (job, pointer arrays): kept alive until admitted

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
        for jid in [j for j in self._inputs if self.status(j) != PENDING]:
            del self._inputs[jid]   # admitted (or failed): inputs no longer read
        return n

    def status(self, jid: int) -> int:
        return self.lib.spb_serve_status(self.h, jid)

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
        _lib.check(self.lib.spb_serve_release(self.h, jid))


def run_stream(server: Server, jobs, arrivals, keep=None, idle_sleep=1e-4):
    """The request loop. jobs[i] arrives `arrivals[i]` seconds after the start
    (sorted). Returns the finished jobs (with results for the indices in
    `keep`) and the wall time of the whole stream."""
    keep = set(keep or ())
    t0 = time.perf_counter()
    i, live, done = 0, {}, []
    while i < len(jobs) or live:
        now = time.perf_counter() - t0
        while i < len(jobs) and arrivals[i] <= now:
            live[server.submit(jobs[i])] = i
            i += 1
        if not live:
            time.sleep(min(idle_sleep, max(0.0, arrivals[i] - now)))
            continue
        server.step()
        for jid, idx in list(live.items()):
            st = server.status(jid)
            if st not in (DONE, FAILED):
                continue
            job = jobs[idx]
            res = {}
            if st == DONE and idx in keep:
                wl = job.wl
                res = {s: server.result(jid, s, p["x"].numel(), wl.nodes)
                       for s, p in enumerate(job.parts)}
            done.append(Finished(jid, job, server.times(jid), st, res))
            server.release(jid)
            del live[jid]
    return done, time.perf_counter() - t0
