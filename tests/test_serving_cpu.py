"""Host logic of the serving form without a GPU: the request loop submits
jobs at their arrival times, steps while anything is queued or running, and
collects each finished job once (a fake engine stands in for spb_serve_*);
the job mix is seeded and respects its caps."""
import time

from sputnipic_b200 import serve


class FakeJob:
    def __init__(self, cycles, n=10):
        self.ncycles, self.n, self.parts, self.wl = cycles, n, [], None

    def particles(self):
        return self.n


class FakeServer:
    """Admits at most `slots` jobs; each step advances every admitted job one
    cycle. Records the step at which each job was submitted and finished, and
    reports the newly finished ids (finished())."""

    def __init__(self, slots=2):
        self.slots, self.t0, self.jobs, self.order, self.steps = slots, time.perf_counter(), {}, [], 0
        self.next_id = 0
        self.newly_done = []

    def submit(self, job):
        jid = self.next_id
        self.next_id += 1
        self.jobs[jid] = {"job": job, "left": job.ncycles, "state": serve.PENDING,
                          "t": [time.perf_counter() - self.t0, -1.0, -1.0]}
        self.order.append(jid)
        return jid

    def step(self):
        active = [j for j in self.jobs.values() if j["state"] == serve.ACTIVE]
        for jid in self.order:
            j = self.jobs[jid]
            if j["state"] == serve.PENDING and len(active) < self.slots:
                j["state"] = serve.ACTIVE
                j["t"][1] = time.perf_counter() - self.t0
                active.append(j)
        for jid, j in self.jobs.items():
            if j in active:
                j["left"] -= 1
                if j["left"] == 0:
                    j["state"] = serve.DONE
                    j["t"][2] = time.perf_counter() - self.t0
                    self.newly_done.append(jid)
        self.steps += 1
        return sum(1 for j in self.jobs.values() if j["state"] == serve.ACTIVE)

    def finished(self):
        out, self.newly_done = self.newly_done, []
        return out

    def status(self, jid):
        return self.jobs[jid]["state"] if jid in self.jobs else -1

    def times(self, jid):
        return tuple(self.jobs[jid]["t"])

    def release(self, jid):
        assert self.jobs[jid]["state"] == serve.DONE
        del self.jobs[jid]
        self.order.remove(jid)


def test_request_loop_runs_every_job_once_in_arrival_order():
    srv = FakeServer(slots=2)
    jobs = [FakeJob(c) for c in (3, 1, 2, 5, 1)]
    arrivals = [0.0, 0.0, 0.002, 0.004, 0.03]
    done, wall = serve.run_stream(srv, jobs, arrivals)
    assert sorted(d.id for d in done) == list(range(5))
    assert all(d.status == serve.DONE for d in done)
    by_id = {d.id: d for d in done}
    for jid, arr in enumerate(arrivals):
        t = by_id[jid].times
        assert t[0] >= arr - 1e-3 and t[0] <= t[1] <= t[2]
        assert by_id[jid].latency >= 0
    # with two slots, the third job cannot start before one of the first two ended
    assert by_id[2].times[1] >= min(by_id[0].times[2], by_id[1].times[2])
    assert wall >= arrivals[-1]
    assert not srv.jobs   # every finished job was released


def test_job_mix_is_seeded_and_capped():
    a = serve.job_mix(n_configs=20, seed=3)
    b = serve.job_mix(n_configs=20, seed=3)
    assert [(w.nxc, w.nyc, w.nzc, w.species[0].ppc, c, s) for w, c, s in a] == \
        [(w.nxc, w.nyc, w.nzc, w.species[0].ppc, c, s) for w, c, s in b]
    for wl, ncycles, species in a:
        assert (wl.nxc, wl.nyc, wl.nzc) in serve.SERVING_GRIDS
        assert 1 <= ncycles <= 50 and len(species) in (2, 4)
        assert wl.species_count(0) <= 5_000_000
        assert wl.nxc % 4 == 0 and wl.nyc % 4 == 0 and wl.nzc % 4 == 0


def test_uniform_job_mix_draws_grids_evenly_without_cap():
    """The configuration's own mix: every grid about equally often, every
    ppc on every grid (up to 65.5M particles per species)."""
    mix = serve.job_mix(n_configs=400, seed=5, uniform=True)
    grids = [(w.nxc, w.nyc, w.nzc) for w, _, _ in mix]
    for g in serve.SERVING_GRIDS:
        assert 0.18 <= grids.count(g) / len(grids) <= 0.32, g
    big = [w for w, _, _ in mix if (w.nxc, w.nyc, w.nzc) == (128, 64, 64)]
    assert max(w.species[0].ppc for w in big) == 125
    assert max(w.species_count(0) for w, _, _ in mix) == 128 * 64 * 64 * 125
