"""Serving form on the GPU: independent frozen-field jobs of different grids
and particle counts, stepped together in shared launches.

Bars:
  - each job's moments after its cycles: relative L2 <= 1e-5 against the FP64
    oracle, and <= 1e-5 between the job run alone and the same job run in a
    mix with others that arrive while it runs;
  - each job's particles (tagged by charge) against the FP64 oracle with the
    precision form's tolerances (positions 1e-5, velocities 1e-5 relative);
  - admission holds a job back while the budget is taken and admits it once
    the running job is released; a job larger than the budget fails with
    SPB_ERR_CAPACITY instead of blocking the queue.
"""
import numpy as np
import pytest

import oracle
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def orc64():
    return oracle.CpuOracle("restated", 64)


def make_job(torch, wl, ncycles, species, tags=False):
    from sputnipic_b200.serve import Job
    fields = [torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in W.gem_fields(wl)]
    parts = []
    for s in species:
        p = W.gem_particles(wl, s)
        d = {k: torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in "xyzuvwq"}
        if tags:
            d["q"] = torch.arange(len(p["x"]), dtype=torch.float32, device="cuda")
        parts.append(d)
    return Job(wl=wl, fields=fields, parts=parts, ncycles=ncycles, species=list(species))


def jobs_spec():
    """Three grids, particle counts and cycle counts (tile 4x4x4)."""
    a = W.small_gem(nxc=16, nyc=8, nzc=8, E_amp=1e-3, species=W.gem_species((8, 8, 8, 8)))
    b = W.small_gem(E_amp=1e-3)
    c = W.small_gem(nxc=8, nyc=8, nzc=4, E_amp=1e-3, species=W.gem_species((40, 40, 40, 40)))
    return [(a, 5, [0, 1]), (b, 3, [0, 1, 2, 3]), (c, 7, [2])]


def oracle_run(orc64, wl, part, qom, ncycles):
    setup = oracle.setup_from(wl)
    F = [f.astype(np.float64) for f in W.gem_fields(wl)]
    p = {k: part[k].astype(np.float64) for k in "xyzuvwq"}
    for _ in range(ncycles):
        orc64.mover_pc(setup, F, p, qom)
    mom = [np.zeros(wl.nodes) for _ in range(10)]
    orc64.interp_p2g(setup, p, mom)
    return p, np.stack(mom)


def rel_l2(a, b):
    nb = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(nb == 0, 1, nb)


def run(torch, specs, arrivals_steps, tags=False, **server_kw):
    """Submits specs[i] before step arrivals_steps[i]; steps until all are done.
    Returns {i: {species: results}} and {i: times}."""
    from sputnipic_b200.serve import DONE, Server
    srv = Server(**server_kw)
    jobs = [make_job(torch, wl, nc, sp, tags) for wl, nc, sp in specs]
    ids, out, times = {}, {}, {}
    step = 0
    while len(out) < len(jobs):
        for i, at in enumerate(arrivals_steps):
            if at == step and i not in ids:
                ids[i] = srv.submit(jobs[i])
        srv.step()
        step += 1
        for i, jid in ids.items():
            if i in out or srv.status(jid) != DONE:
                continue
            wl = jobs[i].wl
            out[i] = {s: {k: v.cpu().numpy() for k, v in
                          srv.result(jid, s, p["x"].numel(), wl.nodes).items()}
                      for s, p in enumerate(jobs[i].parts)}
            times[i] = srv.times(jid)
            srv.release(jid)
        assert step < 200
    srv.close()
    return out, times


def test_results_alone_equal_results_in_mix(cuda, orc64):
    torch = cuda
    specs = jobs_spec()
    alone = {i: run(torch, [spec], [0])[0][0] for i, spec in enumerate(specs)}
    # job 0 starts alone; jobs 1 and 2 arrive while it runs
    mix, times = run(torch, specs, [0, 2, 3])
    assert times[1][1] > times[0][1] and times[1][1] < times[0][2]   # overlapped with job 0
    for i, (wl, nc, species) in enumerate(specs):
        for s, ws in enumerate(species):
            m_alone, m_mix = alone[i][s]["moments"], mix[i][s]["moments"]
            assert (rel_l2(m_mix, m_alone) <= 1e-5).all(), (i, s)
            _, m64 = oracle_run(orc64, wl, W.gem_particles(wl, ws), wl.species[ws].qom, nc)
            assert (rel_l2(m_mix, m64) <= 1e-5).all(), (i, s, rel_l2(m_mix, m64))


def test_particles_in_mix_vs_fp64(cuda, orc64):
    torch = cuda
    specs = jobs_spec()
    mix, _ = run(torch, specs, [0, 1, 1], tags=True)
    for i, (wl, nc, species) in enumerate(specs):
        for s, ws in enumerate(species):
            part = W.gem_particles(wl, ws)
            tagged = dict(part)
            tagged["q"] = np.arange(len(part["x"]), dtype=np.float32)
            ref, _ = oracle_run(orc64, wl, tagged, wl.species[ws].qom, nc)
            got = mix[i][s]
            order = np.argsort(got["q"])
            assert np.array_equal(got["q"][order], np.arange(len(order), dtype=np.float32))
            for k in "xyz":
                assert np.abs(got[k][order].astype(np.float64) - ref[k]).max() <= 1e-5, (i, k)
            for k in "uvw":
                scale = np.abs(ref[k]).max() + 1e-30
                assert np.abs(got[k][order].astype(np.float64) - ref[k]).max() <= 1e-5 * scale


def steps_to_finish(torch, specs, watch, **server_kw):
    """Submits every spec at step 0 and steps until job `watch` is DONE.
    Returns the steps taken and that job's results (species 0)."""
    from sputnipic_b200.serve import DONE, Server
    srv = Server(**server_kw)
    jobs = [make_job(torch, wl, nc, sp) for wl, nc, sp in specs]
    ids = [srv.submit(j) for j in jobs]
    steps = 0
    while srv.status(ids[watch]) != DONE:
        srv.step()
        steps += 1
        assert steps < 200
    wl = jobs[watch].wl
    res = {k: v.cpu().numpy() for k, v in
           srv.result(ids[watch], 0, jobs[watch].parts[0]["x"].numel(), wl.nodes).items()}
    srv.close()
    return steps, res


def test_extra_cycles_for_cheap_jobs(cuda, orc64):
    """A 40-cycle 16x8x8 job (16K particles) beside a 40-cycle 32x16x16 one
    (884K). Each further launch of a step gives one more cycle to every job
    with cycles left whose cost still fits the budget, cheapest first: with
    the default budget (0, read as 1.0 x the first launch's cost) one such
    launch fits both jobs (two cycles a step); with 8.0 all seven further
    launches do (eight cycles a step, one while a check of the job's
    overflow lists is outstanding: 40 cycles in 9 steps); with extra cycles
    off (negative) each job gets one cycle a step. The cheap job's moments are the same in all
    three, within 1e-5 of the FP64 oracle."""
    torch = cuda
    cheap = W.small_gem(nxc=16, nyc=8, nzc=8, E_amp=1e-3, species=W.gem_species((8, 8, 8, 8)))
    big = W.small_gem(E_amp=1e-3)
    specs = [(big, 40, [0, 1, 2, 3]), (cheap, 40, [0, 1])]
    steps, res = {}, {}
    for budget in (0.0, 8.0, -1.0):
        steps[budget], res[budget] = steps_to_finish(torch, specs, 1, extra_budget=budget)
    assert steps[8.0] <= 11, steps
    assert 20 <= steps[0.0] <= 22, steps
    assert steps[-1.0] >= 40, steps
    _, m64 = oracle_run(orc64, cheap, W.gem_particles(cheap, 0), cheap.species[0].qom, 40)
    for budget in res:
        assert (rel_l2(res[budget]["moments"], res[-1.0]["moments"]) <= 1e-5).all(), budget
        assert (rel_l2(res[budget]["moments"], m64) <= 1e-5).all(), budget


def test_admission_waits_for_budget(cuda):
    torch = cuda
    from sputnipic_b200.serve import ACTIVE, PENDING, Server
    wl, nc, species = jobs_spec()[0]
    probe = Server()
    jid = probe.submit(make_job(torch, wl, 1, species))
    probe.step()
    one = probe.counts()["bytes"]
    probe.close()
    assert one > 0
    # room for one job at a time: the second waits until the first is released
    out, times = run(torch, [(wl, nc, species), (wl, nc, species)], [0, 0],
                     hbm_budget=int(1.5 * one))
    assert times[1][1] >= times[0][2]
    srv = Server(hbm_budget=int(1.5 * one))
    a = srv.submit(make_job(torch, wl, nc, species))
    b = srv.submit(make_job(torch, wl, nc, species))
    srv.step()
    assert srv.status(a) == ACTIVE and srv.status(b) == PENDING
    assert srv.counts()["bytes"] <= int(1.5 * one)
    srv.close()
    for s in range(len(species)):
        assert (rel_l2(out[1][s]["moments"], out[0][s]["moments"]) <= 1e-5).all()


def test_job_larger_than_budget_fails(cuda):
    torch = cuda
    from sputnipic_b200 import _lib
    from sputnipic_b200.serve import DONE, FAILED, Server
    wl, nc, species = jobs_spec()[0]
    srv = Server(hbm_budget=1 << 20)
    big = srv.submit(make_job(torch, wl, nc, species))
    srv.step()
    assert srv.status(big) == FAILED
    assert srv.lib.spb_serve_error(srv.h, big) == 8   # SPB_ERR_CAPACITY
    srv.release(big)
    srv.close()
    # a fitting job behind it is not blocked
    srv = Server()
    ok = srv.submit(make_job(torch, wl, 1, species))
    srv.step()
    assert srv.status(ok) == DONE
    srv.close()
    assert _lib.load() is not None
