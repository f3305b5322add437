"""The precision form's deterministic mode (spb_sim_desc.deterministic).

Particles reach their buckets through atomics, so their order inside a
bucket, the overflow lists and the FP64 atomics differ from run to run. In the
deterministic mode every deposit term is rounded down to a power-of-two grid
and summed exactly, and a particle's push is the same whichever path serves it
(staged tile or L2, bucket or overflow list), so:
  - two runs from the same inputs give bitwise identical moments and the same
    particles (compared as sorted multisets), over many cycles with CUDA
    graphs, forced overflows and re-layouts;
  - the moments still match the FP64 oracle (relative L2 <= 1e-5 per moment,
    the precision form's bar), no less closely than the default deposit's.
"""
import numpy as np
import pytest

import oracle
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu


def run(torch, wl, fields, cycles, deterministic, bucket_slots=0, resort_every=2, graph=True):
    from sputnipic_b200.device import gen_particles
    from sputnipic_b200.sim import Simulation
    sim = Simulation(wl, resort_every=resort_every, graph=graph, deterministic=deterministic,
                     bucket_slots=bucket_slots)
    sim.set_fields(fields)
    for s in range(len(wl.species)):
        sim.load_species(s, gen_particles(wl, s))
    sim.cycle(cycles)
    assert sim.check() == 0
    mom = [sim.moments(s).cpu().numpy() for s in range(len(wl.species))]
    parts = []
    for s in range(len(wl.species)):
        p = sim.particles(s)
        a = np.stack([p[k].cpu().numpy().view(np.uint32) for k in "xyzuvwq"], axis=1)
        parts.append(a[np.lexsort(a.T[::-1])])
    overflow = [sim.overflow(s) for s in range(len(wl.species))]
    sim.close()
    return mom, parts, overflow


@pytest.mark.parametrize("bucket_slots", [0, 96])
def test_two_runs_bitwise_identical(cuda, bucket_slots):
    """Uneven species (125, 125, 12.5, 12.5 ppc) on a 64x32x32 GEM grid, 12
    cycles with graphs and overflow checks every 2 cycles; bucket_slots=96
    fixes every bucket below the 125-particle mean, so many particles go
    through the overflow lists (pushed from L2, deposited entry by entry)."""
    torch = cuda
    from sputnipic_b200.device import gen_fields
    wl = W.batching_gem(nxc=64, nyc=32, nzc=32, Lx=10.0, Ly=5.0, Lz=5.0)
    fields = gen_fields(wl)
    m1, p1, o1 = run(torch, wl, fields, 12, True, bucket_slots)
    m2, p2, o2 = run(torch, wl, fields, 12, True, bucket_slots)
    if bucket_slots:                                # the dense species overflowed
        assert min(o1[:2]) > 0 and min(o2[:2]) > 0
    for s in range(len(wl.species)):
        assert np.array_equal(m1[s].view(np.uint64), m2[s].view(np.uint64)), s
        assert np.array_equal(p1[s], p2[s]), s
        assert np.abs(m1[s]).max() > 0


def test_deterministic_moments_match_oracle_and_default(cuda):
    """One cycle of the small GEM configuration: the deterministic moments
    against the FP64 oracle and against the default deposit."""
    torch = cuda
    from sputnipic_b200.sim import Simulation
    wl = W.small_gem(E_amp=1e-3)
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    got = {}
    for det in (False, True):
        sim = Simulation(wl, resort_every=10**6, deterministic=det)
        sim.set_fields([T(f) for f in fields])
        for s, p in enumerate(parts):
            sim.load_species(s, {k: T(p[k]) for k in "xyzuvwq"})
        sim.cycle(1)
        assert sim.check() == 0
        got[det] = [sim.moments(s).cpu().numpy() for s in range(4)]
        sim.close()
    orc64 = oracle.CpuOracle("restated", 64)
    setup = oracle.setup_from(wl)
    F64 = [f.astype(np.float64) for f in fields]
    for s in range(4):
        p = {k: parts[s][k].astype(np.float64) for k in "xyzuvwq"}
        orc64.mover_pc(setup, F64, p, wl.species[s].qom)
        mom = [np.zeros(wl.nodes) for _ in range(10)]
        orc64.interp_p2g(setup, p, mom)
        ref = np.stack(mom)
        err = {}
        for det in (True, False):
            err[det] = np.linalg.norm(got[det][s] - ref, axis=1) / np.linalg.norm(ref, axis=1)
            assert (err[det] <= 1e-5).all(), (s, det, err[det])
        # exact sums of the same FP32 terms: no less accurate than the default
        # deposit's FP32 cell sums
        assert err[True].max() <= err[False].max() + 1e-8, (s, err[True], err[False])


def test_species_loaded_at_rest_stays_exact(cuda):
    """Every particle at rest when loaded (the velocity bound of the grids
    falls back to c/8): six cycles of the small GEM configuration accelerate
    them without any sum leaving its exact range, and two runs agree
    bitwise."""
    torch = cuda
    wl = W.small_gem(E_amp=1e-3)
    fields = [torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in W.gem_fields(wl)]
    out = []
    for _ in range(2):
        from sputnipic_b200.sim import Simulation
        sim = Simulation(wl, resort_every=2, graph=True, deterministic=True)
        sim.set_fields(fields)
        for s in range(len(wl.species)):
            p = W.gem_particles(wl, s)
            for k in "uvw":
                p[k] = np.zeros_like(p[k])
            sim.load_species(s, {k: torch.from_numpy(np.ascontiguousarray(p[k])).cuda()
                                 for k in "xyzuvwq"})
        sim.cycle(6)
        assert sim.check() == 0
        mom = [sim.moments(s).cpu().numpy() for s in range(len(wl.species))]
        assert np.abs(mom[0][1:4]).max() > 0   # the electrons carry current
        out.append(mom)
        sim.close()
    for a, b in zip(*out):
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.mark.parametrize("n, flagged", [(24000, True), (12000, False)])
def test_cell_sum_past_exact_range_is_reported(cuda, n, flagged):
    """n particles at rest near the lower corner of one cell, charge -1e-3
    (max|q| = 1e-3, grid 2^-38 x 2^-9): that cell's rhon sum at the corner node
    is about 0.86 n x 1e-3, against the exact range of 2^13 x 2^-9 = 16. 24,000
    particles (about 20.6) leave it and spb_sim_check reports SPB_ERR_CAPACITY;
    12,000 (about 10.3) stay inside."""
    torch = cuda
    from sputnipic_b200.sim import Simulation
    wl = W.small_gem(E_amp=1e-3)
    sim = Simulation(wl.with_(species=wl.species[:1]), resort_every=10**6, deterministic=True)
    sim.set_fields([torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in W.gem_fields(wl)])
    cell = (11, 7, 5)
    d = {k: torch.full((n,), float((c + 0.05) * h), dtype=torch.float32, device="cuda")
         for k, c, h in zip("xyz", cell, (wl.dx, wl.dy, wl.dz))}
    for k in "uvw":
        d[k] = torch.zeros(n, dtype=torch.float32, device="cuda")
    d["q"] = torch.full((n,), -1e-3, dtype=torch.float32, device="cuda")
    sim.load_species(0, d)
    sim.cycle(1)
    assert sim.check() == (8 if flagged else 0)   # SPB_ERR_CAPACITY
    sim.close()

