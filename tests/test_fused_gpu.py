"""The fused cycle (spb_sim_desc.fused): push and deposit of all species in
one persistent cooperative launch per cycle (the batching form).

Bars:
  - against the FP64 oracle, as the two-kernel precision form: per-moment
    relative L2 <= 1e-5, positions <= 1e-5 (domain units), velocities
    <= 1e-5 relative to the largest, over several cycles with CUDA graphs;
  - particles that jump past their tile's neighbourhood (a 2x2x2 tile and a
    few particles at |u| = 8, over three cells a cycle) take the overflow
    route and are still pushed and deposited correctly;
  - a grid with fewer tiles than resident CTAs;
  - on the batching workload at its real sizes, 8 cycles with graphs: the
    fused cycle and the two-kernel cycle give the same particles (the push
    of a particle is the same on every path; compared as sorted multisets)
    and moments equal up to the order of the FP32 sums (relative L2 1e-6).
"""
import numpy as np
import pytest

import oracle
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def orc64():
    return oracle.CpuOracle("restated", 64)


def rel_l2(a, b):
    nb = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(nb == 0, 1, nb)


def fused_vs_oracle(torch, orc64, wl, parts, tile, ncycles):
    from sputnipic_b200.sim import Simulation
    fields = W.gem_fields(wl)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    got_m, got_p = [], []
    for tagged in (False, True):
        sim = Simulation(wl, tile=tile, resort_every=2, fused=True, graph=True)
        sim.set_fields([T(f) for f in fields])
        for s, p in enumerate(parts):
            d = {k: T(p[k]) for k in "xyzuvwq"}
            if tagged:
                d["q"] = torch.arange(len(p["x"]), dtype=torch.float32, device="cuda")
            sim.load_species(s, d)
        sim.cycle(ncycles)
        assert sim.check() == 0
        for s in range(len(parts)):
            assert sim.count(s) == len(parts[s]["x"])
            if tagged:
                g = {k: v.cpu().numpy() for k, v in sim.particles(s).items()}
                o = np.argsort(g["q"])
                got_p.append({k: g[k][o] for k in "xyzuvw"})
            else:
                got_m.append(sim.moments(s).cpu().numpy())
        sim.close()
    setup = oracle.setup_from(wl)
    F64 = [f.astype(np.float64) for f in fields]
    for s, part in enumerate(parts):
        p = {k: part[k].astype(np.float64) for k in "xyzuvwq"}
        for _ in range(ncycles):
            assert orc64.mover_pc(setup, F64, p, wl.species[s].qom) == 0
        mom = [np.zeros(wl.nodes) for _ in range(10)]
        orc64.interp_p2g(setup, p, mom)
        err = rel_l2(got_m[s], np.stack(mom))
        assert (err <= 1e-5).all(), (s, err)
        for k in "xyz":
            assert np.abs(got_p[s][k] - p[k]).max() <= 1e-5, (s, k)
        for k in "uvw":
            assert np.abs(got_p[s][k] - p[k]).max() <= 1e-5 * np.abs(p[k]).max(), (s, k)


@pytest.mark.parametrize("tile", [(8, 4, 4), (4, 4, 4)])
def test_fused_small_gem_vs_fp64(cuda, orc64, tile):
    wl = W.small_gem(E_amp=1e-3)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    fused_vs_oracle(cuda, orc64, wl, parts, tile, ncycles=6)


def test_fused_far_jumps_take_the_overflow_route(cuda, orc64):
    """At |u| = 8 a particle moves 3.2 cells a cycle (1.6 in the half-step
    prediction). The fast particles start between cells 10 and 22 of 32 in x,
    so that over the two cycles their predictions stay inside the node array
    (past it the reference reads out of bounds and has no defined result)."""
    wl = W.small_gem(E_amp=1e-3, species=W.gem_species((4, 4, 4, 4)))
    parts = [W.gem_particles(wl, s) for s in range(2)]
    rng = np.random.default_rng(3)
    for p in parts:
        mid = np.flatnonzero((p["x"] >= 10 * wl.dx) & (p["x"] <= 22 * wl.dx))
        idx = rng.choice(mid, 64, replace=False)
        p["u"] = p["u"].copy()
        p["u"][idx] = np.float32(8.0) * np.sign(rng.standard_normal(64)).astype(np.float32)
    fused_vs_oracle(cuda, orc64, wl.with_(species=wl.species[:2]), parts, (2, 2, 2), ncycles=2)


def test_fused_grid_with_fewer_tiles_than_ctas(cuda, orc64):
    wl = W.small_gem(nxc=16, nyc=8, nzc=8, Lx=10.0, Ly=5.0, Lz=5.0, E_amp=1e-3)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    fused_vs_oracle(cuda, orc64, wl, parts, (8, 4, 4), ncycles=3)


def test_fused_batching_workload_matches_two_kernel_cycle(cuda):
    torch = cuda
    from sputnipic_b200.device import gen_fields, gen_particles
    from sputnipic_b200.sim import Simulation
    wl = W.batching_gem()
    ns = len(wl.species)
    fields = gen_fields(wl)
    out = {}
    for fused in (False, True):
        sim = Simulation(wl, resort_every=4, graph=True, fused=fused)
        sim.set_fields(fields)
        for s in range(ns):
            sim.load_species(s, gen_particles(wl, s))
            torch.cuda.empty_cache()
        sim.cycle(8)
        assert sim.check() == 0
        mom, parts = [], []
        for s in range(ns):
            assert sim.count(s) == wl.species_count(s)
            mom.append(sim.moments(s).cpu().numpy())
            parts.append(canonical(torch, sim.particles(s)))
        out[fused] = (mom, parts)
        sim.close()
        torch.cuda.empty_cache()
    for s in range(ns):
        assert torch.equal(out[True][1][s], out[False][1][s]), s
        err = rel_l2(out[True][0][s], out[False][0][s])
        assert (err <= 1e-6).all(), (s, err)


def canonical(torch, p):
    """The particles' bit patterns (n x 7 int32, CUDA) in lexicographic order
    of (x, y, z, u, v, w, q): stable sorts from the last key to the first."""
    cols = [p[k].view(torch.int32) for k in "xyzuvwq"]
    idx = torch.arange(cols[0].numel(), device=cols[0].device)
    for c in reversed(cols):
        _, order = torch.sort(c[idx], stable=True)
        idx = idx[order]
    return torch.stack([c[idx] for c in cols], dim=1)
