"""Precision form (per-cell buckets of FP32 offsets, charge and velocities;
FP32 push; FP32 per-cell register sums -> FP64 moments) against the FP64
oracle (the reference's arithmetic with every FP type double) on the same
seeded inputs.

Tolerances:
  moments    per-moment relative L2 error vs the FP64 oracle <= 1e-5
  positions  max |x - x64| <= 1e-5 (domain units, L ~ 10)
  velocities max |u - u64| <= 1e-5 * max|u64|
  cells      particles whose cell differs from the FP64 oracle's: at most
             1e-4 of them (only particles within float rounding of a face)
"""
import numpy as np
import pytest

import oracle
from conftest import edge_workload
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def orc64():
    return oracle.CpuOracle("restated", 64)


def rel_l2(a, b):
    nb = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(nb == 0, 1, nb)


def run_sim(torch, wl, fields, parts, tile=(8, 4, 4), resort_every=1, ncycles=1, tags=False,
            species=None, variant=0, bucket_slots=0, graph=False):
    from sputnipic_b200.sim import Simulation
    sim = Simulation(wl, tile=tile, resort_every=resort_every, species=species, variant=variant,
                     bucket_slots=bucket_slots, graph=graph)
    sim.set_fields([torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in fields])
    for s, p in enumerate(parts):
        d = {k: torch.from_numpy(np.ascontiguousarray(p[k])).cuda() for k in "xyzuvwq"}
        if tags:
            d["q"] = torch.arange(len(p["x"]), dtype=torch.float32, device="cuda")
        sim.load_species(s, d)
    sim.cycle(ncycles)
    assert sim.check() == 0
    return sim


def oracle64(orc64, wl, fields, part, qom, ncycles=1):
    setup = oracle.setup_from(wl)
    F = [f.astype(np.float64) for f in fields]
    p = {k: part[k].astype(np.float64) for k in "xyzuvwq"}
    for _ in range(ncycles):
        orc64.mover_pc(setup, F, p, qom)
    mom = [np.zeros(wl.nodes) for _ in range(10)]
    orc64.interp_p2g(setup, p, mom)
    return p, np.stack(mom)


def compare_particles(sim_p, ref_p, wl):
    order = np.argsort(sim_p["q"])
    assert np.array_equal(sim_p["q"][order], np.arange(len(order), dtype=np.float32))
    d = {k: sim_p[k][order].astype(np.float64) for k in "xyzuvw"}
    for k in "xyz":
        assert np.abs(d[k] - ref_p[k]).max() <= 1e-5, k
    for k in "uvw":
        scale = np.abs(ref_p[k]).max() + 1e-30
        assert np.abs(d[k] - ref_p[k]).max() <= 1e-5 * scale, k
    mism = 0
    for k, dd in (("x", wl.dx), ("y", wl.dy), ("z", wl.dz)):
        mism += int((np.floor(d[k] / dd) != np.floor(ref_p[k] / dd)).sum())
    assert mism <= 1e-4 * len(order) + 2, mism


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("tile", [(8, 4, 4), (4, 4, 4), (2, 2, 2)])
def test_small_gem_moments_vs_fp64(cuda, orc64, tile, variant):
    torch = cuda
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    sim = run_sim(torch, wl, fields, parts, tile=tile, variant=variant)
    for s in range(4):
        _, m64 = oracle64(orc64, wl, fields, parts[s], wl.species[s].qom)
        err = rel_l2(sim.moments(s).cpu().numpy(), m64)
        assert (err <= 1e-5).all(), (s, err)
    sim.close()


def test_small_gem_particles_vs_fp64(cuda, orc64):
    torch = cuda
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    sim = run_sim(torch, wl, fields, parts, tags=True)
    for s in range(4):
        tagged = dict(parts[s])
        tagged["q"] = np.arange(len(parts[s]["x"]), dtype=np.float32)
        ref, _ = oracle64(orc64, wl, fields, tagged, wl.species[s].qom)
        got = {k: v.cpu().numpy() for k, v in sim.particles(s).items()}
        compare_particles(got, ref, wl)
    sim.close()


@pytest.mark.parametrize("resort_every,variant", [(1, 0), (4, 1), (8, 0)])
def test_ten_cycles_vs_fp64(cuda, orc64, resort_every, variant):
    torch = cuda
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    sim = run_sim(torch, wl, fields, parts, resort_every=resort_every, ncycles=10,
                  variant=variant)
    for s in range(4):
        _, m64 = oracle64(orc64, wl, fields, parts[s], wl.species[s].qom, ncycles=10)
        err = rel_l2(sim.moments(s).cpu().numpy(), m64)
        assert (err <= 1e-5).all(), (s, err)
    sim.close()


@pytest.mark.parametrize("qi", [0, 1])
def test_edge_fixture_vs_reference_fp64(cuda, golden_edge, qi):
    """Walls, faces and one-step crossers: moments and particles against the
    reference's own FP64 build (fixture)."""
    torch = cuda
    d = golden_edge
    wl = edge_workload(d)
    wl = wl.with_(species=(W.Species(qom=float(d["qom"][qi]), rho0=1, sheet=False, vth=0,
                                     w0=0, ppc=1),))
    fields = [d[f"field_{n}"] for n in oracle.FIELDS]
    part = {k: d[f"in_{k}"] for k in "xyzuvwq"}
    sim = run_sim(torch, wl, fields, [part], tile=(2, 2, 2), variant=qi)
    err = rel_l2(sim.moments(0).cpu().numpy(), d[f"fp64_q{qi}_p2g"])
    assert (err <= 1e-5).all(), err
    sim.close()
    sim = run_sim(torch, wl, fields, [part], tile=(2, 2, 2), tags=True)
    got = {k: v.cpu().numpy() for k, v in sim.particles(0).items()}
    ref = {k: d[f"fp64_q{qi}_mover_{k}"] for k in "xyzuvw"}
    compare_particles(got, ref, wl)
    sim.close()


@pytest.mark.parametrize("slots,resort_every", [(8, 100), (16, 3)])
def test_overflow_path_vs_fp64(cuda, orc64, slots, resort_every):
    """Buckets far smaller than the cells' counts (27 ppc on average): most
    particles live in the overflow list, are pushed with gathers from L2 and
    deposited by the overflow pass (groups of entries of one cell summed by
    the warp, lone entries one by one; FP64 atomics), and re-enter buckets
    when room appears. Ten
    cycles, with and without re-layouts in between; moments and tagged
    particles against the FP64 oracle."""
    torch = cuda
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(2)]
    sim = run_sim(torch, wl, fields, parts, species=[0, 1], resort_every=resort_every,
                  bucket_slots=slots, ncycles=10)
    for s in range(2):
        assert sim.bucket_slots(s) == slots * wl.cells
        assert sim.overflow(s) > 0
        _, m64 = oracle64(orc64, wl, fields, parts[s], wl.species[s].qom, ncycles=10)
        err = rel_l2(sim.moments(s).cpu().numpy(), m64)
        assert (err <= 1e-5).all(), (s, err)
    sim.close()
    sim = run_sim(torch, wl, fields, parts[:1], species=[0], bucket_slots=slots, ncycles=3,
                  tags=True, resort_every=100)
    tagged = dict(parts[0])
    tagged["q"] = np.arange(len(parts[0]["x"]), dtype=np.float32)
    ref, _ = oracle64(orc64, wl, fields, tagged, wl.species[0].qom, ncycles=3)
    got = {k: v.cpu().numpy() for k, v in sim.particles(0).items()}
    compare_particles(got, ref, wl)
    sim.close()


def test_relayout_keeps_particles_and_moments(cuda, orc64):
    """An explicit re-layout between cycles (compaction into fresh buckets)
    changes nothing: 3 cycles, re-layout, 3 cycles against 6 oracle cycles."""
    torch = cuda
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    part = W.gem_particles(wl, 1)
    tagged = dict(part)
    tagged["q"] = np.arange(len(part["x"]), dtype=np.float32)
    sim = run_sim(torch, wl, fields, [part], species=[1], ncycles=3, tags=True,
                  resort_every=100)
    n0 = sim.count(0)
    sim.resort()
    sim.cycle(3)
    assert sim.check() == 0
    assert sim.count(0) == n0 and sim.overflow(0) == 0
    ref, _ = oracle64(orc64, wl, fields, tagged, wl.species[1].qom, ncycles=6)
    got = {k: v.cpu().numpy() for k, v in sim.particles(0).items()}
    compare_particles(got, ref, wl)
    sim.close()


def test_reload_within_reserved_capacity(cuda, orc64):
    """spb_sim_desc.capacity reserves a species' buffers at its first load:
    half the particles loaded and run two cycles, then the whole set loaded
    in their place and run three cycles, against three FP64 oracle cycles of
    the whole set (moments and tagged particles)."""
    torch = cuda
    from sputnipic_b200.sim import Simulation
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    part = W.gem_particles(wl, 0)
    n = len(part["x"])
    sim = Simulation(wl, species=[0], resort_every=2, capacity=[n])
    sim.set_fields([torch.from_numpy(np.ascontiguousarray(f)).cuda() for f in fields])
    half = {k: torch.from_numpy(np.ascontiguousarray(part[k][: n // 2])).cuda() for k in "xyzuvwq"}
    sim.load_species(0, half)
    sim.cycle(2)
    assert sim.check() == 0 and sim.count(0) == n // 2
    full = {k: torch.from_numpy(np.ascontiguousarray(part[k])).cuda() for k in "xyzuvwq"}
    sim.load_species(0, full)
    sim.cycle(3)
    assert sim.check() == 0 and sim.count(0) == n
    _, m64 = oracle64(orc64, wl, fields, part, wl.species[0].qom, ncycles=3)
    assert (rel_l2(sim.moments(0).cpu().numpy(), m64) <= 1e-5).all()
    full["q"] = torch.arange(n, dtype=torch.float32, device="cuda")
    sim.load_species(0, full)
    sim.cycle(3)
    assert sim.check() == 0
    tagged = dict(part)
    tagged["q"] = np.arange(n, dtype=np.float32)
    ref, _ = oracle64(orc64, wl, fields, tagged, wl.species[0].qom, ncycles=3)
    compare_particles({k: v.cpu().numpy() for k, v in sim.particles(0).items()}, ref, wl)
    sim.close()


def test_bc_on_device_matches_oracle_bc(cuda, orc64):
    torch = cuda
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, 0)]
    sim = run_sim(torch, wl, fields, parts, species=[0])
    raw = sim.moments(0).cpu().numpy()
    bc = sim.moments(0, bc=True).cpu().numpy()
    ref = [a.copy() for a in raw]
    orc64.apply_bc_ids(oracle.setup_from(wl), ref)
    assert np.array_equal(bc, np.stack(ref))
    sim.close()


def test_charge_conservation_and_counts_gem_grid(cuda):
    """Size-independent properties on the full 128x64x64 GEM grid (one species,
    8 ppc, generated on the device): every particle stays in the domain and
    is counted once; the deposited charge equals sum(q) * invVOL."""
    torch = cuda
    from sputnipic_b200.device import gen_fields, gen_particles
    from sputnipic_b200.sim import Simulation
    wl = W.gem(lattice=0, species=W.gem_species((8, 8, 8, 8)))
    sim = Simulation(wl, species=[0, 2])
    sim.set_fields(gen_fields(wl))
    qsum = []
    for i, s in enumerate((0, 2)):
        p = gen_particles(wl, s)
        qsum.append(float(p["q"].double().sum()))
        sim.load_species(i, p)
    sim.cycle(3)
    assert sim.check() == 0
    inv = 1.0 / (wl.dx * wl.dy * wl.dz)
    for i in range(2):
        m = sim.moments(i)
        assert abs(float(m[0].sum()) - qsum[i] * inv) <= 1e-6 * abs(qsum[i] * inv)
        p = sim.particles(i)
        assert p["x"].numel() == wl.species_count((0, 2)[i])
        for k, L in (("x", wl.Lx), ("y", wl.Ly), ("z", wl.Lz)):
            assert float(p[k].min()) >= 0.0 and float(p[k].max()) <= L
    sim.close()


def test_graph_replay_vs_fp64(cuda, orc64):
    """Cycles replayed as CUDA graphs (captured per buffer-parity pattern,
    recaptured after the re-layouts that small buckets force every 3 cycles):
    ten cycles, moments and tagged particles against the FP64 oracle."""
    torch = cuda
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(2)]
    sim = run_sim(torch, wl, fields, parts, species=[0, 1], resort_every=3, ncycles=10,
                  graph=True)
    for s in range(2):
        _, m64 = oracle64(orc64, wl, fields, parts[s], wl.species[s].qom, ncycles=10)
        err = rel_l2(sim.moments(s).cpu().numpy(), m64)
        assert (err <= 1e-5).all(), (s, err)
    sim.close()
    sim = run_sim(torch, wl, fields, parts[:1], species=[0], ncycles=10, tags=True,
                  resort_every=3, bucket_slots=16, graph=True)
    tagged = dict(parts[0])
    tagged["q"] = np.arange(len(parts[0]["x"]), dtype=np.float32)
    ref, _ = oracle64(orc64, wl, fields, tagged, wl.species[0].qom, ncycles=10)
    got = {k: v.cpu().numpy() for k, v in sim.particles(0).items()}
    compare_particles(got, ref, wl)
    sim.close()
