"""Parity at the benchmark configurations' real sizes.

1. Plain drop-in on the full GEM workload (128x64x64 cells, 4 species x
   65,536,000 particles, 125 ppc), through the C-ABI on the reference structs
   in DEVICE residency: mover_PC for every species, interpP2G for every
   species, particles synced back to the host. Bars:
     - the particles of the first SLABS x-slabs of cells are bit-identical
       to the reference's own mover_PC (oracle/_ref where it was built, else
       the restatement pinned to it) run on the same inputs; the plain mover
       keeps the particle order, so those are the first entries of each array;
     - species 0 pushed in COPY residency (the chunked PCIe pipeline) is
       bit-identical to the DEVICE residency result over all 65.5M particles;
     - every particle is counted and inside the domain, and each species'
       deposited charge sum(rhon) equals sum(q) * invVOL (relative 1e-5, FP32
       node sums);
     - the moments on the node planes x = 3 .. SLABS-1, which in one cycle only
       the slabs' particles reach, are within the reordering bound
       |gpu - ref| <= 32 eps32 sum|terms| of the reference FP32 deposit of
       the moved slab particles;
     - the driver's moment section in one call (spb_interp_all_species) on
       the moved particles: each species' moments within relative L2 1e-5 of
       its own interpP2G deposit with applyBCids applied, the net moments
       bit-identical to the float sum of the species' in species order.

2. Batching workload (species of 65.5M, 65.5M, 6.55M and 6.55M particles on
   the GEM grid, background at 12.5 ppc), 20 cycles with CUDA graphs,
   overflow checks every 4 cycles and one forced re-layout. Two tracer
   species (10,000 electrons and 10,000 ions taken from the workload's
   initial state, each with a unique charge as its tag) ride in the same
   launches. Bars after 20 cycles:
     - every species keeps its particles, inside the domain, error word 0;
     - every species' deposited charge equals sum(q) * invVOL (relative 1e-6);
     - the tracers match the FP64 oracle run for 20 cycles particle by
       particle (positions 1e-5 absolute in domain units, velocities 1e-5
       relative to the largest), and their moments match the FP64 oracle's
       deposit of the oracle's particles (relative L2 1e-5 per moment);
     - one more cycle from the state reached (clumped electrons, re-laid-out
       buckets): the FP64 oracle run on the particles of the first x-slabs of
       cells gives the same moments on the node planes that only those
       particles can reach in one cycle (relative L2 1e-5).

3. particle_sort on one full GEM species (65,536,000 particles) after one
   mover_PC step, with GEM_3D's sort_cps = 2: in place on the resident copy
   (DEVICE residency) and through PCIe (COPY residency), both bit-identical
   to the oracle's particle_sort of the same moved particles (all seven
   arrays, order within each bin included).
"""
import numpy as np
import pytest

import oracle
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu

EPS32 = float(np.finfo(np.float32).eps)
SLABS = 4


def ref_oracle32():
    kind = "reference" if oracle.reference_available(32) else "restated"
    return oracle.CpuOracle(kind, 32)


def slab_count(wl, s, slabs):
    return int(W.cell_counts(wl.species[s].ppc, 0, slabs * wl.nyc * wl.nzc).sum())


def rel_l2(a, b):
    nb = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(nb == 0, 1, nb)


def test_plain_dropin_full_gem_device_residency(cuda):
    torch = cuda
    from sputnipic_b200 import dropin as D
    from sputnipic_b200.device import gen_fields, gen_particles
    wl = W.gem()
    ns = len(wl.species)
    orc32 = ref_oracle32()
    orc64 = oracle.CpuOracle("restated", 64)
    setup = oracle.setup_from(wl)
    fields = [f.cpu().numpy() for f in gen_fields(wl)]
    param = D.make_parameters(wl)
    grd = D.setGrid(param)
    field = D.field_allocate(grd, fields)
    P, slab0, qsum, copy0 = [], [], [], None
    for s in range(ns):
        p = gen_particles(wl, s)
        host = {k: p[k].cpu().numpy() for k in "xyzuvwq"}
        del p
        torch.cuda.empty_cache()
        n_s = slab_count(wl, s, SLABS)
        slab0.append({k: host[k][:n_s].copy() for k in "xyzuvwq"})
        qsum.append(float(host["q"].astype(np.float64).sum()))
        if s == 0:
            copy0 = {k: host[k].copy() for k in "xyzuvwq"}
        P.append(D.particle_allocate(param, s, arrays=host))
    try:
        assert D.set_residency(True) == 0
        for s in range(ns):
            assert D.mover_PC(P[s], field, grd, param) == 0, D.last_error()
        ids = [D.interp_dens_species_allocate(grd, s) for s in range(ns)]
        for s in range(ns):
            D.interpP2G(P[s], ids[s], grd, raise_on_error=True)
        for s in range(ns):
            assert D.sync_particles_to_host(P[s]) == 0
    finally:
        D.set_residency(False)
    inv = 1.0 / (wl.dx * wl.dy * wl.dz)
    nodes = np.arange(wl.nodes).reshape(wl.nxn, wl.nyn, wl.nzn)
    keep = nodes[3:SLABS].ravel()
    for s in range(ns):
        out = D.particle_arrays(P[s])
        assert len(out["x"]) == wl.species_count(s)
        for k, L in (("x", wl.Lx), ("y", wl.Ly), ("z", wl.Lz)):
            assert float(out[k].min()) >= 0.0 and float(out[k].max()) <= L, (s, k)
        mom = np.stack(D.moments(ids[s])).astype(np.float64)
        assert abs(mom[0].sum() - qsum[s] * inv) <= 1e-5 * abs(qsum[s] * inv), s
        ref = slab0[s]
        orc32.mover_pc(setup, fields, ref, wl.species[s].qom)
        n_s = len(ref["x"])
        for k in "xyzuvw":
            assert np.array_equal(out[k][:n_s], ref[k]), (s, k)
        ref_m = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
        orc32.interp_p2g(setup, ref, ref_m)
        absm = [np.zeros(wl.nodes) for _ in range(10)]
        pa = {k: np.abs(ref[k].astype(np.float64)) for k in "uvwq"}
        pa.update({k: ref[k].astype(np.float64) for k in "xyz"})
        orc64.interp_p2g(setup, pa, absm)
        bound = 32 * EPS32 * np.stack(absm)[:, keep] + 1e-30
        diff = np.abs(mom[:, keep] - np.stack(ref_m).astype(np.float64)[:, keep])
        assert (diff <= bound).all(), (s, int((diff > bound).sum()))
    # the driver's moment section in one call on the same moved particles:
    # each species' moments match its own interpP2G deposit above with the
    # oracle's applyBCids applied (two FP32 sums in different orders), and the
    # net moments are the float sum of the species' in species order
    ids2 = [D.interp_dens_species_allocate(grd, s) for s in range(ns)]
    idn = D.interp_dens_net_allocate(grd)
    assert D.interp_all_species(P, ids2, idn, grd, param) == 0, D.last_error()
    net = np.zeros((10, wl.nodes), np.float32)
    for s in range(ns):
        sep = [m.copy() for m in D.moments(ids[s])]
        orc32.apply_bc_ids(setup, sep)
        got = np.stack(D.moments(ids2[s]))
        err = rel_l2(got.astype(np.float64), np.stack(sep).astype(np.float64))
        assert (err <= 1e-5).all(), (s, err)
        net = net + got
    assert np.array_equal(np.stack(D.moments(idn)), net)
    # species 0 again in COPY residency (chunked PCIe pipeline): bit-identical
    dev_result = {k: v.copy() for k, v in D.particle_arrays(P[0]).items()}
    D.release_all()
    del P
    param = D.make_parameters(wl)
    grd = D.setGrid(param)
    field = D.field_allocate(grd, fields)
    Pc = D.particle_allocate(param, 0, arrays=copy0)
    assert D.mover_PC(Pc, field, grd, param) == 0, D.last_error()
    got = D.particle_arrays(Pc)
    for k in "xyzuvw":
        assert np.array_equal(got[k], dev_result[k]), k
    D.release_all()


def tracers(parts, n, seed):
    """n particles drawn from a species' initial state (device tensors), each
    with a unique charge (a tag that survives the buckets' reordering)."""
    import torch
    g = torch.Generator(device="cpu").manual_seed(seed)
    idx = torch.randperm(parts["x"].numel(), generator=g)[:n].sort().values.cuda()
    t = {k: parts[k][idx].contiguous() for k in "xyzuvwq"}
    sign = float(np.sign(t["q"][0].item()))
    # |q| from 1e-3 up, 2^-10 relative apart: distinct floats, same magnitude
    t["q"] = (sign * 1e-3 * (1.0 + torch.arange(n, device="cuda", dtype=torch.float64)
                             * 2.0 ** -10)).float()
    return t


def test_batching_workload_twenty_cycles(cuda):
    torch = cuda
    from sputnipic_b200.device import gen_fields, gen_particles
    from sputnipic_b200.sim import Simulation
    wl4 = W.batching_gem()
    sp = wl4.species
    wl = wl4.with_(species=sp + (sp[0], sp[1]))      # + electron and ion tracers
    ns = len(wl.species)
    fields = gen_fields(wl4)
    sim = Simulation(wl, resort_every=4, graph=True)
    sim.set_fields(fields)
    qsum, counts, tr = [], [], []
    for s in range(4):
        p = gen_particles(wl4, s)
        counts.append(p["x"].numel())
        qsum.append(float(p["q"].double().sum()))
        if s < 2:
            tr.append(tracers(p, 10000, seed=s))
        sim.load_species(s, p)
        del p
        torch.cuda.empty_cache()
    for i, t in enumerate(tr):
        sim.load_species(4 + i, t)
        counts.append(t["x"].numel())
        qsum.append(float(t["q"].double().sum()))
    host_tr = [{k: t[k].cpu().numpy().astype(np.float64) for k in "xyzuvwq"} for t in tr]
    sim.cycle(10)
    sim.resort()                                      # at least one re-layout
    sim.cycle(10)
    assert sim.check() == 0
    inv = 1.0 / (wl.dx * wl.dy * wl.dz)
    for s in range(ns):
        assert sim.count(s) == counts[s]
        m = sim.moments(s)
        assert abs(float(m[0].sum()) - qsum[s] * inv) <= 1e-6 * abs(qsum[s] * inv), s
        pts = sim.particles(s)
        assert pts["x"].numel() == counts[s]
        for k, L in (("x", wl.Lx), ("y", wl.Ly), ("z", wl.Lz)):
            assert float(pts[k].min()) >= 0.0 and float(pts[k].max()) <= L, (s, k)
        del pts
    # tracers against the FP64 oracle over the 20 cycles
    orc64 = oracle.CpuOracle("restated", 64)
    setup = oracle.setup_from(wl)
    F64 = [f.cpu().numpy().astype(np.float64) for f in fields]
    for i, ref in enumerate(host_tr):
        s = 4 + i
        for _ in range(20):
            assert orc64.mover_pc(setup, F64, ref, wl.species[s].qom) == 0
        got = {k: v.cpu().numpy() for k, v in sim.particles(s).items()}
        go, ro = np.argsort(got["q"]), np.argsort(ref["q"].astype(np.float32))
        assert np.array_equal(got["q"][go], ref["q"].astype(np.float32)[ro])
        for k in "xyz":
            assert np.abs(got[k][go] - ref[k][ro]).max() <= 1e-5, (s, k)
        for k in "uvw":
            scale = np.abs(ref[k]).max()
            assert np.abs(got[k][go] - ref[k][ro]).max() <= 1e-5 * scale, (s, k)
        mom = [np.zeros(wl.nodes) for _ in range(10)]
        orc64.interp_p2g(setup, ref, mom)
        err = rel_l2(sim.moments(s).cpu().numpy(), np.stack(mom))
        assert (err <= 1e-5).all(), (s, err)
    # one more cycle from the state reached, against the FP64 oracle on the
    # particles of the first S x-slabs. A particle moves at most m cells along
    # x in a cycle (m from the fastest |u| now, with a 1.5x margin for the
    # velocity change within the cycle), so only the slabs' particles reach
    # cells m .. S-m-1, and node planes m+2 .. S-m (node i takes deposits from
    # cells i-2 and i-1)
    parts = [sim.particles(s) for s in range(4)]
    umax = max(float(p["u"].abs().max()) for p in parts)
    m = max(1, int(np.ceil(1.5 * umax * wl.dt / wl.dx)))
    slabs = 4 + 2 * m
    assert slabs < wl.nxc // 2, umax
    start = []
    for p in parts:
        cx = (p["x"].double() / wl.dx).floor().clamp(0, wl.nxc - 1)
        sel = cx < slabs
        start.append({k: p[k][sel].cpu().numpy().astype(np.float64) for k in "xyzuvwq"})
        del cx, sel
    del parts
    sim.cycle(1)
    assert sim.check() == 0
    keep = np.arange(wl.nodes).reshape(wl.nxn, wl.nyn, wl.nzn)[m + 2:slabs - m + 1].ravel()
    for s in range(4):
        ref = start[s]
        assert orc64.mover_pc(setup, F64, ref, wl.species[s].qom) == 0
        mom = [np.zeros(wl.nodes) for _ in range(10)]
        orc64.interp_p2g(setup, ref, mom)
        err = rel_l2(sim.moments(s).cpu().numpy()[:, keep], np.stack(mom)[:, keep])
        assert (err <= 1e-5).all(), (s, err)
    sim.close()
    torch.cuda.empty_cache()


def test_particle_sort_full_gem_species(cuda):
    torch = cuda
    from sputnipic_b200 import dropin as D
    from sputnipic_b200.device import gen_fields, gen_particles
    wl = W.gem()
    orc = oracle.CpuOracle("restated", 32)
    fields = [f.cpu().numpy() for f in gen_fields(wl)]
    param = D.make_parameters(wl)
    grd = D.setGrid(param)
    field = D.field_allocate(grd, fields)
    param.sort_cps = 2
    p = gen_particles(wl, 0)
    host = {k: p[k].cpu().numpy() for k in "xyzuvwq"}
    del p
    torch.cuda.empty_cache()
    a = D.particle_allocate(param, 0, arrays={k: host[k].copy() for k in "xyzuvwq"})
    b = D.particle_allocate(param, 0, arrays=host)
    try:
        # a: moved and sorted where it lies (the device copy is the newest
        # and, after a deposit, holds q too)
        assert D.set_residency(True) == 0
        assert D.mover_PC(a, field, grd, param) == 0, D.last_error()
        D.interpP2G(a, D.interp_dens_species_allocate(grd, 0), grd, raise_on_error=True)
        assert D.particle_sort(param, a, grd) == 0, D.last_error()
        assert D.sync_particles_to_host(a) == 0
    finally:
        D.set_residency(False)
    D.release_all()
    # b: moved in COPY residency (the oracle's input), then sorted through PCIe
    assert D.mover_PC(b, field, grd, param) == 0, D.last_error()
    ref = {k: v.copy() for k, v in D.particle_arrays(b).items()}
    assert D.particle_sort(param, b, grd) == 0, D.last_error()
    D.release_all()
    assert orc.particle_sort(oracle.setup_from(wl), 2, ref) == 0
    got_a, got_b = D.particle_arrays(a), D.particle_arrays(b)
    for k in "xyzuvwq":
        assert np.array_equal(got_a[k].view(np.uint32), ref[k].view(np.uint32)), ("in place", k)
        assert np.array_equal(got_b[k].view(np.uint32), ref[k].view(np.uint32)), ("pcie", k)
