"""The precision form at the benchmark's full sizes, through properties that
do not depend on size and an oracle check on a slab of the domain.

Workloads (generated on the device, as the benchmark does):
  - GEM 128x64x64, 4 species x 65,536,000 particles (125 ppc on the 5x5x5
    jittered sub-lattice), the benchmark's own workload;
  - dense GEM 256x128x128, 4 species x 134,217,728 particles (32 ppc).

Bars, after one cycle of all four species:
  - every particle is still there and inside the domain, the error word is 0;
  - the deposited charge of each species equals sum(q) * invVOL (relative
    1e-6; the charge density is rhon, moment 0, before applyBCids);
  - slab parity: the particles of the first S x-slabs of cells, pushed and
    deposited by the FP64 oracle, give the same moments (relative L2 <= 1e-5
    per moment, the precision form's bar) on the node planes x = 3 .. S-1,
    which in one cycle only particles of those slabs can reach (a particle
    moves less than a cell; node i takes deposits from cells i-2 and i-1, and
    planes 1 and 2 could take periodic inflow from the last slab).
"""
import numpy as np
import pytest

import oracle
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu

SLABS = 6


@pytest.fixture(scope="module")
def orc64():
    return oracle.CpuOracle("restated", 64)


def rel_l2(a, b):
    nb = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(nb == 0, 1, nb)


def full_size_check(torch, orc64, wl):
    from sputnipic_b200.device import gen_fields, gen_particles
    from sputnipic_b200.sim import Simulation
    ns = len(wl.species)
    fields = gen_fields(wl)
    sim = Simulation(wl)
    sim.set_fields(fields)
    slab, qsum = [], []
    plane = wl.nyc * wl.nzc
    for s in range(ns):
        p = gen_particles(wl, s, with_cell=True)
        assert p["x"].numel() == wl.species_count(s)
        qsum.append(float(p["q"].double().sum()))
        sel = (p["cell"] // plane) < SLABS
        slab.append({k: p[k][sel].cpu().numpy().astype(np.float64) for k in "xyzuvwq"})
        sim.load_species(s, {k: p[k] for k in "xyzuvwq"})
        del p, sel
        torch.cuda.empty_cache()
    sim.cycle(1)
    assert sim.check() == 0
    inv = 1.0 / (wl.dx * wl.dy * wl.dz)
    F = [f.cpu().numpy().astype(np.float64) for f in fields]
    setup = oracle.setup_from(wl)
    nodes = np.arange(wl.nodes).reshape(wl.nxn, wl.nyn, wl.nzn)
    keep = nodes[3:SLABS].ravel()
    for s in range(ns):
        assert sim.count(s) == wl.species_count(s)
        m = sim.moments(s).cpu().numpy()
        assert abs(m[0].sum() - qsum[s] * inv) <= 1e-6 * abs(qsum[s] * inv), s
        pts = sim.particles(s)
        for k, L in (("x", wl.Lx), ("y", wl.Ly), ("z", wl.Lz)):
            assert float(pts[k].min()) >= 0.0 and float(pts[k].max()) <= L, (s, k)
        del pts
        p = slab[s]
        orc64.mover_pc(setup, F, p, wl.species[s].qom)
        mom = [np.zeros(wl.nodes) for _ in range(10)]
        orc64.interp_p2g(setup, p, mom)
        err = rel_l2(m[:, keep], np.stack(mom)[:, keep])
        assert (err <= 1e-5).all(), (s, err)
    sim.close()
    torch.cuda.empty_cache()


def test_gem_benchmark_workload(cuda, orc64):
    full_size_check(cuda, orc64, W.gem())


def test_dense_workload(cuda, orc64):
    full_size_check(cuda, orc64, W.dense_gem())
