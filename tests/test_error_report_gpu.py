"""Error of each form against the FP64 oracle, reported and bounded.

Small GEM configuration (32x16x16 cells, 27 ppc, 4 species, seed 0), one
mover + deposit cycle from the same seeded inputs:
  - precision form (FP32 push in cell units, FP64 moments) and
  - plain drop-in (the reference's FP32 arithmetic, bit-identical to it)
against the FP64 oracle (every FP type double). Per moment: relative L2 and
max |error| / max |value| over all species and nodes; per particle
coordinate: max and RMS absolute error (positions in domain units,
velocities relative to the largest |velocity|). `pytest -s` prints the
table as one JSON line.

Bars: precision form, relative L2 <= 1e-5 per moment and position error
<= 1e-5; the plain form within 2e-4 relative L2 (the reference's own FP32
error on this configuration is of that order).
"""
import json

import numpy as np
import pytest

import oracle
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu

MOMENTS = ("rhon", "Jx", "Jy", "Jz", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz")


def moment_errors(got, ref):
    """got, ref: lists (species) of (10, nodes) arrays."""
    out = {}
    for m, name in enumerate(MOMENTS):
        a = np.concatenate([g[m] for g in got])
        b = np.concatenate([r[m] for r in ref])
        d = a - b
        out[name] = {"rel_l2": float(np.linalg.norm(d) / np.linalg.norm(b)),
                     "max_rel": float(np.abs(d).max() / np.abs(b).max())}
    return out


def particle_errors(got, ref):
    """got, ref: lists (species) of dicts x..w in the same particle order."""
    out = {}
    for k in "xyzuvw":
        a = np.concatenate([g[k].astype(np.float64) for g in got])
        b = np.concatenate([r[k] for r in ref])
        d = np.abs(a - b)
        scale = 1.0 if k in "xyz" else float(np.abs(b).max())
        out[k] = {"max_abs": float(d.max() / scale), "rms_abs": float(np.sqrt((d ** 2).mean()) / scale)}
    return out


def test_error_report_small_gem(cuda):
    torch = cuda
    from sputnipic_b200 import dropin as D
    from sputnipic_b200.sim import Simulation
    orc64 = oracle.CpuOracle("restated", 64)
    wl = W.small_gem()
    ns = len(wl.species)
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(ns)]
    setup = oracle.setup_from(wl)
    F64 = [f.astype(np.float64) for f in fields]

    # FP64 oracle, tagged so particles can be matched
    ref_p, ref_m = [], []
    for s in range(ns):
        p = {k: parts[s][k].astype(np.float64) for k in "xyzuvwq"}
        orc64.mover_pc(setup, F64, p, wl.species[s].qom)
        mom = [np.zeros(wl.nodes) for _ in range(10)]
        orc64.interp_p2g(setup, p, mom)
        ref_p.append(p)
        ref_m.append(np.stack(mom))

    # precision form: moments with the real charges, particles with tags
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    got_m, got_p = [], []
    for tagged in (False, True):
        sim = Simulation(wl, resort_every=10**6)
        sim.set_fields([T(f) for f in fields])
        for s in range(ns):
            d = {k: T(parts[s][k]) for k in "xyzuvwq"}
            if tagged:
                d["q"] = torch.arange(len(parts[s]["x"]), dtype=torch.float32, device="cuda")
            sim.load_species(s, d)
        sim.cycle(1)
        assert sim.check() == 0
        for s in range(ns):
            if tagged:
                g = {k: v.cpu().numpy() for k, v in sim.particles(s).items()}
                order = np.argsort(g["q"])
                got_p.append({k: g[k][order] for k in "xyzuvw"})
            else:
                got_m.append(sim.moments(s).cpu().numpy())
        sim.close()
    prec = {"moments": moment_errors(got_m, ref_m), "particles": particle_errors(got_p, ref_p)}

    # plain drop-in (reference precision types)
    param = D.make_parameters(wl)
    grd = D.setGrid(param)
    field = D.field_allocate(grd, fields)
    plain_m, plain_p = [], []
    for s in range(ns):
        part = D.particle_allocate(param, s, arrays={k: parts[s][k].copy() for k in "xyzuvwq"})
        assert D.mover_PC(part, field, grd, param) == 0
        ids = D.interp_dens_species_allocate(grd, s)
        D.interpP2G(part, ids, grd, raise_on_error=True)
        plain_m.append(np.stack([a.astype(np.float64) for a in D.moments(ids)]))
        plain_p.append(D.particle_arrays(part))
    plain = {"moments": moment_errors(plain_m, ref_m), "particles": particle_errors(plain_p, ref_p)}

    print(json.dumps({"config": "small GEM 32x16x16, 27 ppc, 4 species, 1 cycle",
                      "precision": prec, "plain": plain}))
    for name in MOMENTS:
        assert prec["moments"][name]["rel_l2"] <= 1e-5, name
        assert plain["moments"][name]["rel_l2"] <= 2e-4, name
    for k in "xyz":
        assert prec["particles"][k]["max_abs"] <= 1e-5, k


@pytest.mark.parametrize("preset", ["gem", "dense"])
def test_error_report_full_size_slab(cuda, preset):
    """The precision form at the full sizes of the GEM (4 x 65.5M particles,
    128x64x64) and dense (4 x 134M, 256x128x128) workloads, one cycle,
    against the FP64 oracle on the first SLABS x-slabs of cells:
      - moments: the full run's moments on the node planes x = 3..SLABS-1,
        which in one cycle only the slabs' particles reach, against the FP64
        oracle's deposit of the slabs' particles;
      - particles: the slabs' particles loaded alone (each with a unique
        charge as its tag, so that the bucket order can be undone) and
        pushed one cycle, against the FP64 oracle's push of the same
        particles.
    `pytest -s` prints the table (same keys as the small-GEM report). Bars:
    relative L2 <= 1e-5 per moment, positions <= 1e-5 absolute (domain
    units), velocities <= 1e-5 relative to the largest."""
    torch = cuda
    from sputnipic_b200.device import gen_fields, gen_particles
    from sputnipic_b200.sim import Simulation
    SLABS = 6
    wl = W.PRESETS[preset]()
    ns = len(wl.species)
    orc64 = oracle.CpuOracle("restated", 64)
    setup = oracle.setup_from(wl)
    fields = gen_fields(wl)
    F64 = [f.cpu().numpy().astype(np.float64) for f in fields]
    plane = wl.nyc * wl.nzc
    sim = Simulation(wl, resort_every=10**6)
    sim.set_fields(fields)
    slab = []
    for s in range(ns):
        p = gen_particles(wl, s, with_cell=True)
        sel = (p["cell"] // plane) < SLABS
        slab.append({k: p[k][sel].contiguous() for k in "xyzuvwq"})
        sim.load_species(s, {k: p[k] for k in "xyzuvwq"})
        del p, sel
        torch.cuda.empty_cache()
    sim.cycle(1)
    assert sim.check() == 0
    keep = np.arange(wl.nodes).reshape(wl.nxn, wl.nyn, wl.nzn)[3:SLABS].ravel()
    got_m = [sim.moments(s).cpu().numpy()[:, keep] for s in range(ns)]
    sim.close()
    torch.cuda.empty_cache()
    # the slabs alone, tagged
    tag = Simulation(wl, resort_every=10**6)
    tag.set_fields(fields)
    for s in range(ns):
        d = dict(slab[s])
        d["q"] = torch.arange(d["x"].numel(), dtype=torch.float32, device="cuda")
        tag.load_species(s, d)
    tag.cycle(1)
    assert tag.check() == 0
    ref_m, ref_p, got_p = [], [], []
    for s in range(ns):
        p = {k: slab[s][k].cpu().numpy().astype(np.float64) for k in "xyzuvwq"}
        orc64.mover_pc(setup, F64, p, wl.species[s].qom)
        mom = [np.zeros(wl.nodes) for _ in range(10)]
        orc64.interp_p2g(setup, p, mom)
        ref_m.append(np.stack(mom)[:, keep])
        ref_p.append(p)
        g = {k: v.cpu().numpy() for k, v in tag.particles(s).items()}
        order = np.argsort(g["q"])
        assert np.array_equal(g["q"][order], np.arange(len(order), dtype=np.float32))
        got_p.append({k: g[k][order] for k in "xyzuvw"})
    tag.close()
    torch.cuda.empty_cache()
    rep = {"moments": moment_errors(got_m, ref_m), "particles": particle_errors(got_p, ref_p)}
    n_slab = sum(len(p["x"]) for p in ref_p)
    print(json.dumps({"config": f"{wl.name}, {ns} species x {wl.species_count(0):,} particles, "
                                f"1 cycle; first {SLABS} x-slabs ({n_slab:,} particles), node "
                                f"planes 3..{SLABS - 1}", "precision": rep}))
    for name in MOMENTS:
        assert rep["moments"][name]["rel_l2"] <= 1e-5, name
    for k in "xyzuvw":
        assert rep["particles"][k]["max_abs"] <= 1e-5, k
