"""The CPU oracle restatement (oracle/oracle.c) pinned against fixtures made by
the reference's own code (tests/golden/make_golden.py). Bit-exact: both are
the same float arithmetic in the same order, and both deposit serially."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, edge_workload
from sputnipic_b200 import workload as W


def sha(arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("fp", [32, 64])
@pytest.mark.parametrize("qi", [0, 1])
def test_edge_mover_bitexact(golden_edge, fp, qi):
    d = golden_edge
    wl = edge_workload(d)
    O = oracle.CpuOracle("restated", fp)
    dt = O.dtype
    setup = oracle.setup_from(wl)
    F = [d[f"field_{n}"].astype(dt) for n in oracle.FIELDS]
    qom = float(d["qom"][qi])
    for fn, tag in ((O.mover_pc, "mover"), (O.mover_pc_v, "moverv")):
        p = {k: d[f"in_{k}"].astype(dt) for k in "xyzuvwq"}
        fn(setup, F, p, qom)
        for k in "xyzuvw":
            ref = d[f"fp{fp}_q{qi}_{tag}_{k}"]
            assert np.array_equal(p[k], ref), f"{tag} {k}: {np.sum(p[k] != ref)} differ"


@pytest.mark.parametrize("fp", [32, 64])
@pytest.mark.parametrize("qi", [0, 1])
def test_edge_p2g_and_bc_bitexact(golden_edge, fp, qi):
    d = golden_edge
    wl = edge_workload(d)
    O = oracle.CpuOracle("restated", fp)
    dt = O.dtype
    setup = oracle.setup_from(wl)
    p = {k: d[f"fp{fp}_q{qi}_mover_{k}"].astype(dt) for k in "xyzuvw"}
    p["q"] = d["in_q"].astype(dt)
    mom = [np.zeros(wl.nodes, dt) for _ in range(10)]
    O.interp_p2g(setup, p, mom)
    assert np.array_equal(np.stack(mom), d[f"fp{fp}_q{qi}_p2g"])
    O.apply_bc_ids(setup, mom)
    assert np.array_equal(np.stack(mom), d[f"fp{fp}_q{qi}_p2g_bc"])


@pytest.mark.parametrize("fp", [32, 64])
@pytest.mark.parametrize("qi", [0, 1])
def test_edge_fused_bitexact(golden_edge, fp, qi):
    d = golden_edge
    wl = edge_workload(d)
    O = oracle.CpuOracle("restated", fp)
    dt = O.dtype
    setup = oracle.setup_from(wl)
    F = [d[f"field_{n}"].astype(dt) for n in oracle.FIELDS]
    p = {k: d[f"in_{k}"].astype(dt) for k in "xyzuvwq"}
    mom = [np.zeros(wl.nodes, dt) for _ in range(10)]
    O.mover_interp(setup, F, p, float(d["qom"][qi]), mom)
    for k in "xyzuvw":
        assert np.array_equal(p[k], d[f"fp{fp}_q{qi}_fused_{k}"])
    assert np.array_equal(np.stack(mom), d[f"fp{fp}_q{qi}_fused_mom"])


def test_edge_fixture_covers_walls_and_faces(golden_edge):
    """The edge fixture holds particles on x = 0 and x = L, on cell faces, and
    particles that cross both the periodic and the reflecting walls."""
    d = golden_edge
    wl = edge_workload(d)
    x, y = d["in_x"], d["in_y"]
    assert (x == 0).any() and (x == np.float32(wl.Lx)).any()
    assert (y == 0).any() and (y == np.float32(wl.Ly)).any()
    on_face = np.isclose(np.mod(x / wl.dx, 1.0), 0.0, atol=1e-6)
    assert on_face.sum() > 50
    vout = d["fp32_q1_mover_v"]
    flipped = np.sign(vout) != np.sign(d["in_v"])
    crossed_y = (d["in_y"] < 0.06) | (d["in_y"] > wl.Ly - 0.06)
    assert (flipped & crossed_y).sum() > 10          # reflecting wall (y)
    xout = d["fp32_q1_mover_x"]
    assert ((d["in_x"] > wl.Lx - 0.06) & (xout < 0.5)).sum() > 5   # periodic wrap (x)


def test_small_gem_1ppc_ten_cycles(golden_small_1ppc):
    d = golden_small_1ppc
    wl = W.small_gem(species=W.gem_species((1, 1, 1, 1)))
    O = oracle.CpuOracle("restated", 32)
    setup = oracle.setup_from(wl)
    F = [d[f"field_{n}"] for n in oracle.FIELDS]
    for s in range(4):
        p = {k: d[f"in_s{s}_{k}"].copy() for k in "xyzuvwq"}
        qom = wl.species[s].qom
        for cyc in range(1, 11):
            O.mover_pc(setup, F, p, qom)
            mom = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
            O.interp_p2g(setup, p, mom)
            O.apply_bc_ids(setup, mom)
            if cyc in (1, 10):
                for k in "xyzuvw":
                    assert np.array_equal(p[k], d[f"c{cyc}_s{s}_{k}"]), (s, cyc, k)
        assert np.array_equal(np.stack(mom), d[f"c10_s{s}_mom"])


@pytest.mark.slow
def test_small_gem_full_digests():
    """Full small GEM config (4 x 221,184 particles, 10 cycles): the inputs
    regenerate to the pinned digests, and the restatement reproduces the
    reference's particle and moment digests after cycles 1 and 10."""
    with open(os.path.join(GOLDEN, "gem_small.json")) as f:
        doc = json.load(f)
    wl = W.small_gem()
    F = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    assert sha(F) == doc["inputs"]["fields"]
    for s, p in enumerate(parts):
        assert sha([p[k] for k in "xyzuvwq"]) == doc["inputs"]["particles"][s]
    O = oracle.CpuOracle("restated", 32)
    setup = oracle.setup_from(wl)
    ps = [{k: p[k].copy() for k in "xyzuvwq"} for p in parts]
    for cyc in range(1, 11):
        moms = []
        for s, p in enumerate(ps):
            O.mover_pc(setup, F, p, wl.species[s].qom)
            mom = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
            O.interp_p2g(setup, p, mom)
            O.apply_bc_ids(setup, mom)
            moms.append(np.stack(mom))
        if cyc in (1, 10):
            exp = doc["outputs"][f"cycle{cyc}"]
            for s in range(4):
                assert sha([ps[s][k] for k in "xyzuvw"]) == exp["particles"][s], (cyc, s)
                assert sha([moms[s]]) == exp["moments_bc"][s], (cyc, s)


@pytest.mark.skipif(not oracle.reference_available(32), reason="reference oracle not built here")
def test_restated_matches_reference_build_small_gem_cycle():
    """Where oracle/_ref exists, the two oracles agree bit for bit on one full
    driver cycle (mover_PC x4, then interpP2G + applyBCids in an OpenMP team)."""
    wl = W.small_gem()
    F = W.gem_fields(wl)
    setup = oracle.setup_from(wl)
    res = []
    for kind in ("restated", "reference"):
        O = oracle.CpuOracle(kind, 32)
        parts = [W.gem_particles(wl, s) for s in range(4)]
        mom = [np.zeros(wl.nodes, np.float32) for _ in range(40)]
        O.cycle(setup, F, parts, mom)
        res.append((parts, mom))
    for s in range(4):
        for k in "xyzuvw":
            assert np.array_equal(res[0][0][s][k], res[1][0][s][k])
    for a, b in zip(res[0][1], res[1][1]):
        assert np.array_equal(a, b)


@pytest.mark.skipif(not oracle.reference_available(32) or not oracle.reference_available(64),
                    reason="the reference build (oracle/_ref) exists where the reference tree does")
@pytest.mark.parametrize("fp", [32, 64])
@pytest.mark.parametrize("sort_cps", [1, 3, 8])
def test_particle_sort_restated_equals_reference(fp, sort_cps):
    """particle_sort restated against the reference's own, on shuffled GEM
    particles with some outside every bin (the last bin)."""
    wl = W.small_gem(E_amp=1e-3)
    setup = oracle.setup_from(wl)
    p0 = W.gem_particles(wl, 0)
    perm = np.random.default_rng(sort_cps).permutation(len(p0["x"]))
    p = {k: np.ascontiguousarray(p0[k][perm]) for k in "xyzuvwq"}
    p["x"][:5] = np.float32(-1.0)
    p["y"][5:7] = np.float32(11.0)
    if fp == 64:
        p = {k: v.astype(np.float64) for k, v in p.items()}
    a = {k: v.copy() for k, v in p.items()}
    b = {k: v.copy() for k, v in p.items()}
    assert oracle.CpuOracle("restated", fp).particle_sort(setup, sort_cps, a) == 0
    assert oracle.CpuOracle("reference", fp).particle_sort(setup, sort_cps, b) == 0
    for k in "xyzuvwq":
        assert np.array_equal(a[k], b[k]), k
    assert not np.array_equal(a["x"], p["x"])


def hat_case(per):
    """The grid, species qoms and theta of one hat-densities fixture case
    (tests/golden/hat_densities.json)."""
    wl = W.small_gem(nxc=8, nyc=6, nzc=5, periodic=tuple(bool(p) for p in per))
    return wl, [sp.qom for sp in wl.species[:3]], 1.0


@pytest.mark.parametrize("fp", [32, 64])
@pytest.mark.parametrize("per", [(1, 0, 1), (1, 1, 1), (0, 0, 0), (0, 1, 0)])
def test_hat_densities_restated_matches_reference_digests(fp, per):
    """calculateHatDensities (src/MaxwellSolver.cpp:465-603): the restatement
    reproduces the reference build's outputs bit for bit (SHA-256 of Jxh, Jyh,
    Jzh, rhoh), for periodic, reflecting and mixed axes."""
    with open(os.path.join(GOLDEN, "hat_densities.json")) as f:
        doc = json.load(f)
    wl, qom, th = hat_case(per)
    dt = np.float32 if fp == 32 else np.float64
    mom, fields, rhoc = W.hat_inputs(wl, seed=doc["seed"], dtype=dt, ns=doc["species"])
    out = oracle.CpuOracle("restated", fp).hat_densities(oracle.setup_from(wl), th, qom, mom,
                                                         fields, rhoc)
    assert sha(out) == doc["cases"][f"{''.join(map(str, per))}_fp{fp}"]
    assert all(np.isfinite(a).all() for a in out)
