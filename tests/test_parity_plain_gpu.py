"""Parity of the plain form (reference precision types) on the GPU, through
the C-ABI: the drop-in mover_PC / mover_PC_V / interpP2G / mover_interp over
the reference structs, and the device-pointer API.

Bar: particle positions and velocities (hence cell indices, boundary
crossings and counts) bit-identical to the reference CPU code. Moments are
FP32 sums in a different order: every node must satisfy
    |gpu - ref| <= 32 * eps32 * sum_p |term_p|
(the rounding bound of a reordered float sum, with the sum of absolute
summands taken from the FP64 oracle), and the GPU's relative L2 error
against the FP64 oracle must not exceed the reference FP32 code's by more
than 2x + 1e-7.
"""
import threading

import numpy as np
import pytest

import oracle
from conftest import edge_workload
from sputnipic_b200 import dropin
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu

EPS32 = float(np.finfo(np.float32).eps)


@pytest.fixture(scope="module")
def orc32():
    return oracle.CpuOracle("restated", 32)


@pytest.fixture(scope="module")
def orc64():
    return oracle.CpuOracle("restated", 64)


@pytest.fixture(autouse=True)
def _clean_state(cuda):
    dropin.set_residency(False)
    yield
    dropin.release_all()


def abs_moments(orc64, setup, wl, part):
    """Per node sum of |summand| of each moment, in FP64."""
    p = {k: np.abs(part[k].astype(np.float64)) for k in "uvwq"}
    for k in "xyz":
        p[k] = part[k].astype(np.float64)
    mom = [np.zeros(wl.nodes) for _ in range(10)]
    orc64.interp_p2g(setup, p, mom)
    return np.stack(mom)


def check_moments(gpu, ref32, absm, ref64=None):
    gpu, ref32 = np.asarray(gpu, np.float64), np.asarray(ref32, np.float64)
    bound = 32 * EPS32 * absm + 1e-30
    bad = np.abs(gpu - ref32) > bound
    assert not bad.any(), f"{bad.sum()} moment entries outside the reordering bound"
    if ref64 is not None:
        for m in range(10):
            n64 = np.linalg.norm(ref64[m])
            if n64 == 0:
                continue
            e_gpu = np.linalg.norm(gpu[m] - ref64[m]) / n64
            e_cpu = np.linalg.norm(ref32[m] - ref64[m]) / n64
            assert e_gpu <= 2 * e_cpu + 1e-7, (m, e_gpu, e_cpu)


def build(wl, fields, parts, ns=None):
    param = dropin.make_parameters(wl)
    grd = dropin.setGrid(param)
    field = dropin.field_allocate(grd, fields)
    P = [dropin.particle_allocate(param, s, arrays=p) for s, p in enumerate(parts)]
    return param, grd, field, P


def edge_inputs(d, qi):
    wl = edge_workload(d)
    fields = [d[f"field_{n}"] for n in oracle.FIELDS]
    part = {k: d[f"in_{k}"].copy() for k in "xyzuvwq"}
    param, grd, field, (P,) = build(wl, fields, [part])
    P.qom = float(d["qom"][qi])
    return wl, param, grd, field, P


@pytest.mark.parametrize("qi", [0, 1])
@pytest.mark.parametrize("variant", ["mover", "moverv"])
def test_edge_mover_bitexact(golden_edge, qi, variant):
    d = golden_edge
    wl, param, grd, field, P = edge_inputs(d, qi)
    fn = dropin.mover_PC if variant == "mover" else dropin.mover_PC_V
    assert fn(P, field, grd, param) == 0
    out = dropin.particle_arrays(P)
    for k in "xyzuvw":
        ref = d[f"fp32_q{qi}_{variant}_{k}"]
        assert np.array_equal(out[k], ref), f"{k}: {np.sum(out[k] != ref)} of {ref.size} differ"


@pytest.mark.parametrize("qi", [0, 1])
def test_edge_interp_p2g(golden_edge, orc64, qi):
    d = golden_edge
    wl = edge_workload(d)
    part = {k: d[f"fp32_q{qi}_mover_{k}"].copy() for k in "xyzuvw"}
    part["q"] = d["in_q"].copy()
    param, grd, field, (P,) = build(wl, [d[f"field_{n}"] for n in oracle.FIELDS], [part])
    ids = dropin.interp_dens_species_allocate(grd, 0)
    dropin.interpP2G(P, ids, grd, raise_on_error=True)
    once = np.stack(dropin.moments(ids)).copy()
    setup = oracle.setup_from(wl)
    absm = abs_moments(orc64, setup, wl, part)
    check_moments(once, d[f"fp32_q{qi}_p2g"], absm)
    # interpP2G adds into what the caller passes: a second call doubles it
    dropin.interpP2G(P, ids, grd, raise_on_error=True)
    check_moments(np.stack(dropin.moments(ids)), 2.0 * d[f"fp32_q{qi}_p2g"], 2.0 * absm)


@pytest.fixture(params=["accumulator", "direct"])
def deposit_mode(request):
    """Both plain deposit forms: through the node-interleaved accumulator and
    straight into the ten moment arrays (the fallback when the accumulator
    cannot be allocated)."""
    from sputnipic_b200.device import set_plain_deposit_mode
    prev = set_plain_deposit_mode(request.param)
    yield request.param
    set_plain_deposit_mode(prev)


@pytest.mark.parametrize("qi", [0, 1])
def test_edge_mover_interp(golden_edge, orc64, qi, deposit_mode):
    d = golden_edge
    wl, param, grd, field, P = edge_inputs(d, qi)
    ids = dropin.interp_dens_species_allocate(grd, 0)
    assert dropin.mover_interp(P, field, ids, grd, param) == 0
    out = dropin.particle_arrays(P)
    for k in "xyzuvw":
        assert np.array_equal(out[k], d[f"fp32_q{qi}_fused_{k}"]), k
    setup = oracle.setup_from(wl)
    absm = abs_moments(orc64, setup, wl, out)
    check_moments(np.stack(dropin.moments(ids)), d[f"fp32_q{qi}_fused_mom"], absm)


def test_small_gem_1ppc_ten_cycles(golden_small_1ppc):
    d = golden_small_1ppc
    wl = W.small_gem(species=W.gem_species((1, 1, 1, 1)))
    fields = [d[f"field_{n}"] for n in oracle.FIELDS]
    parts = [{k: d[f"in_s{s}_{k}"].copy() for k in "xyzuvwq"} for s in range(4)]
    param, grd, field, P = build(wl, fields, parts)
    for cyc in range(1, 11):
        for s in range(4):
            assert dropin.mover_PC(P[s], field, grd, param) == 0
        if cyc in (1, 10):
            for s in range(4):
                out = dropin.particle_arrays(P[s])
                for k in "xyzuvw":
                    assert np.array_equal(out[k], d[f"c{cyc}_s{s}_{k}"]), (cyc, s, k)


def test_small_gem_full_cycle_vs_oracle(orc32, orc64):
    """The full small GEM config (4 x 221,184 particles), 10 cycles of
    mover_PC then interpP2G + applyBCids, against the restated oracle."""
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    ref = [{k: p[k].copy() for k in "xyzuvwq"} for p in parts]
    param, grd, field, P = build(wl, fields, [{k: p[k].copy() for k in "xyzuvwq"} for p in parts])
    setup = oracle.setup_from(wl)
    ids = [dropin.interp_dens_species_allocate(grd, s) for s in range(4)]
    for cyc in range(10):
        for s in range(4):
            assert dropin.mover_PC(P[s], field, grd, param) == 0
            orc32.mover_pc(setup, fields, ref[s], wl.species[s].qom)
    for s in range(4):
        out = dropin.particle_arrays(P[s])
        for k in "xyzuvw":
            assert np.array_equal(out[k], ref[s][k]), (s, k)
        dropin.setZeroSpeciesDensities(ids[s])
        dropin.interpP2G(P[s], ids[s], grd, raise_on_error=True)
        mom = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
        orc32.interp_p2g(setup, ref[s], mom)
        m64 = [np.zeros(wl.nodes) for _ in range(10)]
        orc64.interp_p2g(setup, {k: ref[s][k].astype(np.float64) for k in "xyzuvwq"}, m64)
        absm = abs_moments(orc64, setup, wl, ref[s])
        check_moments(np.stack(dropin.moments(ids[s])), np.stack(mom), absm, np.stack(m64))


def test_device_api_and_bc_on_device(cuda, orc32, orc64):
    torch = cuda
    from sputnipic_b200.device import GridContext, push_params
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    setup = oracle.setup_from(wl)
    ctx = GridContext(wl)
    ctx.set_fields([torch.from_numpy(f).cuda() for f in fields])
    for s in (0, 1):
        host = W.gem_particles(wl, s)
        dev = {k: torch.from_numpy(host[k]).cuda() for k in "xyzuvwq"}
        ref = {k: host[k].copy() for k in "xyzuvwq"}
        mom = torch.zeros(10, wl.nodes, device="cuda")
        ctx.mover_interp(dev, push_params(wl, s), mom)
        assert ctx.check() == 0
        orc32.mover_pc(setup, fields, ref, wl.species[s].qom)
        for k in "xyzuvw":
            assert np.array_equal(dev[k].cpu().numpy(), ref[k]), (s, k)
        m32 = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
        orc32.interp_p2g(setup, ref, m32)
        absm = abs_moments(orc64, setup, wl, ref)
        check_moments(mom.cpu().numpy(), np.stack(m32), absm)
        # applyBCids on device equals the oracle's applied to the same input
        host_mom = [a.copy() for a in mom.cpu().numpy()]
        ctx.apply_bc_ids(mom, wl.periodic)
        orc32.apply_bc_ids(setup, host_mom)
        assert np.array_equal(mom.cpu().numpy(), np.stack(host_mom))
    ctx.close()


def test_concurrent_interp_from_threads(orc64):
    """interpP2G called from 4 threads at once (the reference's OpenMP team
    over species) gives the same moments as sequential calls."""
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    param, grd, field, P = build(wl, fields, parts)
    seq = []
    for s in range(4):
        ids = dropin.interp_dens_species_allocate(grd, s)
        dropin.interpP2G(P[s], ids, grd, raise_on_error=True)
        seq.append(np.stack(dropin.moments(ids)))
    par = [dropin.interp_dens_species_allocate(grd, s) for s in range(4)]
    errs = []

    def work(s):
        try:
            dropin.interpP2G(P[s], par[s], grd, raise_on_error=True)
        except Exception as e:  # noqa: BLE001
            errs.append(e)

    th = [threading.Thread(target=work, args=(s,)) for s in range(4)]
    [t.start() for t in th]
    [t.join() for t in th]
    assert not errs
    setup = oracle.setup_from(wl)
    for s in range(4):
        absm = abs_moments(orc64, setup, wl, parts[s])
        check_moments(np.stack(dropin.moments(par[s])), seq[s], absm)


def test_device_residency_defers_host_copy(orc64):
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    part = W.gem_particles(wl, 0)
    param, grd, field, (Pc,) = build(wl, fields, [{k: part[k].copy() for k in "xyzuvwq"}])
    assert dropin.mover_PC(Pc, field, grd, param) == 0
    copy_mode = {k: v.copy() for k, v in dropin.particle_arrays(Pc).items()}
    dropin.release_all()
    param, grd, field, (Pd,) = build(wl, fields, [{k: part[k].copy() for k in "xyzuvwq"}])
    assert dropin.set_residency(True) == 0
    assert dropin.mover_PC(Pd, field, grd, param) == 0
    host = dropin.particle_arrays(Pd)
    assert np.array_equal(host["x"], part["x"])            # host not refreshed yet
    assert dropin.set_residency(False) != 0                # refuses while host is stale
    ids = dropin.interp_dens_species_allocate(grd, 0)
    dropin.interpP2G(Pd, ids, grd, raise_on_error=True)    # deposits the device copy
    assert dropin.sync_particles_to_host(Pd) == 0
    for k in "xyzuvw":
        assert np.array_equal(host[k], copy_mode[k])
    ids_c = dropin.interp_dens_species_allocate(grd, 0)
    dropin.set_residency(False)
    dropin.interpP2G(Pd, ids_c, grd, raise_on_error=True)
    moved = {k: host[k].astype(np.float32) for k in "xyzuvwq"}
    absm = abs_moments(orc64, oracle.setup_from(wl), wl, moved)
    check_moments(np.stack(dropin.moments(ids)), np.stack(dropin.moments(ids_c)), absm)


@pytest.mark.parametrize("n", [0, 1, 31, 33, 255, 257, 4097])
def test_ragged_sizes(orc32, n):
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    full = W.gem_particles(wl, 0, 0, 40)
    part = {k: full[k][:n].copy() for k in "xyzuvwq"}
    ref = {k: v.copy() for k, v in part.items()}
    param, grd, field, (P,) = build(wl, fields, [part])
    assert dropin.mover_PC(P, field, grd, param) == 0
    if n:
        orc32.mover_pc(oracle.setup_from(wl), fields, ref, wl.species[0].qom)
    out = dropin.particle_arrays(P)
    for k in "xyzuvw":
        assert np.array_equal(out[k], ref[k])


def test_out_of_grid_particle_is_flagged_not_faulting(orc32):
    """A particle far outside the grid (the reference reads out of bounds for
    it) is clamped to the edge cell and reported as SPB_ERR_OUT_OF_GRID; the
    other particles are still bit-exact."""
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    part = W.gem_particles(wl, 0, 0, 20)
    part = {k: part[k].copy() for k in "xyzuvwq"}
    part["x"][7] = -50.0
    part["y"][11] = np.float32("nan")
    ref = {k: v.copy() for k, v in part.items()}
    param, grd, field, (P,) = build(wl, fields, [part])
    assert dropin.mover_PC(P, field, grd, param) == 3
    assert dropin.last_error()[0] == 3
    good = np.ones(len(ref["x"]), bool)
    good[[7, 11]] = False
    sel = {k: v[good].copy() for k, v in ref.items()}
    orc32.mover_pc(oracle.setup_from(wl), fields, sel, wl.species[0].qom)
    out = dropin.particle_arrays(P)
    for k in "xyzuvw":
        assert np.array_equal(out[k][good], sel[k])


def test_copy_residency_pipeline_over_chunk_boundaries(orc32, orc64, deposit_mode):
    """COPY residency moves species above 4M particles through PCIe in chunks on
    rotating streams. 9.2M particles (several chunk boundaries, chunks of
    unequal sizes): mover_PC bit-identical to the reference code, interpP2G within the
    reordering bound, as for one launch; both deposit forms (the chunks of
    both streams add into one accumulator, folded once)."""
    wl = W.small_gem(nxc=64, nyc=32, nzc=32, E_amp=1e-3,
                     species=W.gem_species((140, 140, 140, 140)))
    fields = W.gem_fields(wl)
    part = W.gem_particles(wl, 0)
    assert len(part["x"]) > 2 * (1 << 22)
    ref = {k: part[k].copy() for k in "xyzuvwq"}
    param, grd, field, P = build(wl, fields, [{k: part[k].copy() for k in "xyzuvwq"}])
    ids = dropin.interp_dens_species_allocate(grd, 0)
    assert dropin.mover_PC(P[0], field, grd, param) == 0
    dropin.interpP2G(P[0], ids, grd, raise_on_error=True)
    setup = oracle.setup_from(wl)
    orc32.mover_pc(setup, fields, ref, wl.species[0].qom)
    out = dropin.particle_arrays(P[0])
    for k in "xyzuvw":
        assert np.array_equal(out[k], ref[k]), k
    mom = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
    orc32.interp_p2g(setup, ref, mom)
    check_moments(np.stack(dropin.moments(ids)), np.stack(mom), abs_moments(orc64, setup, wl, ref))


def test_device_p2g_into_separate_moment_arrays(cuda, orc32, orc64, deposit_mode):
    """spb_grid_p2g into ten moment arrays at irregular offsets (the deposit's
    node-interleaved accumulator is added into them) that already hold
    values: the result is those values plus the deposit, within the
    reordering bound."""
    torch = cuda
    from sputnipic_b200.device import GridContext
    wl = W.small_gem()
    fields = W.gem_fields(wl)
    setup = oracle.setup_from(wl)
    ctx = GridContext(wl)
    ctx.set_fields([torch.from_numpy(f).cuda() for f in fields])
    host = W.gem_particles(wl, 1)
    dev = {k: torch.from_numpy(host[k]).cuda() for k in "xyzuvwq"}
    # slices of one buffer at irregular offsets
    offs = [m * wl.nodes + 4 * m * m for m in range(10)]
    buf = torch.full((offs[-1] + wl.nodes,), 0.25, device="cuda")
    mom = [buf[o:o + wl.nodes] for o in offs]
    steps = {mom[m + 1].data_ptr() - mom[m].data_ptr() for m in range(9)}
    assert len(steps) > 1
    ctx.p2g(dev, mom)
    assert ctx.check() == 0
    m32 = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
    orc32.interp_p2g(setup, host, m32)
    absm = abs_moments(orc64, setup, wl, host)
    got = np.stack([m.cpu().numpy() for m in mom]).astype(np.float64) - 0.25
    check_moments(got, np.stack(m32), absm + 0.25)
    ctx.close()


def test_device_p2g_clumped_shuffled_input(cuda, orc32, orc64, deposit_mode):
    """spb_grid_p2g above the size where the deposit sorts its particles by
    cell first (442K particles): a third of them in one cell (a run longer
    than a CTA's chunk, split over warps and CTAs), the arrays in a seeded
    random order. Nodes the clump does not reach: within the reordering
    bound of the FP32 oracle. The clump's 8 nodes: a sequential FP32 sum of
    147K terms is itself far from exact there (the reference code's own
    result is up to 4 x 32 eps sum|terms| from the FP64 oracle), so they are
    held to the FP64 oracle within 128 eps sum|terms|; a run deposited twice
    or dropped would be off by 1/1150 of the node's value, over 50x that."""
    torch = cuda
    from sputnipic_b200.device import GridContext
    wl = W.small_gem()
    setup = oracle.setup_from(wl)
    ctx = GridContext(wl)
    ctx.set_fields([torch.from_numpy(f).cuda() for f in W.gem_fields(wl)])
    a, b = W.gem_particles(wl, 0), W.gem_particles(wl, 1)
    host = {k: np.concatenate([a[k], b[k]]) for k in "xyzuvwq"}
    n = len(host["x"])
    assert n > 400_000
    rng = np.random.default_rng(5)
    clump = rng.choice(n, n // 3, replace=False)
    for k, c, d in (("x", 17, wl.dx), ("y", 9, wl.dy), ("z", 4, wl.dz)):
        host[k][clump] = ((c + rng.uniform(0.05, 0.95, len(clump))) * d).astype(np.float32)
    order = rng.permutation(n)
    host = {k: np.ascontiguousarray(v[order]) for k, v in host.items()}
    mom = torch.zeros(10, wl.nodes, device="cuda")
    ctx.p2g({k: torch.from_numpy(v).cuda() for k, v in host.items()}, mom)
    assert ctx.check() == 0
    m32 = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
    orc32.interp_p2g(setup, host, m32)
    m64 = [np.zeros(wl.nodes) for _ in range(10)]
    orc64.interp_p2g(setup, {k: v.astype(np.float64) for k, v in host.items()}, m64)
    absm = abs_moments(orc64, setup, wl, host)
    gpu = mom.cpu().numpy().astype(np.float64)
    clumped = np.zeros(wl.nodes, bool)
    cell = {k: ((c + 0.5) * d) for k, c, d in (("x", 17, wl.dx), ("y", 9, wl.dy), ("z", 4, wl.dz))}
    one = {k: np.array([cell[k] if k in cell else 1.0], np.float32) for k in "xyzuvwq"}
    probe = abs_moments(orc64, setup, wl, one)
    clumped[(probe != 0).any(axis=0)] = True
    assert clumped.sum() == 8
    check_moments(gpu[:, ~clumped], np.stack(m32)[:, ~clumped], absm[:, ~clumped])
    err = np.abs(gpu[:, clumped] - np.stack(m64)[:, clumped])
    assert (err <= 128 * EPS32 * absm[:, clumped]).all(), (err / (EPS32 * absm[:, clumped])).max()
    ctx.close()


@pytest.mark.parametrize("residency", ["copy", "device"])
def test_interp_all_species_matches_driver_section(orc32, orc64, residency):
    """spb_interp_all_species against the reference driver's moment section
    (zero, interpP2G per species, applyBCids per species, sumOverSpecies) run
    with the oracle: species moments within the reordering bound (the bound's
    sums of |terms| go through the same linear applyBCids), net moments
    bit-identical to the float sum of the returned species moments in species
    order, rhoc zeroed."""
    wl = W.small_gem(E_amp=1e-3)
    fields = W.gem_fields(wl)
    parts = [W.gem_particles(wl, s) for s in range(4)]
    param, grd, field, P = build(wl, fields, [{k: p[k].copy() for k in "xyzuvwq"} for p in parts])
    if residency == "device":
        assert dropin.set_residency(True) == 0
    # one mover step first, so the deposit sees moved particles
    for s in range(4):
        assert dropin.mover_PC(P[s], field, grd, param) == 0
    ids = [dropin.interp_dens_species_allocate(grd, s) for s in range(4)]
    idn = dropin.interp_dens_net_allocate(grd)
    for i in ids:
        i._arrays["rhoc"][...] = 7.0
    idn._arrays["rhoc"][...] = 7.0
    assert dropin.interp_all_species(P, ids, idn, grd, param) == 0
    if residency == "device":
        for s in range(4):
            assert dropin.sync_particles_to_host(P[s]) == 0
    setup = oracle.setup_from(wl)
    net = np.zeros((10, wl.nodes), np.float32)
    for s in range(4):
        moved = dropin.particle_arrays(P[s])
        ref = [np.zeros(wl.nodes, np.float32) for _ in range(10)]
        orc32.interp_p2g(setup, moved, ref)
        orc32.apply_bc_ids(setup, ref)
        absm = list(abs_moments(orc64, setup, wl, moved))
        orc64.apply_bc_ids(setup, absm)
        got = np.stack(dropin.moments(ids[s]))
        check_moments(got, np.stack(ref), np.stack(absm))
        net = net + got
        assert not ids[s]._arrays["rhoc"].any()
    assert np.array_equal(np.stack(dropin.moments(idn)), net)
    assert not idn._arrays["rhoc"].any()
    dropin.set_residency(False)


@pytest.mark.parametrize("residency", ["copy", "device"])
@pytest.mark.parametrize("sort_cps", [1, 2, 5])
def test_particle_sort_bitexact(orc32, residency, sort_cps):
    """spb_particle_sort against particle_sort (the oracle, itself pinned to the
    reference's own): shuffled GEM particles, a few outside every bin,
    identical arrays after the sort (order within a bin included). DEVICE
    residency sorts the resident copy and syncs on request."""
    wl = W.small_gem(E_amp=1e-3)
    fields = W.gem_fields(wl)
    p0 = W.gem_particles(wl, 1)
    perm = np.random.default_rng(sort_cps).permutation(len(p0["x"]))
    part = {k: np.ascontiguousarray(p0[k][perm]) for k in "xyzuvwq"}
    if residency == "copy":   # outside every bin (the mover would flag them)
        part["x"][:3] = np.float32(-0.5)
        part["z"][3:9] = np.float32(wl.Lz + 1.0)
    param, grd, field, P = build(wl, fields, [{k: part[k].copy() for k in "xyzuvwq"}])
    param.sort_cps = sort_cps
    if residency == "device":
        # the device copy is the newest and holds q: the sort runs where it lies
        assert dropin.set_residency(True) == 0
        assert dropin.mover_PC(P[0], field, grd, param) == 0
        dropin.interpP2G(P[0], dropin.interp_dens_species_allocate(grd, 1), grd,
                         raise_on_error=True)
        orc32.mover_pc(oracle.setup_from(wl), fields, part, wl.species[0].qom)   # allocated as species 0
    assert dropin.particle_sort(param, P[0], grd) == 0
    if residency == "device":
        assert dropin.sync_particles_to_host(P[0]) == 0
    ref = {k: part[k].copy() for k in "xyzuvwq"}
    assert orc32.particle_sort(oracle.setup_from(wl), sort_cps, ref) == 0
    got = dropin.particle_arrays(P[0])
    for k in "xyzuvwq":
        assert np.array_equal(got[k], ref[k]), k
    dropin.set_residency(False)
