"""The particle load + cell sort that allocates nothing
(spb_sort_particles_noalloc), called through the C-ABI, against the existing
entry point that does the same work with scratch it allocates
(spb_sim_load_species, read back with spb_sim_particles).

Callers that cannot call cudaMalloc where they sort (codes whose device
memory belongs to their own pool allocator, loops that cannot take an
allocation's implicit synchronisation) use the no-alloc entry point; its
scratch is a fixed device array shared by all calls, so this file checks two
calls in a row (the second must not see the first call's counters).

Tolerance: the precision-form tests' 1e-5 on positions; velocities and
charges are moved, not computed, so they must be equal. Particle order inside
a cell is not fixed by either sort, so both outputs are put in the order of a
unique tag carried in q.
"""
import ctypes

import numpy as np
import pytest

from sputnipic_b200 import _lib
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu

TILE = (8, 4, 4)


def desc_for(wl, tile=TILE):
    d = _lib.SimDesc()
    d.nxc, d.nyc, d.nzc = wl.nxc, wl.nyc, wl.nzc
    d.Lx, d.Ly, d.Lz = wl.Lx, wl.Ly, wl.Lz
    d.dt, d.c, d.niter = wl.dt, wl.c, wl.niter
    d.ns = 1
    for a in range(3):
        d.tile[a] = tile[a]
    return d


def tile_keys(wl, cx, cy, cz, tile=TILE):
    TX, TY, TZ = tile
    nty, ntz = wl.nyc // TY, wl.nzc // TZ
    return (((cx // TX) * nty + cy // TY) * ntz + cz // TZ) * (TX * TY * TZ) \
        + ((cx % TX) * TY + cy % TY) * TZ + cz % TZ


def noalloc_sort(torch, wl, dev, n, tile=TILE, expect=0):
    lib = _lib.load()
    out = {"cell": torch.empty(n, dtype=torch.int32, device="cuda")}
    for k in ("ox", "oy", "oz", "u", "v", "w", "q"):
        out[k] = torch.empty(n, dtype=torch.float32, device="cuda")
    cs = torch.empty(wl.cells + 1, dtype=torch.int32, device="cuda")
    rc = lib.spb_sort_particles_noalloc(
        ctypes.byref(desc_for(wl, tile)), *[dev[k].data_ptr() for k in "xyzuvwq"], n,
        *[out[k].data_ptr() for k in ("cell", "ox", "oy", "oz", "u", "v", "w", "q")],
        cs.data_ptr(), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == expect, _lib.last_error()
    h = {k: v.cpu().numpy() for k, v in out.items()}
    return h, cs.cpu().numpy()


def positions(wl, h):
    c = h["cell"].view(np.uint32)
    cx, cy, cz = (c >> 21).astype(np.int64), ((c >> 11) & 1023).astype(np.int64), \
        (c & 2047).astype(np.int64)
    # x = (cell + offset) * dx, rounded to float as spb_sim_particles does
    x = ((cx + h["ox"].astype(np.float64)) * wl.dx).astype(np.float32)
    y = ((cy + h["oy"].astype(np.float64)) * wl.dy).astype(np.float32)
    z = ((cz + h["oz"].astype(np.float64)) * wl.dz).astype(np.float32)
    return x, y, z, cx, cy, cz


def check_against_existing(wl, h, cs, ref, n, tile=TILE):
    assert cs[0] == 0 and cs[-1] == n and (np.diff(cs) >= 0).all()
    x, y, z, cx, cy, cz = positions(wl, h)
    # every particle sits in the segment of its own cell
    seg = np.repeat(np.arange(wl.cells), np.diff(cs))
    assert np.array_equal(seg, tile_keys(wl, cx, cy, cz, tile))
    order = np.argsort(h["q"], kind="stable")
    rorder = np.argsort(ref["q"], kind="stable")
    assert np.array_equal(h["q"][order], ref["q"][rorder])
    for k, a in (("x", x), ("y", y), ("z", z)):
        assert np.abs(a[order].astype(np.float64) - ref[k][rorder]).max() <= 1e-5, k
    for k in "uvw":
        assert np.array_equal(h[k][order], ref[k][rorder]), k


@pytest.mark.parametrize("tile", [(8, 4, 4), (4, 4, 4), (2, 2, 2), (8, 8, 4)])
def test_noalloc_sort_matches_allocating_load_two_calls(cuda, tile):
    """Every tile shape the library instantiates: two calls in a row against
    the allocating load, then a smaller call after the larger one."""
    torch = cuda
    from sputnipic_b200.sim import Simulation
    wl = W.small_gem()
    host = W.gem_particles(wl, 0)
    n = len(host["x"])
    host["q"] = np.arange(n, dtype=np.float32)       # unique tags
    dev = {k: torch.from_numpy(host[k]).cuda() for k in "xyzuvwq"}
    sim = Simulation(wl, tile=tile, species=[0])
    sim.load_species(0, dev)
    ref = {k: v.cpu().numpy() for k, v in sim.particles(0).items()}
    sim.close()
    for _ in range(2):                               # two calls in a row
        h, cs = noalloc_sort(torch, wl, dev, n, tile)
        check_against_existing(wl, h, cs, ref, n, tile)
    # a smaller call after a larger one: the counters start from zero again
    m = n // 3
    half = {k: v[:m].contiguous() for k, v in dev.items()}
    sim = Simulation(wl, tile=tile, species=[0])
    sim.load_species(0, half)
    ref_m = {k: v.cpu().numpy() for k, v in sim.particles(0).items()}
    sim.close()
    h, cs = noalloc_sort(torch, wl, half, m, tile)
    check_against_existing(wl, h, cs, ref_m, m, tile)


def test_noalloc_sort_reports_positions_outside_the_domain(cuda):
    """One position beyond Lx: SPB_ERR_OUT_OF_GRID; the next clean call on
    the shared scratch returns 0 again (its error word was cleared)."""
    torch = cuda
    wl = W.small_gem()
    host = W.gem_particles(wl, 0)
    n = len(host["x"])
    host["q"] = np.arange(n, dtype=np.float32)
    bad = {k: host[k].copy() for k in "xyzuvwq"}
    bad["x"][n // 2] = np.float32(wl.Lx * 1.5)
    dev_bad = {k: torch.from_numpy(bad[k]).cuda() for k in "xyzuvwq"}
    noalloc_sort(torch, wl, dev_bad, n, expect=3)     # SPB_ERR_OUT_OF_GRID
    assert b"outside" in _lib.load().spb_last_error_message()
    dev = {k: torch.from_numpy(host[k]).cuda() for k in "xyzuvwq"}
    h, cs = noalloc_sort(torch, wl, dev, n)
    assert cs[-1] == n


def test_noalloc_sort_rejects_grids_beyond_its_scratch(cuda):
    lib = _lib.load()
    big = W.GemWorkload(name="too-big", nxc=256, nyc=128, nzc=64)
    assert big.cells > (1 << 20)
    rc = lib.spb_sort_particles_noalloc(ctypes.byref(desc_for(big)), *([None] * 7), 0,
                                        *([None] * 8), None, None)
    assert rc == 2 == lib.spb_last_error()            # SPB_ERR_INVALID: null cell_start
    # a null cell_start is rejected first; with one given, the capacity check fires
    cs = cuda.empty(1, dtype=cuda.int32, device="cuda")
    rc = lib.spb_sort_particles_noalloc(ctypes.byref(desc_for(big)), *([None] * 7), 0,
                                        *([None] * 8), cs.data_ptr(), None)
    assert rc == 8 == lib.spb_last_error()            # SPB_ERR_CAPACITY
    assert b"cells" in lib.spb_last_error_message()
