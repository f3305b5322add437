"""Synthetic GEM workloads: sizes of the benchmark configurations, placement
inside cells, and that any cell sub-range regenerates the same particles."""
import numpy as np

from sputnipic_b200 import workload as W


def test_config_sizes():
    assert W.small_gem().species_count(0) == 32 * 16 * 16 * 27 == 221184
    g = W.gem()
    assert g.cells == 128 * 64 * 64
    assert [g.species_count(s) for s in range(4)] == [65_536_000] * 4
    assert g.nodes == 131 * 67 * 67 == 588_059
    d = W.dense_gem()
    assert d.species_count(0) == 134_217_728
    b = W.batching_gem()
    assert [b.species_count(s) for s in range(4)] == [65_536_000, 65_536_000, 6_553_600, 6_553_600]


def test_particles_inside_their_cells_and_domain():
    wl = W.small_gem()
    for s in range(4):
        p = W.gem_particles(wl, s)
        cx = p["cell"] // (wl.nyc * wl.nzc)
        cy = (p["cell"] // wl.nzc) % wl.nyc
        cz = p["cell"] % wl.nzc
        for key, c, d, L in (("x", cx, wl.dx, wl.Lx), ("y", cy, wl.dy, wl.Ly), ("z", cz, wl.dz, wl.Lz)):
            a = p[key].astype(np.float64)
            assert (a >= c * d - 1e-6).all() and (a <= (c + 1) * d + 1e-6).all()
            assert (a >= 0).all() and (a <= L).all()
        assert np.isfinite(p["u"]).all()
        assert (np.sign(p["q"]) == np.sign(wl.species[s].qom)).all()


def test_subrange_regenerates_the_same_particles():
    wl = W.gem(nxc=8, nyc=8, nzc=8)
    full = W.gem_particles(wl, 1)
    part = W.gem_particles(wl, 1, 100, 180)
    lo = 100 * 125
    for k in "xyzuvwq":
        assert np.array_equal(full[k][lo:lo + 80 * 125], part[k])


def test_fractional_ppc_alternates():
    c = W.cell_counts(12.5, 0, 10)
    assert c.sum() == 125 and set(c.tolist()) == {12, 13}


def test_jittered_lattice_fills_subcells():
    wl = W.gem(nxc=2, nyc=2, nzc=2)
    p = W.gem_particles(wl, 0, 0, 1)
    sub = np.floor(p["x"] / wl.dx * 5).astype(int)
    assert sorted(np.bincount(sub).tolist()) == [25] * 5


def test_fields_shapes_and_harris_profile():
    wl = W.small_gem()
    F = W.gem_fields(wl)
    assert all(f.dtype == np.float32 and f.size == wl.nodes for f in F)
    Bx = F[3].reshape(wl.nxn, wl.nyn, wl.nzn)
    assert np.sign(Bx[5, 2, 5]) == -1 and np.sign(Bx[5, -3, 5]) == 1
    assert np.abs(F[0]).max() == 0.0
    g = W.gem(nxc=8, nyc=8, nzc=8)
    E = W.gem_fields(g)[0]
    assert 0 < np.abs(E).max() <= 1e-3
