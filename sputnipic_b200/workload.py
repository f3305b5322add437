"""Seeded synthetic GEM (Harris current sheet) workloads for the mover + P2G path.

The reference initialises its particles with ``initGEM`` (src/IC.cpp:7-188):
Harris-sheet B field, sech^2 density for the current-sheet species, uniform
background species, Maxwellian velocities. The workloads here keep that
physics but follow the benchmark descriptions of this project (uniform-random
or jittered-lattice placement, seeded GEM flux perturbation, optional random E),
and are generated from a counter-based hash so that any sub-range of cells can
be regenerated on its own: a bounded CPU sample of a large workload holds
exactly the particles of those cells.

Everything is float64 arithmetic rounded once to float32 (the reference's
PrecisionTypes). Positions use only exactly-rounded operations; velocities and
fields use numpy's transcendental functions. The CUDA generator in the library
(``spb_gen_gem_*``) uses the same hash and formulas, so positions match
bit-for-bit and velocities/fields to within a few float64 ulps before rounding.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

# splitmix64 constants (Steele, Lea, Flood: "Fast splittable pseudorandom
# number generators", OOPSLA 2014).
_GOLD = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def stream_key(seed: int, stream: int) -> np.uint64:
    """64-bit key of one random stream."""
    with np.errstate(over="ignore"):
        z = np.array([(seed & 0xFFFFFFFF) << 32 | (stream & 0xFFFFFFFF)], dtype=np.uint64)
        return _mix(z * _GOLD + _GOLD)[0]


def uniform(seed: int, stream: int, idx: np.ndarray) -> np.ndarray:
    """U[0,1) float64 with 53 random bits, one per counter value."""
    key = stream_key(seed, stream)
    with np.errstate(over="ignore"):
        z = _mix((idx.astype(np.uint64) + np.uint64(1)) * _GOLD + key)
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


# Stream numbering (shared with the CUDA generator).
STREAM_PHASE = 1
STREAM_E = 2            # 2, 3, 4: Ex, Ey, Ez
STREAM_SPECIES = 16     # + 16*species + {0,1,2: position, 3..6: velocity}


@dataclass(frozen=True)
class Species:
    qom: float
    rho0: float
    sheet: bool          # sech^2 current-sheet profile (else uniform)
    vth: float           # thermal speed, all three axes
    w0: float            # drift along z
    ppc: float           # particles per cell (fractional: cells alternate)


def gem_species(ppc=(27, 27, 27, 27)) -> tuple:
    """The four GEM species: sheet electrons, sheet ions, background
    electrons, background ions."""
    return (
        Species(qom=-64.0, rho0=1.0, sheet=True, vth=0.045, w0=-0.0065, ppc=ppc[0]),
        Species(qom=1.0, rho0=1.0, sheet=True, vth=0.0126, w0=0.0065, ppc=ppc[1]),
        Species(qom=-64.0, rho0=0.1, sheet=False, vth=0.045, w0=0.0, ppc=ppc[2]),
        Species(qom=1.0, rho0=0.1, sheet=False, vth=0.0126, w0=0.0, ppc=ppc[3]),
    )


@dataclass(frozen=True)
class GemWorkload:
    name: str
    nxc: int
    nyc: int
    nzc: int
    Lx: float = 20.0
    Ly: float = 10.0
    Lz: float = 10.0
    dt: float = 0.25
    c: float = 1.0
    niter: int = 3
    n_sub_cycles: int = 1
    periodic: tuple = (True, False, True)
    B0: float = 0.0195
    delta: float = 0.5
    pert: float = 0.1
    E_amp: float = 0.0
    lattice: int = 0       # 0: uniform random in the cell; n: n^3 jittered sub-lattice
    cycles: int = 1
    seed: int = 0
    species: tuple = field(default_factory=gem_species)

    # --- grid geometry (src/Grid.cpp:9-27) -----------------------------------
    @property
    def nxn(self):
        return self.nxc + 3

    @property
    def nyn(self):
        return self.nyc + 3

    @property
    def nzn(self):
        return self.nzc + 3

    @property
    def nodes(self) -> int:
        return self.nxn * self.nyn * self.nzn

    @property
    def cells(self) -> int:
        return self.nxc * self.nyc * self.nzc

    @property
    def dx(self):
        return self.Lx / self.nxc

    @property
    def dy(self):
        return self.Ly / self.nyc

    @property
    def dz(self):
        return self.Lz / self.nzc

    @property
    def invVOL(self) -> np.float32:
        return np.float32(1.0 / (self.dx * self.dy * self.dz))

    def species_count(self, s: int) -> int:
        return int(math.floor(self.cells * self.species[s].ppc + 1e-9))

    @property
    def total_particles(self) -> int:
        return sum(self.species_count(s) for s in range(len(self.species)))

    def node_coords(self):
        """1D node coordinates per axis, float32 as setGrid stores them."""
        xs = [(np.arange(n, dtype=np.float64) - 1.0) * d for n, d in
              ((self.nxn, self.dx), (self.nyn, self.dy), (self.nzn, self.dz))]
        return tuple(a.astype(np.float32) for a in xs)

    def with_(self, **kw) -> "GemWorkload":
        return replace(self, **kw)


def small_gem(**kw) -> GemWorkload:
    """Plain method, small GEM cycle: 32x16x16 cells, 27 ppc uniform random,
    4 species, 10 cycles, E = 0."""
    base = GemWorkload(name="gem-small-32x16x16", nxc=32, nyc=16, nzc=16, cycles=10,
                       species=gem_species((27, 27, 27, 27)))
    return replace(base, **kw)


def gem(**kw) -> GemWorkload:
    """Full GEM cycle: 128x64x64 cells, 4 x 65,536,000 particles (125 ppc on a
    5x5x5 jittered sub-lattice), E ~ U(-1e-3, 1e-3), one cycle."""
    base = GemWorkload(name="gem-128x64x64", nxc=128, nyc=64, nzc=64, lattice=5,
                       E_amp=1e-3, cycles=1, species=gem_species((125, 125, 125, 125)))
    return replace(base, **kw)


def dense_gem(**kw) -> GemWorkload:
    """Dense variant: 256x128x128 cells, 4 x 134,217,728 particles (32 ppc;
    the stated count wins over the stated 64 ppc, which would be twice it)."""
    base = GemWorkload(name="gem-dense-256x128x128", nxc=256, nyc=128, nzc=128,
                       E_amp=1e-3, cycles=1, species=gem_species((32, 32, 32, 32)))
    return replace(base, **kw)


def batching_gem(**kw) -> GemWorkload:
    """Batching form: uneven species 65.5M, 65.5M, 6.55M, 6.55M on the GEM
    grid (background at 12.5 ppc), 20 cycles."""
    base = GemWorkload(name="gem-batching-128x64x64", nxc=128, nyc=64, nzc=64,
                       E_amp=1e-3, cycles=20, species=gem_species((125, 125, 12.5, 12.5)))
    return replace(base, **kw)


PRESETS = {"small": small_gem, "gem": gem, "dense": dense_gem, "batching": batching_gem}


# --- fields -------------------------------------------------------------------
def gem_fields(wl: GemWorkload):
    """E and B on all nodes (ghost nodes included), float32, reference layout
    [nxn][nyn][nzn] flattened. B: Harris sheet B0 tanh((y-Ly/2)/delta) along x
    plus a divergence-free GEM flux perturbation of amplitude pert*B0 with a
    seeded phase along x. E: uniform in [-E_amp, E_amp) per node and axis."""
    xn, yn, zn = (a.astype(np.float64) for a in wl.node_coords())
    X = xn[:, None, None]
    Y = yn[None, :, None] - wl.Ly / 2
    phase = 2.0 * math.pi * float(uniform(wl.seed, STREAM_PHASE, np.zeros(1))[0])
    kx = 2.0 * math.pi / wl.Lx
    ky = math.pi / wl.Ly
    amp = wl.pert * wl.B0
    shape = (wl.nxn, wl.nyn, wl.nzn)
    bx = wl.B0 * np.tanh(Y / wl.delta) - amp * np.cos(kx * X + phase) * np.sin(ky * Y)
    by = amp * (kx / ky) * np.sin(kx * X + phase) * np.cos(ky * Y)
    Bx = np.broadcast_to(bx, shape).astype(np.float32).ravel()
    By = np.broadcast_to(by, shape).astype(np.float32).ravel()
    Bz = np.zeros(wl.nodes, np.float32)
    if wl.E_amp != 0.0:
        idx = np.arange(wl.nodes, dtype=np.uint64)
        E = [(wl.E_amp * (2.0 * uniform(wl.seed, STREAM_E + a, idx) - 1.0)).astype(np.float32)
             for a in range(3)]
    else:
        E = [np.zeros(wl.nodes, np.float32) for _ in range(3)]
    return [E[0], E[1], E[2], Bx, By, Bz]


# --- particles ----------------------------------------------------------------
def cell_counts(ppc: float, lo: int, hi: int) -> np.ndarray:
    """Particles in cells [lo, hi): floor((c+1) ppc) - floor(c ppc)."""
    c = np.arange(lo, hi + 1, dtype=np.float64)
    edges = np.floor(c * ppc + 1e-9).astype(np.int64)
    return np.diff(edges)


def gem_particles(wl: GemWorkload, s: int, cell_lo: int = 0, cell_hi: int | None = None) -> dict:
    """Particles of species ``s`` in active cells [cell_lo, cell_hi) (cells in
    x-major order, as initGEM loops, src/IC.cpp:121-125), float32 SoA.

    q = sign(qom) * rho(y_cell) / (4 pi) / ppc / invVOL, the reference's
    statistical weight (src/IC.cpp:139-141) with rho at the cell centre."""
    sp = wl.species[s]
    if cell_hi is None:
        cell_hi = wl.cells
    counts = cell_counts(sp.ppc, cell_lo, cell_hi)
    n = int(counts.sum())
    cell = np.repeat(np.arange(cell_lo, cell_hi, dtype=np.int64), counts)
    first = int(np.floor(cell_lo * sp.ppc + 1e-9))
    pidx = np.arange(first, first + n, dtype=np.int64).astype(np.uint64)
    starts = np.repeat(np.cumsum(counts) - counts, counts)
    k = np.arange(n, dtype=np.int64) - starts            # index inside the cell
    cx = cell // (wl.nyc * wl.nzc)
    cy = (cell // wl.nzc) % wl.nyc
    cz = cell % wl.nzc
    st = STREAM_SPECIES + 16 * s
    offs = [uniform(wl.seed, st + a, pidx) for a in range(3)]
    if wl.lattice:
        m = wl.lattice
        sub = (k // (m * m), (k // m) % m, k % m)
        offs = [(sub[a] + offs[a]) / m for a in range(3)]
    x = ((cx + offs[0]) * wl.dx).astype(np.float32)
    y = ((cy + offs[1]) * wl.dy).astype(np.float32)
    z = ((cz + offs[2]) * wl.dz).astype(np.float32)
    # Maxwellian: two Box-Muller pairs, three normals used
    u1, u2, u3, u4 = (uniform(wl.seed, st + 3 + a, pidx) for a in range(4))
    r1 = np.sqrt(-2.0 * np.log(1.0 - u1))
    r2 = np.sqrt(-2.0 * np.log(1.0 - u3))
    n1 = r1 * np.cos(2.0 * math.pi * u2)
    n2 = r1 * np.sin(2.0 * math.pi * u2)
    n3 = r2 * np.cos(2.0 * math.pi * u4)
    u = (sp.vth * n1).astype(np.float32)
    v = (sp.vth * n2).astype(np.float32)
    w = (sp.w0 + sp.vth * n3).astype(np.float32)
    if sp.sheet:
        yc = (cy + 0.5) * wl.dy - wl.Ly / 2
        rho = sp.rho0 / np.cosh(yc / wl.delta) ** 2
    else:
        rho = np.full(n, sp.rho0)
    q = (math.copysign(1.0, sp.qom) * rho / (4.0 * math.pi) / sp.ppc
         / float(wl.invVOL)).astype(np.float32)
    return {"x": x, "y": y, "z": z, "u": u, "v": v, "w": w, "q": q,
            "qom": sp.qom, "cell": cell.astype(np.int32)}


def _particles_chunk(args):
    wl, s, lo, hi = args
    p = gem_particles(wl, s, lo, hi)
    return lo, {k: p[k] for k in "xyzuvwq"}


def gem_particles_host(wl: GemWorkload, species=None, procs: int | None = None,
                       slabs_per_chunk: int = 2) -> list:
    """gem_particles of every cell for each species in ``species`` (all by
    default), generated by a pool of ``procs`` spawned processes (default:
    the host's cores), chunk by chunk of ``slabs_per_chunk`` x-slabs of cells
    and assembled in cell order: the same arrays as one gem_particles call per
    species. Returns a list of dicts (x..q float32, qom)."""
    import multiprocessing as mp
    import os
    species = range(len(wl.species)) if species is None else species
    plane = wl.nyc * wl.nzc
    step = slabs_per_chunk * plane
    procs = procs or os.cpu_count() or 1
    out = []
    with mp.get_context("spawn").Pool(procs) as pool:
        for s in species:
            ppc = wl.species[s].ppc
            n = wl.species_count(s)
            arr = {k: np.empty(n, np.float32) for k in "xyzuvwq"}
            chunks = [(wl, s, lo, min(lo + step, wl.cells)) for lo in range(0, wl.cells, step)]
            for lo, p in pool.imap_unordered(_particles_chunk, chunks):
                a = int(np.floor(lo * ppc + 1e-9))
                for k in "xyzuvwq":
                    arr[k][a:a + len(p[k])] = p[k]
            arr["qom"] = wl.species[s].qom
            out.append(arr)
    return out


def zero_moments(wl: GemWorkload, dtype=np.float32):
    return [np.zeros(wl.nodes, dtype) for _ in range(10)]


def hat_inputs(wl: GemWorkload, seed: int = 0, dtype=np.float32, ns: int | None = None):
    """Seeded inputs of calculateHatDensities on wl's grid: per species the 10
    node moments (rhon..pzz, magnitudes like a GEM deposit's: rho ~ 1, J ~
    1e-2, pressures ~ 1e-3), the six node fields (E ~ 1e-3, B ~ 0.05) and the
    net charge density on the cell centres (guard cells included)."""
    rng = np.random.default_rng(seed)
    ns = len(wl.species) if ns is None else ns
    scale = (1.0,) + (1e-2,) * 3 + (1e-3,) * 6
    mom = [[(rng.standard_normal(wl.nodes) * sc).astype(dtype) for sc in scale]
           for _ in range(ns)]
    fields = ([rng.uniform(-1e-3, 1e-3, wl.nodes).astype(dtype) for _ in range(3)]
              + [rng.uniform(-0.05, 0.05, wl.nodes).astype(dtype) for _ in range(3)])
    rhoc = rng.standard_normal((wl.nxc + 2) * (wl.nyc + 2) * (wl.nzc + 2)).astype(dtype)
    return mom, fields, rhoc
