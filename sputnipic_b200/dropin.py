"""The reference's interface for the mover + P2G path, in Python.

Same names, argument meaning and results as sputniPIC's C++ functions:

* ``setGrid(param)`` (src/Grid.cpp:5-62), ``field_allocate(grd)``
  (src/EMfield.cpp:4-13), ``particle_allocate(param, is)``
  (src/Particles.cpp:5-54), ``interp_dens_species_allocate(grd, is)``
  (src/InterpDensSpecies.cpp:4-42) build the reference structs over numpy
  arrays (the structs are ctypes mirrors with the reference's layout);
* ``mover_PC``, ``mover_PC_V``, ``interpP2G``, ``mover_interp``
  (include/Mover.h:11-26), ``calculateHatDensities``
  (include/MaxwellSolver.h:37-40) call the CUDA library's drop-in entry
  points with those structs, exactly as the reference's C++ driver would.

mover_PC / mover_PC_V / mover_interp return the library status (0 = ok,
as the reference's always-0 return); interpP2G returns None and leaves its
status in ``last_error()``. Set ``raise_on_error=True`` to get exceptions.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import EMfield, Grid, InterpDensSpecies, Parameters, Particles, MOMENT_NAMES

FIELD_NAMES = ("Ex", "Ey", "Ez", "Bxn", "Byn", "Bzn")


def _keep(obj, name, arr):
    if not hasattr(obj, "_arrays"):
        obj._arrays = {}
    obj._arrays[name] = arr
    return arr.ctypes.data


def make_parameters(wl, ns: int | None = None) -> Parameters:
    """A ``struct parameters`` for a workload (``sputnipic_b200.workload``):
    the members the mover/P2G path reads plus the species table."""
    p = Parameters()
    p.c, p.fourpi, p.dt, p.th = wl.c, 4.0 * np.pi, wl.dt, 1.0
    p.ncycles, p.NiterMover, p.n_sub_cycles = wl.cycles, wl.niter, wl.n_sub_cycles
    p.Lx, p.Ly, p.Lz = wl.Lx, wl.Ly, wl.Lz
    p.nxc, p.nyc, p.nzc = wl.nxc, wl.nyc, wl.nzc
    ns = len(wl.species) if ns is None else ns
    p.ns = ns
    for s in range(ns):
        sp = wl.species[s]
        p.qom[s] = sp.qom
        p.rhoINIT[s] = sp.rho0
        p.uth[s] = p.vth[s] = p.wth[s] = sp.vth
        p.w0[s] = sp.w0
        p.np[s] = p.npMax[s] = wl.species_count(s)
    p.PERIODICX, p.PERIODICY, p.PERIODICZ = (bool(v) for v in wl.periodic)
    p.PERIODICX_P, p.PERIODICY_P, p.PERIODICZ_P = (bool(v) for v in wl.periodic)
    p.delta, p.B0x = wl.delta, wl.B0
    return p


def setGrid(param: Parameters) -> Grid:
    """src/Grid.cpp:5-62: guard cells, spacings, inverses rounded to float,
    node coordinates XN[i][j][k] = (float)(xStart + (i-1)*dx)."""
    g = Grid()
    g.nxc, g.nyc, g.nzc = param.nxc + 2, param.nyc + 2, param.nzc + 2
    g.nxn, g.nyn, g.nzn = g.nxc + 1, g.nyc + 1, g.nzc + 1
    g.dx, g.dy, g.dz = param.Lx / param.nxc, param.Ly / param.nyc, param.Lz / param.nzc
    g.invVOL = float(np.float32(1.0 / (g.dx * g.dy * g.dz)))
    g.invdx = float(np.float32(1.0 / g.dx))
    g.invdy = float(np.float32(1.0 / g.dy))
    g.invdz = float(np.float32(1.0 / g.dz))
    g.xStart, g.xEnd = 0.0, param.Lx
    g.yStart, g.yEnd = 0.0, param.Ly
    g.zStart, g.zEnd = 0.0, param.Lz
    g.Lx, g.Ly, g.Lz = param.Lx, param.Ly, param.Lz
    g.PERIODICX, g.PERIODICY, g.PERIODICZ = param.PERIODICX, param.PERIODICY, param.PERIODICZ
    shape = (g.nxn, g.nyn, g.nzn)
    xs = ((np.arange(g.nxn) - 1) * g.dx).astype(np.float32)
    ys = ((np.arange(g.nyn) - 1) * g.dy).astype(np.float32)
    zs = ((np.arange(g.nzn) - 1) * g.dz).astype(np.float32)
    XN = np.ascontiguousarray(np.broadcast_to(xs[:, None, None], shape)).ravel()
    YN = np.ascontiguousarray(np.broadcast_to(ys[None, :, None], shape)).ravel()
    ZN = np.ascontiguousarray(np.broadcast_to(zs[None, None, :], shape)).ravel()
    g.XN_flat = _keep(g, "XN", XN)
    g.YN_flat = _keep(g, "YN", YN)
    g.ZN_flat = _keep(g, "ZN", ZN)
    return g


def nodes(grd: Grid) -> int:
    return grd.nxn * grd.nyn * grd.nzn


def field_allocate(grd: Grid, arrays=None) -> EMfield:
    """E and B on nodes; ``arrays`` (6 float32 arrays) are adopted if given."""
    f = EMfield()
    for k, name in enumerate(FIELD_NAMES):
        a = (np.zeros(nodes(grd), np.float32) if arrays is None
             else np.ascontiguousarray(arrays[k], dtype=np.float32))
        if a.size != nodes(grd):
            raise ValueError(f"{name} has {a.size} values, grid has {nodes(grd)} nodes")
        setattr(f, name + "_flat", _keep(f, name, a))
    return f


def field_arrays(f: EMfield) -> list:
    return [f._arrays[n] for n in FIELD_NAMES]


def particle_allocate(param: Parameters, is_: int, arrays: dict | None = None,
                      npmax: int | None = None) -> Particles:
    """src/Particles.cpp:5-54. ``arrays`` (x, y, z, u, v, w, q float32) are
    adopted if given; otherwise zeroed arrays of npmax = param.npMax[is]."""
    p = Particles()
    p.species_ID = is_
    n = len(arrays["x"]) if arrays is not None else int(param.np[is_])
    p.nop = n
    p.npmax = max(n, npmax or int(param.npMax[is_]))
    p.NiterMover, p.n_sub_cycles = param.NiterMover, param.n_sub_cycles
    p.qom = param.qom[is_]
    p.uth, p.vth, p.wth = param.uth[is_], param.vth[is_], param.wth[is_]
    p.u0, p.v0, p.w0 = param.u0[is_], param.v0[is_], param.w0[is_]
    for k in "xyzuvwq":
        if arrays is not None:
            a = np.ascontiguousarray(arrays[k], dtype=np.float32)
        else:
            a = np.zeros(p.npmax, np.float32)
        setattr(p, k, _keep(p, k, a))
    return p


def particle_arrays(p: Particles) -> dict:
    return {k: p._arrays[k] for k in "xyzuvwq"}


def interp_dens_species_allocate(grd: Grid, is_: int) -> InterpDensSpecies:
    """src/InterpDensSpecies.cpp:4-42: 10 node moments plus rhoc on centres."""
    ids = InterpDensSpecies()
    ids.species_ID = is_
    for name in MOMENT_NAMES:
        setattr(ids, name + "_flat", _keep(ids, name, np.zeros(nodes(grd), np.float32)))
    ids.rhoc_flat = _keep(ids, "rhoc", np.zeros(grd.nxc * grd.nyc * grd.nzc, np.float32))
    return ids


def moments(ids: InterpDensSpecies) -> list:
    return [ids._arrays[n] for n in MOMENT_NAMES]


def interp_dens_net_allocate(grd: Grid) -> "_lib.InterpDensNet":
    """src/InterpDensNet.cpp (interp_dens_net_allocate): 10 node moments plus
    rhoc on centres, the sums over species."""
    idn = _lib.InterpDensNet()
    for name in MOMENT_NAMES:
        setattr(idn, name + "_flat", _keep(idn, name, np.zeros(nodes(grd), np.float32)))
    idn.rhoc_flat = _keep(idn, "rhoc", np.zeros(grd.nxc * grd.nyc * grd.nzc, np.float32))
    return idn


def _arr3(obj, name: str, n0: int, n1: int, n2: int) -> int:
    """newArr3 (include/Alloc.h:52-60): one zeroed float block with a
    row-pointer and a plane-pointer level over it; returns the top pointer."""
    data = np.zeros(n0 * n1 * n2, np.float32)
    rows = (data.ctypes.data + 4 * n2 * np.arange(n0 * n1, dtype=np.uint64)).astype(np.uint64)
    planes = (rows.ctypes.data + 8 * n1 * np.arange(n0, dtype=np.uint64)).astype(np.uint64)
    _keep(obj, name, data)
    _keep(obj, name + "_rows", rows)
    return _keep(obj, name + "_planes", planes)


def interp_dens_aux_allocate(grd: Grid) -> "_lib.InterpDensAux":
    """interp_dens_aux_allocate (include/InterpDens_aux.h:16-24): rho hat on
    the cell centres, J hat on the nodes, each a 3-level array."""
    aux = _lib.InterpDensAux()
    aux.rhoh = _arr3(aux, "rhoh", grd.nxc, grd.nyc, grd.nzc)
    for n in ("Jxh", "Jyh", "Jzh"):
        setattr(aux, n, _arr3(aux, n, grd.nxn, grd.nyn, grd.nzn))
    return aux


def hat_arrays(aux) -> tuple:
    """The flat (Jxh, Jyh, Jzh, rhoh) arrays of an interp_dens_aux_allocate."""
    return tuple(aux._arrays[n] for n in ("Jxh", "Jyh", "Jzh", "rhoh"))


def setZeroSpeciesDensities(ids: InterpDensSpecies) -> None:
    """src/InterpDensNet.cpp:40-75 for one species."""
    for a in ids._arrays.values():
        a[...] = 0


# --- the drop-in entry points -------------------------------------------------
def _ret(status: int, raise_on_error: bool) -> int:
    if raise_on_error:
        _lib.check(status)
    return status


def mover_PC(part: Particles, field: EMfield, grd: Grid, param: Parameters,
             raise_on_error: bool = False) -> int:
    lib = _lib.load()
    return _ret(lib.spb_mover_PC(ctypes.byref(part), ctypes.byref(field), ctypes.byref(grd),
                                 ctypes.byref(param)), raise_on_error)


def mover_PC_V(part: Particles, field: EMfield, grd: Grid, param: Parameters,
               raise_on_error: bool = False) -> int:
    lib = _lib.load()
    return _ret(lib.spb_mover_PC_V(ctypes.byref(part), ctypes.byref(field), ctypes.byref(grd),
                                   ctypes.byref(param)), raise_on_error)


def interpP2G(part: Particles, ids: InterpDensSpecies, grd: Grid,
              raise_on_error: bool = False) -> None:
    lib = _lib.load()
    lib.spb_clear_error()
    lib.spb_interpP2G(ctypes.byref(part), ctypes.byref(ids), ctypes.byref(grd))
    if raise_on_error:
        _lib.check(lib.spb_last_error())


def interp_all_species(parts: list, ids: list, idn, grd: Grid, param: Parameters,
                       raise_on_error: bool = False) -> int:
    """The driver's moment section (src/sputniPIC_CPU.cpp:247-259) in one call:
    zero, interpP2G every species, applyBCids per species, sumOverSpecies,
    all on the device. param.ns must equal len(parts)."""
    lib = _lib.load()
    ns = len(parts)
    assert param.ns == ns == len(ids)
    parr = (Particles * ns)(*parts)      # copies share the caller's arrays
    iarr = (InterpDensSpecies * ns)(*ids)
    return _ret(lib.spb_interp_all_species(parr, iarr, ctypes.byref(idn), ctypes.byref(grd),
                                           ctypes.byref(param)), raise_on_error)


def calculateHatDensities(aux, idn, ids: list, field: EMfield, grd: Grid, param: Parameters,
                          raise_on_error: bool = False) -> int:
    """calculateHatDensities (src/MaxwellSolver.cpp:465-603) on the device:
    J hat and rho hat into ``aux`` from the species moments ``ids``
    (param.ns of them), the magnetic field and ``idn``'s rhoc."""
    lib = _lib.load()
    ns = len(ids)
    assert param.ns == ns
    iarr = (InterpDensSpecies * ns)(*ids)
    return _ret(lib.spb_calculateHatDensities(ctypes.byref(aux), ctypes.byref(idn), iarr,
                                              ctypes.byref(field), ctypes.byref(grd),
                                              ctypes.byref(param)), raise_on_error)


def particle_sort(param: Parameters, part: Particles, grd: Grid,
                  raise_on_error: bool = False) -> int:
    """particle_sort (src/Particles.cpp:72-234) on the device, over npmax
    entries, with param.sort_cps cells per bin and axis."""
    lib = _lib.load()
    return _ret(lib.spb_particle_sort(ctypes.byref(param), ctypes.byref(part), ctypes.byref(grd)),
                raise_on_error)


def mover_interp(part: Particles, field: EMfield, ids: InterpDensSpecies, grd: Grid,
                 param: Parameters, raise_on_error: bool = False) -> int:
    lib = _lib.load()
    return _ret(lib.spb_mover_interp(ctypes.byref(part), ctypes.byref(field), ctypes.byref(ids),
                                     ctypes.byref(grd), ctypes.byref(param)), raise_on_error)


def last_error():
    return _lib.last_error()


def set_residency(device_resident: bool) -> int:
    return _lib.load().spb_set_residency(1 if device_resident else 0)


def sync_particles_to_host(part: Particles) -> int:
    return _lib.load().spb_sync_particles_to_host(ctypes.byref(part))


def invalidate_particles(part: Particles) -> int:
    return _lib.load().spb_invalidate_particles(ctypes.byref(part))


def release_all() -> int:
    return _lib.load().spb_release_all()
