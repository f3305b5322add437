"""Device-resident plain form: the spb_grid_* C-ABI over torch CUDA tensors.

torch supplies the HBM buffers and the stream; every computation is a kernel
of libsputnipic_b200.so. Particle dicts hold float32 CUDA tensors ``x, y, z,
u, v, w, q``; moments are a float32 CUDA tensor of shape (10, nodes) in the
reference order rhon, Jx, Jy, Jz, pxx, pxy, pxz, pyy, pyz, pzz.
"""
from __future__ import annotations

import ctypes

from . import _lib


def _stream(stream):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


def _ptr(t) -> int:
    import torch
    if not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
        raise TypeError("expected a contiguous float32 CUDA tensor")
    return t.data_ptr()


DEPOSIT_MODES = {"accumulator": 0, "direct": 1}


def set_plain_deposit_mode(mode: str) -> str:
    """How the plain interpP2G / mover_interp deposits, process-wide
    (spb_set_plain_deposit_mode): "accumulator" (a node-interleaved buffer
    from the device pool, then added into the ten moment arrays; the default)
    or "direct" (straight into the ten arrays, no extra memory). Returns the
    previous mode."""
    if mode not in DEPOSIT_MODES:
        raise ValueError(f"unknown deposit mode {mode!r}")
    prev = _lib.load().spb_set_plain_deposit_mode(DEPOSIT_MODES[mode])
    _lib.check(min(prev, 0))
    return {v: k for k, v in DEPOSIT_MODES.items()}[prev]


def push_params(wl, s: int) -> _lib.SpbPush:
    """spb_push of species ``s`` of a workload."""
    p = _lib.SpbPush()
    p.dt, p.c = wl.dt, wl.c
    p.qom = wl.species[s].qom
    p.niter, p.n_sub_cycles = wl.niter, wl.n_sub_cycles
    for a in range(3):
        p.periodic[a] = 1 if wl.periodic[a] else 0
    return p


class GridContext:
    """One spb_grid_ctx: grid geometry, node coordinates, packed fields."""

    def __init__(self, wl=None, grid=None):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        if grid is not None:
            rc = self.lib.spb_grid_create(ctypes.byref(grid), ctypes.byref(h))
        else:
            rc = self.lib.spb_grid_create_uniform(wl.nxc, wl.nyc, wl.nzc, wl.Lx, wl.Ly, wl.Lz,
                                                  ctypes.byref(h))
        _lib.check(rc)
        self.h = h
        self.nodes = self.lib.spb_grid_nodes(h)

    def close(self):
        if self.h:
            self.lib.spb_grid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return self.lib.spb_grid_launches(self.h)

    def set_fields(self, fields, stream=None):
        """fields: six float32 CUDA tensors (Ex, Ey, Ez, Bxn, Byn, Bzn)."""
        arr = (ctypes.c_void_p * 6)(*[_ptr(f) for f in fields])
        _lib.check(self.lib.spb_grid_set_fields(self.h, arr, 1, _stream(stream)))

    def mover(self, part, push, stream=None):
        n = part["x"].numel()
        _lib.check(self.lib.spb_grid_mover(self.h, ctypes.byref(push),
                                           *[_ptr(part[k]) for k in "xyzuvw"], n,
                                           _stream(stream)))

    def p2g(self, part, mom, stream=None):
        n = part["x"].numel()
        m = (ctypes.c_void_p * 10)(*[_ptr(mom[i]) for i in range(10)])
        _lib.check(self.lib.spb_grid_p2g(self.h, *[_ptr(part[k]) for k in "xyzuvwq"], n, m,
                                         _stream(stream)))

    def mover_interp(self, part, push, mom, stream=None):
        n = part["x"].numel()
        m = (ctypes.c_void_p * 10)(*[_ptr(mom[i]) for i in range(10)])
        _lib.check(self.lib.spb_grid_mover_interp(self.h, ctypes.byref(push),
                                                  *[_ptr(part[k]) for k in "xyzuvwq"], n, m,
                                                  _stream(stream)))

    def apply_bc_ids(self, mom, periodic, stream=None):
        per = (ctypes.c_int * 3)(*[1 if p else 0 for p in periodic])
        m = (ctypes.c_void_p * 10)(*[_ptr(mom[i]) for i in range(10)])
        _lib.check(self.lib.spb_grid_apply_bc_ids(self.h, ctypes.byref(per), m, _stream(stream)))

    def check(self, stream=None) -> int:
        """Synchronise and return the status (SPB_ERR_OUT_OF_GRID if a
        particle left the node array since the last check)."""
        return self.lib.spb_grid_check(self.h, _stream(stream))


# --- device-side workload generation -----------------------------------------
def gem_desc(wl) -> _lib.GemDesc:
    d = _lib.GemDesc()
    d.nxc, d.nyc, d.nzc = wl.nxc, wl.nyc, wl.nzc
    d.Lx, d.Ly, d.Lz = wl.Lx, wl.Ly, wl.Lz
    d.B0, d.delta, d.pert, d.E_amp = wl.B0, wl.delta, wl.pert, wl.E_amp
    d.lattice, d.seed = wl.lattice, wl.seed
    return d


def gem_species(wl, s: int) -> _lib.GemSpecies:
    sp = wl.species[s]
    g = _lib.GemSpecies()
    g.qom, g.rho0, g.vth, g.w0, g.ppc, g.sheet = sp.qom, sp.rho0, sp.vth, sp.w0, sp.ppc, int(sp.sheet)
    return g


def gen_fields(wl, stream=None):
    """The workload's six node fields as float32 CUDA tensors."""
    import torch
    F = [torch.empty(wl.nodes, dtype=torch.float32, device="cuda") for _ in range(6)]
    arr = (ctypes.c_void_p * 6)(*[f.data_ptr() for f in F])
    _lib.check(_lib.load().spb_gen_gem_fields(ctypes.byref(gem_desc(wl)), arr, _stream(stream)))
    return F


def gen_particles(wl, s: int, first: int = 0, count: int | None = None, with_cell=False,
                  stream=None):
    """Particles [first, first+count) of species s as float32 CUDA tensors."""
    import torch
    total = wl.species_count(s)
    count = total - first if count is None else count
    part = {k: torch.empty(count, dtype=torch.float32, device="cuda") for k in "xyzuvwq"}
    cell = torch.empty(count, dtype=torch.int32, device="cuda") if with_cell else None
    _lib.check(_lib.load().spb_gen_gem_particles(
        ctypes.byref(gem_desc(wl)), ctypes.byref(gem_species(wl, s)), s, first, count,
        *[part[k].data_ptr() for k in "xyzuvwq"], cell.data_ptr() if cell is not None else None,
        _stream(stream)))
    if with_cell:
        part["cell"] = cell
    return part
