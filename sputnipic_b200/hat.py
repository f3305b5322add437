"""calculateHatDensities on device arrays (spb_hat_densities_f32 / _f64).

The field solver's first consumer of the moments (src/MaxwellSolver.cpp:
465-603): J hat on the nodes and rho hat on the cell centres, bit-identical
to the reference's FP32 build (float32 tensors) or FP64 build (float64). For
the drop-in over the reference's host structs see
``sputnipic_b200.dropin.calculateHatDensities``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def hat_desc(wl, th: float = 1.0, qom=None, fp: int = 32) -> _lib.HatDesc:
    """The descriptor for a workload's grid (``sputnipic_b200.workload``):
    guard cells added, inverse spacings as setGrid stores them (float for the
    FP32 build, src/Grid.cpp:19-27), the field periodicity, dt, c, theta and
    the species' charge-to-mass ratios (default: the workload's)."""
    d = _lib.HatDesc()
    d.nxc, d.nyc, d.nzc = wl.nxc + 2, wl.nyc + 2, wl.nzc + 2
    inv = [1.0 / wl.dx, 1.0 / wl.dy, 1.0 / wl.dz]
    if fp == 32:
        inv = [float(np.float32(v)) for v in inv]
    d.invdx, d.invdy, d.invdz = inv
    for a in range(3):
        d.periodic[a] = 1 if wl.periodic[a] else 0
    d.dt, d.c, d.th = wl.dt, wl.c, th
    qom = [sp.qom for sp in wl.species] if qom is None else list(qom)
    if not 1 <= len(qom) <= _lib.HAT_MAX_SPECIES:
        raise ValueError("1..16 species")
    d.ns = len(qom)
    for s, q in enumerate(qom):
        d.qom[s] = q
    return d


def hat_densities(desc: _lib.HatDesc, mom, B, rhoc, stream=None):
    """J hat (three node tensors) and rho hat (cell-centre tensor) from
    ``mom`` (desc.ns lists of the 10 node moment tensors, interpP2G order),
    ``B`` (Bxn, Byn, Bzn node tensors) and ``rhoc``; all CUDA tensors of one
    dtype (float32 or float64). Returns (Jxh, Jyh, Jzh, rhoh)."""
    import torch
    dtype = rhoc.dtype
    if dtype not in (torch.float32, torch.float64):
        raise TypeError("float32 or float64 tensors")
    tensors = [t for sp in mom for t in sp] + list(B) + [rhoc]
    if any(t.dtype != dtype or not t.is_cuda or not t.is_contiguous() for t in tensors):
        raise TypeError("contiguous CUDA tensors of one dtype")
    if len(mom) != desc.ns or any(len(sp) != 10 for sp in mom):
        raise ValueError("desc.ns lists of 10 moments")
    nodes = (desc.nxc + 1) * (desc.nyc + 1) * (desc.nzc + 1)
    cells = desc.nxc * desc.nyc * desc.nzc
    out = [torch.empty(nodes, dtype=dtype, device=rhoc.device) for _ in range(3)]
    out.append(torch.empty(cells, dtype=dtype, device=rhoc.device))
    mp = (ctypes.c_void_p * (10 * desc.ns))(*[t.data_ptr() for sp in mom for t in sp])
    bp = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in B])
    fn = _lib.load().spb_hat_densities_f32 if dtype == torch.float32 else \
        _lib.load().spb_hat_densities_f64
    st = torch.cuda.current_stream().cuda_stream if stream is None else stream.cuda_stream
    _lib.check(fn(ctypes.byref(desc), mp, bp, ctypes.c_void_p(rhoc.data_ptr()),
                  *[ctypes.c_void_p(t.data_ptr()) for t in out], ctypes.c_void_p(st)))
    return tuple(out)
