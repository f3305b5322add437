"""CPU oracles for the mover + P2G path (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` and
``--impl reference`` legs of ``bench.py`` may import this package, and only
as the checker or the timed CPU baseline. The shipped library
(``sputnipic_b200``) never imports it.

Two implementations share one flat C interface (``oracle_api.h``):

* ``restated``: ``oracle.c``, a plain-C restatement of sputniPIC's
  ``src/Mover.cpp`` (mover_PC :4-162, interpP2G :385-572, mover_interp
  :575-862), ``src/Grid.cpp:5-62`` (setGrid) and ``src/BC.cpp:362-615``
  (applyBCids). Built from committed sources anywhere.
* ``reference``: the reference's own sources compiled into ``oracle/_ref``
  with ``ref_shim.cpp`` (only where the reference tree exists; the built
  libraries travel with the repository snapshot but are never committed).

``fp`` selects the precision: 32 is the reference's PrecisionTypes.h (all
float), 64 makes FPpart/FPfield/FPinterp double (the FP64 oracle).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

MOMENTS = ("rhon", "Jx", "Jy", "Jz", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz")
FIELDS = ("Ex", "Ey", "Ez", "Bxn", "Byn", "Bzn")


class OrcSetup(ctypes.Structure):
    """Mirror of ``orc_setup`` in oracle_api.h."""

    _fields_ = [
        ("nxc", ctypes.c_int), ("nyc", ctypes.c_int), ("nzc", ctypes.c_int),
        ("Lx", ctypes.c_double), ("Ly", ctypes.c_double), ("Lz", ctypes.c_double),
        ("periodic", ctypes.c_int * 3),
        ("dt", ctypes.c_double), ("c", ctypes.c_double),
        ("niter", ctypes.c_int), ("n_sub_cycles", ctypes.c_int),
    ]


def setup_from(wl) -> OrcSetup:
    """Build an ``orc_setup`` from a workload description (any object with the
    attributes of ``sputnipic_b200.workload.GemWorkload``)."""
    s = OrcSetup()
    s.nxc, s.nyc, s.nzc = wl.nxc, wl.nyc, wl.nzc
    s.Lx, s.Ly, s.Lz = wl.Lx, wl.Ly, wl.Lz
    for d in range(3):
        s.periodic[d] = 1 if wl.periodic[d] else 0
    s.dt, s.c = wl.dt, wl.c
    s.niter, s.n_sub_cycles = wl.niter, wl.n_sub_cycles
    return s


def library_path(kind: str, fp: int) -> str:
    if kind == "restated":
        return os.path.join(_HERE, f"liboracle_fp{fp}.so")
    if kind == "reference":
        return os.path.join(_HERE, "_ref", f"libref_fp{fp}.so")
    raise ValueError(kind)


def build_restated() -> None:
    """Compile the restatement (gcc only; safe on any machine)."""
    subprocess.run(["make", "-s", "-C", _HERE, "restated"], check=True)


def reference_available(fp: int = 32) -> bool:
    return os.path.exists(library_path("reference", fp))


_P = ctypes.c_void_p


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


class CpuOracle:
    """ctypes front end of one oracle library."""

    def __init__(self, kind: str = "restated", fp: int = 32):
        path = library_path(kind, fp)
        if not os.path.exists(path):
            if kind == "restated":
                build_restated()
            else:
                raise FileNotFoundError(
                    f"{path} missing: the reference oracle is built by oracle/Makefile "
                    "only where the reference source tree exists")
        self.kind, self.fp = kind, fp
        self.dtype = np.float32 if fp == 32 else np.float64
        lib = ctypes.CDLL(path)
        lib.orc_mover_pc.restype = ctypes.c_int
        lib.orc_mover_pc.argtypes = [ctypes.POINTER(OrcSetup), _P] + [_P] * 6 + [ctypes.c_long, ctypes.c_double]
        lib.orc_mover_pc_v.restype = ctypes.c_int
        lib.orc_mover_pc_v.argtypes = lib.orc_mover_pc.argtypes
        lib.orc_interp_p2g.restype = None
        lib.orc_interp_p2g.argtypes = [ctypes.POINTER(OrcSetup)] + [_P] * 7 + [ctypes.c_long, _P]
        lib.orc_apply_bc_ids.restype = None
        lib.orc_apply_bc_ids.argtypes = [ctypes.POINTER(OrcSetup), _P]
        lib.orc_particle_sort.restype = ctypes.c_int
        lib.orc_particle_sort.argtypes = ([ctypes.POINTER(OrcSetup), ctypes.c_int] + [_P] * 7
                                          + [ctypes.c_long])
        lib.orc_mover_interp.restype = ctypes.c_int
        lib.orc_mover_interp.argtypes = ([ctypes.POINTER(OrcSetup), _P] + [_P] * 7
                                         + [ctypes.c_long, ctypes.c_double, _P])
        lib.orc_cycle.restype = ctypes.c_int
        lib.orc_cycle.argtypes = ([ctypes.POINTER(OrcSetup), _P, ctypes.c_int] + [_P] * 7
                                  + [_P, _P, _P, ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(ctypes.c_double)])
        lib.orc_hat_densities.restype = ctypes.c_int
        lib.orc_hat_densities.argtypes = ([ctypes.POINTER(OrcSetup), ctypes.c_double, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_double)] + [_P] * 7)
        lib.orc_num_threads.restype = ctypes.c_int
        lib.orc_fp_bytes.restype = ctypes.c_int
        assert lib.orc_fp_bytes() * 8 == fp
        self.lib = lib

    # -- helpers ---------------------------------------------------------
    def _chk(self, a: np.ndarray) -> np.ndarray:
        if a.dtype != self.dtype or not a.flags.c_contiguous:
            raise TypeError(f"oracle fp{self.fp} needs C-contiguous {np.dtype(self.dtype).name} arrays")
        return a

    def _arr(self, arrays):
        arrs = [self._chk(a) for a in arrays]
        return (ctypes.c_void_p * len(arrs))(*[_ptr(a) for a in arrs]), arrs

    @property
    def threads(self) -> int:
        return self.lib.orc_num_threads()

    # -- the reference entry points -----------------------------------------
    def mover_pc(self, setup: OrcSetup, fields, part: dict, qom: float) -> int:
        f, keep = self._arr(fields)
        p = [self._chk(part[k]) for k in "xyzuvw"]
        return self.lib.orc_mover_pc(ctypes.byref(setup), f, *[_ptr(a) for a in p],
                                     len(p[0]), float(qom))

    def mover_pc_v(self, setup: OrcSetup, fields, part: dict, qom: float) -> int:
        f, keep = self._arr(fields)
        p = [self._chk(part[k]) for k in "xyzuvw"]
        return self.lib.orc_mover_pc_v(ctypes.byref(setup), f, *[_ptr(a) for a in p],
                                       len(p[0]), float(qom))

    def interp_p2g(self, setup: OrcSetup, part: dict, mom) -> None:
        m, keep = self._arr(mom)
        p = [self._chk(part[k]) for k in "xyzuvwq"]
        self.lib.orc_interp_p2g(ctypes.byref(setup), *[_ptr(a) for a in p], len(p[0]), m)

    def apply_bc_ids(self, setup: OrcSetup, mom) -> None:
        m, keep = self._arr(mom)
        self.lib.orc_apply_bc_ids(ctypes.byref(setup), m)

    def particle_sort(self, setup: OrcSetup, sort_cps: int, part: dict) -> int:
        """particle_sort (src/Particles.cpp:72-234) in place on x..q."""
        p = [self._chk(part[k]) for k in "xyzuvwq"]
        return self.lib.orc_particle_sort(ctypes.byref(setup), int(sort_cps),
                                          *[_ptr(a) for a in p], len(p[0]))

    def mover_interp(self, setup: OrcSetup, fields, part: dict, qom: float, mom) -> int:
        f, keepf = self._arr(fields)
        m, keepm = self._arr(mom)
        p = [self._chk(part[k]) for k in "xyzuvwq"]
        return self.lib.orc_mover_interp(ctypes.byref(setup), f, *[_ptr(a) for a in p],
                                         len(p[0]), float(qom), m)

    def hat_densities(self, setup: OrcSetup, th: float, qom, mom, fields, rhoc):
        """calculateHatDensities (src/MaxwellSolver.cpp:465-603). mom: list of
        ns lists of 10 node arrays; fields: the six node arrays; rhoc: the
        cell-centre net charge density (flat, guard cells included). Returns
        (Jxh, Jyh, Jzh, rhoh) as new arrays."""
        ns = len(mom)
        m, keepm = self._arr([a for sp in mom for a in sp])
        f, keepf = self._arr(fields)
        rc = self._chk(rhoc)
        nodes = len(fields[0])
        out = [np.empty(nodes, dtype=self.dtype) for _ in range(3)]
        out.append(np.empty(len(rc), dtype=self.dtype))
        q = (ctypes.c_double * ns)(*[float(x) for x in qom])
        r = self.lib.orc_hat_densities(ctypes.byref(setup), float(th), ns, q, m, f, _ptr(rc),
                                       *[_ptr(a) for a in out])
        if r != 0:
            raise RuntimeError(f"orc_hat_densities failed: {r}")
        return tuple(out)

    def cycle(self, setup: OrcSetup, fields, species: list, mom):
        """One driver cycle over ``species`` (list of particle dicts with a
        ``qom`` entry); ``mom`` is a list of ns*10 arrays. Returns
        (t_mover, t_interp) in seconds, timed inside the library."""
        ns = len(species)
        f, keepf = self._arr(fields)
        cols = []
        for k in "xyzuvwq":
            cols.append(self._arr([sp[k] for sp in species]))
        nop = (ctypes.c_long * ns)(*[len(sp["x"]) for sp in species])
        qom = (ctypes.c_double * ns)(*[float(sp["qom"]) for sp in species])
        m, keepm = self._arr(mom)
        tm, ti = ctypes.c_double(), ctypes.c_double()
        rc = self.lib.orc_cycle(ctypes.byref(setup), f, ns, *[c[0] for c in cols], nop, qom, m,
                                ctypes.byref(tm), ctypes.byref(ti))
        if rc != 0:
            raise RuntimeError(f"orc_cycle failed: {rc}")
        return tm.value, ti.value
