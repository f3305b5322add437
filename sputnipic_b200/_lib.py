"""ctypes binding of libsputnipic_b200.so and mirrors of the reference structs.

The structs below are the reference's boundary structs, field for field
(include/Particles.h:11-56, include/EMfield.h:8-25, include/Grid.h:11-63,
include/InterpDensSpecies.h:9-40, include/Parameters.h:10-235), so that a
``ctypes.byref`` of them is what the reference's C++ driver passes to
mover_PC / interpP2G. ``check_layout`` compares every offset with the
library's own (``spb_abi_layout_json``).

The library is the product: importing this module fails loudly if the
shared object is missing (build it with ``__graft_entry__.build()`` or
``make -C sputnipic_b200/csrc``). There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import json
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsputnipic_b200.so")

c_int, c_long, c_float, c_double, c_bool = (ctypes.c_int, ctypes.c_long, ctypes.c_float,
                                            ctypes.c_double, ctypes.c_bool)
P = ctypes.c_void_p
NS_MAX = 6


class StdString(ctypes.Structure):
    """Storage of a 64-bit libstdc++ std::string; never read by the library."""
    _fields_ = [("p_", P), ("n_", ctypes.c_size_t), ("buf_", ctypes.c_char * 16)]


class Particles(ctypes.Structure):
    _fields_ = [
        ("species_ID", c_int), ("npmax", c_long), ("nop", c_long),
        ("NiterMover", c_int), ("n_sub_cycles", c_int),
        ("npcel", c_int), ("npcelx", c_int), ("npcely", c_int), ("npcelz", c_int),
        ("qom", c_float), ("u0", c_float), ("v0", c_float), ("w0", c_float),
        ("uth", c_float), ("vth", c_float), ("wth", c_float),
        ("x", P), ("y", P), ("z", P), ("u", P), ("v", P), ("w", P), ("q", P),
        ("track_particle", P),
    ]


class EMfield(ctypes.Structure):
    _fields_ = [(n, P) for f in ("Ex", "Ey", "Ez", "Bxn", "Byn", "Bzn") for n in (f, f + "_flat")]


class Grid(ctypes.Structure):
    _fields_ = [
        ("nxc", c_int), ("nxn", c_int), ("nyc", c_int), ("nyn", c_int),
        ("nzc", c_int), ("nzn", c_int),
        ("dx", c_double), ("dy", c_double), ("dz", c_double),
        ("invdx", c_float), ("invdy", c_float), ("invdz", c_float), ("invVOL", c_float),
        ("xStart", c_double), ("xEnd", c_double), ("yStart", c_double), ("yEnd", c_double),
        ("zStart", c_double), ("zEnd", c_double),
        ("Lx", c_double), ("Ly", c_double), ("Lz", c_double),
        ("PERIODICX", c_bool), ("PERIODICY", c_bool), ("PERIODICZ", c_bool),
        ("XN_flat", P), ("XN", P), ("YN_flat", P), ("YN", P), ("ZN_flat", P), ("ZN", P),
    ]


MOMENT_NAMES = ("rhon", "Jx", "Jy", "Jz", "pxx", "pxy", "pxz", "pyy", "pyz", "pzz")


class InterpDensSpecies(ctypes.Structure):
    _fields_ = ([("species_ID", c_int)]
                + [(n, P) for f in ("rhon", "rhoc") + MOMENT_NAMES[1:] for n in (f, f + "_flat")])


class InterpDensNet(ctypes.Structure):
    _fields_ = [(n, P) for f in ("rhon", "rhoc") + MOMENT_NAMES[1:] for n in (f, f + "_flat")]


class InterpDensAux(ctypes.Structure):
    """Implicit-source densities of the field solver (include/InterpDens_aux.h:6-13)."""
    _fields_ = [(n, P) for n in ("rhoh", "Jxh", "Jyh", "Jzh")]


def _ints(*names):
    return [(n, c_int) for n in names]


class Parameters(ctypes.Structure):
    _fields_ = (
        [("c", c_double), ("fourpi", c_double), ("dt", c_double), ("th", c_double)]
        + _ints("ncycles", "NiterMover", "n_sub_cycles")
        + [("sort", c_bool), ("sort_every_n", c_long), ("sort_cps", c_long),
           ("number_of_batches", c_int), ("threads_per_block", c_long),
           ("track_particles", c_bool), ("n_tracked_particles", c_long),
           ("tracking_start_cycle", c_long), ("tracking_end_cycle", c_long),
           ("tracking_Lx", c_long), ("tracking_Ly", c_long), ("tracking_Lz", c_long),
           ("tracked_particles_filename", StdString),
           ("Lx", c_double), ("Ly", c_double), ("Lz", c_double)]
        + _ints("nxc", "nyc", "nzc")
        + [("x_center", c_double), ("y_center", c_double), ("z_center", c_double),
           ("L_square", c_double), ("ns", c_int),
           ("npcelx", c_int * NS_MAX), ("npcely", c_int * NS_MAX), ("npcelz", c_int * NS_MAX),
           ("np", c_long * NS_MAX), ("npMax", c_long * NS_MAX), ("NpMaxNpRatio", c_double)]
        + [(n, c_double * NS_MAX) for n in ("qom", "rhoINIT", "uth", "vth", "wth", "u0", "v0", "w0")]
        + [(n, c_bool) for n in ("PERIODICX", "PERIODICY", "PERIODICZ",
                                 "PERIODICX_P", "PERIODICY_P", "PERIODICZ_P")]
        + _ints(*[f"bc{k}face{a}{s}" for k in ("P", "PHI", "EM") for a in "XYZ"
                  for s in ("right", "left")])
        + [("Vinj", c_double), ("delta", c_double), ("B0x", c_double), ("B0y", c_double),
           ("B0z", c_double), ("Nwaves", c_int), ("dBoB0", c_double), ("pitch_angle", c_double),
           ("energy", c_double), ("SmoothON", c_bool), ("SmoothValue", c_double),
           ("SmoothTimes", c_int), ("verbose", c_bool), ("RESTART", c_bool),
           ("PoissonCorrection", c_bool), ("CGtol", c_double), ("GMREStol", c_double)]
        + _ints("first_cycle_n", "FieldOutputCycle", "ParticlesOutputCycle",
                "RestartOutputCycle", "DiagnosticsOutputCycle")
        + [(n, StdString) for n in ("inputfile", "SaveDirName", "RestartDirName", "WaveFile")]
    )


STRUCTS = {"particles": Particles, "EMfield": EMfield, "grid": Grid,
           "interpDensSpecies": InterpDensSpecies, "interpDensNet": InterpDensNet,
           "interpDens_aux": InterpDensAux, "parameters": Parameters}


class SpbPush(ctypes.Structure):
    """spb_push of include/sputnipic_b200.h."""
    _fields_ = [("dt", c_double), ("c", c_double), ("qom", c_float), ("niter", c_int),
                ("n_sub_cycles", c_int), ("periodic", c_int * 3)]


class GemDesc(ctypes.Structure):
    """spb_gem_desc of include/sputnipic_b200.h."""
    _fields_ = [("nxc", c_int), ("nyc", c_int), ("nzc", c_int),
                ("Lx", c_double), ("Ly", c_double), ("Lz", c_double),
                ("B0", c_double), ("delta", c_double), ("pert", c_double), ("E_amp", c_double),
                ("lattice", c_int), ("seed", ctypes.c_ulonglong)]


class GemSpecies(ctypes.Structure):
    """spb_gem_species of include/sputnipic_b200.h."""
    _fields_ = [("qom", c_double), ("rho0", c_double), ("vth", c_double), ("w0", c_double),
                ("ppc", c_double), ("sheet", c_int)]


class SimDesc(ctypes.Structure):
    """spb_sim_desc of include/sputnipic_b200.h."""
    _fields_ = [("nxc", c_int), ("nyc", c_int), ("nzc", c_int),
                ("Lx", c_double), ("Ly", c_double), ("Lz", c_double),
                ("dt", c_double), ("c", c_double), ("niter", c_int), ("periodic", c_int * 3),
                ("ns", c_int), ("qom", c_double * 8), ("capacity", c_long * 8),
                ("tile", c_int * 3), ("resort_every", c_int), ("ctas", c_int),
                ("variant", c_int), ("bucket_slots", c_int), ("graph", c_int),
                ("deterministic", c_int), ("fused", c_int), ("overflow_per_mille", c_int)]


HAT_MAX_SPECIES = 16


class HatDesc(ctypes.Structure):
    """spb_hat_desc (include/sputnipic_b200.h)."""
    _fields_ = [("nxc", c_int), ("nyc", c_int), ("nzc", c_int),
                ("invdx", c_double), ("invdy", c_double), ("invdz", c_double),
                ("periodic", c_int * 3), ("dt", c_double), ("c", c_double), ("th", c_double),
                ("ns", c_int), ("qom", c_double * HAT_MAX_SPECIES)]


class ServeDesc(ctypes.Structure):
    """spb_serve_desc of include/sputnipic_b200.h."""
    _fields_ = [("tile", c_int * 3), ("hbm_budget", ctypes.c_longlong), ("max_jobs", c_int),
                ("check_every", c_int), ("reserve_bytes", ctypes.c_longlong),
                ("extra_budget", c_double)]


class JobDesc(ctypes.Structure):
    """spb_job_desc of include/sputnipic_b200.h."""
    _fields_ = [("nxc", c_int), ("nyc", c_int), ("nzc", c_int),
                ("Lx", c_double), ("Ly", c_double), ("Lz", c_double),
                ("dt", c_double), ("c", c_double), ("niter", c_int), ("periodic", c_int * 3),
                ("ns", c_int), ("qom", c_double * 8), ("ncycles", c_int)]


def ctypes_layout() -> dict:
    """Offsets of the ctypes mirrors, keyed like spb_abi_layout_json."""
    out = {}
    for name, cls in STRUCTS.items():
        for fname, _ in cls._fields_:
            out[f"{name}.{fname}"] = getattr(cls, fname).offset
        out[f"sizeof {name}"] = ctypes.sizeof(cls)
    return out


_lib = None


def _proto(lib, name, res, args):
    f = getattr(lib, name)
    f.restype = res
    f.argtypes = args
    return f


def load():
    """Load the shared library (once) and declare every prototype."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python -c 'import __graft_entry__ as g; g.build()')")
    lib = ctypes.CDLL(LIB_PATH)
    R = ctypes.POINTER
    _proto(lib, "spb_last_error", c_int, [])
    _proto(lib, "spb_last_error_message", ctypes.c_char_p, [])
    _proto(lib, "spb_clear_error", None, [])
    _proto(lib, "spb_error_string", ctypes.c_char_p, [c_int])
    _proto(lib, "spb_version", ctypes.c_char_p, [])
    _proto(lib, "spb_launch_count", c_long, [])
    _proto(lib, "spb_set_plain_deposit_mode", c_int, [c_int])
    _proto(lib, "spb_abi_layout_json", ctypes.c_char_p, [])
    _proto(lib, "spb_set_device", c_int, [c_int])
    _proto(lib, "spb_mover_PC", c_int, [R(Particles), R(EMfield), R(Grid), R(Parameters)])
    _proto(lib, "spb_mover_PC_V", c_int, [R(Particles), R(EMfield), R(Grid), R(Parameters)])
    _proto(lib, "spb_interpP2G", None, [R(Particles), R(InterpDensSpecies), R(Grid)])
    _proto(lib, "spb_mover_interp", c_int,
           [R(Particles), R(EMfield), R(InterpDensSpecies), R(Grid), R(Parameters)])
    _proto(lib, "spb_set_residency", c_int, [c_int])
    _proto(lib, "spb_sync_particles_to_host", c_int, [R(Particles)])
    _proto(lib, "spb_invalidate_particles", c_int, [R(Particles)])
    _proto(lib, "spb_release_all", c_int, [])
    _proto(lib, "spb_grid_create", c_int, [R(Grid), R(P)])
    _proto(lib, "spb_grid_create_uniform", c_int,
           [c_int, c_int, c_int, c_double, c_double, c_double, R(P)])
    _proto(lib, "spb_grid_destroy", None, [P])
    _proto(lib, "spb_grid_nodes", c_long, [P])
    _proto(lib, "spb_grid_launches", c_long, [P])
    _proto(lib, "spb_grid_set_fields", c_int, [P, P, c_int, P])
    _proto(lib, "spb_grid_mover", c_int, [P, R(SpbPush)] + [P] * 6 + [c_long, P])
    _proto(lib, "spb_grid_p2g", c_int, [P] + [P] * 7 + [c_long, P, P])
    _proto(lib, "spb_grid_mover_interp", c_int, [P, R(SpbPush)] + [P] * 7 + [c_long, P, P])
    _proto(lib, "spb_grid_apply_bc_ids", c_int, [P, R(c_int * 3), P, P])
    _proto(lib, "spb_grid_check", c_int, [P, P])
    _proto(lib, "spb_gem_species_count", c_long, [R(GemDesc), R(GemSpecies)])
    _proto(lib, "spb_gen_gem_fields", c_int, [R(GemDesc), P, P])
    _proto(lib, "spb_gen_gem_particles", c_int,
           [R(GemDesc), R(GemSpecies), c_int, c_long, c_long] + [P] * 8 + [P])
    _proto(lib, "spb_sim_tile_supported", c_int, [c_int, c_int, c_int])
    _proto(lib, "spb_sim_create", c_int, [R(SimDesc), R(P)])
    _proto(lib, "spb_sim_destroy", None, [P])
    _proto(lib, "spb_sim_nodes", c_long, [P])
    _proto(lib, "spb_sim_count", c_long, [P, c_int])
    _proto(lib, "spb_sim_launches", c_long, [P])
    _proto(lib, "spb_sim_set_fields", c_int, [P, P, c_int, P])
    _proto(lib, "spb_sim_load_species", c_int, [P, c_int] + [P] * 7 + [c_long, c_int, P])
    _proto(lib, "spb_sim_cycle", c_int, [P, c_int, P])
    _proto(lib, "spb_sim_resort", c_int, [P, P])
    _proto(lib, "spb_sim_moments", c_int, [P, c_int, P, c_int, P])
    _proto(lib, "spb_sim_apply_bc_ids", c_int, [P, c_int, P])
    _proto(lib, "spb_sim_moments_device", P, [P, c_int])
    _proto(lib, "spb_sim_particles", c_int, [P, c_int] + [P] * 7 + [c_int, P])
    _proto(lib, "spb_sim_check", c_int, [P, P])
    _proto(lib, "spb_sort_particles_noalloc", c_int,
           [R(SimDesc)] + [P] * 7 + [c_long] + [P] * 8 + [P, P])
    _proto(lib, "spb_sim_set_timing", c_int, [P, c_int])
    _proto(lib, "spb_sim_timing", c_int, [P, R(c_double), R(c_int), R(c_double), R(c_int)])
    _proto(lib, "spb_sim_kernel_timing", c_int,
           [P, R(c_double), R(c_double), R(c_int), R(c_double), R(c_int)])
    _proto(lib, "spb_sim_bucket_slots", c_long, [P, c_int])
    _proto(lib, "spb_sim_overflow", c_long, [P, c_int, P])
    _proto(lib, "spb_interp_all_species", c_int,
           [R(Particles), R(InterpDensSpecies), R(InterpDensNet), R(Grid), R(Parameters)])
    _proto(lib, "spb_particle_sort", c_int, [R(Parameters), R(Particles), R(Grid)])
    _proto(lib, "spb_calculateHatDensities", c_int,
           [R(InterpDensAux), R(InterpDensNet), R(InterpDensSpecies), R(EMfield), R(Grid),
            R(Parameters)])
    for fp in ("f32", "f64"):
        _proto(lib, "spb_hat_densities_" + fp, c_int, [R(HatDesc), P, P, P, P, P, P, P, P])
    _proto(lib, "spb_serve_create", c_int, [R(ServeDesc), R(P)])
    _proto(lib, "spb_release_cached_memory", c_int, [])
    _proto(lib, "spb_serve_destroy", None, [P])
    _proto(lib, "spb_serve_submit", c_long, [P, R(JobDesc), P, P, P, c_int])
    _proto(lib, "spb_serve_step", c_int, [P])
    _proto(lib, "spb_serve_finished", c_int, [P, ctypes.POINTER(c_long), c_int])
    _proto(lib, "spb_serve_status", c_int, [P, c_long])
    _proto(lib, "spb_serve_error", c_int, [P, c_long])
    _proto(lib, "spb_serve_result", c_int, [P, c_long, c_int] + [P] * 8 + [c_int])
    _proto(lib, "spb_serve_times", c_int, [P, c_long, P])
    _proto(lib, "spb_serve_release", c_int, [P, c_long])
    _proto(lib, "spb_serve_stats", c_int, [P, P])
    _proto(lib, "spb_serve_counts", c_int,
           [P, R(c_int), R(c_int), R(c_int), R(ctypes.c_longlong), R(ctypes.c_longlong)])
    _lib = lib
    return lib


def library_layout() -> dict:
    doc = json.loads(load().spb_abi_layout_json().decode())
    doc.pop("end", None)
    return doc


def check_layout() -> None:
    """Raise if the ctypes mirrors disagree with the library's struct layout."""
    lib_doc = library_layout()
    mine = ctypes_layout()
    bad = {k: (mine.get(k), v) for k, v in lib_doc.items() if mine.get(k) != v}
    if bad:
        raise RuntimeError(f"struct layout mismatch (ctypes, library): {bad}")


class SpbError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"spb status {status}: {msg}")
        self.status = status


def last_error():
    lib = load()
    return lib.spb_last_error(), lib.spb_last_error_message().decode()


def check(status: int) -> int:
    """Raise SpbError for a non-zero status of a library call."""
    if status != 0:
        raise SpbError(status, load().spb_last_error_message().decode())
    return status
