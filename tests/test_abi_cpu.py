"""The C-ABI library without a GPU: it loads, exports every symbol that
include/*.h declares, lays out the boundary structs exactly as the reference
headers do, and rejects bad arguments with status codes (no compute)."""
import ctypes
import json
import os
import re
import subprocess

import pytest

from conftest import GOLDEN, ROOT
from sputnipic_b200 import _lib, dropin
from sputnipic_b200 import workload as W

HEADER_DIR = os.path.join(ROOT, "include")

# C++-linkage drop-ins (include/Mover.h:11-26 of the reference)
CXX_DROPINS = [
    "mover_PC(particles*, EMfield*, grid*, parameters*)",
    "mover_PC_V(particles*, EMfield*, grid*, parameters*)",
    "interpP2G(particles*, interpDensSpecies*, grid*)",
    "mover_interp(particles*, EMfield*, interpDensSpecies*, grid*, parameters*)",
    "calculateHatDensities(interpDens_aux*, interpDensNet*, interpDensSpecies*, EMfield*, grid*, "
    "parameters*)",
]


def declared_c_functions():
    names = set()
    for fn in os.listdir(HEADER_DIR):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(HEADER_DIR, fn)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(spb_\w+)\s*\(", text))
    return sorted(names)


def exported_symbols(demangle):
    out = subprocess.run(["nm", "-D", "--defined-only"] + (["-C"] if demangle else [])
                         + [_lib.LIB_PATH], check=True, capture_output=True, text=True).stdout
    return {line.split(" ", 2)[2] for line in out.splitlines() if line.count(" ") >= 2}


def test_library_loads_and_reports_version():
    lib = _lib.load()
    assert b"sm_100a" in lib.spb_version()


def test_every_declared_symbol_is_exported():
    names = declared_c_functions()
    assert len(names) > 20
    lib = _lib.load()
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/ but not exported"
    syms = exported_symbols(demangle=False)
    for n in names:
        assert n in syms
    demangled = exported_symbols(demangle=True)
    for sig in CXX_DROPINS:
        assert sig in demangled, f"C++ drop-in {sig} not exported"


def test_struct_layout_matches_reference_headers():
    with open(os.path.join(GOLDEN, "abi_layout.json")) as f:
        ref = json.load(f)
    assert _lib.library_layout() == ref
    mine = _lib.ctypes_layout()
    assert {k: mine[k] for k in ref} == ref


def test_error_strings():
    lib = _lib.load()
    for code in range(0, 9):
        assert lib.spb_error_string(code)
    assert lib.spb_error_string(0) == b"ok"


def test_dropin_rejects_null_arguments_without_touching_the_gpu():
    lib = _lib.load()
    assert lib.spb_mover_PC(None, None, None, None) == 2
    assert lib.spb_last_error() == 2
    assert b"null" in lib.spb_last_error_message()
    lib.spb_clear_error()
    lib.spb_interpP2G(None, None, None)
    assert lib.spb_last_error() == 2
    assert lib.spb_mover_interp(None, None, None, None, None) == 2


def test_grid_of_2_to_31_nodes_is_rejected_before_any_device_work():
    """The plain kernels index nodes with 32-bit integers: a grid of 2^31
    nodes or more is refused at creation, before the library looks for a
    device."""
    import ctypes
    lib = _lib.load()
    out = ctypes.c_void_p()
    assert lib.spb_grid_create_uniform(1300, 1300, 1300, 1.0, 1.0, 1.0, ctypes.byref(out)) == 6
    assert b"2^31" in lib.spb_last_error_message()
    assert not out.value
    lib.spb_clear_error()


def test_plain_deposit_mode_switch():
    """spb_set_plain_deposit_mode returns the previous mode and rejects
    unknown ones (no device work)."""
    from sputnipic_b200.device import set_plain_deposit_mode
    lib = _lib.load()
    assert lib.spb_set_plain_deposit_mode(7) == 2
    assert lib.spb_last_error() == 2
    lib.spb_clear_error()
    prev = set_plain_deposit_mode("direct")
    try:
        assert set_plain_deposit_mode("accumulator") == "direct"
        assert set_plain_deposit_mode("accumulator") == "accumulator"
    finally:
        set_plain_deposit_mode(prev)


def test_dropin_rejects_bad_mover_parameters():
    wl = W.small_gem()
    param = dropin.make_parameters(wl)
    grd = dropin.setGrid(param)
    field = dropin.field_allocate(grd)
    part = dropin.particle_allocate(param, 0, arrays={k: W.np.zeros(4, W.np.float32)
                                                      for k in "xyzuvwq"})
    part.NiterMover = 0
    assert dropin.mover_PC(part, field, grd, param) == 2
    part.NiterMover = 3
    part.n_sub_cycles = 0
    assert dropin.mover_PC(part, field, grd, param) == 2


def test_set_residency_validates_mode():
    lib = _lib.load()
    assert lib.spb_set_residency(7) == 2
    assert lib.spb_set_residency(0) == 0


def test_python_setgrid_matches_reference_arithmetic():
    """setGrid mirror (src/Grid.cpp:5-62) equals the restated oracle's grid
    arithmetic: same node coordinates and float inverses."""
    wl = W.small_gem()
    grd = dropin.setGrid(dropin.make_parameters(wl))
    xs, ys, zs = wl.node_coords()
    XN = grd._arrays["XN"].reshape(grd.nxn, grd.nyn, grd.nzn)
    assert (XN[:, 3, 5] == xs).all()
    assert grd.nxn == wl.nxc + 3 and grd.nzn == wl.nzc + 3
    assert W.np.float32(grd.invVOL) == wl.invVOL


def test_grid_create_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    lib = _lib.load()
    h = ctypes.c_void_p()
    assert lib.spb_grid_create_uniform(4, 4, 4, 1.0, 1.0, 1.0, ctypes.byref(h)) == 4


def test_library_has_no_unresolved_internal_symbols():
    """Every symbol of the library's own namespace is defined in it (a shared
    library links with undefined symbols; loading would fail later)."""
    out = subprocess.run(["nm", "-u", _lib.LIB_PATH], check=True, capture_output=True,
                         text=True).stdout
    assert not [line for line in out.splitlines() if "3spb" in line or " spb_" in line]
