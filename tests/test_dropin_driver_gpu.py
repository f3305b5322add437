"""The reference's own, unmodified CPU driver (src/sputniPIC_CPU.cpp with the
field solver, BC, IO ...) linked against libsputnipic_b200.so in place of
src/Mover.cpp, against the same driver built with the reference's mover.

Both are built by tests/dropin_driver/Makefile from the reference sources
(single-process MPI and no-op HDF5 header stubs; the binaries travel with the
repository). They run the same small GEM deck for 3 cycles and their VTK
outputs are compared:
  cycle 1 species densities (rhoe, rhoi): relative L2 <= 1e-5 (same
      particles, FP32 sums in another order; see the plain-form parity tests)
  the net density rho_net (electron and ion densities nearly cancel, so its
      relative error is that of the species scaled by their ratio), cycle 1
      E and B, and every output of cycles 2-3: relative L2 <= 1e-3 (the field
      solve iterates to GMRES/CG tolerances, so tiny moment differences move
      the fields within those tolerances)
"""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

BUILD = os.path.join(ROOT, "tests", "dropin_driver", "_build")
DECK = """SaveDirName = data
RestartDirName = data
B0x = 0.0097
B0y = 0.00
B0z = 0.00
delta = 0.5
dt = 0.25
ncycles = 3
th = 1.0
c = 1.0
Lx = 20.0
Ly = 10.0
Lz = 10.0
nxc = 32
nyc = 16
nzc = 16
ns = 4
qom = -64.0 1.0 -64 1.0
rhoINIT = 1.0 1.0 0.02 0.02
npcelx = 3 3 3 3
npcely = 3 3 3 3
npcelz = 3 3 3 3
uth  = 0.045 0.0126 0.045 0.0126
vth  = 0.045 0.0126 0.045 0.0126
wth  = 0.045 0.0126 0.045 0.0126
u0 = 0.0 0.0 0.0 0.0
v0 = 0.0 0.0 0.0 0.0
w0 = 0.0065 -0.0325 0.0 0.0
FieldOutputCycle = 1
ParticlesOutputCycle = 1000
PoissonCorrection = true
n_sub_cycles = 1
"""


def read_vtk(path):
    """Data of a binary legacy VTK file written by VTK_Write_*_Binary
    (src/RW_IO.cpp:674-882): big-endian float32 after the header."""
    raw = open(path, "rb").read()
    m = re.search(rb"POINT_DATA (\d+)\n(VECTORS \S+ float\n|SCALARS \S+ float\nLOOKUP_TABLE default\n)",
                  raw)
    assert m, path
    n = int(m.group(1)) * (3 if m.group(2).startswith(b"VECTORS") else 1)
    return np.frombuffer(raw, dtype=">f4", count=n, offset=m.end()).astype(np.float64)


def run(binary, workdir):
    os.makedirs(os.path.join(workdir, "data"), exist_ok=True)
    with open(os.path.join(workdir, "deck.inp"), "w") as f:
        f.write(DECK)
    env = dict(os.environ, OMP_NUM_THREADS="4")
    p = subprocess.run([binary, "deck.inp"], cwd=workdir, env=env, capture_output=True,
                       text=True, timeout=600)
    assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
    return p.stdout


@pytest.mark.skipif(not os.path.exists(os.path.join(BUILD, "sputnipic_b200")),
                    reason="driver binaries are built where the reference tree exists")
def test_reference_driver_with_dropin_matches_reference_mover(cuda, tmp_path):
    out_ref = run(os.path.join(BUILD, "sputnipic_cpu"), str(tmp_path / "cpu"))
    out_b200 = run(os.path.join(BUILD, "sputnipic_b200"), str(tmp_path / "b200"))
    cg = [re.findall(r"CG converged at iteration # (\d+)", o) for o in (out_ref, out_b200)]
    assert len(cg[0]) == len(cg[1]) == 3
    bad = []
    for cyc in (1, 2, 3):
        for name in ("rhoe", "rhoi", "rho_net", "E", "B"):
            a = read_vtk(str(tmp_path / "cpu" / "data" / f"{name}_{cyc}.vtk"))
            b = read_vtk(str(tmp_path / "b200" / "data" / f"{name}_{cyc}.vtk"))
            err = np.linalg.norm(b - a) / max(np.linalg.norm(a), 1e-300)
            tol = 1e-5 if (cyc == 1 and name in ("rhoe", "rhoi")) else 1e-3
            if not err <= tol:
                bad.append((name, cyc, err, tol))
    assert not bad, bad
