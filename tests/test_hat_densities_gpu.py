"""calculateHatDensities on the GPU (src/MaxwellSolver.cpp:465-603):
spb_hat_densities_f32 / _f64 on device arrays and the drop-in
spb_calculateHatDensities over the reference's host structs.

Bars (bit-exact, the computation has no reordering):
  - the SHA-256 of Jxh, Jyh, Jzh, rhoh equals the reference build's
    (tests/golden/hat_densities.json) in FP32 and FP64, for periodic,
    reflecting and mixed axes, through the device API and through the drop-in;
  - on the GEM grid (128x64x64, 4 species) the FP64 outputs equal the FP64
    oracle's element for element.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN
from sputnipic_b200 import workload as W

pytestmark = pytest.mark.gpu

PERIODIC = [(1, 0, 1), (1, 1, 1), (0, 0, 0), (0, 1, 0)]


def sha(arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def case(per):
    wl = W.small_gem(nxc=8, nyc=6, nzc=5, periodic=tuple(bool(p) for p in per))
    return wl, [sp.qom for sp in wl.species[:3]], 1.0


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(GOLDEN, "hat_densities.json")) as f:
        return json.load(f)


def run_device(torch, wl, qom, th, fp, mom, fields, rhoc):
    from sputnipic_b200.hat import hat_desc, hat_densities
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    out = hat_densities(hat_desc(wl, th, qom, fp), [[T(a) for a in sp] for sp in mom],
                        [T(f) for f in fields[3:]], T(rhoc))
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


@pytest.mark.parametrize("fp", [32, 64])
@pytest.mark.parametrize("per", PERIODIC)
def test_device_api_matches_reference_digests(cuda, golden, fp, per):
    wl, qom, th = case(per)
    dt = np.float32 if fp == 32 else np.float64
    mom, fields, rhoc = W.hat_inputs(wl, seed=golden["seed"], dtype=dt, ns=golden["species"])
    got = run_device(cuda, wl, qom, th, fp, mom, fields, rhoc)
    assert sha(got) == golden["cases"][f"{''.join(map(str, per))}_fp{fp}"]


@pytest.mark.parametrize("per", PERIODIC)
def test_dropin_structs_match_reference_digests(cuda, golden, per):
    from sputnipic_b200 import dropin as D
    wl, qom, th = case(per)
    ns = golden["species"]
    mom, fields, rhoc = W.hat_inputs(wl, seed=golden["seed"], dtype=np.float32, ns=ns)
    param = D.make_parameters(wl, ns=ns)
    param.th = th
    grd = D.setGrid(param)
    field = D.field_allocate(grd, fields)
    ids = [D.interp_dens_species_allocate(grd, s) for s in range(ns)]
    for s in range(ns):
        for dst, src in zip(D.moments(ids[s]), mom[s]):
            dst[...] = src
    idn = D.interp_dens_net_allocate(grd)
    idn._arrays["rhoc"][...] = rhoc
    aux = D.interp_dens_aux_allocate(grd)
    assert D.calculateHatDensities(aux, idn, ids, field, grd, param) == 0
    assert sha(D.hat_arrays(aux)) == golden["cases"][f"{''.join(map(str, per))}_fp32"]


def test_gem_grid_fp64_equals_oracle(cuda):
    wl = W.gem()
    qom = [sp.qom for sp in wl.species]
    mom, fields, rhoc = W.hat_inputs(wl, seed=3, dtype=np.float64)
    ref = oracle.CpuOracle("restated", 64).hat_densities(oracle.setup_from(wl), 1.0, qom, mom,
                                                         fields, rhoc)
    got = run_device(cuda, wl, qom, 1.0, 64, mom, fields, rhoc)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
