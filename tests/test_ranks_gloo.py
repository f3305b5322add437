"""The multi-GPU path's host logic with two gloo ranks on the CPU.

bench.py --gpus N runs one process per GPU. Each rank has its own seeded copy of the
workload, and the moments are summed over the ranks (the reference's particle
decomposition, src/mpi_comm.cpp). Here two CPU processes do the same with the FP64
oracle as the deposit. The summed moments must equal one deposit of both ranks'
particles (linearity; relative 1e-12, an FP64 reordering), every rank must see the
same sum, and the reported time must be the slowest rank's.
"""
import os
import socket
import subprocess
import sys

import numpy as np

from conftest import ROOT

WORKER = os.path.join(ROOT, "tests", "gloo_ranks_worker.py")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_moment_sum_and_slowest_time(tmp_path):
    sys.path.insert(0, os.path.dirname(WORKER))
    import gloo_ranks_worker as gw

    out = str(tmp_path / "rank")
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(free_port()),
               WORLD_SIZE="2", OMP_NUM_THREADS="1")
    procs = [subprocess.Popen([sys.executable, WORKER, out], env=dict(env, RANK=str(r)),
                              stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
             for r in range(2)]
    for p in procs:
        try:
            log, _ = p.communicate(timeout=240)
        except subprocess.TimeoutExpired:
            for q in procs:
                q.kill()
            raise
        assert p.returncode == 0, log.decode()[-2000:]
    res = [np.load(f"{out}.{r}.npz") for r in range(2)]
    # the ranks hold different (independently seeded) particles
    assert int(res[0]["seed"]) != int(res[1]["seed"])
    assert not np.array_equal(res[0]["x"], res[1]["x"])
    # every rank sees the same sum, which is the deposit of all particles
    assert np.array_equal(res[0]["summed"], res[1]["summed"])
    wl0 = gw.tiny()
    both = {}
    for k in "xyzuvwq":
        parts = [gw.W.gem_particles(gw.R.rank_workload(wl0, r), 0)[k] for r in range(2)]
        both[k] = np.concatenate(parts)
    ref = gw.deposit(wl0, both)
    scale = np.abs(ref).max(axis=1, keepdims=True) + 1e-300
    assert (np.abs(res[0]["summed"] - ref) <= 1e-12 * scale).all()
    assert np.allclose(res[0]["local"] + res[1]["local"], ref, rtol=0, atol=1e-12 * scale.max())
    # the reported time is the slowest rank's
    assert float(res[0]["slowest"]) == float(res[1]["slowest"]) == 2.5


def test_bench_gpus_2_launches_two_ranks(tmp_path):
    """bench.py --gpus 2 without a launcher's environment starts two ranks itself
    (torch.distributed.run over 127.0.0.1); its --selftest-ranks mode runs the
    benchmark's rank plumbing on gloo. Each rank has its own seeded particles,
    the charge-weighted x per cell summed over the ranks equals that of both
    ranks' particles together, and the reported time is the slowest's."""
    import gloo_ranks_worker as gw

    out = str(tmp_path / "bench")
    env = {k: v for k, v in os.environ.items()
           if k not in ("RANK", "WORLD_SIZE", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    env["OMP_NUM_THREADS"] = "1"
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                        "--selftest-ranks", out], env=env, capture_output=True, timeout=300)
    assert p.returncode == 0, (p.stdout + p.stderr).decode()[-3000:]
    res = [np.load(f"{out}.{r}.npz") for r in range(2)]
    assert int(res[0]["world"]) == int(res[1]["world"]) == 2
    assert int(res[0]["seed"]) != int(res[1]["seed"])
    wl0 = gw.tiny()
    both = [gw.W.gem_particles(gw.R.rank_workload(wl0, r), 0) for r in range(2)]
    cell = np.concatenate([b["cell"] for b in both])
    qx = np.concatenate([b["q"].astype(np.float64) * b["x"] for b in both])
    ref = np.bincount(cell, weights=qx, minlength=wl0.cells)
    for r in range(2):
        assert np.allclose(res[r]["summed"], ref, rtol=1e-12, atol=0)
    assert np.array_equal(res[0]["summed"], res[1]["summed"])
    assert not np.array_equal(res[0]["local"], res[1]["local"])
    assert float(res[0]["slowest"]) == float(res[1]["slowest"]) == 2.5
