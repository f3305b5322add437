"""One rank of the two-process particle-decomposition test (tests/test_ranks_gloo.py).

Run as `python tests/gloo_ranks_worker.py OUT` with RANK, WORLD_SIZE, MASTER_ADDR and
MASTER_PORT set. Each rank deposits its own seeded particles with the FP64 CPU oracle,
sums the moments over the ranks with sputnipic_b200.ranks over gloo, and writes what it
saw to OUT.<rank>.npz.
"""
import datetime
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import torch  # noqa: E402
import torch.distributed as dist  # noqa: E402

import oracle  # noqa: E402
from sputnipic_b200 import ranks as R  # noqa: E402
from sputnipic_b200 import workload as W  # noqa: E402


def tiny():
    return W.small_gem(nxc=8, nyc=4, nzc=4, species=W.gem_species((8, 8, 8, 8)))


def deposit(wl, part):
    orc = oracle.CpuOracle("restated", 64)
    mom = [np.zeros(wl.nodes) for _ in range(10)]
    orc.interp_p2g(oracle.setup_from(wl), {k: part[k].astype(np.float64) for k in "xyzuvwq"},
                   mom)
    return np.stack(mom)


def main():
    out = sys.argv[1]
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        wl = R.rank_workload(tiny(), rank)
        part = W.gem_particles(wl, 0)
        local = deposit(wl, part)
        mom = torch.from_numpy(local.copy())
        R.reduce_moments(mom, dist)
        slowest = R.max_over_ranks(1.5 + rank, dist, device="cpu")
        np.savez(f"{out}.{rank}.npz", local=local, summed=mom.numpy(), slowest=slowest,
                 x=part["x"], seed=wl.seed)
    finally:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
