"""Precision form: a device-resident simulation of the mover + deposit
(spb_sim_* of libsputnipic_b200.so) over torch CUDA tensors.

Particles are kept in HBM in per-cell buckets (FP32 in-cell offsets, charge
and velocities; the cell is implicit) with an overflow list for full buckets.
A cycle is a push kernel, which writes every particle into its new cell's
bucket of a second buffer set, and a deposit kernel, which sums each bucket
in registers and adds the node sums into FP64 moments. See
include/sputnipic_b200.h.
"""
from __future__ import annotations

import ctypes

from . import _lib


def _stream(stream):
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Simulation:
    def __init__(self, wl, tile=(8, 4, 4), resort_every=4, ctas=0, species=None, variant=0,
                 bucket_slots=0, graph=False, deterministic=False, fused=False, capacity=None,
                 overflow_per_mille=0):
        self.lib = _lib.load()
        self.wl = wl
        species = list(range(len(wl.species))) if species is None else list(species)
        d = _lib.SimDesc()
        d.nxc, d.nyc, d.nzc = wl.nxc, wl.nyc, wl.nzc
        d.Lx, d.Ly, d.Lz = wl.Lx, wl.Ly, wl.Lz
        d.dt, d.c, d.niter = wl.dt, wl.c, wl.niter
        for a in range(3):
            d.periodic[a] = 1 if wl.periodic[a] else 0
        d.ns = len(species)
        for i, s in enumerate(species):
            d.qom[i] = wl.species[s].qom
        for a in range(3):
            d.tile[a] = tile[a]
        d.resort_every, d.ctas, d.variant = resort_every, ctas, variant
        d.bucket_slots = bucket_slots
        d.graph = 1 if graph else 0
        d.deterministic = 1 if deterministic else 0
        d.fused = 1 if fused else 0
        for i, c in enumerate(capacity or []):
            d.capacity[i] = int(c)
        d.overflow_per_mille = int(overflow_per_mille)
        h = ctypes.c_void_p()
        _lib.check(self.lib.spb_sim_create(ctypes.byref(d), ctypes.byref(h)))
        self.h = h
        self.desc = d
        self.ns = d.ns
        self.nodes = self.lib.spb_sim_nodes(h)

    def close(self):
        if self.h:
            self.lib.spb_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def launches(self) -> int:
        return self.lib.spb_sim_launches(self.h)

    def count(self, s: int) -> int:
        return self.lib.spb_sim_count(self.h, s)

    def bucket_slots(self, s: int) -> int:
        """Record slots of species s's bucket layout (summed over cells)."""
        return self.lib.spb_sim_bucket_slots(self.h, s)

    def overflow(self, s: int, stream=None) -> int:
        """Entries in species s's overflow list (synchronises)."""
        n = self.lib.spb_sim_overflow(self.h, s, _stream(stream))
        if n < 0:
            raise RuntimeError("spb_sim_overflow failed")
        return n

    def set_fields(self, fields, stream=None):
        """Six float32 tensors (CUDA or CPU) Ex, Ey, Ez, Bxn, Byn, Bzn."""
        on_dev = int(fields[0].is_cuda)
        arr = (ctypes.c_void_p * 6)(*[f.data_ptr() for f in fields])
        _lib.check(self.lib.spb_sim_set_fields(self.h, arr, on_dev, _stream(stream)))

    def load_species(self, s: int, part: dict, stream=None):
        """part: float32 tensors x, y, z, u, v, w, q (CUDA or CPU)."""
        on_dev = int(part["x"].is_cuda)
        n = part["x"].numel()
        _lib.check(self.lib.spb_sim_load_species(
            self.h, s, *[part[k].data_ptr() for k in "xyzuvwq"], n, on_dev, _stream(stream)))

    def cycle(self, ncycles: int = 1, stream=None):
        _lib.check(self.lib.spb_sim_cycle(self.h, ncycles, _stream(stream)))

    def resort(self, stream=None):
        """Re-lay out every species (compact buckets + overflow list)."""
        _lib.check(self.lib.spb_sim_resort(self.h, _stream(stream)))

    def moments(self, s: int, bc: bool = False, stream=None):
        """FP64 moments of species s as a (10, nodes) CUDA tensor (a copy).
        bc=True applies applyBCids to the simulation's moments first."""
        import torch
        if bc:
            _lib.check(self.lib.spb_sim_apply_bc_ids(self.h, s, _stream(stream)))
        out = torch.empty(10, self.nodes, dtype=torch.float64, device="cuda")
        _lib.check(self.lib.spb_sim_moments(self.h, s, out.data_ptr(), 1, _stream(stream)))
        return out

    def apply_bc_ids(self, s: int, stream=None):
        """applyBCids on species s's FP64 moments, in place."""
        _lib.check(self.lib.spb_sim_apply_bc_ids(self.h, s, _stream(stream)))

    def moments_view(self, s: int):
        """Species s's FP64 moments as a (10, nodes) CUDA tensor sharing the
        simulation's memory (no copy); valid until close(), zeroed by the
        next cycle. Used to sum the moments over ranks in place."""
        import torch
        ptr = self.lib.spb_sim_moments_device(self.h, s)
        if not ptr:
            raise RuntimeError(_lib.last_error())
        iface = {"shape": (10, self.nodes), "typestr": "<f8", "data": (ptr, False),
                 "version": 3, "strides": None}
        view = type("MomentsView", (), {"__cuda_array_interface__": iface})()
        return torch.as_tensor(view, device="cuda")

    def particles(self, s: int, stream=None) -> dict:
        """Positions (domain units), velocities and charges of species s,
        float32 CUDA tensors in cell order (then the overflow list)."""
        import torch
        n = self.count(s)
        out = {k: torch.empty(n, dtype=torch.float32, device="cuda") for k in "xyzuvwq"}
        _lib.check(self.lib.spb_sim_particles(self.h, s, *[out[k].data_ptr() for k in "xyzuvwq"],
                                              1, _stream(stream)))
        return out

    def check(self, stream=None) -> int:
        return self.lib.spb_sim_check(self.h, _stream(stream))

    def set_timing(self, on: bool = True):
        _lib.check(self.lib.spb_sim_set_timing(self.h, 1 if on else 0))

    def timing(self):
        """(cycle kernels ms, cycles, re-layout ms, re-layouts) since the last
        timing query."""
        t = self.kernel_timing()
        return t["push_ms"] + t["deposit_ms"], t["cycles"], t["relayout_ms"], t["relayouts"]

    def kernel_timing(self) -> dict:
        """Summed CUDA-event milliseconds of the push and deposit kernels and
        of the re-layouts since the last timing query (clears them)."""
        p, d, r = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        nc, nr = ctypes.c_int(), ctypes.c_int()
        _lib.check(self.lib.spb_sim_kernel_timing(self.h, ctypes.byref(p), ctypes.byref(d),
                                                  ctypes.byref(nc), ctypes.byref(r),
                                                  ctypes.byref(nr)))
        return {"push_ms": p.value, "deposit_ms": d.value, "cycles": nc.value,
                "relayout_ms": r.value, "relayouts": nr.value}


def autotune(wl, fields, parts, tiles=((8, 4, 4), (4, 4, 4), (8, 8, 4)), variants=(0, 1, 2),
             cycles=3, stream=None):
    """Picks the tile shape and push-kernel residency (variant) with the
    shortest push + deposit time on the given workload (device tensors; left
    intact), timed with CUDA events over `cycles` cycles after one warm-up
    cycle. Returns a dict with the choice and the measurements."""
    import torch
    n = sum(p["x"].numel() for p in parts)
    best, trials = None, []
    for tile in tiles:
        if any(N % t for N, t in zip((wl.nxc, wl.nyc, wl.nzc), tile)):
            continue
        for var in variants:
            sim = Simulation(wl, tile=tile, resort_every=10**6, variant=var)
            sim.set_fields(fields)
            for s, p in enumerate(parts):
                sim.load_species(s, p)
            sim.cycle(1)                       # warm-up (first launch, attributes)
            sim.set_timing(True)
            sim.kernel_timing()
            sim.cycle(cycles)
            t = sim.kernel_timing()
            sim.close()
            per = (t["push_ms"] + t["deposit_ms"]) / max(t["cycles"], 1)
            trials.append({"tile": list(tile), "variant": var, "cycle_ms": per,
                           "push_ms": t["push_ms"] / max(t["cycles"], 1),
                           "deposit_ms": t["deposit_ms"] / max(t["cycles"], 1)})
            if best is None or per < best[0]:
                best = (per, tile, var)
    torch.cuda.synchronize()
    return {"tile": best[1], "variant": best[2], "cycle_ms": best[0], "trials": trials,
            "particles": n}


def autotune_batching(wl, fields, parts, cycles=20, intervals=(1, 2, 4, 8), graph=True,
                      stream=None):
    """The batching form's autotuner: tile shape and push residency as
    ``autotune`` picks them, then the overflow-check (re-layout) interval k
    from ``intervals`` by timing ``cycles`` cycles from the loaded state with
    each (CUDA events around the whole run: cycles, checks and re-layouts).
    Returns the choice, the best run's milliseconds and all trials."""
    import torch
    tune = autotune(wl, fields, parts, stream=stream)
    n = tune["particles"]
    runs = []
    for k in intervals:
        sim = Simulation(wl, tile=tune["tile"], resort_every=k, variant=tune["variant"],
                         graph=graph)
        sim.set_fields(fields)
        for s, p in enumerate(parts):
            sim.load_species(s, p)
        st = torch.cuda.current_stream() if stream is None else stream
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(st)
        sim.cycle(cycles, stream=st)
        ev[1].record(st)
        torch.cuda.synchronize()
        ms = ev[0].elapsed_time(ev[1])
        assert sim.check() == 0
        sim.close()
        runs.append({"check_every": k, "ms": ms, "particles_per_s": n * cycles / (ms * 1e-3)})
    best = min(runs, key=lambda r: r["ms"])
    return {"tile": list(tune["tile"]), "variant": tune["variant"],
            "check_every": best["check_every"], "ms": best["ms"], "cycles": cycles,
            "particles": n, "particles_per_s": best["particles_per_s"], "intervals": runs,
            "tile_trials": tune["trials"]}
