"""Benchmark of the mover + P2G hot path on the GEM cycle.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: 128x64x64 cells, 4 species x 65,536,000 particles (125 ppc on a
5x5x5 jittered sub-lattice), NiterMover = 3, E ~ U(-1e-3, 1e-3) plus the
Harris-sheet B; seeded synthetic inputs generated on the device. One step is
one cycle of the hot section of the reference driver
(src/sputniPIC_CPU.cpp:232-256, with the field refresh of :288-294): the new
fields, mover_PC for every species, zero the moments, interpP2G + applyBCids
for every species, and with N ranks the moment sum over the ranks
(src/sputniPIC_CPU.cpp:262-265).

Keys of the JSON line:
  value       particles pushed+deposited per second with all inputs already
              in HBM (device-timed with CUDA events, max over ranks)
  e2e         the same metric through the reference-facing C-ABI drop-in
              (spb_mover_PC / spb_interpP2G on the reference structs) with
              pinned HOST arrays: every step uploads the particles, fields and
              moments and downloads the results, inside the timed region
  roofline    the dominant kernel's algorithmic bytes per launch / its mean
              CUDA-event duration, against MEASURED_PEAKS.json's HBM copy
              bandwidth; frac_contract is the whole step against the
              compulsory 60 bytes per particle plus the grid bytes
  cpu_baseline  the reference CPU code (oracle/_ref, else the restated port)
              timed on this host's cores over whole cycles of the same
              workload (one warm-up cycle, two timed)
  plain       the plain drop-in (reference precision types) on device
              arrays, per-kernel figures
  serving     Poisson streams of independent frozen-field jobs through the
              serving engine at 10, 50, 200 and 500 jobs/s (a weighted mix of
              grids, a species capped at 5M particles), beside the same jobs
              served one at a time through the plain path; and the
              configuration's own mix (grids drawn uniformly, no cap) at 10
              jobs/s (uniform_mix_10_jobs_per_s)
  batching, hat_densities  the batching workload (uneven species, 20 cycles,
              autotuned) and calculateHatDensities on the GEM grid
  dense       the headline step on the dense variant (256x128x128 cells,
              4 species x 134,217,728 particles)
  next_rows   the drop-in's calls beside the path on the e2e leg's resident
              particles: the driver's moment section in one call
              (spb_interp_all_species) and the binned particle sort
              (spb_particle_sort)
The particle arrays (8.4 GB) are far larger than the 126 MB L2, so no L2
flush is needed between steps.

``--impl reference`` times the reference's own CPU mover_PC + interpP2G +
applyBCids (the CPU driver's hot section) on the full workload, W warm-up and
K timed cycles, with all host threads; under torchrun only rank 0 runs it.

``--gpus N`` without torchrun's environment starts N ranks itself (one per
GPU, torch.distributed.run over 127.0.0.1).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from sputnipic_b200 import ranks as R  # noqa: E402
from sputnipic_b200 import workload as W  # noqa: E402

METRIC = "mover_p2g_particles_per_s"
UNIT = "particles/s"
# the reference GPU build's published times on the same GEM config, 5.208 s and 4.942 s
# per mover+interp cycle of 262,144,000 particles (README.md:76,93)
PUBLISHED_PPS = 262_144_000 / ((5.208 + 4.942) / 2)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        if not self.lines:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[0]))
                smax = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# --- CPU reference arm ------------------------------------------------------------
def cpu_cycles(wl, parts, steps: int, warmup: int):
    """Times whole cycles of the CPU driver's hot section (mover_PC for every
    species, zero, interpP2G + applyBCids per species, timed inside the
    library with omp_get_wtime) on ``parts`` (list of host particle dicts
    with qom). Returns the timed cycles' seconds, the oracle kind ("reference"
    when oracle/_ref was built, else "port") and its threads."""
    import oracle
    kind = "reference" if oracle.reference_available(32) else "restated"
    orc = oracle.CpuOracle(kind, 32)
    fields = W.gem_fields(wl)
    setup = oracle.setup_from(wl)
    mom = [np.zeros(wl.nodes, np.float32) for _ in range(10 * len(parts))]
    times = []
    for i in range(warmup + steps):
        tm, ti = orc.cycle(setup, fields, parts, mom)
        if i >= warmup:
            times.append(tm + ti)
    return times, ("reference" if kind == "reference" else "port"), orc.threads


def run_reference_arm(args, rank):
    if rank != 0:
        return
    wl = W.gem()
    parts = W.gem_particles_host(wl)
    n = sum(len(p["x"]) for p in parts)
    times, kind, cores = cpu_cycles(wl, parts, args.steps, args.warmup)
    t = sum(times)
    pps = n * len(times) / t
    sample = (f"the whole workload every step: {n} particles ({n // len(parts)} per species), "
              f"full 128x64x64 grid; {args.warmup} warm-up and {len(times)} timed cycles")
    line = {
        "impl": "reference", "metric": METRIC, "value": pps, "unit": UNIT,
        "n_gpus": args.gpus, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": 1e3 * t / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": pps / PUBLISHED_PPS,
        "dtype": "fp32", "data": "synthetic (seeded GEM Harris sheet)",
        "config": {"workload": wl.name, "particles": n, "niter": wl.niter,
                   "form": "reference CPU (mover_PC + interpP2G + applyBCids)",
                   "step_seconds": times},
        "cpu_baseline": {"value": pps, "unit": UNIT, "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": pps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# --- our arm ------------------------------------------------------------------------
def algorithmic_bytes(kind: str, n: int, nodes: int, ns: int = 1) -> int:
    """Compulsory HBM bytes of one launch (per-kernel table of the design notes)."""
    if kind == "mover":       # plain: read x..w, write x..w; packed fields once
        return 48 * n + 24 * nodes
    if kind == "p2g":         # plain: read x..w, q; read+write the ten FP32 moments
        return 28 * n + 80 * nodes
    if kind == "push":        # precision: read + write 32-byte records; fields (32 B/node)
        return 64 * n + 32 * nodes
    if kind == "deposit":     # precision: read 32-byte records; FP64 moments written once
        return 32 * n + 80 * nodes * ns
    raise ValueError(kind)


def load_traffic():
    """DRAM bytes per particle of each kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def device_timed(torch, dist, stream, steps, fn):
    """Runs fn() `steps` times between CUDA events; max over ranks (ms)."""
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for _ in range(steps):
        fn()
    t1.record(stream)
    torch.cuda.synchronize()
    return R.max_over_ranks(t0.elapsed_time(t1), dist)


def measure_plain(args, torch, wl, fields, parts, dist, stream):
    """Plain form (reference precision types) on device-resident arrays: the
    CPU driver's sequence mover_PC x ns, zero moments, interpP2G + applyBCids."""
    from sputnipic_b200 import _lib
    from sputnipic_b200.device import GridContext, push_params
    ns = len(parts)
    counts = [p["x"].numel() for p in parts]
    ctx = GridContext(wl)
    ctx.set_fields(fields)
    pushes = [push_params(wl, s) for s in range(ns)]
    mom = torch.zeros(ns, 10, wl.nodes, device="cuda")
    ev = {"mover": [], "p2g": []}
    peak = peaks()[0]

    def timed(kind, n, fn, record):
        if record:
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
        fn()
        if record:
            b.record(stream)
            ev[kind].append((a, b, n))

    def step(record=False):
        for s in range(ns):
            timed("mover", counts[s], lambda: ctx.mover(parts[s], pushes[s]), record)
        mom.zero_()
        for s in range(ns):
            timed("p2g", counts[s], lambda: ctx.p2g(parts[s], mom[s]), record)
            ctx.apply_bc_ids(mom[s], wl.periodic)
        if dist is not None:
            R.reduce_moments(mom, dist)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    rc = ctx.check()
    if rc:
        raise RuntimeError(f"plain warm-up status {rc}: {_lib.last_error()}")
    steps = max(2, args.steps // 2)
    ms = device_timed(torch, dist, stream, steps, lambda: step(True))
    kern = {}
    for k, lst in ev.items():
        durs = [a.elapsed_time(b) for a, b, _ in lst]
        n_mean = statistics.mean(c for _, _, c in lst)
        alg = algorithmic_bytes(k, int(n_mean), wl.nodes)
        ach = alg / (statistics.mean(durs) / 1e3) / 1e9
        kern[k] = {"ms_mean": statistics.mean(durs), "share": sum(durs) / ms,
                   "algorithmic_bytes": alg, "achieved_gbs": ach, "frac": ach / peak,
                   "peak_gbs": peak}
    ctx.close()
    del mom
    return {"value": sum(counts) * steps / (ms / 1e3), "ms_per_step": ms / steps,
            "steps": steps, "kernels": kern}


def measure_precision(args, torch, wl, fields, parts, dist, stream, world):
    """Precision form: per cycle one push kernel and one deposit kernel for
    all species (particles in per-cell buckets, no sort); overflow checks
    every `resort` cycles (counted in the steps)."""
    from sputnipic_b200 import _lib
    from sputnipic_b200.sim import Simulation
    ns = len(parts)
    n = sum(p["x"].numel() for p in parts)
    tune = None
    if args.autotune:
        from sputnipic_b200.sim import autotune
        tune = autotune(wl, fields, parts)
        args.tile, args.variant = list(tune["tile"]), tune["variant"]
    sim = Simulation(wl, tile=tuple(args.tile), resort_every=args.resort, variant=args.variant,
                     graph=not args.no_graph, fused=args.fused,
                     deterministic=args.deterministic)
    sim.set_fields(fields)
    for s, p in enumerate(parts):
        sim.load_species(s, p)
    views = [sim.moments_view(s) for s in range(ns)]

    def step():
        # the driver's cycle: new fields (uploaded from device arrays and
        # packed), mover + deposit of every species, applyBCids per species,
        # and with several ranks the moment sum (mpi_reduce_densities)
        sim.set_fields(fields)
        sim.cycle(1)
        for s in range(ns):
            sim.apply_bc_ids(s)
        if dist is not None:
            for v in views:
                R.reduce_moments(v, dist)

    for _ in range(args.warmup):
        step()
    rc = sim.check()
    if rc:
        raise RuntimeError(f"precision warm-up status {rc}: {_lib.last_error()}")
    lib = _lib.load()
    l0 = lib.spb_launch_count()
    local_rank = torch.cuda.current_device()
    with Clocks(local_rank) as clk:
        ms = device_timed(torch, dist, stream, args.steps, step)
    launches = lib.spb_launch_count() - l0
    # per-kernel breakdown: a separate pass with CUDA events around each kernel
    # (direct launches), outside the timed region above
    sim.set_timing(True)
    sim.kernel_timing()
    for _ in range(min(args.steps, 4)):
        sim.cycle(1)
    kt = sim.kernel_timing()
    sim.set_timing(False)
    rc = sim.check()
    if rc:
        raise RuntimeError(f"precision status {rc}: {_lib.last_error()}")
    overflow = [sim.overflow(s) for s in range(ns)]
    slots = [round(sim.bucket_slots(s) / wl.cells, 2) for s in range(ns)]
    peak, peak_kind = peaks()
    nc = max(kt["cycles"], 1)
    traffic = load_traffic()
    kernels = {}
    for k, name in (("push", "k_push (mover, all species)"),
                    ("deposit", "k_deposit (10-moment deposit, all species)")):
        kms = kt[k + "_ms"] / nc
        alg = algorithmic_bytes(k, n, wl.nodes, ns)
        ach = alg / (kms / 1e3) / 1e9
        tr = traffic.get("k_" + k)
        kernels[k] = {"kernel": name, "ms_mean": kms, "algorithmic_bytes": alg,
                      "achieved": ach, "frac": ach / peak, "share_of_step": kms / (ms / args.steps),
                      "traffic": (tr["dram_bytes_per_particle"] * n +
                                  tr.get("dram_bytes_per_node_species", 0.0) * wl.nodes * ns
                                  if tr else None)}
    dom = max(kernels, key=lambda k: kernels[k]["ms_mean"])
    d = kernels[dom]
    cyc_ms = kernels["push"]["ms_mean"] + kernels["deposit"]["ms_mean"]
    cyc_alg = kernels["push"]["algorithmic_bytes"] + kernels["deposit"]["algorithmic_bytes"]
    # the contract's compulsory bytes of the whole step: 60 B per particle
    # (read 32: int32 cell + 3 fp32 offsets + 3 fp32 velocities + fp32 q;
    # write 28) plus the grid (fields read once, 6 x fp32; every species' ten
    # fp64 moments written once), over the device-timed step
    step_s = ms / args.steps / 1e3
    grid_bytes = wl.nodes * (6 * 4 + ns * 10 * 8)
    contract_bytes = 60 * n + grid_bytes
    roofline = {
        "kernel": d["kernel"], "bound": "hbm", "achieved": d["achieved"], "peak": peak,
        "unit": "GB/s", "frac": d["frac"], "traffic": d["traffic"],
        "traffic_source": ("not measured in this run: DRAM bytes per particle (and per node and "
                           "species) of the committed ncu capture profiles/traffic.json (one "
                           "species, 64x64x64 cells at this workload's cell size and ppc) "
                           "times this launch's particles (and nodes x species)"),
        "frac_contract": contract_bytes / step_s / 1e9 / peak,
        "contract": {"bytes_per_particle": 60, "grid_bytes": grid_bytes,
                     "bytes_per_step": contract_bytes, "achieved": contract_bytes / step_s / 1e9,
                     "basis": "whole device-timed step (fields, push, deposit, applyBCids)"},
        "algorithmic_bytes": d["algorithmic_bytes"], "kernel_ms_mean": d["ms_mean"],
        "peak_source": ("measured: MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured" else
                        "fallback: 6650 GB/s, an earlier copy-bandwidth measurement on B200 "
                        "(MEASURED_PEAKS.json absent)"),
        "share_of_step": d["share_of_step"], "kernels": kernels,
        "cycle": {"kernels_ms": cyc_ms, "algorithmic_bytes": cyc_alg,
                  "achieved": cyc_alg / (cyc_ms / 1e3) / 1e9,
                  "frac": cyc_alg / (cyc_ms / 1e3) / 1e9 / peak},
        "relayouts": {"count": kt["relayouts"], "ms": kt["relayout_ms"]},
    }
    sim.close()
    return {"value": R.aggregate_rate(n, world, args.steps, ms / 1e3), "ms": ms,
            "roofline": roofline,
            "clocks": clk.summary(), "launches": launches, "autotune": tune,
            "buckets": {"mean_slots_per_cell": slots, "overflow_entries": overflow}}


def run_ours(args, rank, world, local_rank):
    import torch
    from sputnipic_b200 import _lib
    from sputnipic_b200.device import gen_fields, gen_particles

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    _lib.load()
    base = W.gem()
    if tuple(args.grid) != (base.nxc, base.nyc, base.nzc):
        # smaller profiling grid with the benchmark's cell size
        g = args.grid
        base = base.with_(nxc=g[0], nyc=g[1], nzc=g[2], Lx=base.Lx * g[0] / base.nxc,
                          Ly=base.Ly * g[1] / base.nyc, Lz=base.Lz * g[2] / base.nzc)
    wl = R.rank_workload(base, rank)
    if args.nspecies != 4 or args.ppc != 125:
        wl = wl.with_(lattice=5 if args.ppc == 125 else 0,
                      species=W.gem_species((args.ppc,) * 4)[:args.nspecies])
    ns = len(wl.species)
    stream = torch.cuda.current_stream()
    fields = gen_fields(wl)
    parts = [gen_particles(wl, s) for s in range(ns)]
    ntot = sum(p["x"].numel() for p in parts)
    host = None
    if not args.no_e2e:
        host = [{k: p[k].cpu().pin_memory() for k in "xyzuvwq"} for p in parts]
        host_f = [f.cpu().pin_memory() for f in fields]

    plain = None
    if not args.no_plain:
        plain = measure_plain(args, torch, wl, fields, [dict(p) for p in parts], dist, stream)
        # the plain run moved the particles: regenerate the initial state
        parts = [gen_particles(wl, s) for s in range(ns)]
    prec = measure_precision(args, torch, wl, fields, parts, dist, stream, world)
    del parts
    torch.cuda.empty_cache()

    e2e = None
    if host is not None:
        e2e = run_e2e(args, wl, host, host_f, world, dist)

    serving = None
    if not args.no_serving:
        # independent replicas under torchrun; rank 0 reports its own
        from sputnipic_b200.serve import measure_stream
        serving = measure_stream(njobs=args.serve_jobs,
                                 rates=[args.serve_rate] + [r for r in (50.0, 200.0, 500.0)
                                                            if r != args.serve_rate])
        torch.cuda.empty_cache()
        # the configuration's own mix (grids drawn uniformly, no cap on a
        # species) at a rate one GPU carries: about 9e8 particle-cycles a job
        lit = measure_stream(njobs=args.serve_jobs, rate=10.0, uniform=True)
        serving["uniform_mix_10_jobs_per_s"] = {
            k: lit[k] for k in ("mix", "jobs", "completed", "failed", "failure_codes", "latency_ms",
                                "single_job_latency_ms",
                                "p99_over_single_job_p99", "slowdown_vs_alone",
                                "throughput_particle_cycles_per_s", "plain_one_at_a_time",
                                "plain_alone_ms")}
        torch.cuda.empty_cache()

    hat = None
    if not args.no_hat:
        hat = measure_hat(torch, wl)

    batching = None
    if not args.no_batching:
        batching = measure_batching(torch, rank)

    dense = None
    if not args.no_dense:
        dense = measure_dense(torch, stream, args, rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # whole cycles of the same workload on the host's cores: the pinned
        # host copies (moved by the e2e leg, which is as good a state of the
        # workload as any) or fresh copies of the device arrays
        if host is None:
            parts = [gen_particles(wl, s) for s in range(ns)]
            host = [{k: p[k].cpu() for k in "xyzuvwq"} for p in parts]
            del parts
        cparts = [dict({k: host[s][k].numpy() for k in "xyzuvwq"}, qom=wl.species[s].qom)
                  for s in range(ns)]
        times, kind, cores = cpu_cycles(wl, cparts, 2, 1)
        cpu = {"value": ntot * len(times) / sum(times), "unit": UNIT, "cores": cores,
               "kind": kind, "ms_per_step": 1e3 * sum(times) / len(times),
               "sample": f"the whole workload ({ntot} particles): one warm-up and "
                         f"{len(times)} timed cycles of mover_PC + interpP2G + applyBCids"}

    if rank == 0:
        value = prec["value"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": prec["ms"] / args.steps,
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / PUBLISHED_PPS, "dtype": "fp32 push, fp64 moments",
            "data": "synthetic (seeded GEM Harris sheet, generated on the device)",
            "config": {"workload": f"{wl.name}: {ns} species x {ntot // ns:,} particles, "
                                   f"{wl.species[0].ppc:g} ppc, NiterMover {wl.niter}, "
                                   "one mover + 10-moment deposit cycle",
                       "form": "precision (per-cell buckets of fp32 offsets, charge and "
                               "velocities; fp32 push; fp32 per-cell register sums -> "
                               "fp64 moments)" + ("; fused cycle" if args.fused else "")
                               + ("; deterministic deposit" if args.deterministic else ""),
                       "step": "the driver's cycle: new fields (six device arrays uploaded "
                               "and packed), mover + deposit of every species, applyBCids "
                               "per species" + (", moment all-reduce over the ranks"
                                                if world > 1 else ""),
                       "tile": list(args.tile), "overflow_check_every": args.resort,
                       "cuda_graph": not args.no_graph,
                       "push_variant": args.variant, "buckets": prec["buckets"],
                       "autotune": prec["autotune"],
                       "particles_per_gpu": ntot, "grid_cells": [wl.nxc, wl.nyc, wl.nzc],
                       "parallelism": f"particle decomposition x{world}" if world > 1 else "1 GPU",
                       "l2": "particle arrays (8.4 GB) exceed the 126 MB L2; no flush needed"},
            "roofline": prec["roofline"], "clocks": prec["clocks"],
            "gpu_launches": prec["launches"],
            "plain": None if plain is None else {
                "value": plain["value"], "unit": UNIT, "ms_per_step": plain["ms_per_step"],
                "kernels": plain["kernels"], "speedup_of_precision_form": value / plain["value"]},
            "e2e": e2e, "cpu_baseline": cpu, "serving": serving, "hat_densities": hat,
            "batching": batching, "dense": dense,
            "next_rows": None if e2e is None else e2e.pop("next_rows", None),
        }
        print(json.dumps(line), flush=True)


def measure_dense(torch, stream, args, rank, steps=5, warmup=3):
    """The precision form's step on the dense variant of the GEM cycle: 256 x
    128 x 128 cells, 4 species x 134,217,728 particles (32 ppc), NiterMover 3,
    generated on the device. The same step as the headline (new fields, push
    and deposit of every species, applyBCids per species), CUDA graphs,
    overflow checks every `args.resort` cycles, device-timed over `steps`
    steps after `warmup`; frac_contract as the headline's (60 B per particle
    plus the grid bytes over the step time)."""
    from sputnipic_b200 import _lib
    from sputnipic_b200.device import gen_fields, gen_particles
    from sputnipic_b200.sim import Simulation
    wl = R.rank_workload(W.PRESETS["dense"](), rank)
    ns = len(wl.species)
    fields = gen_fields(wl)
    sim = Simulation(wl, tile=tuple(args.tile), resort_every=args.resort, graph=True)
    sim.set_fields(fields)
    n = 0
    for s in range(ns):
        p = gen_particles(wl, s)
        n += p["x"].numel()
        sim.load_species(s, p)
        del p
        torch.cuda.empty_cache()

    def step():
        sim.set_fields(fields)
        sim.cycle(1)
        for s in range(ns):
            sim.apply_bc_ids(s)

    for _ in range(warmup):
        step()
    rc = sim.check()
    if rc:
        raise RuntimeError(f"dense warm-up status {rc}: {_lib.last_error()}")
    ms = device_timed(torch, None, stream, steps, step)
    rc = sim.check()
    sim.close()
    torch.cuda.empty_cache()
    if rc:
        raise RuntimeError(f"dense status {rc}: {_lib.last_error()}")
    peak = peaks()[0]
    grid_bytes = wl.nodes * (6 * 4 + ns * 10 * 8)
    contract = (60 * n + grid_bytes) / (ms / steps / 1e3) / 1e9
    return {"workload": f"{wl.name}: {ns} species x {n // ns:,} particles, "
                        f"{wl.species[0].ppc:g} ppc, NiterMover {wl.niter}",
            "value": n * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "warmup": warmup, "tile": list(args.tile),
            "frac_contract": contract / peak, "peak_gbs": peak}


def measure_batching(torch, rank):
    """The batching form: 4 species of uneven counts (65.5M, 65.5M, 6.55M,
    6.55M) on the GEM grid, 20 cycles from the loaded state with CUDA graphs.
    The two-launch cycle with tile shape, push residency and overflow-check
    interval k in {1, 2, 4, 8} picked by the autotuner
    (sputnipic_b200.sim.autotune_batching); then, at the chosen tile shape and
    interval, the fused cycle (one persistent launch per cycle) and the
    deterministic deposit, timed the same way. `value` is the fastest."""
    from sputnipic_b200.device import gen_fields, gen_particles
    from sputnipic_b200.sim import Simulation, autotune_batching
    wl = R.rank_workload(W.batching_gem(), rank)
    fields = gen_fields(wl)
    parts = [gen_particles(wl, s) for s in range(len(wl.species))]
    n = sum(p["x"].numel() for p in parts)
    tune = autotune_batching(wl, fields, parts, cycles=wl.cycles)
    modes = {"two_launch": {"ms_per_cycle": tune["ms"] / tune["cycles"],
                            "particles_per_s": tune["particles_per_s"]}}
    st = torch.cuda.current_stream()
    for name, kw in (("fused", {"fused": True}), ("deterministic", {"deterministic": True})):
        sim = Simulation(wl, tile=tuple(tune["tile"]), resort_every=tune["check_every"],
                         graph=True, **kw)
        sim.set_fields(fields)
        for s, p in enumerate(parts):
            sim.load_species(s, p)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(st)
        sim.cycle(wl.cycles, stream=st)
        ev[1].record(st)
        torch.cuda.synchronize()
        rc = sim.check()
        sim.close()
        if rc:
            raise RuntimeError(f"batching {name} status {rc}")
        ms = ev[0].elapsed_time(ev[1])
        modes[name] = {"ms_per_cycle": ms / wl.cycles,
                       "particles_per_s": n * wl.cycles / (ms * 1e-3)}
    del parts, fields
    torch.cuda.empty_cache()
    best = max(modes, key=lambda k: modes[k]["particles_per_s"])
    counts = [wl.species_count(s) for s in range(len(wl.species))]
    return {"workload": f"{wl.name}: species of {', '.join(f'{c:,}' for c in counts)} "
                        f"particles, {wl.cycles} cycles, CUDA graphs",
            "value": modes[best]["particles_per_s"], "unit": UNIT, "mode": best,
            "ms_per_cycle": modes[best]["ms_per_cycle"], "modes": modes, "tile": tune["tile"],
            "push_variant": tune["variant"], "check_every": tune["check_every"],
            "intervals": tune["intervals"], "tile_trials": tune["tile_trials"]}


def measure_hat(torch, wl, reps=10, warmup=3):
    """calculateHatDensities (src/MaxwellSolver.cpp:465-603) on the workload's
    grid in FP64 (the precision form's moment type), device arrays, timed with
    CUDA events over `reps` calls of spb_hat_densities_f64 after `warmup`
    (arguments built once, so the host's per-call work stays ahead of the
    device's). Algorithmic bytes: the species' J and pressure arrays, B and
    rho_c read once, J hat and rho hat written once."""
    import ctypes

    from sputnipic_b200 import _lib
    from sputnipic_b200.hat import hat_desc, hat_densities
    ns = len(wl.species)
    mom, fields, rhoc = W.hat_inputs(wl, seed=11, dtype=np.float64)
    T = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    dmom = [[T(a) for a in sp] for sp in mom]
    dB = [T(f) for f in fields[3:]]
    drho = T(rhoc)
    desc = hat_desc(wl, 1.0, fp=64)
    out = hat_densities(desc, dmom, dB, drho)   # checks the arguments once
    mp = (ctypes.c_void_p * (10 * ns))(*[t.data_ptr() for sp in dmom for t in sp])
    bp = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in dB])
    st = torch.cuda.current_stream()
    args = (ctypes.byref(desc), mp, bp, ctypes.c_void_p(drho.data_ptr()),
            *[ctypes.c_void_p(t.data_ptr()) for t in out], ctypes.c_void_p(st.cuda_stream))
    fn = _lib.load().spb_hat_densities_f64
    for _ in range(warmup):
        _lib.check(fn(*args))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record(st)
    for _ in range(reps):
        _lib.check(fn(*args))
    ev[1].record(st)
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1]) / reps
    cells = (wl.nxc + 2) * (wl.nyc + 2) * (wl.nzc + 2)
    algo = 8 * ((9 * ns + 3 + 3) * wl.nodes + 2 * cells)
    peak = peaks()[0]
    achieved = algo / (ms * 1e-3) / 1e9
    return {"ms": ms, "species": ns, "dtype": "f64", "algorithmic_bytes": algo,
            "achieved_gbs": achieved, "frac": achieved / peak, "launches": 9,
            "note": "bit-identical to the reference's FP64 build; nine launches for all "
                    "species (divergences, guard fills as gather + scatter, node pass, J hat "
                    "guards, rho hat, rho hat guards)"}


def run_e2e(args, wl, host_parts, host_f, world, dist):
    """Drop-in path with host arrays: COPY residency, pinned host memory."""
    import torch
    from sputnipic_b200 import dropin
    ns = len(wl.species)
    param = dropin.make_parameters(wl)
    grd = dropin.setGrid(param)
    field = dropin.field_allocate(grd, [f.numpy() for f in host_f])
    # the struct adopts the pinned buffers (no copy for contiguous float32)
    P, keep = [], []
    for s in range(ns):
        arrs = {k: host_parts[s][k].numpy() for k in "xyzuvwq"}
        P.append(dropin.particle_allocate(param, s, arrays=arrs))
    ids = []
    for s in range(ns):
        i = dropin.interp_dens_species_allocate(grd, s)
        for name in list(i._arrays):
            t = torch.zeros(i._arrays[name].size, dtype=torch.float32).pin_memory()
            keep.append(t)
            i._arrays[name] = t.numpy()
            setattr(i, name + "_flat", t.numpy().ctypes.data)
        ids.append(i)
    nodes = wl.nodes
    n = [p.nop for p in P]
    h2d = sum(52 * c for c in n) + ns * (24 * nodes + 40 * nodes)
    d2h = sum(24 * c for c in n) + ns * 40 * nodes

    zero_s = [0.0]   # host seconds in the driver's setZeroSpeciesDensities

    def step():
        for s in range(ns):
            if dropin.mover_PC(P[s], field, grd, param) != 0:
                raise RuntimeError(dropin.last_error())
        for s in range(ns):
            z = time.perf_counter()
            dropin.setZeroSpeciesDensities(ids[s])
            zero_s[0] += time.perf_counter() - z
            dropin.interpP2G(P[s], ids[s], grd, raise_on_error=True)

    def timed(steps):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        zero_s[0] = 0.0
        t0 = time.perf_counter()
        for _ in range(steps):
            step()
        return R.max_over_ranks(time.perf_counter() - t0, dist)

    for _ in range(max(1, args.warmup)):
        step()
    steps = max(2, min(args.steps, 5))
    t = timed(steps)
    out = {"value": R.aggregate_rate(sum(n), world, steps, t), "unit": UNIT,
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": steps,
           "ms_per_step": 1e3 * t / steps,
           "host_setzero_ms_per_step": 1e3 * zero_s[0] / steps,
           "path": "spb_mover_PC + spb_interpP2G on reference structs, COPY residency, "
                   "pinned host arrays; timed on the host clock; the step includes the "
                   "driver's own host-side setZeroSpeciesDensities (host_setzero_ms_per_step)"}
    # the same calls with the particles kept in HBM (spb_set_residency): every
    # step still uploads each species' fields and moments and reads the
    # moments back; the particles went up once, before the timed steps
    dropin.release_all()
    if dropin.set_residency(True) == 0:
        try:
            for _ in range(max(1, args.warmup)):
                step()
            steps_d = max(2, min(args.steps, 10))
            td = timed(steps_d)
            for s in range(ns):
                dropin.sync_particles_to_host(P[s])
            out["next_rows"] = measure_next_rows(args, wl, P, ids, field, grd, param, dist)
        finally:
            dropin.set_residency(False)
        out["device_residency"] = {
            "value": R.aggregate_rate(sum(n), world, steps_d, td), "unit": UNIT,
            "h2d_bytes_per_step": ns * (24 * nodes + 40 * nodes),
            "d2h_bytes_per_step": ns * 40 * nodes, "steps": steps_d,
            "ms_per_step": 1e3 * td / steps_d,
            "host_setzero_ms_per_step": 1e3 * zero_s[0] / steps_d,
            "path": "the same calls in DEVICE residency: particles resident in HBM, per step each "
                    "species' fields and moments uploaded and its moments read back"}
    dropin.release_all()
    return out


def measure_next_rows(args, wl, P, ids, field, grd, param, dist):
    """The drop-in's calls beside the mover and the deposit, on the e2e leg's
    reference structs in DEVICE residency (particles resident), host clock
    around the synchronous calls, slowest rank:
      moment_section  spb_interp_all_species, the driver's moment section in
                      one call (src/sputniPIC_CPU.cpp:247-259: zero, interpP2G
                      of every species, applyBCids, sumOverSpecies; the
                      species' and net moments written to the host once)
      particle_sort   spb_particle_sort of every species (src/Particles.cpp:
                      72-234) with GEM_3D's sort_cps = 2: in place on the
                      resident copy when the device holds the newest particles
                      (after a mover_PC step), and through PCIe when the host
                      arrays are the newest (uploaded, sorted, downloaded);
                      algorithmic bytes of the sort: each particle's 28 bytes
                      read and written once"""
    import torch
    from sputnipic_b200 import dropin
    ns = len(P)
    n = sum(p.nop for p in P)
    nodes = wl.nodes
    idn = dropin.interp_dens_net_allocate(grd)
    keep = []
    for name in list(idn._arrays):
        t = torch.zeros(idn._arrays[name].size, dtype=torch.float32).pin_memory()
        keep.append(t)
        idn._arrays[name] = t.numpy()
        setattr(idn, name + "_flat", t.numpy().ctypes.data)

    def timed(call, reps):
        call()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            call()
        torch.cuda.synchronize()
        return R.max_over_ranks(time.perf_counter() - t0, dist) / reps

    def section():
        if dropin.interp_all_species(P, ids, idn, grd, param) != 0:
            raise RuntimeError(dropin.last_error())

    param.sort_cps = 2

    def sort_all():
        for s in range(ns):
            if dropin.particle_sort(param, P[s], grd) != 0:
                raise RuntimeError(dropin.last_error())

    reps = max(3, min(args.steps, 10))
    t_sec = timed(section, reps)
    t_copy = timed(sort_all, reps)          # the host arrays are the newest copy
    for s in range(ns):                     # now the device copy is
        if dropin.mover_PC(P[s], field, grd, param) != 0:
            raise RuntimeError(dropin.last_error())
    t_dev = timed(sort_all, reps)
    peak, peak_kind = peaks()
    sort_bytes = 56 * n
    return {
        "moment_section": {
            "call": "spb_interp_all_species", "residency": "device", "species": ns,
            "ms_per_call": 1e3 * t_sec, "particles_per_s": n / t_sec,
            "d2h_bytes_per_call": (ns + 1) * 40 * nodes},
        "particle_sort": {
            "call": "spb_particle_sort", "sort_cps": 2, "species": ns,
            "in_place": {
                "ms_per_call_all_species": 1e3 * t_dev, "particles_per_s": n / t_dev,
                "algorithmic_bytes": sort_bytes, "achieved_gbs": sort_bytes / t_dev / 1e9,
                "frac": sort_bytes / t_dev / 1e9 / peak, "peak_gbs": peak,
                "peak_source": peak_kind},
            "through_pcie": {
                "ms_per_call_all_species": 1e3 * t_copy, "particles_per_s": n / t_copy,
                "h2d_bytes_per_call": 28 * n, "d2h_bytes_per_call": 28 * n}}}


def launch_ranks(n: int) -> int:
    """Runs this script with the same arguments as n ranks under
    torch.distributed.run on this node (rendezvous on 127.0.0.1); returns the
    launcher's exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def rank_selftest(out: str, rank: int, world: int):
    """The multi-rank plumbing of the benchmark without a GPU: the ranks join
    a gloo process group as the GPU run joins NCCL, each takes its own seeded
    copy of a small GEM workload (sputnipic_b200.ranks.rank_workload), sums
    its particles' charge-weighted x per cell (a linear deposit that depends
    on the seeded positions) over the ranks with the
    same reduce_moments the GPU step uses, and reports the slowest of
    rank-dependent times through max_over_ranks."""
    import datetime

    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        wl = R.rank_workload(W.small_gem(nxc=8, nyc=4, nzc=4,
                                         species=W.gem_species((8, 8, 8, 8))), rank)
        p = W.gem_particles(wl, 0)
        local = np.bincount(p["cell"], weights=p["q"].astype(np.float64) * p["x"],
                            minlength=wl.cells)
        mom = torch.from_numpy(local.copy())
        R.reduce_moments(mom, dist)
        slowest = R.max_over_ranks(1.5 + rank, dist, device="cpu")
        np.savez(f"{out}.{rank}.npz", local=local, summed=mom.numpy(), slowest=slowest,
                 world=world, seed=wl.seed)
    finally:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--tile", type=int, nargs=3, default=[8, 4, 4])
    ap.add_argument("--nspecies", type=int, default=4,
                    help="smaller profiling cases only; the benchmark uses all 4")
    ap.add_argument("--ppc", type=float, default=125,
                    help="smaller profiling cases only; the benchmark uses 125")
    ap.add_argument("--grid", type=int, nargs=3, default=[128, 64, 64],
                    help="smaller profiling cases only (same cell size); the benchmark "
                         "uses 128 64 64")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--resort", type=int, default=4,
                    help="cycles between overflow checks (a species using its overflow "
                         "list is re-laid out)")
    ap.add_argument("--variant", type=int, default=0,
                    help="push kernel residency: 0 three CTAs per SM, 1 two, 2 four")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the tile shape and push variant first (timed on this workload)")
    ap.add_argument("--fused", action="store_true",
                    help="precision form: the fused cycle (one persistent launch per cycle)")
    ap.add_argument("--deterministic", action="store_true",
                    help="precision form: the deterministic deposit")
    ap.add_argument("--no-graph", action="store_true",
                    help="launch each cycle directly instead of replaying a CUDA graph")
    ap.add_argument("--no-serving", action="store_true",
                    help="skip the serving stream (Poisson arrivals of mixed jobs)")
    ap.add_argument("--serve-rate", type=float, default=10.0,
                    help="serving arrivals, jobs/s (the headline rate; 50, 200 and 500 jobs/s "
                         "are swept too)")
    ap.add_argument("--serve-jobs", type=int, default=100, help="jobs in the serving stream")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-hat", action="store_true",
                    help="skip the calculateHatDensities measurement")
    ap.add_argument("--no-dense", action="store_true",
                    help="skip the dense variant (256x128x128, 4 x 134M particles)")
    ap.add_argument("--no-batching", action="store_true",
                    help="skip the batching-form measurement (uneven species, autotuned)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--selftest-ranks", metavar="OUT", default=None,
                    help="check the multi-rank plumbing on the CPU (gloo): every rank sums its "
                         "particles' charge-weighted x per cell over the ranks and writes "
                         "OUT.<rank>.npz")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: run this script again under torch.distributed.run
        sys.exit(launch_ranks(args.gpus))
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}")
    if args.selftest_ranks:
        rank_selftest(args.selftest_ranks, rank, world)
        return
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
        try:
            run_ours(args, rank, world, local_rank)
        finally:
            dist.destroy_process_group()
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
