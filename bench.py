#!/usr/bin/env python
"""Depth-step throughput of the BFPn pencil-beam solver on B200.

Metric: phase-space updates/s -- cells of both species advanced one full
Strang depth step per second.  Default workload: the full paper-scale grid,
the largest single-GPU configuration -- water, 230 MeV beam, sigma_E 2.3 MeV
(1 %), sigma_yz 0.5 cm, 16 x 16 cm lateral domain, Ny = Nz = 80,
Nmu = Nom = 20, Ng = 500, 40 cm depth (Nx = 1000, 1000 steps); 1.31 G cells
per array, both species, about 21 GB of float state resident in HBM.  Inputs
are the reference's water tables (tests/golden/tables/water).  Mixed
precision by default (float state; double energy recursion and IDD),
--precision fp64 for the parity mode.  --workload water230_20 runs the
20 x 20 single-beam configuration, bone230_80 the bone (1.85 g/cm3) grid.

One "step" = one depth step of the whole beam (both species) with the state
resident in HBM.  The four state arrays exceed the 126 MB L2 many times
over, so no flush is needed between timed steps.

Multi-GPU: independent replicas (one beam per GPU, no collective on the data
path); the timed region is bracketed by barriers and the time is the max over
ranks.

--impl reference times the CPU oracle (FP64 restatement of the reference's
eq15 path, all host threads) on a bounded sample of the same workload; that
arm loads only the oracle's library.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

# Single-beam workloads.  The default is the largest single-GPU configuration
# (80 x 80 lateral grid, about 48 GB of device memory in mixed precision).
WORKLOADS = {
    "water230_20": (dict(nx=1000, t_final=40.0, ny=20, nz=20, nmu=20, nom=20, ng=500, ly=8.0, lz=8.0,
                         beam_energy=230.0, sigma_e=2.3, sigma_yz=0.5, material_name="water"),
                    "water 230 MeV pencil beam, 20x20 yz / 20x20 angles / 500 groups, 40 cm (1000 depth steps)"),
    "water230_80": (dict(nx=1000, t_final=40.0, ny=80, nz=80, nmu=20, nom=20, ng=500, ly=16.0, lz=16.0,
                         beam_energy=230.0, sigma_e=2.3, sigma_yz=0.5, material_name="water"),
                    "water 230 MeV pencil beam, 80x80 yz / 20x20 angles / 500 groups, 40 cm (1000 depth steps)"),
    "bone230_80": (dict(nx=1000, t_final=40.0, ny=80, nz=80, nmu=20, nom=20, ng=500, ly=16.0, lz=16.0,
                        beam_energy=230.0, sigma_e=2.3, sigma_yz=0.5, material_name="bone", density=1.85,
                        energy_density=1.85),
                   "bone (1.85 g/cm3) 230 MeV pencil beam, 80x80 yz / 20x20 angles / 500 groups, 40 cm "
                   "(1000 depth steps)"),
}
DEFAULT_WORKLOAD = "water230_80"
WORKLOAD_KEY = DEFAULT_WORKLOAD
WORKLOAD, WORKLOAD_NAME = WORKLOADS[DEFAULT_WORKLOAD]
TABLES = os.path.join(ROOT, "tests", "golden", "tables", "water")
METRIC = "phase-space updates/s"
# Lateral positions per side of the CPU sample (see cpu_sample).
CPU_SAMPLE_NY = 20


def host_cpu():
    """Model name of the host CPU and the cores this process may run on."""
    name = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    name = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count()
    return name, cores


def cpu_sample(workload):
    """The bounded CPU sample of a workload: its central CPU_SAMPLE_NY x
    CPU_SAMPLE_NY lateral positions at the same spacing (dy, dz unchanged),
    with the full angular and energy grids, tables, beam and depth step.
    Every operator's work is per cell (the energy sweep, the source and the
    DST per lane; transport per plane cell), so updates/s carries over to the
    full grid.  Returns (workload dict, description)."""
    w = dict(workload)
    if w["ny"] <= CPU_SAMPLE_NY:
        return w, "the whole grid"
    w["ly"] = w["ly"] * CPU_SAMPLE_NY / w["ny"]
    w["lz"] = w["lz"] * CPU_SAMPLE_NY / w["nz"]
    w["ny"] = w["nz"] = CPU_SAMPLE_NY
    return w, ("the central %dx%d lateral positions (%.1f x %.1f cm at the workload's %.2f cm spacing) with "
               "the full %dx%d angles x %d groups" % (CPU_SAMPLE_NY, CPU_SAMPLE_NY, w["ly"], w["lz"],
                                                      w["ly"] / CPU_SAMPLE_NY, w["nmu"], w["nom"], w["ng"]))


def product_library_loaded():
    """True when this process has mapped the solver library (the reference
    arm must not)."""
    try:
        with open("/proc/self/maps") as f:
            return any("libbfpn_b200" in line for line in f)
    except OSError:
        return False


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(mode="w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.flush()
        self.out.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.out.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.out.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(backend="nccl"):
    """Rank / world from the torchrun environment; a process group when N > 1
    (nccl on GPUs; gloo for the CPU tests of this path)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, init_method="env://", world_size=world, rank=rank,
                                timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, local, device=None):
    """Max of a per-rank float over the ranks (device time of the slowest replica)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device if device is not None else "cuda:%d" % local)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, updates_per_step_per_rank, steps, max_ms):
    """Whole-job updates/s: every replica's updates over the slowest replica's time."""
    return world * updates_per_step_per_rank * steps / (max_ms / 1e3)


def kernel_bytes(cls, cells, elem, n_groups, nyz, NA, fused=False):
    """Algorithmic bytes (hbm) or flops (tensor) of one launch of a kernel class."""
    if cls == "energy":
        # F, f read + written; the secondary's launches also read the source (2 of the 4 separate passes, 2
        # of the 3 when the primary's passes are fused)
        return "hbm", (5.0 if fused else 4.5) * cells * elem
    if cls == "energy_fused":
        # F, f read + written once for two half-steps, the source groups' split-bf16 operand written
        return "hbm", 4.0 * cells * elem + 8.0 * nyz * NA * n_groups
    if cls == "transport":
        return "hbm", 2.0 * cells * elem
    if cls == "angle":
        return "hbm", 2.0 * cells * elem
    if cls == "source_energy":
        return "hbm", 3.0 * cells * elem  # A1, A2 read, S written
    if cls == "source_angular":
        return "tensor", 2.0 * 2.0 * nyz * NA * NA * n_groups  # two operands
    return "hbm", 0.0


# DRAM bytes (read + write) per cell of one launch of each kernel class, from ncu
# captures of the same kernels on a smaller state of the same lateral and
# angular grid (profiles/*.txt: the 20x20 kernels at 250 groups, the 80x80
# kernels at 40 groups), mixed precision; traffic grows in proportion to the
# cells, so a full launch is this times its cells.
NCU_DRAM_BYTES_PER_CELL = {
    "water230_20": {
        "transport": (176.52e6 + 122.73e6) / 44.1e6,
        "angle": (176.85e6 + 119.49e6) / 44.1e6,
        "energy": (352.90e6 + 295.12e6) / 44.1e6,
        "source_angular": (190.52e6 + 153.69e6 + 284.85e6 + 154.88e6) / 44.1e6,  # pack + GEMM
        "source_energy": (249.24e6 + 132.63e6) / 44.1e6,
    },
    "water230_80": {
        "transport": (420.0e6 + 366.8e6) / 104.976e6,  # transport_stream_kernel, 81x81x400x40
    },
}
NCU_DRAM_BYTES_PER_CELL["bone230_80"] = NCU_DRAM_BYTES_PER_CELL["water230_80"]


def run_ours(args):
    import torch
    from bfpn_gpu_b200 import Context, capi, make_config, read_tables

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    cfg = make_config(**WORKLOAD)
    prec = capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64
    elem = 4 if prec == capi.PREC_MIXED else 8
    mu, sig = read_tables(TABLES, cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), prec, device=local)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    ctx.step(1 + max(args.warmup, 3), fetch=False)  # first step (no secondary) + warm-up (graph capture)
    cells = ctx.cells
    updates_per_step = 2 * cells

    sampler = ClockSampler(local)
    torch.cuda.synchronize()
    barrier(world)
    sampler.start()
    ms = ctx.timed_steps(args.steps)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = max_over_ranks(ms, world, local)
    value = job_throughput(world, updates_per_step, args.steps, ms)
    kps = ctx.kernels_per_step()

    # per-kernel device times, eager launches bracketed by CUDA events
    ctx.set_profiling(True)
    ctx.kernel_profile(reset=True)
    prof_steps = 8  # one call: its first step opens and its last closes separately when the passes are fused
    ctx.step(prof_steps, fetch=False)
    prof = ctx.kernel_profile()
    ctx.set_profiling(False)
    nyz = (cfg.ny + 1) * (cfg.nz + 1)
    NA = cfg.nmu * cfg.nom
    n_groups = ctx.source_groups()
    fused = prof.get("energy_fused", (0.0, 0))[1] > 0
    pk, pk_kind = peaks()
    per_kernel = {}
    for cls, (tot, n) in prof.items():
        if n == 0:
            continue
        bound, work = kernel_bytes(cls, cells, elem, n_groups, nyz, NA, fused)
        avg = tot / n
        entry = {"launches_per_step": n / prof_steps, "ms_per_launch": avg, "share": tot / sum(v[0] for v in prof.values())}
        if work > 0:
            if bound == "hbm":
                entry["achieved_GBps"] = work / (avg / 1e3) / 1e9
            else:
                entry["achieved_TFLOPs"] = work / (avg / 1e3) / 1e12
        per_kernel[cls] = entry
    dom = max(prof.items(), key=lambda kv: kv[1][0])[0]
    bound, work = kernel_bytes(dom, cells, elem, n_groups, nyz, NA, fused)
    avg_s = prof[dom][0] / prof[dom][1] / 1e3
    per_cell = NCU_DRAM_BYTES_PER_CELL.get(WORKLOAD_KEY, {}).get(dom) if prec == capi.PREC_MIXED else None
    traffic = per_cell * cells if per_cell and args.ng is None else None  # bytes per launch
    if bound == "hbm":
        achieved = work / avg_s / 1e9
        peak = pk["hbm_gbs"]
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": pk_kind}
    else:
        achieved = work / avg_s / 1e12
        peak = pk.get("bf16_tflops_sustained", pk["bf16_tflops"])
        roof = {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": traffic, "peak_source": pk_kind}
    ctx.close()

    out = {"metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 state / f64 recursion" if prec == capi.PREC_MIXED else "f64",
           "data": "reference water tables; synthetic initial beam (Gaussian y/z/E, near-delta angle)",
           "config": {"workload": WORKLOAD_NAME, "precision": args.precision, "cells_per_array": cells,
                      "species": 2, "l2": "state arrays 4 x %.2f GB > L2; no flush" % (cells * elem / 1e9),
                      "parallelism": "replicas x%d" % world},
           "gpu_launches": kps * args.steps, "kernels_per_step": kps, "roofline": roof, "per_kernel": per_kernel}
    if clocks:
        out["clocks"] = clocks

    idd_e2e = None
    if rank == 0 and not args.no_e2e:
        out["e2e"], idd_e2e = e2e_job(cfg, prec, local)
    if rank == 0 and world == 1 and not args.no_accuracy and prec == capi.PREC_MIXED:
        out["accuracy"] = accuracy(cfg, local, mu, sig, args.accuracy_steps, idd_e2e)
    if rank == 0 and world == 1 and not args.no_cpu:
        out["cpu_baseline"] = cpu_baseline(args.cpu_steps)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def e2e_job(cfg, prec, device):
    """The whole beam solve through the public C ABI: host tables in, IDD
    history out.  Returns the e2e record and the IDD curve."""
    from bfpn_gpu_b200 import Context, capi, read_tables

    steps = cfg.max_steps()
    t0 = time.perf_counter()
    mu, sig = read_tables(TABLES, cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), prec, device=device)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    idd, proxy = ctx.step(steps)
    t1 = time.perf_counter()
    cells = ctx.cells
    elem = 4 if prec == capi.PREC_MIXED else 8
    NA = cfg.nmu * cfg.nom
    nyz = (cfg.ny + 1) * (cfg.nz + 1)
    h2d = (cfg.ng * NA * NA * elem + 2 * cfg.ng * cfg.ng * 8 + nyz * NA * 8 + 2 * cfg.ng * NA * elem
           + cfg.ng * 40 * 8)
    ctx.close()
    updates = cells * (2 * steps - 1)  # the first step advances the primary only
    rec = {"value": updates / (t1 - t0), "unit": "updates/s", "h2d_bytes_per_step": h2d / steps,
           "d2h_bytes_per_step": 16, "steps": steps, "seconds": t1 - t0,
           "what": "create + load tables + initial beam + %d depth steps + IDD/proxy history to host" % steps}
    return rec, idd


def accuracy(cfg, device, mu, sig, nsteps, idd_mixed=None):
    """IDD of the mixed-precision run against the FP64 run of the same beam
    (the FP64 path is pinned to the oracle at 1e-10 by the parity tests; the
    oracle itself needs days for this grid).  idd_mixed: the mixed curve of
    the e2e job, when it ran over the same steps."""
    from bfpn_gpu_b200 import Context, capi
    from bfpn_gpu_b200.validation import idd_accuracy

    idds = {}
    if idd_mixed is not None and len(idd_mixed) == nsteps:
        idds[capi.PREC_MIXED] = idd_mixed
    t0 = time.perf_counter()
    for prec in (capi.PREC_FP64, capi.PREC_MIXED):
        if prec in idds:
            continue
        ctx = Context(cfg.grid(), cfg.phys(), prec, device=device)
        ctx.load_tables(mu, sig)
        ctx.init_beam()
        idds[prec], _ = ctx.step(nsteps)
        ctx.close()
    res = idd_accuracy(idds[capi.PREC_MIXED], idds[capi.PREC_FP64], cfg.dt())
    res["against"] = "the FP64 GPU path over the same depth steps"
    res["seconds"] = time.perf_counter() - t0
    return res


def oracle_sample(steps, budget_s=None, warmup=0):
    """The oracle (FP64 restatement of the reference's path) on the host
    cores, on the bounded CPU sample of the workload (cpu_sample): regular
    depth steps (both species) from the initial beam, the first step's
    primary-only half skipped.  Loads only the oracle's library: the tables
    come through the oracle's own loader."""
    from bfpn_gpu_b200.config import make_config
    from oracle import oracle as O

    w, what = cpu_sample(WORKLOAD)
    cfg = make_config(**w)
    mu, sig = O.read_tables(TABLES, cfg.ng)
    threads = O.max_threads()
    o = O.Oracle(cfg.grid(), cfg.phys(), mu, sig)
    o.set_steps_done(1)  # regular steps: the secondary is advanced from the first one
    if warmup:
        o.step(warmup)
    done = 0
    t0 = time.perf_counter()
    while done < steps:
        o.step(1)
        done += 1
        if budget_s is not None and time.perf_counter() - t0 > budget_s:
            break
    sec = time.perf_counter() - t0
    cells = o.cells
    o.close()
    model, _ = host_cpu()
    return {"value": 2 * cells * done / sec, "unit": "updates/s", "cores": threads, "kind": "port",
            "sample": "%d regular depth step(s) (both species, FP64) of %s: %d cells per array; updates/s per "
                      "cell carries to the full workload" % (done, what, cells),
            "cpu": model, "seconds": sec, "steps": done}


def cpu_baseline(nsteps):
    """The oracle on the host cores, a bounded sample of the same workload."""
    return oracle_sample(nsteps)


def run_reference(args):
    """CPU reference arm: the oracle port on all host threads, rank 0 only,
    on the bounded CPU sample of the workload, time-bounded."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    rec = oracle_sample(args.steps, budget_s=args.reference_budget_s, warmup=min(args.warmup, 1))
    if product_library_loaded():
        raise RuntimeError("the reference arm mapped the solver library")
    done = rec["steps"]
    value = rec["value"]
    cpu = dict(rec)
    cpu.pop("steps")
    out = {"metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": done,
           "warmup": min(args.warmup, 1), "ms_per_step": rec["seconds"] * 1e3 / done, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "reference %s tables; synthetic initial beam" % WORKLOAD["material_name"],
           "config": {"workload": WORKLOAD_NAME, "precision": "fp64",
                      "sample": rec["sample"], "time_bound_s": args.reference_budget_s},
           "impl": "reference", "cpu_baseline": cpu,
           "e2e": {"value": value, "unit": "updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def _plain_run(r):
    """One beam through a fresh single context: create, tables, beam, all
    steps, IDD history to the host."""
    from bfpn_gpu_b200 import Context
    ctx = Context(r.cfg.grid(), r.cfg.phys(), r.precision)
    ctx.load_tables(r.mu, r.sigma)
    ctx.init_beam()
    idd, _ = ctx.step(r.nsteps)
    ctx.close()
    return idd


def _serve(reqs, arrivals, workers=2):
    """Submit each request at its arrival time (seconds from the start) to a
    continuous-batching server; returns (IDDs, makespan s, latencies ms)."""
    from bfpn_gpu_b200 import capi
    with capi.Server(devices=(0,), workers_per_device=workers) as srv:
        start = time.perf_counter()
        tickets, submit_t = [], []
        for r, at in zip(reqs, arrivals):
            delay = at - (time.perf_counter() - start)
            if delay > 0:
                time.sleep(delay)
            submit_t.append(time.perf_counter())
            tickets.append(srv.submit(r.beam()))
        out, lat = [], []
        for r, t, t0 in zip(reqs, tickets, submit_t):
            idd, _, info = srv.wait(t, r.nsteps)
            out.append(idd)
            lat.append(info["queue_ms"] + info["run_ms"])
        return out, time.perf_counter() - start, np.array(lat)


def _max_rel_diff(got, ref):
    return max(float(np.abs(a - b).max() / np.abs(b).max()) for a, b in zip(got, ref))


def run_batch(args):
    """Config 4: the seeded set of uneven beams (energy 70-230 MeV, water or
    bone, sigma_yz 0.3-0.8 cm, Ny = Nz in {16,32,48,64}, Nmu = Nom in
    {12,16,20}, Ng ~ 2 E0, depth 1.2 x CSDA range) served by continuous
    batching -- bundles by shape class, admitted by device footprint -- against
    the plain path, one beam at a time through a fresh context.  Beams/s of
    both, every batched IDD against the same beam run alone."""
    import torch  # noqa: F401
    from bfpn_gpu_b200 import beams, capi

    reqs = [r for r in beams.uneven_beams(args.batch_beams, seed=args.serve_seed) if r.cfg.ny <= args.batch_max_ny]
    for r in reqs:
        r.precision = capi.PREC_MIXED
    updates = sum(r.cells * (2 * r.nsteps - 1) for r in reqs)
    _plain_run(reqs[0])  # warm-up: module load
    t0 = time.perf_counter()
    alone = [_plain_run(r) for r in reqs]
    t_plain = time.perf_counter() - t0
    batched, t_batch, lat = _serve(reqs, np.zeros(len(reqs)))
    name, cores = host_cpu()
    out = {"metric": "beams/s", "value": len(reqs) / t_batch, "unit": "beams/s", "n_gpus": 1,
           "higher_is_better": True, "dtype": "f32 state / f64 recursion", "data": "synthetic seeded beam set, "
           "reference water / bone tables",
           "config": {"workload": "%d uneven beams (E 70-230 MeV, water/bone, Ny=Nz in 16/32/48/64 up to %d, "
                                  "Nmu=Nom in 12/16/20, Ng ~ 2 E0, depth 1.2 CSDA range; the first %d of the seeded "
                                  "set), all submitted at t=0" % (len(reqs), args.batch_max_ny, args.batch_beams),
                      "mode": "continuous batching (bundles by shape class, footprint admission)"},
           "plain_beams_per_s": len(reqs) / t_plain, "speedup_vs_plain": t_plain / t_batch,
           "seconds_batched": t_batch, "seconds_plain": t_plain,
           "updates_per_s_batched": updates / t_batch, "updates_per_s_plain": updates / t_plain,
           "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
           "max_idd_diff_batched_vs_alone_rel_to_peak": _max_rel_diff(batched, alone),
           "timing": "host wall clock around whole beam solves (set-up included)", "host_cpu": name}
    print(json.dumps(out), flush=True)


def run_serve(args):
    """Config 5: Poisson streams of beam requests at each rate of a sweep,
    drawn from the config-4 distribution with a share of full 80x80 paper-grid
    requests, served by continuous batching.  Per rate: beams/s, latency
    percentiles, and every served IDD against the same beam run alone."""
    import dataclasses

    import torch  # noqa: F401
    from bfpn_gpu_b200 import beams, capi, make_config, read_tables

    rates = [float(x) for x in args.serve_rates.split(",")]
    rng = np.random.default_rng(args.serve_seed + 7)
    small = beams.uneven_beams(args.serve_beams, seed=args.serve_seed)
    big_w, _ = WORKLOADS["water230_80"]
    big_cfg = make_config(**big_w)
    big_mu, big_sig = read_tables(os.path.join(ROOT, "tests", "golden", "tables", "water"), big_cfg.ng)
    reqs = []
    for r in small:
        if rng.random() < args.serve_large_frac:
            reqs.append(beams.BeamRequest(dataclasses.replace(big_cfg), big_mu, big_sig, big_cfg.max_steps(),
                                          capi.PREC_MIXED))
        else:
            r.precision = capi.PREC_MIXED
            reqs.append(r)
    n_large = sum(1 for r in reqs if r.cfg.ny == 80)
    alone = {}
    for k, r in enumerate(reqs):  # solo IDD of each distinct beam (the large requests are one beam)
        key = "large" if r.cfg.ny == 80 else k
        if key not in alone:
            alone[key] = _plain_run(r)
    ref = [alone["large" if r.cfg.ny == 80 else k] for k, r in enumerate(reqs)]
    sweep = []
    for rate in rates:
        arrivals = beams.poisson_arrivals(len(reqs), rate, seed=args.serve_seed + int(rate))
        print("serve: rate %g/s, %d requests ..." % (rate, len(reqs)), file=sys.stderr, flush=True)
        got, t, lat = _serve(reqs, arrivals)
        print("serve: rate %g/s done in %.1f s" % (rate, t), file=sys.stderr, flush=True)
        sweep.append({"rate_per_s": rate, "beams_per_s": len(reqs) / t, "makespan_s": t,
                      "latency_ms": {q: float(np.percentile(lat, float(q[1:]))) for q in ("p50", "p99", "p99.9")},
                      "max_idd_diff_vs_alone_rel_to_peak": _max_rel_diff(got, ref)})
    best = max(sweep, key=lambda x: x["beams_per_s"])
    out = {"metric": "served beams/s", "value": best["beams_per_s"], "unit": "beams/s", "n_gpus": 1,
           "higher_is_better": True, "dtype": "f32 state / f64 recursion",
           "data": "synthetic seeded requests, reference water / bone tables",
           "config": {"workload": "%d requests: config-4 beams with %d full 80x80x20x20x500 water 230 MeV "
                                  "requests, Poisson arrivals" % (len(reqs), n_large),
                      "rates_per_s": rates, "mode": "continuous batching (bundles by shape class, footprint "
                                                    "admission)"},
           "sweep": sweep, "timing": "host wall clock from each submit to its result"}
    print(json.dumps(out), flush=True)


def run_out_of_core(args):
    """The out-of-core mode (the reference's --streaming-full): the state in
    pinned host memory, each step streamed through the GPU in chunks.  K steps
    timed with CUDA events on the context stream; one replica."""
    import dataclasses
    import torch
    from bfpn_gpu_b200 import Context, capi, make_config, read_tables

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    cfg = dataclasses.replace(make_config(**WORKLOAD), streaming_full=True)
    prec = capi.PREC_MIXED if args.precision == "mixed" else capi.PREC_FP64
    mu, sig = read_tables(TABLES, cfg.ng)
    ctx = Context(cfg.grid(), cfg.phys(), prec, device=local)
    ctx.set_option(capi.OPT_LANE_CHUNK, args.lane_chunk)
    ctx.set_option(capi.OPT_ENERGY_CHUNK, args.energy_chunk)
    ctx.load_tables(mu, sig)
    ctx.init_beam()
    ctx.step(2, fetch=False)  # the first step (no secondary) and one regular step
    sampler = ClockSampler(local)
    torch.cuda.synchronize()
    barrier(world)
    sampler.start()
    ms = ctx.timed_steps(args.steps)
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms = max_over_ranks(ms, world, local)
    updates_per_step = 2 * ctx.cells
    value = job_throughput(world, updates_per_step, args.steps, ms)
    elem = 4 if prec == capi.PREC_MIXED else 8
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": 2, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 state / f64 recursion" if prec == capi.PREC_MIXED else "f64",
            "data": "reference tables; synthetic initial beam", "mode": "out-of-core",
            "config": {"workload": WORKLOAD_NAME, "precision": args.precision, "cells_per_array": ctx.cells,
                       "host_state_bytes": 4 * ctx.cells * elem, "lane_chunk": args.lane_chunk,
                       "energy_chunk": args.energy_chunk, "parallelism": "replicas x%d" % world},
            "gpu_launches": ctx.kernels_per_step() * args.steps, "clocks": clocks}), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--accuracy-steps", type=int, default=1000)
    ap.add_argument("--cpu-steps", type=int, default=1)
    ap.add_argument("--reference-budget-s", type=float, default=120.0)
    ap.add_argument("--batch", action="store_true",
                    help="the uneven beam set by continuous batching against the plain one-beam-at-a-time path")
    ap.add_argument("--batch-beams", type=int, default=64)
    ap.add_argument("--batch-max-ny", type=int, default=64, help="keep the beams of the set with Ny <= this")
    ap.add_argument("--serve", action="store_true",
                    help="Poisson request streams at each rate of --serve-rates, served by continuous batching")
    ap.add_argument("--serve-beams", type=int, default=20)
    ap.add_argument("--serve-rates", default="10,30,100,300,1000")
    ap.add_argument("--serve-large-frac", type=float, default=0.1)
    ap.add_argument("--serve-seed", type=int, default=20261203)
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD,
                    help="single-beam workload (default: the 80x80 paper-scale grid)")
    ap.add_argument("--ng", type=int, default=None,
                    help="energy groups (profiling captures on a smaller state; not for bench lines)")
    ap.add_argument("--out-of-core", action="store_true",
                    help="time the out-of-core mode (state in pinned host memory) on --workload")
    ap.add_argument("--lane-chunk", type=int, default=262144)
    ap.add_argument("--energy-chunk", type=int, default=128)
    args = ap.parse_args()
    global WORKLOAD, WORKLOAD_NAME, TABLES, WORKLOAD_KEY
    WORKLOAD_KEY = args.workload
    WORKLOAD, WORKLOAD_NAME = WORKLOADS[args.workload]
    WORKLOAD = dict(WORKLOAD)
    TABLES = os.path.join(ROOT, "tests", "golden", "tables", WORKLOAD["material_name"])
    if args.ng:
        WORKLOAD["ng"] = args.ng
    if args.batch:
        run_batch(args)
    elif args.serve:
        run_serve(args)
    elif args.out_of_core:
        run_out_of_core(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
