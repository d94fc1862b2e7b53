"""Benchmark of the B200 cell-grid Lennard-Jones path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config c2]

A step is one pass of the hot path over one synthetic system: the cell-grid
build (count, scan, scatter, within-cell sort) and the truncated-LJ pair
kernel (energy, force, totals).  Default workload: 10,000,000 particles
uniform in [0,1)^3 from the seeded drand48 generator, cutoff 0.01, cell
width = cutoff (100^3 cells), eps = 1, sigma = cutoff / 2.5.

value  = interacting ordered pairs per second over all ranks (inputs resident
         in HBM; L2 flushed between steps, flush excluded from the timing).
e2e    = the same metric through the host-buffer entry with host buffers:
         positions host->device, step, energy/force device->host in the
         caller's order, every step; steps back to back through
         lj_simulate_host_inorder_async() (one step's upload and compute overlap
         the previous step's download), the sorted-order entry
         (lj_simulate_host_async, + index) and the one-call lj_simulate_host()
         times beside it.
roofline: the pair kernel, algorithmic flops 8 per candidate pair of the
         reference's 27-cell stencil + 18 per interacting pair, against the
         FP32 CUDA-core peak 148 SMs x 128 lanes x 2 flop x the SM clock
         sampled during the timed region.
--impl reference times the CPU restatement of the reference's cell-grid
loop (the reference has no CPU path of its own) on the host cores, and adds
the reference's own GPU kernels (cudaLJ.cu built from source) timed on the
same seeded positions.

Under torchrun each rank runs its own independent system (seed + rank):
replicas, weak scaling, no collective on the data path.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "particle-interaction-with-optix_b200"))

METRIC = "LJ pairs/sec @10M particles, plain vs mixed-precision/batched at ≤1e-5 err"
FLOP_CANDIDATE = 8
FLOP_INTERACTING = 18
KERNEL_NAMES = {1: "k_pair_config", 6: "k_pair_pass", 10: "k_pair_pass2", 11: "k_pair_config (whole rows)",
                12: "k_pair_cellpair"}
RETIRED = {2: 1, 3: 1, 4: 1, 5: 6, 7: 6, 8: 10, 9: 10}   # tuning values of retired variants -> the kernel they run


def kernel_name(k: int) -> str:
    return KERNEL_NAMES[RETIRED.get(k, k)]
SCATTER_REGION = 56 << 20   # bytes of scattered records per binning scatter pass (the library's default)


def bin_launches(n: int, ncells: int) -> int:
    """Kernels one lj_bin launches: count, scan, the scatter passes, rank, large-cell sort."""
    passes = max(1, min(8, ncells, -(-16 * n // SCATTER_REGION)))
    return 4 + passes

CONFIGS = {
    "c1": dict(workload="uniform 100k, rc=0.05", n=100_000, dist="uniform", lo=(0, 0, 0), hi=(1, 1, 1), rc=0.05),
    "c2": dict(workload="uniform 10M, rc=0.01", n=10_000_000, dist="uniform", lo=(0, 0, 0), hi=(1, 1, 1), rc=0.01),
    "c3": dict(workload="sphere-shell 4M, rc=0.005", n=4_000_000, dist="sphere", lo=(-0.5,) * 3, hi=(1.5,) * 3,
               rc=0.005),
    "c4": dict(workload="uniform 10M, rc=0.02", n=10_000_000, dist="uniform", lo=(0, 0, 0), hi=(1, 1, 1), rc=0.02),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer end-to-end leg (profiling runs)")
    ap.add_argument("--pair-kernel", type=int, default=0,
                    help="run the headline with this lj_tuning.pair_kernel instead of the autotuner's choice (profiling)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other workloads (batched 512 systems, sphere shell, dense) reported beside the headline")
    ap.add_argument("--n", type=int, default=None, help="particles per GPU (overrides the --config preset)")
    ap.add_argument("--rc", type=float, default=None, help="cutoff = cell width (overrides the --config preset)")
    ap.add_argument("--dist", default=None, choices=["uniform", "shell"],
                    help="uniform in [0,1)^3, or a unit sphere shell in [-0.5,1.5)^3 (overrides the preset)")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slab"],
                    help="under torchrun: replicas (one system per rank, weak scaling; the default) or slab (one "
                         "system split into z slabs with a one-layer halo exchange, strong scaling)")
    ap.add_argument("--mode", default="config", choices=["config", "compat", "mixed"],
                    help="config: truncated law with forces (the benchmark); compat: the reference's law over the "
                         "27 cells (value counts candidate pairs); mixed: binary16 cell-relative records")
    return ap.parse_args()


def workload(args) -> dict:
    """The --config preset with the --n / --rc / --dist overrides applied."""
    cfg = dict(CONFIGS[args.config])
    if args.dist == "uniform":
        cfg.update(dist="uniform", lo=(0, 0, 0), hi=(1, 1, 1))
    elif args.dist == "shell":
        cfg.update(dist="sphere", lo=(-0.5,) * 3, hi=(1.5,) * 3)
    if args.n is not None:
        cfg["n"] = args.n
    if args.rc is not None:
        cfg["rc"] = args.rc
    if args.n is not None or args.rc is not None or args.dist is not None:
        kind = "uniform" if cfg["dist"] == "uniform" else "sphere-shell"
        cfg["workload"] = f"{kind} {cfg['n']}, rc={cfg['rc']}"
    return cfg


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.1)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------- dist
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(backend):
    import torch.distributed as dist
    from datetime import timedelta

    ws, rank, _ = dist_env()
    if ws > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=timedelta(seconds=120))
    return ws, rank


def allreduce_max(v: float, ws: int, device=None) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum(v: float, ws: int, device=None) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ----------------------------------------------------------------------------- cpu baseline
class CpuBaseline:
    """The oracle's restatement of the reference's cell-grid loop (27-cell
    stencil per particle, config law, FP32) on the host cores.  Set-up
    generates and bins the whole system once (timed, one thread); each step
    runs the pair loop over the first targets in cell order, sized to a time
    budget, and charges the binning time per target."""

    def __init__(self, cfg, seed):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ljoracle as O

        self.O = O
        n = cfg["n"]
        if cfg["dist"] == "uniform":
            x, y, z = O.generate_uniform(seed, n, cfg["lo"], cfg["hi"])
        else:
            x, y, z = O.generate_sphere(seed, n, (0.5, 0.5, 0.5), 1.0)
        self.g = O.grid_from_box(cfg["lo"], cfg["hi"], cfg["rc"])
        t0 = time.perf_counter()
        self.b = O.bin_particles(self.g, x, y, z, O.ORDER_INDEX)
        self.t_bin = time.perf_counter() - t0
        self.n, self.rc = n, cfg["rc"]
        self.sigma = float(np.float32(self.rc) / np.float32(2.5))
        self.e = np.empty(n, np.float32)
        self.f = np.empty((n, 3), np.float32)
        self.threads = O.max_threads()
        self.k1 = min(n, 20_000)

    def step(self, budget_s):
        while True:
            t0 = time.perf_counter()
            pairs = self.O.config_forces_f32_range(self.g, self.b, 0, self.k1, self.rc, 1.0, self.sigma, self.e,
                                                   self.f, self.threads)
            dt = time.perf_counter() - t0
            if dt > budget_s / 3 or self.k1 == self.n:
                break
            self.k1 = min(self.n, int(self.k1 * min(8.0, max(1.5, budget_s / max(dt, 1e-4)))))
        t_step = dt + self.t_bin * (self.k1 / self.n)
        self.last = {"value": pairs / t_step, "unit": "pairs/s", "cores": self.threads, "kind": "port",
                     "sample": f"binning of all {self.n} particles once ({self.t_bin:.2f}s, 1 thread, charged per "
                               f"target) + pair loop over the first {self.k1} sorted targets ({pairs} pairs, "
                               f"{dt:.2f}s, {self.threads} threads)"}
        return self.last


def run_reference(args, cfg):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    cb = CpuBaseline(cfg, args.seed)
    per_step = max(0.3, min(4.0, 150.0 / max(1, args.steps + args.warmup)))
    for _ in range(max(args.warmup, 0)):
        cb.step(per_step)
    vals = [cb.step(per_step)["value"] for _ in range(args.steps)]
    value = float(np.median(vals))
    info = cb.last
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded drand48)",
            "config": {"workload": cfg["workload"], "n": cfg["n"], "cutoff": cfg["rc"], "path": "cpu cell-grid loop"},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": info["cores"], "kind": "port",
                             "sample": info["sample"]},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_ref_gpu:
        try:
            rg = reference_gpu(cfg, args.seed)
        except Exception as exc:  # the harness needs a GPU; the CPU figure above stands without it
            rg = {"unavailable": f"{type(exc).__name__}: {exc}"}
        if rg:
            line["reference_gpu"] = rg
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------- ours
def run_ours(args, cfg):
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
    init_dist("nccl" if ws > 1 else "gloo")
    import ljcell

    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    ctx = ljcell.Context(dev.index, stream)
    seed = args.seed + rank
    n, rc = cfg["n"], cfg["rc"]
    g = ljcell.grid_from_box(cfg["lo"], cfg["hi"], rc)
    p = ljcell.params(rc)
    if cfg["dist"] == "uniform":
        soa, _ = ctx.generate_uniform(seed, n, cfg["lo"], cfg["hi"])
    else:
        soa, _ = ctx.generate_sphere(seed, n, (0.5, 0.5, 0.5), 1.0)
    x, y, z = soa["x"], soa["y"], soa["z"]
    mode = args.mode
    order = ljcell.ORDER_INDEX if mode == "compat" else ljcell.ORDER_X
    b = ctx.alloc_binned(g, n, order)
    energy, force, tot = ctx.alloc_outputs(n)
    rec = ctx.pack_mixed(g, ctx.bin(g, x, y, z, order=order, out=b)) if mode == "mixed" else None
    cand = torch.zeros(1, dtype=torch.int64, device=dev)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    def bin_stage():
        ctx.bin(g, x, y, z, order=order, out=b)

    def pair_stage():
        if mode == "config":
            ctx.compute(g, p, b, energy, force, tot)
        elif mode == "mixed":        # records packed in every step, counted in the pair stage
            ctx.pack_mixed(g, b, rec)
            ctx.compute_mixed(g, p, b, rec, energy, force, tot)
        else:                        # the reference's law (energies only, every particle of the 27 cells)
            ctx.compute_compat(g, b, energy)

    def step():
        bin_stage()
        pair_stage()

    for _ in range(max(args.warmup, 3)):
        step()
    ctx.sync()
    if mode != "config":
        pair_kernel = args.pair_kernel
        ctx.set_tuning(pair_kernel)
    elif args.pair_kernel:
        pair_kernel = args.pair_kernel
        ctx.set_tuning(pair_kernel)
    else:
        pair_kernel, _ = ctx.autotune_compute(g, p, b)   # outside the timed region
    step()
    ctx.sync()
    ctx.count_candidates(g, b.offsets, cand)
    ctx.sync()
    c_ref = int(cand.item())
    # compat: every candidate is an interaction of the reference's law (no cutoff)
    pairs = c_ref if mode == "compat" else ljcell.totals_from_tensor(tot)["pairs"]

    K = args.steps
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(K)]
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index) as clk:
        for k in range(K):
            flush.fill_(k & 0xFF)                      # L2 flush, outside the timed events
            ev[k][0].record(stream)
            bin_stage()
            ev[k][1].record(stream)
            pair_stage()
            ev[k][2].record(stream)
        torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    ctx.sync()
    t_bin = np.array([ev[k][0].elapsed_time(ev[k][1]) for k in range(K)])
    t_pair = np.array([ev[k][1].elapsed_time(ev[k][2]) for k in range(K)])
    t_step_ms = float(np.median(t_bin + t_pair))   # median of the K timed steps
    t_max_ms = allreduce_max(t_step_ms, ws, dev)
    total_pairs = allreduce_sum(float(pairs), ws, dev)
    value = total_pairs / (t_max_ms * 1e-3)

    clocks = clk.summary()
    sm_mhz = clocks["sm_mhz"] or 1965.0
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    peak_tflops = sms * 128 * 2 * sm_mhz * 1e6 / 1e12
    # compat: the reference's own count, 18 flop per candidate (cudaLJ.cu:550)
    algo_flops = 18 * c_ref if mode == "compat" else FLOP_CANDIDATE * c_ref + FLOP_INTERACTING * pairs
    pair_ms = float(np.median(t_pair))
    achieved = algo_flops / (pair_ms * 1e-3) / 1e12
    useful = (algo_flops if mode == "compat" else FLOP_INTERACTING * pairs) / (pair_ms * 1e-3) / 1e12
    kname = {"config": kernel_name(pair_kernel) if pair_kernel else "", "mixed": "k_pair_mixed_pass2",
             "compat": "k_pair_compat"}[mode]
    traffic = read_traffic(kname, cfg["workload"])

    # errors of the last step's outputs against an FP64 reference on a stratified target sample
    errors = None
    if rank == 0 and mode != "compat":
        smp = fp64_sample(g, b.offsets, b.cell[:n], b.xyzi[:n, :3].double(), rc, p.sigma)
        errors = error_stats(*smp, energy[:n], force[:n])
        errors["reference"] = "FP64 (torch, on the GPU) on the same positions, every particle of the 27-cell stencil"
        del smp

    # the reference law on the same particles (our compat kernel), comparable with the reference arm's pair kernel
    compat = None
    if rank == 0 and ws == 1 and cfg["dist"] == "uniform" and mode == "config":
        gc = ljcell.grid_compat(float(cfg["hi"][0]), rc) if tuple(cfg["lo"]) == (0, 0, 0) else g
        bc = ctx.bin(gc, x, y, z, order=ljcell.ORDER_INDEX)
        vc = ctx.compute_compat(gc, bc)
        cc = torch.zeros(1, dtype=torch.int64, device=dev)
        ctx.count_candidates(gc, bc.offsets, cc)
        compat_ms = time_events(lambda: ctx.compute_compat(gc, bc, vc), 5, flush)
        ctx.sync()
        ccand = int(cc.item())
        rate = ccand / (compat_ms * 1e-3)
        compat = {"ms": compat_ms, "kernel": "k_pair_compat", "candidate_pairs": ccand,
                  "candidate_pairs_per_s": rate,
                  "gflops_reference_definition": 18 * rate / 1e9,   # NbFlopsPerInteraction = 18, cudaLJ.cu:550
                  "fp32_frac": 18 * rate / 1e12 / peak_tflops,
                  "mufu_frac": rate / (sms * 16 * sm_mhz * 1e6),  # one reciprocal square root per candidate
                  "mufu_peak": f"{sms} SMs x 16 MUFU results per clock x {sm_mhz:.0f} MHz"}
        del bc, vc, cc

    e2e = None
    if not args.no_e2e and mode == "config":   # the host-buffer entry computes the truncated law
        e2e = run_e2e(ctx, g, p, x, y, z, n, K, ws, dev, total_pairs, pairs)


    extras = None
    if rank == 0 and ws == 1 and not args.no_extras and mode == "config":
        extras = run_extras(ctx, dev, flush, peak_tflops)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cb = CpuBaseline(cfg, args.seed)
        cb.step(2.0)
        c = cb.step(12.0)
        cpu = {k: c[k] for k in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": ws, "steps": K, "warmup": args.warmup,
            "ms_per_step": t_max_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded drand48, device generated)",
            "config": {"workload": cfg["workload"], "n_per_gpu": n, "cutoff": rc, "sigma": p.sigma,
                       "cells": g.ncells,
                       "order": "x-sorted within cells" if order == ljcell.ORDER_X else "index order within cells",
                       "mode": {"config": "plain fp32", "mixed": "mixed: binary16 cell-relative y, z records",
                                "compat": "reference law over the 27 cells; pairs = candidate pairs"}[mode],
                       "pair_kernel": f"{pair_kernel} ({kname}, " + ("set by --pair-kernel)" if args.pair_kernel else
                                                                     "chosen by lj_autotune_compute)")
                       if mode == "config" else kname,
                       "l2": "flushed between steps (256 MiB write), flush excluded from timing",
                       "parallelism": f"replicas x{ws}" if ws > 1 else "single gpu"},
            "stage_ms": {"bin": float(np.median(t_bin)), "pair": pair_ms, "statistic": f"median of {K} steps",
                         "step_mean": float((t_bin + t_pair).mean())},
            "pairs_per_step": pairs, "candidate_pairs_per_step": c_ref,
            "candidate_pairs_per_s": c_ref * ws / (t_max_ms * 1e-3),
            "particles_per_s": n * ws / (t_max_ms * 1e-3),
            "roofline": {"kernel": kname, "bound": "fp32", "achieved": achieved, "peak": peak_tflops,
                         "unit": "TFLOP/s", "frac": achieved / peak_tflops, "traffic": traffic,
                         "useful_frac": useful / peak_tflops,   # 18 flop per interacting pair only
                         "peak_source": f"{sms} SMs x 128 FP32 lanes x 2 flop x {sm_mhz:.0f} MHz (median sampled "
                                        "SM clock; MEASURED_PEAKS.json has no FP32 CUDA-core figure)",
                         "algorithmic_flops": algo_flops},
            "e2e": e2e,
            "gpu_launches": (bin_launches(n, g.ncells) + (2 if mode == "mixed" else 1)) * K,
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if errors:
            line["errors_vs_fp64"] = errors
        if compat is not None:
            line["reference_law_pair_kernel_ms"] = compat["ms"]
            line["reference_law_pair_kernel"] = compat
        if extras:
            line["workloads"] = extras
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def fp64_sample(g, offsets, cell, pos64, rc, sigma, sample=4096, eps=1.0):
    """FP64 reference of the truncated law for a stratified sample of sorted targets (torch, on the
    GPU): each sample target against every particle of its 27-cell stencil, pairs i != j with
    r < rc in FP64.  pos64: (n, 3) float64 positions in sorted order (the caller's, or the ones a
    storage format keeps).  Returns (targets, energy, force, energy scale, force scale): the scales
    are 4 eps sum (s^12 + s^6) and 24 eps sum (2 s^12 + s^6) / r, each pair term before the
    cancellation between its repulsive and attractive parts."""
    import torch

    n = pos64.shape[0]
    dev = pos64.device
    gx, gy, gz = g.dim[0], g.dim[1], g.dim[2]
    tgt = torch.linspace(0, n - 1, min(sample, n), device=dev).round().long().unique()
    c = cell[tgt].long()
    cx, cy, cz = c % gx, (c // gx) % gy, c // (gx * gy)
    starts, lens = [], []
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            z, y = cz + dz, cy + dy
            ok = (z >= 0) & (z < gz) & (y >= 0) & (y < gy)
            rb = (z.clamp(0, gz - 1) * gy + y.clamp(0, gy - 1)) * gx
            s = offsets[(rb + (cx - 1).clamp(min=0))].long()
            e = offsets[(rb + (cx + 1).clamp(max=gx - 1) + 1)].long()
            starts.append(torch.where(ok, s, torch.zeros_like(s)))
            lens.append(torch.where(ok, e - s, torch.zeros_like(s)))
    starts, lens = torch.stack(starts, 1).reshape(-1), torch.stack(lens, 1).reshape(-1)
    owner = torch.repeat_interleave(torch.arange(len(tgt), device=dev).repeat_interleave(9), lens)
    first = torch.cumsum(lens, 0) - lens
    j = torch.repeat_interleave(starts - first, lens) + torch.arange(int(lens.sum()), device=dev)
    i = tgt[owner]
    d = pos64[j] - pos64[i]
    r2 = (d * d).sum(1)
    keep = (j != i) & (r2 < float(rc) ** 2)
    d, r2, own = d[keep], r2[keep], owner[keep]
    s2 = float(sigma) ** 2 / r2
    s6 = s2 ** 3
    s12 = s6 * s6
    m = len(tgt)
    e = torch.zeros(m, dtype=torch.float64, device=dev).index_add_(0, own, 4 * eps * (s12 - s6))
    es = torch.zeros(m, dtype=torch.float64, device=dev).index_add_(0, own, 4 * eps * (s12 + s6))
    fmag = 24 * eps * (2 * s12 - s6) / r2
    f = torch.zeros((m, 3), dtype=torch.float64, device=dev).index_add_(0, own, -fmag[:, None] * d)
    fs = torch.zeros(m, dtype=torch.float64, device=dev).index_add_(0, own, 24 * eps * (2 * s12 + s6) / r2.sqrt())
    return tgt, e, f, es, fs


def error_stats(tgt, e64, f64, es, fs, energy, force):
    """Errors of float outputs (sorted order) against an FP64 sample: norm-wise force error, max and
    p99 relative |F| error, max error over the force scale, relative error of the sample's total
    energy and max energy error over its scale; particles whose FP64 results exceed the float range
    are left out (and counted)."""
    import torch

    f = force.reshape(-1, 3)[tgt].double()
    e = energy[tgt].double()
    ok = (f64.abs() < 1e38).all(1) & (e64.abs() < 1e38) & (fs < 1e38) & (es < 1e38)
    df = (f - f64)[ok].norm(dim=1)
    fn = f64[ok].norm(dim=1)
    rel = df[fn > 0] / fn[fn > 0]
    q = lambda t: float(t.max()) if t.numel() else 0.0
    return {"targets": int(len(tgt)), "excluded": int((~ok).sum()),
            "force_normwise": float((f - f64)[ok].norm() / f64[ok].norm().clamp(min=1e-300)),
            "force_max_rel": q(rel), "force_p99_rel": float(torch.quantile(rel, 0.99)) if rel.numel() else 0.0,
            "force_max_over_scale": q(df[fs[ok] > 0] / fs[ok][fs[ok] > 0]),
            "energy_sample_total_rel": float(abs(e[ok].sum() - e64[ok].sum()) / e64[ok].sum().abs().clamp(min=1e-300)),
            "energy_max_over_scale": q((e - e64)[ok].abs()[es[ok] > 0] / es[ok][es[ok] > 0])}


def time_events(fn, reps, flush=None):
    """Mean device time (ms) of fn() over reps calls, L2 flushed before each (outside the events)."""
    import torch

    fn()
    torch.cuda.synchronize()
    ts = []
    for i in range(reps):
        if flush is not None:
            flush.fill_(i & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        torch.cuda.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.mean(ts))


def single_workload(ctx, cfg, seed, flush, peak_tflops, reps=10):
    """Plain FP32 step on one more single-system workload: stage times, pairs/s,
    FP32 roofline of the pair kernel and, for the sphere shell, the HBM figure of
    the whole step (76 B per particle + 16 B per cell, algorithmic)."""
    import torch
    import ljcell

    n, rc = cfg["n"], cfg["rc"]
    g = ljcell.grid_from_box(cfg["lo"], cfg["hi"], rc)
    p = ljcell.params(rc)
    if cfg["dist"] == "uniform":
        soa, _ = ctx.generate_uniform(seed, n, cfg["lo"], cfg["hi"])
    else:
        soa, _ = ctx.generate_sphere(seed, n, (0.5, 0.5, 0.5), 1.0)
    b = ctx.alloc_binned(g, n, ljcell.ORDER_X)
    e, f, tot = ctx.alloc_outputs(n)
    cand = torch.zeros(1, dtype=torch.int64, device=ctx.device)
    t_bin = time_events(lambda: ctx.bin(g, soa["x"], soa["y"], soa["z"], order=ljcell.ORDER_X, out=b), reps, flush)
    saved = ctx.get_tuning()["pair_kernel"]
    kern, _ = ctx.autotune_compute(g, p, b)
    t_pair = time_events(lambda: ctx.compute(g, p, b, e, f, tot), reps, flush)
    ctx.set_tuning(saved)
    ctx.count_candidates(g, b.offsets, cand)
    ctx.sync()
    pairs = ljcell.totals_from_tensor(tot)["pairs"]
    c_ref = int(cand.item())
    step = t_bin + t_pair
    ach = (FLOP_CANDIDATE * c_ref + FLOP_INTERACTING * pairs) / (t_pair * 1e-3) / 1e12
    out = {"workload": cfg["workload"], "n": n, "cells": g.ncells, "ms_per_step": step,
           "stage_ms": {"bin": t_bin, "pair": t_pair}, "pairs_per_step": pairs, "pairs_per_s": pairs / (step * 1e-3),
           "particles_per_s": n / (step * 1e-3),
           "pair_kernel_fp32": {"kernel": kernel_name(kern), "achieved_tflops": ach, "frac": ach / peak_tflops}}
    if cfg["dist"] == "sphere":
        algo_bytes = 76 * n + 16 * g.ncells
        out["step_hbm"] = {"algorithmic_bytes": algo_bytes, "achieved_gbs": algo_bytes / (step * 1e-3) / 1e9,
                           "peak_gbs": hbm_peak(), "frac": algo_bytes / (step * 1e-3) / 1e9 / hbm_peak()}
    del soa, b, e, f, tot
    torch.cuda.empty_cache()
    return out


def hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(path))["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        return 6650.0


def batched_workload(ctx, flush, reps=10):
    """512 uneven systems (log-uniform N in [1e3, 2e5], 25% sphere shells): the
    batched step replayed as one CUDA graph after autotuning, against the same
    results from 512 per-system plain launches."""
    import torch
    import ljcell

    w = ljcell.batch_workload()
    b = ljcell.Batch(ctx, w)
    x, y, z = b.generate()
    e, f, idx, tot = b.alloc_outputs()
    ctx.sync()
    t0 = time.perf_counter()
    cfg, _ = b.autotune(x, y, z)
    tune_s = time.perf_counter() - t0
    t_graph = time_events(lambda: b.run(x, y, z, e, f, None, tot, mode="graph"), reps, flush)
    pairs = sum(t["pairs"] for t in ljcell.totals_from_array(tot))
    t_sep = time_events(lambda: b.run(x, y, z, e, f, None, tot, mode="separate"), max(3, reps // 3), flush)
    pairs_sep = sum(t["pairs"] for t in ljcell.totals_from_array(tot))
    ctx.sync()
    out = {"workload": "512 systems, N log-uniform [1e3, 2e5], 25% sphere shells, 20-200 neighbours",
           "particles": b.ntotal, "pairs_per_step": pairs, "autotuned": cfg, "autotune_s": tune_s,
           "ms_per_step_batched_graph": t_graph, "ms_per_step_per_system_launches": t_sep,
           "speedup_vs_per_system": t_sep / t_graph, "pairs_per_s": pairs / (t_graph * 1e-3),
           "pairs_match": pairs == pairs_sep}
    b.close()
    del x, y, z, e, f, idx, tot
    torch.cuda.empty_cache()
    return out


def mixed_workload(ctx, cfg, seed, flush, reps=10):
    """Mixed-precision form beside the plain FP32 form on the same binned
    particles: device times of the pair stage (records packed once per step,
    counted)."""
    import torch
    import ljcell

    n, rc = cfg["n"], cfg["rc"]
    g = ljcell.grid_from_box(cfg["lo"], cfg["hi"], rc)
    p = ljcell.params(rc)
    soa, _ = ctx.generate_uniform(seed, n, cfg["lo"], cfg["hi"])
    b = ctx.bin(g, soa["x"], soa["y"], soa["z"], order=ljcell.ORDER_X)
    e, f, tot = ctx.alloc_outputs(n)
    rec = ctx.pack_mixed(g, b)
    saved = ctx.get_tuning()["pair_kernel"]
    kern, _ = ctx.autotune_compute(g, p, b)
    t_plain = time_events(lambda: ctx.compute(g, p, b, e, f, tot), reps, flush)
    plain_pairs = ljcell.totals_from_tensor(tot)["pairs"]
    ctx.set_tuning(saved)

    def mixed_step():
        ctx.pack_mixed(g, b, rec)
        ctx.compute_mixed(g, p, b, rec, e, f, tot)

    t_pack = time_events(lambda: ctx.pack_mixed(g, b, rec), reps, flush)
    mixed_ms = {}
    for mk in (0, 1, 2):   # the mixed walks (two-target row passes, flat with two window layouts); keep the fastest
        ctx.set_tuning(mk)
        mixed_ms[mk] = time_events(mixed_step, reps, flush)
    mk = min(mixed_ms, key=mixed_ms.get)
    ctx.set_tuning(mk)
    t_mixed = time_events(mixed_step, reps, flush)
    ctx.set_tuning(saved)
    ctx.sync()
    mixed_pairs = ljcell.totals_from_tensor(tot)["pairs"]
    # errors of the mixed outputs against FP64 on the caller's positions and on the stored positions
    # (FP32 x; y, z = origin + (cell + binary16 offset) * width), and of the plain outputs
    caller = b.xyzi[:n, :3].double()
    c = b.cell[:n].long()
    gx, gy = g.dim[0], g.dim[1]
    uyz = rec[:n, 1].contiguous().view(torch.int32)
    uy = (uyz & 0xFFFF).to(torch.int16).view(torch.float16).double()
    uz = ((uyz >> 16) & 0xFFFF).to(torch.int16).view(torch.float16).double()
    w = float(g.width)
    stored = torch.stack([rec[:n, 0].double(), g.origin[1] + (((c // gx) % gy).double() + uy) * w,
                          g.origin[2] + ((c // (gx * gy)).double() + uz) * w], 1)
    ref_caller = fp64_sample(g, b.offsets, b.cell[:n], caller, rc, p.sigma)
    ref_stored = fp64_sample(g, b.offsets, b.cell[:n], stored, rc, p.sigma)
    err_mixed_caller = error_stats(*ref_caller, e[:n], f[:n])
    err_mixed_stored = error_stats(*ref_stored, e[:n], f[:n])
    ctx.set_tuning(kern)
    ctx.compute(g, p, b, e, f, tot)
    ctx.set_tuning(saved)
    err_plain = error_stats(*ref_caller, e[:n], f[:n])
    out = {"workload": cfg["workload"] + ", mixed precision", "ms_pair_plain": t_plain,
           "plain_kernel": kernel_name(kern), "ms_pack_mixed": t_pack, "ms_pack_and_pair_mixed": t_mixed,
           "mixed_kernel": {0: "k_pair_mixed_pass2", 1: "k_pair_mixed", 2: "k_pair_mixed_reg"}[mk],
           "speedup_vs_plain": t_plain / t_mixed, "pairs_plain": plain_pairs, "pairs_mixed": mixed_pairs,
           "errors_vs_fp64": {
               "mixed_vs_caller_positions": err_mixed_caller,
               "mixed_vs_stored_positions": err_mixed_stored,
               "plain_vs_caller_positions": err_plain,
               "reference": "FP64 (torch, on the GPU) on a stratified sample of targets, every particle of the "
                            "27-cell stencil; stored positions: FP32 x, y and z rebuilt from the binary16 offsets",
               "bound_met": "1e-5 relative force error holds against the stored positions only: binary16 offsets "
                            "move y, z by up to 2^-12 cell widths, and r^-13 forces turn that into percent-level "
                            "errors against the caller's positions"}}
    del soa, b, e, f, tot, rec, caller, stored, ref_caller, ref_stored
    torch.cuda.empty_cache()
    return out


def half_workload(ctx, cfg, seed, flush, peak_tflops, reps=5):
    """Half-shell evaluation (lj_compute_half: each unordered pair once, reactions applied to the
    partner, deterministic colour phases) beside the full-shell default on the same binned particles."""
    import torch
    import ljcell

    n, rc = cfg["n"], cfg["rc"]
    g = ljcell.grid_from_box(cfg["lo"], cfg["hi"], rc)
    p = ljcell.params(rc)
    soa, _ = ctx.generate_uniform(seed, n, cfg["lo"], cfg["hi"])
    b = ctx.bin(g, soa["x"], soa["y"], soa["z"], order=ljcell.ORDER_X)
    e, f, tot = ctx.alloc_outputs(n)
    cand = torch.zeros(1, dtype=torch.int64, device=ctx.device)
    ctx.count_candidates(g, b.offsets, cand)
    saved = ctx.get_tuning()["pair_kernel"]
    kern, _ = ctx.autotune_compute(g, p, b)
    t_full = time_events(lambda: ctx.compute(g, p, b, e, f, tot), reps, flush)
    pairs_full = ljcell.totals_from_tensor(tot)["pairs"]
    ctx.set_tuning(saved)
    t_half = time_events(lambda: ctx.compute_half(g, p, b, e, f, tot), reps, flush)
    ctx.sync()
    pairs_half = ljcell.totals_from_tensor(tot)["pairs"]
    c_ref = int(cand.item())
    ach = (FLOP_CANDIDATE * c_ref + FLOP_INTERACTING * pairs_half) / (t_half * 1e-3) / 1e12
    out = {"workload": cfg["workload"] + ", half shell", "ms_pair_half": t_half, "ms_pair_full": t_full,
           "full_kernel": kernel_name(kern), "speedup_vs_full": t_full / t_half,
           "pairs_half": pairs_half, "pairs_full": pairs_full, "pairs_match": pairs_half == pairs_full,
           "fp32_frac_half": ach / peak_tflops}
    del soa, b, e, f, tot, cand
    torch.cuda.empty_cache()
    return out


def slab_workload(ctx, cfg, seed, flush, worlds=(2, 4, 8), reps=5):
    """Slab decomposition of one system (ljcell.slab) with its W ranks emulated in turn on this
    GPU: each rank's step (halo layers picked from its own particles, binning of own + halo on the
    global grid, lj_compute_range over its own sorted range) timed on the device.  The exchange
    itself is an in-memory hand-off here; the bytes a rank would receive over NVLink are reported
    beside it.  Against the single-domain step (bin + compute) of the same system."""
    import torch
    import ljcell
    from ljcell import slab

    n, rc = cfg["n"], cfg["rc"]
    g = ljcell.grid_from_box(cfg["lo"], cfg["hi"], rc)
    p = ljcell.params(rc)
    soa, _ = ctx.generate_uniform(seed, n, cfg["lo"], cfg["hi"])
    xyz = torch.stack([soa["x"], soa["y"], soa["z"]], 1).contiguous()
    del soa
    x, y, z = (xyz[:, k].contiguous() for k in range(3))
    b = ctx.alloc_binned(g, n, ljcell.ORDER_X)
    e, f, tot = ctx.alloc_outputs(n)

    def single():
        ctx.bin(g, x, y, z, order=ljcell.ORDER_X, out=b)
        ctx.compute(g, p, b, e, f, tot)

    t_single = time_events(single, reps, flush)
    ctx.sync()
    pairs_single = ljcell.totals_from_tensor(tot)["pairs"]
    del x, y, z, b, e, f, tot
    torch.cuda.empty_cache()
    out = {"workload": cfg["workload"] + ", slab ranks emulated on one GPU", "ms_single_domain": t_single,
           "pairs_single": pairs_single, "ranks": {}}
    for w in worlds:
        doms = [slab.SlabDomain.of(g, r, w) for r in range(w)]
        owns = [d.own(xyz) for d in doms]
        halos = [d.halo_out(o) for d, o in zip(doms, owns)]
        empty = xyz[:0]
        ms, pairs, recv = [], 0, []
        for r, d in enumerate(doms):
            below = halos[r - 1][1] if r > 0 else empty
            above = halos[r + 1][0] if r < w - 1 else empty
            res = []

            def rank_step(r=r, d=d, a=below, c=above):
                res[:] = [slab.step(ctx, g, p, d, owns[r], exchange=lambda dom, dn, up: (a, c))]

            ms.append(time_events(rank_step, reps, flush))
            ctx.sync()
            pairs += ljcell.totals_from_tensor(res[0].totals)["pairs"]
            recv.append(12 * res[0].halo)
            del res
        out["ranks"][str(w)] = {"max_rank_ms": max(ms), "mean_rank_ms": float(np.mean(ms)),
                                "pairs_match": pairs == pairs_single,
                                "single_over_max_rank": t_single / max(ms),
                                "halo_bytes_in_max": max(recv),
                                "halo_us_at_770_gbs": max(recv) / 770e9 * 1e6}
        del doms, owns, halos
        torch.cuda.empty_cache()
    del xyz
    torch.cuda.empty_cache()
    return out


def verlet_workload(ctx, flush, side=215, reps=10, seed=5):
    """Time stepping (lj_step_verlet: half kick and drift in the sorted order, rebinning from the
    previous order, the pair stage, closing half kick) on a jittered cubic lattice of side^3 particles
    (about 10M) with sigma = spacing / 1.12 and r_c = 2.5 sigma, dt = 2e-4: device time per step
    beside a step that bins the same particles from a shuffled input order."""
    import torch
    import ljcell

    rng = np.random.default_rng(seed)
    a = 1.0 / side
    gl = (np.arange(side) + 0.5) * a
    X, Y, Z = np.meshgrid(gl, gl, gl, indexing="ij")
    pts = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    pts += rng.uniform(-0.05 * a, 0.05 * a, pts.shape)
    pts = pts[rng.permutation(len(pts))].astype(np.float32)
    n = len(pts)
    sigma = a / 1.12
    rc = 2.5 * sigma
    g = ljcell.grid_from_box((0, 0, 0), (1, 1, 1), rc)
    p = ljcell.params(rc, sigma=sigma)
    d = [torch.from_numpy(np.ascontiguousarray(pts[:, k])).to(ctx.device) for k in range(3)]
    b = ctx.bin(g, *d, order=ljcell.ORDER_X)
    e, f, tot = ctx.alloc_outputs(n)
    t_random = time_events(lambda: (ctx.bin(g, *d, order=ljcell.ORDER_X, out=b), ctx.compute(g, p, b, e, f, tot)),
                           reps, flush)
    vel = torch.from_numpy((rng.standard_normal((n, 3)) * 0.5).astype(np.float32)).to(ctx.device)
    ctx.bin(g, *d, order=ljcell.ORDER_X, out=b)
    ctx.compute(g, p, b, e, f, tot)
    t_step = time_events(lambda: ctx.step_verlet(g, p, b, vel, f, 2e-4, 1.0, e, tot), reps, flush)
    ctx.sync()
    pairs = ljcell.totals_from_tensor(tot)["pairs"]
    out = {"workload": f"jittered lattice {n} ({side}^3), rc={rc:.5f}, sigma=spacing/1.12, dt=2e-4",
           "ms_per_verlet_step": t_step, "pairs_per_step": pairs, "pairs_per_s": pairs / (t_step * 1e-3),
           "ms_bin_and_compute_from_shuffled_order": t_random}
    del d, b, e, f, tot, vel
    torch.cuda.empty_cache()
    return out


def run_extras(ctx, dev, flush, peak_tflops):
    out = {}
    out["verlet_lattice10M"] = verlet_workload(ctx, flush)
    out["slab_c2"] = slab_workload(ctx, CONFIGS["c2"], 1234, flush)
    out["half_shell_c2"] = half_workload(ctx, CONFIGS["c2"], 1234, flush, peak_tflops)
    out["half_shell_c4"] = half_workload(ctx, CONFIGS["c4"], 1234, flush, peak_tflops)
    out["mixed_c4"] = mixed_workload(ctx, CONFIGS["c4"], 1234, flush)
    out["batched_c5"] = batched_workload(ctx, flush)
    out["shell_c3"] = single_workload(ctx, CONFIGS["c3"], 1234, flush, peak_tflops)
    out["dense_c4"] = single_workload(ctx, CONFIGS["c4"], 1234, flush, peak_tflops)
    return out


def run_e2e(ctx, g, p, x, y, z, n, K, ws, dev, total_pairs, pairs):
    """Same metric through the host-buffer entry: pinned host positions in,
    energy and force out every step, copies inside the timed region; steps back
    to back through lj_simulate_host_inorder_async() (results in the caller's
    order), with lj_simulate_host_async() (sorted order + index) and one
    lj_simulate_host() call timed beside them."""
    import torch

    hx, hy, hz = (torch.empty(n, dtype=torch.float32, pin_memory=True) for _ in range(3))
    hx.copy_(x)
    hy.copy_(y)
    hz.copy_(z)
    he = torch.empty(n, dtype=torch.float32, pin_memory=True)
    hf = torch.empty((n, 3), dtype=torch.float32, pin_memory=True)
    hidx = torch.empty(n, dtype=torch.int32, pin_memory=True)
    hxn, hyn, hzn, hen, hfn, hin = (t.numpy() for t in (hx, hy, hz, he, hf, hidx))
    for _ in range(2):
        ctx.simulate_host(g, p, hxn, hyn, hzn, hen, hfn, hin)
    steps = 30   # fixed: the pipelined steps need a run long enough that filling and draining it do not count
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(steps):
        tt = ctx.simulate_host(g, p, hxn, hyn, hzn, hen, hfn, hin)
    one_s = allreduce_max((time.perf_counter() - t0) / steps, ws, dev)
    if tt.pairs != pairs:
        raise RuntimeError(f"end-to-end pair count {tt.pairs} differs from the device path {pairs}")
    # steps back to back through lj_simulate_host_async: step k + 1's upload overlaps step k's download
    for _ in range(2):
        ctx.simulate_host_async(g, p, hxn, hyn, hzn, hen, hfn, hin)
    ctx.simulate_host_wait()
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    tots = [ctx.simulate_host_async(g, p, hxn, hyn, hzn, hen, hfn, hin) for _ in range(steps)]
    ctx.simulate_host_wait()
    sorted_s = allreduce_max((time.perf_counter() - t0) / steps, ws, dev)
    if any(t.pairs != pairs for t in tots):
        raise RuntimeError("pipelined end-to-end pair count differs from the device path")
    # the same steps with energy and force returned in the caller's order (16 B per particle down, no index)
    for _ in range(2):
        ctx.simulate_host_inorder_async(g, p, hxn, hyn, hzn, hen, hfn)
    ctx.simulate_host_wait()
    if ws > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    tots = [ctx.simulate_host_inorder_async(g, p, hxn, hyn, hzn, hen, hfn) for _ in range(steps)]
    ctx.simulate_host_wait()
    e2e_s = allreduce_max((time.perf_counter() - t0) / steps, ws, dev)
    if any(t.pairs != pairs for t in tots):
        raise RuntimeError("input-order end-to-end pair count differs from the device path")
    return {"value": total_pairs / e2e_s, "unit": "pairs/s", "h2d_bytes_per_step": 12 * n,
            "d2h_bytes_per_step": 16 * n + 32, "ms_per_step": e2e_s * 1e3, "steps": steps,
            "api": "lj_simulate_host_inorder_async, steps back to back (one lj_simulate_host_wait at the end): "
                   "energy and force in the caller's order",
            "ms_per_step_sorted_order": sorted_s * 1e3,
            "sorted_order_api": "lj_simulate_host_async (sorted order + index, 20 B per particle down)",
            "ms_per_step_one_call": one_s * 1e3}


def read_traffic(kernel, workload):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(path):
        return None
    for ln in open(path):
        parts = [s.strip() for s in ln.split("|")]
        if len(parts) >= 3 and parts[0] == kernel and parts[1] == workload:
            try:
                return float(parts[2])
            except ValueError:
                return None
    return None


def reference_gpu(cfg, seed):
    """The reference's own kernels (cudaLJ.cu built from source for sm_100a into
    oracle/_ref) on the same seeded positions, reference law and stencil: stage
    times and candidate pairs/s of its pair kernel.  Reference arm only."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ljoracle as O

    if not O.ref_available() or cfg["dist"] != "uniform" or tuple(cfg["lo"]) != (0, 0, 0):
        return None
    box = float(cfg["hi"][0])
    w = np.float32(cfg["rc"])
    G = int(np.float32(box) / w)
    below = np.nextafter(np.float32(box), np.float32(0))
    while np.float32(below) / w >= np.float32(G):   # the reference indexes int(x / w) without clamping
        below = np.nextafter(below, np.float32(0))
    x, y, z = (np.minimum(a, below).astype(np.float32) for a in O.generate_uniform(seed, cfg["n"], cfg["lo"],
                                                                                      cfg["hi"]))
    r = O.ref_run(x, y, z, box, cfg["rc"], reps=3)
    ms = r.stage_ms
    return {"what": "reference cudaLJ.cu kernels built from source for sm_100a, same seeded positions, "
                    "reference law (ComputeParticleInterationsParPartNoLoop)",
            "candidate_pairs": r.nbinter, "pair_kernel_ms": float(ms[5]), "binning_ms": float(ms[6]),
            "scan_ms": float(ms[1]), "candidate_pairs_per_s": r.nbinter / (float(ms[5]) * 1e-3)}


def run_slab(args, cfg):
    """One system split over the ranks in slabs of z layers (ljcell.slab): each rank keeps its own
    particles, and a step is the halo exchange with its neighbours (NCCL point-to-point), the binning
    of own + halo particles and the pair stage over its own sorted range.  Every rank generates the
    same system (one seed) and keeps its layers.  The step time is the median over the timed steps
    of each rank's device time, the maximum over ranks; value = the whole system's interacting pairs
    over it (strong scaling)."""
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
    init_dist("nccl" if ws > 1 else "gloo")
    import ljcell
    from ljcell import slab

    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.current_stream()
    ctx = ljcell.Context(dev.index, stream)
    n, rc = cfg["n"], cfg["rc"]
    g = ljcell.grid_from_box(cfg["lo"], cfg["hi"], rc)
    p = ljcell.params(rc)
    if cfg["dist"] == "uniform":
        soa, _ = ctx.generate_uniform(args.seed, n, cfg["lo"], cfg["hi"])
    else:
        soa, _ = ctx.generate_sphere(args.seed, n, (0.5, 0.5, 0.5), 1.0)
    xyz = torch.stack([soa["x"], soa["y"], soa["z"]], 1).contiguous()
    del soa
    dom = slab.SlabDomain.of(g, rank, ws)
    own = dom.own(xyz)
    del xyz
    torch.cuda.empty_cache()
    if ws > 1:
        torch.distributed.barrier()
    res = None
    for _ in range(max(args.warmup, 3)):
        res = slab.step(ctx, g, p, dom, own)
    torch.cuda.synchronize()
    K = args.steps
    times = []
    with ClockSampler(dev.index) as clk:
        for _ in range(K):
            if ws > 1:
                torch.distributed.barrier()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            res = slab.step(ctx, g, p, dom, own)
            b.record(stream)
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b))
    ctx.sync()
    t_max = allreduce_max(float(np.median(times)), ws, dev)
    tot = slab.allreduce_totals(res.totals) if ws > 1 else ljcell.totals_from_tensor(res.totals)
    halo = allreduce_max(float(res.halo), ws, dev)
    if rank == 0:
        clocks = clk.summary()
        line = {"metric": METRIC, "value": tot["pairs"] / (t_max * 1e-3), "unit": "pairs/s", "n_gpus": ws,
                "steps": K, "warmup": args.warmup, "ms_per_step": t_max, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded drand48, device generated)",
                "config": {"workload": cfg["workload"], "n_total": n, "cutoff": rc, "cells": g.ncells,
                           "parallelism": f"slab x{ws} (z layers, one-layer halo, NCCL point-to-point)",
                           "l2": "not flushed (each rank's step reads its own and halo particles)"},
                "pairs_per_step": tot["pairs"], "energy": tot["energy"], "max_halo_particles": int(halo),
                "e2e": None, "gpu_launches": None,
                "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")}}
        print(json.dumps(line), flush=True)
    ctx.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def main():
    args = parse()
    cfg = workload(args)
    if args.impl == "reference":
        return run_reference(args, cfg)
    if args.decomp == "slab":
        return run_slab(args, cfg)
    return run_ours(args, cfg)


if __name__ == "__main__":
    sys.exit(main())
