"""Benchmark: spin-flip attempts per second of simulated annealing on one B200.

Workload (the configuration the headline metric is quoted on): simulated
annealing of a sparse random Ising problem -- N=2000 spins on a random
3-regular graph, couplings J_ij ~ N(0,1) and biases h_i ~ N(0, 0.1^2) (f32,
seeded synthetic data), a linear beta schedule 0.1 -> 10 over 1000 sweeps and
1024 independent restarts.  One step = one full anneal of all restarts =
2000 * 1024 * 1000 = 2.048e9 flip attempts.

  value : device-resident throughput: instance, schedule and outputs already in
          HBM, kernel time from CUDA events on the launching stream; L2 is
          flushed (a 256 MiB write) between timed steps.
  e2e   : the same anneal through the reference-facing C ABI call with host
          buffers (tamc_gpu_sa_run: host schedule in, host energies and
          bit-packed states out), copies inside the timed region.
  roofline: HBM bound of the per-flip algorithmic bytes (one spin bit read and
          written, plus the CSR row of the site amortised over the restarts
          sharing one pass): B = 2/8 + (4 + 8*3 + 4)/1024 bytes per flip.
  cpu_baseline: the CPU restatement of the reference (oracle/, OpenMP over
          SA partitions as the reference's rayon code), on a bounded sample
          of the same schedule.

`--impl reference` times that CPU implementation on the same workload and
prints the reference arm's line.  Under torchrun (N > 1) every rank anneals
its own 1024 restarts (independent seeds; weak scaling, no collective on the
data path) and the line reports all ranks' flips over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SPINS, DEGREE, N_REPLICAS, N_SWEEPS = 2000, 3, 1024, 1000
BETA0, BETA1 = 0.1, 10.0
FLIPS_PER_STEP = N_SPINS * N_REPLICAS * N_SWEEPS
BYTES_PER_FLIP = 2 / 8 + (4 + 8 * DEGREE + 4) / N_REPLICAS
METRIC = "spin-flip attempts/s (SA, 1 B200)"
CONFIG = {"workload": "SA: N=2000 random 3-regular Ising, J~N(0,1), h~N(0,0.01), linear beta 0.1->10 x 1000 "
                      "sweeps, 1024 restarts", "n": N_SPINS, "degree": DEGREE, "restarts": N_REPLICAS,
          "sweeps": N_SWEEPS, "l2": "flushed between timed steps (256 MiB write)"}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_traffic():
    """dram bytes per launch of the SA kernel from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "sa_fast_c2.md")
    try:
        txt = open(path).read()
        m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", txt)
        return float(m.group(1)) if m else None
    except OSError:
        return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if len(r) > 5 + k and r[5 + k] == "Active"})
        load = sorted(sm)[len(sm) // 2:] if sm else []
        return {"sm_mhz": float(np.median(load)) if load else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_sample(text: str, betas: np.ndarray, budget_s: float = 12.0, threads: int | None = None):
    """Times the oracle (CPU restatement of the reference, all host threads) on a
    bounded, schedule-spread sample of the workload: all 1024 restarts, a
    strided subset of the 1000 betas.  Returns (flips/s, description, cores)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    cores = threads or os.cpu_count() or 1
    inst = po.Instance.from_text(text)
    probe = betas[:: max(1, len(betas) // 4)][:4]
    t0 = time.perf_counter()
    po.sa_run(inst, probe, N_REPLICAS, cores, 1, nthreads=cores)
    per_sweep = (time.perf_counter() - t0) / len(probe)
    k = int(min(len(betas), max(4, budget_s / max(per_sweep, 1e-9))))
    sample = betas[np.linspace(0, len(betas) - 1, k).astype(int)]
    t0 = time.perf_counter()
    po.sa_run(inst, sample, N_REPLICAS, cores, 2, nthreads=cores)
    dt = time.perf_counter() - t0
    flips = N_SPINS * N_REPLICAS * len(sample)
    desc = (f"oracle SA, {N_REPLICAS} restarts in {cores} partitions x {len(sample)} of the 1000 betas "
            f"(evenly spread), {flips:.3g} flips in {dt:.1f} s")
    return flips / dt, desc, cores


def run_reference(args):
    world, rank, _ = _dist()
    if rank != 0:
        return 0
    from tamc_b200 import instances as gi
    text = gi.sa_regular(N_SPINS, DEGREE, 0)
    betas = np.linspace(BETA0, BETA1, N_SWEEPS).astype(np.float32)
    vals = []
    desc, cores = "", 1
    for i in range(args.warmup + args.steps):
        v, desc, cores = cpu_sample(text, betas, budget_s=max(2.0, 60.0 / max(1, args.warmup + args.steps)))
        if i >= args.warmup:
            vals.append(v)
    value = float(np.median(vals))
    line = {"metric": METRIC, "value": value, "unit": "flips/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": FLIPS_PER_STEP / value * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "config": CONFIG,
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "flips/s", "cores": cores, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "flips/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_gpu(args):
    import torch
    import tamc_b200 as tb
    from tamc_b200 import instances as gi

    world, rank, local = _dist()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    gpu = tb.Gpu(local)
    text = gi.sa_regular(N_SPINS, DEGREE, 0)
    inst = tb.HostInstance.parse(text)
    dinst = gpu.upload(inst)
    betas_h = np.linspace(BETA0, BETA1, N_SWEEPS).astype(np.float32)
    betas = torch.from_numpy(betas_h).to(dev)
    energies = torch.empty(N_REPLICAS, dtype=torch.float32, device=dev)
    words = torch.empty(((N_REPLICAS + 31) // 32) * N_SPINS, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    seed0 = 1000 * (rank + 1)

    def step(k):
        tb.sa_run_device(dinst, betas.data_ptr(), N_SWEEPS, N_REPLICAS, seed0 + k, energies.data_ptr(),
                         words.data_ptr(), stream.cuda_stream)

    for k in range(args.warmup):
        step(k)
        flush.fill_(k & 0xFF)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches0 = gpu.launches
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        for k in range(args.steps):
            evs[k][0].record(stream)
            step(args.warmup + k)
            evs[k][1].record(stream)
            flush.fill_((k + 7) & 0xFF)
        torch.cuda.synchronize()
    launches = gpu.launches - launches0
    times = [a.elapsed_time(b) for a, b in evs]
    ms = float(np.sum(times))
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = FLIPS_PER_STEP * args.steps * world / (ms_max / 1e3)
    e_min = float(energies.min().item())

    # end-to-end through the C ABI with host buffers
    reff = 0
    t_e2e = []
    for k in range(max(1, min(args.steps, 5)) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_h, packed = tb.sa_run(dinst, betas_h, N_REPLICAS, 1, seed0 + 10 ** 6 + k, tb.MODE_FAST)
        t_e2e.append(time.perf_counter() - t0)
        reff = len(e_h)
    e2e_s = float(np.median(t_e2e[1:]))
    e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_value = FLIPS_PER_STEP * world / float(e2e_t.item())
    h2d = N_SWEEPS * 4
    d2h = reff * 4 + ((N_REPLICAS + 31) // 32) * N_SPINS * 4

    out = None
    if rank == 0:
        peak, kind = _peaks()
        per_launch_ms = float(np.mean(times))
        achieved = BYTES_PER_FLIP * FLIPS_PER_STEP / (per_launch_ms / 1e3) / 1e9
        traffic = _profile_traffic()
        out = {"metric": METRIC, "value": value, "unit": "flips/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
               "config": dict(CONFIG, parallelism=f"replicas x{world}" if world > 1 else "1 GPU"),
               "e2e": {"value": e2e_value, "unit": "flips/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
               "gpu_launches": int(launches),
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{kind} burst",
                            "bytes_per_flip": BYTES_PER_FLIP},
               "clocks": clk.summary(), "best_energy": e_min}
        if not args.no_cpu and world == 1:
            v, desc, cores = cpu_sample(text, betas_h)
            out["cpu_baseline"] = {"value": v, "unit": "flips/s", "cores": cores, "kind": "port", "sample": desc}
        elif world > 1:
            out["cpu_baseline"] = None
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)
    del gpu
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
