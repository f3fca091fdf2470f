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
  issue_roofline: the bound that binds (state stays in shared memory): warp
          instructions per launch from the committed ncu summary over the live
          launch time, against 4 issue slots per SM per cycle at the sampled clock.
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


def _profile_value(key):
    """A per-launch figure of the SA kernel (`key: value` line) from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "sa_fast_c2.md")
    try:
        txt = open(path).read()
        m = re.search(key + r":\s*([0-9.eE+]+)", txt)
        return float(m.group(1)) if m else None
    except OSError:
        return None


def _profile_traffic():
    """dram bytes per launch of the SA kernel from the committed ncu summary, if present."""
    return _profile_value("traffic_bytes_per_launch")


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
    torch.cuda.set_device(local)  # before the process group, so NCCL binds this rank's GPU
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
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
    # a dedicated stream: its handle is never 0, so the library launches on it
    # and the CUDA events below time exactly those launches
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
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
    # the reported quality of an anneal: best energy and the share of restarts reaching it
    frac_best = float((energies <= e_min + 1e-4 * max(1.0, abs(e_min))).float().mean().item())
    # time to target with 99 % confidence, target = this run's best energy: one anneal
    # of all restarts succeeds with P = 1 - (1 - frac)^restarts
    p_anneal = 1.0 - (1.0 - frac_best) ** N_REPLICAS

    # end-to-end through the C ABI with host buffers
    reff = 0
    t_e2e = []
    # host buffers of the end-to-end call in pinned memory: the schedule in, energies and states out
    betas_pin = torch.from_numpy(betas_h).pin_memory().numpy()
    e_pin = torch.empty(N_REPLICAS, dtype=torch.float32).pin_memory().numpy()
    packed_pin = torch.empty((N_REPLICAS, (N_SPINS + 7) // 8), dtype=torch.uint8).pin_memory().numpy()
    for k in range(max(1, min(args.steps, 5)) + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e_h, packed = tb.sa_run(dinst, betas_pin, N_REPLICAS, 1, seed0 + 10 ** 6 + k, tb.MODE_FAST,
                                out=(e_pin, packed_pin))
        t_e2e.append(time.perf_counter() - t0)
        reff = len(e_h)
    e2e_s = float(np.median(t_e2e[1:]))
    e2e_t = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_value = FLIPS_PER_STEP * world / float(e2e_t.item())
    h2d = betas_pin.nbytes  # the instance is resident; the schedule goes in every step
    d2h = e_pin[:reff].nbytes + packed_pin[:reff].nbytes  # energies and AnnealState bytes out

    out = None
    if rank == 0:
        peak, kind = _peaks()
        per_launch_ms = float(np.mean(times))
        achieved = BYTES_PER_FLIP * FLIPS_PER_STEP / (per_launch_ms / 1e3) / 1e9
        traffic = _profile_traffic()
        clocks = clk.summary()
        # The kernel keeps its state on chip, so instruction issue binds, not HBM:
        # warp instructions per launch (ncu, same workload and tile) over the live
        # launch time, against 4 issue slots per SM per cycle at the sampled clock.
        inst = _profile_value("warp_instructions_per_launch")
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
        issue = None
        if inst and mhz:
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            ach, pk = inst / (per_launch_ms / 1e3), sms * 4 * mhz * 1e6
            issue = {"achieved": ach, "peak": pk, "unit": "warp instructions/s", "frac": ach / pk,
                     "instructions_per_launch": inst, "clock_mhz": mhz,
                     "source": "profiles/sa_fast_c2.md (smsp__inst_executed.sum of one launch)"}
        out = {"metric": METRIC, "value": value, "unit": "flips/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
               "config": dict(CONFIG, parallelism=f"replicas x{world}" if world > 1 else "1 GPU"),
               "e2e": {"value": e2e_value, "unit": "flips/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
               "gpu_launches": int(launches),
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{kind} burst",
                            "bytes_per_flip": BYTES_PER_FLIP},
               "issue_roofline": issue,
               "clocks": clocks, "best_energy": e_min, "restarts_at_best": frac_best,
               "tts99_s": per_launch_ms / 1e3 * (1.0 if p_anneal >= 0.99 else
                                                math.log(0.01) / math.log(1.0 - p_anneal))}
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


# ------------------------------------------------------- other workloads ----
# The remaining benchmark configurations, run with --workload; each prints one
# JSON line.  They are measured separately from the headline line above.
def _lattice_params(tb, nt, sweeps, sample=None, states=None, level=0, threads=8):
    b = tb.geometric_betas(0.2, 5.0, nt)
    lo = int(np.argmax(b >= np.float32(1.0))) if np.any(b >= np.float32(1.0)) else nt - 1
    return tb.PtParams(sweeps, b, lo, 0.5, True, 2, threads, sample, states, level)


def _time_run(tb, dinst, p, seed):
    import torch
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = tb.PtRun(dinst, p, seed).run().sync()
    torch.cuda.synchronize()
    return time.perf_counter() - t0, r


def _time_to_target(tb, dinst, p, seed, target, t_sweep):
    """Time to target: the ground-state log is kept only after the warm-up
    (src/pt.rs:542-583), so a second run with warm-up 0 records the running
    minimum from the first sweep; returns the first sweep whose minimum reaches
    `target` (or None) and that many sweeps at the measured time per sweep."""
    q = tb.PtParams(p.num_sweeps, p.betas, p.lo_beta_idx, 0.0, p.icm, p.num_replica_chains, p.threads,
                    p.sample, p.sample_states, p.sample_limiting)
    steps, en, _ = tb.PtRun(dinst, q, seed).run().sync().gs()
    hit = [int(st) for st, e in zip(steps, en) if e <= target + 1e-4 * max(1.0, abs(target))]
    if not hit:
        return None, None
    return hit[0], (hit[0] + 1) * t_sweep


def workload_pt_c1(args, tb, gi, gpu):
    """2-D EA +-J, L=16, nt=32, 2 chains, ICM, 2000 sweeps, sample 32 / states 32 / limiting 2."""
    text = gi.lattice(16, 2, "pm", 0)
    d = gpu.upload(tb.HostInstance.parse(text))
    p = _lattice_params(tb, 32, 2000, 32, 32, 2, threads=1)
    flips = 256 * 32 * 2 * 2000
    _time_run(tb, d, p, 1)
    t_fast, r = _time_run(tb, d, p, 2)
    t0 = time.perf_counter()
    rr = tb.PtRun(d, p, 3, tb.MODE_REF).run().sync()
    t_ref = time.perf_counter() - t0
    best = float(r.gs()[1][-1])
    out = {"workload": "pt_c1", "flips": flips, "fast_flips_per_s": flips / t_fast, "fast_s": t_fast,
           "ref_mode_flips_per_s": flips / t_ref, "ref_mode_s": t_ref,
           "best_energy_fast": best, "best_energy_ref_mode": float(rr.gs()[1][-1])}
    target = best
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        inst = po.Instance.from_text(text)
        runs = {}
        for threads in (1, os.cpu_count() or 1):  # the reference's run (threads: 1) and run_parallel on all cores
            t0 = time.perf_counter()
            orc = po.PtRun(inst, p.betas, 2000, 0.5, p.lo_beta_idx, True, 2, threads, sample=32, sample_states=32,
                           sample_limiting=2, seed=3)
            orc.run(nthreads=threads)
            runs[threads] = (time.perf_counter() - t0, float(orc.gs()[-1][1]))
        t1, e1 = runs[1]
        tn, en = runs[max(runs)]
        out.update(cpu_flips_per_s=flips / t1, cpu_s=t1, cpu_kind="oracle, threads: 1 (serial reference loop)",
                   cpu_best_energy=e1, cpu_allcore_flips_per_s=flips / tn, cpu_allcore_threads=max(runs),
                   cpu_allcore_best_energy=en)
        target = min(e1, en, best)
    first, tts = _time_to_target(tb, d, p, 2, target, t_fast / 2000)
    out.update(target_energy=target, target_first_sweep=first, time_to_target_s=tts)
    return out


def workload_batch_c3(args, tb, gi, gpu):
    """256 uneven 2-D +-J instances, L in {8..32}, nt in {16,24,32}, 5000 sweeps: batched vs plain."""
    rng = np.random.default_rng(0)
    jobs = []
    for k in range(256):
        L = int(rng.choice([8, 12, 16, 24, 32]))
        nt = int(rng.choice([16, 24, 32]))
        jobs.append((L, nt))
    sweeps = args.c3_sweeps
    dinsts = {}
    batch = tb.Batch(gpu)
    flips = 0
    for k, (L, nt) in enumerate(jobs):
        key = (L, k)
        d = gpu.upload(tb.HostInstance.parse(gi.lattice(L, 2, "pm", 1000 + k)))
        dinsts[key] = d
        batch.add(d, _lattice_params(tb, nt, sweeps), 7 + k)
        flips += L * L * nt * 2 * sweeps
    import torch
    torch.cuda.synchronize()
    l0 = gpu.launches
    t0 = time.perf_counter()
    batch.run()
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    l_batch = gpu.launches - l0
    # plain form (one instance at a time, one launch per sweep phase) on a subset
    os.environ["TAMC_PT_FORM"] = "plain"
    sub = list(range(0, 256, 256 // args.c3_plain)) if args.c3_plain > 0 else []
    f_sub, t_sub = 0, 0.0
    for k in sub:
        L, nt = jobs[k]
        d = dinsts[(L, k)]
        p = _lattice_params(tb, nt, sweeps)
        t, _ = _time_run(tb, d, p, 7 + k)
        t_sub += t
        f_sub += L * L * nt * 2 * sweeps
    del os.environ["TAMC_PT_FORM"]
    plain_rate = f_sub / t_sub if t_sub > 0 else None
    return {"workload": "batch_c3", "instances": 256, "sweeps": sweeps, "flips": flips,
            "batched_flips_per_s": flips / t_batch, "batched_s": t_batch, "batched_launches": int(l_batch),
            "plain_flips_per_s": plain_rate, "plain_sample": f"{len(sub)} of 256 instances",
            "batched_over_plain": (flips / t_batch) / plain_rate if plain_rate else None}


def workload_pt_c4(args, tb, gi, gpu):
    """3-D Gaussian L=16 (N=4096), nt=64, 2 chains, ICM, 20000 sweeps, sampling every 32, suscepts."""
    L = 16
    text = gi.lattice(L, 3, "gauss", 0)
    h = tb.HostInstance.parse(text)
    w = [gi.fourier_weights(L, 3, 0), gi.fourier_weights(L, 3, 1)]
    for row in w:
        h.add_suscept(row)
    d = gpu.upload(h)
    sweeps = args.c4_sweeps
    p = _lattice_params(tb, 64, sweeps, 32, 32, 0, threads=64)
    flips = 4096 * 64 * 2 * sweeps
    _time_run(tb, d, _lattice_params(tb, 64, 64, 32, 32, 0, threads=64), 1)  # autotune + warm-up
    t_gpu, r = _time_run(tb, d, p, 2)
    best = float(r.gs()[1][-1])
    first, tts = _time_to_target(tb, d, p, 2, best, t_gpu / sweeps)
    out = {"workload": "pt_c4", "sweeps": sweeps, "flips": flips, "gpu_flips_per_s": flips / t_gpu, "gpu_s": t_gpu,
           "gpu_best_energy": best, "target_energy": best, "target_first_sweep": first, "time_to_target_s": tts}
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        inst = po.Instance.from_text(text)
        for row in w:
            inst.add_suscept(row)
        k = args.c4_cpu_sweeps
        cores = os.cpu_count() or 1
        orc = po.PtRun(inst, p.betas, k, 0.0, p.lo_beta_idx, True, 2, 64, sample=32, sample_states=32,
                       sample_limiting=0, seed=3)
        t0 = time.perf_counter()
        orc.run(nthreads=cores)
        t_cpu = time.perf_counter() - t0
        cpu_rate = 4096 * 64 * 2 * k / t_cpu
        out.update(cpu_flips_per_s=cpu_rate, cpu_sample=f"oracle run_parallel (threads: 64), first {k} sweeps "
                   f"measured every sweep, {cores} OpenMP threads", cpu_cores=cores,
                   gpu_over_cpu=(flips / t_gpu) / cpu_rate)
    return out


def workload_serve_c5(args, tb, gi, gpu):
    """Poisson stream of QUBO requests, N log-uniform in [64, 8192], PT-ICM 16-32 temps, 1000 sweeps."""
    rng = np.random.default_rng(5)
    nreq = args.c5_requests
    reqs = []
    for k in range(nreq):
        n = int(round(math.exp(rng.uniform(math.log(64), math.log(8192)))))
        nt = int(rng.integers(16, 33))
        reqs.append((n, nt))
    texts = [gi.qubo_er(n, 6.0, 100 + k) for k, (n, _) in enumerate(reqs)]
    hosts = [tb.HostInstance.parse(t, qubo=True) for t in texts]
    rate = args.c5_rate
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq))
    srv = tb.Server(gpu, hbm_budget_bytes=64 << 30, max_active=512, chunk_sweeps=125)
    ids = {}
    t0 = time.perf_counter()
    nxt = 0
    while True:
        now = time.perf_counter() - t0
        while nxt < nreq and arrivals[nxt] <= now:
            n, nt = reqs[nxt]
            b = tb.geometric_betas(0.2, 5.0, nt)
            lo = int(np.argmax(b >= np.float32(1.0)))
            ids[nxt] = srv.submit(hosts[nxt], tb.PtParams(1000, b, lo, 0.5, True, 2, 8), 900 + nxt)
            nxt += 1
        a, q = srv.step()
        if nxt >= nreq and a == 0 and q == 0:
            break
        if a == 0 and q == 0 and nxt < nreq:
            time.sleep(max(0.0, min(0.01, arrivals[nxt] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    lat = np.array([srv.result(ids[k])[3] for k in range(nreq)])
    flips = sum(n * nt * 2 * 1000 for n, nt in reqs)
    return {"workload": "serve_c5", "requests": nreq, "offered_rate_per_s": rate, "wall_s": wall,
            "flips": flips, "aggregate_flips_per_s": flips / wall, "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean())}


def run_workload(args):
    import torch
    import tamc_b200 as tb
    from tamc_b200 import instances as gi
    torch.cuda.set_device(0)
    gpu = tb.Gpu(0)
    fn = {"pt_c1": workload_pt_c1, "batch_c3": workload_batch_c3, "pt_c4": workload_pt_c4,
          "serve_c5": workload_serve_c5}[args.workload]
    with ClockSampler(0) as clk:
        out = fn(args, tb, gi, gpu)
    out["metric"] = "spin-flip attempts/s"
    out["clocks"] = clk.summary()
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--workload", default="sa_c2", choices=["sa_c2", "pt_c1", "batch_c3", "pt_c4", "serve_c5"])
    ap.add_argument("--c3-sweeps", type=int, default=5000)
    ap.add_argument("--c3-plain", type=int, default=16, help="instances of the plain-form comparison (0 skips it)")
    ap.add_argument("--c4-sweeps", type=int, default=20000)
    ap.add_argument("--c4-cpu-sweeps", type=int, default=200)
    ap.add_argument("--c5-requests", type=int, default=1000)
    ap.add_argument("--c5-rate", type=float, default=100.0)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload != "sa_c2":
        return run_workload(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
