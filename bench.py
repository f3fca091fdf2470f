"""Benchmark: spin-flip attempts per second of batched PT-ICM against the plain
form, on one B200.

Default workload (--workload batch_c3): 256 uneven 2-D +-J spin-glass
instances -- periodic L x L lattices with L drawn uniformly from
{8, 12, 16, 24, 32}, J_ij uniform in {-1, +1} (f32, seeded synthetic data) --
each a PT-ICM run with a geometric beta ladder 0.2 -> 5.0 of 16, 24 or 32
temperatures (drawn uniformly), 2 replica chains, Houdayer moves from
lo_beta = 1.0, 5000 sweeps.  One step = the whole batch run to the end =
sum_j L_j^2 * nt_j * 2 * 5000 flip attempts (about 2.5e10).

  value   : batched form (tamc_gpu_batch_*: all jobs in one persistent kernel
            per chunk of rounds, each chunk a replayed CUDA graph), instances
            resident in HBM; CUDA events on the library's stream around the
            whole run, L2 flushed (256 MiB write) between steps.
  plain_flips_per_s / batched_over_plain : the plain form (one instance at a
            time, one launch per sweep phase) on a fixed systematic sample of
            the same jobs, same seeds, CUDA-event time.
  e2e     : the same batch through the C ABI from host instances: upload every
            instance, create the batch, run, read every job's ground-state
            trajectory and acceptance counts, free; wall clock, with the
            library's own count of host<->device bytes.
  roofline: HBM bound of the per-flip algorithmic bytes, job by job
            B_j = 2/8 + (4 + 8*4 + 4) / (2 nt_j) (one spin bit read and written,
            plus the CSR row of the site amortised over the replicas sharing
            one pass), over the device time of the chunk launches.
  issue_roofline: the bound that applies (the replicas stay in shared memory):
            warp instructions per step from the committed ncu summary over the
            same device time, against 4 issue slots per SM per cycle.
  cpu_baseline: the CPU restatement of the reference (oracle/) on a fixed
            subset of the same jobs at their full 5000 sweeps, one job per host
            thread on all cores, median of 3 runs, in a child process.
  c4      : 3-D L=16 Gaussian PT-ICM (64 temperatures, 20000 sweeps, samples
            every 32) on the GPU, against whole oracle runs of the same method
            with fewer sweeps on all cores (gpu_over_cpu).

`--impl reference` times the CPU restatement on the same jobs and prints the
reference arm's line.  `--workload sa_c2 | pt_c1 | pt_c4 | serve_c5` measures
the other configurations (one JSON line each).  Under torchrun (N > 1) every
rank runs its own 256-job batch (same shapes, its own couplings and seeds; weak
scaling, no collective on the data path) and the line reports all ranks'
flips over the slowest rank's time.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
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

METRIC = "spin-flip attempts/s (batched PT-ICM vs plain, 1 B200)"
C3_JOBS, C3_SWEEPS = 256, 5000
C3_L, C3_NT = (8, 12, 16, 24, 32), (16, 24, 32)
C3_CONFIG = {"workload": "batch_c3: 256 uneven 2-D +-J PT-ICM instances, L~U{8,12,16,24,32} periodic, "
                         "nt~U{16,24,32} geometric beta 0.2->5.0, 2 chains, ICM from beta 1.0, 5000 sweeps",
             "instances": C3_JOBS, "sweeps": C3_SWEEPS, "chains": 2, "mode": "colour-ordered (TAMC_MODE_FAST)",
             "l2": "flushed between timed steps (256 MiB write)"}


# ------------------------------------------------------------ helpers ----
def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _profile_value(name, key):
    """A `key: value` figure from a committed ncu summary under profiles/, if present."""
    try:
        txt = open(os.path.join(ROOT, "profiles", name)).read()
        m = re.search(key + r":\s*([0-9.eE+]+)", txt)
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


def _child_json(argv, timeout=900):
    """Runs `python bench.py <argv>` in a fresh process (no torch, no CUDA
    context, its own OpenMP runtime) and returns the JSON it prints last."""
    r = subprocess.run([sys.executable, os.path.abspath(__file__)] + argv, capture_output=True, text=True,
                       timeout=timeout, cwd=ROOT)
    if r.returncode != 0:
        raise RuntimeError(f"CPU leg failed: {r.stderr[-2000:]}")
    return json.loads(r.stdout.strip().splitlines()[-1])


# ------------------------------------------------------- C3 job list ----
def c3_jobs(rank: int = 0):
    """(L, nt, instance seed, run seed) of the 256 jobs; shapes are the same on
    every rank, couplings and run seeds differ per rank."""
    rng = np.random.default_rng(0)
    out = []
    for k in range(C3_JOBS):
        L = int(rng.choice(C3_L))
        nt = int(rng.choice(C3_NT))
        out.append((L, nt, 1000 + k + 100003 * rank, 7 + k + 100003 * rank))
    return out


def c3_flips(jobs, sweeps=C3_SWEEPS):
    return sum(L * L * nt * 2 * sweeps for L, nt, _, _ in jobs)


def c3_bytes(jobs, sweeps=C3_SWEEPS):
    """Algorithmic HBM bytes of the jobs: per flip 2/8 + (4 + 8*4 + 4)/R, R = 2 nt."""
    return sum(L * L * nt * 2 * sweeps * (0.25 + 40.0 / (2 * nt)) for L, nt, _, _ in jobs)


def _lattice_params(tb, nt, sweeps, sample=None, states=None, level=0, threads=8):
    b = tb.geometric_betas(0.2, 5.0, nt)
    lo = int(np.argmax(b >= np.float32(1.0))) if np.any(b >= np.float32(1.0)) else nt - 1
    return tb.PtParams(sweeps, b, lo, 0.5, True, 2, threads, sample, states, level)


# ---------------------------------------------------- CPU (oracle) legs ----
def cpu_c3(stride: int, runs: int, threads: int | None = None):
    """The oracle (CPU restatement of the reference) on jobs 0, stride, 2*stride, ...
    of the batch, each a whole 5000-sweep run; one job per host thread (a
    thread pool over ctypes calls, which release the GIL), longest jobs first.
    Returns the per-run flips/s and a description."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from tamc_b200 import instances as gi
    cores = threads or os.cpu_count() or 1
    jobs = c3_jobs()[::stride]
    texts = [gi.lattice(L, 2, "pm", si) for L, _, si, _ in jobs]
    insts = [po.Instance.from_text(t) for t in texts]
    order = sorted(range(len(jobs)), key=lambda k: -jobs[k][0] ** 2 * jobs[k][1])
    flips = c3_flips(jobs)

    def one(k):
        L, nt, _, seed = jobs[k]
        b = po.geometric_betas(0.2, 5.0, nt)
        lo = po.lo_beta_idx(b, lo_beta=1.0)
        r = po.PtRun(insts[k], b, C3_SWEEPS, 0.5, lo, True, 2, 8, seed=seed)
        r.run(nthreads=1)
        return r.gs()[-1][1] if r.gs() else None

    rates = []
    for _ in range(runs):
        t0 = time.perf_counter()
        with cf.ThreadPoolExecutor(max_workers=cores) as ex:
            list(ex.map(one, order))
        rates.append(flips / (time.perf_counter() - t0))
    desc = (f"oracle PT-ICM (method as the GPU run, threads: 8 semantics), {len(jobs)} of the 256 jobs "
            f"(every {stride}th), 5000 sweeps each, {flips:.3g} flips per run, one job per thread on {cores} "
            f"threads, median of {runs} runs in a child process")
    return rates, desc, cores


def cpu_c4(sweeps: int, runs: int, threads: int | None = None):
    """Whole oracle runs of the C4 method (run_parallel, threads: 64) with `sweeps`
    sweeps on all host cores (OpenMP over the replicas)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from tamc_b200 import instances as gi
    cores = threads or os.cpu_count() or 1
    L = 16
    inst = po.Instance.from_text(gi.lattice(L, 3, "gauss", 0))
    for ax in (0, 1):
        inst.add_suscept(gi.fourier_weights(L, 3, ax))
    b = po.geometric_betas(0.2, 5.0, 64)
    lo = po.lo_beta_idx(b, lo_beta=1.0)
    rates = []
    for k in range(runs):
        r = po.PtRun(inst, b, sweeps, 0.5, lo, True, 2, 64, sample=32, sample_states=32, sample_limiting=0,
                     seed=3 + k)
        t0 = time.perf_counter()
        r.run(nthreads=cores)
        rates.append(4096 * 64 * 2 * sweeps / (time.perf_counter() - t0))
    desc = (f"oracle run_parallel (threads: 64), whole runs of {sweeps} sweeps (warm-up 0.5, samples every 32), "
            f"{cores} OpenMP threads, median of {runs} runs in a child process")
    return rates, desc, cores


def cpu_sa(budget_s: float, threads: int | None = None):
    """The oracle's SA on whole anneals of the C2 instance (all 1000 betas) with as
    many of the 1024 restarts as fit the budget, in `cores` partitions."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    from tamc_b200 import instances as gi
    cores = threads or os.cpu_count() or 1
    inst = po.Instance.from_text(gi.sa_regular(2000, 3, 0))
    betas = np.linspace(0.1, 10.0, 1000).astype(np.float32)
    t0 = time.perf_counter()
    po.sa_run(inst, betas, cores, cores, 1, nthreads=cores)  # one restart per thread
    per = time.perf_counter() - t0
    reps = int(max(1, min(1024 // cores, budget_s / max(per, 1e-9))))
    R = reps * cores
    rates = []
    for k in range(3):
        t0 = time.perf_counter()
        po.sa_run(inst, betas, R, cores, 2 + k, nthreads=cores)
        rates.append(2000 * R * 1000 / (time.perf_counter() - t0))
    desc = (f"oracle SA run_parallel, whole anneals (all 1000 betas) of {R} of the 1024 restarts in {cores} "
            f"partitions, median of 3 runs in a child process")
    return rates, desc, cores


def run_cpu_leg(args):
    if args.cpu_leg == "c3":
        rates, desc, cores = cpu_c3(args.cpu_stride, args.cpu_runs)
    elif args.cpu_leg == "c4":
        rates, desc, cores = cpu_c4(args.c4_cpu_sweeps, args.cpu_runs)
    else:
        rates, desc, cores = cpu_sa(args.cpu_budget)
    print(json.dumps({"value": float(np.median(rates)), "runs": rates, "sample": desc, "cores": cores}))
    return 0


def run_reference(args):
    """The reference arm: the CPU restatement of the reference on the C3 jobs,
    on rank 0 only (other ranks exit without work)."""
    world, rank, _ = _dist()
    if rank != 0:
        return 0
    if args.workload == "sa_c2":
        rates, desc, cores = [], "", 1
        for i in range(args.warmup + args.steps):
            r, desc, cores = cpu_sa(max(1.0, 60.0 / max(1, args.warmup + args.steps)))
            if i >= args.warmup:
                rates.append(float(np.median(r)))
        config, metric = SA_CONFIG, SA_METRIC
    else:
        # each step: one whole-run sample of the batch; the subset is sized so
        # that all warm-up and timed steps end within a few minutes
        stride = args.cpu_stride
        t0 = time.perf_counter()
        r, desc, cores = cpu_c3(stride, 1)
        first = time.perf_counter() - t0
        budget = 180.0 / max(1, args.warmup + args.steps)
        while first > budget and stride < 64:
            stride *= 2
            first /= 2
        rates = []
        for i in range(args.warmup - 1 + args.steps):
            r, desc, cores = cpu_c3(stride, 1)
            if i >= args.warmup - 1:
                rates.append(r[0])
        desc = desc.replace("median of 1 runs in a child process", f"one run per step, median of {len(rates)} steps")
        config, metric = C3_CONFIG, METRIC
    value = float(np.median(rates))
    flips = c3_flips(c3_jobs()) if args.workload != "sa_c2" else SA_FLIPS
    line = {"metric": metric, "value": value, "unit": "flips/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": flips / value * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)", "config": config,
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "flips/s", "cores": cores, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": "flips/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------- GPU: C3 ----
def run_c3(args):
    import torch
    import tamc_b200 as tb
    from tamc_b200 import instances as gi

    world, rank, local = _dist()
    torch.cuda.set_device(local)  # before the process group, so NCCL binds this rank's GPU
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    gpu = tb.Gpu(local)
    lib_stream = torch.cuda.ExternalStream(gpu.stream, device=dev)
    jobs = c3_jobs(rank)
    hosts = [tb.HostInstance.parse(gi.lattice(L, 2, "pm", si)) for L, _, si, _ in jobs]
    sweeps = args.c3_sweeps
    params = [_lattice_params(tb, nt, sweeps) for _, nt, _, _ in jobs]
    dinsts = [gpu.upload(h) for h in hosts]
    flips = c3_flips(jobs, sweeps)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def make_batch(k):
        b = tb.Batch(gpu)
        for j, (d, p) in enumerate(zip(dinsts, params)):
            b.add(d, p, jobs[j][3] + 7919 * k)
        return b

    def flush_l2(k):
        with torch.cuda.stream(lib_stream):
            flush.fill_(k & 0xFF)

    for k in range(args.warmup):  # the first warm-up step also autotunes every job shape
        b = make_batch(k)
        b.run()
        gpu.sync()
        del b
        flush_l2(k)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    step_ms, dev_ms, launches = [], 0.0, 0
    nlaunch = 0
    best = None
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            b = make_batch(args.warmup + k)
            gpu.sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            l0 = gpu.launches
            e0.record(lib_stream)
            b.run()
            e1.record(lib_stream)
            e1.synchronize()
            launches += gpu.launches - l0
            step_ms.append(e0.elapsed_time(e1))
            ms, n = b.device_time()
            dev_ms += ms
            nlaunch += n
            if k == args.steps - 1:
                best = [float(b.gs(j)[1][-1]) if len(b.gs(j)[1]) else None for j in (0, 1, 2, 3)]
            del b
            flush_l2(k)
        torch.cuda.synchronize()
    ms_total = float(np.sum(step_ms))
    ms_t = torch.tensor([ms_total], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    value = flips * args.steps * world / (float(ms_t.item()) / 1e3)

    # end to end through the C ABI: host instances in, results out, per step
    e2e_s, h2d, d2h = [], 0, 0
    for k in range(max(1, min(args.steps, 3)) + 1):
        gpu.sync()
        c0 = tb.copy_bytes()
        t0 = time.perf_counter()
        di = gpu.upload_many(hosts)
        b = tb.Batch(gpu)
        for j, (d, p) in enumerate(zip(di, params)):
            b.add(d, p, jobs[j][3] + 31 * k)
        b.run()
        res = list(zip(b.gs_all(), b.acceptance_all()))
        del b, di
        gpu.sync()
        t1 = time.perf_counter()
        c1 = tb.copy_bytes()
        if k > 0:  # the first pass warms the host allocator and the graph cache
            e2e_s.append(t1 - t0)
            h2d, d2h = c1[0] - c0[0], c1[1] - c0[1]
        assert len(res) == len(jobs)
    e2e_t = torch.tensor([float(np.median(e2e_s))], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    e2e_value = flips * world / float(e2e_t.item())

    out = None
    if rank == 0:
        clocks = clk.summary()
        peak, kind = _peaks()
        dev_ms_step = dev_ms / args.steps
        bytes_step = c3_bytes(jobs, sweeps)
        achieved = bytes_step / (dev_ms_step / 1e3) / 1e9
        traffic = _profile_value("pt_fused_c3.md", "dram_bytes_per_step")
        inst = _profile_value("pt_fused_c3.md", "warp_instructions_per_step")
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
        issue = None
        if inst and mhz:
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            ach, pk = inst / (dev_ms_step / 1e3), sms * 4 * mhz * 1e6
            issue = {"achieved": ach, "peak": pk, "unit": "warp instructions/s", "frac": ach / pk,
                     "instructions_per_step": inst, "clock_mhz": mhz,
                     "source": "profiles/pt_fused_c3.md (smsp__inst_executed.sum over one step's chunk launches)"}
        out = {"metric": METRIC, "value": value, "unit": "flips/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": float(ms_t.item()) / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
               "config": C3_CONFIG if sweeps == C3_SWEEPS else dict(C3_CONFIG, sweeps=sweeps),
               "flips_per_step": flips,
               "e2e": {"value": e2e_value, "unit": "flips/s", "h2d_bytes_per_step": int(h2d),
                       "d2h_bytes_per_step": int(d2h),
                       "path": "tamc_gpu_instance_upload_many (256 instances), tamc_gpu_batch_create/add/run, "
                               "tamc_gpu_batch_gs_all + tamc_gpu_batch_acceptance_all, destroy; wall clock",
                       "s_per_step": float(e2e_t.item())},
               "gpu_launches": int(launches),
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{kind} burst",
                            "bytes_per_step": bytes_step, "kernel": "k_pt_fused (one per chunk launch)",
                            "launch_ms_avg": dev_ms / max(1, nlaunch), "launches_per_step": nlaunch / args.steps},
               "issue_roofline": issue,
               "clocks": clocks, "best_energy_jobs_0_3": best}
        if world == 1 and args.c3_plain > 0:
            out.update(c3_plain(args, tb, gpu, lib_stream, jobs, dinsts, params, value, sweeps))
        if world == 1 and not args.no_cpu:
            cpu = _child_json(["--cpu-leg", "c3", "--cpu-stride", str(args.cpu_stride), "--cpu-runs", "3"])
            out["cpu_baseline"] = {"value": cpu["value"], "unit": "flips/s", "cores": cpu["cores"], "kind": "port",
                                   "sample": cpu["sample"], "runs": cpu["runs"]}
        elif world > 1:
            out["cpu_baseline"] = None
        if world == 1 and not args.no_c4:
            out["c4"] = c4_summary(args, tb, gi, gpu)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)
    del gpu
    return 0


def c3_plain(args, tb, gpu, lib_stream, jobs, dinsts, params, batched, sweeps):
    """The plain form on jobs 0, s, 2s, ... (s = 256 / --c3-plain): one run at a
    time, CUDA events around each run's sweep loop."""
    import torch
    stride = max(1, C3_JOBS // args.c3_plain)
    sub = list(range(0, C3_JOBS, stride))
    os.environ["TAMC_PT_FORM"] = "plain"
    try:
        f, ms = 0, 0.0
        for k in sub:
            r = tb.PtRun(dinsts[k], params[k], jobs[k][3])
            gpu.sync()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(lib_stream)
            r.run()
            e1.record(lib_stream)
            r.sync()
            e1.synchronize()
            ms += e0.elapsed_time(e1)
            L, nt = jobs[k][0], jobs[k][1]
            f += L * L * nt * 2 * sweeps
            del r
    finally:
        del os.environ["TAMC_PT_FORM"]
    plain = f / (ms / 1e3)
    return {"plain_flips_per_s": plain, "batched_over_plain": batched / plain,
            "plain_sample": f"{len(sub)} of the 256 jobs (every {stride}th), one at a time, plain form "
                            f"(one launch per sweep phase over all SMs), CUDA events, {f:.3g} flips in {ms / 1e3:.2f} s"}


def c4_summary(args, tb, gi, gpu):
    """C4 on the GPU (whole 20000-sweep run) against whole oracle runs on all cores."""
    r = workload_pt_c4(args, tb, gi, gpu, cpu=False)
    if not args.no_cpu:
        cpu = _child_json(["--cpu-leg", "c4", "--c4-cpu-sweeps", str(args.c4_cpu_sweeps), "--cpu-runs", "3"])
        r.update(cpu_flips_per_s=cpu["value"], cpu_runs=cpu["runs"], cpu_sample=cpu["sample"],
                 cpu_cores=cpu["cores"], gpu_over_cpu=r["gpu_flips_per_s"] / cpu["value"])
    return r


# ------------------------------------------------------- other workloads ----
SA_N, SA_DEG, SA_R, SA_SWEEPS = 2000, 3, 1024, 1000
SA_FLIPS = SA_N * SA_R * SA_SWEEPS
SA_METRIC = "spin-flip attempts/s (SA, 1 B200)"
SA_CONFIG = {"workload": "sa_c2: N=2000 random 3-regular Ising, J~N(0,1), h~N(0,0.01), linear beta 0.1->10 x 1000 "
                         "sweeps, 1024 restarts", "n": SA_N, "degree": SA_DEG, "restarts": SA_R, "sweeps": SA_SWEEPS,
             "l2": "flushed between timed steps (256 MiB write)"}


def run_sa_c2(args):
    """Simulated annealing, N=2000 random 3-regular, 1024 restarts x 1000 sweeps."""
    import torch
    import tamc_b200 as tb
    from tamc_b200 import instances as gi

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    gpu = tb.Gpu(local)
    dinst = gpu.upload(tb.HostInstance.parse(gi.sa_regular(SA_N, SA_DEG, 0)))
    betas_h = np.linspace(0.1, 10.0, SA_SWEEPS).astype(np.float32)
    betas = torch.from_numpy(betas_h).to(dev)
    energies = torch.empty(SA_R, dtype=torch.float32, device=dev)
    words = torch.empty(((SA_R + 31) // 32) * SA_N, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    seed0 = 1000 * (rank + 1)

    def step(k):
        tb.sa_run_device(dinst, betas.data_ptr(), SA_SWEEPS, SA_R, seed0 + k, energies.data_ptr(), words.data_ptr(),
                         stream.cuda_stream)

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
    ms_t = torch.tensor([float(np.sum(times))], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(ms_t, op=torch.distributed.ReduceOp.MAX)
    value = SA_FLIPS * args.steps * world / (float(ms_t.item()) / 1e3)
    e_min = float(energies.min().item())
    frac_best = float((energies <= e_min + 1e-4 * max(1.0, abs(e_min))).float().mean().item())
    p_anneal = 1.0 - (1.0 - frac_best) ** SA_R
    betas_pin = torch.from_numpy(betas_h).pin_memory().numpy()
    e_pin = torch.empty(SA_R, dtype=torch.float32).pin_memory().numpy()
    packed_pin = torch.empty((SA_R, (SA_N + 7) // 8), dtype=torch.uint8).pin_memory().numpy()
    t_e2e, h2d, d2h = [], 0, 0
    for k in range(max(1, min(args.steps, 5)) + 1):
        torch.cuda.synchronize()
        c0 = tb.copy_bytes()
        t0 = time.perf_counter()
        tb.sa_run(dinst, betas_pin, SA_R, 1, seed0 + 10 ** 6 + k, tb.MODE_FAST, out=(e_pin, packed_pin))
        t_e2e.append(time.perf_counter() - t0)
        c1 = tb.copy_bytes()
        h2d, d2h = c1[0] - c0[0], c1[1] - c0[1]
    e2e_t = torch.tensor([float(np.median(t_e2e[1:]))], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.all_reduce(e2e_t, op=torch.distributed.ReduceOp.MAX)
    out = None
    if rank == 0:
        peak, kind = _peaks()
        per_launch_ms = float(np.mean(times))
        bpf = 2 / 8 + (4 + 8 * SA_DEG + 4) / SA_R
        achieved = bpf * SA_FLIPS / (per_launch_ms / 1e3) / 1e9
        clocks = clk.summary()
        inst = _profile_value("sa_fast_c2.md", "warp_instructions_per_launch")
        mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz")
        issue = None
        if inst and mhz:
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            ach, pk = inst / (per_launch_ms / 1e3), sms * 4 * mhz * 1e6
            issue = {"achieved": ach, "peak": pk, "unit": "warp instructions/s", "frac": ach / pk,
                     "instructions_per_launch": inst, "clock_mhz": mhz,
                     "source": "profiles/sa_fast_c2.md (smsp__inst_executed.sum of one launch)"}
        out = {"metric": SA_METRIC, "value": value, "unit": "flips/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": float(ms_t.item()) / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
               "config": SA_CONFIG,
               "e2e": {"value": SA_FLIPS * world / float(e2e_t.item()), "unit": "flips/s", "h2d_bytes_per_step": h2d,
                       "d2h_bytes_per_step": d2h},
               "gpu_launches": int(launches),
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak,
                            "traffic": _profile_value("sa_fast_c2.md", "traffic_bytes_per_launch"),
                            "peak_kind": f"{kind} burst", "bytes_per_flip": bpf},
               "issue_roofline": issue, "clocks": clocks, "best_energy": e_min, "restarts_at_best": frac_best,
               "tts99_s": per_launch_ms / 1e3 * (1.0 if p_anneal >= 0.99 else
                                                math.log(0.01) / math.log(1.0 - p_anneal))}
        if not args.no_cpu and world == 1:
            cpu = _child_json(["--cpu-leg", "sa", "--cpu-budget", "12"])
            out["cpu_baseline"] = {"value": cpu["value"], "unit": "flips/s", "cores": cpu["cores"], "kind": "port",
                                   "sample": cpu["sample"], "runs": cpu["runs"]}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if out is not None:
        print(json.dumps(out), flush=True)
    return 0


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


def workload_pt_c4(args, tb, gi, gpu, cpu=True):
    """3-D Gaussian L=16 (N=4096), nt=64, 2 chains, ICM, 20000 sweeps, sampling every 32, suscepts."""
    L = 16
    text = gi.lattice(L, 3, "gauss", 0)
    h = tb.HostInstance.parse(text)
    for ax in (0, 1):
        h.add_suscept(gi.fourier_weights(L, 3, ax))
    d = gpu.upload(h)
    sweeps = args.c4_sweeps
    p = _lattice_params(tb, 64, sweeps, 32, 32, 0, threads=64)
    flips = 4096 * 64 * 2 * sweeps
    _time_run(tb, d, _lattice_params(tb, 64, 64, 32, 32, 0, threads=64), 1)  # autotune + warm-up
    t_gpu, r = _time_run(tb, d, p, 2)
    best = float(r.gs()[1][-1])
    first, tts = _time_to_target(tb, d, p, 2, best, t_gpu / sweeps)
    out = {"workload": "pt_c4: 3-D L=16 Gaussian, 64 temperatures, 2 chains, ICM, samples every 32",
           "sweeps": sweeps, "flips": flips, "gpu_flips_per_s": flips / t_gpu, "gpu_s": t_gpu,
           "round_us": t_gpu / sweeps * 1e6,
           "gpu_best_energy": best, "target_energy": best,
           "target_first_sweep": first, "time_to_target_s": tts}
    if cpu and not args.no_cpu:
        c = _child_json(["--cpu-leg", "c4", "--c4-cpu-sweeps", str(args.c4_cpu_sweeps), "--cpu-runs", "3"])
        out.update(cpu_flips_per_s=c["value"], cpu_runs=c["runs"], cpu_sample=c["sample"], cpu_cores=c["cores"],
                   gpu_over_cpu=(flips / t_gpu) / c["value"])
    return out


def workload_batch_c3(args, tb, gi, gpu):
    raise SystemExit("batch_c3 is the default line: run bench.py without --workload")


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
    fn = {"pt_c1": workload_pt_c1, "pt_c4": workload_pt_c4, "serve_c5": workload_serve_c5}[args.workload]
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
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline legs")
    ap.add_argument("--no-c4", action="store_true", help="skip the C4 keys of the default line")
    ap.add_argument("--workload", default="batch_c3", choices=["batch_c3", "sa_c2", "pt_c1", "pt_c4", "serve_c5"])
    ap.add_argument("--c3-plain", type=int, default=64, help="jobs of the plain-form comparison (0 skips it)")
    ap.add_argument("--c3-sweeps", type=int, default=C3_SWEEPS, help="sweeps per job (profiling runs only)")
    ap.add_argument("--c4-sweeps", type=int, default=20000)
    ap.add_argument("--c4-cpu-sweeps", type=int, default=1000)
    ap.add_argument("--c5-requests", type=int, default=1000)
    ap.add_argument("--c5-rate", type=float, default=100.0)
    ap.add_argument("--cpu-leg", choices=["c3", "c4", "sa"], help=argparse.SUPPRESS)
    ap.add_argument("--cpu-stride", type=int, default=8, help="C3 CPU sample: every k-th job")
    ap.add_argument("--cpu-runs", type=int, default=3)
    ap.add_argument("--cpu-budget", type=float, default=12.0)
    args = ap.parse_args()
    if args.cpu_leg:
        return run_cpu_leg(args)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch_c3":
        return run_c3(args)
    if args.workload == "sa_c2":
        return run_sa_c2(args)
    return run_workload(args)


if __name__ == "__main__":
    sys.exit(main())
