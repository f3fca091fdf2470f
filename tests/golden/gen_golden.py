"""Generates the golden fixtures under tests/golden/ from the CPU oracle.

The reference (Rust) cannot be built in this environment and its own tests
hold no known answers, so these fixtures record the oracle's restatement of
the reference for fixed seeds: final replica states, cached energies,
acceptance counts, round-trip bookkeeping, the ground-state trajectory and the
thermal samples of PT-ICM runs (serial and threaded exchange), and SA runs.
They pin the oracle against regressions and are the bit-exact targets of the
reference-order GPU mode.  Run:  python tests/golden/gen_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import pyoracle as po  # noqa: E402
from tamc_b200 import instances as gi  # noqa: E402

PT_CASES = {
    # name: (instance generator, qubo, betas, lo, chains, threads, sweeps, sample, sample_states, level, suscept, seed)
    "pt_2d_pm_L4_threaded": (lambda: gi.lattice(4, 2, "pm", 11), False, (0.2, 5.0, 8), ("lo_beta", 1.0), 2, 4, 60,
                             4, 8, 0, True, 1234),
    "pt_2d_pm_L4_serial": (lambda: gi.lattice(4, 2, "pm", 11), False, (0.2, 5.0, 8), ("lo_beta", 1.0), 2, 1, 60,
                           4, 8, 0, True, 1234),
    "pt_rrg_gauss_threaded": (lambda: gi.sa_regular(24, 3, 5), False, (0.3, 4.0, 6), ("lo_num", 3), 4, 3, 40,
                              3, 5, 1, False, 77),
    "pt_qubo_serial": (lambda: gi.qubo_er(20, 4, 9), True, (0.2, 2.0, 4), ("lo_beta", 0.5), 2, 1, 30, 5, 7, 2,
                       False, 5),
    "pt_2d_pm_L16_threaded": (lambda: gi.lattice(16, 2, "pm", 3), False, (0.2, 5.0, 32), ("lo_beta", 1.0), 2, 8,
                              200, 32, 32, 2, False, 42),
    "pt_3d_gauss_L4_threaded": (lambda: gi.lattice(4, 3, "gauss", 8), False, (0.2, 5.0, 16), ("lo_beta", 1.0), 2,
                                16, 50, 10, 10, 0, True, 99),
}

SA_CASES = {
    # name: (instance, qubo, betas, num_replicas, threads, seed)
    "sa_rrg_parallel": (lambda: gi.sa_regular(24, 3, 6), False, np.linspace(0.1, 3.0, 40), 8, 4, 21),
    "sa_rrg_single": (lambda: gi.sa_regular(24, 3, 6), False, np.linspace(0.1, 3.0, 40), 1, 4, 22),
    "sa_2d_pm_parallel": (lambda: gi.lattice(8, 2, "pm", 4), False, np.linspace(0.1, 2.0, 30), 10, 3, 23),
}


def run_pt_case(name, spec):
    gen, qubo, (b0, b1, nb), lo_spec, C, threads, sweeps, sample, sstates, level, sus, seed = spec
    text = gen()
    inst = po.Instance.from_text(text, qubo=qubo)
    betas = po.geometric_betas(b0, b1, nb)
    lo = po.lo_beta_idx(betas, lo_beta=lo_spec[1]) if lo_spec[0] == "lo_beta" else po.lo_beta_idx(betas, lo_num=lo_spec[1])
    w = None
    if sus:
        L = int(round(inst.n ** 0.5)) if name.startswith("pt_2d") else int(round(inst.n ** (1 / 3)))
        dim = 2 if name.startswith("pt_2d") else 3
        w = np.stack([gi.fourier_weights(L, dim, 0), gi.fourier_weights(L, dim, 1)])
        for row in w:
            inst.add_suscept(row)
    run = po.PtRun(inst, betas, sweeps, 0.5, lo, True, C, threads, sample=sample, sample_states=sstates,
                   sample_limiting=level, seed=seed)
    run.run()
    S, E, F = run.states()
    acc = run.acceptance()
    gs = run.gs()
    e, q, su, smp = run.thermal(nchi=0 if w is None else len(w))
    tags = []
    rts = []
    dh = []
    for c in range(C):
        t, r, d = run.tags(c)
        tags.append(t)
        rts.append(r)
        dh.append(d)
    out = dict(
        text=np.frombuffer(text.encode(), np.uint8), qubo=qubo, betas=betas, lo=lo, chains=C, threads=threads,
        sweeps=sweeps, sample=sample, sample_states=sstates, level=level, seed=seed,
        suscept=np.zeros((0, inst.n)) if w is None else w,
        spins=S, energies=E, acceptance=acc, tags=np.array(tags), round_trips=np.array(rts), dhist=np.array(dh),
        gs_steps=np.array([g[0] for g in gs], np.uint32), gs_energies=np.array([g[1] for g in gs], np.float32),
        gs_states=np.array([g[2] for g in gs], np.uint64).reshape(len(gs), -1),
        e=np.array(e, np.float32), q=np.array(q, np.int32),
        sus=(np.zeros((len(betas), 0, 0), np.float32) if w is None else
             np.array(su, np.float32).reshape(len(betas), len(w), -1)),
        samples=np.array(smp, np.uint8).reshape(len(smp), -1, (inst.n + 7) // 8),
    )
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    return out


def run_sa_case(name, spec):
    gen, qubo, betas, R, threads, seed = spec
    text = gen()
    inst = po.Instance.from_text(text, qubo=qubo)
    betas = np.asarray(betas, np.float32)
    en, st = po.sa_run(inst, betas, R, threads, seed)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), text=np.frombuffer(text.encode(), np.uint8), qubo=qubo,
                        betas=betas, num_replicas=R, threads=threads, seed=seed, energies=en, spins=st)


def main():
    for k, v in PT_CASES.items():
        run_pt_case(k, v)
        print("wrote", k)
    for k, v in SA_CASES.items():
        run_sa_case(k, v)
        print("wrote", k)


if __name__ == "__main__":
    main()
