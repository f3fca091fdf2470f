"""Parity on the benchmark configurations themselves, not toy sizes.

* C1 (2-D L=16 +-J, 32 temperatures, lo_beta 1.0, 2 chains, 2000 sweeps,
  warm-up 0.5, measured every 32 sweeps): colour-ordered mode against the
  oracle over 16 independent seeds each -- per temperature <E>, <|q|> and the
  two Fourier-mode <chi^2> -- and the same best energy; reference-order mode
  bit-exact against the live oracle over the whole run, with serial (threads:
  1) and threaded (threads: 16) exchange semantics.
* C2 (SA, N=2000 random 3-regular, 1024 restarts x 1000 linear betas 0.1->10):
  final-energy distribution and best energy against the oracle's run_parallel.
* C4 shortened (3-D L=16 Gaussian, 64 temperatures, 1000 sweeps, 8 seeds):
  <E> over the paramagnetic temperatures against the oracle.

Statistical rule (tests/stat_rule.py, fixed before any run): z = (mean_gpu -
mean_oracle) / sqrt(se_gpu^2 + se_oracle^2) over independent seeds; every
|z| <= 4 and at least 95 % of them <= 3.
"""
import concurrent.futures as cf
import math
import os

import numpy as np
import pytest

from tamc_b200 import instances as gi

pytestmark = pytest.mark.gpu

CORES = os.cpu_count() or 1


def _z_ok(g, o, label):
    from stat_rule import z_ok
    return z_ok(g, o, label)


def _thermal_stats(e, q, sus, nt, chains=2):
    e = np.array(e, np.float64).reshape(nt, -1, chains).mean(axis=(1, 2))
    q = np.abs(np.array(q, np.float64)).reshape(nt, -1).mean(axis=1)
    x = (np.array(sus, np.float64) ** 2).mean(axis=2)  # [nt][nchi]
    return np.concatenate([e, q, x.T.ravel()])


def _pool(fn, items):
    # ctypes calls release the GIL: one oracle run per host thread
    with cf.ThreadPoolExecutor(max_workers=CORES) as ex:
        return list(ex.map(fn, items))


# --------------------------------------------------------------------- C1 ----
C1_L, C1_NT, C1_SWEEPS, C1_SEEDS = 16, 32, 2000, 16


def _c1(tb, po):
    text = gi.lattice(C1_L, 2, "pm", 0)
    w = [gi.fourier_weights(C1_L, 2, 0), gi.fourier_weights(C1_L, 2, 1)]
    b = po.geometric_betas(0.2, 5.0, C1_NT)
    lo = po.lo_beta_idx(b, lo_beta=1.0)
    return text, w, b, lo


def test_c1_colour_order_thermal_statistics_and_ground_state(tb, po, gpu):
    text, w, b, lo = _c1(tb, po)
    h = tb.HostInstance.parse(text)
    inst = po.Instance.from_text(text)
    for row in w:
        h.add_suscept(row)
        inst.add_suscept(row)
    d = gpu.upload(h)
    p = tb.PtParams(C1_SWEEPS, b, lo, 0.5, True, 2, 1, 32, None, 0)
    batch = tb.Batch(gpu)
    for s in range(C1_SEEDS):
        batch.add(d, p, 1000 + s)
    batch.run()
    g, g_best = [], []
    for s in range(C1_SEEDS):
        ts = batch.samples(s)
        assert len(ts.e[0]) == 2 * 33  # 32 samples after the warm-up, plus the last sweep
        g.append(_thermal_stats(ts.e, ts.q, ts.suscept, C1_NT))
        g_best.append(float(batch.gs(s)[1][-1]))

    def oracle(s):
        r = po.PtRun(inst, b, C1_SWEEPS, 0.5, lo, True, 2, 1, sample=32, seed=2000 + s)
        r.run(nthreads=1)
        e, q, sus, _ = r.thermal(nchi=2)
        return _thermal_stats(e, q, sus, C1_NT), r.gs()[-1][1]

    res = _pool(oracle, range(C1_SEEDS))
    o = [x[0] for x in res]
    o_best = [x[1] for x in res]
    _z_ok(g, o, "C1 <E>, <|q|>, <chi^2> per temperature")
    # the same ground state: lowest energy over the seeds, and both find it often
    assert min(g_best) == min(o_best)
    assert sum(e == min(o_best) for e in g_best) >= C1_SEEDS // 2
    assert sum(e == min(o_best) for e in o_best) >= C1_SEEDS // 2


@pytest.mark.parametrize("threads", [1, 16])
def test_c1_reference_order_bit_exact_whole_run(tb, po, gpu, threads):
    """The whole C1 run (2000 sweeps, e/q every 32 sweeps, states of every
    temperature every 32 sweeps) replayed bit for bit."""
    text, w, b, lo = _c1(tb, po)
    inst = po.Instance.from_text(text)
    h = tb.HostInstance.parse(text)
    for row in w:
        h.add_suscept(row)
        inst.add_suscept(row)
    seed = 77 + threads
    orc = po.PtRun(inst, b, C1_SWEEPS, 0.5, lo, True, 2, threads, sample=32, sample_states=32, sample_limiting=0,
                   seed=seed)
    orc.run(nthreads=min(threads, CORES))
    run = tb.PtRun(gpu.upload(h), tb.PtParams(C1_SWEEPS, b, lo, 0.5, True, 2, threads, 32, 32, 0), seed,
                   tb.MODE_REF).run().sync()
    S0, E0, _ = orc.states()
    S1, E1 = run.state()
    assert np.array_equal(S0, S1)
    assert np.array_equal(E0.view(np.uint32), E1.view(np.uint32))
    assert np.array_equal(orc.acceptance().sum(0), run.acceptance())
    for c in range(2):
        t0, rt0, dh0 = orc.tags(c)
        t1, rt1, dh1 = run.round_trips()
        assert np.array_equal(t0, t1[c]) and rt0 == rt1[c] and np.array_equal(dh0, dh1[c])
    gs0 = orc.gs()
    steps, en, st = run.gs()
    assert [x[0] for x in gs0] == steps.tolist()
    assert np.array_equal(np.array([x[1] for x in gs0], np.float32).view(np.uint32), en.view(np.uint32))
    assert np.array_equal(np.array([x[2] for x in gs0]), st)
    e, q, sus, smp = orc.thermal(nchi=2)
    ts = run.samples()
    assert np.array_equal(np.array(e).view(np.uint32), np.array(ts.e).view(np.uint32))
    assert np.array_equal(np.array(q), np.array(ts.q))
    assert np.array_equal(np.array(sus, np.float32).view(np.uint32), np.array(ts.suscept).view(np.uint32))
    assert np.array_equal(np.array(smp), np.array(ts.samples))


# --------------------------------------------------------------------- C2 ----
def test_c2_sa_energies_and_best_state_match_oracle(tb, po, gpu):
    """Final-energy distribution of 1024 restarts within the statistical rule
    (mean and lower quantiles over independent restarts), and the best state:
    the lowest energy the oracle's 1024 restarts reach is reached by the GPU's
    restarts at a rate consistent with the oracle's (a binomial test)."""
    text = gi.sa_regular(2000, 3, 0)
    betas = np.linspace(0.1, 10.0, 1000).astype(np.float32)
    d = gpu.upload(tb.HostInstance.parse(text))
    inst = po.Instance.from_text(text)
    anneals = 8
    eg = np.concatenate([tb.sa_run(d, betas, 1024, 1, 500 + k)[0] for k in range(anneals)]).astype(np.float64)
    eo, so = po.sa_run(inst, betas, 1024, CORES, 9, nthreads=CORES)
    eo = eo.astype(np.float64)
    # distribution: mean, and the share below fixed energy levels, as per-restart means
    se = math.sqrt(eg[:1024].var(ddof=1) / 1024 + eo.var(ddof=1) / 1024)
    assert abs(eg[:1024].mean() - eo.mean()) <= 3 * se, (eg.mean(), eo.mean(), se)
    for lvl in np.quantile(eo, [0.1, 0.25, 0.5]):
        pg, po_ = np.mean(eg <= lvl), np.mean(eo <= lvl)
        pp = (pg * len(eg) + po_ * len(eo)) / (len(eg) + len(eo))
        assert abs(pg - po_) <= 3.5 * math.sqrt(pp * (1 - pp) * (1 / len(eg) + 1 / len(eo))) + 1e-12, lvl
    # best state: compare f64 energies of the spins (the two modes sum in different orders)
    best_o = min(inst.energy_f64(s) for s in so[eo <= eo.min() + 1e-3])
    tol = 1e-3
    hit_o = np.mean(eo <= best_o + tol)
    hit_g = np.mean(eg <= best_o + tol)
    pp = (hit_o * len(eo) + hit_g * len(eg)) / (len(eo) + len(eg))
    assert hit_g > 0, "no GPU restart reaches the oracle's best energy"
    assert abs(hit_g - hit_o) <= 3.5 * math.sqrt(pp * (1 - pp) * (1 / len(eg) + 1 / len(eo)))


# --------------------------------------------------------------------- C4 ----
def test_c4_shortened_paramagnetic_energies_match_oracle(tb, po, gpu):
    L, nt, sweeps, seeds = 16, 64, 1000, 8
    text = gi.lattice(L, 3, "gauss", 0)
    b = po.geometric_betas(0.2, 5.0, nt)
    lo = po.lo_beta_idx(b, lo_beta=1.0)
    hot = np.flatnonzero(b <= 0.8)  # the paramagnetic end, equilibrated within the run
    assert len(hot) >= 20
    d = gpu.upload(tb.HostInstance.parse(text))
    inst = po.Instance.from_text(text)
    p = tb.PtParams(sweeps, b, lo, 0.5, True, 2, 64, 8, None, 0)
    g = []
    for s in range(seeds):
        ts = tb.PtRun(d, p, 300 + s).run().sync().samples()
        g.append(np.array(ts.e, np.float64).mean(axis=1)[hot])

    def oracle(s):
        r = po.PtRun(inst, b, sweeps, 0.5, lo, True, 2, 64, sample=8, seed=400 + s)
        r.run(nthreads=max(1, CORES // seeds))
        e, _, _, _ = r.thermal()
        return np.array(e, np.float64).mean(axis=1)[hot]

    o = _pool(oracle, range(seeds))
    _z_ok(g, o, "C4 <E> at beta <= 0.8")
