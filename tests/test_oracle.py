"""The CPU oracle against independent restatements, physics known answers and
the committed golden fixtures (CPU only)."""
import itertools

import numpy as np
import pytest

from conftest import load_golden

M64 = (1 << 64) - 1


# ---- an independent pure-Python restatement of the RNG stack ---------------
def py_splitmix(seed, n):
    st, out = seed, []
    for _ in range(n):
        st = (st + 0x9E3779B97F4A7C15) & M64
        z = st
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        out.append(z ^ (z >> 31))
    return out


def rotl(x, k):
    return ((x << k) | (x >> (64 - k))) & M64


def py_xo_next(s):
    r = (rotl((s[0] + s[3]) & M64, 23) + s[0]) & M64
    t = (s[1] << 17) & M64
    s[2] ^= s[0]
    s[3] ^= s[1]
    s[1] ^= s[2]
    s[0] ^= s[3]
    s[2] ^= t
    s[3] = rotl(s[3], 45)
    return r


def py_xo_jump(s):
    J = [0x180EC6D33CFD0ABA, 0xD5A61266F0C9392C, 0xA9582618E03FC9AA, 0x39ABDC4529B1661C]
    t = [0, 0, 0, 0]
    for j in J:
        for b in range(64):
            if (j >> b) & 1:
                t = [a ^ c for a, c in zip(t, s)]
            py_xo_next(s)
    s[:] = t


@pytest.mark.parametrize("seed", [0, 1, 1234, 2 ** 63 + 5])
def test_rng_matches_independent_restatement(po, seed):
    assert list(po.splitmix64(seed, 8)) == py_splitmix(seed, 8)
    s = po.xoshiro_seed(seed)
    ps = py_splitmix(seed, 4)
    assert list(s) == ps
    got = po.xoshiro_next(s, 50)
    want = [py_xo_next(ps) for _ in range(50)]
    assert list(got) == want
    po.xoshiro_jump(s)
    py_xo_jump(ps)
    assert list(s) == ps
    assert list(po.xoshiro_next(s, 5)) == [py_xo_next(ps) for _ in range(5)]


@pytest.mark.parametrize("rng_range", [1, 2, 3, 7, 1000, 2 ** 31 + 1])
def test_gen_range_semantics(po, rng_range):
    s = po.xoshiro_seed(99)
    ps = [int(x) for x in s]
    got = po.gen_range(s, rng_range, 200)
    zone = ((rng_range << (32 - rng_range.bit_length())) & 0xFFFFFFFF) - 1
    want = []
    while len(want) < 200:
        v = py_xo_next(ps) >> 32
        m = v * rng_range
        if (m & 0xFFFFFFFF) <= zone:
            want.append(m >> 32)
    assert list(got) == want
    assert got.max() < rng_range


def test_geometric_betas_and_lo_idx(po):
    b = po.geometric_betas(0.2, 5.0, 32)
    assert b[0] == np.float32(0.2) and abs(b[-1] - 5.0) < 1e-6
    assert np.all(np.diff(b) > 0)
    assert po.lo_beta_idx(b, lo_beta=1.0) == int(np.argmax(b >= np.float32(1.0)))
    assert po.lo_beta_idx(b, lo_beta=100.0) == 31
    assert po.lo_beta_idx(b, lo_num=4) == 28
    assert po.lo_beta_idx(b, lo_num=100, lo_beta=1.0) == 0


# ---- physics known answers -----------------------------------------------
def _ferro(L, dim):
    from tamc_b200 import instances as gi
    return gi.lattice(L, dim, "ferro", 0)


@pytest.mark.parametrize("L,dim,gs", [(8, 2, -128.0), (4, 3, -192.0)])
def test_ferromagnet_ground_state(po, L, dim, gs):
    inst = po.Instance.from_text(_ferro(L, dim))
    assert inst.energy_ref(np.ones(inst.n, np.int8)) == gs
    assert inst.energy_ref(-np.ones(inst.n, np.int8)) == gs
    b = po.geometric_betas(0.2, 5.0, 12)
    r = po.PtRun(inst, b, 300, 0.5, po.lo_beta_idx(b, lo_beta=1.0), True, 2, 4, seed=3)
    r.run()
    assert r.gs()[-1][1] == gs


def test_brute_force_ground_state(po):
    from tamc_b200 import instances as gi
    text = gi.sa_regular(14, 3, 2)
    inst = po.Instance.from_text(text)
    n = inst.n
    states = 1 - 2 * ((np.arange(2 ** n)[:, None] >> np.arange(n)) & 1).astype(np.int8)
    e = np.array([inst.energy_f64(s) for s in states])
    b = po.geometric_betas(0.3, 6.0, 10)
    r = po.PtRun(inst, b, 400, 0.25, 5, True, 2, 2, seed=8)
    r.run()
    assert abs(r.gs()[-1][1] - e.min()) < 1e-4


def test_delta_energy_consistent(po):
    from tamc_b200 import instances as gi
    inst = po.Instance.from_text(gi.sa_regular(30, 3, 4))
    rng = np.random.default_rng(0)
    s = rng.choice(np.array([-1, 1], np.int8), inst.n)
    for i in range(inst.n):
        s2 = s.copy()
        s2[i] = -s2[i]
        assert abs(inst.energy_f64(s2) - inst.energy_f64(s) - inst.delta_energy(s, i)) < 1e-4


def test_icm_preserves_pair_energy_and_overlap_structure(po):
    # Houdayer moves swap clusters between two replicas: the multiset of
    # (s1_i, s2_i) pairs per site is preserved.
    inst = po.Instance.from_text(_ferro(6, 2))
    b = po.geometric_betas(1.0, 2.0, 2)
    r = po.PtRun(inst, b, 1, 0.0, 0, True, 2, 2, seed=5)
    S0, _, _ = r.states()
    r.run(1)
    sizes = r.icm_sizes()
    assert len(sizes) == 2


# ---- golden fixtures ------------------------------------------------------
PT_GOLDEN = ["pt_2d_pm_L4_threaded", "pt_2d_pm_L4_serial", "pt_rrg_gauss_threaded", "pt_qubo_serial",
             "pt_2d_pm_L16_threaded", "pt_3d_gauss_L4_threaded"]
SA_GOLDEN = ["sa_rrg_parallel", "sa_rrg_single", "sa_2d_pm_parallel"]


@pytest.mark.parametrize("name", PT_GOLDEN)
def test_oracle_reproduces_pt_golden(po, name):
    g = load_golden(name)
    inst = po.Instance.from_text(bytes(g["text"]).decode(), qubo=bool(g["qubo"]))
    for w in g["suscept"]:
        inst.add_suscept(w)
    r = po.PtRun(inst, g["betas"], int(g["sweeps"]), 0.5, int(g["lo"]), True, int(g["chains"]), int(g["threads"]),
                 sample=int(g["sample"]), sample_states=int(g["sample_states"]), sample_limiting=int(g["level"]),
                 seed=int(g["seed"]))
    r.run()
    S, E, _ = r.states()
    assert np.array_equal(S, g["spins"])
    assert np.array_equal(E.view(np.uint32), g["energies"].view(np.uint32))
    assert np.array_equal(r.acceptance(), g["acceptance"])
    gs = r.gs()
    assert [x[0] for x in gs] == list(g["gs_steps"])
    assert np.array_equal(np.array([x[1] for x in gs], np.float32), g["gs_energies"])
    e, q, sus, smp = r.thermal(nchi=len(g["suscept"]))
    assert np.array_equal(np.array(e, np.float32), g["e"])
    assert np.array_equal(np.array(q, np.int32), g["q"])
    if len(g["suscept"]):
        assert np.array_equal(np.array(sus, np.float32), g["sus"])
    assert np.array_equal(np.array(smp, np.uint8).reshape(g["samples"].shape), g["samples"])


@pytest.mark.parametrize("name", SA_GOLDEN)
def test_oracle_reproduces_sa_golden(po, name):
    g = load_golden(name)
    inst = po.Instance.from_text(bytes(g["text"]).decode(), qubo=bool(g["qubo"]))
    e, s = po.sa_run(inst, g["betas"], int(g["num_replicas"]), int(g["threads"]), int(g["seed"]))
    assert np.array_equal(e, g["energies"])
    assert np.array_equal(s, g["spins"])


def test_threaded_run_independent_of_omp_threads(po):
    g = load_golden("pt_3d_gauss_L4_threaded")
    inst = po.Instance.from_text(bytes(g["text"]).decode())
    outs = []
    for nth in (1, 3):
        r = po.PtRun(inst, g["betas"], 20, 0.5, int(g["lo"]), True, 2, 16, seed=4)
        r.run(nthreads=nth)
        outs.append(r.states()[0])
    assert np.array_equal(outs[0], outs[1])


def test_oracle_serial_exchange_samples_exact_boltzmann_and_threaded_does_not(po):
    """<E>(beta) of a 4x4 +-J torus against exact enumeration of its 65536
    states.  Serial exchange (threads: 1, tamc-core/src/pt.rs:120-132)
    updates the next pair's energy difference after a swap: every |z| <= 4 over
    6 runs.  The threaded exchange (tamc-core/src/parallel/pt.rs:46-58) decides
    every pair on the differences of the round's start; the oracle keeps that,
    and its coldest slot is visibly hotter than the Boltzmann average."""
    from tamc_b200 import instances as gi
    text = gi.lattice(4, 2, "pm", 21)
    betas = np.linspace(0.1, 1.6, 8).astype(np.float32)
    spins = ((np.arange(1 << 16)[:, None] >> np.arange(16)[None, :]) & 1).astype(np.int8) * -2 + 1
    E = np.zeros(1 << 16)
    for ln in text.strip().splitlines():
        a, c, k = ln.split()
        E += float(k) * spins[:, int(a)] * spins[:, int(c)]
    exact = np.array([(np.exp(-float(b) * (E - E.min())) * E).sum() / np.exp(-float(b) * (E - E.min())).sum()
                      for b in betas])
    inst = po.Instance.from_text(text)

    def means(threads):
        out = []
        for s in range(6):
            r = po.PtRun(inst, betas, 20000, 0.1, 4, True, 2, threads, sample=1, seed=900 + s)
            r.run(nthreads=1)
            out.append(np.array(r.thermal()[0], np.float64).mean(axis=1))
        out = np.array(out)
        return out.mean(0), out.std(0, ddof=1) / np.sqrt(len(out))

    m1, se1 = means(1)
    assert np.all(np.abs(m1 - exact) <= 4 * se1), (m1, exact, se1)
    m4, se4 = means(4)
    assert m4[-1] - exact[-1] > 0.2 and m4[-1] - exact[-1] > 20 * se4[-1], (m4, exact)


@pytest.mark.parametrize("threads", [1, 3])
def test_oracle_qubo_cached_energy_rule(po, threads):
    """The oracle's cached energies on a QUBO follow the reference's rule
    (self-coupling drift between Houdayer refreshes), predicted exactly with an
    all-zero ladder; pins the predictor the GPU test uses."""
    from qubo_rule import check_cached_energies, self_coupling_sum
    from tamc_b200 import instances as gi
    inst = po.Instance.from_text(gi.qubo_er(48, 5, 2), qubo=True)
    rp, col, K, _ = inst.csr()
    ksum = self_coupling_sum(rp, col, K)
    assert ksum != 0.0
    nt, lo, rounds, C = 6, 3, 14, 2
    orc = po.PtRun(inst, np.zeros(nt, np.float32), rounds, 0.0, lo, True, C, threads, sample=1, sample_states=1,
                   sample_limiting=0, seed=5)
    orc.run()
    e, _, _, samples = orc.thermal()
    assert check_cached_energies(e, samples, inst.energy_f64, nt, lo, rounds, C, ksum, inst.n) >= 3


@pytest.mark.parametrize("case", range(8))
def test_pt_opt_step_matches_restatement(tb, case):
    """tamc_pt_opt_step (the library's ladder update) against the oracle's
    float32 restatement of pt_optimize_beta's iteration, bit for bit, on
    synthetic round-trip statistics (including zero round trips and too few
    to form the density)."""
    import ctypes as C
    import ptopt
    rng = np.random.default_rng(case)
    nt = [8, 12, 16, 32, 24, 9, 16, 5][case]
    ninst = [1, 3, 5, 2, 4, 1, 6, 2][case]
    betas = tb.geometric_betas(0.2, 5.0, nt)
    mom = betas * np.float32(1.03) if case % 2 else betas.copy()
    rts = rng.integers(0, 40, ninst).astype(np.uint32)
    if case == 5:
        rts[:] = 0
    frac = 1 / (1 + np.exp(-np.linspace(-4, 4, nt) + rng.normal(0, 0.3, nt)))
    tot = rng.integers(500, 5000, (ninst, nt))
    dh = np.stack([tot - np.round(tot * frac), np.round(tot * frac)], -1).astype(np.uint32)
    if case == 7:
        dh[:] = 0  # no flow at all: every fraction 1/2, no density
    want = ptopt.step(betas, mom, rts, dh, 2000, 2, 0.2, 0.85)
    b, m = betas.copy(), mom.copy().astype(np.float32)
    tau = np.zeros(ninst, np.float32)
    err = C.c_float()
    L = tb.lib()
    L.tamc_pt_opt_step.restype = C.c_int
    rc = L.tamc_pt_opt_step(nt, b.ctypes.data_as(C.POINTER(C.c_float)), m.ctypes.data_as(C.POINTER(C.c_float)),
                            ninst, np.ascontiguousarray(rts).ctypes.data_as(C.POINTER(C.c_uint32)),
                            np.ascontiguousarray(dh).ctypes.data_as(C.POINTER(C.c_uint32)), 2000, 2,
                            C.c_float(0.2), C.c_float(0.85), tau.ctypes.data_as(C.POINTER(C.c_float)),
                            C.byref(err))
    assert rc == want[0]
    assert np.array_equal(tau.view(np.uint32), np.array(want[3], np.float32).view(np.uint32))
    assert np.array_equal(b.view(np.uint32), np.array(want[1], np.float32).view(np.uint32))
    assert np.array_equal(m.view(np.uint32), np.array(want[2], np.float32).view(np.uint32))
    if rc == 0:
        assert np.float32(err.value) == want[4]
        assert np.all(np.diff(b) > 0) and b[0] == betas[0]
