"""Edge shapes on the GPU: a one-site instance, an odd number of replica
chains with a single temperature, a single sweep, the largest and the first
too-large fast-mode shapes, and an instance without sites.  Reference-order
results must equal the oracle's bit for bit; fast-mode energies must match an
FP64 recomputation."""
import numpy as np
import pytest

from tamc_b200 import instances as gi

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _ref_vs_oracle(tb, po, gpu, text, betas, sweeps, warm, lo, icm, chains, threads, sample, states, level, seed):
    orc = po.PtRun(po.Instance.from_text(text), betas, sweeps, warm, lo, icm, chains, threads, sample=sample,
                   sample_states=states, sample_limiting=level, seed=seed)
    orc.run()
    p = tb.PtParams(sweeps, betas, lo, warm, icm, chains, threads, sample, states, level)
    run = tb.PtRun(gpu.upload(tb.HostInstance.parse(text)), p, seed, tb.MODE_REF).run().sync()
    S0, E0, _ = orc.states()
    S1, E1 = run.state()
    assert np.array_equal(S0, S1)
    assert np.array_equal(_bits(E0), _bits(E1))
    assert np.array_equal(orc.acceptance().sum(0), run.acceptance())
    gs = orc.gs()
    steps, en, st = run.gs()
    assert [g[0] for g in gs] == list(steps)
    assert np.array_equal(_bits([g[1] for g in gs]), _bits(en))
    return run


def test_ref_single_site_instance(tb, po, gpu):
    betas = np.array([0.5, 1.0, 2.0], np.float32)
    _ref_vs_oracle(tb, po, gpu, "0 0 0.7\n", betas, 10, 0.0, 0, False, 2, 1, 2, None, 0, 3)


def test_sa_single_site_instance(tb, po, gpu):
    betas = np.linspace(0.1, 10, 50).astype(np.float32)
    d = gpu.upload(tb.HostInstance.parse("0 0 0.7\n"))
    e0, s0 = po.sa_run(po.Instance.from_text("0 0 0.7\n"), betas, 8, 2, 4)
    e1, p1 = tb.sa_run(d, betas, 8, 2, 4, tb.MODE_REF)
    assert np.array_equal(_bits(e0), _bits(e1))
    assert np.array_equal(tb.unpack_bits(p1, 1), s0)
    e2, _ = tb.sa_run(d, betas, 64, 1, 4, tb.MODE_FAST)
    assert np.all(e2 == np.float32(-0.7))  # the ground state, reached by every restart at beta = 10


@pytest.mark.parametrize("threads", [1, 5])
def test_ref_odd_chains_single_temperature(tb, po, gpu, threads):
    text = gi.lattice(6, 2, "gauss", 5)
    betas = np.array([1.5], np.float32)
    _ref_vs_oracle(tb, po, gpu, text, betas, 30, 0.3, 0, True, 3, threads, 3, 4, 0, 8)


@pytest.mark.parametrize("threads", [1, 4])
def test_ref_single_sweep(tb, po, gpu, threads):
    text = gi.lattice(8, 2, "pm", 2)
    betas = tb.geometric_betas(0.2, 5.0, 12)
    _ref_vs_oracle(tb, po, gpu, text, betas, 1, 0.0, 6, True, 2, threads, 1, 1, 1, 21)


def test_fast_single_sweep_and_largest_shape(tb, po, gpu):
    text = gi.lattice(4, 2, "gauss", 9)
    inst = po.Instance.from_text(text)
    d = gpu.upload(tb.HostInstance.parse(text))
    # 64 temperatures x 32 chains = 2048 replicas: the largest fast-mode run
    for sweeps, chains in ((1, 2), (20, 32)):
        betas = tb.geometric_betas(0.2, 5.0, 64)
        p = tb.PtParams(sweeps, betas, 32, 0.5, True, chains, 8, None, None, 0)
        S, E = tb.PtRun(d, p, 12).run().sync().state()
        ef = np.array([[inst.energy_f64(S[c, t]) for t in range(64)] for c in range(chains)])
        assert np.all(np.abs(E - ef) <= 1e-5 * np.maximum(np.abs(ef), 1.0))


def test_fast_rejects_shapes_beyond_its_limits(tb, gpu):
    d = gpu.upload(tb.HostInstance.parse(gi.lattice(4, 2, "gauss", 9)))
    with pytest.raises(tb.TamcError) as e:  # 65 temperatures per chain
        tb.PtRun(d, tb.PtParams(5, tb.geometric_betas(0.2, 5.0, 65), 0, 0.5, True, 2, 8), 1)
    assert e.value.code == -7
    with pytest.raises(tb.TamcError) as e:  # 34 chains x 64 temperatures > 2048 replicas
        tb.PtRun(d, tb.PtParams(5, tb.geometric_betas(0.2, 5.0, 64), 0, 0.5, True, 34, 8), 1)
    assert e.value.code == -7


def test_instance_without_sites_is_refused(tb, gpu):
    h = tb.HostInstance.parse("")
    assert h.n == 0
    with pytest.raises(tb.TamcError) as e:
        gpu.upload(h)
    assert e.value.code == -1
