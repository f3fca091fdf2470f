"""Reference-order mode (TAMC_MODE_REF) on the GPU against the golden fixtures
and the live CPU oracle: spin states, cached f32 energies, ICM choices,
exchange decisions (acceptance counts, round-trip tags), the ground-state
trajectory and every thermal sample must be bit-exact."""
import numpy as np
import pytest

from conftest import load_golden
from test_oracle import PT_GOLDEN, SA_GOLDEN

pytestmark = pytest.mark.gpu


def _pt_params(tb, g):
    return tb.PtParams(num_sweeps=int(g["sweeps"]), betas=g["betas"], lo_beta_idx=int(g["lo"]),
                       warmup_fraction=0.5, icm=True, num_replica_chains=int(g["chains"]),
                       threads=int(g["threads"]), sample=int(g["sample"]), sample_states=int(g["sample_states"]),
                       sample_limiting=int(g["level"]))


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("name", PT_GOLDEN)
def test_ref_pt_matches_golden(tb, gpu, name):
    g = load_golden(name)
    inst = tb.HostInstance.parse(bytes(g["text"]).decode(), qubo=bool(g["qubo"]))
    for w in g["suscept"]:
        inst.add_suscept(w)
    run = tb.PtRun(gpu.upload(inst), _pt_params(tb, g), int(g["seed"]), tb.MODE_REF).run().sync()
    S, E = run.state()
    assert np.array_equal(S, g["spins"])
    assert np.array_equal(_bits(E), _bits(g["energies"]))
    # acceptance_counts = per-chain counts summed over chains (count_acc, src/pt.rs:585-591)
    assert np.array_equal(run.acceptance(), g["acceptance"].sum(0))
    tags, rts, dh = run.round_trips()
    assert np.array_equal(tags, g["tags"]) and np.array_equal(rts, g["round_trips"])
    assert np.array_equal(dh, g["dhist"])
    steps, en, st = run.gs()
    assert np.array_equal(steps, g["gs_steps"])
    assert np.array_equal(_bits(en), _bits(g["gs_energies"]))
    assert np.array_equal(st, g["gs_states"])
    ts = run.samples()
    assert np.array_equal(_bits(np.array(ts.e)), _bits(g["e"]))
    assert np.array_equal(np.array(ts.q), g["q"])
    if len(g["suscept"]):
        assert np.array_equal(_bits(np.array(ts.suscept)), _bits(g["sus"]))
    assert np.array_equal(np.array(ts.samples).reshape(g["samples"].shape), g["samples"])


@pytest.mark.parametrize("name", SA_GOLDEN)
def test_ref_sa_matches_golden(tb, gpu, name):
    g = load_golden(name)
    inst = tb.HostInstance.parse(bytes(g["text"]).decode(), qubo=bool(g["qubo"]))
    e, packed = tb.sa_run(gpu.upload(inst), g["betas"], int(g["num_replicas"]), int(g["threads"]), int(g["seed"]),
                          tb.MODE_REF)
    assert np.array_equal(_bits(e), _bits(g["energies"]))
    assert np.array_equal(tb.unpack_bits(packed, inst.n), g["spins"])


@pytest.mark.parametrize("threads", [1, 5])
@pytest.mark.parametrize("seed", [3, 2024])
def test_ref_pt_live_oracle_chunked(tb, po, gpu, threads, seed):
    """Runs in uneven chunks (resumable) against the oracle after every chunk."""
    from tamc_b200 import instances as gi
    text = gi.lattice(6, 2, "gauss", seed)
    b = po.geometric_betas(0.25, 4.0, 10)
    lo = po.lo_beta_idx(b, lo_beta=1.0)
    orc = po.PtRun(po.Instance.from_text(text), b, 45, 0.4, lo, True, 4, threads, sample=3, sample_states=4,
                   sample_limiting=1, seed=seed)
    p = tb.PtParams(45, b, lo, 0.4, True, 4, threads, 3, 4, 1)
    run = tb.PtRun(gpu.upload(tb.HostInstance.parse(text)), p, seed, tb.MODE_REF)
    for end in (1, 7, 20, 45):
        orc.run(end)
        run.run(end).sync()
        S0, E0, _ = orc.states()
        S1, E1 = run.state()
        assert np.array_equal(S0, S1), end
        assert np.array_equal(_bits(E0), _bits(E1)), end
    assert np.array_equal(orc.acceptance().sum(0), run.acceptance())


def test_ref_qubo_self_loop_quirk(tb, po, gpu):
    from tamc_b200 import instances as gi
    text = gi.qubo_er(30, 5, 17)
    b = po.geometric_betas(0.1, 1.5, 6)
    orc = po.PtRun(po.Instance.from_text(text, qubo=True), b, 25, 0.5, 2, True, 2, 3, sample=2, seed=9)
    orc.run()
    p = tb.PtParams(25, b, 2, 0.5, True, 2, 3, 2, None, 0)
    run = tb.PtRun(gpu.upload(tb.HostInstance.parse(text, qubo=True)), p, 9, tb.MODE_REF).run().sync()
    S0, E0, _ = orc.states()
    S1, E1 = run.state()
    assert np.array_equal(S0, S1)
    assert np.array_equal(_bits(E0), _bits(E1))


def test_ref_isolated_seed_site_reports_reference_panic(tb, gpu):
    # the highest-index site has no coupling: petgraph's node range ends before
    # it and the reference panics when ICM picks it; the backend reports it.
    text = "0 1 1.0\n1 2 -1.0\n3 3 0.5\n"
    p = tb.PtParams(50, np.array([0.1, 0.2], np.float32), 0, 0.0, True, 2, 1)
    run = tb.PtRun(gpu.upload(tb.HostInstance.parse(text)), p, 1, tb.MODE_REF)
    with pytest.raises(tb.TamcError) as e:
        run.run().sync()
    assert e.value.code == -8
