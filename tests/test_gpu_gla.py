"""GLA partitioned solves (run_gla, src/gla.rs:121-195) on the GPU.

Reference order: every sub-instance replayed on its jumped Xoshiro256++
stream must give the oracle's partition energies, boundary energies (same
groups, same order), total energy and joined state bit for bit.  Colour
order: all sub-instances in one batch; the joined state's FP64 energy equals
the reported total within 1e-5 relative.  The CLI writes GlaResults in
bincode and pickle like the reference's write_data."""
import pickle
import subprocess

import numpy as np
import pytest

from tamc_b200 import instances as gi

pytestmark = pytest.mark.gpu


def _blocks(L, k):
    """k x k blocks of an L x L lattice (site index x*L + y), in a scrambled order."""
    rng = np.random.default_rng(L + k)
    parts = [[] for _ in range(k * k)]
    for x in range(L):
        for y in range(L):
            parts[(x * k // L) * k + (y * k // L)].append(x * L + y)
    for p in parts:
        rng.shuffle(p)  # the file order of a partition's sites does not matter
    order = rng.permutation(len(parts))
    return [parts[i] for i in order]


def _text(parts):
    return "\n".join(" ".join(str(i) for i in p) for p in parts) + "\n"


def _params(tb, po, nt=8, sweeps=120, chains=2, threads=4, sample=None):
    b = po.geometric_betas(0.2, 5.0, nt)
    return b, po.lo_beta_idx(b, lo_beta=1.0), tb.PtParams(sweeps, b, po.lo_beta_idx(b, lo_beta=1.0), 0.5, True,
                                                         chains, threads, sample, None, 0)


@pytest.mark.parametrize("case", ["2d_pm_blocks", "qubo_random_parts", "3d_gauss_slabs"])
def test_gla_reference_order_matches_oracle(tb, po, gpu, case):
    if case == "2d_pm_blocks":
        text, qubo, parts = gi.lattice(12, 2, "pm", 4), False, _blocks(12, 3)
    elif case == "qubo_random_parts":
        text, qubo = gi.qubo_er(90, 5, 7), True
        rng = np.random.default_rng(3)
        lab = rng.integers(0, 5, 90)
        parts = [np.flatnonzero(lab == k).tolist() for k in range(5)]
    else:
        text, qubo = gi.lattice(6, 3, "gauss", 2), False
        parts = [list(range(72 * k, 72 * (k + 1))) for k in range(3)]
    h = tb.HostInstance.parse(text, qubo=qubo)
    part = tb.Partition.parse(_text(parts), h.n)
    assert part.parts == parts
    b, lo, p = _params(tb, po, sample=7)
    r = tb.gla_run(gpu, h, part, p, 21, tb.MODE_REF)
    o = po.gla_run(po.Instance.from_text(text, qubo=qubo), parts, b, p.num_sweeps, 0.5, lo, True, 2, sample=7,
                   seed=21)
    assert r.instance_size == h.n and r.num_partitions == len(parts)
    assert np.array_equal(r.partition_energies.view(np.uint32), o["partition_energies"].view(np.uint32))
    assert [(a, c) for a, c, _ in r.boundary_energies] == [(a, c) for a, c, _ in o["boundary_energies"]]
    assert np.array_equal(np.array([e for _, _, e in r.boundary_energies], np.float32).view(np.uint32),
                          o["bnd_energies"].view(np.uint32))
    assert np.float32(r.total_energy).view(np.uint32) == o["total_energy"].view(np.uint32)
    assert np.array_equal(r.state, o["state"])
    if not qubo:  # sub-instances drop the offset; without one the total is the joined state's energy
        assert abs(po.Instance.from_text(text).energy_f64(r.state) - r.total_energy) <= 1e-5 * abs(r.total_energy)


def test_gla_colour_order_batch(tb, po, gpu):
    text = gi.lattice(16, 2, "gauss", 9)
    h = tb.HostInstance.parse(text)
    parts = _blocks(16, 4)
    b, lo, p = _params(tb, po, nt=16, sweeps=400)
    r = tb.gla_run(gpu, h, tb.Partition.parse(_text(parts), h.n), p, 5, tb.MODE_FAST)
    inst = po.Instance.from_text(text)
    e = inst.energy_f64(r.state)
    assert abs(e - r.total_energy) <= 1e-5 * abs(e)
    # each partition energy is its sub-instance's energy of the joined state's restriction
    for k, pk in enumerate(parts):
        sub = sorted(pk)
        sinst = tb.HostInstance.parse(text)
        rp, col, J, bias = sinst.csr()
        es = 0.0
        for i in sub:
            f = bias[i]
            for x in range(rp[i], rp[i + 1]):
                if col[x] in pk:
                    f += J[x] * r.state[col[x]] / 2
            es += f * r.state[i]
        assert abs(es - r.partition_energies[k]) <= 1e-4 * max(1.0, abs(es))
    assert len(r.boundary_energies) > 0
    # deterministic for a fixed seed
    r2 = tb.gla_run(gpu, h, tb.Partition.parse(_text(parts), h.n), p, 5, tb.MODE_FAST)
    assert np.array_equal(r.state, r2.state) and r.total_energy == r2.total_energy


def test_gla_reference_panics(tb, po, gpu):
    b, lo, p = _params(tb, po, sweeps=20)
    h = tb.HostInstance.parse(gi.lattice(6, 2, "pm", 1))
    with pytest.raises(tb.TamcError) as e:  # site 35 in no partition
        tb.gla_run(gpu, h, tb.Partition.parse("0 1 2 3\n" + " ".join(map(str, range(4, 35))) + "\n", 36), p, 1,
                   tb.MODE_REF)
    assert e.value.code == -8
    h2 = tb.HostInstance.parse("0 1 1.0\n1 2 -1.0\n3 3 0.5\n")  # the last site has no coupling
    with pytest.raises(tb.TamcError) as e:
        tb.gla_run(gpu, h2, tb.Partition.parse("0 1\n2 3\n", 4), p, 1, tb.MODE_REF)
    assert e.value.code == -8


def _decode_gla_bincode(b):
    import struct
    o = 0

    def take(fmt):
        nonlocal o
        v = struct.unpack_from("<" + fmt, b, o)
        o += struct.calcsize("<" + fmt)
        return v if len(v) > 1 else v[0]
    out = {"instance_size": take("I"), "num_partitions": take("I")}
    out["partition_energies"] = [take("f") for _ in range(take("Q"))]
    out["boundary_energies"] = [take("IIf") for _ in range(take("Q"))]
    out["final_state"] = [take("B") for _ in range(take("Q"))]
    out["total_energy"] = take("f")
    assert o == len(b)
    return out


def test_cli_gla_writes_results_like_the_reference(tb, po, tmp_path):
    text = gi.lattice(10, 2, "pm", 6)
    parts = _blocks(10, 2)
    (tmp_path / "i.txt").write_text(text)
    (tmp_path / "parts.txt").write_text(_text(parts))
    (tmp_path / "m.yml").write_text(f"""GLA:
  num_threads: 4
  partition_file: {tmp_path / "parts.txt"}
  pt_params:
    num_sweeps: 80
    warmup_fraction: 0.5
    beta:
      Geometric:
        beta_min: 0.2
        beta_max: 5.0
        num_beta: 8
    lo_beta: 1.0
    icm: true
    num_replica_chains: 2
    threads: 4
""")
    outs = {}
    for out in ("r.bin", "r.pkl"):
        cmd = [tb.CLI_PATH, str(tmp_path / "m.yml"), str(tmp_path / "i.txt"), str(tmp_path / out), "--seed", "9",
               "--mode", "ref"]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        assert "tamc finished successfully" in r.stdout and "Total energy" in r.stderr
        outs[out] = (tmp_path / out).read_bytes()
    bn = _decode_gla_bincode(outs["r.bin"])
    pk = pickle.loads(outs["r.pkl"])
    b = po.geometric_betas(0.2, 5.0, 8)
    o = po.gla_run(po.Instance.from_text(text), parts, b, 80, 0.5, po.lo_beta_idx(b, lo_beta=1.0), True, 2, seed=9)
    assert bn["instance_size"] == pk["instance_size"] == 100
    assert bn["num_partitions"] == pk["num_partitions"] == 4
    assert np.array_equal(np.array(bn["partition_energies"], np.float32), o["partition_energies"])
    assert pk["partition_energies"] == [float(x) for x in o["partition_energies"]]
    want = [(a, c, float(e)) for a, c, e in o["boundary_energies"]]
    assert [(a, c, float(np.float32(e))) for a, c, e in bn["boundary_energies"]] == want
    assert [tuple(x) for x in pk["boundary_energies"]] == want and isinstance(pk["boundary_energies"][0], tuple)
    assert bn["final_state"] == [] and pk["final_state"] == []
    assert np.float32(bn["total_energy"]) == o["total_energy"] and pk["total_energy"] == float(o["total_energy"])
