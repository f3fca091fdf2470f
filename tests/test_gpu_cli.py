"""The tamc_b200 CLI as a drop-in for `tamc`: same arguments and result files.
Reference-order runs are compared with the oracle value by value; the binary
layouts are decoded independently with `struct` (bincode) and `pickle`."""
import os
import pickle
import struct
import subprocess

import numpy as np
import pytest
import yaml

from tamc_b200 import instances as gi

pytestmark = pytest.mark.gpu


class Bin:
    def __init__(self, b):
        self.b, self.o = b, 0

    def take(self, fmt):
        v = struct.unpack_from("<" + fmt, self.b, self.o)
        self.o += struct.calcsize("<" + fmt)
        return v if len(v) > 1 else v[0]

    def vec(self, f):
        return [f() for _ in range(self.take("Q"))]


def decode_thermal(b):
    r = Bin(b)
    out = {"compression_level": r.take("B"), "instance_size": r.take("Q")}
    out["beta_arr"] = r.vec(lambda: r.take("f"))
    out["samples"] = r.vec(lambda: r.vec(lambda: bytes(r.vec(lambda: r.take("B")))))
    out["e"] = r.vec(lambda: r.vec(lambda: r.take("f")))
    out["q"] = r.vec(lambda: r.vec(lambda: r.take("i")))
    out["suscept"] = r.vec(lambda: r.vec(lambda: r.vec(lambda: r.take("f"))))
    assert r.o == len(b)
    return out


METHOD = """---
PT:
  num_sweeps: 60
  warmup_fraction: 0.5
  beta:
    Geometric:
      beta_min: 0.2
      beta_max: 5.0
      num_beta: 8
  lo_beta: 1.0
  icm: true
  num_replica_chains: 2
  threads: {threads}
  sample: 4
  sample_states: 8
  sample_limiting: 0
"""


@pytest.mark.parametrize("threads", [1, 4])
def test_cli_pt_reference_mode_matches_oracle(tb, po, tmp_path, threads):
    L = 6
    text = gi.lattice(L, 2, "pm", 3)
    (tmp_path / "m.yml").write_text(METHOD.format(threads=threads))
    (tmp_path / "i.txt").write_text(text)
    w = [gi.fourier_weights(L, 2, 0), gi.fourier_weights(L, 2, 1)]
    for k, row in enumerate(w):
        (tmp_path / f"s{k}.txt").write_text(gi.weights_text(row))
    cmd = [tb.CLI_PATH, str(tmp_path / "m.yml"), str(tmp_path / "i.txt"), str(tmp_path / "out.yml"),
           "--suscepts", str(tmp_path / "s0.txt"), str(tmp_path / "s1.txt"), "--sample-output",
           str(tmp_path / "samples.bin"), "--seed", "77", "--mode", "ref"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "tamc finished successfully" in r.stdout
    res = yaml.safe_load((tmp_path / "out.yml").read_text())
    inst = po.Instance.from_text(text)
    for k in range(2):
        inst.add_suscept(po_read_vec(tmp_path / f"s{k}.txt"))
    b = po.geometric_betas(0.2, 5.0, 8)
    orc = po.PtRun(inst, b, 60, 0.5, po.lo_beta_idx(b, lo_beta=1.0), True, 2, threads, sample=4, sample_states=8,
                   sample_limiting=0, seed=77)
    orc.run()
    gs = orc.gs()
    assert res["gs_time_steps"] == [g[0] for g in gs]
    assert np.array_equal(np.array(res["gs_energies"], np.float32), np.array([g[1] for g in gs], np.float32))
    assert res["gs_states"] == [[int(x) for x in g[2]] for g in gs]
    assert res["acceptance_counts"] == orc.acceptance().sum(0).tolist()
    assert res["instance_size"] == L * L and res["num_measurements"] == 0
    assert res["params"]["beta"]["Geometric"]["num_beta"] == 8 and res["params"]["lo_num_beta"] is None
    t = decode_thermal((tmp_path / "samples.bin").read_bytes())
    e, q, sus, smp = orc.thermal(nchi=2)
    assert t["compression_level"] == 0 and t["instance_size"] == L * L
    assert np.array_equal(np.array(t["beta_arr"], np.float32), b)
    assert np.array_equal(np.array(t["e"], np.float32), np.array(e, np.float32))
    assert np.array_equal(np.array(t["q"]), np.array(q))
    assert np.array_equal(np.array(t["suscept"], np.float32), np.array(sus, np.float32))
    assert [[bytes(x) for x in z] for z in smp] == t["samples"]


def po_read_vec(path):
    return np.array([float(x) for x in open(path).read().split()], np.float64)


def test_cli_sa_outputs(tb, tmp_path):
    text = gi.sa_regular(100, 3, 1)
    (tmp_path / "i.txt").write_text(text)
    (tmp_path / "m.yml").write_text("SA:\n  beta:\n    Arr: [" + ", ".join(f"{x:.4f}" for x in np.linspace(0.1, 3, 50))
                                    + "]\n  num_replicas: 64\n  threads: 4\n")
    for out, so in (("r.yml", "gs.bin"), ("r.pkl", "gs.pkl")):
        r = subprocess.run([tb.CLI_PATH, str(tmp_path / "m.yml"), str(tmp_path / "i.txt"), str(tmp_path / out),
                            "--sample-output", str(tmp_path / so), "--seed", "5"], capture_output=True, text=True,
                           timeout=300)
        assert r.returncode == 0, r.stderr
    res = yaml.safe_load((tmp_path / "r.yml").read_text())
    assert res["params"]["num_replicas"] == 64 and len(res["energies"]) == 64
    assert res["min_energy"] == min(res["energies"])
    pk = pickle.loads((tmp_path / "r.pkl").read_bytes())
    assert pk["params"]["threads"] == 4 and len(pk["energies"]) == 64
    b = Bin((tmp_path / "gs.bin").read_bytes())
    n, nrep = b.take("I"), b.take("I")
    nbytes = b.take("Q")
    assert n == 100 and nbytes == nrep * 13
    st = pickle.loads((tmp_path / "gs.pkl").read_bytes())
    assert st["instance_size"] == 100 and len(st["bytes"]) == st["num_replicas"] * 13


def test_cli_errors(tb, tmp_path):
    (tmp_path / "m.yml").write_text("PT:\n  num_sweeps: 1\n")
    (tmp_path / "i.txt").write_text("0 1 1.0\n")
    r = subprocess.run([tb.CLI_PATH, str(tmp_path / "m.yml"), str(tmp_path / "i.txt"), str(tmp_path / "o.yml")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "tamc terminated with an error" in r.stderr
    r = subprocess.run([tb.CLI_PATH, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "--sample-output" in r.stdout


@pytest.mark.parametrize("level", [0, 1, 2])
def test_cli_pt_pickle_samples_match_bincode_and_oracle(tb, po, tmp_path, level):
    """`--sample-output x.pkl` (src/pt.rs:645-654 via write_data, src/util.rs:26-36)
    writes the same PtIcmThermalSamples as the bincode file, field by field, and
    both equal the oracle's run for every compression level."""
    L = 5
    text = gi.lattice(L, 2, "gauss", 8)
    (tmp_path / "m.yml").write_text(METHOD.format(threads=3).replace("sample_limiting: 0",
                                                                      f"sample_limiting: {level}"))
    (tmp_path / "i.txt").write_text(text)
    (tmp_path / "s0.txt").write_text(gi.weights_text(gi.fourier_weights(L, 2, 1)))
    outs = {}
    for so in ("samples.bin", "samples.pkl"):
        cmd = [tb.CLI_PATH, str(tmp_path / "m.yml"), str(tmp_path / "i.txt"), str(tmp_path / "out.yml"),
               "--suscepts", str(tmp_path / "s0.txt"), "--sample-output", str(tmp_path / so), "--seed", "31",
               "--mode", "ref"]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs[so] = (tmp_path / so).read_bytes()
    t = decode_thermal(outs["samples.bin"])
    pk = pickle.loads(outs["samples.pkl"])
    assert set(pk) == {"compression_level", "instance_size", "beta_arr", "samples", "e", "q", "suscept"}
    assert pk["compression_level"] == t["compression_level"] == level
    assert pk["instance_size"] == t["instance_size"] == L * L
    assert pk["beta_arr"] == [float(np.float32(x)) for x in t["beta_arr"]]
    assert [[bytes(x) for x in z] for z in pk["samples"]] == t["samples"]
    assert pk["e"] == [[float(np.float32(x)) for x in row] for row in t["e"]]
    assert pk["q"] == t["q"]
    assert pk["suscept"] == [[[float(np.float32(x)) for x in c] for c in row] for row in t["suscept"]]
    inst = po.Instance.from_text(text)
    inst.add_suscept(po_read_vec(tmp_path / "s0.txt"))
    b = po.geometric_betas(0.2, 5.0, 8)
    orc = po.PtRun(inst, b, 60, 0.5, po.lo_beta_idx(b, lo_beta=1.0), True, 2, 3, sample=4, sample_states=8,
                   sample_limiting=level, seed=31)
    orc.run()
    e, q, sus, smp = orc.thermal(nchi=1)
    assert np.array_equal(np.array(pk["e"], np.float32), np.array(e, np.float32))
    assert np.array_equal(np.array(pk["q"]), np.array(q))
    assert np.array_equal(np.array(pk["suscept"], np.float32), np.array(sus, np.float32))
    assert [[bytes(x) for x in z] for z in smp] == [[bytes(x) for x in z] for z in pk["samples"]]


def test_cli_sa_reference_mode_values_match_oracle(tb, po, tmp_path):
    """SA through the CLI in reference order: every energy of AnnealMinResults
    (YAML and pickle) and every ground-state sample of AnnealState (bincode and
    pickle) equal the oracle's SaRunner::run_parallel (src/sa.rs:136-199,
    src/sa.rs:242-270)."""
    text = gi.sa_regular(100, 3, 1)
    betas = np.linspace(0.1, 3, 50)
    (tmp_path / "i.txt").write_text(text)
    (tmp_path / "m.yml").write_text("SA:\n  beta:\n    Arr: [" + ", ".join(f"{x:.4f}" for x in betas)
                                    + "]\n  num_replicas: 64\n  threads: 4\n")
    for out, so in (("r.yml", "gs.bin"), ("r.pkl", "gs.pkl")):
        r = subprocess.run([tb.CLI_PATH, str(tmp_path / "m.yml"), str(tmp_path / "i.txt"), str(tmp_path / out),
                            "--sample-output", str(tmp_path / so), "--seed", "5", "--mode", "ref"],
                           capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
    inst = po.Instance.from_text(text)
    b32 = np.array([float(f"{x:.4f}") for x in betas], np.float32)
    eo, so_ = po.sa_run(inst, b32, 64, 4, 5)
    res = yaml.safe_load((tmp_path / "r.yml").read_text())
    pk = pickle.loads((tmp_path / "r.pkl").read_bytes())
    for got in (res["energies"], pk["energies"]):
        assert np.array_equal(np.array(got, np.float32).view(np.uint32), eo.view(np.uint32))
    assert np.float32(res["min_energy"]) == eo.min() == np.float32(pk["min_energy"])
    gs = [k for k in range(64) if eo[k] <= eo.min() + np.float32(1e-8)]
    want = b"".join(np.packbits(so_[k] < 0, bitorder="little").tobytes() for k in gs)
    bn = Bin((tmp_path / "gs.bin").read_bytes())
    assert (bn.take("I"), bn.take("I")) == (100, len(gs))
    assert bytes(bn.vec(lambda: bn.take("B"))) == want
    st = pickle.loads((tmp_path / "gs.pkl").read_bytes())
    assert st["instance_size"] == 100 and st["num_replicas"] == len(gs) and bytes(st["bytes"]) == want
