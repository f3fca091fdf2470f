"""tamc-pt-opt on the GPU (src/bin/tamc-pt-opt.rs): the CLI's first ladder
update equals tamc_pt_opt_step applied to the statistics of the same batched
runs gathered through the Python API, and the CLI writes the optimised PT
method (YAML, ladder as `Arr`, num_sweeps doubled) and the round-trip-time
history (CSV rows ending in a comma)."""
import subprocess

import numpy as np
import pytest
import yaml

from tamc_b200 import instances as gi

pytestmark = pytest.mark.gpu

METHOD = """PT:
  num_sweeps: 400
  warmup_fraction: 0.5
  beta:
    Geometric:
      beta_min: 0.1
      beta_max: 3.0
      num_beta: 10
  lo_beta: 1.0
  icm: true
  num_replica_chains: 2
  threads: 4
"""


def _splitmix(seed, n):
    M = (1 << 64) - 1
    st, out = seed, []
    for _ in range(n):
        st = (st + 0x9E3779B97F4A7C15) & M
        z = st
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        out.append(z ^ (z >> 31))
    return out


def test_pt_opt_cli_first_update_and_outputs(tb, gpu, tmp_path):
    texts = [gi.lattice(6, 2, "gauss", 40 + k) for k in range(3)]
    files = []
    for k, t in enumerate(texts):
        (tmp_path / f"i{k}.txt").write_text(t)
        files.append(str(tmp_path / f"i{k}.txt"))
    (tmp_path / "m.yml").write_text(METHOD)
    seed = 12345
    cmd = [tb.PT_OPT_CLI_PATH, "--max-iters", "1", "--opt-params", str(tmp_path / "opt.yml"), "--tau-hist",
           str(tmp_path / "tau.csv"), "--seed", str(seed), str(tmp_path / "m.yml")] + files
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert "Writing to" in r.stdout
    opt = yaml.safe_load((tmp_path / "opt.yml").read_text())["PT"]
    assert opt["num_sweeps"] == 800 and opt["threads"] == 4 and opt["lo_beta"] == 1.0
    new = np.array(opt["beta"]["Arr"], np.float32)
    # the same runs through the API: iteration 0, run k seeded with the k-th SplitMix64 output
    b0 = tb.geometric_betas(0.1, 3.0, 10)
    lo = int(np.argmax(b0 >= np.float32(1.0)))
    p = tb.PtParams(400, b0, lo, 0.5, True, 2, 1)
    batch = tb.Batch(gpu)
    for k, t in enumerate(texts):
        batch.add(gpu.upload(tb.HostInstance.parse(t)), p, _splitmix(seed, 3)[k])
    batch.run()
    rts = np.array([batch.round_trips(k)[1].sum() for k in range(3)], np.uint32)
    dh = np.array([batch.round_trips(k)[2].sum(axis=0) for k in range(3)], np.uint32)
    ok, want, mom, tau, err = tb.pt_opt_step(b0, b0, rts, dh, 400, 2, 0.2, 0.85)
    assert ok and rts.sum() > 0
    assert np.array_equal(new.view(np.uint32), want.view(np.uint32))
    assert np.all(np.diff(new) > 0) and new[0] == b0[0]
    rows = (tmp_path / "tau.csv").read_text().splitlines()
    assert len(rows) == 1 and rows[0].endswith(",")
    assert np.array_equal(np.array([float(x) for x in rows[0].split(",")[:-1]], np.float32), tau)


def test_pt_opt_cli_iterates_to_a_spread_ladder(tb, tmp_path):
    """Several iterations from a ladder crowded at low beta: the optimiser moves
    interior temperatures and keeps the ladder increasing with fixed ends."""
    (tmp_path / "i.txt").write_text(gi.lattice(8, 2, "pm", 3))
    (tmp_path / "m.yml").write_text(METHOD.replace("num_beta: 10", "num_beta: 12"))
    cmd = [tb.PT_OPT_CLI_PATH, "--max-iters", "6", "--opt-params", str(tmp_path / "opt.yml"), "--tau-hist",
           str(tmp_path / "tau.csv"), "--seed", "3", str(tmp_path / "m.yml"), str(tmp_path / "i.txt")]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    b = np.array(yaml.safe_load((tmp_path / "opt.yml").read_text())["PT"]["beta"]["Arr"], np.float32)
    b0 = np.array(tb.geometric_betas(0.1, 3.0, 12))
    assert len(b) == 12 and np.all(np.diff(b) > 0) and b[0] == b0[0]
    assert abs(b[-1] - b0[-1]) <= 1e-6 * b0[-1]
    assert not np.array_equal(b, b0)
    assert 1 <= len((tmp_path / "tau.csv").read_text().splitlines()) <= 6
