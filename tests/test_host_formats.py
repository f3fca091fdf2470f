"""Host-side boundary (no GPU): instance parser quirks, QUBO conversion, YAML
method files, beta ladders, colouring, and the C ABI's exported symbols."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def _same_csr(tb, po, text, qubo=False):
    a = tb.HostInstance.parse(text, qubo=qubo)
    b = po.Instance.from_text(text, qubo=qubo)
    assert a.n == b.n and a.nnz == b.nnz
    assert np.float32(a.offset).view(np.uint32) == np.float32(b.offset).view(np.uint32)
    for x, y in zip(a.csr(), b.csr()):
        assert np.array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))
    assert a.graph_nodes == b.graph_nodes
    return a


PARSER_CASES = {
    "exponent_prefix_only": "0 1 1e-5\n1 2 -2.5\n",          # K parses as 1 (exponent ignored)
    "plus_sign_ignored": "0 1 +1.0\n1 2 1.0\n",              # '+' line is ignored
    "leading_dot_ignored": "0 1 .5\n0 2 1\n",
    "trailing_dot": "  3 4 -2.\n",
    "tabs": "0\t1\t0.5\n",
    "comments_ignored": "# header\n0 1 1.0\n% other\n",
    "duplicates_overwrite": "0 1 1.0\n1 0 2.0\n0 1 3.0\n",
    "bias_line": "0 1 1.0\n2 2 0.5\n",
    "trailing_text": "0 1 1.5 extra text\n1 2 -0.25;\n",
    "crlf": "0 1 1.0\r\n1 2 -1.0\r\n",
    "isolated_last_site": "0 1 1.0\n5 5 0.25\n",
    "empty": "",
    "many_digits": "0 1 0.123456789012345678901234567890\n",
}


@pytest.mark.parametrize("name", sorted(PARSER_CASES))
def test_parser_matches_oracle(tb, po, name):
    _same_csr(tb, po, PARSER_CASES[name])


def test_parser_known_values(tb):
    a = tb.HostInstance.parse(PARSER_CASES["exponent_prefix_only"])
    rp, col, J, h = a.csr()
    assert J[0] == 1.0 and a.n == 3
    a = tb.HostInstance.parse(PARSER_CASES["plus_sign_ignored"])
    assert a.n == 3 and a.nnz == 2
    a = tb.HostInstance.parse(PARSER_CASES["duplicates_overwrite"])
    rp, col, J, h = a.csr()
    assert list(J) == [3.0, 3.0]
    a = tb.HostInstance.parse(PARSER_CASES["bias_line"])
    rp, col, J, h = a.csr()
    assert a.n == 3 and h[2] == 0.5 and a.nnz == 2
    a = tb.HostInstance.parse(PARSER_CASES["isolated_last_site"])
    assert a.n == 6 and a.graph_nodes == 2


def test_parser_overflow_is_an_error(tb):
    with pytest.raises(tb.TamcError):
        tb.HostInstance.parse("0 99999999999 1.0\n")


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_qubo_conversion_matches_oracle(tb, po, seed):
    from tamc_b200 import instances as gi
    a = _same_csr(tb, po, gi.qubo_er(40, 6, seed), qubo=True)
    rp, col, J, h = a.csr()
    # the reference keeps the diagonal as a self-coupling (src/ising.rs:308-310)
    self_loops = sum(1 for i in range(a.n) for e in range(rp[i], rp[i + 1]) if col[e] == i)
    assert self_loops == a.n


def test_generators_round_trip(tb, po):
    from tamc_b200 import instances as gi
    for text in (gi.lattice(6, 2, "pm", 1), gi.lattice(4, 3, "gauss", 2), gi.sa_regular(100, 3, 3)):
        _same_csr(tb, po, text)


def test_energy_ref_matches_oracle(tb, po):
    from tamc_b200 import instances as gi
    text = gi.qubo_er(30, 5, 4)
    a = tb.HostInstance.parse(text, qubo=True)
    b = po.Instance.from_text(text, qubo=True)
    rng = np.random.default_rng(1)
    for _ in range(10):
        s = rng.choice(np.array([-1, 1], np.int8), a.n)
        assert np.float32(a.energy_ref(s)).view(np.uint32) == np.float32(b.energy_ref(s)).view(np.uint32)


def test_coloring_is_proper(tb):
    from tamc_b200 import instances as gi
    for text in (gi.lattice(8, 2, "pm", 1), gi.lattice(5, 2, "pm", 1), gi.sa_regular(200, 3, 1),
                 gi.qubo_er(100, 6, 1)):
        a = tb.HostInstance.parse(text)
        nc, col = a.coloring()
        rp, c, _, _ = a.csr()
        for i in range(a.n):
            for e in range(rp[i], rp[i + 1]):
                if c[e] != i:
                    assert col[i] != col[c[e]]
        assert col.max() < nc
    nc, col = tb.HostInstance.parse(gi.lattice(8, 2, "pm", 1)).coloring()
    assert nc == 2 and np.bincount(col).tolist() == [32, 32]


PT_YAML = """---
PT:
  num_sweeps: 2000
  warmup_fraction: 0.5
  beta:
    Geometric:
      beta_min: 0.2
      beta_max: 5.0
      num_beta: 32
  lo_beta: 1.0
  icm: true
  num_replica_chains: 2
  threads: 1
  sample: 32
  sample_states: 32
  sample_limiting: 2
"""


def test_method_pt(tb, po):
    p = tb.Method.parse(PT_YAML).pt()
    assert p.num_sweeps == 2000 and p.warmup_fraction == 0.5 and p.icm and p.num_replica_chains == 2
    assert p.sample == 32 and p.sample_states == 32 and p.sample_limiting == 2 and p.threads == 1
    assert np.array_equal(p.betas, po.geometric_betas(0.2, 5.0, 32))
    assert p.lo_beta_idx == po.lo_beta_idx(p.betas, lo_beta=1.0)


def test_method_variants(tb, po):
    y = PT_YAML.replace("  sample: 32\n", "").replace("lo_beta: 1.0", "lo_num_beta: 4\n  lo_beta: 1.0")
    p = tb.Method.parse(y).pt()
    assert p.sample is None and p.lo_beta_idx == 28
    y = """PT: {num_sweeps: 10, warmup_fraction: 0.1, beta: {Arr: [0.1, 0.5, 1.0]}, lo_beta: 0.5,
  icm: false, num_replica_chains: 4, threads: 8}  # flow style
"""
    p = tb.Method.parse(y).pt()
    assert list(p.betas) == [np.float32(0.1), np.float32(0.5), np.float32(1.0)] and p.lo_beta_idx == 1
    y = "SA:\n  beta:\n    Arr:\n      - 0.1\n      - 0.2\n  num_replicas: 16\n  threads: 4\n"
    m = tb.Method.parse(y)
    b, r, t = m.sa()
    assert m.kind == "SA" and r == 16 and t == 4 and list(b) == [np.float32(0.1), np.float32(0.2)]


@pytest.mark.parametrize("yaml_text,code", [
    (PT_YAML.replace("  icm: true\n", ""), -5),                          # missing field
    (PT_YAML.replace("Geometric", "Linear"), -5),                        # unknown variant
    (PT_YAML.replace("  lo_beta: 1.0\n", ""), -8),                         # icm without lo_beta: reference panics
    ("PT:\n  num_sweeps: 1\n  warmup_fraction: 0.5\n  beta: {Arr: [1.0, 0.5]}\n  icm: false\n"
     "  num_replica_chains: 2\n  threads: 1\n", -8),                     # decreasing betas
    ("XX: 1\n", -5),
])
def test_method_errors(tb, yaml_text, code):
    with pytest.raises(tb.TamcError) as e:
        tb.Method.parse(yaml_text)
    assert e.value.code == code


def test_geometric_betas_match_oracle(tb, po):
    for spec in [(0.2, 5.0, 32), (0.1, 10.0, 64), (0.3, 4.0, 6), (1.0, 1.0, 3)]:
        assert np.array_equal(tb.geometric_betas(*spec), po.geometric_betas(*spec))


def _header_functions():
    h = open(os.path.join(ROOT, "include", "tamc_gpu.h")).read()
    h = re.sub(r"/\*.*?\*/", "", h, flags=re.S)
    return sorted(set(re.findall(r"\b(tamc_\w+)\s*\(", h)))


def test_library_exports_every_header_symbol(tb):
    L = ctypes.CDLL(tb.LIB_PATH)
    names = _header_functions()
    assert len(names) > 50
    for name in names:
        assert hasattr(L, name), name
    assert sorted(tb.exported_symbols()) == names


def test_ref_expf_matches_glibc(tb):
    libm = ctypes.CDLL("libm.so.6")
    libm.expf.restype = ctypes.c_float
    libm.expf.argtypes = [ctypes.c_float]
    rng = np.random.default_rng(0)
    xs = np.concatenate([
        -rng.exponential(3.0, 40000), rng.uniform(-110, 89, 40000), -np.abs(rng.standard_normal(20000)) * 1e-3,
        np.array([0.0, -0.0, -87.3, -103.97, -104.0, 88.72, 89.0, -110.0, -200.0]),
    ]).astype(np.float32)
    # plus every exception-table key
    table = os.path.join(ROOT, "_build", "tamc_b200", "expf_table.bin")
    if os.path.exists(table):
        raw = np.fromfile(table, np.uint32)
        nb, ne = int(raw[1]), int(raw[2])
        keys = raw[3 + nb + 1: 3 + nb + 1 + ne]
        xs = np.concatenate([xs, keys.view(np.float32)[::7]])
    L = tb.lib()
    bad = [x for x in xs if np.float32(L.tamc_ref_expf(float(x))).view(np.uint32)
           != np.float32(libm.expf(float(x))).view(np.uint32)]
    assert not bad, bad[:5]


def _py_read_u32_lines(text):
    """read_u32_lines (src/util.rs:142-172) restated: per line, whitespace-separated
    leading u32 values (space0 before, multispace0 after each), the rest ignored;
    lines without a leading value skipped."""
    out = []
    for line in text.split("\n"):
        if line.endswith("\r"):
            line = line[:-1]  # BufRead::lines strips "\r\n"
        vals, k = [], 0
        while True:
            j = k
            while j < len(line) and line[j] in " \t":
                j += 1
            m = j
            while m < len(line) and line[m].isdigit() and line[m].isascii():
                m += 1
            if m == j:
                break
            vals.append(int(line[j:m]))
            while m < len(line) and line[m] in " \t\r\n":
                m += 1
            k = m
        if vals:
            out.append(vals)
    return out


@pytest.mark.parametrize("text", [
    "0 1 2\n3 4 5\n",
    "  0\t1  \r\n2 3 4\r\n\n\n5\n",
    "0 1 x 9\n# comment 2\n2,3\n4 5",
    "5 4 3\n\n2 1 0 \n",
    "",
])
def test_partition_parse_matches_restatement(tb, text):
    p = tb.Partition.parse(text, 10)
    assert p.parts == _py_read_u32_lines(text)


def test_partition_errors_follow_read_graph_partition(tb):
    with pytest.raises(tb.TamcError) as e:
        tb.Partition.parse("0 1\n2 10\n", 10)
    assert e.value.code == -1 and "Found index 10" in str(e.value)
    with pytest.raises(tb.TamcError) as e:
        tb.Partition.parse("0 1\n2 1\n", 10)
    assert e.value.code == -1 and "Index 1 specified more than once in partition 1" in str(e.value)
    with pytest.raises(tb.TamcError) as e:  # u32::from_str(..).unwrap() panics
        tb.Partition.parse("0 99999999999\n", 10)
    assert e.value.code == -8
    with pytest.raises(tb.TamcError) as e:
        tb.Partition.read("/nonexistent/parts.txt", 10)
    assert e.value.code == -6


def test_gla_method_file(tb):
    m = tb.Method.parse("""GLA:
  num_threads: 6
  pt_params:
    num_sweeps: 100
    warmup_fraction: 0.25
    beta:
      Arr: [0.1, 0.5, 1.0, 2.0]
    lo_num_beta: 2
    icm: true
    num_replica_chains: 4
    threads: 3
    sample: 10
  partition_file: "parts/p.txt"
""")
    assert m.kind == "GLA"
    nt, pf, p = m.gla()
    assert nt == 6 and pf == "parts/p.txt"
    assert p.num_sweeps == 100 and p.lo_beta_idx == 2 and p.num_replica_chains == 4 and p.sample == 10
    assert np.array_equal(p.betas, np.array([0.1, 0.5, 1.0, 2.0], np.float32))
    with pytest.raises(tb.TamcError):
        tb.Method.parse("GLA:\n  num_threads: 1\n  partition_file: x\n")  # pt_params missing
