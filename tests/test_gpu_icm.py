"""Colour-ordered (fast) mode: the on-device Houdayer cluster move is integer
work and must pick and flip exactly the cluster a CPU breadth-first search
picks, in the fused and in the plain form, with either cluster search (frontier
BFS from the seeds, or union-find labelling of the whole subgraph).

With every coupling and bias zero, each Metropolis flip has dE = 0 and is
accepted and every exchange has probability one, so one PT round is: the
Houdayer move on each chain pair and slot >= lo, a permutation of slots inside
each chain, and one sweep that flips every spin.  The expected states follow
from the initial states alone: the seed site is the k-th disagreeing site in
colour order, k = (u * count) >> 32 with u the first word of
Philox4x32-10(counter = (slot, round, pair, 'IC'), key = seed), and the
cluster is the seed's connected component of the disagreement subgraph
(src/pt.rs:31-77 grows the same cluster by BFS over the coupling graph).
"""
import numpy as np
import pytest

from tamc_b200 import instances as gi

pytestmark = pytest.mark.gpu

PTAG_ICM = 0x4943
M32 = 0xFFFFFFFF


def philox4x32_10(ctr, key):
    """Philox4x32-10 (Salmon et al., SC'11), one block."""
    c0, c1, c2, c3 = ctr
    k0, k1 = key
    for _ in range(10):
        p0 = 0xD2511F53 * c0
        p1 = 0xCD9E8D57 * c2
        c0, c1, c2, c3 = ((p1 >> 32) ^ c1 ^ k0) & M32, p1 & M32, ((p0 >> 32) ^ c3 ^ k1) & M32, p0 & M32
        k0 = (k0 + 0x9E3779B9) & M32
        k1 = (k1 + 0xBB67AE85) & M32
    return c0, c1, c2, c3


def zero_coupling_text(text):
    rows = [ln.split() for ln in text.strip().splitlines()]
    return "".join(f"{a} {b} 0.0\n" for a, b, _ in rows)


def neighbours(text, n):
    adj = [set() for _ in range(n)]
    for ln in text.strip().splitlines():
        a, b, _ = ln.split()
        a, b = int(a), int(b)
        if a != b:
            adj[a].add(b)
            adj[b].add(a)
    return adj


def expected_round(S0, adj, colour, lo, seed):
    """One round at zero couplings: Houdayer move per (pair, slot >= lo), then every spin flipped."""
    C, nt, n = S0.shape
    order = np.argsort(colour, kind="stable")  # colour-ordered index -> site
    S = S0.copy()
    key = (seed & M32, seed >> 32)
    for p in range(C // 2):
        for t in range(lo, nt):
            a, b = S[2 * p, t], S[2 * p + 1, t]
            dis = [s for s in order if a[s] != b[s]]  # colour order
            if not dis:
                continue
            u = philox4x32_10((t, 0, p, PTAG_ICM), key)[0]
            k = (u * len(dis)) >> 32
            start = dis[k]
            seen = {start}
            stack = [start]
            while stack:
                x = stack.pop()
                for y in adj[x]:
                    if y not in seen and a[y] != b[y]:
                        seen.add(y)
                        stack.append(y)
            idx = np.fromiter(seen, np.int64)
            a[idx] *= -1
            b[idx] *= -1
    return -S


def _case(kind):
    if kind == "2d_L16":
        return gi.lattice(16, 2, "pm", 1), 16 * 16
    if kind == "2d_L32":
        return gi.lattice(32, 2, "pm", 2), 32 * 32
    if kind == "3d_L8":
        return gi.lattice(8, 3, "gauss", 3), 8 ** 3
    if kind == "regular":
        return gi.to_text(300, [(a, b, 1.0) for a, b in gi.random_regular(300, 3, 4)]), 300
    raise ValueError(kind)


@pytest.mark.parametrize("search", ["bfs", "uf"])
@pytest.mark.parametrize("form", ["fused", "plain"])
@pytest.mark.parametrize("kind,nt,C", [("2d_L16", 32, 2), ("2d_L32", 24, 4), ("3d_L8", 16, 2), ("regular", 40, 2)])
def test_fast_icm_cluster_matches_cpu_bfs(tb, gpu, monkeypatch, form, search, kind, nt, C):
    text, n = _case(kind)
    text = zero_coupling_text(text)
    h = tb.HostInstance.parse(text)
    assert h.n == n
    _, colour = h.coloring()
    adj = neighbours(text, n)
    lo = nt // 3
    betas = np.linspace(0.2, 3.0, nt).astype(np.float32)
    p = tb.PtParams(1, betas, lo, 0.0, True, C, 4, None, None, 0)
    seed = 0x1234_5678_9ABC_DEF1
    rng = np.random.default_rng(n + nt)
    monkeypatch.setenv("TAMC_PT_FORM", form)
    monkeypatch.setenv("TAMC_ICM", search)
    for trial in range(2):
        # mixes of heavy and light disagreement: large percolating clusters and small ones
        frac = rng.uniform(0.2, 0.8, size=(C // 2, nt, 1))
        base = rng.choice(np.array([-1, 1], np.int8), size=(C, nt, n))
        flip = rng.random((C // 2, nt, n)) < frac
        base[1::2] = np.where(flip, -base[0::2], base[0::2])
        run = tb.PtRun(gpu.upload(h), p, seed)
        run.set_state(base)
        run.run().sync()
        S, E = run.state()
        want = expected_round(base.astype(np.int64), adj, colour, lo, seed)
        assert np.all(E == 0)
        for c in range(C):
            # exchange permutes the slots of a chain: compare the sets of states
            got = sorted(r.tobytes() for r in S[c].astype(np.int8))
            exp = sorted(r.tobytes() for r in want[c].astype(np.int8))
            assert got == exp, (kind, form, trial, c)
