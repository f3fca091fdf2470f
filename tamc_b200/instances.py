"""Seeded synthetic instances in tamc's `i j K` text format.

Each edge is written once with i < j (the reader symmetrises it) and every K
is written in fixed-point notation, because the reference's parser accepts
only `-?digits(.digits)?` (src/util.rs:43-54).  Generators cover the shapes of
the benchmark workloads: periodic 2-D / 3-D lattices with +-J or Gaussian
couplings, random 3-regular graphs with Gaussian couplings and biases, and
Erdos-Renyi QUBOs with integer weights.
"""
from __future__ import annotations

import numpy as np


def _fmt(x: float) -> str:
    s = f"{x:.8f}"
    if s.startswith("-") and float(s) == 0.0:
        s = s[1:]
    return s


def to_text(n: int, edges, biases=None) -> str:
    """edges: iterable of (i, j, K); biases: optional length-n array."""
    lines = []
    if biases is not None:
        for i, h in enumerate(biases):
            lines.append(f"{i} {i} {_fmt(float(h))}")
    for i, j, k in edges:
        lines.append(f"{int(i)} {int(j)} {_fmt(float(k))}")
    if n > 0 and biases is None:
        # make sure the last site exists even when it has no written coupling
        pass
    return "\n".join(lines) + "\n"


def lattice_edges(L: int, dim: int):
    """Periodic hypercubic lattice, index (x*L + y) [*L + z], +1 neighbours per axis."""
    n = L ** dim
    idx = np.arange(n).reshape((L,) * dim)
    out = []
    for ax in range(dim):
        nb = np.roll(idx, -1, axis=ax)
        for a, b in zip(idx.ravel(), nb.ravel()):
            out.append((min(a, b), max(a, b)))
    # L = 2 produces each bond twice; keep unique pairs (the reader would overwrite)
    return sorted(set(out))


def lattice(L: int, dim: int, couplings: str, seed: int) -> str:
    rng = np.random.default_rng(seed)
    e = lattice_edges(L, dim)
    if couplings == "pm":
        J = rng.choice(np.array([-1.0, 1.0]), size=len(e))
    elif couplings == "gauss":
        J = rng.standard_normal(len(e))
    elif couplings == "ferro":
        J = -np.ones(len(e))
    else:
        raise ValueError(couplings)
    return to_text(L ** dim, [(i, j, k) for (i, j), k in zip(e, J)])


def random_regular(n: int, d: int, seed: int, max_tries: int = 1000):
    """Random d-regular simple graph by the configuration model with rejection."""
    rng = np.random.default_rng(seed)
    for _ in range(max_tries):
        stubs = np.repeat(np.arange(n), d)
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        a, b = pairs.min(1), pairs.max(1)
        if np.any(a == b):
            continue
        key = a.astype(np.int64) * n + b
        if len(np.unique(key)) != len(key):
            continue
        return sorted(zip(a.tolist(), b.tolist()))
    raise RuntimeError("could not draw a simple regular graph")


def sa_regular(n: int = 2000, d: int = 3, seed: int = 0) -> str:
    """Sparse random Ising problem: d-regular graph, J ~ N(0,1), h ~ N(0, 0.1^2)."""
    e = random_regular(n, d, seed)
    rng = np.random.default_rng(seed + 1)
    J = rng.standard_normal(len(e))
    h = 0.1 * rng.standard_normal(n)
    return to_text(n, [(i, j, k) for (i, j), k in zip(e, J)], biases=h)


def qubo_er(n: int, mean_degree: float, seed: int) -> str:
    """Erdos-Renyi QUBO: Q_ij uniform integers in [-5,5], Q_ii in [-10,10] (for --qubo)."""
    rng = np.random.default_rng(seed)
    p = mean_degree / max(n - 1, 1)
    m = rng.binomial(n * (n - 1) // 2, p)
    a = rng.integers(0, n, size=3 * m + 16)
    b = rng.integers(0, n, size=3 * m + 16)
    keep = a != b
    a, b = np.minimum(a[keep], b[keep]), np.maximum(a[keep], b[keep])
    key = np.unique(a.astype(np.int64) * n + b)[:m]
    rng.shuffle(key)
    i, j = key // n, key % n
    q = rng.integers(-5, 6, size=len(key))
    diag = rng.integers(-10, 11, size=n)
    lines = [f"{k} {k} {float(diag[k]):.1f}" for k in range(n)]
    lines += [f"{x} {y} {float(v):.1f}" for x, y, v in zip(i.tolist(), j.tolist(), q.tolist())]
    return "\n".join(lines) + "\n"


def fourier_weights(L: int, dim: int, axis: int) -> np.ndarray:
    """cos(2 pi x_axis / L) over site coordinates (index (x*L + y)[*L + z])."""
    coords = np.indices((L,) * dim).reshape(dim, -1)
    return np.cos(2 * np.pi * coords[axis] / L)


def weights_text(w) -> str:
    return "\n".join(_fmt(float(x)) for x in w) + "\n"
