"""The reference's cached-energy rule on QUBO instances, in a setting where it
can be predicted exactly (test helper, no GPU).

On a QUBO the reference keeps the diagonal as a self-coupling K_ii in the
coupling rows (src/ising.rs:308-310), so the local field of delta_energy
(src/ising.rs:468-480) includes K_ii s_i: every accepted flip adds
delta_E_true - 2 K_ii to the cached energy (src/ising.rs:225-233), which drifts
from energy_ref by -2 K_ii per flip.  A Houdayer move with a non-empty
disagreement invalidates both caches (src/pt.rs:74-75); the exchange that
follows recomputes energy_ref (tamc-core/src/pt.rs:126-129).

With every beta zero, each Metropolis proposal is accepted (every site flips
every sweep: drift -2 sum_i K_ii per sweep) and each exchange swaps
(tamc-core/src/pt.rs:132-139), so the swaps j = 0..nt-2 compose to a cyclic
shift: a state at slot p moves to p - 1, the state at slot 0 to nt - 1.  Two
chains that differ somewhere keep differing (sweeps flip both, a Houdayer move
swaps the disagreeing cluster between them), so every round's move at a slot
>= lo invalidates.  A state at slot t after round r was at slot (t + k) mod nt
at the start of round r + 1 - k; its cache was last refreshed k rounds back for
the smallest such k with that slot >= lo (k <= r + 1), else it has carried its
initial energy_ref through all r + 1 sweeps.
"""
import numpy as np


def sweeps_since_refresh(nt: int, lo: int, rounds: int) -> np.ndarray:
    """m[r][t]: sweeps the cache of the state at slot t after round r has run
    since its last refresh."""
    m = np.zeros((rounds, nt), np.int64)
    for r in range(rounds):
        for t in range(nt):
            m[r, t] = next((k for k in range(1, r + 2) if (t + k) % nt >= lo), r + 1)
    return m


def self_coupling_sum(row_ptr, col, K) -> float:
    """sum_i K_ii over the coupling rows (the stored self-couplings)."""
    rows = np.repeat(np.arange(len(row_ptr) - 1), np.diff(row_ptr.astype(np.int64)))
    return float(np.sum(K[col == rows], dtype=np.float64))


def check_cached_energies(e, samples, energy_f64, nt, lo, rounds, chains, ksum, n):
    """e[t][r*C + c] against energy_f64(state) - 2 m[r][t] ksum, where the state
    is samples[t][r*C + c] (level-0 packed states).  Returns the largest m seen
    (so a caller can check that the drift was exercised)."""
    m = sweeps_since_refresh(nt, lo, rounds)
    for t in range(nt):
        assert len(e[t]) == rounds * chains and len(samples[t]) == rounds * chains
        for r in range(rounds):
            for c in range(chains):
                bits = np.unpackbits(np.asarray(samples[t][r * chains + c], np.uint8), bitorder="little")[:n]
                s = (1 - 2 * bits.astype(np.int8)).astype(np.int8)
                want = energy_f64(s) - 2.0 * m[r, t] * ksum
                got = float(e[t][r * chains + c])
                assert abs(got - want) <= 1e-5 * max(1.0, abs(want)), (t, r, c, got, want, m[r, t])
    return int(m.max())
