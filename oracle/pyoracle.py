"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Imported only by tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
bench.py.  The product never loads it.  Parity with the reference is
*unpinned*: the reference (Rust) cannot be built here and carries no golden
vectors, so the oracle is a line-by-line restatement (see tamc_oracle.cpp).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtamc_oracle.so")
_lib = None

u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i8p = C.POINTER(C.c_int8)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
u8p = C.POINTER(C.c_uint8)


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "orc_splitmix64": (None, [C.c_uint64, u64p, C.c_uint32]),
            "orc_xoshiro_seed": (None, [C.c_uint64, u64p]),
            "orc_xoshiro_next": (None, [u64p, u64p, C.c_uint32]),
            "orc_xoshiro_jump": (None, [u64p]),
            "orc_gen_range": (None, [u64p, C.c_uint32, u32p, C.c_uint32]),
            "orc_expf": (C.c_float, [C.c_float]),
            "orc_geometric_betas": (None, [C.c_float, C.c_float, C.c_uint32, f32p]),
            "orc_lo_beta_idx": (C.c_uint32, [f32p, C.c_uint32, C.c_int, C.c_uint32, C.c_int, C.c_float]),
            "orc_inst_from_text": (C.c_void_p, [C.c_char_p, C.c_uint64, C.c_int, C.c_char_p, C.c_uint64]),
            "orc_inst_from_csr": (C.c_void_p, [C.c_uint32, u32p, u32p, f32p, f32p, C.c_float]),
            "orc_inst_add_suscept": (C.c_int, [C.c_void_p, f64p, C.c_uint32]),
            "orc_inst_free": (None, [C.c_void_p]),
            "orc_inst_n": (C.c_uint32, [C.c_void_p]),
            "orc_inst_nnz": (C.c_uint64, [C.c_void_p]),
            "orc_inst_offset": (C.c_float, [C.c_void_p]),
            "orc_inst_graph_nodes": (C.c_uint32, [C.c_void_p]),
            "orc_inst_csr": (None, [C.c_void_p, u32p, u32p, f32p, f32p]),
            "orc_energy_ref": (C.c_float, [C.c_void_p, i8p]),
            "orc_energy_f64": (C.c_double, [C.c_void_p, i8p]),
            "orc_delta_energy": (C.c_float, [C.c_void_p, i8p, C.c_uint32]),
            "orc_pt_new": (C.c_void_p, [C.c_void_p, C.c_uint32, C.c_double, f32p, C.c_uint32, C.c_uint32,
                                        C.c_int, C.c_uint32, C.c_uint32, C.c_int64, C.c_int64,
                                        C.c_uint32, C.c_uint64]),
            "orc_pt_free": (None, [C.c_void_p]),
            "orc_pt_error": (C.c_char_p, [C.c_void_p]),
            "orc_pt_run": (C.c_int, [C.c_void_p, C.c_uint32, C.c_int]),
            "orc_pt_state": (None, [C.c_void_p, C.c_uint32, C.c_uint32, i8p, f32p, C.POINTER(C.c_int)]),
            "orc_pt_set_state": (None, [C.c_void_p, C.c_uint32, C.c_uint32, i8p]),
            "orc_pt_acceptance": (None, [C.c_void_p, C.c_uint32, u32p]),
            "orc_pt_tags": (None, [C.c_void_p, C.c_uint32, u8p, u32p, u32p]),
            "orc_pt_rng": (None, [C.c_void_p, C.c_int, C.c_int, u64p]),
            "orc_pt_gs_count": (C.c_uint32, [C.c_void_p]),
            "orc_pt_gs_entry": (None, [C.c_void_p, C.c_uint32, u32p, f32p, u64p]),
            "orc_pt_num_e": (C.c_uint32, [C.c_void_p, C.c_uint32]),
            "orc_pt_e": (None, [C.c_void_p, C.c_uint32, f32p]),
            "orc_pt_num_q": (C.c_uint32, [C.c_void_p, C.c_uint32]),
            "orc_pt_q": (None, [C.c_void_p, C.c_uint32, i32p]),
            "orc_pt_sus": (None, [C.c_void_p, C.c_uint32, C.c_uint32, f32p]),
            "orc_pt_num_sample_slots": (C.c_uint32, [C.c_void_p]),
            "orc_pt_num_samples": (C.c_uint32, [C.c_void_p, C.c_uint32]),
            "orc_pt_sample": (None, [C.c_void_p, C.c_uint32, C.c_uint32, u8p]),
            "orc_pt_icm_count": (C.c_uint32, [C.c_void_p]),
            "orc_pt_icm_sizes": (None, [C.c_void_p, i64p]),
            "orc_sa_run": (C.c_uint32, [C.c_void_p, f32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                                        C.c_int, f32p, i8p]),
            "orc_gla_run": (C.c_int, [C.c_void_p, u32p, u32p, C.c_uint32, C.c_uint32, C.c_double, f32p,
                                      C.c_uint32, C.c_uint32, C.c_int, C.c_uint32, C.c_int64, C.c_int64,
                                      C.c_uint32, C.c_uint64, f32p, C.c_uint32, u32p, u32p, u32p, f32p, f32p,
                                      i8p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


# ------------------------------------------------------------------ RNG ----
def splitmix64(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint64)
    lib().orc_splitmix64(seed, _p(out, u64p), n)
    return out


def xoshiro_seed(seed: int) -> np.ndarray:
    s = np.zeros(4, np.uint64)
    lib().orc_xoshiro_seed(seed, _p(s, u64p))
    return s


def xoshiro_next(state: np.ndarray, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint64)
    lib().orc_xoshiro_next(_p(state, u64p), _p(out, u64p), n)
    return out


def xoshiro_jump(state: np.ndarray) -> None:
    lib().orc_xoshiro_jump(_p(state, u64p))


def gen_range(state: np.ndarray, rng: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint32)
    lib().orc_gen_range(_p(state, u64p), rng, _p(out, u32p), n)
    return out


def expf(x: float) -> float:
    return lib().orc_expf(x)


def geometric_betas(bmin: float, bmax: float, n: int) -> np.ndarray:
    out = np.zeros(n, np.float32)
    lib().orc_geometric_betas(bmin, bmax, n, _p(out, f32p))
    return out


def lo_beta_idx(betas, lo_num=None, lo_beta=None) -> int:
    b = np.ascontiguousarray(betas, np.float32)
    return lib().orc_lo_beta_idx(_p(b, f32p), len(b), lo_num is not None, lo_num or 0,
                                 lo_beta is not None, lo_beta or 0.0)


# ------------------------------------------------------------- instance ----
class Instance:
    def __init__(self, handle):
        self.h = handle
        L = lib()
        self.n = L.orc_inst_n(self.h)
        self.nnz = L.orc_inst_nnz(self.h)
        self.offset = L.orc_inst_offset(self.h)
        self.graph_nodes = L.orc_inst_graph_nodes(self.h)

    @classmethod
    def from_text(cls, text: str, qubo: bool = False) -> "Instance":
        b = text.encode()
        err = C.create_string_buffer(256)
        h = lib().orc_inst_from_text(b, len(b), int(qubo), err, 256)
        if not h:
            raise ValueError(err.value.decode())
        return cls(h)

    @classmethod
    def from_csr(cls, row_ptr, col, K, bias, offset=0.0) -> "Instance":
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        cl = np.ascontiguousarray(col, np.uint32)
        kk = np.ascontiguousarray(K, np.float32)
        bb = np.ascontiguousarray(bias, np.float32)
        h = lib().orc_inst_from_csr(len(bb), _p(rp, u32p), _p(cl, u32p), _p(kk, f32p), _p(bb, f32p), offset)
        return cls(h)

    def add_suscept(self, w) -> None:
        a = np.ascontiguousarray(w, np.float64)
        lib().orc_inst_add_suscept(self.h, _p(a, f64p), len(a))

    def csr(self):
        rp = np.zeros(self.n + 1, np.uint32)
        cl = np.zeros(self.nnz, np.uint32)
        kk = np.zeros(self.nnz, np.float32)
        bb = np.zeros(self.n, np.float32)
        lib().orc_inst_csr(self.h, _p(rp, u32p), _p(cl, u32p), _p(kk, f32p), _p(bb, f32p))
        return rp, cl, kk, bb

    def energy_ref(self, s) -> float:
        a = np.ascontiguousarray(s, np.int8)
        return lib().orc_energy_ref(self.h, _p(a, i8p))

    def energy_f64(self, s) -> float:
        a = np.ascontiguousarray(s, np.int8)
        return lib().orc_energy_f64(self.h, _p(a, i8p))

    def delta_energy(self, s, i) -> float:
        a = np.ascontiguousarray(s, np.int8)
        return lib().orc_delta_energy(self.h, _p(a, i8p), i)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_inst_free(self.h)
            self.h = None


# ------------------------------------------------------------------- PT ----
class PtRun:
    """PtIcmRunner::run (threads<=1) / run_parallel (threads>1) with a fixed seed."""

    def __init__(self, inst: Instance, betas, num_sweeps, warmup_fraction=0.5, lo_beta_idx=0,
                 icm=True, num_chains=2, threads=1, sample=None, sample_states=None,
                 sample_limiting=0, seed=0):
        self.inst = inst
        self.betas = np.ascontiguousarray(betas, np.float32)
        self.nb = len(self.betas)
        self.nc = num_chains
        self.num_sweeps = num_sweeps
        self.h = lib().orc_pt_new(inst.h, num_sweeps, warmup_fraction, _p(self.betas, f32p), self.nb,
                                  lo_beta_idx, int(icm), num_chains, threads,
                                  -1 if sample is None else sample,
                                  -1 if sample_states is None else sample_states, sample_limiting, seed)

    def run(self, end=None, nthreads=0):
        end = self.num_sweeps if end is None else end
        if lib().orc_pt_run(self.h, end, nthreads) != 0:
            raise RuntimeError(lib().orc_pt_error(self.h).decode())

    def state(self, c, t):
        a = np.zeros(self.inst.n, np.int8)
        e = C.c_float()
        i = C.c_int()
        lib().orc_pt_state(self.h, c, t, _p(a, i8p), C.byref(e), C.byref(i))
        return a, e.value, bool(i.value)

    def states(self):
        """[chain][slot] spins (int8), cached energies and init flags."""
        S = np.zeros((self.nc, self.nb, self.inst.n), np.int8)
        E = np.zeros((self.nc, self.nb), np.float32)
        F = np.zeros((self.nc, self.nb), bool)
        for c in range(self.nc):
            for t in range(self.nb):
                S[c, t], E[c, t], F[c, t] = self.state(c, t)
        return S, E, F

    def set_state(self, c, t, s):
        a = np.ascontiguousarray(s, np.int8)
        lib().orc_pt_set_state(self.h, c, t, _p(a, i8p))

    def acceptance(self):
        out = np.zeros((self.nc, self.nb), np.uint32)
        for c in range(self.nc):
            row = np.zeros(self.nb, np.uint32)
            lib().orc_pt_acceptance(self.h, c, _p(row, u32p))
            out[c] = row
        return out

    def tags(self, c):
        t = np.zeros(self.nb, np.uint8)
        rt = C.c_uint32()
        dh = np.zeros(2 * self.nb, np.uint32)
        lib().orc_pt_tags(self.h, c, _p(t, u8p), C.byref(rt), _p(dh, u32p))
        return t, rt.value, dh.reshape(self.nb, 2)

    def rng(self, c=-1, t=0):
        s = np.zeros(4, np.uint64)
        lib().orc_pt_rng(self.h, c, t, _p(s, u64p))
        return s

    def gs(self):
        L = lib()
        nw = (self.inst.n + 63) // 64
        out = []
        for k in range(L.orc_pt_gs_count(self.h)):
            st = C.c_uint32()
            en = C.c_float()
            w = np.zeros(nw, np.uint64)
            L.orc_pt_gs_entry(self.h, k, C.byref(st), C.byref(en), _p(w, u64p))
            out.append((st.value, en.value, w))
        return out

    def thermal(self, nchi=0):
        L = lib()
        e, q, sus, samples = [], [], [], []
        for t in range(self.nb):
            a = np.zeros(L.orc_pt_num_e(self.h, t), np.float32)
            L.orc_pt_e(self.h, t, _p(a, f32p))
            e.append(a)
            b = np.zeros(L.orc_pt_num_q(self.h, t), np.int32)
            L.orc_pt_q(self.h, t, _p(b, i32p))
            q.append(b)
            rows = []
            for k in range(nchi):
                c = np.zeros(len(b), np.float32)
                L.orc_pt_sus(self.h, t, k, _p(c, f32p))
                rows.append(c)
            sus.append(rows)
        nbytes = (self.inst.n + 7) // 8
        for s in range(L.orc_pt_num_sample_slots(self.h)):
            lst = []
            for k in range(L.orc_pt_num_samples(self.h, s)):
                a = np.zeros(nbytes, np.uint8)
                L.orc_pt_sample(self.h, s, k, _p(a, u8p))
                lst.append(a)
            samples.append(lst)
        return e, q, sus, samples

    def icm_sizes(self):
        L = lib()
        a = np.zeros(L.orc_pt_icm_count(self.h), np.int64)
        L.orc_pt_icm_sizes(self.h, _p(a, i64p))
        return a

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_pt_free(self.h)
            self.h = None


def sa_run(inst: Instance, betas, num_replicas, threads, seed, nthreads=0):
    """SaRunner::run/run_parallel with a fixed seed: (energies, states[int8])."""
    b = np.ascontiguousarray(betas, np.float32)
    per = num_replicas // threads if num_replicas > 1 else 1
    parts = threads if num_replicas > 1 else 1
    r = parts * per
    e = np.zeros(r, np.float32)
    s = np.zeros((r, inst.n), np.int8)
    got = lib().orc_sa_run(inst.h, _p(b, f32p), len(b), num_replicas, threads, seed, nthreads,
                           _p(e, f32p), _p(s, i8p))
    if got != r:
        raise ValueError("bad SA parameters")
    return e, s


def gla_run(inst: Instance, parts, betas, num_sweeps, warmup_fraction=0.5, lo_beta_idx=0, icm=True,
            num_chains=2, sample=None, sample_states=None, sample_limiting=0, seed=0):
    """run_gla (src/gla.rs:121-195) with the master stream seed_from_u64(seed):
    dict of GlaResults fields plus the joined state; None where the reference panics."""
    b = np.ascontiguousarray(betas, np.float32)
    ptr = np.zeros(len(parts) + 1, np.uint32)
    ptr[1:] = np.cumsum([len(p) for p in parts])
    sites = np.ascontiguousarray(np.concatenate([np.asarray(p, np.uint32) for p in parts]) if parts else
                                 np.zeros(0, np.uint32), np.uint32)
    cap = max(1, len(parts) * len(parts))
    pe = np.zeros(len(parts), np.float32)
    nb = C.c_uint32()
    bs, bd = np.zeros(cap, np.uint32), np.zeros(cap, np.uint32)
    be = np.zeros(cap, np.float32)
    tot = C.c_float()
    joined = np.zeros(inst.n, np.int8)
    rc = lib().orc_gla_run(inst.h, _p(ptr, u32p), _p(sites, u32p), len(parts), num_sweeps, warmup_fraction,
                           _p(b, f32p), len(b), lo_beta_idx, int(icm), num_chains,
                           -1 if sample is None else sample, -1 if sample_states is None else sample_states,
                           sample_limiting, seed, _p(pe, f32p), cap, C.byref(nb), _p(bs, u32p), _p(bd, u32p),
                           _p(be, f32p), C.byref(tot), _p(joined, i8p))
    if rc == -2:
        return None
    if rc != 0:
        raise ValueError("bad GLA input")
    k = nb.value
    return {"instance_size": inst.n, "num_partitions": len(parts), "partition_energies": pe,
            "boundary_energies": list(zip(bs[:k].tolist(), bd[:k].tolist(), be[:k].tolist())),
            "bnd_energies": be[:k], "total_energy": np.float32(tot.value), "state": joined}
