"""tamc_b200 -- B200 (sm_100a) backend of tamc's PT-ICM and SA Monte-Carlo runners.

Python host mirror of the C ABI declared in include/tamc_gpu.h (loaded with
ctypes from the in-tree libtamc_b200.so).  The classes follow the reference's
runner interface: ``PtIcmRunner`` (src/pt.rs:298-593) and ``SaRunner``
(src/sa.rs:90-211) take the reference's parameters and return the reference's
result structures; ``Batch`` and ``Server`` are the batched and serving forms.
There is no CPU fallback: every compute call goes through the CUDA library and
raises if it is missing or no GPU is present.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

__all__ = [
    "TamcError", "lib", "HostInstance", "Method", "PtParams", "Gpu", "DeviceInstance", "PtRun", "sa_run",
    "sa_run_device", "Batch", "Server", "PtIcmRunner", "SaRunner", "geometric_betas", "MODE_REF", "MODE_FAST",
    "Partition", "GlaResults", "gla_run", "pt_opt_step",
]

MODE_REF = 0
MODE_FAST = 1
_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtamc_b200.so")
CLI_PATH = os.path.join(_HERE, "bin", "tamc_b200")
PT_OPT_CLI_PATH = os.path.join(_HERE, "bin", "tamc_b200_pt_opt")

ERRORS = {-1: "INVAL", -2: "NOMEM", -3: "CUDA", -4: "TIMEOUT", -5: "PARSE", -6: "IO", -7: "UNSUPPORTED",
          -8: "REFPANIC", -9: "ADMISSION"}


class TamcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)
f32p = C.POINTER(C.c_float)
f64p = C.POINTER(C.c_double)
i8p = C.POINTER(C.c_int8)
i32p = C.POINTER(C.c_int32)
u8p = C.POINTER(C.c_uint8)
vp = C.c_void_p


class _PtParams(C.Structure):
    _fields_ = [
        ("num_sweeps", C.c_uint32), ("warmup_fraction", C.c_double), ("num_beta", C.c_uint32),
        ("betas", f32p), ("lo_beta_idx", C.c_uint32), ("icm", C.c_int32), ("num_replica_chains", C.c_uint32),
        ("threads", C.c_uint32), ("sample", C.c_int64), ("sample_states", C.c_int64),
        ("sample_limiting", C.c_uint32),
    ]


_SIGS = {
    "tamc_last_error": (C.c_char_p, []),
    "tamc_version": (C.c_char_p, []),
    "tamc_ref_expf": (C.c_float, [C.c_float]),
    "tamc_instance_parse": (C.c_int, [C.c_char_p, C.c_uint64, C.c_int, C.POINTER(vp)]),
    "tamc_instance_read": (C.c_int, [C.c_char_p, C.c_int, C.POINTER(vp)]),
    "tamc_instance_from_csr": (C.c_int, [C.c_uint32, u32p, u32p, f32p, f32p, C.c_float, C.POINTER(vp)]),
    "tamc_instance_add_suscept_file": (C.c_int, [vp, C.c_char_p]),
    "tamc_instance_add_suscept": (C.c_int, [vp, f64p, C.c_uint32]),
    "tamc_instance_dims": (C.c_int, [vp, u32p, u64p, f32p, u32p]),
    "tamc_instance_csr": (C.c_int, [vp, u32p, u32p, f32p, f32p]),
    "tamc_instance_graph_nodes": (C.c_uint32, [vp]),
    "tamc_instance_coloring": (C.c_int, [vp, u32p, u32p]),
    "tamc_instance_energy_ref": (C.c_float, [vp, i8p]),
    "tamc_instance_free": (None, [vp]),
    "tamc_method_parse": (C.c_int, [C.c_char_p, C.c_uint64, C.POINTER(vp)]),
    "tamc_method_read": (C.c_int, [C.c_char_p, C.POINTER(vp)]),
    "tamc_method_kind": (C.c_int, [vp]),
    "tamc_method_pt": (C.c_int, [vp, C.POINTER(_PtParams)]),
    "tamc_method_sa": (C.c_int, [vp, C.POINTER(f32p), u32p, u32p, u32p]),
    "tamc_method_free": (None, [vp]),
    "tamc_method_gla": (C.c_int, [vp, u32p, C.POINTER(C.c_char_p), C.POINTER(_PtParams)]),
    "tamc_partition_parse": (C.c_int, [C.c_char_p, C.c_uint64, C.c_uint32, C.POINTER(vp)]),
    "tamc_partition_read": (C.c_int, [C.c_char_p, C.c_uint32, C.POINTER(vp)]),
    "tamc_partition_dims": (C.c_int, [vp, u32p, u64p]),
    "tamc_partition_get": (C.c_int, [vp, u32p, u32p]),
    "tamc_partition_free": (None, [vp]),
    "tamc_gla_run": (C.c_int, [vp, vp, vp, C.POINTER(_PtParams), C.c_uint64, C.c_int, C.POINTER(vp)]),
    "tamc_gla_dims": (C.c_int, [vp, u32p, u32p, u32p]),
    "tamc_gla_results": (C.c_int, [vp, f32p, u32p, u32p, f32p, f32p]),
    "tamc_gla_state": (C.c_int, [vp, i8p]),
    "tamc_gla_write": (C.c_int, [vp, C.c_char_p]),
    "tamc_gla_free": (None, [vp]),
    "tamc_geometric_betas": (C.c_int, [C.c_float, C.c_float, C.c_uint32, f32p]),
    "tamc_gpu_open": (C.c_int, [C.c_int, C.POINTER(vp)]),
    "tamc_gpu_close": (C.c_int, [vp]),
    "tamc_gpu_sync": (C.c_int, [vp]),
    "tamc_gpu_stream": (vp, [vp]),
    "tamc_gpu_launch_count": (C.c_uint64, [vp]),
    "tamc_copy_bytes": (None, [u64p, u64p]),
    "tamc_gpu_instance_upload": (C.c_int, [vp, vp, C.POINTER(vp)]),
    "tamc_gpu_instance_upload_many": (C.c_int, [vp, C.c_uint32, C.POINTER(vp), C.POINTER(vp)]),
    "tamc_gpu_instance_destroy": (C.c_int, [vp]),
    "tamc_gpu_batch_gs_all": (C.c_int, [vp, C.c_uint64, C.c_uint64, u32p, u32p, f32p, u64p]),
    "tamc_gpu_batch_acceptance_all": (C.c_int, [vp, C.c_uint64, u32p]),
    "tamc_gpu_pt_create": (C.c_int, [vp, C.POINTER(_PtParams), C.c_uint64, C.c_int, C.POINTER(vp)]),
    "tamc_gpu_pt_run": (C.c_int, [vp, C.c_uint32]),
    "tamc_gpu_pt_sync": (C.c_int, [vp]),
    "tamc_gpu_pt_get_state": (C.c_int, [vp, i8p, f32p]),
    "tamc_gpu_pt_set_state": (C.c_int, [vp, i8p]),
    "tamc_gpu_pt_acceptance": (C.c_int, [vp, u32p]),
    "tamc_gpu_pt_round_trips": (C.c_int, [vp, u8p, u32p, u32p]),
    "tamc_gpu_pt_gs": (C.c_int, [vp, C.c_uint32, u32p, u32p, f32p, u64p]),
    "tamc_gpu_pt_samples_dims": (C.c_int, [vp, u32p, u32p, u32p, u32p]),
    "tamc_gpu_pt_samples": (C.c_int, [vp, f32p, i32p, f32p, u8p]),
    "tamc_gpu_pt_timing_us": (C.c_double, [vp]),
    "tamc_gpu_pt_phase_cycles": (C.c_int, [vp, u64p]),
    "tamc_gpu_pt_destroy": (C.c_int, [vp]),
    "tamc_gpu_sa_run": (C.c_int, [vp, f32p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64, C.c_int, f32p, u8p,
                                  u32p]),
    "tamc_gpu_sa_run_device": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint64, vp, vp, vp]),
    "tamc_gpu_sa_scratch_bytes": (C.c_uint64, [vp, C.c_uint32]),
    "tamc_gpu_sa_run_noalloc": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, C.c_uint64, vp, vp, vp]),
    "tamc_gpu_batch_create": (C.c_int, [vp, C.POINTER(vp)]),
    "tamc_gpu_batch_add": (C.c_int, [vp, vp, C.POINTER(_PtParams), C.c_uint64, u32p]),
    "tamc_gpu_batch_run": (C.c_int, [vp]),
    "tamc_gpu_batch_sync": (C.c_int, [vp]),
    "tamc_gpu_batch_get_state": (C.c_int, [vp, C.c_uint32, i8p, f32p]),
    "tamc_gpu_batch_acceptance": (C.c_int, [vp, C.c_uint32, u32p]),
    "tamc_gpu_batch_gs": (C.c_int, [vp, C.c_uint32, C.c_uint32, u32p, u32p, f32p, u64p]),
    "tamc_gpu_batch_samples_dims": (C.c_int, [vp, C.c_uint32, u32p, u32p, u32p, u32p]),
    "tamc_gpu_batch_samples": (C.c_int, [vp, C.c_uint32, f32p, i32p, f32p, u8p]),
    "tamc_gpu_batch_device_time": (C.c_int, [vp, f64p, u64p]),
    "tamc_gpu_batch_set_state": (C.c_int, [vp, C.c_uint32, i8p]),
    "tamc_gpu_batch_round_trips": (C.c_int, [vp, C.c_uint32, u8p, u32p, u32p]),
    "tamc_pt_opt_step": (C.c_int, [C.c_uint32, f32p, f32p, C.c_uint32, u32p, u32p, C.c_uint32, C.c_uint32,
                                   C.c_float, C.c_float, f32p, f32p]),
    "tamc_gpu_batch_tile": (C.c_int, [vp, C.c_uint32, u32p, u32p, i32p]),
    "tamc_gpu_batch_destroy": (C.c_int, [vp]),
    "tamc_serve_create": (C.c_int, [vp, C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(vp)]),
    "tamc_serve_submit": (C.c_int, [vp, vp, C.POINTER(_PtParams), C.c_uint64, C.c_float, u64p]),
    "tamc_serve_step": (C.c_int, [vp, u32p, u32p]),
    "tamc_serve_result": (C.c_int, [vp, C.c_uint64, i32p, f32p, u32p, f64p]),
    "tamc_serve_state": (C.c_int, [vp, C.c_uint64, i8p, f32p]),
    "tamc_serve_status": (C.c_int, [vp, C.c_uint64, i32p, C.POINTER(C.c_char_p)]),
    "tamc_serve_cancel": (C.c_int, [vp, C.c_uint64]),
    "tamc_serve_destroy": (C.c_int, [vp]),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libtamc_b200.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing; build it with `python tamc_b200/build.py`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def _check(rc: int) -> None:
    if rc != 0:
        raise TamcError(rc, lib().tamc_last_error().decode())


def _p(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def copy_bytes():
    """(host->device, device->host) bytes the library has copied since load."""
    h, d = C.c_uint64(), C.c_uint64()
    lib().tamc_copy_bytes(C.byref(h), C.byref(d))
    return h.value, d.value


def geometric_betas(beta_min: float, beta_max: float, n: int) -> np.ndarray:
    """geometric_beta_schedule (tamc-core/src/sa.rs:13-22) cast to f32."""
    out = np.zeros(n, np.float32)
    _check(lib().tamc_geometric_betas(beta_min, beta_max, n, _p(out, f32p)))
    return out


# ----------------------------------------------------------------- instances
class HostInstance:
    """BqmIsingInstance on the host (src/ising.rs:257-324)."""

    def __init__(self, handle):
        self.h = handle
        n, nnz, off, nchi = C.c_uint32(), C.c_uint64(), C.c_float(), C.c_uint32()
        _check(lib().tamc_instance_dims(self.h, C.byref(n), C.byref(nnz), C.byref(off), C.byref(nchi)))
        self.n, self.nnz, self.offset, self.nchi = n.value, nnz.value, off.value, nchi.value

    def _refresh(self):
        self.__init__(self.h)

    @classmethod
    def parse(cls, text: str | bytes, qubo: bool = False) -> "HostInstance":
        b = text.encode() if isinstance(text, str) else text
        h = vp()
        _check(lib().tamc_instance_parse(b, len(b), int(qubo), C.byref(h)))
        return cls(h)

    @classmethod
    def read(cls, path: str, qubo: bool = False) -> "HostInstance":
        h = vp()
        _check(lib().tamc_instance_read(path.encode(), int(qubo), C.byref(h)))
        return cls(h)

    @classmethod
    def from_csr(cls, row_ptr, col, J, bias, offset: float = 0.0) -> "HostInstance":
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        cl = np.ascontiguousarray(col, np.uint32)
        jj = np.ascontiguousarray(J, np.float32)
        bb = np.ascontiguousarray(bias, np.float32)
        h = vp()
        _check(lib().tamc_instance_from_csr(len(bb), _p(rp, u32p), _p(cl, u32p), _p(jj, f32p), _p(bb, f32p),
                                            offset, C.byref(h)))
        return cls(h)

    def add_suscept(self, w) -> None:
        a = np.ascontiguousarray(w, np.float64)
        _check(lib().tamc_instance_add_suscept(self.h, _p(a, f64p), len(a)))
        self._refresh()

    def add_suscept_file(self, path: str) -> None:
        _check(lib().tamc_instance_add_suscept_file(self.h, path.encode()))
        self._refresh()

    def csr(self):
        rp = np.zeros(self.n + 1, np.uint32)
        cl = np.zeros(self.nnz, np.uint32)
        jj = np.zeros(self.nnz, np.float32)
        bb = np.zeros(self.n, np.float32)
        _check(lib().tamc_instance_csr(self.h, _p(rp, u32p), _p(cl, u32p), _p(jj, f32p), _p(bb, f32p)))
        return rp, cl, jj, bb

    @property
    def graph_nodes(self) -> int:
        return lib().tamc_instance_graph_nodes(self.h)

    def coloring(self):
        nc = C.c_uint32()
        col = np.zeros(self.n, np.uint32)
        _check(lib().tamc_instance_coloring(self.h, C.byref(nc), _p(col, u32p)))
        return nc.value, col

    def energy_ref(self, spins) -> float:
        a = np.ascontiguousarray(spins, np.int8)
        return lib().tamc_instance_energy_ref(self.h, _p(a, i8p))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.tamc_instance_free(self.h)
            self.h = None


@dataclass
class PtParams:
    """PtIcmParams (src/pt.rs:259-272) with the ladder and lo_beta_idx resolved."""
    num_sweeps: int
    betas: np.ndarray
    lo_beta_idx: int = 0
    warmup_fraction: float = 0.5
    icm: bool = True
    num_replica_chains: int = 2
    threads: int = 1
    sample: Optional[int] = None
    sample_states: Optional[int] = None
    sample_limiting: int = 0
    _keep: list = field(default_factory=list, repr=False)

    def to_c(self) -> _PtParams:
        b = np.ascontiguousarray(self.betas, np.float32)
        self._keep = [b]
        return _PtParams(self.num_sweeps, self.warmup_fraction, len(b), _p(b, f32p), self.lo_beta_idx,
                         int(self.icm), self.num_replica_chains, self.threads,
                         -1 if self.sample is None else self.sample,
                         -1 if self.sample_states is None else self.sample_states, self.sample_limiting)

    @property
    def meas_init(self) -> int:
        return max(0, int(self.warmup_fraction * self.num_sweeps))


class Method:
    """A parsed YAML method file (`PT:` / `SA:`; src/lib.rs:80-113)."""

    def __init__(self, handle):
        self.h = handle
        self.kind = {1: "PT", 2: "SA", 3: "GLA"}[lib().tamc_method_kind(self.h)]

    @classmethod
    def parse(cls, yaml_text: str) -> "Method":
        b = yaml_text.encode()
        h = vp()
        _check(lib().tamc_method_parse(b, len(b), C.byref(h)))
        return cls(h)

    @classmethod
    def read(cls, path: str) -> "Method":
        h = vp()
        _check(lib().tamc_method_read(path.encode(), C.byref(h)))
        return cls(h)

    def pt(self) -> PtParams:
        p = _PtParams()
        _check(lib().tamc_method_pt(self.h, C.byref(p)))
        betas = np.ctypeslib.as_array(p.betas, shape=(p.num_beta,)).copy()
        return PtParams(p.num_sweeps, betas, p.lo_beta_idx, p.warmup_fraction, bool(p.icm), p.num_replica_chains,
                        p.threads, None if p.sample < 0 else p.sample,
                        None if p.sample_states < 0 else p.sample_states, p.sample_limiting)

    def gla(self):
        """GLA: (num_threads, partition_file, the sub-solvers' PtParams)."""
        nt = C.c_uint32()
        pf = C.c_char_p()
        p = _PtParams()
        _check(lib().tamc_method_gla(self.h, C.byref(nt), C.byref(pf), C.byref(p)))
        betas = np.ctypeslib.as_array(p.betas, shape=(p.num_beta,)).copy()
        pt = PtParams(p.num_sweeps, betas, p.lo_beta_idx, p.warmup_fraction, bool(p.icm), p.num_replica_chains,
                      p.threads, None if p.sample < 0 else p.sample,
                      None if p.sample_states < 0 else p.sample_states, p.sample_limiting)
        return nt.value, pf.value.decode(), pt

    def sa(self):
        b = f32p()
        nb, r, t = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(lib().tamc_method_sa(self.h, C.byref(b), C.byref(nb), C.byref(r), C.byref(t)))
        betas = np.ctypeslib.as_array(b, shape=(nb.value,)).copy() if nb.value else np.zeros(0, np.float32)
        return betas, r.value, t.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.tamc_method_free(self.h)
            self.h = None


# --------------------------------------------------------------------- device
class Gpu:
    """A device context (one CUDA stream) -- tamc_gpu_open."""

    def __init__(self, device: int = 0):
        self.h = vp()
        _check(lib().tamc_gpu_open(device, C.byref(self.h)))
        self.device = device

    @property
    def stream(self) -> int:
        return lib().tamc_gpu_stream(self.h) or 0

    @property
    def launches(self) -> int:
        return lib().tamc_gpu_launch_count(self.h)

    def sync(self):
        _check(lib().tamc_gpu_sync(self.h))

    def upload(self, inst: HostInstance) -> "DeviceInstance":
        return DeviceInstance(self, inst)

    def upload_many(self, insts) -> list:
        """Uploads several instances in one call (tamc_gpu_instance_upload_many:
        host preparation on several threads), as many upload() calls would."""
        insts = list(insts)
        k = len(insts)
        his = (vp * max(k, 1))(*[i.h for i in insts])
        outs = (vp * max(k, 1))()
        _check(lib().tamc_gpu_instance_upload_many(self.h, k, his, outs))
        return [DeviceInstance(self, i, handle=outs[j]) for j, i in enumerate(insts)]

    def close(self):
        if getattr(self, "h", None):
            lib().tamc_gpu_close(self.h)
            self.h = None

    def __del__(self):
        if _lib is not None:
            self.close()


class DeviceInstance:
    def __init__(self, gpu: Gpu, inst: HostInstance, handle=None):
        self.gpu, self.host = gpu, inst
        if handle is not None:  # uploaded by Gpu.upload_many
            self.h = vp(handle)
        else:
            self.h = vp()
            _check(lib().tamc_gpu_instance_upload(gpu.h, inst.h, C.byref(self.h)))
        self.n = inst.n

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.tamc_gpu_instance_destroy(self.h)
            self.h = None


@dataclass
class ThermalSamples:
    """PtIcmThermalSamples (src/pt.rs:117-125), nested as the reference stores it."""
    compression_level: int
    instance_size: int
    beta_arr: np.ndarray
    samples: list
    e: list
    q: list
    suscept: list


class PtRun:
    """One PT-ICM run on the device (plain form: tamc_gpu_pt_*)."""

    def __init__(self, dinst: DeviceInstance, params: PtParams, seed: int, mode: int = MODE_FAST):
        self.dinst, self.params, self.mode = dinst, params, mode
        self.nt, self.C, self.n = len(params.betas), params.num_replica_chains, dinst.n
        cp = params.to_c()
        self.h = vp()
        _check(lib().tamc_gpu_pt_create(dinst.h, C.byref(cp), seed, mode, C.byref(self.h)))

    def run(self, sweep_end: Optional[int] = None) -> "PtRun":
        _check(lib().tamc_gpu_pt_run(self.h, self.params.num_sweeps if sweep_end is None else sweep_end))
        return self

    def sync(self) -> "PtRun":
        _check(lib().tamc_gpu_pt_sync(self.h))
        return self

    def state(self):
        s = np.zeros((self.C, self.nt, self.n), np.int8)
        e = np.zeros((self.C, self.nt), np.float32)
        _check(lib().tamc_gpu_pt_get_state(self.h, _p(s, i8p), _p(e, f32p)))
        return s, e

    def set_state(self, spins) -> None:
        a = np.ascontiguousarray(spins, np.int8)
        _check(lib().tamc_gpu_pt_set_state(self.h, _p(a, i8p)))

    def acceptance(self) -> np.ndarray:
        a = np.zeros(self.nt, np.uint32)
        _check(lib().tamc_gpu_pt_acceptance(self.h, _p(a, u32p)))
        return a

    def round_trips(self):
        t = np.zeros((self.C, self.nt), np.uint8)
        r = np.zeros(self.C, np.uint32)
        d = np.zeros((self.C, self.nt, 2), np.uint32)
        _check(lib().tamc_gpu_pt_round_trips(self.h, _p(t, u8p), _p(r, u32p), _p(d, u32p)))
        return t, r, d

    def gs(self):
        cnt = C.c_uint32()
        _check(lib().tamc_gpu_pt_gs(self.h, 0, C.byref(cnt), None, None, None))
        k = cnt.value
        nw = (self.n + 63) // 64
        steps = np.zeros(k, np.uint32)
        en = np.zeros(k, np.float32)
        st = np.zeros((k, nw), np.uint64)
        _check(lib().tamc_gpu_pt_gs(self.h, k, C.byref(cnt), _p(steps, u32p), _p(en, f32p), _p(st, u64p)))
        return steps, en, st

    def samples(self) -> ThermalSamples:
        M, S, Z, nchi = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(lib().tamc_gpu_pt_samples_dims(self.h, C.byref(M), C.byref(S), C.byref(Z), C.byref(nchi)))
        M, S, Z, nchi = M.value, S.value, Z.value, nchi.value
        nt, Cc, P, nb = self.nt, self.C, self.C // 2, (self.n + 7) // 8
        e = np.zeros((nt, M * Cc), np.float32)
        q = np.zeros((nt, M * P), np.int32)
        sus = np.zeros((nt, nchi, M * P), np.float32)
        smp = np.zeros((Z, S * Cc, nb), np.uint8)
        _check(lib().tamc_gpu_pt_samples(self.h, _p(e, f32p), _p(q, i32p), _p(sus, f32p), _p(smp, u8p)))
        return ThermalSamples(self.params.sample_limiting, self.n, np.asarray(self.params.betas, np.float32),
                              [list(z) for z in smp], list(e), list(q), [list(r) for r in sus])

    @property
    def timing_us(self) -> float:
        return lib().tamc_gpu_pt_timing_us(self.h)

    PHASES = ("icm_scan", "icm_init", "icm_jump", "icm_grow", "icm_mark", "icm_apply", "exchange", "sweep", "measure",
              "other", "sweep_levels_per_warp", "sweep_flip_per_warp", "sweep_energy_per_warp", "sweep_wait_per_warp")

    def phase_cycles(self) -> dict:
        """Cycles per round phase (fast mode, TAMC_PHASE_PROF=1 at creation)."""
        a = np.zeros(len(self.PHASES), np.uint64)
        _check(lib().tamc_gpu_pt_phase_cycles(self.h, _p(a, u64p)))
        return dict(zip(self.PHASES, a.tolist()))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.tamc_gpu_pt_destroy(self.h)
            self.h = None


def sa_run(dinst: DeviceInstance, betas, num_replicas: int, threads: int, seed: int, mode: int = MODE_FAST,
           out=None):
    """SaRunner::run / run_parallel on the device: (energies, packed states [r_eff, ceil(n/8)]).
    `out` = (energies float32[r], packed uint8[r, ceil(n/8)]) receives the results
    in caller-owned (e.g. pinned) host buffers with room for every replica."""
    b = np.ascontiguousarray(betas, np.float32)
    parts = threads if num_replicas > 1 else 1
    per = num_replicas // threads if num_replicas > 1 and threads else 1
    rmax = max(parts * per, 1)
    if out is None:
        e = np.zeros(rmax, np.float32)
        packed = np.zeros((rmax, (dinst.n + 7) // 8), np.uint8)
    else:
        e, packed = out
        if (e.dtype != np.float32 or packed.dtype != np.uint8 or len(e) < rmax or packed.shape[0] < rmax
                or packed.shape[1] != (dinst.n + 7) // 8 or not e.flags.c_contiguous
                or not packed.flags.c_contiguous):
            raise ValueError("out buffers must be contiguous float32[r] and uint8[r, ceil(n/8)]")
    reff = C.c_uint32()
    _check(lib().tamc_gpu_sa_run(dinst.h, _p(b, f32p), len(b), num_replicas, threads, seed, mode, _p(e, f32p),
                                 _p(packed, u8p), C.byref(reff)))
    r = reff.value
    return e[:r], packed[:r]


def sa_run_device(dinst: DeviceInstance, d_betas: int, nbeta: int, num_replicas: int, seed: int, d_energies: int,
                  d_words: int, stream: int = 0) -> None:
    """Device-resident SA (all pointers are device addresses, e.g. torch tensor data_ptr())."""
    _check(lib().tamc_gpu_sa_run_device(dinst.h, d_betas, nbeta, num_replicas, seed, d_energies, d_words,
                                        stream or None))


# largest ceil(num_replicas/32) * n * 4 that sa_run_noalloc accepts (TAMC_SA_NOALLOC_SCRATCH_BYTES)
SA_NOALLOC_SCRATCH_BYTES = 4 << 20


def sa_run_noalloc(dinst: DeviceInstance, d_betas: int, nbeta: int, num_replicas: int, seed: int, d_energies: int,
                   d_packed: int, stream: int = 0) -> None:
    """Fast-mode SA with no device allocation: energies and packed states into
    caller-owned device buffers; replica words in a static device array shared
    by all calls on the device (calls must not overlap)."""
    _check(lib().tamc_gpu_sa_run_noalloc(dinst.h, d_betas, nbeta, num_replicas, seed, d_energies, d_packed,
                                         stream or None))


def unpack_bits(packed: np.ndarray, n: int) -> np.ndarray:
    """Bit-packed states (bit i%8 of byte i/8 set = spin -1) to int8 +-1."""
    bits = np.unpackbits(packed, axis=-1, bitorder="little")[..., :n]
    return (1 - 2 * bits.astype(np.int8)).astype(np.int8)


def u64_to_spins(words: np.ndarray, n: int) -> np.ndarray:
    b = words.astype("<u8").view(np.uint8)
    return unpack_bits(b, n)


# ----------------------------------------------------------------- batched
class Batch:
    """Batched PT-ICM: many uneven instances in one persistent kernel (tamc_gpu_batch_*)."""

    def __init__(self, gpu: Gpu):
        self.gpu = gpu
        self.h = vp()
        _check(lib().tamc_gpu_batch_create(gpu.h, C.byref(self.h)))
        self.jobs = []

    def add(self, dinst: DeviceInstance, params: PtParams, seed: int) -> int:
        cp = params.to_c()
        j = C.c_uint32()
        _check(lib().tamc_gpu_batch_add(self.h, dinst.h, C.byref(cp), seed, C.byref(j)))
        self.jobs.append((dinst, params))
        return j.value

    def run(self) -> "Batch":
        _check(lib().tamc_gpu_batch_run(self.h))
        return self

    def state(self, job: int):
        d, p = self.jobs[job]
        s = np.zeros((p.num_replica_chains, len(p.betas), d.n), np.int8)
        e = np.zeros((p.num_replica_chains, len(p.betas)), np.float32)
        _check(lib().tamc_gpu_batch_get_state(self.h, job, _p(s, i8p), _p(e, f32p)))
        return s, e

    def gs(self, job: int):
        d, p = self.jobs[job]
        cnt = C.c_uint32()
        _check(lib().tamc_gpu_batch_gs(self.h, job, 0, C.byref(cnt), None, None, None))
        k = cnt.value
        steps = np.zeros(k, np.uint32)
        en = np.zeros(k, np.float32)
        st = np.zeros((k, (d.n + 63) // 64), np.uint64)
        _check(lib().tamc_gpu_batch_gs(self.h, job, k, C.byref(cnt), _p(steps, u32p), _p(en, f32p), _p(st, u64p)))
        return steps, en, st

    def acceptance(self, job: int) -> np.ndarray:
        _, p = self.jobs[job]
        a = np.zeros(len(p.betas), np.uint32)
        _check(lib().tamc_gpu_batch_acceptance(self.h, job, _p(a, u32p)))
        return a

    def gs_all(self) -> list:
        """gs() of every job, read in two calls (tamc_gpu_batch_gs_all)."""
        nj = len(self.jobs)
        cnt = np.zeros(max(nj, 1), np.uint32)
        _check(lib().tamc_gpu_batch_gs_all(self.h, 0, 0, _p(cnt, u32p), None, None, None))
        wpj = np.array([(d.n + 63) // 64 for d, _ in self.jobs], np.uint64)
        cnt = cnt[:nj].astype(np.uint64)
        ne, nwd = int(cnt.sum()), int((cnt * wpj).sum())
        steps = np.zeros(max(ne, 1), np.uint32)
        en = np.zeros(max(ne, 1), np.float32)
        st = np.zeros(max(nwd, 1), np.uint64)
        _check(lib().tamc_gpu_batch_gs_all(self.h, ne, nwd, _p(np.zeros(max(nj, 1), np.uint32), u32p),
                                           _p(steps, u32p), _p(en, f32p), _p(st, u64p)))
        out, eo, wo = [], 0, 0
        for j in range(nj):
            c, w = int(cnt[j]), int(wpj[j])
            out.append((steps[eo:eo + c], en[eo:eo + c], st[wo:wo + c * w].reshape(c, w)))
            eo += c
            wo += c * w
        return out

    def acceptance_all(self) -> list:
        """acceptance() of every job in one call (tamc_gpu_batch_acceptance_all)."""
        nts = [len(p.betas) for _, p in self.jobs]
        a = np.zeros(max(sum(nts), 1), np.uint32)
        _check(lib().tamc_gpu_batch_acceptance_all(self.h, sum(nts), _p(a, u32p)))
        out, o = [], 0
        for nt in nts:
            out.append(a[o:o + nt])
            o += nt
        return out

    def set_state(self, job: int, spins) -> None:
        a = np.ascontiguousarray(spins, np.int8)
        _check(lib().tamc_gpu_batch_set_state(self.h, job, _p(a, i8p)))

    def round_trips(self, job: int):
        _, p = self.jobs[job]
        nt, Cc = len(p.betas), p.num_replica_chains
        t = np.zeros((Cc, nt), np.uint8)
        r = np.zeros(Cc, np.uint32)
        d = np.zeros((Cc, nt, 2), np.uint32)
        _check(lib().tamc_gpu_batch_round_trips(self.h, job, _p(t, u8p), _p(r, u32p), _p(d, u32p)))
        return t, r, d

    def samples(self, job: int) -> "ThermalSamples":
        """PtIcmThermalSamples of one job (as PtRun.samples)."""
        d, p = self.jobs[job]
        M, S, Z, nchi = C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(lib().tamc_gpu_batch_samples_dims(self.h, job, C.byref(M), C.byref(S), C.byref(Z), C.byref(nchi)))
        M, S, Z, nchi = M.value, S.value, Z.value, nchi.value
        nt, Cc, nb = len(p.betas), p.num_replica_chains, (d.n + 7) // 8
        P = Cc // 2
        e = np.zeros((nt, M * Cc), np.float32)
        q = np.zeros((nt, M * P), np.int32)
        sus = np.zeros((nt, nchi, M * P), np.float32)
        smp = np.zeros((Z, S * Cc, nb), np.uint8)
        _check(lib().tamc_gpu_batch_samples(self.h, job, _p(e, f32p), _p(q, i32p), _p(sus, f32p), _p(smp, u8p)))
        return ThermalSamples(p.sample_limiting, d.n, np.asarray(p.betas, np.float32), [list(z) for z in smp],
                              list(e), list(q), [list(r) for r in sus])

    def device_time(self):
        """(summed CUDA-event ms of the chunk launches, number of launches)."""
        ms, n = C.c_double(), C.c_uint64()
        _check(lib().tamc_gpu_batch_device_time(self.h, C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def tile(self, job: int):
        t, s, c = C.c_uint32(), C.c_uint32(), C.c_int32()
        _check(lib().tamc_gpu_batch_tile(self.h, job, C.byref(t), C.byref(s), C.byref(c)))
        return t.value, s.value, bool(c.value)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.tamc_gpu_batch_destroy(self.h)
            self.h = None


class Server:
    """Continuous-batching solve server (tamc_serve_*)."""

    def __init__(self, gpu: Gpu, hbm_budget_bytes: int, max_active: int = 256, chunk_sweeps: int = 100):
        self.gpu = gpu
        self.h = vp()
        _check(lib().tamc_serve_create(gpu.h, hbm_budget_bytes, max_active, chunk_sweeps, C.byref(self.h)))
        self.params = {}

    def submit(self, inst: HostInstance, params: PtParams, seed: int, target_energy: float = math.nan) -> int:
        cp = params.to_c()
        rid = C.c_uint64()
        _check(lib().tamc_serve_submit(self.h, inst.h, C.byref(cp), seed, target_energy, C.byref(rid)))
        self.params[rid.value] = (inst.n, params)
        return rid.value

    def step(self):
        a, q = C.c_uint32(), C.c_uint32()
        _check(lib().tamc_serve_step(self.h, C.byref(a), C.byref(q)))
        return a.value, q.value

    def result(self, rid: int):
        d, b, s, l = C.c_int32(), C.c_float(), C.c_uint32(), C.c_double()
        _check(lib().tamc_serve_result(self.h, rid, C.byref(d), C.byref(b), C.byref(s), C.byref(l)))
        return bool(d.value), b.value, s.value, l.value

    STATUS = ("queued", "active", "done", "cancelled", "failed")

    def status(self, rid: int):
        """(state name, error message for a failed request or '')."""
        st = C.c_int32()
        err = C.c_char_p()
        _check(lib().tamc_serve_status(self.h, rid, C.byref(st), C.byref(err)))
        return self.STATUS[st.value], (err.value or b"").decode()

    def cancel(self, rid: int) -> None:
        _check(lib().tamc_serve_cancel(self.h, rid))

    def state(self, rid: int):
        n, p = self.params[rid]
        s = np.zeros((p.num_replica_chains, len(p.betas), n), np.int8)
        e = np.zeros((p.num_replica_chains, len(p.betas)), np.float32)
        _check(lib().tamc_serve_state(self.h, rid, _p(s, i8p), _p(e, f32p)))
        return s, e

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.tamc_serve_destroy(self.h)
            self.h = None


# ------------------------------------------------------------- pt-opt
def pt_opt_step(betas, momentum, round_trips, diffusion_hist, num_sweeps: int, num_chains: int, alpha: float,
                m: float):
    """One ladder update of tamc-pt-opt (tamc_pt_opt_step).  round_trips[I] and
    diffusion_hist[I][nt][2] are per instance, summed over chains.  Returns
    (updated, betas, momentum, tau, err); `updated` False when the runs saw too
    few round trips (ladder and momentum unchanged, err None)."""
    b = np.array(betas, np.float32)
    mo = np.array(momentum, np.float32)
    rt = np.ascontiguousarray(round_trips, np.uint32)
    dh = np.ascontiguousarray(diffusion_hist, np.uint32)
    tau = np.zeros(len(rt), np.float32)
    err = C.c_float()
    rc = lib().tamc_pt_opt_step(len(b), _p(b, f32p), _p(mo, f32p), len(rt), _p(rt, u32p), _p(dh, u32p), num_sweeps,
                                num_chains, alpha, m, _p(tau, f32p), C.byref(err))
    if rc == 1:
        return False, b, mo, tau, None
    _check(rc)
    return True, b, mo, tau, err.value


# ---------------------------------------------------------------- GLA
class Partition:
    """A site partition for GLA (GlaParams::read_graph_partition, src/gla.rs:37-58)."""

    def __init__(self, handle):
        self.h = handle
        npart, nsite = C.c_uint32(), C.c_uint64()
        _check(lib().tamc_partition_dims(self.h, C.byref(npart), C.byref(nsite)))
        ptr = np.zeros(npart.value + 1, np.uint32)
        sites = np.zeros(nsite.value, np.uint32)
        _check(lib().tamc_partition_get(self.h, _p(ptr, u32p), _p(sites, u32p)))
        self.parts = [sites[ptr[k]:ptr[k + 1]].tolist() for k in range(npart.value)]

    @classmethod
    def parse(cls, text: str | bytes, n: int) -> "Partition":
        b = text.encode() if isinstance(text, str) else text
        h = vp()
        _check(lib().tamc_partition_parse(b, len(b), n, C.byref(h)))
        return cls(h)

    @classmethod
    def read(cls, path: str, n: int) -> "Partition":
        h = vp()
        _check(lib().tamc_partition_read(path.encode(), n, C.byref(h)))
        return cls(h)

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.tamc_partition_free(self.h)
            self.h = None


@dataclass
class GlaResults:
    """GlaResults (src/gla.rs:61-69), plus the joined ground state."""
    instance_size: int
    num_partitions: int
    partition_energies: np.ndarray
    boundary_energies: list
    total_energy: float
    state: np.ndarray


def gla_run(gpu: Gpu, inst: HostInstance, part: Partition, params: PtParams, seed: int, mode: int = MODE_FAST,
            output: Optional[str] = None) -> GlaResults:
    """run_gla (src/gla.rs:121-195) on the device; `output` writes the result
    file as the reference does (pickle for .pkl, else bincode)."""
    cp = params.to_c()
    h = vp()
    _check(lib().tamc_gla_run(gpu.h, inst.h, part.h, C.byref(cp), seed, mode, C.byref(h)))
    try:
        n, npart, nb = C.c_uint32(), C.c_uint32(), C.c_uint32()
        _check(lib().tamc_gla_dims(h, C.byref(n), C.byref(npart), C.byref(nb)))
        pe = np.zeros(npart.value, np.float32)
        bs, bd = np.zeros(nb.value, np.uint32), np.zeros(nb.value, np.uint32)
        be = np.zeros(nb.value, np.float32)
        tot = C.c_float()
        _check(lib().tamc_gla_results(h, _p(pe, f32p), _p(bs, u32p), _p(bd, u32p), _p(be, f32p), C.byref(tot)))
        st = np.zeros(n.value, np.int8)
        _check(lib().tamc_gla_state(h, _p(st, i8p)))
        if output:
            _check(lib().tamc_gla_write(h, output.encode()))
    finally:
        lib().tamc_gla_free(h)
    return GlaResults(n.value, npart.value, pe, list(zip(bs.tolist(), bd.tolist(), be.tolist())),
                      np.float32(tot.value), st)


# ------------------------------------------------- reference-named runners
class PtIcmRunner:
    """Mirror of PtIcmRunner (src/pt.rs:298-593): construct with an instance and
    PtIcmParams, then ``run()`` returns (PtIcmMinResults dict, ThermalSamples,
    final states).  `threads` keeps the reference's meaning: <=1 selects `run`
    (one stream, serial exchange), >1 `run_parallel` (per-slot streams)."""

    def __init__(self, gpu: Gpu, instance: HostInstance, params: PtParams, seed: int, mode: int = MODE_FAST):
        self.dinst = gpu.upload(instance)
        self.params, self.seed, self.mode = params, seed, mode

    def run(self):
        r = PtRun(self.dinst, self.params, self.seed, self.mode).run().sync()
        steps, en, st = r.gs()
        res = {"timing": r.timing_us, "gs_time_steps": steps.tolist(), "gs_energies": en.tolist(),
               "gs_states": [list(map(int, w)) for w in st], "num_measurements": 0,
               "instance_size": self.dinst.n, "acceptance_counts": r.acceptance().tolist()}
        return res, r.samples(), r.state()


class SaRunner:
    """Mirror of SaRunner (src/sa.rs:90-211)."""

    def __init__(self, gpu: Gpu, instance: HostInstance, betas, num_replicas: int, threads: int, seed: int,
                 mode: int = MODE_FAST):
        self.dinst = gpu.upload(instance)
        self.betas, self.num_replicas, self.threads, self.seed, self.mode = betas, num_replicas, threads, seed, mode

    def run(self):
        e, packed = sa_run(self.dinst, self.betas, self.num_replicas, self.threads, self.seed, self.mode)
        return {"min_energy": float(e.min()) if len(e) else 0.0, "energies": e.tolist(),
                "num_replicas": len(e)}, packed
