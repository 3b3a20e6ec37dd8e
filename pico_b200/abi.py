"""ctypes binding of libpico_gpu.so (the C ABI declared in include/pico_gpu.h).

The library is built in-tree by pico_b200/build.py.  Loading never falls back
to anything else: if the shared object is missing or stale and cannot be
built, import of the GPU entry points fails loudly.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

from . import build as _build

PICO_OK = 0
PICO_ERR_INVALID_ARG = 1
PICO_ERR_OUT_OF_MEMORY = 2
PICO_ERR_CUDA = 3
PICO_ERR_UNSUPPORTED = 4
PICO_ERR_TIMEOUT = 5
PICO_ERR_NOT_READY = 6
PICO_ERR_CANCELLED = 7
STATUS_NAMES = {
    0: "PICO_OK",
    1: "PICO_ERR_INVALID_ARG",
    2: "PICO_ERR_OUT_OF_MEMORY",
    3: "PICO_ERR_CUDA",
    4: "PICO_ERR_UNSUPPORTED",
    5: "PICO_ERR_TIMEOUT",
    6: "PICO_ERR_NOT_READY",
    7: "PICO_ERR_CANCELLED",
    8: "PICO_ERR_NO_DEVICE",
}

PICO_KOALABEAR = 0
PICO_BABYBEAR = 1

PICO_INPUT_DEVICE = 0x1
PICO_COMMIT_PLAIN = 0x2
PICO_OUTPUT_DEVICE = 0x4
PICO_LDE_NATURAL_ORDER = 0x8
PICO_P2_FOUR_LANES = 0x10
PICO_QUOTIENT_CHUNKS = 0x20


class PicoError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


PICO_MATRIX_EXT4 = 0x1


class Matrix(C.Structure):
    _fields_ = [
        ("values", C.c_void_p),
        ("log_height", C.c_uint32),
        ("width", C.c_uint32),
        ("shift", C.c_uint32),
        ("flags", C.c_uint32),
    ]


class Config(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_uint64),
        ("n_streams", C.c_uint32),
        ("flags", C.c_uint32),
        ("max_inflight", C.c_uint32),
        ("max_group", C.c_uint32),
        ("reserved", C.c_uint32 * 4),
    ]


class Challenger(C.Structure):
    _fields_ = [
        ("sponge", C.c_uint32 * 16),
        ("in_buf", C.c_uint32 * 8),
        ("in_len", C.c_uint32),
        ("out_buf", C.c_uint32 * 8),
        ("out_len", C.c_uint32),
    ]


class CommitStats(C.Structure):
    _fields_ = [
        ("total_ms", C.c_double),
        ("h2d_ms", C.c_double),
        ("lde_ms", C.c_double),
        ("leaves_ms", C.c_double),
        ("tree_ms", C.c_double),
        ("cells", C.c_uint64),
        ("lde_cells", C.c_uint64),
        ("permutations", C.c_uint64),
        ("leaf_permutations", C.c_uint64),
        ("lde_bytes", C.c_uint64),
        ("launches", C.c_uint64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class OpenBatch(C.Structure):
    _fields_ = [("commit", C.c_void_p), ("n_points", C.c_void_p), ("points", C.c_void_p)]


class FriParams(C.Structure):
    _fields_ = [
        ("log_blowup", C.c_uint32),
        ("num_queries", C.c_uint32),
        ("proof_of_work_bits", C.c_uint32),
        ("reserved", C.c_uint32),
    ]


class OpenStats(C.Structure):
    _fields_ = [
        ("ms_values", C.c_float),
        ("ms_reduce", C.c_float),
        ("ms_fri", C.c_float),
        ("ms_grind", C.c_float),
        ("ms_queries", C.c_float),
        ("ms_total", C.c_float),
        ("value_cells", C.c_uint64),
        ("reduce_cells", C.c_uint64),
        ("launches", C.c_uint32),
        ("rounds", C.c_uint32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class TraceRef(C.Structure):
    _fields_ = [("commit", C.c_void_p), ("mat_idx", C.c_uint32), ("reserved", C.c_uint32)]


_u32p = C.POINTER(C.c_uint32)
_vp = C.c_void_p
_u32 = C.c_uint32
_u64 = C.c_uint64

# name -> (restype, argtypes); every symbol the header declares
SIGNATURES = {
    "pico_gpu_init": (C.c_int, [C.c_int, C.POINTER(Config), C.POINTER(_vp)]),
    "pico_gpu_shutdown": (C.c_int, [_vp]),
    "pico_gpu_last_error": (C.c_char_p, []),
    "pico_gpu_abi_version": (_u32, []),
    "pico_gpu_memory": (C.c_int, [_vp, C.POINTER(_u64), C.POINTER(_u64)]),
    "pico_gpu_reserve_pool": (C.c_int, [_vp, _u64, C.POINTER(C.c_uint64)]),
    "pico_gpu_commit_bytes": (C.c_int, [C.c_int, C.POINTER(Matrix), _u32, _u32, _u32, C.POINTER(_u64),
                                        C.POINTER(_u64)]),
    "pico_gpu_commit": (C.c_int, [_vp, C.c_int, C.POINTER(Matrix), _u32, _u32, _u32, C.POINTER(_vp), _u32p]),
    "pico_gpu_release": (C.c_int, [_vp, _vp]),
    "pico_gpu_commit_stats": (C.c_int, [_vp, C.POINTER(CommitStats)]),
    "pico_gpu_last_commit_stats": (C.c_int, [C.POINTER(CommitStats)]),
    "pico_gpu_lde_rows": (C.c_int, [_vp, _vp, _u32, _u64, _u64, _vp, _u32]),
    "pico_gpu_lde_shape": (C.c_int, [_vp, _u32, _u32p, _u32p]),
    "pico_gpu_evaluations_on_domain": (C.c_int, [_vp, _vp, _u32, _u32, _vp, _u32]),
    "pico_gpu_digest_layer": (C.c_int, [_vp, _vp, _u32, _vp, _u32]),
    "pico_gpu_open_batch": (C.c_int, [_vp, _vp, _u64, _vp, _vp]),
    "pico_gpu_coset_lde_batch": (C.c_int, [_vp, C.c_int, _vp, _u32, _u32, _u32, _u32, _vp, _u32]),
    "pico_gpu_coset_lde_batch_noalloc": (C.c_int, [C.c_int, _vp, _u32, _u32, _u32, _u32, _vp, _vp]),
    "pico_gpu_noalloc_status": (C.c_int, [_vp]),
    "pico_gpu_mmcs_commit": (C.c_int, [_vp, C.c_int, C.POINTER(Matrix), _u32, _u32, C.POINTER(_vp), _u32p]),
    "pico_gpu_commit_shard": (C.c_int, [_vp, C.c_int, C.POINTER(Matrix), _u32, _u32, _u32, _u32, _u32,
                                        C.POINTER(_vp), _u32p]),
    "pico_gpu_merkle_top": (C.c_int, [C.c_int, _u32p, _u32, _u32p]),
    "pico_gpu_merkle_top_path": (C.c_int, [C.c_int, _u32p, _u32, _u32, _u32p]),
    "pico_gpu_fri_shard_begin": (C.c_int, [_vp, C.c_int, _vp, _u32, _u32, _u32, _u32, C.POINTER(_vp), _u32p]),
    "pico_gpu_fri_shard_fold": (C.c_int, [_vp, _u32p, _u32p]),
    "pico_gpu_fri_shard_rows": (C.c_int, [_vp, _vp, _u32]),
    "pico_gpu_fri_shard_release": (C.c_int, [_vp]),
    "pico_gpu_poseidon2_permute": (C.c_int, [_vp, C.c_int, _vp, _u64, _u32]),
    "pico_gpu_fri_commit_phase": (
        C.c_int,
        [_vp, C.c_int, _vp, _u32, _u32, _u32, _vp, C.POINTER(Challenger), _u32, _vp, _vp, _vp, _u32p,
         C.POINTER(_vp)],
    ),
    "pico_gpu_fri_release": (C.c_int, [_vp, _vp]),
    "pico_gpu_fri_layer": (C.c_int, [_vp, _vp, _u32, _vp, _u32]),
    "pico_gpu_submit_commit": (C.c_int, [_vp, C.c_int, C.POINTER(Matrix), _u32, _u32, _u32, C.POINTER(_vp)]),
    "pico_gpu_poll": (C.c_int, [_vp, _vp]),
    "pico_gpu_wait": (C.c_int, [_vp, _vp, C.c_int64, C.POINTER(_vp), _u32p]),
    "pico_gpu_cancel": (C.c_int, [_vp, _vp]),
    "pico_gpu_request_times": (C.c_int, [_vp, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "pico_gpu_request_free": (C.c_int, [_vp, _vp]),
    "pico_gpu_autotune": (C.c_int, [_vp, C.c_int, _u32, _u32, C.POINTER(C.c_float)]),
    "pico_gpu_lde_split": (C.c_int, [_vp, C.c_int, _u32, _u32, C.POINTER(_u32)]),
    "pico_gpu_open_sizes": (C.c_int, [C.POINTER(OpenBatch), _u32, _u32, C.POINTER(_u64), C.POINTER(_u32),
                                      C.POINTER(_u64)]),
    "pico_gpu_pcs_open": (
        C.c_int,
        [_vp, C.POINTER(OpenBatch), _u32, C.POINTER(FriParams), C.POINTER(Challenger), _vp, _vp, _vp, _vp,
         C.POINTER(_u32), _vp, _vp, C.POINTER(OpenStats)],
    ),
    "pico_gpu_open_values": (C.c_int, [_vp, C.POINTER(OpenBatch), _u32, _u32, _vp]),
    "pico_gpu_reduced_opening": (C.c_int, [_vp, C.POINTER(OpenBatch), _u32, _u32, _vp, _vp, _u32, _vp]),
    "pico_gpu_test_fail_allocations": (C.c_int, [C.c_int64]),
    "pico_gpu_quotient_values": (
        C.c_int,
        [_vp, TraceRef, TraceRef, TraceRef, _u32, _u32, _vp, _u32, _vp, _u32, _vp, _u32, _vp, _vp, _vp, _vp, _u32],
    ),
    "pico_gpu_challenger_observe": (C.c_int, [C.c_int, C.POINTER(Challenger), _vp, _u64]),
    "pico_gpu_challenger_sample": (C.c_int, [C.c_int, C.POINTER(Challenger), _vp, _u64]),
}

_lib = None
_lock = threading.Lock()


def lib_path() -> Path:
    return _build.LIB


def load(build_if_needed: bool = True) -> C.CDLL:
    """Load libpico_gpu.so, building it first if it is missing or stale."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_needed and not _build.up_to_date():
            _build.build()
        path = _build.LIB
        if not path.exists():
            raise RuntimeError(f"{path} is missing; run pico_b200/build.py (requires nvcc)")
        lib = C.CDLL(str(path))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int) -> None:
    if status != PICO_OK:
        msg = load().pico_gpu_last_error()
        raise PicoError(status, msg.decode() if msg else "")
