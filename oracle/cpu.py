"""ctypes wrapper of the C oracle (oracle/oracle.c) -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker or the timed CPU baseline; the product never does.
All arrays are numpy uint32 in Montgomery form unless a name says canonical.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
_lib = None
_lock = threading.Lock()


class Challenger(C.Structure):
    _fields_ = [
        ("sponge", C.c_uint32 * 16),
        ("in_buf", C.c_uint32 * 8),
        ("in_len", C.c_uint32),
        ("out_buf", C.c_uint32 * 8),
        ("out_len", C.c_uint32),
    ]


class OpenBatch(C.Structure):
    _fields_ = [
        ("n_mats", C.c_uint32),
        ("ldes", C.c_void_p),
        ("log_heights", C.c_void_p),
        ("widths", C.c_void_p),
        ("n_points", C.c_void_p),
        ("points", C.c_void_p),
        ("layers", C.c_void_p),
        ("root", C.c_void_p),
    ]


def build(force: bool = False) -> Path:
    srcs = [HERE / "oracle.c", HERE / "oracle.h", HERE.parent / "pico_b200" / "csrc" / "p2_rc_table.inc"]
    if force or not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "all"], check=True, capture_output=True)
    return LIB


def load():
    global _lib
    with _lock:
        if _lib is None:
            build()
            lib = C.CDLL(str(LIB))
            u32, vp, u64 = C.c_uint32, C.c_void_p, C.c_uint64
            for name, res, args in [
                ("orc_prime", u32, [C.c_int]),
                ("orc_to_monty", u32, [C.c_int, u32]),
                ("orc_from_monty", u32, [C.c_int, u32]),
                ("orc_two_adic_generator", u32, [C.c_int, u32]),
                ("orc_generator", u32, [C.c_int]),
                ("orc_num_threads", C.c_int, []),
                ("orc_set_threads", None, [C.c_int]),
                ("orc_uniform_monty", None, [C.c_int, u64, u64, vp]),
                ("orc_permute", C.c_int, [C.c_int, vp, C.c_size_t]),
                ("orc_permute_canonical", C.c_int, [C.c_int, vp]),
                ("orc_hash", C.c_int, [C.c_int, vp, C.c_size_t, vp]),
                ("orc_compress", C.c_int, [C.c_int, vp, vp, vp]),
                ("orc_mmcs_commit", C.c_int, [C.c_int, u32, vp, vp, vp, vp, vp]),
                ("orc_coset_lde", C.c_int, [C.c_int, vp, u32, u32, u32, u32, C.c_int, vp]),
                ("orc_pcs_commit", C.c_int, [C.c_int, u32, vp, vp, vp, vp, u32, vp, vp, vp]),
                ("orc_challenger_init", None, [C.POINTER(Challenger)]),
                ("orc_challenger_observe", None, [C.c_int, C.POINTER(Challenger), u32]),
                ("orc_challenger_sample", u32, [C.c_int, C.POINTER(Challenger)]),
                ("orc_fri_commit_phase", C.c_int,
                 [C.c_int, vp, u32, u32, u32, vp, C.POINTER(Challenger), vp, vp, vp, vp]),
                ("orc_ext_mul", None, [C.c_int, vp, vp, vp]),
                ("orc_ext_inv", None, [C.c_int, vp, vp]),
                ("orc_open_values", C.c_int, [C.c_int, C.POINTER(OpenBatch), u32, vp]),
                ("orc_reduce_openings", C.c_int, [C.c_int, C.POINTER(OpenBatch), u32, vp, vp, u32, vp]),
                ("orc_open_query_words", u64, [C.POINTER(OpenBatch), u32, u32]),
                ("orc_pcs_open", C.c_int,
                 [C.c_int, C.POINTER(OpenBatch), u32, u32, u32, u32, C.POINTER(Challenger), vp, vp, vp, vp, vp,
                  vp, vp, vp]),
                ("orc_quotient_values", C.c_int,
                 [C.c_int, u32, u32, vp, u32, vp, u32, vp, u32, vp, u32, vp, u32, vp, u32, vp, vp, vp, vp]),
                ("orc_verify_open", C.c_int,
                 [C.c_int, C.POINTER(OpenBatch), u32, u32, u32, u32, C.POINTER(Challenger), vp, vp, u32, vp, u32,
                  vp, vp]),
            ]:
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
        return _lib


def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"oracle {what} failed with code {rc}")


def _u32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.uint32)


def set_threads(n: int):
    load().orc_set_threads(n)


def num_threads() -> int:
    return load().orc_num_threads()


def random_matrix(field: int, log_height: int, width: int, seed: int) -> np.ndarray:
    """The seeded synthetic matrix of pico_b200.fields.random_matrix (the same
    SplitMix64 stream, Monty form), generated in C for matrices too large for
    the vectorised numpy form."""
    out = np.empty((1 << log_height, width), dtype=np.uint32)
    if out.size:
        load().orc_uniform_monty(field, seed & 0xFFFFFFFFFFFFFFFF, out.size, out.ctypes.data)
    return out


def permute_canonical(field: int, state) -> np.ndarray:
    s = _u32(state).copy()
    _check(load().orc_permute_canonical(field, s.ctypes.data), "permute")
    return s


def permute(field: int, states) -> np.ndarray:
    s = _u32(states).copy()
    _check(load().orc_permute(field, s.ctypes.data, s.size // 16), "permute")
    return s


def hash_elems(field: int, elems) -> np.ndarray:
    a = _u32(elems)
    out = np.zeros(8, dtype=np.uint32)
    _check(load().orc_hash(field, a.ctypes.data if a.size else None, a.size, out.ctypes.data), "hash")
    return out


def compress(field: int, left, right) -> np.ndarray:
    l, r = _u32(left), _u32(right)
    out = np.zeros(8, dtype=np.uint32)
    _check(load().orc_compress(field, l.ctypes.data, r.ctypes.data, out.ctypes.data), "compress")
    return out


def mmcs_commit(field: int, mats, want_layers: bool = False):
    mats = [_u32(m) for m in mats]
    n = len(mats)
    ptrs = (C.c_void_p * n)(*[m.ctypes.data for m in mats])
    heights = np.array([m.shape[0] for m in mats], dtype=np.uint64)
    widths = np.array([m.shape[1] for m in mats], dtype=np.uint32)
    root = np.zeros(8, dtype=np.uint32)
    layers = None
    if want_layers:
        hmax = int(heights.max())
        layers = np.zeros(((2 * hmax - 1), 8), dtype=np.uint32)
    _check(load().orc_mmcs_commit(field, n, ptrs, heights.ctypes.data, widths.ctypes.data, root.ctypes.data,
                                  layers.ctypes.data if layers is not None else None), "mmcs_commit")
    return (root, layers) if want_layers else root


def coset_lde(field: int, mat, log_blowup: int, shift_monty: int, bitrev: bool = True) -> np.ndarray:
    m = _u32(mat)
    n, w = m.shape
    logn = n.bit_length() - 1
    out = np.zeros((n << log_blowup, w), dtype=np.uint32)
    _check(load().orc_coset_lde(field, m.ctypes.data, logn, w, log_blowup, shift_monty, int(bitrev),
                                out.ctypes.data), "coset_lde")
    return out


def pcs_commit(field: int, mats, shifts, log_blowup: int, want_ldes: bool = False, want_layers: bool = False):
    mats = [_u32(m) for m in mats]
    n = len(mats)
    ptrs = (C.c_void_p * n)(*[m.ctypes.data for m in mats])
    logh = np.array([m.shape[0].bit_length() - 1 for m in mats], dtype=np.uint32)
    widths = np.array([m.shape[1] for m in mats], dtype=np.uint32)
    sh = _u32(shifts)
    root = np.zeros(8, dtype=np.uint32)
    ldes = None
    ldep = None
    if want_ldes:
        ldes = [np.zeros((m.shape[0] << log_blowup, m.shape[1]), dtype=np.uint32) for m in mats]
        ldep = (C.c_void_p * n)(*[l.ctypes.data for l in ldes])
    layers = None
    if want_layers:
        hmax = max(m.shape[0] for m in mats) << log_blowup
        layers = np.zeros((2 * hmax - 1, 8), dtype=np.uint32)
    _check(load().orc_pcs_commit(field, n, ptrs, logh.ctypes.data, widths.ctypes.data, sh.ctypes.data, log_blowup,
                                 root.ctypes.data, ldep, layers.ctypes.data if layers is not None else None),
           "pcs_commit")
    return root, ldes, layers


def new_challenger() -> Challenger:
    ch = Challenger()
    load().orc_challenger_init(C.byref(ch))
    return ch


def challenger_observe(field: int, ch: Challenger, v: int):
    load().orc_challenger_observe(field, C.byref(ch), v)


def challenger_sample(field: int, ch: Challenger) -> int:
    return load().orc_challenger_sample(field, C.byref(ch))


def fri_commit_phase(field: int, codeword, log_blowup: int, log_final_len: int = 0, betas=None, challenger=None):
    cw = _u32(codeword)
    log_n = cw.shape[0].bit_length() - 1
    rounds = log_n - log_blowup - log_final_len
    roots = np.zeros((max(rounds, 1), 8), dtype=np.uint32)
    out_betas = np.zeros((max(rounds, 1), 4), dtype=np.uint32)
    final = np.zeros((1 << log_final_len, 4), dtype=np.uint32)
    ch = challenger if challenger is not None else new_challenger()
    b = _u32(betas) if betas is not None else None
    nr = C.c_uint32()
    _check(load().orc_fri_commit_phase(field, cw.ctypes.data, log_n, log_blowup, log_final_len,
                                       b.ctypes.data if b is not None else None, C.byref(ch), roots.ctypes.data,
                                       out_betas.ctypes.data, final.ctypes.data, C.byref(nr)), "fri_commit_phase")
    return roots[:rounds], out_betas[:rounds], final, ch


def ext_mul(field: int, a, b) -> np.ndarray:
    x, y = _u32(a), _u32(b)
    out = np.zeros(4, dtype=np.uint32)
    load().orc_ext_mul(field, x.ctypes.data, y.ctypes.data, out.ctypes.data)
    return out


def ext_inv(field: int, a) -> np.ndarray:
    x = _u32(a)
    out = np.zeros(4, dtype=np.uint32)
    load().orc_ext_inv(field, x.ctypes.data, out.ctypes.data)
    return out


class _Batches:
    """ctypes view of opening batches.  Each batch is a dict with `ldes`
    (committed LDEs, bit-reversed rows, Monty) -- or, for the verifier alone,
    `shapes` [(LDE height, width)] --, `points` (per matrix an array of shape
    (k, 4)), and optionally `layers` and `root`."""

    def __init__(self, batches):
        self.keep = []
        arr = (OpenBatch * len(batches))()
        for b, B in enumerate(batches):
            if "ldes" in B:
                ldes = [_u32(m) for m in B["ldes"]]
                shapes = [m.shape for m in ldes]
                ptrs = (C.c_void_p * len(ldes))(*[m.ctypes.data for m in ldes])
            else:  # verifier only: LDE shapes without data
                ldes = None
                shapes = B["shapes"]
                ptrs = (C.c_void_p * len(shapes))()
            n = len(shapes)
            logh = np.array([h.bit_length() - 1 for h, _ in shapes], dtype=np.uint32)
            widths = np.array([w for _, w in shapes], dtype=np.uint32)
            pts = [np.asarray(P, dtype=np.uint32).reshape(-1, 4) for P in B["points"]]
            npts = np.array([len(P) for P in pts], dtype=np.uint32)
            flat = _u32(np.concatenate(pts) if sum(len(P) for P in pts) else np.zeros((1, 4), np.uint32))
            layers = _u32(B["layers"]) if B.get("layers") is not None else None
            root = _u32(B["root"]) if B.get("root") is not None else None
            self.keep += [ldes, ptrs, logh, widths, npts, flat, layers, root]
            arr[b] = OpenBatch(n, C.cast(ptrs, C.c_void_p), logh.ctypes.data, widths.ctypes.data,
                               npts.ctypes.data, flat.ctypes.data,
                               layers.ctypes.data if layers is not None else None,
                               root.ctypes.data if root is not None else None)
        self.arr = arr
        self.n = len(batches)
        self.value_words = sum(4 * len(np.asarray(P).reshape(-1, 4)) * w
                               for B in batches
                               for (_, w), P in zip(B["shapes"] if "shapes" in B else [m.shape for m in B["ldes"]],
                                                    B["points"]))


def open_values(field: int, batch, log_blowup: int) -> np.ndarray:
    bs = _Batches([batch])
    out = np.zeros(max(bs.value_words, 4), dtype=np.uint32)
    _check(load().orc_open_values(field, bs.arr, log_blowup, out.ctypes.data), "open_values")
    return out[: bs.value_words].reshape(-1, 4)


def reduce_openings(field: int, batches, values, alpha, log_height: int) -> np.ndarray:
    bs = _Batches(batches)
    v = _u32(values)
    a = _u32(alpha)
    out = np.zeros((1 << log_height, 4), dtype=np.uint32)
    _check(load().orc_reduce_openings(field, bs.arr, bs.n, v.ctypes.data, a.ctypes.data, log_height,
                                      out.ctypes.data), "reduce_openings")
    return out


def open_query_words(batches, log_blowup: int) -> int:
    return int(load().orc_open_query_words(_Batches(batches).arr, len(batches), log_blowup))


def pcs_open(field: int, batches, log_blowup: int, num_queries: int, pow_bits: int, challenger=None):
    """TwoAdicFriPcs::open; returns a dict of the opened values and the proof."""
    bs = _Batches(batches)
    log_max = max(m.shape[0].bit_length() - 1 for B in batches for m in B["ldes"])
    rounds = log_max - log_blowup
    qw = int(load().orc_open_query_words(bs.arr, bs.n, log_blowup))
    values = np.zeros(max(bs.value_words, 4), dtype=np.uint32)
    roots = np.zeros((max(rounds, 1), 8), dtype=np.uint32)
    betas = np.zeros((max(rounds, 1), 4), dtype=np.uint32)
    final = np.zeros(4, dtype=np.uint32)
    wit = C.c_uint32()
    idx = np.zeros(max(num_queries, 1), dtype=np.uint32)
    queries = np.zeros((max(num_queries, 1), qw), dtype=np.uint32)
    nr = C.c_uint32()
    ch = challenger if challenger is not None else new_challenger()
    _check(load().orc_pcs_open(field, bs.arr, bs.n, log_blowup, num_queries, pow_bits, C.byref(ch),
                               values.ctypes.data, roots.ctypes.data, betas.ctypes.data, final.ctypes.data,
                               C.byref(wit), idx.ctypes.data, queries.ctypes.data, C.byref(nr)), "pcs_open")
    return {
        "values": values[: bs.value_words].reshape(-1, 4),
        "roots": roots[:rounds],
        "betas": betas[:rounds],
        "final": final,
        "pow_witness": int(wit.value),
        "indices": idx[:num_queries],
        "queries": queries[:num_queries],
        "challenger": ch,
    }


def verify_open(field: int, batches, log_blowup: int, num_queries: int, pow_bits: int, proof, challenger=None):
    """The Pico verifier's checks; returns (code, indices), code 0 = verifies."""
    bs = _Batches(batches)
    ch = challenger if challenger is not None else new_challenger()
    v = _u32(proof["values"])
    roots = _u32(proof["roots"])
    fin = _u32(proof["final"])
    q = _u32(proof["queries"])
    idx = np.zeros(max(num_queries, 1), dtype=np.uint32)
    rc = load().orc_verify_open(field, bs.arr, bs.n, log_blowup, num_queries, pow_bits, C.byref(ch),
                                v.ctypes.data, roots.ctypes.data, len(proof["roots"]), fin.ctypes.data,
                                int(proof["pow_witness"]), q.ctypes.data, idx.ctypes.data)
    return rc, idx[:num_queries]


def quotient_values(field: int, log_trace: int, log_qd: int, program, main_q, prep_q=None, perm_q=None,
                    public_values=(), perm_challenges=None, regional_sum=None, global_sum=None, alpha=None):
    """compute_quotient_values (vm/src/machine/utils.rs:201-350) from the traces'
    evaluations on the quotient domain in natural order (Monty form): main_q and
    prep_q are (Q, w) base matrices, perm_q is (Q, w, 4) (extension columns).
    Returns (Q, 4) Monty words."""
    Q = 1 << (log_trace + log_qd)
    ops = _u32(program).reshape(-1, 4)
    m = _u32(main_q)
    pr = _u32(prep_q) if prep_q is not None else None
    pe = _u32(perm_q) if perm_q is not None else None
    pub = _u32(np.asarray(public_values, dtype=np.uint32).reshape(-1))
    ch = _u32(np.zeros((0, 4), np.uint32) if perm_challenges is None else perm_challenges).reshape(-1, 4)
    reg = _u32(np.zeros(4, np.uint32) if regional_sum is None else regional_sum)
    glob = _u32(np.zeros(14, np.uint32) if global_sum is None else global_sum)
    al = _u32(alpha)
    out = np.zeros((Q, 4), dtype=np.uint32)
    _check(load().orc_quotient_values(
        field, log_trace, log_qd, pr.ctypes.data if pr is not None else None, pr.shape[1] if pr is not None else 0,
        m.ctypes.data, m.shape[1], pe.ctypes.data if pe is not None else None, pe.shape[1] if pe is not None else 0,
        ops.ctypes.data, ops.shape[0], pub.ctypes.data if pub.size else None, pub.size,
        ch.ctypes.data if ch.size else None, ch.shape[0], reg.ctypes.data, glob.ctypes.data, al.ctypes.data,
        out.ctypes.data), "quotient_values")
    return out


def on_quotient_domain(field: int, trace, log_qd: int):
    """A trace's evaluations on the quotient domain GENERATOR * <w_Q> in natural
    order: its coset LDE with blowup 2^log_qd and shift GENERATOR, not
    bit-reversed (what get_evaluations_on_domain returns, prover.rs:469-489)."""
    from pico_b200 import fields as F

    t = _u32(trace)
    if t.ndim == 3:  # extension columns: flatten, extend, restore
        h, w, _ = t.shape
        return coset_lde(field, t.reshape(h, 4 * w), log_qd, F.lde_shift(field), bitrev=False).reshape(-1, w, 4)
    return coset_lde(field, t, log_qd, F.lde_shift(field), bitrev=False)
