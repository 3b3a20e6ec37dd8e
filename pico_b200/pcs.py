"""Host-side mirror of the prover's commitment interface, over the C ABI.

Names and argument meanings follow the Plonky3 types the reference binds in
vm/src/configs/stark_config/kb_poseidon2.rs:15-27 (and bb_poseidon2.rs):
TwoAdicFriPcs (commit, get_evaluations_on_domain, the FRI commit phase),
MerkleTreeMmcs (commit, open_batch), Radix2DitParallel (coset_lde_batch) and
the Poseidon2 permutation.  Errors surface as PicoError with the library's
status code and message, the way the Rust shim would panic on misuse.

Matrices are numpy uint32 arrays (host, Monty form) or CUDA tensors whose
int32/uint32 storage holds the same bit patterns (device).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import abi
from . import fields as F


def _is_device(a) -> bool:
    return hasattr(a, "is_cuda") and bool(a.is_cuda)


def _ptr(a) -> int:
    if _is_device(a):
        if not a.is_contiguous():
            raise ValueError("device matrices must be contiguous")
        return a.data_ptr()
    if not (isinstance(a, np.ndarray) and a.dtype == np.uint32 and a.flags["C_CONTIGUOUS"]):
        raise ValueError("host matrices must be C-contiguous numpy uint32 arrays")
    return a.ctypes.data


def _log2_exact(n: int) -> int:
    if n <= 0 or n & (n - 1):
        raise ValueError(f"height {n} is not a power of two")
    return n.bit_length() - 1


class GpuContext:
    """One device context (pico_gpu_init).  Thread-safe; close() when done."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0, n_streams: int = 0, max_inflight: int = 0,
                 max_group: int = 0):
        self.lib = abi.load()
        cfg = abi.Config()
        cfg.hbm_budget_bytes = hbm_budget_bytes
        cfg.n_streams = n_streams
        cfg.max_inflight = max_inflight
        cfg.max_group = max_group
        h = C.c_void_p()
        abi.check(self.lib.pico_gpu_init(device, C.byref(cfg), C.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            abi.check(self.lib.pico_gpu_shutdown(self.handle))
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def memory(self):
        r, b = C.c_uint64(), C.c_uint64()
        abi.check(self.lib.pico_gpu_memory(self.handle, C.byref(r), C.byref(b)))
        return r.value, b.value

    def reserve_pool(self, nbytes: int) -> int:
        """Grow the device memory pool to hold at least nbytes (pico_gpu_reserve_pool);
        returns the bytes the pool then holds."""
        out = C.c_uint64()
        abi.check(self.lib.pico_gpu_reserve_pool(self.handle, nbytes, C.byref(out)))
        return out.value

    def autotune(self, field, log_n_min: int = 12, log_n_max: int = 22) -> dict:
        """Time the LDE's four-step splits per height and the row-hashing block
        size on this device and keep the fastest (pico_gpu_autotune).  Returns
        {log_n: {"log_n1": chosen, "ms": {log_n1: ms}}, "hash_block": {block: ms}}."""
        f = F.field_id(field)
        heights = log_n_max - log_n_min + 1
        ms = (C.c_float * (3 * heights + 3))()
        abi.check(self.lib.pico_gpu_autotune(self.handle, f, log_n_min, log_n_max, ms))
        out = {}
        for i, l in enumerate(range(log_n_min, log_n_max + 1)):
            if any(ms[3 * i + c] < 0 for c in range(3)):  # taken from the PICO_TUNE_CACHE file
                out[l] = {"log_n1": self.lde_split(f, l), "ms": {}, "cached": True}
                continue
            times = {(l + 1) // 2 - 1 + c: ms[3 * i + c] for c in range(3) if ms[3 * i + c] > 0}
            if times:
                out[l] = {"log_n1": self.lde_split(f, l), "ms": times}
        hb = [ms[3 * heights + c] for c in range(3)]
        if any(v < 0 for v in hb):
            out["hash_block"] = {64 << c: (1.0 if hb[c] < 0 else 2.0) for c in range(3)}  # cached choice ranks first
            out["hash_block_cached"] = True
        else:
            out["hash_block"] = {64 << c: hb[c] for c in range(3)}
        return out

    def lde_split(self, field, log_n: int, set_log_n1: int = 0) -> int:
        """log2 n1 of the LDE's four-step split at height 2^log_n (0: one pass); set it if set_log_n1."""
        v = C.c_uint32()
        abi.check(self.lib.pico_gpu_lde_split(self.handle, F.field_id(field), log_n, set_log_n1, C.byref(v)))
        return v.value


@dataclass
class TwoAdicDomain:
    """TwoAdicMultiplicativeCoset: shift * <w_{2^log_n}> (shift canonical)."""

    log_n: int
    shift: int = 1


class ProverData:
    """Resident prover data of one commit (pico_commit): LDEs + digest layers."""

    def __init__(self, ctx: GpuContext, handle: C.c_void_p, root: np.ndarray, n_mats: int, field: int):
        self.ctx, self.handle, self.root, self.n_mats, self.field = ctx, handle, root, n_mats, field

    def release(self):
        if self.handle:
            abi.check(self.ctx.lib.pico_gpu_release(self.ctx.handle, self.handle))
            self.handle = None

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                self.release()
        except Exception:
            pass

    def stats(self) -> dict:
        st = abi.CommitStats()
        abi.check(self.ctx.lib.pico_gpu_commit_stats(self.handle, C.byref(st)))
        return st.as_dict()

    def lde_shape(self, i: int):
        lh, w = C.c_uint32(), C.c_uint32()
        abi.check(self.ctx.lib.pico_gpu_lde_shape(self.handle, i, C.byref(lh), C.byref(w)))
        return 1 << lh.value, w.value

    @property
    def log_max_height(self) -> int:
        return max(self.lde_shape(i)[0] for i in range(self.n_mats)).bit_length() - 1

    def lde_rows(self, i: int, begin: int = 0, end: int | None = None, out=None):
        """Committed (bit-reversed) rows [begin, end) of LDE i; host numpy unless `out` is a CUDA tensor."""
        h, w = self.lde_shape(i)
        end = h if end is None else end
        flags = 0
        if out is None:
            out = np.empty((end - begin, w), dtype=np.uint32)
        if _is_device(out):
            flags |= abi.PICO_OUTPUT_DEVICE
        abi.check(self.ctx.lib.pico_gpu_lde_rows(self.ctx.handle, self.handle, i, begin, end, _ptr(out), flags))
        return out

    def evaluations_on_domain(self, i: int, log_domain: int, out=None):
        """Pcs::get_evaluations_on_domain for g * H_(2^log_domain): natural row order
        (vm/src/machine/prover.rs:469-489)."""
        _, w = self.lde_shape(i)
        if out is None:
            out = np.zeros((1 << log_domain, w), dtype=np.uint32)
        flags = abi.PICO_OUTPUT_DEVICE if _is_device(out) else 0
        abi.check(self.ctx.lib.pico_gpu_evaluations_on_domain(self.ctx.handle, self.handle, i, log_domain,
                                                               _ptr(out), flags))
        return out

    def lde(self, i: int):
        return self.lde_rows(i)

    def digest_layer(self, level: int) -> np.ndarray:
        n = 1 << (self.log_max_height - level)
        out = np.empty((n, 8), dtype=np.uint32)
        abi.check(self.ctx.lib.pico_gpu_digest_layer(self.ctx.handle, self.handle, level, out.ctypes.data, 0))
        return out


class MerkleTreeMmcs:
    """MerkleTreeMmcs<_, _, PaddingFreeSponge<Perm,16,8,8>, TruncatedPermutation<Perm,2,8,16>, 8>
    (kb_poseidon2.rs:17-20; mixed heights as vm/src/compiler/recursion/circuit/fri.rs:389-436 verifies them)."""

    def __init__(self, ctx: GpuContext, field):
        self.ctx, self.field = ctx, F.field_id(field)

    def commit(self, matrices, plain: bool = False):
        mats = (abi.Matrix * len(matrices))()
        flags = abi.PICO_COMMIT_PLAIN if plain else 0
        dev = [_is_device(m) for m in matrices]
        if any(dev) and not all(dev):
            raise ValueError("matrices must be all host or all device")
        if all(dev):
            flags |= abi.PICO_INPUT_DEVICE
        for k, m in enumerate(matrices):
            mats[k].values = _ptr(m)
            mats[k].log_height = _log2_exact(m.shape[0])
            mats[k].width = m.shape[1]
        root = np.zeros(8, dtype=np.uint32)
        h = C.c_void_p()
        abi.check(self.ctx.lib.pico_gpu_mmcs_commit(
            self.ctx.handle, self.field, mats, len(matrices), flags, C.byref(h),
            root.ctypes.data_as(C.POINTER(C.c_uint32))))
        return root, ProverData(self.ctx, h, root, len(matrices), self.field)

    def open_batch(self, index: int, prover_data: ProverData):
        """(opened rows per matrix, sibling path) at `index` of the tallest matrix
        (the BatchOpening fri.rs:389-436 checks)."""
        widths = [prover_data.lde_shape(i)[1] for i in range(prover_data.n_mats)]
        rows = np.zeros(sum(widths), dtype=np.uint32)
        path = np.zeros((prover_data.log_max_height, 8), dtype=np.uint32)
        abi.check(self.ctx.lib.pico_gpu_open_batch(self.ctx.handle, prover_data.handle, index,
                                                   rows.ctypes.data, path.ctypes.data))
        out, off = [], 0
        for w in widths:
            out.append(rows[off:off + w].copy())
            off += w
        return out, path


class Radix2DitParallel:
    """SC_Dft: coset LDE of a batch of columns (kb_poseidon2.rs:25; committed row i
    is x = g * w_N^rev(i), fri.rs:155-171)."""

    def __init__(self, ctx: GpuContext, field):
        self.ctx, self.field = ctx, F.field_id(field)

    def coset_lde_batch_bitrev(self, mat, added_bits: int, shift_monty: int, out=None):
        """LDE rows in the committed (bit-reversed) order."""
        n, w = mat.shape
        flags = abi.PICO_INPUT_DEVICE if _is_device(mat) else 0
        if out is None:
            out = np.empty((n << added_bits, w), dtype=np.uint32)
        if _is_device(out):
            flags |= abi.PICO_OUTPUT_DEVICE
        abi.check(self.ctx.lib.pico_gpu_coset_lde_batch(self.ctx.handle, self.field, _ptr(mat), _log2_exact(n), w,
                                                        added_bits, shift_monty, _ptr(out), flags))
        return out

    def coset_lde_batch(self, mat, added_bits: int, shift_monty: int) -> np.ndarray:
        """Natural row order, as the Dft trait returns it (host result)."""
        br = self.coset_lde_batch_bitrev(mat, added_bits, shift_monty)
        logn = _log2_exact(br.shape[0])
        idx = np.arange(br.shape[0])
        rev = np.zeros_like(idx)
        for b in range(logn):
            rev |= ((idx >> b) & 1) << (logn - 1 - b)
        return br[rev]


class Poseidon2:
    def __init__(self, ctx: GpuContext, field):
        self.ctx, self.field = ctx, F.field_id(field)

    def permute(self, states, four_lanes: bool = False):
        """In place on (n, 16) states (host numpy or CUDA tensor); four_lanes:
        four threads per state (the latency form)."""
        flags = abi.PICO_INPUT_DEVICE if _is_device(states) else 0
        if four_lanes:
            flags |= abi.PICO_P2_FOUR_LANES
        abi.check(self.ctx.lib.pico_gpu_poseidon2_permute(self.ctx.handle, self.field, _ptr(states),
                                                          states.shape[0], flags))
        return states


@dataclass
class FriCommitResult:
    roots: np.ndarray
    betas: np.ndarray
    final_poly: np.ndarray
    rounds: int
    data: "FriData | None"


class FriData:
    def __init__(self, ctx, handle, log_n):
        self.ctx, self.handle, self.log_n = ctx, handle, log_n

    def layer(self, r: int) -> np.ndarray:
        out = np.empty(((1 << (self.log_n - r)), 4), dtype=np.uint32)
        abi.check(self.ctx.lib.pico_gpu_fri_layer(self.ctx.handle, self.handle, r, out.ctypes.data, 0))
        return out

    def release(self):
        if self.handle:
            abi.check(self.ctx.lib.pico_gpu_fri_release(self.ctx.handle, self.handle))
            self.handle = None

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                self.release()
        except Exception:
            pass


def last_commit_stats() -> dict:
    """Device timings of the calling thread's last synchronous commit."""
    st = abi.CommitStats()
    abi.check(abi.load().pico_gpu_last_commit_stats(C.byref(st)))
    return st.as_dict()


def new_challenger() -> abi.Challenger:
    """DuplexChallenger::new: zero sponge, empty buffers (observe / sample as
    vm/src/compiler/recursion/circuit/challenger.rs:89-106, 223-234)."""
    return abi.Challenger()


class _OpenBatches:
    """ctypes view of [(ProverData, points per matrix)] for the opening calls."""

    def __init__(self, rounds):
        self.keep = []
        self.arr = (abi.OpenBatch * len(rounds))()
        self.n = len(rounds)
        for b, (pd, points) in enumerate(rounds):
            pts = [np.asarray(P, dtype=np.uint32).reshape(-1, 4) for P in points]
            if len(pts) != pd.n_mats:
                raise ValueError(f"batch {b}: {len(pts)} point lists for {pd.n_mats} matrices")
            npts = np.array([len(P) for P in pts], dtype=np.uint32)
            flat = np.ascontiguousarray(np.concatenate(pts) if npts.sum() else np.zeros((1, 4), np.uint32))
            self.keep += [npts, flat]
            self.arr[b] = abi.OpenBatch(pd.handle.value, npts.ctypes.data, flat.ctypes.data)

    def sizes(self, log_blowup: int):
        vw, r, qw = C.c_uint64(), C.c_uint32(), C.c_uint64()
        abi.check(abi.load().pico_gpu_open_sizes(self.arr, self.n, log_blowup, C.byref(vw), C.byref(r),
                                                 C.byref(qw)))
        return vw.value, r.value, qw.value


class TwoAdicFriPcs:
    """SC_Pcs = TwoAdicFriPcs<Val, Dft, ValMmcs, ChallengeMmcs>."""

    def __init__(self, ctx: GpuContext, field, log_blowup: int):
        self.ctx, self.field, self.log_blowup = ctx, F.field_id(field), log_blowup

    def natural_domain_for_degree(self, n: int) -> TwoAdicDomain:
        return TwoAdicDomain(_log2_exact(n), 1)

    def commit_bytes(self, domains_and_traces, plain: bool = False):
        """(resident, scratch) device bytes a commit of these traces reserves
        against the context's HBM budget (pico_gpu_commit_bytes); no device needed."""
        mats, flags = self._descriptors(domains_and_traces, plain)
        res, scr = C.c_uint64(), C.c_uint64()
        abi.check(abi.load().pico_gpu_commit_bytes(self.field, mats, len(domains_and_traces), self.log_blowup, flags,
                                                   C.byref(res), C.byref(scr)))
        return res.value, scr.value

    def _descriptors(self, domains_and_traces, plain: bool):
        n = len(domains_and_traces)
        mats = (abi.Matrix * n)()
        flags = abi.PICO_COMMIT_PLAIN if plain else 0
        traces = [t for _, t in domains_and_traces]
        dev = [_is_device(t) for t in traces]
        if any(dev) and not all(dev):
            raise ValueError("traces must be all host or all device")
        if all(dev):
            flags |= abi.PICO_INPUT_DEVICE
        for k, (dom, t) in enumerate(domains_and_traces):
            if t.shape[0] != 1 << dom.log_n:
                raise ValueError(f"trace {k}: height {t.shape[0]} != domain size {1 << dom.log_n}")
            ext = len(t.shape) == 3
            if ext and t.shape[2] != 4:
                raise ValueError(f"trace {k}: extension traces have 4 words per element")
            mats[k].values = _ptr(t)
            mats[k].log_height = dom.log_n
            mats[k].width = t.shape[1]
            mats[k].shift = F.lde_shift(self.field, dom.shift)
            # (n, w, 4) extension traces commit as their base flattening (flatten_to_base)
            mats[k].flags = abi.PICO_MATRIX_EXT4 if ext else 0
        return mats, flags

    def commit(self, domains_and_traces, plain: bool = False, keep: bool = True):
        """[(domain, trace)] -> (root, ProverData).  LDE shift per matrix is
        GENERATOR / domain.shift, as TwoAdicFriPcs::commit computes it (called at
        vm/src/machine/prover.rs:102,244,415,540)."""
        n = len(domains_and_traces)
        mats, flags = self._descriptors(domains_and_traces, plain)
        root = np.zeros(8, dtype=np.uint32)
        h = C.c_void_p()
        abi.check(self.ctx.lib.pico_gpu_commit(
            self.ctx.handle, self.field, mats, n, self.log_blowup, flags,
            C.byref(h) if keep else None, root.ctypes.data_as(C.POINTER(C.c_uint32))))
        pd = ProverData(self.ctx, h, root, n, self.field) if keep else None
        return root, pd

    def commit_shard(self, domains_and_traces, log_shards: int, shard: int, keep: bool = True):
        """Shard `shard` of 2^log_shards of the same commit split by rows
        (pico_gpu_commit_shard): its rows of every committed LDE and the root
        of their subtree.  log_shards <= log_blowup."""
        n = len(domains_and_traces)
        mats, flags = self._descriptors(domains_and_traces, False)
        root = np.zeros(8, dtype=np.uint32)
        h = C.c_void_p()
        abi.check(self.ctx.lib.pico_gpu_commit_shard(
            self.ctx.handle, self.field, mats, n, self.log_blowup, log_shards, shard, flags,
            C.byref(h) if keep else None, root.ctypes.data_as(C.POINTER(C.c_uint32))))
        pd = ProverData(self.ctx, h, root, n, self.field) if keep else None
        return root, pd

    def get_evaluations_on_domain(self, prover_data: ProverData, idx: int):
        """The committed LDE of matrix idx (bit-reversed rows, as stored)."""
        return prover_data.lde(idx)

    def fri_commit_phase(self, codeword, log_final_len: int = 0, betas=None, challenger=None,
                         keep: bool = False) -> FriCommitResult:
        """FRI commit phase over an EF4 codeword ((2^k, 4) Monty words, bit-reversed order;
        fold and layer commits as fri.rs:288-387 verifies them)."""
        log_n = _log2_exact(codeword.shape[0])
        rounds = log_n - self.log_blowup - log_final_len
        if rounds < 0:
            raise ValueError("codeword shorter than the final length")
        flags = abi.PICO_INPUT_DEVICE if _is_device(codeword) else 0
        roots = np.zeros((max(rounds, 1), 8), dtype=np.uint32)
        out_betas = np.zeros((max(rounds, 1), 4), dtype=np.uint32)
        final = np.zeros((1 << log_final_len, 4), dtype=np.uint32)
        if betas is not None:
            betas = np.ascontiguousarray(betas, dtype=np.uint32)
        ch = challenger if challenger is not None else (new_challenger() if betas is None else None)
        nr = C.c_uint32()
        h = C.c_void_p()
        abi.check(self.ctx.lib.pico_gpu_fri_commit_phase(
            self.ctx.handle, self.field, _ptr(codeword), log_n, self.log_blowup, log_final_len,
            betas.ctypes.data if betas is not None else None,
            C.byref(ch) if ch is not None else None, flags, roots.ctypes.data, out_betas.ctypes.data,
            final.ctypes.data, C.byref(nr), C.byref(h) if keep else None))
        data = FriData(self.ctx, h, log_n) if keep else None
        return FriCommitResult(roots[:rounds], out_betas[:rounds], final, nr.value, data)

    def open(self, rounds, challenger, num_queries: int = 84, proof_of_work_bits: int = 16):
        """TwoAdicFriPcs::open over [(ProverData, points per matrix)] (called at
        vm/src/machine/prover.rs:589; the proof is what
        vm/src/compiler/recursion/circuit/fri.rs:77-436 verifies): returns the
        opened values (per batch, matrix, point: (width, 4)) and the proof pieces.
        The challenger is advanced in place, as the prover's is."""
        ob = _OpenBatches(rounds)
        vw, R, qw = ob.sizes(self.log_blowup)
        values = np.zeros(max(vw, 4), dtype=np.uint32)
        roots = np.zeros((max(R, 1), 8), dtype=np.uint32)
        betas = np.zeros((max(R, 1), 4), dtype=np.uint32)
        final = np.zeros(4, dtype=np.uint32)
        wit = C.c_uint32()
        idx = np.zeros(max(num_queries, 1), dtype=np.uint32)
        queries = np.zeros((max(num_queries, 1), qw), dtype=np.uint32)
        params = abi.FriParams(self.log_blowup, num_queries, proof_of_work_bits, 0)
        st = abi.OpenStats()
        abi.check(self.ctx.lib.pico_gpu_pcs_open(
            self.ctx.handle, ob.arr, ob.n, C.byref(params), C.byref(challenger), values.ctypes.data, roots.ctypes.data,
            betas.ctypes.data, final.ctypes.data, C.byref(wit), idx.ctypes.data, queries.ctypes.data, C.byref(st)))
        return {
            "values": values[:vw].reshape(-1, 4),
            "roots": roots[:R],
            "betas": betas[:R],
            "final": final,
            "pow_witness": wit.value,
            "indices": idx[:num_queries],
            "queries": queries[:num_queries],
            "stats": st.as_dict(),
        }


    def open_values(self, rounds):
        """Opened values p(z) of every matrix at each of its points, (n, 4) Monty words."""
        ob = _OpenBatches(rounds)
        vw, _, _ = ob.sizes(self.log_blowup)
        values = np.zeros(max(vw, 4), dtype=np.uint32)
        abi.check(self.ctx.lib.pico_gpu_open_values(self.ctx.handle, ob.arr, ob.n, self.log_blowup, values.ctypes.data))
        return values[:vw].reshape(-1, 4)


    def reduced_opening(self, rounds, values, alpha, log_height: int):
        """The reduced opening of LDE height 2^log_height for given values and alpha."""
        ob = _OpenBatches(rounds)
        v = np.ascontiguousarray(values, dtype=np.uint32)
        a = np.ascontiguousarray(alpha, dtype=np.uint32)
        out = np.zeros((1 << log_height, 4), dtype=np.uint32)
        abi.check(self.ctx.lib.pico_gpu_reduced_opening(self.ctx.handle, ob.arr, ob.n, self.log_blowup,
                                                         v.ctypes.data if v.size else None, a.ctypes.data, log_height,
                                                         out.ctypes.data))
        return out


class CommitRequest:
    def __init__(self, server: "CommitServer", handle: C.c_void_p, n_mats: int, field: int):
        self.server, self.handle, self.n_mats, self.field = server, handle, n_mats, field

    def poll(self) -> bool:
        s = self.server.ctx.lib.pico_gpu_poll(self.server.ctx.handle, self.handle)
        if s == 6:  # PICO_ERR_NOT_READY
            return False
        abi.check(s)
        return True

    def wait(self, timeout_ms: int = -1, keep: bool = True):
        root = np.zeros(8, dtype=np.uint32)
        h = C.c_void_p()
        abi.check(self.server.ctx.lib.pico_gpu_wait(
            self.server.ctx.handle, self.handle, timeout_ms, C.byref(h) if keep else None,
            root.ctypes.data_as(C.POINTER(C.c_uint32))))
        pd = ProverData(self.server.ctx, h, root, self.n_mats, self.field) if keep else None
        return root, pd

    def times(self):
        q, r = C.c_double(), C.c_double()
        abi.check(self.server.ctx.lib.pico_gpu_request_times(self.handle, C.byref(q), C.byref(r)))
        return q.value, r.value

    def cancel(self):
        abi.check(self.server.ctx.lib.pico_gpu_cancel(self.server.ctx.handle, self.handle))

    def free(self):
        if self.handle:
            abi.check(self.server.ctx.lib.pico_gpu_request_free(self.server.ctx.handle, self.handle))
            self.handle = None


class CommitServer:
    """Serving front end: asynchronous commits admitted by free HBM."""

    def __init__(self, ctx: GpuContext):
        self.ctx = ctx

    def submit(self, field, traces, log_blowup: int, shifts=None, plain: bool = False) -> CommitRequest:
        f = F.field_id(field)
        n = len(traces)
        mats = (abi.Matrix * n)()
        dev = [_is_device(t) for t in traces]
        if any(dev) and not all(dev):
            raise ValueError("traces must be all host or all device")
        flags = abi.PICO_INPUT_DEVICE if all(dev) else 0
        if plain:
            flags |= abi.PICO_COMMIT_PLAIN
        for k, t in enumerate(traces):
            mats[k].values = _ptr(t)
            mats[k].log_height = _log2_exact(t.shape[0])
            mats[k].width = t.shape[1]
            mats[k].shift = shifts[k] if shifts is not None else F.lde_shift(f)
        h = C.c_void_p()
        abi.check(self.ctx.lib.pico_gpu_submit_commit(self.ctx.handle, f, mats, n, log_blowup, flags, C.byref(h)))
        return CommitRequest(self, h, n, f)


def merkle_top(field, shard_roots) -> np.ndarray:
    """Root of a Merkle tree from its 2^k subtree roots at depth k, in order
    (pico_gpu_merkle_top; host only)."""
    roots = np.ascontiguousarray(np.asarray(shard_roots, dtype=np.uint32).reshape(-1, 8))
    k = _log2_exact(roots.shape[0])
    out = np.zeros(8, dtype=np.uint32)
    abi.check(abi.load().pico_gpu_merkle_top(F.field_id(field), roots.ctypes.data_as(C.POINTER(C.c_uint32)), k,
                                             out.ctypes.data_as(C.POINTER(C.c_uint32))))
    return out


def merkle_top_path(field, shard_roots, shard: int) -> np.ndarray:
    """The siblings above shard `shard`'s subtree root, lowest first
    (pico_gpu_merkle_top_path): appended to the shard's own open_batch path,
    the path through the whole row-split commit."""
    roots = np.ascontiguousarray(np.asarray(shard_roots, dtype=np.uint32).reshape(-1, 8))
    k = _log2_exact(roots.shape[0])
    out = np.zeros((k, 8), dtype=np.uint32)
    abi.check(abi.load().pico_gpu_merkle_top_path(F.field_id(field), roots.ctypes.data_as(C.POINTER(C.c_uint32)), k,
                                                  shard, out.ctypes.data_as(C.POINTER(C.c_uint32))))
    return out
