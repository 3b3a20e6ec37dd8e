"""A commit split by rows across the ranks of a process group, one GPU per
rank (the split of one `pcs.commit`, vm/src/machine/prover.rs:102, that the
reference runs on one host).

Shard s of 2^k holds rows [s N / 2^k, (s + 1) N / 2^k) of every committed LDE:
the LDE's coset blocks s 2^(b-k) .. (s + 1) 2^(b-k) - 1, which each rank
computes from the whole trace (pico_gpu_commit_shard), so no trace or LDE data
crosses devices and k <= log_blowup.  Its Merkle tree is the full tree's
subtree under node s at depth k.  One all-gather of the 2^k eight-word shard
roots, then the top k compression levels on every rank (pico_gpu_merkle_top),
give every rank the commitment root.  Rank r of the group computes shard r.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from . import fields as F
from .pcs import _is_device, _ptr, merkle_top, new_challenger


def _log2_world(world: int) -> int:
    k = world.bit_length() - 1
    if world <= 0 or (1 << k) != world:
        raise ValueError(f"a row-split commit needs a power-of-two number of ranks, not {world}")
    return k


def gather_root(field, shard_root, group=None) -> np.ndarray:
    """All-gather this rank's shard root over `group` (torch.distributed; the
    tensors live on the current CUDA device under NCCL, on the host under
    gloo) and return the commitment root, the same on every rank."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    _log2_world(world)
    t = torch.from_numpy(np.ascontiguousarray(shard_root, dtype=np.uint32).view(np.int32).copy())
    if dist.get_backend(group) == "nccl":
        t = t.to(torch.device("cuda", torch.cuda.current_device()))
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    roots = np.stack([p.cpu().numpy().view(np.uint32) for p in parts])
    return merkle_top(field, roots)


def commit_sharded(pcs, domains_and_traces, group=None, keep: bool = True):
    """Commit `domains_and_traces` split by rows over `group`: returns (root
    of the whole commit, this rank's prover data, this rank's shard root)."""
    import torch.distributed as dist

    k = _log2_world(dist.get_world_size(group))
    shard_root, pd = pcs.commit_shard(domains_and_traces, k, dist.get_rank(group), keep=keep)
    return gather_root(pcs.field, shard_root, group), pd, shard_root


# ---------------------------------------------------------------- FRI commit phase
class FriShard:
    """One shard's part of a FRI commit phase split by rows
    (pico_gpu_fri_shard_*): `rows` are this shard's 2^(log_n - k) rows of the
    2^log_n-row EF4 codeword, (rows, 4) Monty words, host or device."""

    def __init__(self, ctx, field, rows, log_n: int, log_shards: int, shard: int):
        self.ctx, self.field = ctx, F.field_id(field)
        self.log_len, self.log_shards = log_n, log_shards
        self.root = np.zeros(8, dtype=np.uint32)
        h = C.c_void_p()
        flags = abi.PICO_INPUT_DEVICE if _is_device(rows) else 0
        if not _is_device(rows):
            rows = np.ascontiguousarray(rows, dtype=np.uint32)
        self._keep = rows
        abi.check(ctx.lib.pico_gpu_fri_shard_begin(ctx.handle, self.field, _ptr(rows), log_n, log_shards, shard,
                                                   flags, C.byref(h), self.root.ctypes.data_as(C.POINTER(C.c_uint32))))
        self.handle = h

    def log_rows(self) -> int:
        return self.log_len - self.log_shards

    def fold(self, beta) -> np.ndarray:
        b = np.ascontiguousarray(beta, dtype=np.uint32).reshape(4)
        abi.check(self.ctx.lib.pico_gpu_fri_shard_fold(self.handle, b.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                       self.root.ctypes.data_as(C.POINTER(C.c_uint32))))
        self.log_len -= 1
        return self.root

    def rows(self) -> np.ndarray:
        out = np.zeros((1 << self.log_rows(), 4), dtype=np.uint32)
        abi.check(self.ctx.lib.pico_gpu_fri_shard_rows(self.handle, out.ctypes.data, 0))
        return out

    def release(self):
        if self.handle:
            abi.check(self.ctx.lib.pico_gpu_fri_shard_release(self.handle))
            self.handle = None


def _observe(field, ch, words):
    w = np.ascontiguousarray(words, dtype=np.uint32).reshape(-1)
    abi.check(abi.load().pico_gpu_challenger_observe(field, C.byref(ch), w.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                     w.size))


def _sample(field, ch, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint32)
    abi.check(abi.load().pico_gpu_challenger_sample(field, C.byref(ch), out.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                    n))
    return out


def _split_rounds(pcs, log_n: int, k: int, shard_roots, fold, codeword, log_final_len: int, challenger,
                  min_log_rows: int):
    """The round loop of a row-split commit phase: while every shard keeps more
    than 2^min_log_rows rows, the round's root from the shard roots, observed,
    beta sampled (the prover's DuplexChallenger, on the host) and every shard
    folded; then the short codeword gathered and the rest of the phase run on
    this device by pcs.fri_commit_phase with the same challenger."""
    f = pcs.field
    ch = challenger if challenger is not None else new_challenger()
    roots, betas = [], []
    L, stop = log_n, pcs.log_blowup + log_final_len
    while L - k > max(min_log_rows, 1) and L - 1 > stop:
        root = merkle_top(f, np.stack(shard_roots()))
        _observe(f, ch, root)
        beta = _sample(f, ch, 4)
        roots.append(root)
        betas.append(beta)
        fold(beta)
        L -= 1
    rest = pcs.fri_commit_phase(codeword(), log_final_len=log_final_len, challenger=ch)
    all_roots = np.concatenate([np.stack(roots).reshape(-1, 8), rest.roots]) if roots else rest.roots
    all_betas = np.concatenate([np.stack(betas).reshape(-1, 4), rest.betas]) if betas else rest.betas
    return all_roots, all_betas, rest.final_poly, ch


def fri_commit_phase_split(pcs, codeword, log_shards: int, log_final_len: int = 0, challenger=None,
                           min_log_rows: int = 10):
    """A row-split commit phase with every shard on this device, one after the
    other (what 2^log_shards ranks do side by side): returns (roots, betas,
    final polynomial, challenger), equal to pcs.fri_commit_phase's."""
    n = codeword.shape[0]
    log_n = n.bit_length() - 1
    per = n >> log_shards
    shards = [FriShard(pcs.ctx, pcs.field, codeword[s * per:(s + 1) * per], log_n, log_shards, s)
              for s in range(1 << log_shards)]
    try:
        return _split_rounds(pcs, log_n, log_shards, lambda: [fs.root.copy() for fs in shards],
                             lambda beta: [fs.fold(beta) for fs in shards],
                             lambda: np.concatenate([fs.rows() for fs in shards]), log_final_len, challenger,
                             min_log_rows)
    finally:
        for fs in shards:
            fs.release()


def fri_commit_phase_sharded(pcs, rows, log_n: int, group=None, log_final_len: int = 0, challenger=None,
                             min_log_rows: int = 10):
    """The commit phase of a 2^log_n-row codeword split by rows over `group`:
    rank r passes its rows [r N / 2^k, (r + 1) N / 2^k); one all-gather of 8
    words per rank per round, and of the short codeword at the end.  Every
    rank returns (roots, betas, final polynomial, challenger)."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    k = _log2_world(world)
    fs = FriShard(pcs.ctx, pcs.field, rows, log_n, k, dist.get_rank(group))
    nccl = dist.get_backend(group) == "nccl"

    def gather(a):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32).copy())
        if nccl:
            t = t.to(torch.device("cuda", torch.cuda.current_device()))
        parts = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(parts, t, group=group)
        return [p.cpu().numpy().view(np.uint32) for p in parts]

    try:
        return _split_rounds(pcs, log_n, k, lambda: gather(fs.root), fs.fold,
                             lambda: np.concatenate(gather(fs.rows())), log_final_len, challenger, min_log_rows)
    finally:
        fs.release()
