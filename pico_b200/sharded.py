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

import numpy as np

from .pcs import merkle_top


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
