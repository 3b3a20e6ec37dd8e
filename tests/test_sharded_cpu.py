"""A commit split by rows over two gloo ranks, on CPU.

The shard arithmetic is checked against the oracle: shard s of 2^k is the
MMCS of rows [s N / 2^k, (s + 1) N / 2^k) of every committed LDE, its root is
the full tree's node at depth k, and pico_gpu_merkle_top over the 2^k shard
roots is the commitment root.  The two ranks stand in for two GPUs: each
computes its shard root with the oracle and the product's gather_root does
the all-gather and the top levels."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

SHAPES = [(7, 5), (7, 2), (5, 3), (3, 1), (0, 2)]  # log heights 7..0 and a height-1 trace


def _traces(f):
    from pico_b200 import fields as F

    return [F.random_matrix(f, lh, w, 8800 + 13 * i + f) for i, (lh, w) in enumerate(SHAPES)]


def _shard_root(orc, f, mats, b, k, s):
    """The oracle's shard: rows block s of 2^k of every committed LDE, as an MMCS."""
    from pico_b200 import fields as F

    _, ldes, _ = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b, want_ldes=True)
    blocks = [l[s * (l.shape[0] >> k):(s + 1) * (l.shape[0] >> k)] for l in ldes]
    return orc.mmcs_commit(f, blocks)


@pytest.mark.parametrize("f,b,k", [(0, 1, 1), (1, 2, 2), (0, 2, 1)])
def test_shard_roots_are_the_tree_at_depth_k(orc, f, b, k):
    from pico_b200 import fields as F
    from pico_b200.pcs import merkle_top

    mats = _traces(f)
    root, _, layers = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b, want_layers=True)
    subs = np.stack([_shard_root(orc, f, mats, b, k, s) for s in range(1 << k)])
    # the layers array holds the levels leaves first; depth k is the 2^k nodes before the top 2^k - 1
    depth_k = layers[len(layers) - (2 << k) + 1: len(layers) - (1 << k) + 1]
    assert np.array_equal(subs, depth_k)
    assert merkle_top(f, subs).tolist() == root.tolist()
    assert merkle_top(f, root.reshape(1, 8)).tolist() == root.tolist()


def _rank_main(rank, world, port, out_dir, f, b):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle import cpu as orc
        from pico_b200.sharded import gather_root

        k = world.bit_length() - 1
        sub = _shard_root(orc, f, _traces(f), b, k, rank)
        root = gather_root(f, sub)
        np.save(Path(out_dir) / f"rank{rank}.npy", np.concatenate([sub, root]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("f,b", [(0, 1), (1, 2)])
def test_two_rank_row_split_gloo(tmp_path, orc, f, b):
    import socket

    import torch.multiprocessing as mp

    from pico_b200 import fields as F

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path), f, b), nprocs=world, start_method="spawn",
                       join=True)
    mats = _traces(f)
    want, _, _ = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b)
    got = [np.load(tmp_path / f"rank{r}.npy").astype(np.uint32) for r in range(world)]
    assert got[0][:8].tolist() != got[1][:8].tolist()  # distinct shards
    for g in got:
        assert g[8:].tolist() == want.tolist()  # every rank holds the commitment root


def test_merkle_top_refuses_bad_arguments():
    from pico_b200 import PicoError
    from pico_b200.pcs import merkle_top

    with pytest.raises(ValueError):
        merkle_top(0, np.zeros((3, 8), dtype=np.uint32))  # not a power of two
    with pytest.raises(PicoError):
        merkle_top(7, np.zeros((2, 8), dtype=np.uint32))  # unknown field


@pytest.mark.parametrize("f,b,k", [(0, 1, 1), (1, 2, 2)])
def test_merkle_top_path_is_the_upper_path(orc, f, b, k):
    """pico_gpu_merkle_top_path: the siblings of shard s's subtree root up to
    the root, the last k digests of every Merkle path through that shard."""
    from pico_b200 import fields as F
    from pico_b200.pcs import merkle_top_path

    mats = _traces(f)
    _, _, layers = orc.pcs_commit(f, mats, [F.lde_shift(f)] * len(mats), b, want_layers=True)
    depth = lambda d: layers[len(layers) - (2 << d) + 1: len(layers) - (1 << d) + 1]
    roots = depth(k)
    for s in range(1 << k):
        want = np.stack([depth(d)[(s >> (k - d)) ^ 1] for d in range(k, 0, -1)])
        assert np.array_equal(merkle_top_path(f, roots, s), want)
    assert merkle_top_path(f, roots[:1], 0).shape == (0, 8)
