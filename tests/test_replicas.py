"""Replica (N > 1) host logic of bench.py on CPU ranks over gloo.

Each rank commits its own shard with the CPU oracle (the GPU path is not
needed to exercise the per-rank seeding, the barrier and the max-over-ranks
timing), then rank 0 checks the job throughput against the slowest rank."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        from oracle import cpu as orc
        from pico_b200 import fields as F

        seed = bench.replica_seed(11, rank)
        shapes = [(6, 5), (4, 3)]
        mats = [F.random_matrix(0, lh, w, seed * 1000 + i) for i, (lh, w) in enumerate(shapes)]
        root, _, _ = orc.pcs_commit(0, mats, [F.lde_shift(0)] * len(mats), 1)
        bench.barrier(world)
        fake_ms = 10.0 * (rank + 1)  # rank r "took" 10 (r + 1) ms
        slowest = bench.allmax(world, fake_ms)
        cells = sum(w << lh for lh, w in shapes)
        np.save(Path(out_dir) / f"rank{rank}.npy",
                np.array([*root.tolist(), slowest, bench.job_rate(world, cells, 1, slowest)], dtype=np.float64))
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo(tmp_path):
    import socket

    import torch.multiprocessing as mp

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    world = 2
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn", join=True)
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    # distinct shards per rank, each the commitment of that rank's seeded shard
    import bench
    from oracle import cpu as orc
    from pico_b200 import fields as F

    for rank, got in ((0, r0), (1, r1)):
        seed = bench.replica_seed(11, rank)
        mats = [F.random_matrix(0, lh, w, seed * 1000 + i) for i, (lh, w) in enumerate([(6, 5), (4, 3)])]
        want, _, _ = orc.pcs_commit(0, mats, [F.lde_shift(0)] * 2, 1)
        assert got[:8].tolist() == want.tolist()
    assert r0[:8].tolist() != r1[:8].tolist()
    # max over ranks seen by every rank; throughput over the slowest rank
    assert r0[8] == r1[8] == 20.0
    cells = (5 << 6) + (3 << 4)
    assert r0[9] == pytest.approx(2 * cells / 0.020)
