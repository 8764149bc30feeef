"""Multi-rank host logic on CPU: world_size 2 with the gloo backend.

Each rank fakes its shard's tracking output (no GPU); the test checks the
contiguous seed split, the all-gather of counts and that the jointly written
TRX equals the rank-ordered concatenation.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _fake_rank_output(rank, seeds):
    rng = np.random.default_rng(100 + rank)
    lens = rng.integers(1, 30, 2 * len(seeds)).astype(np.int32)
    pts = rng.normal(size=(int(lens.sum()), 3)).astype(np.float32) + 10 * rank
    return lens, pts


def _worker(rank, world, port, tmp, nseeds):
    import torch.distributed as dist

    from gpustreamlines_b200 import distributed as D

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        start, stop = D.shard(nseeds, rank, world)
        seeds = np.arange(nseeds * 3, dtype=np.float32).reshape(nseeds, 3)[start:stop]
        lens, pts = _fake_rank_output(rank, seeds)
        counts, sl_off, pt_off = D.gather_counts(len(lens), len(pts))
        if rank == 0:
            D.create_shared_trx(tmp, counts)
        dist.barrier()
        D.write_shard_trx(tmp, rank, counts, sl_off, pt_off, lens, pts,
                          {"DIMENSIONS": [4, 4, 4], "VOXEL_TO_RASMM": np.eye(4).tolist()})
        dist.barrier()
        if rank == 0:
            D.seal_trx(tmp, os.path.join(tmp, "all.trx"))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nseeds", [7, 10])
def test_two_rank_shards_and_trx(tmp_path, nseeds):
    from gpustreamlines_b200 import distributed as D
    from gpustreamlines_b200 import io

    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), nseeds), nprocs=world,
                       join=True, start_method="spawn")
    hdr, seq = io.load_trx(str(tmp_path / "all.trx"))
    want_l, want_p = [], []
    for r in range(world):
        a, b = D.shard(nseeds, r, world)
        l, p = _fake_rank_output(r, np.zeros((b - a, 3)))
        want_l.append(l)
        want_p.append(p)
    wl = np.concatenate(want_l)
    assert hdr["NB_STREAMLINES"] == len(wl)
    assert np.array_equal(seq._lengths, wl)
    assert np.array_equal(seq._data, np.concatenate(want_p))


def test_shard_matches_reference_split():
    from gpustreamlines_b200 import distributed as D

    # cu_propagate_seeds.py:45-54: ceil(n/ngpus) per GPU, the last one short
    assert [D.shard(10, r, 3) for r in range(3)] == [(0, 4), (4, 8), (8, 10)]
    assert [D.shard(2, r, 4) for r in range(4)] == [(0, 1), (1, 2), (2, 2), (2, 2)]
