"""Multi-rank host logic on CPU: world_size 2 with the gloo backend.

Each rank tracks its contiguous seed shard with the CPU oracle (standing in
for its GPU's tracker), all-gathers the counts and writes its slice of a
shared TRX layout (gpustreamlines_b200.distributed.track_shard_to_trx).  The
merged file is compared with a one-rank oracle run over all seeds:
  * global Philox indices (each seed's streams follow its index in the whole
    run): identical to the one-rank run, streamline for streamline;
  * the reference's per-GPU indices (each rank restarts at 0): identical to
    the per-shard runs concatenated in rank order.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

AFF = [[2.0, 0, 0, -24.0], [0, 2.0, 0, -28.0], [0, 0, 2.0, -20.0], [0, 0, 0, 1]]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _oracle_track(seeds, rng_index_base):
    from oracle import api, cases

    inp = cases.inputs("prob_s")
    _, L, S, P = api.Oracle(inp).track(seeds, threads=2, rng_index_base=rng_index_base)
    return L, S, P


def _worker(rank, world, port, tmp, nseeds, global_index):
    import torch.distributed as dist

    from gpustreamlines_b200 import distributed as D
    from oracle import cases

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        seeds = cases.seeds("prob_s", nseeds, seed=61)
        D.track_shard_to_trx(_oracle_track, seeds, rank, world, tmp, AFF, cases.inputs("prob_s")["stop_map"].shape,
                             global_rng_index=global_index)
    finally:
        dist.destroy_process_group()


def _world(P):
    a = np.asarray(AFF)
    return (P.astype(np.float64) @ a[:3, :3].T + a[:3, 3]).astype(np.float32)


@pytest.mark.parametrize("global_index", [True, False])
def test_two_rank_tracking_matches_one_rank(tmp_path, global_index):
    from gpustreamlines_b200 import distributed as D
    from gpustreamlines_b200 import io
    from oracle import cases

    world, nseeds = 2, 301
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), nseeds, global_index), nprocs=world,
                       join=True, start_method="spawn")
    hdr, seq = io.load_trx(str(tmp_path / "all.trx"))
    seeds = cases.seeds("prob_s", nseeds, seed=61)
    if global_index:
        L, _, P = _oracle_track(seeds, 0)
    else:
        parts = [_oracle_track(seeds[slice(*D.shard(nseeds, r, world))], 0) for r in range(world)]
        L = np.concatenate([p[0] for p in parts])
        P = np.concatenate([p[2] for p in parts])
    assert hdr["NB_STREAMLINES"] == len(L) > 0
    assert np.array_equal(np.asarray(seq._lengths), L)
    assert np.array_equal(np.asarray(seq._data), _world(P))


def test_shard_matches_reference_split():
    from gpustreamlines_b200 import distributed as D

    # cu_propagate_seeds.py:45-54: ceil(n/ngpus) per GPU, the last one short
    assert [D.shard(10, r, 3) for r in range(3)] == [(0, 4), (4, 8), (8, 10)]
    assert [D.shard(2, r, 4) for r in range(4)] == [(0, 1), (1, 2), (2, 2), (2, 2)]
