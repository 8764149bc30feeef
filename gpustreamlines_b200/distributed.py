"""Multi-GPU seed sharding: one process per GPU, no data-path collective.

The reference splits each chunk's seeds into contiguous per-GPU blocks of
``ceil(n / ngpus)`` (``cu_propagate_seeds.py:45-54``) and gathers results
through host memory.  Here each rank (one process per GPU, torch.distributed)
tracks its contiguous shard; the only exchange is an all-gather of the
per-rank (streamline, point) counts, which gives every rank its offsets in
the global tractogram.  Each rank then writes its compacted slice directly
into a shared memory-mapped TRX layout at those offsets; rank 0 seals the file.
"""

from __future__ import annotations

import json
import os

import numpy as np


def shard(n: int, rank: int, world: int):
    """[start, stop) of this rank's contiguous seed block (reference split)."""
    per = (n + world - 1) // world
    start = min(n, rank * per)
    return start, min(n, start + per)


def gather_counts(n_streamlines: int, n_points: int, group=None, device=None):
    """All-gather per-rank counts -> (counts [world,2], streamline offset, point offset)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([n_streamlines, n_points], dtype=torch.int64, device=device)
    world = dist.get_world_size(group)
    out = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    counts = torch.stack(out).cpu().numpy()
    rank = dist.get_rank(group)
    sl_off = int(counts[:rank, 0].sum())
    pt_off = int(counts[:rank, 1].sum())
    return counts, sl_off, pt_off


def write_shard_trx(directory: str, rank: int, counts: np.ndarray, sl_off: int, pt_off: int,
                    lengths: np.ndarray, points_rasmm: np.ndarray, header: dict,
                    pos_dtype=np.float32):
    """Write this rank's slice into the shared TRX arrays under ``directory``.

    Every rank opens the same memmaps (created with the global sizes) and
    writes disjoint ranges, so no data crosses between GPUs.
    """
    nsl = int(counts[:, 0].sum())
    nv = int(counts[:, 1].sum())
    pos = np.memmap(os.path.join(directory, "positions.bin"), dtype=pos_dtype, mode="r+",
                    shape=(nv, 3))
    offs = np.memmap(os.path.join(directory, "offsets.bin"), dtype=np.uint64, mode="r+",
                     shape=(nsl + 1,))
    n = len(lengths)
    pos[pt_off:pt_off + len(points_rasmm)] = points_rasmm
    local = np.zeros(n, dtype=np.uint64)
    if n:
        np.cumsum(np.asarray(lengths[:-1], dtype=np.uint64), out=local[1:])
    offs[sl_off:sl_off + n] = local + np.uint64(pt_off)
    if rank == 0:
        offs[nsl] = nv
        hdr = dict(header)
        hdr["NB_STREAMLINES"], hdr["NB_VERTICES"] = nsl, nv
        with open(os.path.join(directory, "header.json"), "w") as f:
            json.dump(hdr, f)
    pos.flush()
    offs.flush()


def track_shard_to_trx(track, seeds: np.ndarray, rank: int, world: int, directory: str, affine,
                       dims, global_rng_index: bool = True, group=None):
    """One rank's whole share of a multi-GPU run into a shared TRX layout.

    ``track(seeds, rng_index_base) -> (lengths, seed_index, points_vox)`` runs
    this rank's tracker (``Handle.propagate`` + ``fetch`` on its GPU).  Seeds
    are split contiguously (the reference's split); with ``global_rng_index``
    seed s of the run uses the Philox streams of index s on every rank, so the
    merged tractogram equals a one-GPU run over all seeds; without it each rank
    restarts at index 0, which reproduces the reference's multi-GPU streams
    (its rng offset is ignored by its kernels).  The only exchange is the
    counts all-gather.  Rank 0 creates and seals ``directory/all.trx``.
    """
    import torch.distributed as dist

    start, stop = shard(len(seeds), rank, world)
    lengths, seed_idx, pts = track(seeds[start:stop], start if global_rng_index else 0)
    counts, sl_off, pt_off = gather_counts(len(lengths), len(pts), group=group)
    if rank == 0:
        create_shared_trx(directory, counts)
    dist.barrier(group)
    aff = np.asarray(affine, dtype=np.float64)
    world_pts = (np.asarray(pts, dtype=np.float64) @ aff[:3, :3].T + aff[:3, 3]).astype(np.float32)
    write_shard_trx(directory, rank, counts, sl_off, pt_off, lengths, world_pts,
                    {"DIMENSIONS": list(dims), "VOXEL_TO_RASMM": aff.tolist()})
    dist.barrier(group)
    if rank == 0:
        seal_trx(directory, os.path.join(directory, "all.trx"))
    dist.barrier(group)
    return counts


def create_shared_trx(directory: str, counts: np.ndarray, pos_dtype=np.float32):
    """Rank 0: allocate the shared arrays with the global sizes."""
    os.makedirs(directory, exist_ok=True)
    nsl = int(counts[:, 0].sum())
    nv = int(counts[:, 1].sum())
    np.memmap(os.path.join(directory, "positions.bin"), dtype=pos_dtype, mode="w+",
              shape=(max(nv, 1), 3)).flush()
    np.memmap(os.path.join(directory, "offsets.bin"), dtype=np.uint64, mode="w+",
              shape=(nsl + 1,)).flush()


def seal_trx(directory: str, filename: str, pos_dtype=np.float32):
    """Rank 0: pack the shared arrays into a TRX zip."""
    import zipfile

    with open(os.path.join(directory, "header.json")) as f:
        hdr = json.load(f)
    nv, nsl = hdr["NB_VERTICES"], hdr["NB_STREAMLINES"]
    pos = np.memmap(os.path.join(directory, "positions.bin"), dtype=pos_dtype, mode="r",
                    shape=(max(nv, 1), 3))[:nv]
    offs = np.memmap(os.path.join(directory, "offsets.bin"), dtype=np.uint64, mode="r",
                     shape=(nsl + 1,))
    with zipfile.ZipFile(filename, "w", compression=zipfile.ZIP_STORED) as z:
        z.writestr("header.json", json.dumps(hdr))
        z.writestr(f"positions.3.{np.dtype(pos_dtype).name}", np.ascontiguousarray(pos).tobytes())
        z.writestr("offsets.uint64", np.ascontiguousarray(offs).tobytes())
