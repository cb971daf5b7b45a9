"""Multi-GPU sharding of the imaging path (one process per GPU).

The reference runs one consumer thread per GPU, each imaging whatever traces
it pops into a private image, and sums the per-GPU images on the host after
every offset group (src/q-psdm.cu:1711-1757).  Here each rank (one process,
one GPU, one engine) images its own whole shot gathers -- shots are kept whole
so that the batched form can share source terms and receiver positions
within a rank -- and the images are summed once per offset group with one
collective (NCCL over NVLink on GPUs, gloo on CPU).  Imaging itself needs no
communication, so scaling is weak: per-rank work stays fixed as ranks grow.
"""
from __future__ import annotations

import numpy as np

SU_SX, SU_SY = 72, 76


def source_runs(records: np.ndarray, big_endian: bool = True) -> np.ndarray:
    """Shot index of every SU record: consecutive records with the same
    source position form one shot (first-occurrence numbering)."""
    e = ">i4" if big_endian else "<i4"
    sx = records[:, SU_SX:SU_SX + 4].copy().view(e).ravel()
    sy = records[:, SU_SY:SU_SY + 4].copy().view(e).ravel()
    if sx.size == 0:
        return np.zeros(0, np.int64)
    new = np.ones(sx.size, bool)
    new[1:] = (sx[1:] != sx[:-1]) | (sy[1:] != sy[:-1])
    return np.cumsum(new) - 1


def shard_records(records: np.ndarray, rank: int, world: int, big_endian: bool = True):
    """Records of the shots this rank images (shot k goes to rank k % world),
    in their original order, and the indices they came from."""
    if world <= 1:
        return records, np.arange(records.shape[0])
    shot = source_runs(records, big_endian)
    idx = np.nonzero(shot % world == rank)[0]
    return records[idx], idx


def reduce_image(img, dist, dst: int = 0, all_ranks: bool = False):
    """Sum the per-rank images (a torch tensor, in place) with one collective:
    a reduce to `dst` (the rank that writes the output, as the reference's
    host sum) or an all-reduce when every rank needs the image."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return img
    if all_ranks:
        dist.all_reduce(img, op=dist.ReduceOp.SUM)
    else:
        dist.reduce(img, dst=dst, op=dist.ReduceOp.SUM)
    return img
