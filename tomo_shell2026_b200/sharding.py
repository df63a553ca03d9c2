"""Orientation sharding across ranks (one process per GPU).

Orientations are independent, so a sweep partitions into contiguous shards
of the YPR array with no exchange on the data path.  The one cross-rank
step is the final argmin, which must reproduce _find1stOptimal
(Tomo_Shell_vc_src/Tomo_Shell2026.cpp:89-97): the first index whose Mss is
strictly below the running minimum, the running minimum starting at 1e5
(result 0 when nothing is below 1e5, or when there is at most one
orientation).  Each rank reduces its shard to (first minimal Mss, global
index); ranks combine with one MIN all-reduce on a 64-bit key that orders by
Mss first and global index second.
"""
from __future__ import annotations

import numpy as np

NO_CANDIDATE = np.iinfo(np.int64).max


def shard_range(n: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [begin, end) of orientation indices owned by `rank`."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    per, rem = divmod(n, world)
    begin = rank * per + min(rank, rem)
    return begin, begin + per + (1 if rank < rem else 0)


def _order_key(value: np.float32) -> int:
    """Monotone map float32 -> uint32 (negative floats below positive ones)."""
    b = int(np.float32(value).view(np.uint32))
    return (b ^ 0xFFFFFFFF) if (b & 0x80000000) else (b | 0x80000000)


def local_candidate(mss_shard: np.ndarray, begin: int) -> int:
    """Packed (Mss, global index) key of the shard's first strict minimum
    below 1e5, or NO_CANDIDATE."""
    best = np.float32(1e5)
    idx = -1
    for i, v in enumerate(np.asarray(mss_shard, np.float32)):
        if v < best:
            best, idx = v, i
    if idx < 0:
        return NO_CANDIDATE
    return (_order_key(best) << 31) | (begin + idx)


def first_optimal(mss: np.ndarray) -> int:
    """_find1stOptimal on one array (Tomo_Shell2026.cpp:89-97)."""
    if len(mss) <= 1:
        return 0
    key = local_candidate(mss, 0)
    return 0 if key == NO_CANDIDATE else int(key & ((1 << 31) - 1))


def global_first_optimal(mss_shard: np.ndarray, begin: int, n_total: int, group=None) -> int:
    """Combine shard candidates across the process group (torch.distributed)."""
    if n_total <= 1:
        return 0
    import torch
    import torch.distributed as dist
    key = local_candidate(mss_shard, begin)
    backend = dist.get_backend(group) if dist.is_initialized() else "gloo"
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([key], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    k = int(t.item())
    return 0 if k == NO_CANDIDATE else int(k & ((1 << 31) - 1))
