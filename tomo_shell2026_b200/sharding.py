"""Orientation sharding across ranks (one process per GPU).

Orientations are independent, so a sweep partitions into contiguous shards
of the YPR array with no exchange on the data path.  The one cross-rank
step is the final argmin, which must reproduce _find1stOptimal
(Tomo_Shell_vc_src/Tomo_Shell2026.cpp:89-97): the first index whose Mss is
strictly below the running minimum, the running minimum starting at 1e5
(result 0 when nothing is below 1e5, or when there is at most one
orientation).  Each rank reduces its shard to (first minimal Mss, global
index); ranks combine with one MIN all-reduce on a 64-bit key that orders by
Mss first and global index second.  ``sweep_shard`` runs one rank's part
of a single mesh's sweep and returns the global optimum.
"""
from __future__ import annotations

from dataclasses import dataclass

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


@dataclass
class ShardSweep:
    """One rank's part of a sharded sweep.

    ``optID`` is the global first optimum (the same index one undivided
    sweep returns); ``begin``/``end`` bound this rank's orientations;
    ``shard`` is the engine's result for them.  With ``gather`` the
    per-orientation arrays of the whole grid (``Mss``, ``Mo``, ``Vo64``,
    ``Vss64``) are filled on every rank, else they are None.
    """

    optID: int
    begin: int
    end: int
    shard: object
    Mss: np.ndarray | None = None
    Mo: np.ndarray | None = None
    Vo64: np.ndarray | None = None
    Vss64: np.ndarray | None = None


def _field(res, name):
    return res[name] if isinstance(res, dict) else getattr(res, name)


def _all_gather(local: np.ndarray, n: int, rank: int, world: int, group) -> np.ndarray:
    """Concatenate every rank's contiguous shard of a 1-D array (shards may
    differ in length by one, so each is padded to the longest first)."""
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend(group) == "nccl" else "cpu"
    longest = max(e - b for b, e in (shard_range(n, r, world) for r in range(world)))
    bits = np.ascontiguousarray(local).view(np.int32 if local.dtype.itemsize == 4 else np.int64)
    buf = torch.zeros(max(longest, 1), dtype=torch.int32 if bits.dtype == np.int32 else torch.int64, device=dev)
    if bits.size:
        buf[: bits.size] = torch.from_numpy(bits).to(dev)
    outs = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(outs, buf, group=group)
    parts = []
    for r in range(world):
        b, e = shard_range(n, r, world)
        parts.append(outs[r][: e - b].cpu().numpy())
    return np.concatenate(parts).view(local.dtype)


def sweep_shard(mesh, ypr, opts, rank: int | None = None, world: int | None = None, group=None,
                engine=None, gather: bool = False) -> ShardSweep:
    """Sweep this rank's contiguous shard of one mesh's orientation grid.

    Each rank evaluates ``ypr[begin:end]`` (``shard_range``) with ``engine``
    -- by default the CUDA library's ``TomoSh_CUDA`` (``native.sweep``) on
    the rank's current device -- and the ranks combine their first minima
    with one MIN all-reduce (``global_first_optimal``), so every rank
    returns the optID of the undivided sweep (_find1stOptimal,
    Tomo_Shell_vc_src/Tomo_Shell2026.cpp:89-97).  Orientations are
    independent, so nothing else crosses ranks unless ``gather`` asks for
    the whole grid's per-orientation arrays.

    ``engine(mesh, ypr_shard, opts)`` returns an object or dict with at
    least ``Mss`` (and ``Mo``, ``Vo64``, ``Vss64`` when gathering).
    Without an initialised process group the call is the undivided sweep.
    """
    import torch.distributed as dist
    live = dist.is_available() and dist.is_initialized()
    if rank is None:
        rank = dist.get_rank(group) if live else 0
    if world is None:
        world = dist.get_world_size(group) if live else 1
    if world > 1 and not live:
        raise RuntimeError("a sharded sweep over several ranks needs an initialised process group")
    if engine is None:
        from . import native
        engine = native.sweep
    n = int(ypr.shape[0])
    b, e = shard_range(n, rank, world)
    res = engine(mesh, np.ascontiguousarray(ypr[b:e], np.float32), opts) if e > b else None
    empty = {"Mss": np.zeros(0, np.float32), "Mo": np.zeros(0, np.float32), "Vo64": np.zeros(0, np.int64),
             "Vss64": np.zeros(0, np.int64)}
    src = res if res is not None else empty
    mss = np.asarray(_field(src, "Mss"), np.float32)
    if world == 1:
        opt = first_optimal(mss)
    else:
        opt = global_first_optimal(mss, b, n, group)
    out = ShardSweep(opt, b, e, res)
    if gather:
        if world == 1:
            out.Mss, out.Mo = mss.copy(), np.asarray(_field(src, "Mo"), np.float32).copy()
            out.Vo64 = np.asarray(_field(src, "Vo64"), np.int64).copy()
            out.Vss64 = np.asarray(_field(src, "Vss64"), np.int64).copy()
        else:
            out.Mss = _all_gather(mss, n, rank, world, group)
            out.Mo = _all_gather(np.asarray(_field(src, "Mo"), np.float32), n, rank, world, group)
            out.Vo64 = _all_gather(np.asarray(_field(src, "Vo64"), np.int64), n, rank, world, group)
            out.Vss64 = _all_gather(np.asarray(_field(src, "Vss64"), np.int64), n, rank, world, group)
    return out
