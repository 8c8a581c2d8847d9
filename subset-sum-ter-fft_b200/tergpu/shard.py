"""One root split over the ranks of a process group (one GPU per rank).

The root's 4096 cells are independent: every pair (a, b) lands in exactly one
target family u = (key_a + key_b) mod 2^fb, and the reference groups its cells
the same way (the 64 target families of ``RootIndex``, reference
ter2_root/frozen/ter_root_queue_kernels.hpp:63-67).  Shard g of G (G a power of
two <= 64) is the set of pairs with key_a + key_b == g (mod G), i.e. the D
entries with key_d == g (mod G); the G shards are disjoint and their union is
the whole root.

Rank r of a world of W > 1 ranks takes the shards r, r + W, r + 2W, ... of
G = 64 (the finest split the cell grid allows: a rank's share is at most
ceil(64 / W) / (64 / W) of the mean, 1.10 for W <= 8, whatever W is), runs them
through the backend (each rank
reads all of A and B and the D families of its shards; there is no exchange
inside the join), and the only collective is one gather of the triples (a count
plus a few 12-byte records) and of the telemetry sums, so every rank ends with
the whole root's result.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from .root import Config, RootKeys, RootResult, Telemetry, run_gpu_root

MAX_SHARDS = 64


def shard_count_for(world: int) -> int:
    """Shards a world of `world` ranks splits one root into: 1 for a single
    rank, else all 64 (dealt round-robin, so non-power-of-two worlds stay
    balanced)."""
    if world < 1 or world > MAX_SHARDS:
        raise ValueError(f"world size {world} outside [1, {MAX_SHARDS}]")
    return 1 if world == 1 else MAX_SHARDS


def shards_of_rank(rank: int, world: int) -> list[int]:
    """The shard indices rank `rank` runs (every shard exactly once over the world)."""
    g = shard_count_for(world)
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    return list(range(rank, g, world))


def shard_cells(index: int, count: int) -> np.ndarray:
    """The 4096-byte cell mask (index s * 64 + t over the low 6 key bits of the
    A and B entries) that selects exactly the pairs of shard `index` of `count`."""
    if count < 1 or count > MAX_SHARDS or count & (count - 1) or not 0 <= index < count:
        raise ValueError("shard count must be a power of two <= 64 with the index below it")
    s = np.arange(64)[:, None]
    t = np.arange(64)[None, :]
    return (((s + t) % count) == index).astype(np.uint8).reshape(4096)


_TELEMETRY_SUMS = ("logical_pairs", "filter_survivors", "fast_hits", "full_hits",
                   "projected_hits", "kernel_launches")


def run_sharded_root(keys: RootKeys, config: Config | None = None, cells: np.ndarray | None = None,
                     group=None, runner=run_gpu_root) -> RootResult:
    """This rank's shards of one root, then one gather: every rank returns the
    whole root's triples (sorted) and summed telemetry; ``join_ms`` is the
    slowest rank's device time.

    `group` is a torch.distributed process group (None: the default group, or a
    world of one when torch.distributed is not initialised).  `runner` is the
    backend call (run_gpu_root); it receives a Config with shard_index and
    shard_count set."""
    config = config or Config()
    rank, world, dist = 0, 1, None
    try:
        import torch.distributed as _dist

        if _dist.is_available() and _dist.is_initialized():
            dist = _dist
            rank, world = dist.get_rank(group), dist.get_world_size(group)
    except ImportError:
        pass
    count = shard_count_for(world)
    parts: list[np.ndarray] = []
    tel = Telemetry()
    local_ms = 0.0
    for index in shards_of_rank(rank, world):
        cfg = dataclasses.replace(config, shard_index=index, shard_count=count)
        res = runner(keys, cfg, cells)
        parts.append(np.asarray(res.triples, dtype=np.uint32).reshape(-1, 3))
        for k in _TELEMETRY_SUMS:
            setattr(tel, k, getattr(tel, k) + getattr(res.telemetry, k))
        local_ms += res.telemetry.join_ms
        tel.family_bits = res.telemetry.family_bits
        tel.filter_bits = res.telemetry.filter_bits
    mine = np.concatenate(parts) if parts else np.zeros((0, 3), dtype=np.uint32)
    if dist is None or world == 1:
        tel.join_ms = local_ms
        return RootResult(status=0, triples=_sorted(mine), telemetry=tel)
    return _gather(dist, group, mine, tel, local_ms)


def _sorted(t: np.ndarray) -> np.ndarray:
    if len(t) == 0:
        return t.reshape(0, 3)
    order = np.lexsort((t[:, 2], t[:, 1], t[:, 0]))
    return t[order]


def _gather(dist, group, mine: np.ndarray, tel: Telemetry, local_ms: float) -> RootResult:
    import torch

    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    world = dist.get_world_size(group)
    sums = torch.tensor([getattr(tel, k) for k in _TELEMETRY_SUMS] + [len(mine)], dtype=torch.int64,
                        device=dev)
    dist.all_reduce(sums, group=group)
    slow = torch.tensor([local_ms], dtype=torch.float64, device=dev)
    dist.all_reduce(slow, op=dist.ReduceOp.MAX, group=group)
    counts = [torch.zeros(1, dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(counts, torch.tensor([len(mine)], dtype=torch.int64, device=dev), group=group)
    width = max(1, max(int(c.item()) for c in counts))
    pad = np.zeros((width, 3), dtype=np.int64)
    pad[: len(mine)] = mine
    bufs = [torch.zeros((width, 3), dtype=torch.int64, device=dev) for _ in range(world)]
    dist.all_gather(bufs, torch.from_numpy(pad).to(dev), group=group)
    merged = np.concatenate([b[: int(c.item())].cpu().numpy() for b, c in zip(bufs, counts)])
    out = Telemetry(family_bits=tel.family_bits, filter_bits=tel.filter_bits,
                    join_ms=float(slow.item()))
    for k, v in zip(_TELEMETRY_SUMS, sums.tolist()):
        setattr(out, k, int(v))
    if len(merged) != int(sums[-1].item()):
        raise RuntimeError("gathered triple count differs from the summed count")
    return RootResult(status=0, triples=_sorted(merged.astype(np.uint32).reshape(-1, 3)),
                      telemetry=out)
