"""The multi-GPU split of one root (tergpu.shard) on the CPU: the shard masks
partition the reference's cell grid, the shards' union is the whole root, and
the gather over a gloo process group (world sizes 2 and 3) returns the whole
root to every rank.  The per-shard join here is the oracle (the GPU backend
runs the same shards in test_gpu_root.py)."""
import os
import socket

import numpy as np
import pytest

from conftest import hexint

DIGEST_KEYS = ("triples", "triple_sum", "triple_xor", "triple_sum2")


def _oracle_runner(keys, cfg, cells):
    import oracle

    from tergpu import RootResult, Telemetry
    from tergpu.shard import shard_cells

    mask = shard_cells(cfg.shard_index, cfg.shard_count)
    if cells is not None:
        mask = mask & np.asarray(cells, dtype=np.uint8)
    d, trip = oracle.root_join(keys.quotient_bits, keys.lo, keys.hi, cells=mask, capacity=1 << 14)
    sizes = [len(a) for a in keys.lo]
    s6 = np.bincount(np.asarray(keys.lo[0], dtype=np.uint64) & np.uint64(63), minlength=64)
    t6 = np.bincount(np.asarray(keys.lo[1], dtype=np.uint64) & np.uint64(63), minlength=64)
    pairs = int((np.outer(s6, t6).reshape(4096) * mask).sum())
    assert sizes[0] == s6.sum()
    return RootResult(status=0, triples=trip,
                      telemetry=Telemetry(full_hits=d["triples"], logical_pairs=pairs, join_ms=1.0))


def _keys(oracle_mod, golden, case=0):
    from tergpu import RootKeys

    g = golden["synthetic_roots"][case]
    lo, hi = oracle_mod.synthetic_root(g["bits"], g["seed"], g["size"], g["pool"])
    return g, RootKeys(g["bits"], lo, [h.astype(np.uint8) for h in hi])


@pytest.mark.parametrize("count", [1, 2, 4, 8, 64])
def test_shard_masks_partition_the_cell_grid(count):
    from tergpu.shard import shard_cells

    total = sum(shard_cells(i, count).astype(int) for i in range(count))
    assert np.array_equal(total, np.ones(4096, dtype=int))


def test_shard_assignment_covers_each_shard_once():
    from tergpu.shard import shard_count_for, shards_of_rank

    for world in (1, 2, 3, 4, 5, 7, 8, 13, 64):
        g = shard_count_for(world)
        assert g >= world and g & (g - 1) == 0
        got = sorted(i for r in range(world) for i in shards_of_rank(r, world))
        assert got == list(range(g))
        # balance: no rank holds more than ceil(64 / W) shards of 64
        if world > 1:
            most = max(len(shards_of_rank(r, world)) for r in range(world))
            assert g == 64 and most == -(-64 // world)
    with pytest.raises(ValueError):
        shard_count_for(65)
    with pytest.raises(ValueError):
        from tergpu.shard import shard_cells
        shard_cells(3, 6)


def test_shards_union_is_the_whole_root(oracle_mod, golden):
    from tergpu import workload
    from tergpu.shard import run_sharded_root

    g, keys = _keys(oracle_mod, golden, 1)
    res = run_sharded_root(keys, runner=_oracle_runner)
    got = workload.digest(res.triples)
    for k in DIGEST_KEYS:
        assert got[k] == hexint(g["brute"][k]), k
    assert res.telemetry.logical_pairs == g["arwlf"]["logical_pairs"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, case, out_dir):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    import conftest  # noqa: F401  (puts the package and the oracle on sys.path)
    import json

    import torch.distributed as dist

    import oracle
    from tergpu import workload
    from tergpu.shard import run_sharded_root

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        golden = json.loads(open(os.path.join(here, "golden", "reference_golden.json")).read())
        g = golden["synthetic_roots"][case]
        lo, hi = oracle.synthetic_root(g["bits"], g["seed"], g["size"], g["pool"])
        from tergpu import RootKeys

        keys = RootKeys(g["bits"], lo, [h.astype(np.uint8) for h in hi])
        res = run_sharded_root(keys, runner=_oracle_runner)
        d = workload.digest(res.triples)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"digest": {k: int(d[k]) for k in DIGEST_KEYS},
                       "pairs": res.telemetry.logical_pairs,
                       "full": res.telemetry.full_hits,
                       "n": int(len(res.triples))}, f)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_gather_the_whole_root(golden, tmp_path, world):
    import json

    import torch.multiprocessing as mp

    case = 3
    mp.start_processes(_rank_main, args=(world, _free_port(), case, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    g = golden["synthetic_roots"][case]
    for r in range(world):
        row = json.loads((tmp_path / f"rank{r}.json").read_text())
        for k in DIGEST_KEYS:
            assert row["digest"][k] == hexint(g["brute"][k]), (r, k)
        assert row["full"] == row["n"] == g["brute"]["triples"]
        assert row["pairs"] == g["arwlf"]["logical_pairs"]
