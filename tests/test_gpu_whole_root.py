"""Whole authentic roots with the reference's planted final output.

The reference's whole-root runner plants one positive output on the anchor
microproblem (seed 0xB1A57001) and every exact backend must report exactly
that output over the whole root (the published n=108 0x1001 run reports
[1753507, 754371, 6896564] on cell 2730).  Here the device attempt pipeline
produces the L1 lists, the planted D key from the reference (golden
whole_root_plants) is appended, and the device root must return exactly the
planted triple: nothing missed, nothing extra, over all 2.5e13 pairs at n=108.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _planted_keys(g):
    import tergpu
    from tergpu import attempt, instance, snapshot

    inst = instance.benchmark_instance(g["n"], g["seed"])
    cfg = attempt.FullTerConfig(seed=g["seed"], attempt_first=g["attempt"], attempt_limit=1,
                                capture_only=True, export_l1_capacity=7_500_000)
    snap = attempt.solve_full_ter(inst, cfg).snapshot
    q, lo, hi, _ = snapshot.root_keys(snap)
    assert len(lo[2]) == g["first_planted"]
    lo[2] = np.concatenate([lo[2], np.array(g["d_lo"], dtype=np.uint64)])
    hi[2] = np.concatenate([hi[2], np.array(g["d_hi"], dtype=np.uint8)])
    return tergpu.RootKeys(quotient_bits=q, lo=lo, hi=hi)


@pytest.mark.parametrize("index", [0, 1])
def test_whole_root_reports_exactly_the_planted_output(golden, index):
    import tergpu

    g = golden["whole_root_plants"][index]
    keys = _planted_keys(g)
    res = tergpu.run_gpu_root(keys)
    assert sorted(map(list, res.triples.tolist())) == g["expected"]
    assert res.telemetry.logical_pairs == len(keys.lo[0]) * len(keys.lo[1])


def test_sharded_whole_root_reports_the_planted_output(golden):
    import tergpu
    from tergpu.shard import shard_count_for

    g = golden["whole_root_plants"][0]
    keys = _planted_keys(g)
    count = shard_count_for(4)
    got = []
    for i in range(count):
        res = tergpu.run_gpu_root(keys, tergpu.Config(shard_index=i, shard_count=count))
        got.extend(map(list, res.triples.tolist()))
    assert sorted(got) == g["expected"]
