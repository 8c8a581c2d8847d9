"""n=108 roots of the six published seeds against the reference.

For every seed the device attempt pipeline makes the authentic attempt-0 L1
lists of the benchmark instance and the device runs the records root (keys
derived on the device, join, authority) over the reference's declared 16-cell
sample; the reference's own capture and frozen ARWLF on the same sample
(golden seed_roots, printed by the reference harness) must agree on the level
sizes, the full-Q triple multiset (count and the three sink hashes), the
residue-exact and structural counts, the witnesses, the logical pairs and the
32-bit projected hits (about 1.6e8 per seed: the strong check, since the full-Q
outputs of a 16-cell sample are almost always empty).
"""
import pytest

from conftest import hexint

pytestmark = pytest.mark.gpu

CELLS = 16


@pytest.mark.parametrize("index", range(6))
def test_seed_root_sample_matches_reference_arwlf(oracle_mod, golden, index):
    import tergpu
    from tergpu import attempt, instance, workload

    g = golden["seed_roots"][index]
    seed = g["seed"]
    inst = instance.benchmark_instance(108, seed)
    res = attempt.solve_full_ter(inst, attempt.FullTerConfig(seed=seed, attempt_limit=1,
                                                             capture_only=True,
                                                             export_l1_capacity=7_500_000))
    assert res.attempts[0]["level1"] == g["level1"]
    assert res.attempts[0]["level2"] == g["level2"]
    root = tergpu.run_gpu_root_records(res.snapshot, tergpu.Config(projected_bits=32),
                                       cells=oracle_mod.select_cells(CELLS))
    ref = g["arwlf16"]
    got = workload.digest(root.triples)
    for k in ("triples", "triple_sum", "triple_xor", "triple_sum2"):
        assert got[k] == hexint(ref[k]), (hex(seed), k)
    assert root.telemetry.logical_pairs == ref["pairs"]
    assert root.telemetry.projected_hits == ref["projected_hits"] > 0
    assert root.residue_exact == ref["residue"]
    assert sorted(map(list, root.triples[root.flags & 1 == 1].tolist())) == ref["witnesses"]
