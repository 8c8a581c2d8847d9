"""GPU root parity: libtergpu.so through its C ABI against the oracle and the
reference's own outputs (golden fixtures, and the reference harness when it
was built)."""
import numpy as np
import pytest

from conftest import GOLDEN_DIR, hexint

pytestmark = pytest.mark.gpu

ANCHOR_SEED = 19797034556212562
DIGEST_KEYS = ("triples", "triple_sum", "triple_xor", "triple_sum2")


@pytest.fixture(scope="module")
def tg():
    import tergpu

    if tergpu.device_count() < 1:
        raise RuntimeError("the GPU tests need a CUDA device and libtergpu.so")
    return tergpu


def keys_of(oracle_mod, bits, seed, size, pool):
    import tergpu

    lo, hi = oracle_mod.synthetic_root(bits, seed, size, pool)
    return lo, hi, tergpu.RootKeys(quotient_bits=bits, lo=lo, hi=[h.astype(np.uint8) for h in hi])


def vcfg(variant):
    """Config keywords selecting sweep variant 1, 2, 3 (the default) or 4."""
    return {"sweep_v1": variant == 1, "sweep_v2": variant == 2, "sweep_v4": variant == 4}


def assert_digest(got, expected):
    for k in DIGEST_KEYS:
        assert got[k] == hexint(expected[k]), (k, got[k], expected[k])


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
@pytest.mark.parametrize("case", range(6))
def test_synthetic_roots_match_reference(tg, oracle_mod, golden, case, variant):
    from tergpu import workload

    g = golden["synthetic_roots"][case]
    lo, hi, keys = keys_of(oracle_mod, g["bits"], g["seed"], g["size"], g["pool"])
    res = tg.run_gpu_root(keys, tg.Config(projected_bits=g["arwlf"]["projected_bits"], **vcfg(variant)))
    assert_digest(workload.digest(res.triples), g["brute"])
    assert res.telemetry.logical_pairs == g["arwlf"]["logical_pairs"]
    assert res.telemetry.projected_hits == g["arwlf"]["projected_hits"]
    assert res.telemetry.full_hits == g["brute"]["triples"]
    # the reference's declared 700-cell subsample
    sub = tg.run_gpu_root(keys, tg.Config(**vcfg(variant)), cells=oracle_mod.select_cells(700))
    assert_digest(workload.digest(sub.triples), g["subsample700"])
    assert sub.telemetry.logical_pairs == g["subsample700"]["logical_pairs"]


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
@pytest.mark.parametrize("fb,filt", [(6, 10), (6, 19), (7, 12), (8, 15), (9, 20), (10, 11)])
def test_result_is_independent_of_tuning(tg, oracle_mod, golden, fb, filt, variant):
    from tergpu import workload

    g = golden["synthetic_roots"][0]
    _, _, keys = keys_of(oracle_mod, g["bits"], g["seed"], g["size"], g["pool"])
    res = tg.run_gpu_root(keys, tg.Config(family_bits=fb, filter_bits=filt, **vcfg(variant)))
    assert res.telemetry.family_bits == fb and res.telemetry.filter_bits == filt
    assert_digest(workload.digest(res.triples), g["brute"])


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
@pytest.mark.parametrize("bits", [24, 33, 40, 47, 58, 64, 65, 69, 72])
def test_widths_against_oracle(tg, oracle_mod, bits, variant):
    """Every key width from the n=36 root (24) to the one-byte high limit (72),
    with the carry, multiplicity and high-bit plants; projected counts at two k."""
    from tergpu import workload

    lo, hi, keys = keys_of(oracle_mod, bits, 0xABC0 + bits, 3000, 0)
    expected, _ = oracle_mod.root_join(bits, lo, hi)
    k = min(bits, 64) - 3
    res = tg.run_gpu_root(keys, tg.Config(projected_bits=k, **vcfg(variant)))
    got = workload.digest(res.triples)
    for key in DIGEST_KEYS:
        assert got[key] == expected[key], key
    assert res.telemetry.projected_hits == oracle_mod.projected_count(k, lo)


def test_dense_skewed_families_against_oracle(tg, oracle_mod):
    """pool=1: every key shares its low 19 bits, so one family holds everything."""
    from tergpu import workload

    lo, hi, keys = keys_of(oracle_mod, 69, 0x3131, 3000, 1)
    expected, _ = oracle_mod.root_join(69, lo, hi)
    res = tg.run_gpu_root(keys, tg.Config())
    assert workload.digest(res.triples)["triple_sum"] == expected["triple_sum"]
    assert res.telemetry.full_hits == expected["triples"]


def test_output_capacity_retry_and_count_only(tg, oracle_mod, golden):
    from tergpu import workload

    g = golden["synthetic_roots"][1]
    _, _, keys = keys_of(oracle_mod, g["bits"], g["seed"], g["size"], g["pool"])
    res = tg.run_gpu_root(keys, tg.Config(capacity=1))
    assert_digest(workload.digest(res.triples), g["brute"])
    cnt = tg.run_gpu_root(keys, tg.Config(count_only=True))
    assert cnt.telemetry.full_hits == g["brute"]["triples"] and len(cnt.triples) == 0


def test_resource_limit_and_invalid_width(tg, oracle_mod):
    _, _, keys = keys_of(oracle_mod, 69, 1, 500, 0)
    with pytest.raises(tg.TergpuError) as e:
        tg.run_gpu_root(keys, tg.Config(memory_limit_bytes=4096))
    assert e.value.status == 7  # ResourceLimit, refused before any allocation
    bad = tg.RootKeys(quotient_bits=100, lo=keys.lo, hi=keys.hi)
    with pytest.raises(tg.TergpuError) as e:
        tg.run_gpu_root(bad)
    assert e.value.status == 11  # UnsupportedWidth


def test_empty_and_ragged_lists(tg):
    from tergpu import workload

    Q = 47
    rng = np.random.default_rng(5)
    a = rng.integers(0, 1 << Q, 1000, dtype=np.uint64)
    b = rng.integers(0, 1 << Q, 7, dtype=np.uint64)
    d = np.array([(int(a[3]) + int(b[5])) % (1 << Q)], dtype=np.uint64)
    z = np.zeros
    keys = tg.RootKeys(Q, [a, b, d], [z(1000, np.uint8), z(7, np.uint8), z(1, np.uint8)])
    res = tg.run_gpu_root(keys)
    assert [tuple(t) for t in res.triples] == [(3, 5, 0)]
    empty = tg.RootKeys(Q, [a, b[:0], d], [z(1000, np.uint8), z(0, np.uint8), z(1, np.uint8)])
    assert len(tg.run_gpu_root(empty).triples) == 0


def test_n36_records_root_matches_reference(tg, oracle_mod, golden):
    """The reference's n=36 capture through the records entry: device key
    derivation, join and authority, against the reference's root stage and the
    oracle's projected counts on host-derived keys."""
    from tergpu import snapshot

    snap = snapshot.load(GOLDEN_DIR / golden["n36_snapshot"]["path"])
    Q, lo, hi, tau = snapshot.root_keys(snap)
    row = golden["n36_attempts"][0]["attempts"][0]
    for k in (12, 16, 20, 24):
        res = tg.run_gpu_root_records(snap, tg.Config(projected_bits=k))
        assert res.tau == tau
        assert res.telemetry.projected_hits == oracle_mod.projected_count(k, lo), k
        assert res.telemetry.full_hits == row["root_modular"]
        assert res.valid_roots == row["valid_roots"]


def _n72_snapshot(oracle_mod, tmp_path, seed, attempt):
    from tergpu import snapshot

    if not oracle_mod.ref_available():
        pytest.skip("reference harness not built on this host")
    path = tmp_path / f"n72_{seed:x}_{attempt}.snap"
    oracle_mod.ref_run("capture", 72, seed, attempt, "auth", path)
    return snapshot.load(path)


@pytest.mark.parametrize("case", range(3))
def test_n72_authentic_roots_match_frozen_backends(tg, oracle_mod, golden, tmp_path, case):
    from tergpu import workload

    g = golden["n72_roots"][case]
    snap = _n72_snapshot(oracle_mod, tmp_path, g["seed"], g["attempt"])
    assert snap.entries == g["level1"]
    res = tg.run_gpu_root_records(snap, tg.Config(projected_bits=32))
    assert_digest(workload.digest(res.triples), g["k2wide"])
    assert res.telemetry.logical_pairs == g["k2wide"]["pairs"]
    assert res.telemetry.projected_hits == g["arwlf_k32_projected_hits"] == g["k2"]["full_q"]
    assert res.residue_exact == g["k2wide"]["residue"]
    assert sorted(map(list, res.triples[res.flags & 1 == 1].tolist())) == g["k2wide"]["witnesses"]
    p25 = tg.run_gpu_root_records(snap, tg.Config(projected_bits=25, count_only=True))
    assert p25.telemetry.projected_hits == g["k2wide"]["projected_hits_25"]
    sub = tg.run_gpu_root_records(snap, tg.Config(), cells=oracle_mod.select_cells(512))
    assert_digest(workload.digest(sub.triples), g["k2wide_subsample512"])
    if g["attempt"] == 21:
        # the reference's positive attempt: one residue-exact triple, a valid root
        assert res.valid_roots == 1 and res.residue_exact == 1


def test_n72_adapter_through_reference_sink(tg, oracle_mod, golden, tmp_path):
    """run_gpu_root as a fifth backend of the reference harness, through the
    reference's own Dataset / FamilyKeys / RootSink (authority chain on)."""
    g = golden["n72_roots"][2]
    _n72_snapshot(oracle_mod, tmp_path, g["seed"], g["attempt"])
    path = tmp_path / f"n72_{g['seed']:x}_{g['attempt']}.snap"
    row = oracle_mod.ref_run("snaproot", path, "gpu", 4096, 32)[0]
    assert row["backend_status"] == "Completed"
    for k in ("triples", "triple_sum", "triple_xor", "triple_sum2", "residue", "residue_sum",
              "structural", "witnesses"):
        assert row[k] == g["k2wide"][k], k
    assert row["projected_hits"] == g["arwlf_k32_projected_hits"]


def test_large_planted_root_is_exact_and_deterministic(tg):
    """2e10 logical pairs at Q=69: every planted triple is reported, every
    reported triple satisfies the root equation exactly, two runs and two
    tunings agree."""
    from tergpu import workload

    keys = workload.synthetic_root(sizes=(100_000, 200_000, 200_000), quotient_bits=69,
                                   seed=0xBEEF, planted=64)
    r1 = tg.run_gpu_root(keys)
    r2 = tg.run_gpu_root(keys, tg.Config(family_bits=9, filter_bits=17, sweep_v1=True))
    r3 = tg.run_gpu_root(keys, tg.Config(family_bits=11, filter_bits=18, sweep_v2=True))
    t1 = sorted(map(tuple, r1.triples.tolist()))
    assert t1 == sorted(map(tuple, r2.triples.tolist())) == sorted(map(tuple, r3.triples.tolist()))
    n = [len(x) for x in keys.lo]
    planted = {(n[0] - 1 - i, n[1] - 1 - i, n[2] - 1 - i) for i in range(64)}
    assert planted <= set(t1)
    for a, b, c in t1:
        va = int(keys.lo[0][a]) | (int(keys.hi[0][a]) << 64)
        vb = int(keys.lo[1][b]) | (int(keys.hi[1][b]) << 64)
        vd = int(keys.lo[2][c]) | (int(keys.hi[2][c]) << 64)
        assert (va + vb - vd) % (1 << 69) == 0
    assert r1.telemetry.logical_pairs == n[0] * n[1]


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
@pytest.mark.parametrize("count", [2, 8, 64])
def test_shards_union_equals_whole_root(tg, oracle_mod, golden, count, variant):
    """The multi-GPU split run shard by shard on one device: disjoint shards
    whose union is the whole root (and, under the 700-cell subsample, the
    subsample), every triple in the shard its D key names."""
    from tergpu import workload

    g = golden["synthetic_roots"][0]
    lo, _, keys = keys_of(oracle_mod, g["bits"], g["seed"], g["size"], g["pool"])
    sub = oracle_mod.select_cells(700)
    trip, pairs, sub_trip = [], 0, []
    for i in range(count):
        res = tg.run_gpu_root(keys, tg.Config(shard_index=i, shard_count=count, **vcfg(variant)))
        assert all(int(lo[2][c]) % count == i for _, _, c in res.triples)
        trip.extend(map(tuple, res.triples.tolist()))
        pairs += res.telemetry.logical_pairs
        part = tg.run_gpu_root(keys, tg.Config(shard_index=i, shard_count=count, **vcfg(variant)),
                               cells=sub)
        sub_trip.extend(map(tuple, part.triples.tolist()))
    assert len(trip) == g["brute"]["triples"]
    assert_digest(workload.digest(trip), g["brute"])
    assert pairs == g["arwlf"]["logical_pairs"]
    assert_digest(workload.digest(sub_trip), g["subsample700"])


def test_sharded_root_in_one_process_and_bad_shard_counts(tg, oracle_mod, golden):
    from tergpu import workload
    from tergpu.shard import run_sharded_root

    g = golden["synthetic_roots"][2]
    _, _, keys = keys_of(oracle_mod, g["bits"], g["seed"], g["size"], g["pool"])
    res = run_sharded_root(keys)  # a world of one: the whole root
    assert_digest(workload.digest(res.triples), g["brute"])
    for index, count in ((0, 3), (2, 2), (0, 128)):
        with pytest.raises(tg.TergpuError) as e:
            tg.run_gpu_root(keys, tg.Config(shard_index=index, shard_count=count))
        assert e.value.status == 66  # InvalidInput


def test_autotune_is_exact_and_cached(tg, oracle_mod, golden):
    """The autotuner times candidate tunings on 1/64 of the target families and
    caches the pick per shape; the result is the reference's either way."""
    from tergpu import workload

    g = golden["synthetic_roots"][1]
    _, _, keys = keys_of(oracle_mod, g["bits"], g["seed"], g["size"], g["pool"])
    first = tg.run_gpu_root(keys, tg.Config(autotune=True))
    second = tg.run_gpu_root(keys, tg.Config(autotune=True))
    for res in (first, second):
        assert_digest(workload.digest(res.triples), g["brute"])
        assert res.telemetry.sweep_variant in (2, 3)
    assert first.telemetry.tune_ms > 0 and second.telemetry.tune_ms == 0
    assert (first.telemetry.family_bits, first.telemetry.filter_bits,
            first.telemetry.sweep_variant) == (second.telemetry.family_bits,
                                               second.telemetry.filter_bits,
                                               second.telemetry.sweep_variant)
    plain = tg.run_gpu_root(keys, tg.Config(sweep_v1=True))
    assert plain.telemetry.sweep_variant == 1 and plain.telemetry.tune_ms == 0


def test_v4_large_a_families_and_ragged_rows(tg):
    """Variant 4 with A families of several staged segments (about 940 entries
    at 6 family bits) and B families of every row count: the same triples as
    variant 2 on the same keys."""
    from tergpu import workload

    keys = workload.synthetic_root(sizes=(60_000, 9_000, 9_000), quotient_bits=69, seed=0xA4,
                                   planted=24)
    want = tg.run_gpu_root(keys, tg.Config(sweep_v2=True, family_bits=6))
    for fb in (6, 7, 9):
        got = tg.run_gpu_root(keys, tg.Config(family_bits=fb, sweep_v4=True))
        assert got.telemetry.sweep_variant == 4
        assert workload.digest(got.triples) == workload.digest(want.triples)
        assert got.telemetry.logical_pairs == want.telemetry.logical_pairs


def test_v4_dense_target_family(tg):
    """Every A + B sum on one 14-bit window that a dense D family holds: every
    probe passes the table, so a warp's survivors overflow its buffer and
    resolve in place; one class of B entries (no balanced layout: the family
    keeps its order) and A families of many staged segments.  The result
    equals variant 2's, including planted exact sums."""
    import numpy as np

    import tergpu
    from tergpu import workload

    rng = np.random.default_rng(5)
    Q, fb = 69, 6
    low_b = (0x1357 << fb) | 5
    mask = (1 << Q) - 1

    def keys(n, low):
        return [(int(v) << 20 | low) & mask for v in rng.integers(0, 1 << 49, n, dtype=np.uint64)]

    a, b = keys(3_000, 0), keys(3_000, low_b)
    d = keys(500, low_b) + keys(1_000, int(rng.integers(0, 1 << 20)))
    d += [(a[int(i)] + b[int(j)]) & mask for i, j in rng.integers(0, 3_000, (10, 2))]
    lists = [a, b, d]
    k = tergpu.RootKeys(quotient_bits=Q,
                        lo=[np.array([v & ((1 << 64) - 1) for v in l], dtype=np.uint64) for l in lists],
                        hi=[np.array([v >> 64 for v in l], dtype=np.uint8) for l in lists])
    want = tg.run_gpu_root(k, tg.Config(sweep_v2=True, family_bits=fb))
    got = tg.run_gpu_root(k, tg.Config(family_bits=fb, sweep_v4=True))
    assert got.telemetry.sweep_variant == 4
    assert got.telemetry.filter_survivors >= 3_000 * 3_000
    assert len(want.triples) >= 10
    assert workload.digest(got.triples) == workload.digest(want.triples)


@pytest.mark.parametrize("fb", [6, 7, 8, 9, 10, 12, 14])
def test_staged_partition_equals_one_pass(tg, fb):
    """Lists of 2^20 or more entries go to their families through the staged
    two-pass scatter (one staged pass at 7 family bits or fewer); on the same
    keys every count and the triple multiset equal the one-pass scatter's.  A
    (1.1 M entries) is always staged; D holds about 1,500 entries per family
    (the sweep's exact lookup takes 2,048), so it is staged from 10 family bits
    on; B stays short."""
    from tergpu import workload

    n_d = min(1_200_000, 1500 << fb)
    keys = workload.synthetic_root(sizes=(1_100_000, 40_000, n_d), quotient_bits=69,
                                   seed=0x5EED + fb, planted=40)
    cfg = dict(family_bits=fb, projected_bits=fb + 20)
    staged = tg.run_gpu_root(keys, tg.Config(**cfg))
    plain = tg.run_gpu_root(keys, tg.Config(one_pass_partition=True, **cfg))
    assert len(staged.triples) >= 40
    assert workload.digest(staged.triples) == workload.digest(plain.triples)
    for k in ("logical_pairs", "filter_survivors", "fast_hits", "full_hits", "projected_hits"):
        assert getattr(staged.telemetry, k) == getattr(plain.telemetry, k), k
    if fb >= 8:  # two passes instead of one per staged list (the scan fills the bucket table)
        extra = sum(1 for n in (1_100_000, 40_000, n_d) if n >= 1 << 20)
        assert staged.telemetry.kernel_launches == plain.telemetry.kernel_launches + extra


def test_staged_partition_with_empty_buckets_and_no_high_byte(tg):
    """Q = 47 (no high byte) and an A list whose families take three values,
    so most buckets and families are empty and one tile spans few digits."""
    import numpy as np

    import tergpu
    from tergpu import workload

    rng = np.random.default_rng(3)
    for fb in (7, 12):
        keys = workload.synthetic_root(sizes=(1_300_000, 30_000, 1200 << fb if fb < 10 else 1_100_000),
                                       quotient_bits=47, seed=0xE3 + fb, planted=16)
        low = np.array([0, 5, 4077], dtype=np.uint64)[rng.integers(0, 3, len(keys.lo[0]))]
        lo_a = (keys.lo[0] & ~np.uint64(0xFFF)) | low
        skew = tergpu.RootKeys(quotient_bits=47, lo=[lo_a, keys.lo[1], keys.lo[2]], hi=keys.hi)
        cfg = dict(family_bits=fb, projected_bits=fb + 18)
        staged = tg.run_gpu_root(skew, tg.Config(**cfg))
        plain = tg.run_gpu_root(skew, tg.Config(one_pass_partition=True, **cfg))
        assert staged.telemetry.projected_hits > 0
        assert workload.digest(staged.triples) == workload.digest(plain.triples)
        for k in ("logical_pairs", "filter_survivors", "projected_hits"):
            assert getattr(staged.telemetry, k) == getattr(plain.telemetry, k), (fb, k)
