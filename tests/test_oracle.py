"""The oracle restatement pinned against the reference's own outputs (CPU only)."""
import numpy as np
import pytest

from conftest import hexint

ANCHOR_SEED = 19797034556212562


def test_params_known_answers(oracle_mod, golden):
    # n=36 from the reference run; n=72 / n=108 from the reference's published
    # snapshot records (r1 = 25 / 39, r2 = 7 / 12).
    final = golden["n36_attempts"][0]["final"]
    assert oracle_mod.params(36) == (final["r1"], final["r2"]) == (12, 3)
    assert oracle_mod.params(72) == (25, 7)
    assert oracle_mod.params(108) == (39, 12)
    for n in (48, 60, 84, 96, 0, 35):
        assert oracle_mod.params(n) is None


@pytest.mark.parametrize("case", range(6))
def test_n36_attempts_match_reference(oracle_mod, golden, case):
    g = golden["n36_attempts"][case]
    for row in g["attempts"]:
        got = oracle_mod.attempt(36, g["seed"], row["attempt"], kind=g["kind"])
        for key in ("level2", "level1", "level0", "l3_modular", "l2_modular", "root_prefilter",
                    "root_quotient_rejects", "root_modular", "valid_roots"):
            assert got[key] == row[key], (g["kind"], g["seed"], row["attempt"], key)
        assert got["status"] == (1 if row["status"] == 1 else 0)
        if got["status"] == 1:
            assert got["witness_verified"] == 1


@pytest.mark.parametrize("case", range(6))
def test_synthetic_roots_match_reference_brute_force(oracle_mod, golden, case):
    g = golden["synthetic_roots"][case]
    lo, hi = oracle_mod.synthetic_root(g["bits"], g["seed"], g["size"], g["pool"])
    assert [len(a) for a in lo] == g["sizes"]
    d, trip = oracle_mod.root_join(g["bits"], lo, hi, capacity=4096)
    for k in ("triples", "triple_sum", "triple_xor", "triple_sum2"):
        assert d[k] == hexint(g["brute"][k]), k
    # the same multiset from the explicit triple list
    assert oracle_mod.digest_of(trip)["triple_sum"] == d["triple_sum"]
    # ARWLF's projected hits (k = 19 + mid bits) by brute force
    assert oracle_mod.projected_count(g["arwlf"]["projected_bits"], lo) == g["arwlf"]["projected_hits"]
    # the reference's declared 700-cell subsample
    cells = oracle_mod.select_cells(700)
    assert int(cells.sum()) == 700
    ds, _ = oracle_mod.root_join(g["bits"], lo, hi, cells=cells)
    for k in ("triples", "triple_sum", "triple_xor", "triple_sum2"):
        assert ds[k] == hexint(g["subsample700"][k]), k


def test_planted_synthetic_triples_satisfy_equation(oracle_mod):
    lo, hi = oracle_mod.synthetic_root(69, 0x1234, 200, 0)
    _, trip = oracle_mod.root_join(69, lo, hi, capacity=1000)
    for a, b, c in trip:
        va = int(lo[0][a]) | (int(hi[0][a]) << 64)
        vb = int(lo[1][b]) | (int(hi[1][b]) << 64)
        vd = int(lo[2][c]) | (int(hi[2][c]) << 64)
        assert (va + vb - vd) % (1 << 69) == 0


def test_n72_anchor_level_sizes(n72_anchor_attempt, golden):
    g = golden["n72_roots"][0]
    got = n72_anchor_attempt
    assert got["level1"] == g["level1"] == [19109, 32496, 33505]
    assert got["level2"] == g["level2"]


def test_instance_generators(oracle_mod):
    values, target, planted = oracle_mod.build_instance(108, 0x1001, "auth")
    assert planted.sum() == 54 and planted[:27].all() and planted[54:81].all()
    v, t, p = oracle_mod.build_instance(36, 7, "build")
    assert p.sum() == 18
    acc = 0
    for i in range(36):
        if p[i]:
            acc += int(v[i][0])
    assert acc % (1 << 36) == int(t[0])


def test_config3_goldens_cover_32_seeds(golden):
    """Config 3's golden set, printed by the reference: 32 n=108 seeds (six
    published, 26 fresh), each with its capture's three L1 checksums and frozen
    ARWLF's 16-cell sample, and whole unplanted roots merged from cell slices
    that cover all 4,096 cells."""
    rows = golden["seed_roots"]
    assert len(rows) == 32 and len({g["seed"] for g in rows}) == 32
    assert sum(1 for g in rows if g["published"]) == 6
    for g in rows:
        assert len(g["checksums"]) == 3 and len(g["level1"]) == 3
        assert g["arwlf16"]["projected_hits"] > 0
    whole = [g for g in golden["whole_roots"] if "arwlf" in g]
    assert len(whole) >= 2
    for g in whole:
        assert g["arwlf"]["cells"] == 4096 and len(g["slice_rows"]) == g["slices"]
        assert g["arwlf"]["pairs"] == g["level1"][0] * g["level1"][1]


def test_wide_quotient_truncation_fixture(oracle_mod):
    """The reference's Q = 69 known answer (tests/full_ter_tests.cpp:805-838):
    the two A entries agree on the low 64 quotient bits, so a truncated window
    cannot separate them; the full 69-bit join keeps only the arithmetic root,
    whose residue sum equals the root target and whose parent has the root shape."""
    from conftest import wide_quotient_capture
    from tergpu import snapshot

    snap = wide_quotient_capture()
    Q, lo, hi, tau = snapshot.root_keys(snap)
    assert Q == 69 and tau == 0
    assert lo[0].tolist() == [0, 0] and hi[0].tolist() == [0, 1]
    assert oracle_mod.projected_count(32, lo) == 2
    digest, trip = oracle_mod.root_join(Q, lo, hi, capacity=16)
    assert digest["triples"] == 1 and trip.tolist() == [[0, 0, 0]]
    mod = 1 << snap.n
    target = snapshot.words_to_int(snap.root_target)
    for a, accepted in ((0, True), (1, False)):
        total = sum(snapshot.words_to_int(snap.residues(l)[i]) for l, i in ((0, a), (1, 0), (2, 0)))
        assert (total % mod == target) is accepted
    pos = [snap.masks(l)[0][0] for l in range(3)]
    parent = [int(pos[0][k]) | int(pos[1][k]) | int(pos[2][k]) for k in range(snap.words64)]
    assert sum(bin(w).count("1") for w in parent) == snap.n // 2


def test_witness_verification_fails_closed(golden):
    """verify_full_ter_witness's refusals as the reference's guided test checks
    them (tests/full_ter_tests.cpp:331-350), on the witness the reference found
    for its balanced n=36 instance (seed 0x544552F, the benchmark instance): a
    -1 digit, one selected item dropped, and the target's lowest bit flipped are
    each refused; the witness itself is the planted support."""
    import dataclasses

    from tergpu import instance

    g = golden["guided_replay"][0]
    inst = instance.benchmark_instance(g["n"], g["seed"])
    witness = [int(c) for c in g["final"]["witness"]]
    assert witness == inst.planted.tolist()
    assert instance.verify_witness(inst, witness)
    negative = list(witness)
    negative[0] = -1
    assert not instance.verify_witness(inst, negative)
    light = list(witness)
    light[light.index(1)] = 0
    assert not instance.verify_witness(inst, light)
    target = inst.target_le.copy()
    target[0] ^= 1
    assert not instance.verify_witness(dataclasses.replace(inst, target_le=target), witness)


def test_early_root_fixture_multiplicity(oracle_mod):
    """The reference's deterministic root-report fixture
    (tests/full_ter_tests.cpp:423-485): every one of the 4 x 4 x 4 triples is an
    exact root (all keys 0 at Q = 24), 64 pre-dedup roots with two distinct
    parents, each of them the root shape."""
    from conftest import early_root_capture
    from tergpu import snapshot

    snap = early_root_capture()
    Q, lo, hi, tau = snapshot.root_keys(snap)
    assert Q == 24 and tau == 0 and all(not v.any() for v in lo)
    digest, trip = oracle_mod.root_join(Q, lo, hi, capacity=128)
    assert digest["triples"] == 64 and len(trip) == 64
    pos = [snap.masks(l)[0][:, 0] for l in range(3)]
    parents = {int(pos[0][a]) | int(pos[1][b]) | int(pos[2][c]) for a, b, c in trip.tolist()}
    assert len(parents) == 2 and all(bin(p).count("1") == 18 for p in parents)


def test_guided_goldens_hold_the_reference_tests_assertions(golden):
    """The golden guided_replay rows, printed by the reference's solve_full_ter,
    satisfy what the reference's own tests assert of those solves
    (tests/full_ter_tests.cpp:249-330, 372-421, 578-595): the guided solves are
    Found with the planted root as witness; audited roots report
    FullCanonicalOutput without an early stop; FirstWitness stops early with one
    retained root; the random-target run exhausts its budget with an empty root."""
    from tergpu import instance

    rows = golden["guided_replay"]
    assert len(rows) == 8
    for g in rows:
        final, root = g["final"], g["rows"][0]["root"]
        if "guided" in g["modes"]:
            assert final["status"] == 1
            inst = instance.benchmark_instance(g["n"], g["seed"])
            assert [int(c) for c in final["witness"]] == inst.planted.tolist()
            assert g["rows"][0]["level0"] == 1
            if g["audit"]:
                assert root["policy"] == 2 and root["early_stopped"] == 0
            else:
                assert root["policy"] == 0 and root["early_stopped"] == 1 and root["valid_roots"] == 1
        else:
            assert final["status"] == 3 and g["rows"][0]["level0"] == 0 and root["early_stopped"] == 0
    n72 = [g for g in rows if g["n"] == 72]
    assert n72 and n72[0]["rows"][0]["root"]["quotient_bits"] == 47


def test_product_instances_equal_the_oracle_generator(oracle_mod):
    """tergpu.instance, which builds every device request, gives the same
    weights, target and planted support as the oracle's restatement of the
    reference's generators (build_instance, src/instance.cpp:61-120, and the
    benchmark instance with the planted support on the first n/4 coordinates
    of each half, bench/ter_full_bench.cpp:218-245)."""
    from tergpu import instance

    for n in (36, 72, 108):
        for seed in (1, 0x1001, ANCHOR_SEED, 0x544552F):
            for kind, make in (("auth", instance.benchmark_instance), ("build", instance.build_instance)):
                values, target, planted = oracle_mod.build_instance(n, seed, kind)
                inst = make(n, seed)
                assert np.array_equal(inst.values_le.reshape(values.shape), values), (n, seed, kind)
                assert np.array_equal(inst.target_le, target), (n, seed, kind)
                assert np.array_equal(inst.planted, planted), (n, seed, kind)


@pytest.mark.parametrize("case", range(6))
def test_product_digest_equals_reference_brute_force(oracle_mod, golden, case):
    """tergpu.workload.digest (the RootSink multiset hashes every GPU root test
    compares, ter2_root/frozen/ter_root_queue_kernels.cpp:165-175) over the
    oracle's triples of the six synthetic roots equals the reference's
    brute-force digest."""
    from tergpu import workload

    g = golden["synthetic_roots"][case]
    lo, hi = oracle_mod.synthetic_root(g["bits"], g["seed"], g["size"], g["pool"])
    _, trip = oracle_mod.root_join(g["bits"], lo, hi, capacity=1 << 16)
    got = workload.digest(trip)
    for k in ("triples", "triple_sum", "triple_xor", "triple_sum2"):
        assert got[k] == hexint(g["brute"][k]), k


def test_packed_add_matches_every_ternary_truth_table_row(oracle_mod):
    """The oracle's packed ternary add (add_packed_word, src/packed.cpp:15-38)
    on the reference's own truth-table test (tests/packed_tests.cpp:85-113):
    valid exactly when a + b + c stays in {-1, 0, 1}, and then its sign; and
    on seeded words of 64 independent digits against the scalar digit sums."""
    for a in (-1, 0, 1):
        for b in (-1, 0, 1):
            for c in (-1, 0, 1):
                ok, pos, neg = oracle_mod.add_packed_word(int(a == 1), int(a == -1), int(b == 1),
                                                          int(b == -1), int(c == 1), int(c == -1))
                total = a + b + c
                assert ok == (-1 <= total <= 1), (a, b, c)
                if ok:
                    assert (pos & 1, neg & 1) == (int(total == 1), int(total == -1)), (a, b, c)
    rng = np.random.default_rng(0x5041434B)
    for _ in range(200):
        digits = rng.integers(-1, 2, size=(3, 64))
        # keep the sums in range most of the time, so both outcomes occur
        if rng.random() < 0.7:
            digits[2] = np.clip(-(digits[0] + digits[1]) + rng.integers(-1, 2, size=64), -1, 1)
        masks = [(int(sum(1 << i for i in range(64) if d[i] == 1)),
                  int(sum(1 << i for i in range(64) if d[i] == -1))) for d in digits]
        ok, pos, neg = oracle_mod.add_packed_word(*masks[0], *masks[1], *masks[2])
        total = digits.sum(axis=0)
        assert ok == bool(np.all(np.abs(total) <= 1))
        if ok:
            assert pos == sum(1 << i for i in range(64) if total[i] == 1)
            assert neg == sum(1 << i for i in range(64) if total[i] == -1)


def test_boundary_roots_are_exact(oracle_mod):
    """The reporter's boundary cases at every device key width: the oracle's
    full-Q join finds exactly the triples exact integer arithmetic finds, and
    the reference's own expectations hold (the (0, 0, 1) singleton is the one
    miss; the duplicated keys give 3 x 2 x 4 = 24 triples)."""
    from conftest import boundary_roots

    wants = []
    for Q, lo, hi, want in boundary_roots():
        digest, _ = oracle_mod.root_join(Q, lo, [h.astype(np.uint64) for h in hi], capacity=64)
        assert digest["triples"] == want, (Q, [int(v[0]) for v in lo])
        wants.append(want)
    assert wants == [1, 0, 1, 1, 1, 1, 1, 1, 24] * 5
