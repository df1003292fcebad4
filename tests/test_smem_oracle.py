"""CPU checks of the SMEM-seeding oracle (the restatement of BWT.occ,
BackwardSearch.backwardExt and SMEMFinder.findAllSMEMs) and of the FM-index
builders the tests and the benchmark use for synthetic references.

The reference pins this path only with properties on its lambda-phage index
(Tests/FMIndexTests/FMIndexIntegrationTests.swift:131-234: intervals are
non-empty and shrink, SMEMs of a reference substring exist, lie inside the
query, are at least minSeedLen long and occur).  Here the same properties
are checked, and more strictly against brute force on small references:
every checkpoint count is the rank of its BWT prefix, every SMEM's interval
size is the number of occurrences of its substring in the indexed text
(forward strand + reverse complement), and no SMEM extends by one base on
either side without dropping below the occurrence threshold."""
import numpy as np
import pytest

from oracle import oracle

RC = np.array([3, 2, 1, 0], np.uint8)


def _text(ref):
    return np.concatenate([ref, RC[ref[::-1]]])


def _count(text_bytes, pat_bytes):
    n, k = 0, -1
    while True:
        k = text_bytes.find(pat_bytes, k + 1)
        if k < 0:
            return n
        n += 1


def _ref(seed, n, tandem=True):
    rng = np.random.default_rng(seed)
    ref = rng.integers(0, 4, n).astype(np.uint8)
    if tandem:
        unit = rng.integers(0, 4, 3).astype(np.uint8)
        ref[n // 3: n // 3 + 300] = np.resize(unit, 300)
        ref[2 * n // 3: 2 * n // 3 + 200] = ref[100:300]     # an exact repeat
    return ref


def test_checkpoints_are_prefix_ranks():
    ref = _ref(1, 3000)
    idx = oracle.bwt_build(ref)
    N = 2 * ref.size + 1
    assert idx.length == N and idx.count[4] == N and idx.count[0] == 1
    assert 0 <= idx.sentinel < N
    # counts: 1 + characters below c in the text (BWT.swift: each count +1 for '$')
    t = _text(ref)
    for c in range(4):
        assert idx.count[c + 1] - idx.count[c] == int(np.sum(t == c))
    # the BWT decoded from the bitstrings; checkpoint counts are its prefix ranks
    bwt = np.full(N, 4, np.uint8)
    for b in range(idx.cp.size):
        for y in range(64):
            i = 64 * b + y
            if i >= N:
                break
            for c in range(4):
                if (int(idx.cp["bits"][b, c]) >> (63 - y)) & 1:
                    bwt[i] = c
    assert np.sum(bwt == 4) == 1 and bwt[idx.sentinel] == 4
    for b in range(idx.cp.size):
        for c in range(4):
            assert idx.cp["counts"][b, c] == int(np.sum(bwt[: 64 * b] == c))


def _reads(ref, seed, n, L):
    rng = np.random.default_rng(seed)
    t = _text(ref)
    reads = []
    for _ in range(n):
        p = int(rng.integers(0, t.size - L))
        r = t[p:p + L].copy()
        m = rng.random(L)
        r[m < 0.03] = rng.integers(0, 4, int(np.sum(m < 0.03)))
        r[rng.random(L) < 0.01] = 4
        if rng.random() < 0.1:
            r = rng.integers(0, 4, L).astype(np.uint8)
        reads.append(r)
    return reads


@pytest.mark.parametrize("min_intv", [1, 3])
def test_smems_are_exact_maximal_matches(min_intv):
    ref = _ref(2, 4000)
    idx = oracle.bwt_build(ref)
    tb = _text(ref).tobytes()
    reads = _reads(ref, 3, 60, 80)
    bases = np.concatenate(reads)
    off = np.arange(len(reads), dtype=np.uint64) * 80
    ln = np.full(len(reads), 80, np.int32)
    out, n_out, over = oracle.smem_batch(idx, bases, off, ln, min_seed_len=12, min_intv=min_intv, cap=256)
    assert over == 0 and n_out.sum() > 0
    for r, q in enumerate(reads):
        sm = out[r * 256: r * 256 + n_out[r]]
        keys = list(zip(sm["qb"].tolist(), (-(sm["qe"] - sm["qb"])).tolist()))
        assert keys == sorted(keys)                                   # by begin, longer first
        for s in sm:
            qb, qe = int(s["qb"]), int(s["qe"])
            assert 0 <= qb < qe <= 80 and qe - qb >= 12
            sub = q[qb:qe]
            assert np.all(sub < 4)
            occ = _count(tb, sub.tobytes())
            assert occ == int(s["l"] - s["k"] + 1) >= min_intv
            if qb > 0 and q[qb - 1] < 4:
                assert _count(tb, q[qb - 1:qe].tobytes()) < min_intv
            if qe < 80 and q[qe] < 4:
                assert _count(tb, q[qb:qe + 1].tobytes()) < min_intv


def test_reference_substring_properties():
    """FMIndexIntegrationTests.swift:174-234 on a synthetic reference: a
    50-base reference substring yields SMEMs (minSeedLen 19) within the query,
    at least 19 long, with positive counts; a 30-base one (minSeedLen 15)
    covers part of the query."""
    ref = _ref(4, 20000, tandem=False)
    idx = oracle.bwt_build(ref)
    for start, L, msl in ((0, 50, 19), (1000, 30, 15)):
        q = ref[start:start + L].copy()
        out, n_out, _ = oracle.smem_batch(idx, q, np.array([0]), np.array([L]), min_seed_len=msl, cap=64)
        sm = out[: n_out[0]]
        assert n_out[0] > 0
        assert np.all(sm["qb"] >= 0) and np.all(sm["qe"] <= L) and np.all(sm["qe"] > sm["qb"])
        assert np.all(sm["qe"] - sm["qb"] >= msl) and np.all(sm["l"] - sm["k"] + 1 > 0)
        assert int(sm["qe"].max()) > 0
        assert (int(sm["qb"][0]), int(sm["qe"][0])) == (0, L)       # the whole substring matches


def test_overflowing_window_is_reported():
    ref = _ref(5, 3000)
    idx = oracle.bwt_build(ref)
    reads = _reads(ref, 6, 20, 100)
    bases = np.concatenate(reads)
    off = np.arange(20, dtype=np.uint64) * 100
    full, n_full, over0 = oracle.smem_batch(idx, bases, off, np.full(20, 100, np.int32), 10, cap=512)
    small, n_small, over = oracle.smem_batch(idx, bases, off, np.full(20, 100, np.int32), 10, cap=1)
    assert over0 == 0 and np.array_equal(n_full, n_small)
    assert over == int(np.sum(n_full > 1))


@pytest.mark.parametrize("n,tandem", [(1, 0.0), (5000, 0.2), (30000, 0.2)])
def test_workload_index_builder_matches_oracle_builder(n, tandem):
    """The benchmark's FM-index builder (prefix doubling on torch sorts, here
    on the CPU) gives the oracle builder's arrays exactly."""
    pytest.importorskip("torch")
    from swiftbwa_b200 import workloads as W
    ref = W.reference(W.SEED_BASE + 40 + n, n, tandem_frac=tandem).codes if n > 1 else np.array([1], np.uint8)
    a = oracle.bwt_build(ref)
    b = W.fm_index(ref, device="cpu")
    assert np.array_equal(a.cp, b.cp) and np.array_equal(a.count, b.count)
    assert (a.length, a.sentinel) == (b.length, b.sentinel)


def test_internal_reseed_adds_exact_more_specific_seeds():
    """BWAMemAligner.internalReseed (the arena form, BWAMemAligner.swift:259-305):
    the first pass's SMEMs are kept, and every added one is an exact match of
    at least minSeedLen found from the midpoint of a first-pass SMEM at least
    split_len long with at most split_width occurrences, with more occurrences
    than that SMEM; the list stays sorted by begin, longer first."""
    assert oracle.split_len_of(19, 1.5) == 28
    ref = _ref(7, 6000)
    ref[3000:3200] = ref[500:700]                    # extra copies make lower-count sub-seeds
    ref[4000:4100] = ref[520:620]
    idx = oracle.bwt_build(ref)
    tb = _text(ref).tobytes()
    reads = _reads(ref, 8, 80, 100)
    bases = np.concatenate(reads)
    off = np.arange(len(reads), dtype=np.uint64) * 100
    ln = np.full(len(reads), 100, np.int32)
    base, nb, _ = oracle.smem_batch(idx, bases, off, ln, 19, cap=512)
    rs, nr, over = oracle.smem_batch(idx, bases, off, ln, 19, cap=512, split_len=28, split_width=10)
    assert over == 0 and np.all(nr >= nb) and nr.sum() > nb.sum()
    for r, q in enumerate(reads):
        a = base[r * 512: r * 512 + nb[r]]
        b = rs[r * 512: r * 512 + nr[r]]
        keys = list(zip(b["qb"].tolist(), (-(b["qe"] - b["qb"])).tolist()))
        assert keys == sorted(keys)
        first = {tuple(x) for x in a.tolist()}
        assert first <= {tuple(x) for x in b.tolist()}
        parents = [s for s in a if s["qe"] - s["qb"] >= 28 and s["l"] - s["k"] + 1 <= 10]
        for s in b:
            if tuple(s.tolist()) in first:
                continue
            qb, qe = int(s["qb"]), int(s["qe"])
            occ = _count(tb, q[qb:qe].tobytes())
            assert qe - qb >= 19 and occ == int(s["l"] - s["k"] + 1)
            assert any(p["qb"] <= (int(p["qb"]) + int(p["qe"])) // 2 < p["qe"] and
                       (int(p["qb"]) + int(p["qe"])) // 2 in range(qb, qe) and occ > int(p["l"] - p["k"] + 1)
                       for p in parents)
