"""Host-side checks of the synthetic workloads (no GPU): the seed chains'
seeds are exact matches at their BWT coordinates through the oracle's
FMIndex.getReference, and the oracle's ExtensionAligner.extend turns each
chain into regions that contain their first seed."""
import numpy as np

from swiftbwa_b200 import workloads as W
from swiftbwa_b200.abi import Scoring


def test_chain_seeds_are_exact_matches(oracle_mod):
    ref = W.reference(W.SEED_BASE + 60, 100_000)
    wl = W.chains(ref, 11, 400, 150, spurious_frac=0.0)
    assert len(wl.seeds) >= len(wl.chains)          # most reads have a seed
    rev = 0
    for c in wl.chains:
        read = wl.bases[int(c["read_off"]):int(c["read_off"]) + int(c["read_len"])]
        for s in wl.seeds[int(c["seed_off"]):int(c["seed_off"]) + int(c["n_seeds"])]:
            got = oracle_mod.get_reference(ref.pac, ref.n, int(s["rbeg"]), int(s["len"]))
            q = read[int(s["qbeg"]):int(s["qbeg"]) + int(s["len"])]
            assert np.array_equal(got, q)
            assert int(s["len"]) >= 19 and int(s["score"]) == int(s["len"])
            rev += int(s["rbeg"]) >= ref.n
    assert rev > 0                                   # both strands present


def test_chain_generation_is_deterministic():
    ref = W.reference(W.SEED_BASE + 61, 50_000)
    a = W.chains(ref, 5, 300, 100)
    b = W.chains(ref, 5, 300, 100)
    assert np.array_equal(a.bases, b.bases) and np.array_equal(a.seeds, b.seeds)
    assert np.array_equal(a.chains, b.chains)


def test_oracle_extend_regions_contain_first_seed(oracle_mod):
    ref = W.reference(W.SEED_BASE + 62, 100_000)
    wl = W.chains(ref, 12, 100, 150)
    sc = Scoring.default()
    for c in wl.chains:
        so, ns = int(c["seed_off"]), int(c["n_seeds"])
        if ns == 0:
            continue
        seeds = [(int(s["rbeg"]), int(s["qbeg"]), int(s["len"]), int(s["score"])) for s in wl.seeds[so:so + ns]]
        read = wl.bases[int(c["read_off"]):int(c["read_off"]) + int(c["read_len"])]
        regs, calls, _ = oracle_mod.extend(seeds, 0, read, ref.pac, sc, ref_mode=1, genome_len=ref.n)
        best = max(range(ns), key=lambda k: (seeds[k][3], -k))
        r0 = regs[0]
        rb, qb, ln, _ = seeds[best]
        assert r0["qb"] <= qb and qb + ln <= r0["qe"] and r0["rb"] <= rb and rb + ln <= r0["re"]
        assert r0["seed_len0"] == ln and calls >= 1 or (qb == 0 and qb + ln == len(read))


def test_oracle_extend_batch_equals_per_chain(oracle_mod):
    from swiftbwa_b200.abi import REGION_DTYPE
    ref = W.reference(W.SEED_BASE + 63, 80_000, tandem_frac=0.05)
    wl = W.chains(ref, 13, 300, 150, sub=0.03, indel=0.01, spurious_frac=0.3)
    sc = Scoring.default()
    regs, counts, cells = oracle_mod.extend_batch(sc, wl.bases, ref.pac, ref.n, wl.seeds, wl.chains, n_threads=4)
    assert cells > 0
    for k, c in enumerate(wl.chains):
        so, ns = int(c["seed_off"]), int(c["n_seeds"])
        seeds = [(int(s["rbeg"]), int(s["qbeg"]), int(s["len"]), int(s["score"])) for s in wl.seeds[so:so + ns]]
        read = wl.bases[int(c["read_off"]):int(c["read_off"]) + int(c["read_len"])]
        exp, _, _ = oracle_mod.extend(seeds, int(c["rid"]), read, ref.pac, sc, ref_mode=1, genome_len=ref.n)
        assert int(counts[k]) == len(exp)
        for j, e in enumerate(exp):
            assert tuple(int(regs[so + j][f]) for f in REGION_DTYPE.names) == tuple(e[f] for f in REGION_DTYPE.names)
