"""MateRescue.rescue known answers from the reference's suite
(Tests/BWAMemTests/BWAMemTests.swift:860-1013), pinned on the oracle, and
host-side checks of the rescue workload generator.  No GPU."""
import numpy as np

from swiftbwa_b200.abi import ANCHOR_DTYPE, ORIENTATION_DTYPE, RESCUE_JOB_DTYPE, Scoring

FR = 1


def acgt_reference():
    """makeTestReference (:862-883): 1000 bp of repeating ACGT, one contig chr1."""
    pac = np.full(250 + 16, 0x1B, np.uint8)
    codes = np.tile(np.array([0, 1, 2, 3], np.uint8), 250)
    return pac, codes


def fr_stats():
    """FR stats of the tests (:904-911); every other orientation failed (the
    InsertSizeDistribution() default)."""
    st = np.zeros(4, ORIENTATION_DTYPE)
    st["failed"] = 1
    st[FR] = (0, 0, 150, 450)
    return st


def run(oracle_mod, mate, templates, mate_regions):
    pac, _ = acgt_reference()
    jobs = np.zeros(1, RESCUE_JOB_DTYPE)
    jobs[0] = (0, len(mate), 0, 0, len(templates), 0, len(mate_regions))
    t = np.array([(rb, rid, 0) for rb, rid in templates], ANCHOR_DTYPE)
    m = np.array([(rb, rid, 0) for rb, rid in mate_regions], ANCHOR_DTYPE)
    out, n_out, _, _ = oracle_mod.mate_rescue_batch(Scoring.default(), np.asarray(mate, np.uint8), pac, 1000, jobs,
                                                    t, m, fr_stats(), FR, np.array([0]), np.array([1000]))
    return out[:n_out[0]]


def test_rescue_finds_mate_in_fr(oracle_mod):
    """testRescueFR (:885-932): template at 100, mate = reverse complement of
    ref[380, 400) -> at least one region, score >= minSeedLength * A, rid 0."""
    _, codes = acgt_reference()
    mate = (3 - codes[380:400])[::-1]
    got = run(oracle_mod, mate, [(100, 0)], [])
    sc = Scoring.default()
    assert len(got) >= 1
    assert got[0]["score"] >= sc.min_seed_len * sc.a
    assert got[0]["rid"] == 0


def test_rescue_skips_existing_hit(oracle_mod):
    """testRescueSkipsExisting (:934-983): a mate region at rb 1599 satisfies
    FR at distance 300 -> nothing rescued."""
    got = run(oracle_mod, [0] * 20, [(100, 0)], [(1599, 0)])
    assert len(got) == 0


def test_rescue_empty_templates(oracle_mod):
    """testRescueEmptyTemplates (:985-1006) -> nothing rescued."""
    got = run(oracle_mod, [0, 1, 2, 3], [], [])
    assert len(got) == 0


def test_rescue_workload_shapes(oracle_mod):
    """The rescue workload: jobs index valid template/mate-region ranges, the
    contigs tile the genome, and the oracle rescues a good share of the mates
    placed at their true insert offset."""
    from swiftbwa_b200 import workloads as W
    wl = W.rescue_jobs(W.reference(W.SEED_BASE + 70, 200_000), 71, 300, n_contigs=5)
    assert int(wl.contig_offsets[0]) == 0
    assert int(wl.contig_offsets[-1]) + int(wl.contig_lengths[-1]) == wl.ref.n
    assert np.all(np.diff(wl.contig_offsets) > 0)
    j = wl.jobs
    assert np.all(j["tmpl_off"].astype(np.int64) + j["n_tmpl"] <= len(wl.templates))
    assert np.all(j["mreg_off"].astype(np.int64) + j["n_mreg"] <= len(wl.mate_regions))
    out, n_out, n_cand, cells = oracle_mod.mate_rescue_batch(
        Scoring.default(), wl.bases, wl.ref.pac, wl.ref.n, wl.jobs, wl.templates, wl.mate_regions, wl.stats,
        wl.primary, wl.contig_offsets, wl.contig_lengths, n_threads=4)
    assert cells > 0 and n_cand.sum() > 0
    assert (n_out > 0).mean() > 0.3
