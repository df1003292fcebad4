"""MateRescue.rescue on the GPU (swb_mate_rescue) against the oracle's
restatement (MateRescue.swift:29-171 with fetchSequence, hasMateHit and
LocalSWAligner.align): every region field, counts and candidate counts,
bit-exact; plus the reference's own rescue tests."""
import numpy as np
import pytest

from swiftbwa_b200 import abi
from swiftbwa_b200.abi import ANCHOR_DTYPE, RESCUE_JOB_DTYPE, Scoring

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from swiftbwa_b200.alignment import Engine
    from swiftbwa_b200.build import build
    build()
    e = Engine(0)
    yield e
    e.close()


def _compare(engine, oracle_mod, sc, wl):
    engine.upload_reference(wl.ref.pac, wl.ref.n)
    args = (wl.bases, wl.jobs, wl.templates, wl.mate_regions, wl.stats, wl.primary, wl.contig_offsets,
            wl.contig_lengths, wl.ref.n)
    got, n, nc = engine.mate_rescue(sc, *args)
    exp, en, enc, _ = oracle_mod.mate_rescue_batch(sc, wl.bases, wl.ref.pac, wl.ref.n, wl.jobs, wl.templates,
                                                   wl.mate_regions, wl.stats, wl.primary, wl.contig_offsets,
                                                   wl.contig_lengths, n_threads=8)
    assert np.array_equal(nc, enc), "candidate counts differ"
    assert np.array_equal(n, en), "rescued counts differ"
    for j, job in enumerate(wl.jobs):
        o = 4 * int(job["tmpl_off"])
        for k in range(int(n[j])):
            assert got[o + k] == exp[o + k], (j, k, got[o + k], exp[o + k])
    return int(n.sum())


SCORINGS = {"default": {}, "affine": dict(a=2, b=5, o_ins=7, e_ins=2, o_del=5, e_del=3, min_seed_len=15),
            "a8": dict(a=8)}


@pytest.mark.parametrize("name", list(SCORINGS))
def test_rescue_matches_oracle(engine, oracle_mod, name):
    from swiftbwa_b200 import workloads as W
    sc = Scoring.default(**SCORINGS[name])
    ref = W.reference(W.SEED_BASE + 80, 400_000, tandem_frac=0.05)
    wl = W.rescue_jobs(ref, 81 + len(name), 1500, 150, n_contigs=7, more_orientations=True)
    assert _compare(engine, oracle_mod, sc, wl) > 0


def test_rescue_short_contigs_and_mates(engine, oracle_mod):
    """Many short contigs (windows clamped and crossing contigs), 100 bp
    mates, insert close to the mate length, primary orientation FR only."""
    from swiftbwa_b200 import workloads as W
    ref = W.reference(W.SEED_BASE + 82, 60_000)
    wl = W.rescue_jobs(ref, 83, 800, 100, n_contigs=40, ins_mean=180.0, ins_sd=30.0, hit_frac=0.5)
    _compare(engine, oracle_mod, Scoring.default(), wl)


def test_rescue_reference_cases(engine, oracle_mod):
    """The reference suite's three MateRescue tests (BWAMemTests.swift:885-1006)
    as one batch of jobs on the 1000 bp ACGT reference."""
    from swiftbwa_b200 import workloads as W
    from test_rescue_host import acgt_reference, fr_stats, FR
    pac, codes = acgt_reference()
    mate_fr = ((3 - codes[380:400])[::-1]).astype(np.uint8)
    bases = np.concatenate([mate_fr, np.zeros(20, np.uint8), np.array([0, 1, 2, 3], np.uint8)])
    jobs = np.zeros(3, RESCUE_JOB_DTYPE)
    jobs[0] = (0, 20, 0, 0, 1, 0, 0)
    jobs[1] = (20, 20, 0, 1, 1, 0, 1)
    jobs[2] = (40, 4, 0, 2, 0, 1, 0)
    templates = np.array([(100, 0, 0), (100, 0, 0)], ANCHOR_DTYPE)
    mregs = np.array([(1599, 0, 0)], ANCHOR_DTYPE)
    ref = W.Reference(codes, pac, np.zeros((0, 2), np.int64))
    wl = W.RescueJobs(ref, bases, jobs, templates, mregs, fr_stats(), FR, np.array([0], np.int64),
                      np.array([1000], np.int32))
    engine.upload_reference(pac, 1000)
    got, n, _ = engine.mate_rescue(Scoring.default(), bases, jobs, templates, mregs, wl.stats, FR,
                                   wl.contig_offsets, wl.contig_lengths, 1000)
    assert n[0] >= 1 and got[0]["score"] >= 19 and got[0]["rid"] == 0
    assert n[1] == 0 and n[2] == 0
    _compare(engine, oracle_mod, Scoring.default(), wl)


def test_rescue_primary_failed_and_errors(engine, oracle_mod):
    from swiftbwa_b200 import workloads as W
    from swiftbwa_b200.alignment import SWBError
    ref = W.reference(W.SEED_BASE + 84, 50_000)
    wl = W.rescue_jobs(ref, 85, 100, 150, n_contigs=2)
    wl.stats["failed"][1] = 1                      # primary failed -> nothing at all
    wl.stats["failed"][0] = 0
    assert _compare(engine, oracle_mod, Scoring.default(), wl) == 0
    bad = wl.jobs.copy()
    bad[0]["n_tmpl"] = len(wl.templates) + 5
    with pytest.raises(SWBError) as ei:
        engine.mate_rescue(Scoring.default(), wl.bases, bad, wl.templates, wl.mate_regions, wl.stats, 1,
                           wl.contig_offsets, wl.contig_lengths, ref.n)
    assert ei.value.status == abi.SWB_ERR_INVALID_ARG
