"""SMEM seeding on the GPU (swb_upload_bwt + swb_smem_batch) against the
oracle's restatement of SMEMFinder.findAllSMEMs: every read's SMEM list
(SA interval, query span, order) equal, at occurrence thresholds 1 and 20
(the re-seeding pass's minIntv), for reads from both strands with N bases,
random reads, ragged and zero lengths; a window too small for a read's
SMEMs is reported with the full counts; calls without an index or with bad
spans fail cleanly and leave the context usable."""
import numpy as np
import pytest

from swiftbwa_b200 import abi

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from swiftbwa_b200.alignment import Engine
    from swiftbwa_b200.build import build
    build()
    e = Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def index(oracle_mod):
    from swiftbwa_b200 import workloads as W
    ref = W.reference(W.SEED_BASE + 77, 300_000, tandem_frac=0.2)
    return ref, oracle_mod.bwt_build(ref.codes)


def _reads(ref, seed, n, L):
    rng = np.random.default_rng(seed)
    out, lens = np.zeros((n, L), np.uint8), np.full(n, L, np.int32)
    for r in range(n):
        p = int(rng.integers(0, ref.n - L))
        x = ref.codes[p:p + L].copy()
        if rng.random() < 0.5:
            x = (3 - x[::-1]).astype(np.uint8)
        m = rng.random(L)
        x[m < 0.02] = rng.integers(0, 4, int(np.sum(m < 0.02)))
        x[rng.random(L) < 0.005] = 4
        if rng.random() < 0.1:
            x = rng.integers(0, 4, L).astype(np.uint8)
        out[r] = x
        if rng.random() < 0.1:
            lens[r] = int(rng.integers(0, L))
    return out.reshape(-1), np.arange(n, dtype=np.uint64) * L, lens


@pytest.mark.parametrize("min_intv,split_len", [(1, 0), (20, 0), (1, 28)])
def test_smems_equal_oracle(engine, oracle_mod, index, min_intv, split_len):
    """min_intv 20: the re-seeding pass's threshold; split_len 28: with the
    internal re-seeding of BWAMemAligner.internalReseed (split width 10)."""
    ref, idx = index
    engine.upload_bwt(idx.cp, idx.count, idx.length, idx.sentinel)
    bases, off, lens = _reads(ref, 5 + min_intv + split_len, 3000, 150)
    cap = 128
    got, gn, goff = engine.smem_batch(bases, off, lens, 19, min_intv=min_intv, cap_per_read=cap,
                                      split_len=split_len)
    exp, en, over = oracle_mod.smem_batch(idx, bases, off, lens, 19, min_intv=min_intv, cap=cap, n_threads=8,
                                          split_len=split_len, split_width=10)
    assert over == 0 and np.array_equal(gn, en) and en.sum() > 0
    assert np.array_equal(goff, np.concatenate([[0], np.cumsum(en.astype(np.uint64))[:-1]]))
    for r in range(len(lens)):
        assert np.array_equal(got[goff[r]: goff[r] + gn[r]], exp[r * cap: r * cap + en[r]]), f"read {r}"


def test_long_and_ragged_reads(engine, oracle_mod, index):
    """Reads of 0 to 1500 bases in one batch (long ones keep many candidate
    intervals, past those a lane holds in shared memory; short and empty
    ones finish while their warp's other lanes walk on), with re-seeding."""
    ref, idx = index
    engine.upload_bwt(idx.cp, idx.count, idx.length, idx.sentinel)
    rng = np.random.default_rng(99)
    n = 700
    lens = rng.integers(1, 1500, n).astype(np.int32)
    lens[:60] = rng.integers(0, 4, 60)
    rng.shuffle(lens)
    chunks = []
    for L in lens:
        p = int(rng.integers(0, ref.n - max(int(L), 1)))
        x = ref.codes[p:p + int(L)].copy()
        if rng.random() < 0.5:
            x = (3 - x[::-1]).astype(np.uint8)
        x[rng.random(len(x)) < 0.01] = rng.integers(0, 4)
        x[rng.random(len(x)) < 0.003] = 4
        chunks.append(x)
    bases = np.concatenate(chunks).astype(np.uint8)
    off = np.concatenate([[0], np.cumsum(lens.astype(np.uint64))[:-1]]).astype(np.uint64)
    cap = 512
    got, gn, goff = engine.smem_batch(bases, off, lens, 15, cap_per_read=cap, split_len=28)
    exp, en, over = oracle_mod.smem_batch(idx, bases, off, lens, 15, cap=cap, n_threads=8, split_len=28,
                                          split_width=10)
    assert over == 0 and np.array_equal(gn, en) and en.sum() > 0
    for r in range(n):
        assert np.array_equal(got[goff[r]: goff[r] + gn[r]], exp[r * cap: r * cap + en[r]]), f"read {r}"
    # Pinned reads and outputs: copied straight to and from the device, the same SMEMs.
    import torch
    from swiftbwa_b200.abi import SMEM_DTYPE
    tot = int(gn.sum())
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).pin_memory().numpy().view(a.dtype)
    out = (pin(np.full((tot + 1) * SMEM_DTYPE.itemsize, 0xA5, np.uint8)).view(SMEM_DTYPE),
           pin(np.zeros(n, np.uint32)), pin(np.zeros(n, np.uint64)))
    pg, pn, po = engine.smem_batch(pin(bases), pin(off), pin(lens), 15, cap_per_read=cap, split_len=28, out=out)
    assert np.array_equal(pn, gn) and np.array_equal(po, goff) and np.array_equal(pg[:tot], got[:tot])


def test_small_window_reports_counts(engine, oracle_mod, index):
    from swiftbwa_b200.alignment import SWBError
    ref, idx = index
    engine.upload_bwt(idx.cp, idx.count, idx.length, idx.sentinel)
    bases, off, lens = _reads(ref, 11, 500, 150)
    _, en, _ = oracle_mod.smem_batch(idx, bases, off, lens, 15, cap=256)
    assert en.max() > 1
    with pytest.raises(SWBError) as ei:
        engine.smem_batch(bases, off, lens, 15, cap_per_read=1)
    assert ei.value.status == abi.SWB_ERR_TOO_LARGE
    first = int(np.nonzero(en > 1)[0][0])
    assert f"read {first}:".encode() in engine.lib.swb_last_error_message()
    got, gn, _ = engine.smem_batch(bases, off, lens, 15, cap_per_read=256)   # usable afterwards
    assert np.array_equal(gn, en)
    with pytest.raises(SWBError) as ei:                          # output array too small
        engine.smem_batch(bases, off, lens, 15, cap_per_read=256, out_cap=int(en.sum()) - 1)
    assert ei.value.status == abi.SWB_ERR_TOO_LARGE and b"out_cap" in engine.lib.swb_last_error_message()


def test_empty_and_invalid_inputs(engine, index):
    from swiftbwa_b200.alignment import Engine, SWBError
    ref, idx = index
    fresh = Engine(0)
    try:
        with pytest.raises(SWBError) as ei:                      # no index uploaded
            fresh.smem_batch(np.zeros(10, np.uint8), np.array([0]), np.array([10]), 19)
        assert ei.value.status == abi.SWB_ERR_NO_REFERENCE
    finally:
        fresh.close()
    engine.upload_bwt(idx.cp, idx.count, idx.length, idx.sentinel)
    out, n, o = engine.smem_batch(np.zeros(1, np.uint8), np.zeros(0, np.uint64), np.zeros(0, np.int32), 19)
    assert n.size == 0 and o.size == 0
    with pytest.raises(SWBError) as ei:                          # span beyond the bases buffer
        engine.smem_batch(np.zeros(10, np.uint8), np.array([5]), np.array([10]), 19)
    assert ei.value.status == abi.SWB_ERR_INVALID_ARG
    bases, off, lens = _reads(ref, 13, 50, 100)
    got, gn, _ = engine.smem_batch(bases, off, lens, 19)
    assert gn.sum() > 0
