"""Edge cases through the C ABI on the GPU: empty batches of every batch
entry point, rejected inputs (each followed by a valid call on the same
context), and extension queries beyond 4096 bases (the global-scratch
thread kernel) mixed with short ones, against the oracle."""
import numpy as np
import pytest

from swiftbwa_b200 import abi
from swiftbwa_b200.abi import (CIGAR_TASK_DTYPE, EXT_TASK_DTYPE, GLOBAL_TASK_DTYPE, LOCAL_TASK_DTYPE, Scoring)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from swiftbwa_b200.alignment import Engine
    from swiftbwa_b200.build import build
    build()
    e = Engine(0)        # a context of its own: no reference uploaded yet
    yield e
    e.close()


def _ext(q_off, t_off, qlen, tlen, w=20, h0=30, flags=0):
    t = np.zeros(1, EXT_TASK_DTYPE)
    t[0] = (q_off, t_off, qlen, tlen, w, h0, 5, flags)
    return t


def _small_batch(rng, n=200):
    q = rng.integers(0, 4, 150 * n).astype(np.uint8)
    tasks = np.concatenate([_ext(150 * k, 150 * k, 100, 120) for k in range(n)])
    return q, tasks


def test_empty_batches(engine):
    sc = Scoring.default()
    b = np.zeros(1, np.uint8)
    assert len(engine.ext_batch(sc, b, np.zeros(0, EXT_TASK_DTYPE))) == 0
    res, _ = engine.global_batch(sc, b, np.zeros(0, GLOBAL_TASK_DTYPE))
    assert len(res) == 0
    assert len(engine.local_batch(sc, b, np.zeros(0, LOCAL_TASK_DTYPE))) == 0
    res, _, _ = engine.cigar_batch_raw(sc, b, np.zeros(0, CIGAR_TASK_DTYPE))
    assert len(res) == 0


def test_rejected_inputs_leave_the_context_usable(engine, oracle_mod):
    from swiftbwa_b200.alignment import SWBError
    sc = Scoring.default()
    rng = np.random.default_rng(11)
    bases, good = _small_batch(rng)
    exp, _ = oracle_mod.ext_batch(sc, bases, good, n_threads=8)
    cases = [
        (_ext(len(bases) - 10, 0, 100, 100), abi.SWB_ERR_INVALID_ARG),        # query span outside bases
        (_ext(0, 0, -1, 10), abi.SWB_ERR_INVALID_ARG),                        # negative length
        (_ext(0, 0, 70_000, 10), abi.SWB_ERR_TOO_LARGE),                      # above 65535
        (_ext(0, 0, 50, 60, flags=abi.SWB_T_FROM_REF), abi.SWB_ERR_NO_REFERENCE),
    ]
    for bad, status in cases:
        batch = np.concatenate([good[:50], bad, good[50:]])
        with pytest.raises(SWBError) as ei:
            engine.ext_batch(sc, bases, batch)
        assert ei.value.status == status
        assert np.array_equal(engine.ext_batch(sc, bases, good), exp)
    # a reference span past the uploaded reference
    ref = rng.integers(0, 4, 1000).astype(np.uint8)
    from gen import pack_ref
    engine.upload_reference(pack_ref(ref), len(ref))
    with pytest.raises(SWBError) as ei:
        engine.ext_batch(sc, bases, np.concatenate([good, _ext(0, 950, 50, 60, flags=abi.SWB_T_FROM_REF)]))
    assert ei.value.status == abi.SWB_ERR_INVALID_ARG
    assert np.array_equal(engine.ext_batch(sc, bases, good), exp)


def test_long_queries_global_scratch_path(engine, oracle_mod):
    """Queries of 4.1k-6k bases (above the warp kernel's 4096, so one thread
    each over rows in global scratch), 300-4096 (warp per extension) and
    short ones in one batch."""
    sc = Scoring.default()
    rng = np.random.default_rng(12)
    chunks, tasks, off = [], [], 0
    for k, qlen in enumerate([4100, 5000, 6000, 4500, 300, 1200, 4096, 100, 150, 80] * 3):
        w = int(rng.choice([5, 20, 60]))
        base = rng.integers(0, 4, qlen + w + 10).astype(np.uint8)
        q = base[:qlen].copy()
        t = base.copy()
        t[rng.random(len(t)) < 0.02] = rng.integers(0, 4)
        chunks += [q, t]
        tasks.append(_ext(off, off + qlen, qlen, len(t), w=w, h0=int(rng.integers(10, 60))))
        off += qlen + len(t)
    bases = np.concatenate(chunks)
    tasks = np.concatenate(tasks)
    exp, cells = oracle_mod.ext_batch(sc, bases, tasks, n_threads=8)
    got = engine.ext_batch(sc, bases, tasks)
    assert np.array_equal(got, exp)
    assert engine.last_batch_stats()[1] == cells
