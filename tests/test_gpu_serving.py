"""The continuous-batching request loop (swb_server_*): every request's
results equal the oracle's (the C++ restatement of BandedSWScalar.align)
and are the same alone and in the mix, in served and both plain modes;
waits are bounded; admission waits for arena space; oversized requests are
rejected at submit."""
import numpy as np
import pytest

import gen
from swiftbwa_b200 import abi
from swiftbwa_b200.abi import Scoring

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine():
    from swiftbwa_b200.alignment import Engine
    from swiftbwa_b200.build import build
    build()
    e = Engine(0)
    yield e
    e.close()


def _pool(engine, seed=31, n=6000, with_ref=False):
    d = gen.ext_tasks(seed, n, qmax=280, ref_len=8000)
    engine.upload_reference(d["pac"], d["ref_bases"])
    if with_ref:
        return d["bases"], d["tasks"], d["pac"], d["ref_bases"]
    return d["bases"], d["tasks"]


def _requests(n_pool, seed=7, k=40):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(k):
        n = int(np.exp(rng.uniform(np.log(1), np.log(1500))))
        lo = int(rng.integers(0, n_pool - n + 1))
        out.append((lo, lo + n))
    return out


@pytest.mark.parametrize("plain", [0, 1, 2])
def test_same_alone_and_in_mix(engine, oracle_mod, plain):
    from swiftbwa_b200.serving import Server, slice_request
    sc = Scoring.default()
    bases, tasks, pac, ref_bases = _pool(engine, with_ref=True)
    reqs = [slice_request(bases, tasks, lo, hi) for lo, hi in _requests(len(tasks))]
    alone = [engine.ext_batch(sc, b, t) for b, t in reqs]
    for k, (b, t) in enumerate(reqs):
        exp, _ = oracle_mod.ext_batch(sc, b, t, pac=pac, ref_bases=ref_bases)
        assert np.array_equal(alone[k], exp), f"request {k} alone differs from the oracle"
    # Small waves force large requests across several waves and both lanes.
    srv = Server(engine, sc, arena_bytes=1 << 24, max_wave_tasks=700, plain=plain)
    try:
        tickets = [srv.submit(b, t) for b, t in reqs]
        for k, tk in enumerate(tickets):
            out, s_ns, d_ns = srv.wait(tk)
            assert d_ns >= s_ns
            assert np.array_equal(out, alone[k]), f"request {k} differs in the mix"
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["tasks_completed"] == sum(len(t) for _, t in reqs)
    finally:
        srv.stop()


def test_bounded_wait_and_resume(engine):
    from swiftbwa_b200.alignment import SWBError
    from swiftbwa_b200.serving import Server, slice_request
    sc = Scoring.default()
    bases, tasks = _pool(engine, seed=32, n=500)
    b, t = slice_request(bases, tasks, 0, 500)
    srv = Server(engine, sc, arena_bytes=1 << 22, start_paused=True)
    try:
        tk = srv.submit(b, t)
        with pytest.raises(SWBError) as ei:
            srv.wait(tk, timeout_ms=50)
        assert ei.value.status == abi.SWB_ERR_TIMEOUT
        assert srv.poll(tk)[0] is False
        srv.resume()
        out, _, _ = srv.wait(tk)
        assert np.array_equal(out, engine.ext_batch(sc, b, t))
        with pytest.raises(SWBError) as ei:
            srv.poll(tk)          # released by the successful wait
        assert ei.value.status == abi.SWB_ERR_NOT_FOUND
    finally:
        srv.stop()


def test_admission_waits_for_arena_space(engine):
    from swiftbwa_b200.serving import Server, slice_request
    sc = Scoring.default()
    bases, tasks = _pool(engine, seed=33, n=3000)
    reqs = [slice_request(bases, tasks, lo, lo + 300) for lo in range(0, 3000, 300)]
    need = max(b.size for b, _ in reqs)
    srv = Server(engine, sc, arena_bytes=((need + 255) // 256) * 256 * 2, max_wave_tasks=1000)
    try:
        tickets = [srv.submit(b, t) for b, t in reqs]
        for k, tk in enumerate(tickets):
            out, _, _ = srv.wait(tk)
            assert np.array_equal(out, engine.ext_batch(sc, *reqs[k]))
        big = np.zeros(4 * need + 1024, np.uint8)
        from swiftbwa_b200.alignment import SWBError
        with pytest.raises(SWBError) as ei:
            srv.submit(big, tasks[:1].copy())
        assert ei.value.status == abi.SWB_ERR_TOO_LARGE
    finally:
        srv.stop()


@pytest.mark.parametrize("plain", [0, 2])
def test_pinned_zero_copy_pool(engine, oracle_mod, plain):
    """Requests as views of a pinned pool (span_origin, device-side rebase),
    served and through the plain single-launch kernel: same as alone and as
    the oracle."""
    torch = pytest.importorskip("torch")
    from swiftbwa_b200 import workloads as W
    from swiftbwa_b200.abi import EXT_RESULT_DTYPE
    from swiftbwa_b200.serving import Server, pool_request
    sc = Scoring.default()
    ref = W.reference(W.SEED_BASE + 9, 2_000_000)
    engine.upload_reference(ref.pac, ref.n)
    pool = W.uneven(ref, 99, 40_000)
    pb = torch.from_numpy(pool.bases).pin_memory().numpy()
    pt = torch.from_numpy(pool.tasks.view(np.uint8)).pin_memory().numpy().view(pool.tasks.dtype)
    po = torch.zeros(len(pool.tasks) * EXT_RESULT_DTYPE.itemsize, dtype=torch.uint8).pin_memory().numpy().view(EXT_RESULT_DTYPE)
    expected = engine.ext_batch(sc, pool.bases, pool.tasks)
    oracle_out, _ = oracle_mod.ext_batch(sc, pool.bases, pool.tasks, pac=ref.pac, ref_bases=ref.n, n_threads=8)
    assert np.array_equal(expected, oracle_out)
    rng = np.random.default_rng(3)
    cuts = np.sort(rng.choice(np.arange(1, len(pool.tasks)), 30, replace=False))
    bounds = list(zip([0, *cuts], [*cuts, len(pool.tasks)]))     # disjoint requests covering the pool
    srv = Server(engine, sc, arena_bytes=1 << 26, max_wave_tasks=5000, plain=plain)
    try:
        tickets = []
        for lo, hi in bounds:
            b, origin, t, o = pool_request(pb, pt, po, int(lo), int(hi))
            tickets.append(srv.submit(b, t, o, span_origin=origin))
        for tk in tickets:
            srv.wait(tk)
    finally:
        srv.stop()
    assert np.array_equal(po, expected)
    assert np.array_equal(po, oracle_out)


def test_multiserver_on_one_gpu(engine, oracle_mod):
    """The multi-GPU router over this GPU's server (one device here): results
    equal the oracle and the direct batch call, whole and split into slices."""
    from swiftbwa_b200.serving import MultiServer, Server
    sc = Scoring.default()
    d = gen.ext_tasks(404, 4000, qmax=200)
    expected = engine.ext_batch(sc, d["bases"], d["tasks"])
    assert np.array_equal(expected, oracle_mod.ext_batch(sc, d["bases"], d["tasks"])[0])
    srv = Server(engine, sc)
    try:
        ms = MultiServer([srv], split_tasks=1000)
        h = ms.submit(d["bases"], d["tasks"])
        out, s_ns, d_ns = ms.wait(h)
        assert np.array_equal(out, expected) and s_ns <= d_ns
        assert ms.load() == [0]
    finally:
        srv.stop()
