"""The allocation-free extension entry point, swb_ext_batch_static.

It exists for callers that cannot let the library call cudaMalloc -- a
server whose own arena already holds the free HBM, or a batching loop that
cannot afford cudaMalloc/cudaFree stalling its other streams -- and works
from one static device array instead.  These tests call it through the C
ABI on device buffers the test owns and hold it to the oracle (the C++
restatement of BandedSWScalar.align) and to the allocating entry point
(swb_ext_batch) bit for bit, on two calls in a row (the second call sees
the array the first one left behind), check that the second call leaves the
device's free memory unchanged, and check that a task beyond its stated
limit is rejected with a clear error.

This file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import gen
from swiftbwa_b200 import abi
from swiftbwa_b200.abi import EXT_RESULT_DTYPE, EXT_TASK_DTYPE, Scoring

pytestmark = pytest.mark.gpu


def _mixed_tasks():
    """Shared-memory-path tasks (queries <= 256, int16-safe) mixed with
    int32-path tasks (queries up to 300, and h0 above 30000)."""
    a = gen.ext_tasks(4242, 2500, qmax=300, ref_len=6000)
    b = gen.ext_tasks(4343, 400, qmax=120, big_scores=True)
    shift = a["bases"].size
    tb = b["tasks"].copy()
    tb["q_off"] += shift
    explicit = (tb["flags"] & abi.SWB_T_FROM_REF) == 0
    tb["t_off"][explicit] += shift
    bases = np.concatenate([a["bases"], b["bases"]])
    tasks = np.concatenate([a["tasks"], tb]).astype(EXT_TASK_DTYPE)
    return bases, tasks, a["pac"], a["ref_bases"]


def _dev(torch, arr: np.ndarray):
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.uint8)).to("cuda:0")


def _call_static(lib, torch, sc, d_bases, d_pac, d_tasks, n, d_out):
    torch.cuda.synchronize()
    return lib.swb_ext_batch_static(C.byref(sc), C.c_void_p(d_bases.data_ptr()),
                                    C.c_void_p(d_pac.data_ptr() if d_pac is not None else 0),
                                    C.c_void_p(d_tasks.data_ptr()), n, C.c_void_p(d_out.data_ptr()),
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream))


def test_static_entry_matches_allocating_entry_twice(oracle_mod):
    torch = pytest.importorskip("torch")
    from swiftbwa_b200.alignment import Engine
    from swiftbwa_b200.build import build
    build()
    lib = abi.load_library()
    bases, tasks, pac, ref_bases = _mixed_tasks()
    for scoring in (Scoring.default(), Scoring.default(a=2, b=3, o_ins=5, e_ins=2, o_del=4, e_del=3, zdrop=10)):
        eng = Engine(0)
        try:
            eng.upload_reference(pac, ref_bases)
            expected = eng.ext_batch(scoring, bases, tasks)
        finally:
            eng.close()
        oracle_out, _ = oracle_mod.ext_batch(scoring, bases, tasks, pac=pac, ref_bases=ref_bases, n_threads=8)
        assert np.array_equal(expected, oracle_out)
        d_bases, d_pac, d_tasks = _dev(torch, bases), _dev(torch, pac), _dev(torch, tasks)
        outs = [torch.full((len(tasks) * EXT_RESULT_DTYPE.itemsize,), 0xA5, dtype=torch.uint8, device="cuda:0")
                for _ in range(2)]
        for call in range(2):
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info(0)[0]
            rc = _call_static(lib, torch, scoring, d_bases, d_pac, d_tasks, len(tasks), outs[call])
            assert rc == abi.SWB_OK, (rc, lib.swb_last_error_message())
            torch.cuda.synchronize()
            if call == 1:   # the set-up of the first call may load the library's device code
                assert torch.cuda.mem_get_info(0)[0] == free_before, "the second call changed free device memory"
            got = outs[call].cpu().numpy().view(EXT_RESULT_DTYPE)
            bad = np.nonzero(got != oracle_out)[0]
            assert bad.size == 0, f"call {call}: {bad.size} tasks differ from the oracle, first {bad[:5]}"
            assert np.array_equal(got, expected)


def test_static_entry_rejects_query_beyond_limit():
    torch = pytest.importorskip("torch")
    lib = abi.load_library()
    rng = np.random.default_rng(5)
    q = rng.integers(0, 4, 1500).astype(np.uint8)
    t = np.concatenate([q, rng.integers(0, 4, 50).astype(np.uint8)])
    bases = np.concatenate([q[:100], t[:200], q, t])
    tasks = np.zeros(2, EXT_TASK_DTYPE)
    tasks[0] = (0, 100, 100, 200, 100, 19, 5, 0)                      # fits the limit
    tasks[1] = (300, 300 + 1500, 1500, len(t), 100, 19, 5, 0)         # int32 path, 1500 > 1024 bases
    d_bases, d_tasks = _dev(torch, bases), _dev(torch, tasks)
    d_out = torch.zeros(2 * EXT_RESULT_DTYPE.itemsize, dtype=torch.uint8, device="cuda:0")
    rc = _call_static(lib, torch, Scoring.default(), d_bases, None, d_tasks, 2, d_out)
    assert rc == abi.SWB_ERR_TOO_LARGE
    assert b"task 1" in lib.swb_last_error_message()
    got = d_out.cpu().numpy().view(EXT_RESULT_DTYPE)
    assert got[1]["score"] == 0 and got[0]["score"] > 0
