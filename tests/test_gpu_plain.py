"""The plain one-launch-per-batch extension kernel (swb_ext_batch_plain_device),
the baseline that batching is measured against: the dispatch shape of
BandedSWDispatcher.dispatchBatch8/16 (one launch, one task per thread, input
order) over the same two-row kernel code.  Its results must equal the oracle
(the C++ restatement of BandedSWScalar.align) for batches whose rows are int8
only, int16, mixed with int32-path tasks (long queries, large scores) and
empty tasks, under several scorings."""
import numpy as np
import pytest

import gen
from swiftbwa_b200 import abi
from swiftbwa_b200.abi import EXT_RESULT_DTYPE, EXT_TASK_DTYPE, Scoring

pytestmark = pytest.mark.gpu

SCORINGS = [Scoring.default(), Scoring.default(a=2, b=3, o_ins=5, e_ins=2, o_del=4, e_del=3, zdrop=10),
            Scoring.default(zdrop=0)]


@pytest.fixture(scope="module")
def engine():
    from swiftbwa_b200.alignment import Engine
    from swiftbwa_b200.build import build
    build()
    e = Engine(0)
    yield e
    e.close()


def _run_plain(engine, sc, bases, tasks):
    torch = pytest.importorskip("torch")
    d_b = torch.from_numpy(np.ascontiguousarray(bases)).to("cuda:0")
    d_t = torch.from_numpy(np.ascontiguousarray(tasks).view(np.uint8)).to("cuda:0")
    d_o = torch.full((max(len(tasks), 1) * EXT_RESULT_DTYPE.itemsize,), 0xA5, dtype=torch.uint8, device="cuda:0")
    s = torch.cuda.Stream()
    engine.ext_batch_plain_device(sc, d_b.data_ptr(), d_t.data_ptr(), len(tasks), d_o.data_ptr(), s.cuda_stream)
    s.synchronize()
    return d_o.cpu().numpy().view(EXT_RESULT_DTYPE)[: len(tasks)]


def _mixed(seed):
    a = gen.ext_tasks(seed, 3000, qmax=300, ref_len=6000)
    b = gen.ext_tasks(seed + 1, 300, qmax=120, big_scores=True)
    shift = a["bases"].size
    tb = b["tasks"].copy()
    tb["q_off"] += shift
    explicit = (tb["flags"] & abi.SWB_T_FROM_REF) == 0
    tb["t_off"][explicit] += shift
    return (np.concatenate([a["bases"], b["bases"]]), np.concatenate([a["tasks"], tb]).astype(EXT_TASK_DTYPE),
            a["pac"], a["ref_bases"])


@pytest.mark.parametrize("si", range(len(SCORINGS)))
def test_plain_mixed_batch_equals_oracle(engine, oracle_mod, si):
    sc = SCORINGS[si]
    bases, tasks, pac, ref_bases = _mixed(700 + si)
    engine.upload_reference(pac, ref_bases)
    got = _run_plain(engine, sc, bases, tasks)
    exp, _ = oracle_mod.ext_batch(sc, bases, tasks, pac=pac, ref_bases=ref_bases, n_threads=8)
    bad = np.nonzero(got != exp)[0]
    assert bad.size == 0, f"{bad.size} tasks differ, first {bad[:5]}"


@pytest.mark.parametrize("kind", ["int8_rows", "int16_rows", "empty_only", "int32_only"])
def test_plain_row_shapes(engine, oracle_mod, kind):
    sc = Scoring.default()
    d = gen.ext_tasks(811, 2000, qmax=200)
    bases, tasks = d["bases"], d["tasks"].copy()
    if kind == "int8_rows":      # every score bound within a byte: the int8-row launch
        tasks = tasks[tasks["qlen"].astype(np.int64) + np.maximum(tasks["h0"], 0) <= 255]
    elif kind == "int16_rows":
        tasks["h0"] = 200
    elif kind == "empty_only":
        tasks = tasks[:50].copy()
        tasks["qlen"][::2] = 0
        tasks["tlen"][1::2] = 0
    else:                        # scores beyond int16: only the int32 kernels run
        tasks["h0"] = 33000
    got = _run_plain(engine, sc, bases, tasks)
    exp, _ = oracle_mod.ext_batch(sc, bases, tasks, n_threads=8)
    assert np.array_equal(got, exp)
