"""Multi-GPU request routing on CPU: MultiServer over fake per-GPU servers
(least-loaded routing, load accounting, cell-balanced slicing of large
requests into views of one output), and the batch partition it uses."""
import numpy as np
import pytest

from swiftbwa_b200.abi import EXT_RESULT_DTYPE, EXT_TASK_DTYPE
from swiftbwa_b200.serving import MultiServer
from swiftbwa_b200.sharding import partition_by_cells, task_cells_estimate


class FakeServer:
    """Stands in for one GPU's Server: remembers what it was given and, on
    wait, writes a result that is a pure function of each task."""

    def __init__(self, name):
        self.name, self.calls, self.next, self.open = name, [], 0, {}

    def submit(self, bases, tasks, out, span_origin=0):
        assert tasks.flags["C_CONTIGUOUS"] and out.flags["C_CONTIGUOUS"]
        t = self.next
        self.next += 1
        self.calls.append((len(tasks), span_origin))
        self.open[t] = (tasks, out)
        return t

    def poll(self, t):
        return True, 0

    def wait(self, t, timeout_ms=0):
        tasks, out = self.open.pop(t)
        out["score"] = tasks["qlen"] * 3 + tasks["tlen"]
        out["qle"] = tasks["w"]
        return out, 100 + t, 200 + t

    def stop(self):
        pass


def _tasks(rng, n):
    t = np.zeros(n, EXT_TASK_DTYPE)
    t["qlen"] = rng.integers(1, 250, n)
    t["tlen"] = t["qlen"] + rng.integers(0, 100, n)
    t["w"] = rng.integers(10, 100, n)
    t["q_off"] = np.arange(n) * 300
    return t


def test_partition_by_cells_properties():
    rng = np.random.default_rng(3)
    t = _tasks(rng, 5000)
    c = task_cells_estimate(t)
    for parts in (1, 2, 3, 8, 64):
        b = partition_by_cells(t, parts)
        assert b[0] == 0 and b[-1] == len(t) and len(b) == parts + 1
        assert all(x <= y for x, y in zip(b, b[1:]))
        share = c.sum() / parts
        for k in range(parts):
            assert abs(int(c[b[k]:b[k + 1]].sum()) - share) <= c.max() + 1
    assert partition_by_cells(t[:0], 3) == [0, 0, 0, 0]
    with pytest.raises(ValueError):
        partition_by_cells(t, 0)


def test_least_loaded_routing_and_load_accounting():
    rng = np.random.default_rng(5)
    srv = [FakeServer(k) for k in range(3)]
    ms = MultiServer(srv)
    reqs = [_tasks(rng, n) for n in (500, 20, 20, 300, 10)]
    hs = [ms.submit(np.zeros(1, np.uint8), r) for r in reqs]
    # replay the policy: each request to the server with the least outstanding cells (lowest index on ties)
    sim, expect = [0, 0, 0], [[], [], []]
    for r in reqs:
        k = min(range(3), key=lambda j: (sim[j], j))
        sim[k] += int(task_cells_estimate(r).sum())
        expect[k].append(len(r))
    assert [[c[0] for c in s.calls] for s in srv] == expect
    load = ms.load()
    assert load == sim
    assert sum(load) == sum(int(task_cells_estimate(r).sum()) for r in reqs)
    assert srv[0].calls[0][0] == 500 and srv[1].calls[0][0] == 20 and srv[2].calls[0][0] == 20
    for h, r in zip(hs, reqs):
        out, s_ns, d_ns = ms.wait(h)
        assert np.array_equal(out["score"], r["qlen"] * 3 + r["tlen"])
        assert s_ns <= d_ns
    assert ms.load() == [0, 0, 0]


def test_large_request_split_into_balanced_slices():
    rng = np.random.default_rng(7)
    srv = [FakeServer(k) for k in range(4)]
    ms = MultiServer(srv, split_tasks=1000)
    t = _tasks(rng, 10_000)
    out = np.zeros(len(t), EXT_RESULT_DTYPE)
    h = ms.submit(np.zeros(1, np.uint8), t, out, span_origin=123)
    sizes = [s.calls[0][0] for s in srv]
    assert sum(sizes) == len(t) and all(n > 0 for n in sizes)
    assert all(s.calls[0][1] == 123 for s in srv)            # every slice keeps the request's span origin
    assert ms.poll(h) == (True, 0)
    got, _, _ = ms.wait(h)
    assert got is out                                         # the slices wrote views of one output
    assert np.array_equal(out["score"], t["qlen"] * 3 + t["tlen"])
    assert np.array_equal(out["qle"], t["w"])
    b = partition_by_cells(t, 4)
    assert sizes == [b[k + 1] - b[k] for k in range(4)]
    small = ms.submit(np.zeros(1, np.uint8), t[:999])         # below the split size: one server
    assert sum(len(s.calls) for s in srv) == 5
    ms.wait(small)
