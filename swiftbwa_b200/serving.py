"""Python side of the continuous-batching request loop (swb_server_* in
include/swb_cuda.h) and the config-4 request-stream driver used by bench.py.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

from . import abi
from .abi import EXT_RESULT_DTYPE, EXT_TASK_DTYPE, Scoring, ptr
from .alignment import Engine, _check


class Server:
    """A request loop on one Engine's GPU.  Keeps every submitted request's
    arrays alive until its ticket has been waited for."""

    def __init__(self, engine: Engine, scoring: Scoring, arena_bytes: int = 0, max_wave_tasks: int = 0,
                 plain: int = 0, start_paused: bool = False, latency_cells: int = 0):
        self.lib = engine.lib
        self.engine = engine
        opts = abi.ServerOpts(arena_bytes, max_wave_tasks, int(plain), int(start_paused), int(latency_cells), 0)
        h = C.c_void_p()
        _check(self.lib.swb_server_start(engine.h, C.byref(scoring), C.byref(opts), C.byref(h)), "swb_server_start")
        self.h = h
        self._keep = {}
        self._lock = threading.Lock()

    def submit(self, bases: np.ndarray, tasks: np.ndarray, out: Optional[np.ndarray] = None,
               span_origin: int = 0) -> int:
        """Queue one request; task offsets address bases[x - span_origin]."""
        assert tasks.dtype == EXT_TASK_DTYPE and tasks.flags["C_CONTIGUOUS"]
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        if out is None:
            out = np.zeros(len(tasks), EXT_RESULT_DTYPE)
        t = C.c_uint64()
        _check(self.lib.swb_server_submit(self.h, ptr(bases), bases.size, span_origin, tasks.ctypes.data,
                                          len(tasks), out.ctypes.data, C.byref(t)), "swb_server_submit")
        with self._lock:
            self._keep[t.value] = (bases, tasks, out)
        return t.value

    def poll(self, ticket: int):
        done, status = C.c_int(), C.c_int()
        _check(self.lib.swb_server_poll(self.h, ticket, C.byref(done), C.byref(status)), "swb_server_poll")
        return bool(done.value), status.value

    def wait(self, ticket: int, timeout_ms: int = 60_000):
        """-> (results array, submit_ns, done_ns); raises SWBError on timeout."""
        status, s_ns, d_ns = C.c_int(), C.c_uint64(), C.c_uint64()
        _check(self.lib.swb_server_wait(self.h, ticket, timeout_ms, C.byref(status), C.byref(s_ns), C.byref(d_ns)),
               "swb_server_wait")
        _check(status.value, "request")
        with self._lock:
            _, _, out = self._keep.pop(ticket)
        return out, s_ns.value, d_ns.value

    def resume(self):
        _check(self.lib.swb_server_resume(self.h), "swb_server_resume")

    def stats(self) -> dict:
        st = abi.ServerStats()
        _check(self.lib.swb_server_stats_get(self.h, C.byref(st)), "swb_server_stats_get")
        return {f: getattr(st, f) for f, _ in abi.ServerStats._fields_}

    def stop(self):
        if self.h:
            _check(self.lib.swb_server_stop(self.h), "swb_server_stop")
            self.h = None

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


class MultiServer:
    """Requests over several GPUs, one Server each (one per device's Engine):
    every request goes to the server with the fewest outstanding estimated
    DP cells, and a request of at least `split_tasks` tasks is cut into
    cell-balanced contiguous slices, one per server, each writing its own
    view of the request's output.  No data crosses GPUs; every GPU holds its
    own copy of the resident reference."""

    def __init__(self, servers, split_tasks: int = 0):
        if not servers:
            raise ValueError("MultiServer needs at least one server")
        self.servers = list(servers)
        self.split_tasks = int(split_tasks)
        self._load = [0] * len(self.servers)      # outstanding estimated cells per server
        self._handles = {}
        self._next = 0
        self._lock = threading.Lock()

    def _pick(self) -> int:
        return min(range(len(self.servers)), key=lambda k: (self._load[k], k))

    def submit(self, bases: np.ndarray, tasks: np.ndarray, out: Optional[np.ndarray] = None,
               span_origin: int = 0) -> int:
        from .sharding import partition_by_cells, task_cells_estimate
        assert tasks.dtype == EXT_TASK_DTYPE and tasks.flags["C_CONTIGUOUS"]
        if out is None:
            out = np.zeros(len(tasks), EXT_RESULT_DTYPE)
        cells = task_cells_estimate(tasks)
        n_srv = len(self.servers)
        if n_srv > 1 and self.split_tasks and len(tasks) >= self.split_tasks:
            b = partition_by_cells(tasks, n_srv)
            pieces = [(b[k], b[k + 1]) for k in range(n_srv) if b[k + 1] > b[k]]
        else:
            pieces = [(0, len(tasks))]
        parts = []
        with self._lock:
            order = sorted(range(n_srv), key=lambda k: (self._load[k], k))
            for j, (lo, hi) in enumerate(pieces):
                k = order[j % n_srv] if len(pieces) > 1 else self._pick()
                c = int(cells[lo:hi].sum())
                t = self.servers[k].submit(bases, tasks[lo:hi], out[lo:hi], span_origin=span_origin)
                self._load[k] += c
                parts.append((k, t, c))
            h = self._next
            self._next += 1
            self._handles[h] = (parts, out)
        return h

    def poll(self, handle: int):
        """(done, status): done when every slice is; the first nonzero status."""
        parts, _ = self._handles[handle]
        done, status = True, 0
        for k, t, _ in parts:
            d, st = self.servers[k].poll(t)
            done = done and d
            status = status or st
        return done, status

    def wait(self, handle: int, timeout_ms: int = 60_000):
        """-> (results array, first submit_ns, last done_ns)."""
        with self._lock:
            parts, out = self._handles.pop(handle)
        s_ns, d_ns = None, 0
        for k, t, c in parts:
            try:
                _, s, d = self.servers[k].wait(t, timeout_ms)
            finally:
                with self._lock:
                    self._load[k] -= c
            s_ns = s if s_ns is None else min(s_ns, s)
            d_ns = max(d_ns, d)
        return out, s_ns, d_ns

    def load(self):
        """Outstanding estimated cells per server."""
        with self._lock:
            return list(self._load)

    def stop(self):
        for srv in self.servers:
            srv.stop()


@dataclass
class Request:
    lo: int          # task range in the pool
    hi: int
    at: float        # arrival time (s from start)


def request_stream(seed: int, n_pool: int, rate: float, duration: float, min_tasks=1_000,
                   max_tasks=1_000_000) -> List[Request]:
    """Poisson arrivals at `rate`/s for `duration` s; sizes log-uniform in
    [min_tasks, max_tasks]; each request is a random contiguous slice of a
    task pool of n_pool tasks."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            break
        n = int(np.exp(rng.uniform(np.log(min_tasks), np.log(max_tasks))))
        n = min(n, n_pool)
        lo = int(rng.integers(0, n_pool - n + 1))
        out.append(Request(lo, lo + n, t))
    return out


def slice_request(bases: np.ndarray, tasks: np.ndarray, lo: int, hi: int):
    """A request's own (bases, tasks): the pool slice with offsets rebased to
    its own bases buffer (targets from the resident reference keep theirs)."""
    t = tasks[lo:hi].copy()
    explicit = (t["flags"] & abi.SWB_T_FROM_REF) == 0
    starts = [t["q_off"]] + ([t["t_off"][explicit]] if explicit.any() else [])
    ends = [t["q_off"] + t["qlen"].astype(np.uint64)]
    if explicit.any():
        ends.append(t["t_off"][explicit] + t["tlen"][explicit].astype(np.uint64))
    b0 = int(min(int(x.min()) for x in starts))
    b1 = int(max(int(x.max()) for x in ends))
    t["q_off"] -= np.uint64(b0)
    t["t_off"][explicit] -= np.uint64(b0)
    return bases[b0:max(b1, b0 + 1)], t


def pool_request(bases: np.ndarray, tasks: np.ndarray, out: np.ndarray, lo: int, hi: int):
    """Zero-copy request over a pool whose queries are laid out in task order
    and whose targets are reference spans: (bases slice, span_origin, tasks
    slice, out slice), all views of the pool arrays."""
    q0 = int(tasks["q_off"][lo])
    q1 = int(tasks["q_off"][hi - 1]) + int(tasks["qlen"][hi - 1])
    return bases[q0:max(q1, q0 + 1)], q0, tasks[lo:hi], out[lo:hi]


def run_pool_stream(server: Server, bases: np.ndarray, tasks: np.ndarray, out: np.ndarray, reqs: List[Request],
                    open_loop: bool = True):
    """Like run_stream for a pool of reference-target tasks with queries in
    task order; requests are views of the (ideally pinned) pool arrays, so the
    submitter does no host work besides the call."""
    tickets = [None] * len(reqs)
    lat = [None] * len(reqs)
    t0 = time.perf_counter()

    def submitter():
        for k, r in enumerate(reqs):
            if open_loop:
                delay = r.at - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            b, origin, t, o = pool_request(bases, tasks, out, r.lo, r.hi)
            tickets[k] = server.submit(b, t, o, span_origin=origin)

    th = threading.Thread(target=submitter)
    th.start()
    for k in range(len(reqs)):
        while tickets[k] is None:
            time.sleep(0.0002)
        _, s_ns, d_ns = server.wait(tickets[k], timeout_ms=600_000)
        lat[k] = (d_ns - s_ns) * 1e-9
    th.join()
    makespan = time.perf_counter() - t0
    return [(r.hi - r.lo, lat[k]) for k, r in enumerate(reqs)], makespan


def run_stream(server: Server, bases: np.ndarray, tasks: np.ndarray, reqs: List[Request], open_loop: bool = True):
    """Submits the requests (at their arrival times when open_loop, else all at
    once) and waits for them; returns per-request (n_tasks, latency_s) and the
    makespan in seconds."""
    # Closed loop: every request prepared up front, then submitted at once.
    # Open loop: each request is prepared just before its arrival time, so
    # host memory holds only the requests in flight.
    prepared = [slice_request(bases, tasks, r.lo, r.hi) for r in reqs] if not open_loop else None
    tickets = [None] * len(reqs)
    lat = [None] * len(reqs)
    t0 = time.perf_counter()

    def submitter():
        for k, r in enumerate(reqs):
            if open_loop:
                b, t = slice_request(bases, tasks, r.lo, r.hi)
                delay = r.at - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
            else:
                b, t = prepared[k]
                prepared[k] = None
            tickets[k] = server.submit(b, t)

    th = threading.Thread(target=submitter)
    th.start()
    for k in range(len(reqs)):
        while tickets[k] is None:
            time.sleep(0.0002)
        _, s_ns, d_ns = server.wait(tickets[k], timeout_ms=600_000)
        lat[k] = (d_ns - s_ns) * 1e-9
    th.join()
    makespan = time.perf_counter() - t0
    return [(r.hi - r.lo, lat[k]) for k, r in enumerate(reqs)], makespan
