"""The multi-GPU plumbing of bench.py on CPU: two gloo ranks, each with its
own seeded shard (weak scaling) extended by the oracle, no data exchange;
the process group carries only barriers and the max over ranks."""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, outdir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle
        from swiftbwa_b200 import workloads as W
        from swiftbwa_b200.abi import Scoring
        from swiftbwa_b200.sharding import dist_env, max_over_ranks, whole_job_rate
        ws, r, local = dist_env()
        assert (ws, r, local) == (world, rank, rank)
        wl = W.config0(rank=r)                      # this rank's shard
        res, cells = oracle.ext_batch(Scoring.default(), wl.bases, wl.tasks, pac=wl.ref.pac, ref_bases=wl.ref.n,
                                      n_threads=2)
        dist.barrier()
        t = 1.0 + rank                              # a per-rank step time
        tmax = max_over_ranks(t, dist)
        rate = whole_job_rate(len(wl.tasks), ws, tmax)
        np.savez(os.path.join(outdir, f"rank{rank}.npz"), tasks=wl.tasks.view(np.uint8), res=res.view(np.uint8),
                 tmax=tmax, rate=rate, cells=cells)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_weak_scaling(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    from oracle import oracle
    from swiftbwa_b200 import workloads as W
    from swiftbwa_b200.abi import EXT_RESULT_DTYPE, EXT_TASK_DTYPE, Scoring
    got = [np.load(tmp_path / f"rank{r}.npz") for r in range(world)]
    # Shards differ between ranks; each equals the shard one process makes
    # for that rank, and so do its results (nothing crossed ranks).
    assert not np.array_equal(got[0]["tasks"], got[1]["tasks"])
    for r in range(world):
        wl = W.config0(rank=r)
        assert np.array_equal(got[r]["tasks"].view(EXT_TASK_DTYPE), wl.tasks)
        exp, _ = oracle.ext_batch(Scoring.default(), wl.bases, wl.tasks, pac=wl.ref.pac, ref_bases=wl.ref.n,
                                  n_threads=2)
        assert np.array_equal(got[r]["res"].view(EXT_RESULT_DTYPE), exp)
        # Every rank sees the slowest rank's time; the rate counts all ranks' units.
        assert float(got[r]["tmax"]) == 2.0
        assert float(got[r]["rate"]) == pytest.approx(len(wl.tasks) * world / 2.0)


def test_single_process_defaults(monkeypatch):
    from swiftbwa_b200.sharding import dist_env, max_over_ranks, whole_job_rate
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert dist_env() == (1, 0, 0)
    assert max_over_ranks(3.5) == 3.5
    assert whole_job_rate(100, 1, 2.0) == 50.0
