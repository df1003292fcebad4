"""CUDA kernels vs the oracle, through the C ABI: known answers, the
reference's GPU-vs-CPU differential shapes, and seeded fuzz sets.  Every
field must match bit for bit."""
import numpy as np
import pytest

import gen
import known
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


class GpuBackend:
    def __init__(self, e, o):
        self.e, self.o = e, o

    def ext(self, q, t, sc, w, h0, eb):
        return self.e.banded_sw_align(q, t, sc, w, h0, eb).as_tuple()

    def global_(self, q, t, sc, w):
        r = self.e.global_align(q, t, sc, w)
        return r.score, list(r.cigar)

    def compute_nm(self, cigar, q, t):
        return self.o.compute_nm(cigar, q, t)

    def cigar(self, q, r, qb, qe, rl, rev, ts, iw, sc, pos):
        return self.e.cigar_generate(q, r, qb, qe, rl, rev, ts, iw, sc, pos)

    def local(self, q, t, sc, ms):
        r = self.e.local_align(q, t, sc, ms)
        return None if r is None else r.as_tuple()


CASES = known.load()["known_answers"]


@pytest.mark.parametrize("case", [c for c in CASES if c["fn"] in ("ext", "global", "global_w_pair", "local", "cigar")],
                         ids=lambda c: c["name"])
def test_known_answer_on_gpu(case, engine, oracle_mod):
    fails = known.evaluate(case, GpuBackend(engine, oracle_mod))
    assert fails is not None and not fails, "\n".join(fails or [])


def test_differential_shapes(engine, oracle_mod):
    for d in known.load()["differential_shapes"]:
        sc = Scoring.default(**d["scoring"])
        if d["kind"] == "ext":
            g = engine.banded_sw_align(d["q"], d["t"], sc, d["w"], d["h0"]).as_tuple()
            o = oracle_mod.banded_sw_scalar(d["q"], d["t"], sc, d["w"], d["h0"])[0]
        else:
            r = engine.local_align(d["q"], d["t"], sc, 0)
            g = None if r is None else r.as_tuple()
            o = oracle_mod.local_align(d["q"], d["t"], sc, 0)[0]
        assert g == o, (d["source"], g, o)


SCORINGS = [
    dict(),
    dict(zdrop=0),
    dict(zdrop=10),
    dict(a=2, b=3, o_ins=5, e_ins=2, o_del=4, e_del=3),
    dict(a=1, b=1, o_ins=1, e_ins=1, o_del=1, e_del=1, zdrop=5),
    dict(a=8),
]


def _cmp_struct(got, exp, fields):
    bad = np.nonzero(np.any(np.stack([got[f] != exp[f] for f in fields]), axis=0))[0]
    return bad


@pytest.mark.parametrize("si", range(len(SCORINGS)))
def test_ext_fuzz(engine, oracle_mod, si):
    sc = Scoring.default(**SCORINGS[si])
    d = gen.ext_tasks(1000 + si, 3000, qmax=300, ref_len=5000)
    engine.upload_reference(d["pac"], d["ref_bases"])
    got = engine.ext_batch(sc, d["bases"], d["tasks"])   # host entry: the one-launch form at this size
    exp, cells = oracle_mod.ext_batch(sc, d["bases"], d["tasks"], pac=d["pac"], ref_bases=d["ref_bases"],
                                      n_threads=8)
    bad = _cmp_struct(got, exp, got.dtype.names)
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]}: {got[bad[:3]]} vs {exp[bad[:3]]} tasks {d['tasks'][bad[:3]]}"
    ms, gcells = engine.last_batch_stats()
    assert gcells == cells
    binned = gen.ext_batch_binned(engine, sc, d["bases"], d["tasks"])
    bad = _cmp_struct(binned, exp, got.dtype.names)
    assert bad.size == 0, f"binned: {bad.size} mismatches, first {bad[:5]}"


@pytest.mark.parametrize("si", [0, 1, 3])
def test_ext_ring_rows(engine, oracle_mod, si):
    """Queries above the last length class (256 bases; here up to 2500, w
    1-150) whose band is narrower than the query keep a ring of 2w+3 columns
    in the shared-memory bins instead of taking the int32 bin: the oracle's
    results, with first-row values (h0 up to 120) entering the ring late."""
    sc = Scoring.default(**SCORINGS[si])
    d = gen.ext_tasks(4242 + si, 1500, qmax=2500, ref_len=20000)
    engine.upload_reference(d["pac"], d["ref_bases"])
    engine.profile(True)
    engine.profile_reset()
    try:
        got = gen.ext_batch_binned(engine, sc, d["bases"], d["tasks"])
        prof = engine.profile_read()
    finally:
        engine.profile(False)
    exp, cells = oracle_mod.ext_batch(sc, d["bases"], d["tasks"], pac=d["pac"], ref_bases=d["ref_bases"],
                                      n_threads=8)
    bad = _cmp_struct(got, exp, got.dtype.names)
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]}: {got[bad[:3]]} vs {exp[bad[:3]]} tasks {d['tasks'][bad[:3]]}"
    assert sum(v[2] for k, v in prof.items() if k.startswith("ext_")) == cells


def test_ext_host_entry_small_batch_threshold(engine, oracle_mod):
    """The host entry runs batches of up to 16384 tasks in one launch and
    larger ones through the bins: both sides of the threshold give the
    oracle's results and cell counts."""
    sc = Scoring.default()
    d = gen.ext_tasks(515, 16385, qmax=300, ref_len=8000)
    engine.upload_reference(d["pac"], d["ref_bases"])
    exp, _ = oracle_mod.ext_batch(sc, d["bases"], d["tasks"], pac=d["pac"], ref_bases=d["ref_bases"], n_threads=8)
    for n in (16384, 16385):
        got = engine.ext_batch(sc, d["bases"], d["tasks"][:n])
        bad = _cmp_struct(got, exp[:n], got.dtype.names)
        assert bad.size == 0, f"{n} tasks: {bad.size} mismatches, first {bad[:5]}"
        _, cells = oracle_mod.ext_batch(sc, d["bases"], d["tasks"][:n], pac=d["pac"], ref_bases=d["ref_bases"],
                                        n_threads=8)
        assert engine.last_batch_stats()[1] == cells


def test_ext_fuzz_int32_path(engine, oracle_mod):
    sc = Scoring.default()
    d = gen.ext_tasks(77, 500, qmax=120, big_scores=True)
    got = engine.ext_batch(sc, d["bases"], d["tasks"])
    exp, _ = oracle_mod.ext_batch(sc, d["bases"], d["tasks"], n_threads=8)
    bad = _cmp_struct(got, exp, got.dtype.names)
    assert bad.size == 0, f"{bad.size} mismatches: {got[bad[:3]]} vs {exp[bad[:3]]}"


@pytest.mark.parametrize("bins", [[64, 256], list(range(32, 257, 16)), [256], [8, 40, 100], [24, 200, 232]])
def test_ext_length_classes(engine, oracle_mod, bins):
    """Any set of length classes gives the oracle's results: coarse, fine,
    one class, and low bounds that send long queries to the int32 bin."""
    sc = Scoring.default()
    d = gen.ext_tasks(2024, 3000, qmax=300, ref_len=5000)
    engine.upload_reference(d["pac"], d["ref_bases"])
    exp, cells = oracle_mod.ext_batch(sc, d["bases"], d["tasks"], pac=d["pac"], ref_bases=d["ref_bases"], n_threads=8)
    default = engine.ext_bins()
    try:
        engine.set_ext_bins(bins)
        assert engine.ext_bins() == bins
        got = gen.ext_batch_binned(engine, sc, d["bases"], d["tasks"])
        bad = _cmp_struct(got, exp, got.dtype.names)
        assert bad.size == 0, f"{bins}: {bad.size} mismatches, first {bad[:5]}"
    finally:
        engine.set_ext_bins(default)


def test_ext_bins_autotuner(engine, oracle_mod):
    """The tuner keeps the fastest candidate, never slower than the defaults
    on its sample, and results stay equal to the oracle under it."""
    from swiftbwa_b200 import workloads as W
    sc = Scoring.default()
    wl = W.config2(n=200_000, ref_len=10_000_000)
    engine.upload_reference(wl.ref.pac, wl.ref.n)
    default = engine.ext_bins()
    try:
        assert default == [32, 48, 64, 80, 96, 112, 128, 160, 192, 256]
        rep = engine.tune_ext_bins(sc, wl.bases, wl.tasks)
        assert 1 <= len(rep["bins"]) <= 15 and rep["bins"] == sorted(set(rep["bins"]))
        assert min(rep["bins"]) >= 8 and max(rep["bins"]) <= 256
        assert engine.ext_bins() == rep["bins"]
        assert 0 < rep["ms"] <= rep["default_ms"]
        sub = slice(0, 20_000)
        got = engine.ext_batch(sc, wl.bases, wl.tasks[sub])
        exp, _ = oracle_mod.ext_batch(sc, wl.bases, wl.tasks[sub], pac=wl.ref.pac, ref_bases=wl.ref.n, n_threads=8)
        assert np.array_equal(got, exp)
        with pytest.raises(Exception):
            engine.set_ext_bins([64, 32])          # not ascending
        with pytest.raises(Exception):
            engine.set_ext_bins([512])             # above the shared-memory rows' 256
    finally:
        engine.set_ext_bins(default)


# Gap and mismatch costs high enough that long tasks leave the int16 rows.
BIG_PENALTIES = dict(a=1, b=60, o_ins=50, e_ins=30, o_del=45, e_del=35)


@pytest.mark.parametrize("si,qmax", [(0, 200), (3, 200), (4, 200), (0, 420), (5, 420), ("big", 200)])
def test_global_fuzz(engine, oracle_mod, si, qmax):
    """qmax 420 mixes the shared-memory kernels (queries up to 256 bases) with
    the global-scratch kernel; the "big" scoring mixes int16 and int32 rows
    within the shared-memory kernels."""
    sc = Scoring.default(**(BIG_PENALTIES if si == "big" else SCORINGS[si]))
    d = gen.global_tasks(2000 + (7 if si == "big" else si) + qmax, 1500, qmax=qmax)
    res, cig = engine.global_batch(sc, d["bases"], d["tasks"])
    eres, ecig, _ = oracle_mod.global_batch(sc, d["bases"], d["tasks"], n_threads=8)
    for k in range(len(res)):
        assert res["score"][k] == eres["score"][k], k
        assert res["n_cigar"][k] == eres["n_cigar"][k], k
        assert res["w_used"][k] == eres["w_used"][k] and res["attempts"][k] == eres["attempts"][k], k
        o, n = int(res["cigar_off"][k]), int(res["n_cigar"][k])
        eo = int(eres["cigar_off"][k])
        assert np.array_equal(cig[o:o + n], ecig[eo:eo + n]), k


@pytest.mark.parametrize("si", [0, 3, 4, 5])
def test_local_fuzz(engine, oracle_mod, si):
    sc = Scoring.default(**SCORINGS[si])
    d = gen.local_tasks(3000 + si, 1200)
    got = engine.local_batch(sc, d["bases"], d["tasks"])
    exp, _ = oracle_mod.local_batch(sc, d["bases"], d["tasks"], n_threads=8)
    bad = _cmp_struct(got, exp, got.dtype.names)
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]}: {got[bad[:3]]} vs {exp[bad[:3]]} tasks {d['tasks'][bad[:3]]}"


def test_local_many_claims_per_half_warp(oracle_mod):
    """60k mate-rescue pairs of one stripe count (150-base mates, ~700-base
    windows): the striped kernel's grid is the device's resident blocks, so
    each half-warp claims about ten tasks of the bin from its counter, longest
    target first; every field against the oracle."""
    from swiftbwa_b200 import workloads as W
    from swiftbwa_b200.alignment import Engine
    sc = Scoring.default()
    wl = W.config3(n=60_000)
    eng = Engine(0)
    try:
        eng.upload_reference(wl.ref.pac, wl.ref.n)
        got = eng.local_batch(sc, wl.bases, wl.tasks)
    finally:
        eng.close()
    exp, _ = oracle_mod.local_batch(sc, wl.bases, wl.tasks, pac=wl.ref.pac, ref_bases=wl.ref.n, n_threads=8)
    bad = _cmp_struct(got, exp, got.dtype.names)
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]}"
    assert (exp["score"] > 0).sum() > 50_000


def test_ext_config_workloads_chunked(engine, oracle_mod):
    """Config-0 and a 2.6M-task config-1 shard through the host entry point
    (the latter runs as pipelined chunks), every task against the oracle."""
    import os
    from swiftbwa_b200 import workloads as W
    sc = Scoring.default()
    for wl in (W.config0(), W.config1(n_reads=1_300_000, ref_len=10_000_000)):
        engine.upload_reference(wl.ref.pac, wl.ref.n)
        got = engine.ext_batch(sc, wl.bases, wl.tasks)
        exp, cells = oracle_mod.ext_batch(sc, wl.bases, wl.tasks, pac=wl.ref.pac, ref_bases=wl.ref.n,
                                          n_threads=os.cpu_count() or 8)
        bad = _cmp_struct(got, exp, got.dtype.names)
        assert bad.size == 0, f"{wl.name}: {bad.size} mismatches, first {bad[:5]}"
        assert engine.last_batch_stats()[1] == cells


def test_ext_large_batch_chunk_schedules(engine):
    """A batch large enough for the host entry point's growing chunks (from
    1/32 of the batch, then two short ones at the end) gives the same results
    as its two halves, each cut into equal chunks."""
    from swiftbwa_b200 import workloads as W
    sc = Scoring.default()
    wl = W.config1(n_reads=4_300_000, ref_len=10_000_000)
    assert len(wl.tasks) >= 16 * (1 << 19)
    engine.upload_reference(wl.ref.pac, wl.ref.n)
    whole = engine.ext_batch(sc, wl.bases, wl.tasks)
    h = len(wl.tasks) // 2
    parts = np.concatenate([engine.ext_batch(sc, wl.bases, wl.tasks[:h]), engine.ext_batch(sc, wl.bases, wl.tasks[h:])])
    assert np.array_equal(whole, parts)


@pytest.mark.parametrize("si", [0, 3])
def test_cigar_generate_fuzz(engine, oracle_mod, si):
    """CIGARGenerator.generate: fast path, device DP with retries, squeeze,
    NM, MD and soft clips against the oracle, task by task."""
    from swiftbwa_b200.abi import CIGAR_TASK_DTYPE
    sc = Scoring.default(**SCORINGS[si])
    rng = np.random.default_rng(5000 + si)
    chunks, rows, cases = [], [], []
    off = 0
    for k in range(1500):
        rl_read = int(rng.integers(20, 200))
        read = rng.integers(0, 4, rl_read).astype(np.uint8)
        qb = int(rng.integers(0, rl_read // 3))
        qe = int(rng.integers(max(qb + 1, rl_read - rl_read // 3), rl_read + 1))
        qseg = read[qb:qe].copy()
        rseg = gen.mutate(rng, qseg, sub=rng.choice([0.0, 0.01, 0.05]), indel=rng.choice([0.0, 0.0, 0.02, 0.05]))
        if rng.random() < 0.2:   # leading/trailing reference bases -> squeezed deletions
            rseg = np.concatenate([rng.integers(0, 4, int(rng.integers(0, 4))).astype(np.uint8), rseg,
                                   rng.integers(0, 4, int(rng.integers(0, 4))).astype(np.uint8)])
        if len(rseg) == 0:
            rseg = np.array([2], np.uint8)
        true_score = int(len(qseg) * sc.a - rng.integers(0, 30))
        iw = int(rng.choice([1, 5, 20, 100]))
        is_rev = bool(rng.random() < 0.5)
        pos = int(rng.integers(0, 10**9))
        chunks += [qseg, rseg]
        rows.append((off, off + len(qseg), len(qseg), len(rseg), qb, qe, rl_read, int(is_rev), true_score, iw, pos, 0, 0))
        cases.append((qseg, rseg, qb, qe, rl_read, is_rev, true_score, iw, pos))
        off += len(qseg) + len(rseg)
    tasks = np.array(rows, dtype=CIGAR_TASK_DTYPE)
    bases = np.concatenate(chunks)
    got = engine.cigar_batch(sc, bases, tasks)
    for k, c in enumerate(cases):
        exp = oracle_mod.cigar_generate(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], sc, c[8])
        g = got[k]
        assert (g["cigar"], g["nm"], g["md"], g["score"], g["pos"], g["used_dp"]) == \
            (exp["cigar"], exp["nm"], exp["md"], exp["score"], exp["pos"], exp["used_dp"]), (k, g, exp)
    # Pinned inputs are copied straight to the device: the same results.
    import torch
    pb = torch.from_numpy(bases).pin_memory().numpy()
    pt = torch.from_numpy(tasks.view(np.uint8)).pin_memory().numpy().view(CIGAR_TASK_DTYPE)
    ra, ca, ma = engine.cigar_batch_raw(sc, bases, tasks)
    rb, cb, mb = engine.cigar_batch_raw(sc, pb, pt)
    assert np.array_equal(ra, rb)
    nc = int((ra["cigar_off"] + ra["n_cigar"].astype(np.uint64)).max())
    nm = int((ra["md_off"] + ra["md_len"].astype(np.uint64)).max())
    assert np.array_equal(ca[:nc], cb[:nc]) and np.array_equal(ma[:nm], mb[:nm])
    # Pinned output buffers are written by the device directly: the same results.
    from swiftbwa_b200.abi import CIGAR_RESULT_DTYPE
    ccap, mcap = engine.cigar_caps(tasks)
    po = (torch.full((len(tasks) * CIGAR_RESULT_DTYPE.itemsize,), 0xA5, dtype=torch.uint8).pin_memory().numpy()
          .view(CIGAR_RESULT_DTYPE),
          torch.full((ccap,), -1, dtype=torch.int32).pin_memory().numpy().view(np.uint32),
          torch.full((mcap,), 0xA5, dtype=torch.uint8).pin_memory().numpy())
    rc, cc, mc = engine.cigar_batch_raw(sc, pb, pt, out=po)
    assert rc is po[0] and np.array_equal(ra, rc)
    assert np.array_equal(ca[:nc], cc[:nc]) and np.array_equal(ma[:nm], mc[:nm])


def test_alu_probes(engine):
    """The roofline denominators: int32 add/max and packed 16-bit DPX add/max
    rates are positive and of B200 magnitude (tens of T ops/s)."""
    i32 = engine.int_alu_peak()
    i16 = engine.int16x2_alu_peak()
    assert 5e12 < i32 < 5e14
    assert 5e12 < i16 < 5e14
