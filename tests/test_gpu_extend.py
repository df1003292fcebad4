"""ExtensionAligner.extend for many chains (swb_extend_chains) against the
oracle's restatement of ExtensionAligner.extend with FMIndex.getReference on
the packed forward strand (ExtensionAligner.swift:114-346,
FMIndex.swift:147-170): every region field, bit-exact."""
import numpy as np
import pytest

from swiftbwa_b200 import abi
from swiftbwa_b200.abi import Scoring

pytestmark = pytest.mark.gpu

FIELDS = ["rb", "re", "qb", "qe", "rid", "score", "true_score", "sub", "sub_n", "w", "seed_cov", "seed_len0"]


@pytest.fixture(scope="module")
def engine():
    from swiftbwa_b200.alignment import Engine
    from swiftbwa_b200.build import build
    build()
    e = Engine(0)
    yield e
    e.close()


def _oracle_regions(oracle_mod, sc, wl, gl):
    out = []
    for c in wl.chains:
        so, ns = int(c["seed_off"]), int(c["n_seeds"])
        seeds = [(int(s["rbeg"]), int(s["qbeg"]), int(s["len"]), int(s["score"])) for s in wl.seeds[so:so + ns]]
        read = wl.bases[int(c["read_off"]):int(c["read_off"]) + int(c["read_len"])]
        regs, _, _ = oracle_mod.extend(seeds, int(c["rid"]), read, wl.ref.pac, sc, ref_mode=1, genome_len=gl)
        out.append(regs)
    return out


def _compare(engine, oracle_mod, sc, wl):
    gl = wl.ref.n
    engine.upload_reference(wl.ref.pac, gl)
    regs, counts, rounds = engine.extend_chains(sc, wl.bases, wl.seeds, wl.chains, gl)
    exp = _oracle_regions(oracle_mod, sc, wl, gl)
    for k, c in enumerate(wl.chains):
        so = int(c["seed_off"])
        got = regs[so:so + int(counts[k])]
        assert len(got) == len(exp[k]), f"chain {k}: {len(got)} regions, oracle {len(exp[k])}"
        for j, e in enumerate(exp[k]):
            for f in FIELDS:
                assert int(got[j][f]) == e[f], f"chain {k} region {j} field {f}: {int(got[j][f])} != {e[f]}"
    return rounds


SCORINGS = {
    "default": {},
    "narrow_band": dict(band_width=8),          # band retries fire often
    "clips_zdrop": dict(pen_clip5=0, pen_clip3=30, zdrop=20),
    "affine": dict(a=2, b=5, o_ins=7, e_ins=2, o_del=5, e_del=3, min_seed_len=25),
}


@pytest.mark.parametrize("name", list(SCORINGS))
def test_extend_chains_matches_oracle(engine, oracle_mod, name):
    from swiftbwa_b200 import workloads as W
    sc = Scoring.default()
    for k, v in SCORINGS[name].items():
        setattr(sc, k, v)
    ref = W.reference(W.SEED_BASE + 50, 300_000, tandem_frac=0.05)
    wl = W.chains(ref, 77 + len(name), 1500, 150, sub=0.03, indel=0.01, spurious_frac=0.3, a=sc.a)
    rounds = _compare(engine, oracle_mod, sc, wl)
    assert rounds >= 1
    if name == "default":   # pinned inputs and outputs: copied straight to and from the device
        import torch
        from swiftbwa_b200.abi import REGION_DTYPE
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8)).pin_memory().numpy().view(a.dtype)
        regs, counts, _ = engine.extend_chains(sc, wl.bases, wl.seeds, wl.chains, ref.n)
        out = (pin(np.zeros(len(wl.seeds), REGION_DTYPE)), pin(np.full(len(wl.chains), 7, np.uint32)))
        pr, pc, _ = engine.extend_chains(sc, pin(wl.bases), pin(wl.seeds), pin(wl.chains), ref.n, out=out)
        assert pr is out[0] and np.array_equal(pc, counts) and np.array_equal(pr, regs)


def test_extend_chains_edges(engine, oracle_mod):
    """Seeds at both genome ends and both strand boundaries, equal-score ties,
    empty chains, a read with no flanks and long reads (int32 DP path)."""
    from swiftbwa_b200 import workloads as W
    sc = Scoring.default()
    gl = 50_000
    ref = W.reference(W.SEED_BASE + 51, gl)
    rng = np.random.default_rng(5)
    full = np.concatenate([ref.codes, 3 - ref.codes[::-1]])
    reads, seeds, chains = [], [], []

    def add(rbeg, qbeg, rl, slen, extra=()):
        read = full[max(rbeg - qbeg, 0):max(rbeg - qbeg, 0) + rl].copy()
        if read.size < rl:
            read = np.concatenate([read, rng.integers(0, 4, rl - read.size).astype(np.uint8)])
        read[rng.random(rl) < 0.02] = rng.integers(0, 4)
        off = sum(r.size for r in reads)
        reads.append(read)
        ss = [(rbeg, qbeg, slen, slen)] + list(extra)
        chains.append((off, rl, len(chains), len(seeds), len(ss)))
        seeds.extend(ss)

    add(0, 0, 150, 30)                       # genome start, no left flank
    add(40, 40, 150, 30)                     # left target clipped at 0
    add(gl - 30, 120, 150, 30)               # right target runs off the forward strand
    add(gl, 0, 150, 40)                      # first reverse-strand base
    add(gl + 20, 60, 150, 25)                # left target crosses the strand boundary
    add(2 * gl - 30, 120, 150, 30)           # reverse strand end
    add(1000, 10, 150, 20, [(1090, 100, 20, 20), (1050, 60, 20, 20)])      # equal-score ties, covered seeds
    add(5000, 0, 150, 150)                   # seed spans the read: no extension at all
    add(7000, 300, 900, 40, [(7400, 700, 30, 30)])                          # long read: int32 path
    add(9000, 20, 100, 20, [(30000, 20, 20, 20)])                           # repeat seed elsewhere
    chains.append((0, 0, len(chains), len(seeds), 0))                       # empty chain
    bases = np.concatenate(reads).astype(np.uint8)
    seeds_a = np.array([(r, q, l, s, 0) for r, q, l, s in seeds], abi.SEED_DTYPE)
    chains_a = np.array(chains, abi.CHAIN_DTYPE)
    wl = W.ChainWorkload(ref, bases, seeds_a, chains_a, 0)
    _compare(engine, oracle_mod, sc, wl)


def test_extend_chains_rejects_bad_input(engine):
    from swiftbwa_b200 import workloads as W
    from swiftbwa_b200.alignment import SWBError
    sc = Scoring.default()
    ref = W.reference(W.SEED_BASE + 52, 10_000)
    engine.upload_reference(ref.pac, ref.n)
    wl = W.chains(ref, 3, 10, 150)
    bad = wl.seeds.copy()
    bad[0]["qbeg"] = 149          # seed runs past the read end
    with pytest.raises(SWBError) as ei:
        engine.extend_chains(sc, wl.bases, bad, wl.chains, ref.n)
    assert ei.value.status == abi.SWB_ERR_INVALID_ARG
    with pytest.raises(SWBError) as ei:
        engine.extend_chains(sc, wl.bases, wl.seeds, wl.chains, ref.n + 1)   # longer than the uploaded strand
    assert ei.value.status == abi.SWB_ERR_NO_REFERENCE
