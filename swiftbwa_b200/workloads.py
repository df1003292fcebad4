"""Seeded synthetic workloads for the five benchmark configurations
(libswb_workload.so, built from csrc/swb_workload.cpp).

The reference publishes no dataset for this path; every config is a seeded
synthetic stand-in with the shapes, sizes and error rates the configs
state.  Seeds are 0x5EED0000 + config (+ rank for multi-GPU shards).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .abi import (ANCHOR_DTYPE, CHAIN_DTYPE, EXT_TASK_DTYPE, GLOBAL_TASK_DTYPE, LOCAL_TASK_DTYPE, ORIENTATION_DTYPE,
                  RESCUE_JOB_DTYPE, SEED_DTYPE, SWB_GLB_RETRY)
from .build import WORKLOAD_OUT, build_workload

SEED_BASE = 0x5EED0000

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(WORKLOAD_OUT):
            build_workload()
        L = C.CDLL(WORKLOAD_OUT)
        vp, i64, u64, dbl, i32 = C.c_void_p, C.c_int64, C.c_uint64, C.c_double, C.c_int
        L.swbw_reference.argtypes = [u64, u64, dbl, vp, vp, vp, i64]
        L.swbw_reference.restype = i64
        L.swbw_ext_tasks.argtypes = [u64, vp, i64, vp, i64, dbl, i64, i32, dbl, dbl, dbl, i32, i32, i32, i32,
                                     i32, i32, i32, vp, vp, vp]
        L.swbw_ext_tasks.restype = i64
        L.swbw_uneven_tasks.argtypes = [u64, vp, i64, i64, i32, i32, vp, i32, i32, i32, i32, i32, dbl, dbl, i32,
                                        vp, vp]
        L.swbw_uneven_tasks.restype = i64
        L.swbw_rescue_tasks.argtypes = [u64, vp, i64, i64, i32, i32, dbl, dbl, dbl, dbl, i32, vp, vp]
        L.swbw_rescue_tasks.restype = None
        L.swbw_chains.argtypes = [u64, vp, i64, i64, i32, dbl, dbl, dbl, i32, i32, i32, dbl, vp, vp, vp]
        L.swbw_chains.restype = i64
        L.swbw_rescue_jobs.argtypes = [u64, vp, i64, vp, i64, i64, i32, dbl, dbl, dbl, dbl, dbl, vp, vp, vp, vp]
        L.swbw_rescue_jobs.restype = u64
        _lib = L
    return _lib


@dataclass
class Reference:
    codes: np.ndarray          # one byte per base, 0-3
    pac: np.ndarray            # .pac layout
    blocks: np.ndarray         # (n, 2) tandem blocks [start, len]

    @property
    def n(self) -> int:
        return int(self.codes.size)


def reference(seed: int, n: int, tandem_frac: float = 0.0, max_blocks: int = 1 << 16) -> Reference:
    codes = np.empty(n, np.uint8)
    pac = np.empty((n + 3) // 4 + 16, np.uint8)
    blocks = np.zeros((max_blocks, 2), np.int64)
    nb = lib().swbw_reference(seed, n, tandem_frac, codes.ctypes.data, pac.ctypes.data, blocks.ctypes.data,
                              max_blocks)
    return Reference(codes, pac, blocks[:nb].copy())


@dataclass
class ExtWorkload:
    ref: Reference
    bases: np.ndarray                  # reads (or queries), one byte per base
    tasks: np.ndarray                  # EXT_TASK_DTYPE
    read_info: Optional[np.ndarray] = None   # (n_reads, 4): ref_start, ref_end, n_sub, indel_bases
    read_len: int = 0
    name: str = ""
    meta: dict = field(default_factory=dict)


def ext_from_reads(ref: Reference, seed: int, n_reads: int, read_len: int, *, sub=0.01, indel=0.001,
                   n_rate=0.005, w=100, h0=19, end_bonus5=5, end_bonus3=5, left=True, random_seed_pos=True,
                   tandem_read_frac=0.0, bases_out: Optional[np.ndarray] = None,
                   tasks_out: Optional[np.ndarray] = None) -> ExtWorkload:
    per = 2 if left else 1
    reads = bases_out if bases_out is not None else np.empty(n_reads * read_len, np.uint8)
    tasks = tasks_out if tasks_out is not None else np.empty(n_reads * per, EXT_TASK_DTYPE)
    info = np.empty((n_reads, 4), np.int64)
    nt = lib().swbw_ext_tasks(seed, ref.codes.ctypes.data, ref.n, ref.blocks.ctypes.data, len(ref.blocks),
                              tandem_read_frac, n_reads, read_len, sub, indel, n_rate, 19, int(random_seed_pos),
                              w, h0, end_bonus5, end_bonus3, int(left), reads.ctypes.data, tasks.ctypes.data,
                              info.ctypes.data)
    return ExtWorkload(ref, reads, tasks[:nt], info, read_len)


def config0(rank: int = 0) -> ExtWorkload:
    """10,000 right extensions: 100 bp reads off a 50 kbp reference, 1% subs,
    0.1% 1-3 bp indels, 0.5% N; query = suffix after the first exact 19-mer,
    target = qlen + w window; w=100, h0=19, end bonus 5."""
    ref = reference(SEED_BASE + 0 + 1000 * rank, 50_000)
    wl = ext_from_reads(ref, SEED_BASE + 0 + 1000 * rank + 1, 10_000, 100, left=False, random_seed_pos=False)
    wl.name = "config0: 10k right extensions, 100 bp reads, 50 kbp reference"
    return wl


def config1(rank: int = 0, n_reads: int = 5_000_000, ref_len: int = 100_000_000) -> ExtWorkload:
    """10M extension tasks (left on reversed prefixes + right) from 150 bp
    reads off a 100 Mbp reference in which 20% of reads come from inserted
    tandem-repeat blocks (period 2-6, 1-5 kbp); error rates as config 0."""
    ref = reference(SEED_BASE + 1 + 1000 * rank, ref_len, tandem_frac=0.02)
    wl = ext_from_reads(ref, SEED_BASE + 1 + 1000 * rank + 1, n_reads, 150, left=True, random_seed_pos=True,
                        tandem_read_frac=0.2)
    wl.name = f"config1: {len(wl.tasks)} left+right extensions, {n_reads} x 150 bp reads, {ref_len // 10**6} Mbp reference, 20% tandem-repeat reads"
    return wl


def global_from_reads(wl: ExtWorkload, scoring_a: int = 1, w: int = 100, only_non_fast_path: bool = True):
    """Banded NW + CIGAR task per read hit span (config 1): query = read,
    target = the reference span the read was drawn from.  With
    only_non_fast_path, reads CIGARGenerator would answer with its pure-M
    fast path (equal lengths, no indel, deficit < open+extend of both gaps,
    CIGARGenerator.swift:59-80) are left out, as the reference skips their DP."""
    info = wl.read_info
    L = wl.read_len
    rs, re_, nsub, nind = info[:, 0], info[:, 1], info[:, 2], info[:, 3]
    rlen = np.minimum(re_ - rs, 10_000).astype(np.int64)
    est = L * scoring_a - nsub * 5 - nind * 2
    fast = (rlen == L) & (nind == 0) & (L * scoring_a - est < 14)
    keep = ~fast if only_non_fast_path else np.ones(len(info), bool)
    idx = np.nonzero(keep & (rlen > 0))[0]
    t = np.zeros(len(idx), GLOBAL_TASK_DTYPE)
    t["q_off"] = idx.astype(np.uint64) * L
    t["t_off"] = rs[idx].astype(np.uint64)
    t["qlen"] = L
    t["tlen"] = rlen[idx]
    t["w"] = w
    t["true_score"] = est[idx]
    t["flags"] = SWB_GLB_RETRY | 0x8    # SWB_T_FROM_REF
    return t


def config2(rank: int = 0, n: int = 20_000_000, ref_len: int = 100_000_000) -> ExtWorkload:
    """20M uneven extensions: qlen log-uniform 30-250, w uniform 10-100,
    target qlen + w, h0 uniform 19-60, 2% subs, 0.3% indels."""
    ref = reference(SEED_BASE + 2 + 1000 * rank, ref_len)
    return uneven(ref, SEED_BASE + 2 + 1000 * rank + 1, n, name=f"config2: {n} uneven extensions")


def uneven(ref: Reference, seed: int, n: int, qmin=30, qmax=250, mix=None, wmin=10, wmax=100, h0min=19, h0max=60,
           sub=0.02, indel=0.003, end_bonus=5, name="uneven") -> ExtWorkload:
    bases = np.empty(n * qmax, np.uint8)
    tasks = np.empty(n, EXT_TASK_DTYPE)
    mix_arr = np.asarray(mix or [], np.int32)
    used = lib().swbw_uneven_tasks(seed, ref.codes.ctypes.data, ref.n, n, qmin, qmax,
                                   mix_arr.ctypes.data if mix_arr.size else None, int(mix_arr.size),
                                   wmin, wmax, h0min, h0max, sub, indel, end_bonus, bases.ctypes.data,
                                   tasks.ctypes.data)
    return ExtWorkload(ref, bases[:used], tasks, None, 0, name)


@dataclass
class RescueWorkload:
    ref: Reference
    bases: np.ndarray
    tasks: np.ndarray
    name: str = ""


def config3(rank: int = 0, n: int = 2_000_000, ref_len: int = 100_000_000) -> RescueWorkload:
    """2M mate-rescue local SW: 150 bp mate (2% subs) vs a ~700 bp window
    (insert 400 +- 50, window = mean +- 4 SD plus the mate), 10% no hit,
    minSubScore = 19."""
    ref = reference(SEED_BASE + 3 + 1000 * rank, ref_len)
    bases = np.empty(n * 150, np.uint8)
    tasks = np.empty(n, LOCAL_TASK_DTYPE)
    lib().swbw_rescue_tasks(SEED_BASE + 3 + 1000 * rank + 1, ref.codes.ctypes.data, ref.n, n, 150, 700, 400.0,
                            50.0, 0.02, 0.10, 19, bases.ctypes.data, tasks.ctypes.data)
    return RescueWorkload(ref, bases, tasks, f"config3: {n} mate-rescue local SW, 150 bp vs 700 bp")


@dataclass
class ChainWorkload:
    ref: Reference
    bases: np.ndarray          # reads, read_len bytes each
    seeds: np.ndarray          # SEED_DTYPE, BWT coordinates [0, 2 * ref.n)
    chains: np.ndarray         # CHAIN_DTYPE, one chain per read
    read_len: int
    name: str = ""


def chains(ref: Reference, seed: int, n_reads: int, read_len: int = 150, *, sub=0.01, indel=0.001, n_rate=0.005,
           min_seed=19, max_seeds=6, a=1, spurious_frac=0.1) -> ChainWorkload:
    """One seed chain per read for ExtensionAligner.extend: reads from either
    strand with errors; seeds = the clean runs of >= min_seed bases at the
    true location (score len * a), plus an offset copy of one of them in a
    fraction spurious_frac of chains."""
    bases = np.empty(n_reads * read_len, np.uint8)
    seeds = np.empty(n_reads * (max_seeds + 1), SEED_DTYPE)
    ch = np.empty(n_reads, CHAIN_DTYPE)
    ns = lib().swbw_chains(seed, ref.codes.ctypes.data, ref.n, n_reads, read_len, sub, indel, n_rate, min_seed,
                           max_seeds, a, spurious_frac, bases.ctypes.data, seeds.ctypes.data, ch.ctypes.data)
    return ChainWorkload(ref, bases, seeds[:ns].copy(), ch, read_len)


def config5(rank: int = 0, n_reads: int = 1_000_000, ref_len: int = 100_000_000) -> ChainWorkload:
    """ExtensionAligner.extend over 1M seed chains of 150 bp reads (both
    strands, config-1 error rates) off a 100 Mbp reference."""
    ref = reference(SEED_BASE + 5 + 1000 * rank, ref_len)
    wl = chains(ref, SEED_BASE + 5 + 1000 * rank + 1, n_reads, 150)
    wl.name = f"config5: {n_reads} seed chains of 150 bp reads ({len(wl.seeds)} seeds), {ref_len // 10**6} Mbp reference"
    return wl


@dataclass
class RescueJobs:
    ref: Reference
    bases: np.ndarray              # mates, mate_len bytes each
    jobs: np.ndarray               # RESCUE_JOB_DTYPE
    templates: np.ndarray          # ANCHOR_DTYPE
    mate_regions: np.ndarray       # ANCHOR_DTYPE
    stats: np.ndarray              # ORIENTATION_DTYPE[4] (FF, FR, RF, RR)
    primary: int
    contig_offsets: np.ndarray     # int64, ascending
    contig_lengths: np.ndarray     # int32
    name: str = ""


def rescue_jobs(ref: Reference, seed: int, n: int, mate_len: int = 150, *, n_contigs: int = 1, ins_mean=400.0,
                ins_sd=50.0, sub=0.02, no_hit_frac=0.1, hit_frac=0.2, more_orientations=False) -> RescueJobs:
    """MateRescue.rescue jobs: FR pairs (insert N(ins_mean, ins_sd)), 1-3
    template regions per mate (the first the true anchor), existing mate
    regions that already satisfy FR in a fraction hit_frac, random mates in a
    fraction no_hit_frac, the genome cut into n_contigs contigs.  Stats: FR
    with proper range mean +- 4 sd (InsertSizeEstimator.swift:209-210); with
    more_orientations also FF and RR, with the same range."""
    rng = np.random.default_rng(seed)
    cuts = np.sort(rng.choice(np.arange(1, ref.n), n_contigs - 1, replace=False)) if n_contigs > 1 else np.array([], np.int64)
    offs = np.concatenate([[0], cuts]).astype(np.int64)
    lens = np.diff(np.concatenate([offs, [ref.n]])).astype(np.int32)
    bases = np.empty(n * mate_len, np.uint8)
    jobs = np.empty(n, RESCUE_JOB_DTYPE)
    tmpl = np.empty(3 * n, ANCHOR_DTYPE)
    mreg = np.empty(3 * n, ANCHOR_DTYPE)
    packed = lib().swbw_rescue_jobs(seed, ref.codes.ctypes.data, ref.n, offs.ctypes.data, len(offs), n, mate_len,
                                    ins_mean, ins_sd, sub, no_hit_frac, hit_frac, bases.ctypes.data,
                                    jobs.ctypes.data, tmpl.ctypes.data, mreg.ctypes.data)
    nt, nm = int(packed >> 32), int(packed & 0xFFFFFFFF)
    stats = np.zeros(4, ORIENTATION_DTYPE)
    stats["failed"] = 1
    lo, hi = max(1, int(ins_mean - 4 * ins_sd + 0.5)), int(ins_mean + 4 * ins_sd + 0.5)
    stats[1] = (0, 0, lo, hi)
    if more_orientations:
        stats[0] = (0, 0, lo, hi)
        stats[3] = (0, 0, lo, hi)
    return RescueJobs(ref, bases, jobs, tmpl[:nt].copy(), mreg[:nm].copy(), stats, 1, offs, lens)


def config3_jobs(rank: int = 0, n: int = 1_000_000, ref_len: int = 100_000_000) -> RescueJobs:
    """MateRescue.rescue over 1M 150 bp mates (config-3 insert 400 +- 50, 2%
    substitutions, 10% random mates) against a 100 Mbp reference in 24 contigs."""
    ref = reference(SEED_BASE + 3 + 1000 * rank, ref_len)
    wl = rescue_jobs(ref, SEED_BASE + 3 + 1000 * rank + 7, n, 150, n_contigs=24)
    wl.name = f"config3 rescue driver: {n} mates, {len(wl.templates)} template regions, {ref_len // 10**6} Mbp reference, 24 contigs"
    return wl


# ------------------------------------------------------------ FM index (seeding)
@dataclass
class FMIndexData:
    """An FM index in the layout the reference loads (BWT.swift, CheckpointOCC.swift)."""
    cp: np.ndarray             # BWT_CHECKPOINT_DTYPE, (length >> 6) + 1 entries
    count: np.ndarray          # int64[5]: 1 + the characters below each base; count[4] = length
    length: int
    sentinel: int


def fm_index(codes: np.ndarray, device: str = "cuda") -> FMIndexData:
    """FM index of a synthetic forward strand (codes 0-3): the text is the
    strand, its reverse complement and '$'; the suffix array comes from
    prefix doubling with torch sorts on `device` (ranks of 27-base prefixes
    packed in base 5, then doubled until every suffix has its own rank), the
    BWT is text[SA-1], and one checkpoint per 64 BWT positions holds the
    base counts before it and one bitstring per base (bit 63-y for position
    y).  Workload generation for the seeding tests and benchmark, not part of
    the seeding path: the same arrays as the oracle's builder, faster."""
    import torch
    from .abi import BWT_CHECKPOINT_DTYPE
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    n = int(codes.size)
    N = 2 * n + 1
    T = np.empty(N, np.int64)
    T[:n] = codes.astype(np.int64) + 1
    T[n:2 * n] = 4 - codes[::-1].astype(np.int64)          # complement c -> 3 - c, then + 1
    T[2 * n] = 0                                            # '$'
    dev = torch.device(device)
    t = torch.from_numpy(T).to(dev)
    K = 27                                                  # 5**27 < 2**63
    key = torch.zeros(N, dtype=torch.int64, device=dev)
    for j in range(K):
        nxt = torch.zeros(N, dtype=torch.int64, device=dev)
        if j < N:
            nxt[: N - j] = t[j:]
        key = key * 5 + nxt
    del t

    def ranks_of(sorted_keys, order):
        r = torch.empty(N, dtype=torch.int64, device=dev)
        new = torch.ones(N, dtype=torch.int64, device=dev)
        new[0] = 0
        new[1:] = (sorted_keys[1:] != sorted_keys[:-1]).to(torch.int64)
        r[order] = torch.cumsum(new, 0)
        return r

    sk, sa = torch.sort(key)
    rank = ranks_of(sk, sa)
    h = K
    while int(rank.max()) < N - 1:
        second = torch.zeros(N, dtype=torch.int64, device=dev)
        if h < N:
            second[: N - h] = rank[h:] + 1
        key = rank * (N + 1) + second
        sk, sa = torch.sort(key)
        rank = ranks_of(sk, sa)
        h *= 2
    del key, sk, rank
    tt = torch.from_numpy(T).to(dev)
    prev = torch.where(sa > 0, tt[(sa - 1).clamp(min=0)], torch.zeros_like(sa))   # 0 = '$' (the sentinel)
    sentinel = int(torch.nonzero(sa == 0)[0, 0])
    n_cp = (N >> 6) + 1
    pad = torch.zeros(n_cp * 64, dtype=torch.int64, device=dev)
    pad[:N] = prev
    blk = pad.view(n_cp, 64)
    cp = np.zeros(n_cp, BWT_CHECKPOINT_DTYPE)
    shift = (63 - torch.arange(64, device=dev, dtype=torch.int64))
    for c in range(4):
        m = (blk == c + 1).to(torch.int64)
        cnt = m.sum(1)
        before = torch.cumsum(cnt, 0) - cnt
        cp["counts"][:, c] = before.cpu().numpy()
        hi = (m[:, :32] << (shift[:32] - 32)).sum(1).cpu().numpy().astype(np.uint64)   # bits 63..32
        lo = (m[:, 32:] << shift[32:]).sum(1).cpu().numpy().astype(np.uint64)          # bits 31..0
        cp["bits"][:, c] = (hi << np.uint64(32)) | lo
    tot = np.array([int(np.sum(codes == c)) + int(np.sum(codes == 3 - c)) for c in range(4)], np.int64)
    count = np.zeros(5, np.int64)
    count[0] = 1
    count[1:] = 1 + np.cumsum(tot)
    return FMIndexData(cp, count, N, sentinel)
