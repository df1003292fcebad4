"""TEST INFRASTRUCTURE, NOT PRODUCT CODE.

ctypes wrapper of oracle/build/libswb_oracle.so, the C++ restatement of the
reference's Swift CPU Alignment functions (see oracle/swb_oracle.cpp for the
file:line each function follows).  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from swiftbwa_b200.abi import (ExtResult, LocalResult, Scoring, ptr, BWT_CHECKPOINT_DTYPE, CIGAR_RESULT_DTYPE,
                               EXT_RESULT_DTYPE, GLOBAL_RESULT_DTYPE, LOCAL_RESULT_DTYPE, SMEM_DTYPE)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "libswb_oracle.so")


class Region(C.Structure):
    _fields_ = [("rb", C.c_int64), ("re", C.c_int64), ("qb", C.c_int32), ("qe", C.c_int32),
                ("rid", C.c_int32), ("score", C.c_int32), ("true_score", C.c_int32),
                ("sub", C.c_int32), ("sub_n", C.c_int32), ("w", C.c_int32),
                ("seed_cov", C.c_int32), ("seed_len0", C.c_int32)]


class Seed(C.Structure):
    _fields_ = [("rbeg", C.c_int64), ("qbeg", C.c_int32), ("len", C.c_int32),
                ("score", C.c_int32), ("pad", C.c_int32)]


def build() -> str:
    """Compile the oracle (make -C oracle); returns the library path."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        P, u8p = C.POINTER, C.POINTER(C.c_uint8)
        L.orc_banded_sw_scalar.argtypes = [u8p, C.c_int32, u8p, C.c_int32, P(Scoring), C.c_int32,
                                           C.c_int32, C.c_int32, P(ExtResult), P(C.c_uint64)]
        L.orc_banded_sw16.argtypes = [u8p, C.c_int32, u8p, C.c_int32, P(Scoring), C.c_int32,
                                      C.c_int32, P(ExtResult)]
        L.orc_banded_sw8.argtypes = L.orc_banded_sw16.argtypes
        L.orc_banded_sw8.restype = C.c_int
        L.orc_global_align.argtypes = [u8p, C.c_int32, u8p, C.c_int32, P(Scoring), C.c_int32,
                                       P(C.c_int32), P(C.c_uint32), P(C.c_int32), P(C.c_uint64)]
        L.orc_compute_nm.argtypes = [P(C.c_uint32), C.c_int32, u8p, C.c_int32, u8p, C.c_int32]
        L.orc_compute_nm.restype = C.c_int32
        L.orc_infer_band_width.argtypes = [C.c_int32, C.c_int32, C.c_int32, P(Scoring)]
        L.orc_infer_band_width.restype = C.c_int32
        L.orc_cigar_generate.argtypes = [u8p, C.c_int32, u8p, C.c_int32, C.c_int32, C.c_int32,
                                         C.c_int32, C.c_int32, C.c_int32, C.c_int32, P(Scoring),
                                         C.c_int64, P(C.c_uint32), P(C.c_int32), P(C.c_int32),
                                         C.c_char_p, C.c_int32, P(C.c_int32), P(C.c_int64),
                                         P(C.c_uint64), P(C.c_int32)]
        L.orc_cigar_postprocess.argtypes = [P(C.c_uint32), C.c_int32, C.c_int32, u8p, C.c_int32,
                                            u8p, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                                            C.c_int32, C.c_int64, P(C.c_uint32), P(C.c_int32),
                                            P(C.c_int32), C.c_char_p, C.c_int32, P(C.c_int32),
                                            P(C.c_int64)]
        L.orc_local_align.argtypes = [u8p, C.c_int32, u8p, C.c_int32, P(Scoring), C.c_int32,
                                      P(LocalResult), P(C.c_uint64), P(C.c_int32)]
        L.orc_local_align.restype = C.c_int
        L.orc_pac_base.argtypes = [u8p, C.c_int64]
        L.orc_pac_base.restype = C.c_uint8
        L.orc_get_reference.argtypes = [u8p, C.c_int64, C.c_int64, C.c_int32, u8p]
        L.orc_get_reference.restype = C.c_int32
        L.orc_extend.argtypes = [P(Seed), C.c_int32, C.c_int32, u8p, C.c_int32, u8p, C.c_int64,
                                 C.c_int32, P(Scoring), P(Region), C.c_int32, P(C.c_uint64),
                                 P(C.c_uint64)]
        L.orc_extend.restype = C.c_int
        for name in ("orc_ext_batch", "orc_global_batch", "orc_local_batch"):
            getattr(L, name).restype = C.c_int
        L.orc_ext_batch.argtypes = [P(Scoring), u8p, u8p, C.c_uint64, C.c_void_p, C.c_size_t,
                                    C.c_void_p, C.c_int, P(C.c_uint64)]
        L.orc_global_batch.argtypes = [P(Scoring), u8p, u8p, C.c_uint64, C.c_void_p, C.c_size_t,
                                       C.c_void_p, P(C.c_uint32), C.c_size_t, C.c_int,
                                       P(C.c_uint64)]
        L.orc_local_batch.argtypes = L.orc_ext_batch.argtypes
        L.orc_cigar_batch.argtypes = [P(Scoring), u8p, u8p, C.c_void_p, C.c_size_t, C.c_void_p, P(C.c_uint32),
                                      C.c_size_t, C.c_char_p, C.c_size_t, C.c_int, P(C.c_uint64)]
        L.orc_cigar_batch.restype = C.c_int
        L.orc_bwt_build.argtypes = [u8p, C.c_int64, C.c_void_p, C.c_int64, P(C.c_int64), P(C.c_int64),
                                    P(C.c_int64), C.c_int]
        L.orc_bwt_build.restype = C.c_int
        L.orc_smem_batch.argtypes = [C.c_void_p, P(C.c_int64), C.c_int64, C.c_int64, u8p, C.c_void_p, C.c_void_p,
                                     C.c_size_t, C.c_int32, C.c_int64, C.c_int32, C.c_int32, C.c_uint32, C.c_void_p,
                                     C.c_void_p, C.c_int]
        L.orc_smem_batch.restype = C.c_int64
        L.orc_extend_batch.argtypes = [P(Scoring), u8p, u8p, C.c_int64, C.c_void_p, C.c_void_p, C.c_size_t,
                                       C.c_void_p, P(C.c_uint32), C.c_int, P(C.c_uint64)]
        L.orc_extend_batch.restype = C.c_int
        L.orc_mate_rescue_batch.argtypes = [P(Scoring), u8p, u8p, C.c_int64, C.c_void_p, C.c_size_t, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_size_t,
                                            C.c_void_p, P(C.c_uint32), P(C.c_uint32), C.c_int, P(C.c_uint64)]
        L.orc_mate_rescue_batch.restype = C.c_int
        _lib = L
    return _lib


def _u8(seq) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(seq, dtype=np.uint8))
    return a if a.size else np.zeros(1, np.uint8)


def banded_sw_scalar(q, t, sc: Scoring, w, h0, end_bonus=0):
    """BandedSWScalar.align -> (score, qle, tle, gtle, gscore, max_off), cells."""
    qa, ta = _u8(q), _u8(t)
    out, cells = ExtResult(), C.c_uint64()
    lib().orc_banded_sw_scalar(ptr(qa), len(q), ptr(ta), len(t), C.byref(sc), w, h0, end_bonus,
                               C.byref(out), C.byref(cells))
    return out.as_tuple(), cells.value


def banded_sw16(q, t, sc: Scoring, w, h0):
    qa, ta = _u8(q), _u8(t)
    out = ExtResult()
    lib().orc_banded_sw16(ptr(qa), len(q), ptr(ta), len(t), C.byref(sc), w, h0, C.byref(out))
    return out.as_tuple()


def banded_sw8(q, t, sc: Scoring, w, h0):
    """BandedSW8.align; None for nil."""
    qa, ta = _u8(q), _u8(t)
    out = ExtResult()
    ok = lib().orc_banded_sw8(ptr(qa), len(q), ptr(ta), len(t), C.byref(sc), w, h0, C.byref(out))
    return out.as_tuple() if ok else None


def global_align(q, t, sc: Scoring, w):
    """GlobalAligner.align -> (score, [packed ops]), cells."""
    qa, ta = _u8(q), _u8(t)
    cap = len(q) + len(t) + 1
    cig = (C.c_uint32 * cap)()
    n = C.c_int32(cap)
    score, cells = C.c_int32(), C.c_uint64()
    rc = lib().orc_global_align(ptr(qa), len(q), ptr(ta), len(t), C.byref(sc), w, C.byref(score),
                                cig, C.byref(n), C.byref(cells))
    if rc != 0:
        raise ValueError("global_align: undefined input (w < 1 with equal lengths)")
    return (score.value, list(cig[: n.value])), cells.value


def compute_nm(cigar, q, t):
    qa, ta = _u8(q), _u8(t)
    arr = (C.c_uint32 * max(len(cigar), 1))(*cigar)
    return lib().orc_compute_nm(arr, len(cigar), ptr(qa), len(q), ptr(ta), len(t))


def infer_band_width(qlen, rlen, score, sc: Scoring):
    return lib().orc_infer_band_width(qlen, rlen, score, C.byref(sc))


def cigar_generate(qseg, rseg, qb, qe, read_len, is_rev, true_score, initial_w, sc: Scoring,
                   ref_pos):
    """CIGARGenerator.generate -> dict(cigar, nm, md, score, pos, cells, used_dp)."""
    qa, ra = _u8(qseg), _u8(rseg)
    cap = len(qseg) + len(rseg) + 4
    cig = (C.c_uint32 * cap)()
    n = C.c_int32(cap)
    nm, score, used = C.c_int32(), C.c_int32(), C.c_int32()
    pos, cells = C.c_int64(), C.c_uint64()
    md = C.create_string_buffer(8 * cap + 16)
    rc = lib().orc_cigar_generate(ptr(qa), len(qseg), ptr(ra), len(rseg), qb, qe, read_len,
                                  int(is_rev), true_score, initial_w, C.byref(sc), ref_pos, cig,
                                  C.byref(n), C.byref(nm), md, len(md), C.byref(score),
                                  C.byref(pos), C.byref(cells), C.byref(used))
    if rc != 0:
        raise ValueError("cigar_generate failed")
    return dict(cigar=list(cig[: n.value]), nm=nm.value, md=md.value.decode(), score=score.value,
                pos=pos.value, cells=cells.value, used_dp=bool(used.value))


def cigar_postprocess(raw, score, qseg, rseg, qb, qe, read_len, is_rev, ref_pos):
    qa, ra = _u8(qseg), _u8(rseg)
    cap = len(raw) + 4
    rawa = (C.c_uint32 * max(len(raw), 1))(*raw)
    cig = (C.c_uint32 * cap)()
    n = C.c_int32(cap)
    nm, sc_out, pos = C.c_int32(), C.c_int32(), C.c_int64()
    md = C.create_string_buffer(8 * (len(qseg) + len(rseg)) + 16)
    rc = lib().orc_cigar_postprocess(rawa, len(raw), score, ptr(qa), len(qseg), ptr(ra), len(rseg),
                                     qb, qe, read_len, int(is_rev), ref_pos, cig, C.byref(n),
                                     C.byref(nm), md, len(md), C.byref(sc_out), C.byref(pos))
    if rc != 0:
        raise ValueError("cigar_postprocess failed")
    return dict(cigar=list(cig[: n.value]), nm=nm.value, md=md.value.decode(),
                score=sc_out.value, pos=pos.value)


def local_align(q, t, sc: Scoring, min_sub_score=0):
    """LocalSWAligner.align -> (score, qb, qe, tb, te, score2) or None, cells, path."""
    qa, ta = _u8(q), _u8(t)
    out, cells, path = LocalResult(), C.c_uint64(), C.c_int32()
    ok = lib().orc_local_align(ptr(qa), len(q), ptr(ta), len(t), C.byref(sc), min_sub_score,
                               C.byref(out), C.byref(cells), C.byref(path))
    return (out.as_tuple() if ok else None), cells.value, path.value


def get_reference(pac: np.ndarray, genome_len: int, pos: int, length: int) -> np.ndarray:
    buf = np.zeros(max(length, 1), np.uint8)
    n = lib().orc_get_reference(ptr(pac), genome_len, pos, length, ptr(buf))
    return buf[:n].copy()


def extend(seeds, rid, read, ref, sc: Scoring, ref_mode=0, genome_len=None):
    """ExtensionAligner.extend.  seeds: [(rbeg, qbeg, len, score)]."""
    sa = (Seed * max(len(seeds), 1))(*[Seed(r, q, l, s, 0) for (r, q, l, s) in seeds])
    ra, fa = _u8(read), _u8(ref)
    cap = max(len(seeds), 1)
    out = (Region * cap)()
    calls, cells = C.c_uint64(), C.c_uint64()
    ref_len = len(ref) if ref_mode == 0 else genome_len
    n = lib().orc_extend(sa, len(seeds), rid, ptr(ra), len(read), ptr(fa), ref_len, ref_mode,
                         C.byref(sc), out, cap, C.byref(calls), C.byref(cells))
    if n < 0:
        raise ValueError("extend failed")
    return [dict((f, getattr(out[i], f)) for f, _ in Region._fields_) for i in range(n)], \
        calls.value, cells.value


def ext_batch(sc: Scoring, bases: np.ndarray, tasks: np.ndarray, pac=None, ref_bases=0,
              n_threads: int = 1):
    """Batch BandedSWScalar over EXT_TASK_DTYPE tasks -> (results array, cells)."""
    out = np.zeros(len(tasks), EXT_RESULT_DTYPE)
    cells = C.c_uint64()
    rc = lib().orc_ext_batch(C.byref(sc), ptr(_u8(bases) if bases is None or bases.size == 0 else bases),
                             ptr(pac), ref_bases, tasks.ctypes.data, len(tasks), out.ctypes.data,
                             n_threads, C.byref(cells))
    assert rc == 0
    return out, cells.value


def global_batch(sc: Scoring, bases: np.ndarray, tasks: np.ndarray, pac=None, ref_bases=0,
                 n_threads: int = 1):
    cap = int((tasks["qlen"].astype(np.int64) + tasks["tlen"]).sum()) + 1
    res = np.zeros(len(tasks), GLOBAL_RESULT_DTYPE)
    cig = np.zeros(cap, np.uint32)
    cells = C.c_uint64()
    rc = lib().orc_global_batch(C.byref(sc), ptr(bases), ptr(pac), ref_bases, tasks.ctypes.data,
                                len(tasks), res.ctypes.data, ptr(cig, C.c_uint32), cap, n_threads,
                                C.byref(cells))
    if rc != 0:
        raise ValueError("global_batch failed")
    return res, cig, cells.value


def cigar_batch(sc: Scoring, bases: np.ndarray, tasks: np.ndarray, pac=None, n_threads: int = 1):
    """CIGARGenerator.generate over CIGAR_TASK_DTYPE tasks, host threads ->
    (CIGAR_RESULT_DTYPE results, CIGAR words, MD bytes, cells); task k's CIGAR
    is words[cigar_off : cigar_off + n_cigar], its MD md[md_off : md_off + md_len]."""
    qr = tasks["qlen"].astype(np.int64).clip(0) + tasks["rlen"].astype(np.int64).clip(0)
    ccap = int((qr + 2).sum()) + 1
    mcap = int((6 * qr + 8).sum()) + 1
    res = np.zeros(len(tasks), CIGAR_RESULT_DTYPE)
    cig = np.zeros(ccap, np.uint32)
    md = C.create_string_buffer(mcap)
    cells = C.c_uint64()
    rc = lib().orc_cigar_batch(C.byref(sc), ptr(bases), ptr(pac), tasks.ctypes.data, len(tasks), res.ctypes.data,
                               ptr(cig, C.c_uint32), ccap, md, mcap, n_threads, C.byref(cells))
    if rc != 0:
        raise ValueError("cigar_batch failed")
    return res, cig, np.frombuffer(md.raw, np.uint8), cells.value


class FMIndex:
    """The FM index of a forward strand as the reference loads it (BWT.swift):
    checkpoints, count[5], length, sentinel."""

    def __init__(self, cp, count, length, sentinel):
        self.cp, self.count, self.length, self.sentinel = cp, count, int(length), int(sentinel)


def bwt_build(codes: np.ndarray) -> FMIndex:
    """FM index of `codes` (0-3) and its reverse complement, with '$' (test infrastructure)."""
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    n = codes.size
    n_cp = ((2 * n + 1) >> 6) + 1
    cp = np.zeros(n_cp, BWT_CHECKPOINT_DTYPE)
    count = np.zeros(5, np.int64)
    length, sentinel = C.c_int64(), C.c_int64()
    rc = lib().orc_bwt_build(ptr(codes), n, cp.ctypes.data, n_cp, count.ctypes.data_as(C.POINTER(C.c_int64)),
                             C.byref(length), C.byref(sentinel), 1)
    if rc != 0:
        raise ValueError(f"bwt_build failed ({rc})")
    return FMIndex(cp, count, length.value, sentinel.value)


def split_len_of(min_seed_len: int, seed_split_ratio: float = 1.5) -> int:
    """Int(Float(minSeedLength) * seedSplitRatio + 0.499) in single precision
    (BWAMemAligner.swift:265): 28 for the defaults 19 and 1.5."""
    f = np.float32(min_seed_len) * np.float32(seed_split_ratio)
    return int(np.float32(f + np.float32(0.499)))


def smem_batch(idx: FMIndex, bases: np.ndarray, read_off: np.ndarray, read_len: np.ndarray, min_seed_len: int,
               min_intv: int = 1, cap: int = 64, n_threads: int = 1, split_len: int = 0, split_width: int = 10):
    """SMEMFinder.findAllSMEMs per read, then (split_len > 0) internalReseed ->
    (SMEM_DTYPE [n_reads * cap], n_out, reads over cap)."""
    read_off = np.ascontiguousarray(read_off, dtype=np.uint64)
    read_len = np.ascontiguousarray(read_len, dtype=np.int32)
    n = read_off.size
    out = np.zeros(max(n * cap, 1), SMEM_DTYPE)
    n_out = np.zeros(n, np.uint32)
    over = lib().orc_smem_batch(idx.cp.ctypes.data, idx.count.ctypes.data_as(C.POINTER(C.c_int64)), idx.length,
                                idx.sentinel, ptr(bases), read_off.ctypes.data, read_len.ctypes.data, n,
                                min_seed_len, min_intv, split_len, split_width, cap, out.ctypes.data,
                                n_out.ctypes.data, n_threads)
    return out, n_out, int(over)


def local_batch(sc: Scoring, bases: np.ndarray, tasks: np.ndarray, pac=None, ref_bases=0,
                n_threads: int = 1):
    out = np.zeros(len(tasks), LOCAL_RESULT_DTYPE)
    cells = C.c_uint64()
    rc = lib().orc_local_batch(C.byref(sc), ptr(bases), ptr(pac), ref_bases, tasks.ctypes.data,
                               len(tasks), out.ctypes.data, n_threads, C.byref(cells))
    assert rc == 0
    return out, cells.value


def extend_batch(sc: Scoring, bases: np.ndarray, pac: np.ndarray, genome_len: int, seeds: np.ndarray,
                 chains: np.ndarray, n_threads: int = 1):
    """ExtensionAligner.extend (FMIndex.getReference targets) for every chain
    -> (regions array laid out like swb_extend_chains' output, counts, cells)."""
    from swiftbwa_b200.abi import REGION_DTYPE
    out = np.zeros(max(len(seeds), 1), REGION_DTYPE)
    counts = np.zeros(max(len(chains), 1), np.uint32)
    cells = C.c_uint64()
    rc = lib().orc_extend_batch(C.byref(sc), ptr(bases), ptr(pac), genome_len, seeds.ctypes.data,
                                chains.ctypes.data, len(chains), out.ctypes.data, ptr(counts, C.c_uint32),
                                n_threads, C.byref(cells))
    if rc != 0:
        raise ValueError("extend_batch failed")
    return out, counts[:len(chains)], cells.value


def mate_rescue_batch(sc: Scoring, bases: np.ndarray, pac: np.ndarray, genome_len: int, jobs: np.ndarray,
                      templates: np.ndarray, mate_regions: np.ndarray, stats: np.ndarray, primary: int,
                      contig_offsets: np.ndarray, contig_lengths: np.ndarray, n_threads: int = 1):
    """MateRescue.rescue for every job (RESCUE_JOB_DTYPE) -> (RESCUED_DTYPE array
    laid out like swb_mate_rescue's output, per-job counts, per-job local
    alignments run, cells)."""
    from swiftbwa_b200.abi import ANCHOR_DTYPE, RESCUED_DTYPE
    out = np.zeros(max(4 * len(templates), 1), RESCUED_DTYPE)
    n_out = np.zeros(max(len(jobs), 1), np.uint32)
    n_cand = np.zeros(max(len(jobs), 1), np.uint32)
    cells = C.c_uint64()
    mr = mate_regions if len(mate_regions) else np.zeros(1, ANCHOR_DTYPE)
    tp = templates if len(templates) else np.zeros(1, ANCHOR_DTYPE)
    offs = np.ascontiguousarray(contig_offsets, np.int64)
    lens = np.ascontiguousarray(contig_lengths, np.int32)
    bases = np.ascontiguousarray(bases, np.uint8) if bases.size else np.zeros(1, np.uint8)
    rc = lib().orc_mate_rescue_batch(C.byref(sc), ptr(bases), ptr(pac),
                                     genome_len, jobs.ctypes.data, len(jobs), tp.ctypes.data, mr.ctypes.data,
                                     stats.ctypes.data, primary, offs.ctypes.data, lens.ctypes.data, len(offs),
                                     out.ctypes.data, ptr(n_out, C.c_uint32), ptr(n_cand, C.c_uint32), n_threads,
                                     C.byref(cells))
    if rc != 0:
        raise ValueError("mate_rescue_batch failed")
    return out, n_out[:len(jobs)], n_cand[:len(jobs)], cells.value
