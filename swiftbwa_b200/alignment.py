"""Host-side mirror of swiftbwa's Alignment API over libswb_cuda.so.

Same names, argument meaning and nil behaviour as the reference's Swift
functions, so a caller (or a parity test) reads like the reference's own
code; every call goes through the C ABI (include/swb_cuda.h) to the sm_100a
kernels.  There is no CPU fallback: if the library or a GPU is missing the
calls raise.

    BandedSWScalar.align(query, target, scoring, w, h0, end_bonus) -> SWResult
        Sources/Alignment/BandedSWScalar.swift:21-28
    GlobalAligner.align(query, target, scoring, w) -> GlobalAlignResult
        Sources/Alignment/GlobalAligner.swift:19-25
    LocalSWAligner.align(query, target, scoring, min_sub_score) -> LocalSWResult | None
        Sources/Alignment/LocalSWAligner.swift:42-45
and the batch dispatchers that replace the Metal ones
(Sources/MetalSW/BandedSWDispatcher.swift:48,107, GlobalSWDispatcher.swift:40,
LocalSWDispatcher.swift:31).
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import abi
from .abi import (BWT_CHECKPOINT_DTYPE, EXT_RESULT_DTYPE, EXT_TASK_DTYPE, GLOBAL_RESULT_DTYPE, GLOBAL_TASK_DTYPE,
                  LOCAL_RESULT_DTYPE, LOCAL_TASK_DTYPE, SMEM_DTYPE, ExtResult, LocalResult, Scoring, ptr)


class SWBError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = abi.load_library()
        msg = lib.swb_strerror(status).decode()
        detail = lib.swb_last_error_message().decode()
        super().__init__(f"{where}: {msg} ({status}){': ' + detail if detail else ''}")
        self.status = status


def _check(rc: int, where: str):
    if rc != abi.SWB_OK:
        raise SWBError(rc, where)


@dataclass(frozen=True)
class SWResult:
    """Sources/BWACore/SWResult.swift:2-24."""
    score: int = 0
    queryEnd: int = 0
    targetEnd: int = 0
    globalTargetEnd: int = 0
    globalScore: int = 0
    maxOff: int = 0

    def as_tuple(self):
        return (self.score, self.queryEnd, self.targetEnd, self.globalTargetEnd,
                self.globalScore, self.maxOff)


@dataclass(frozen=True)
class GlobalAlignResult:
    """Sources/Alignment/GlobalAlignResult.swift:2-14."""
    score: int = 0
    cigar: tuple = ()
    nm: int = 0


@dataclass(frozen=True)
class LocalSWResult:
    """Sources/Alignment/LocalSWAligner.swift:4-23."""
    score: int
    queryBegin: int
    queryEnd: int
    targetBegin: int
    targetEnd: int
    score2: int = 0

    def as_tuple(self):
        return (self.score, self.queryBegin, self.queryEnd, self.targetBegin, self.targetEnd,
                self.score2)


def _u8(seq) -> np.ndarray:
    a = np.ascontiguousarray(np.asarray(seq, dtype=np.uint8))
    return a


class Engine:
    """One library context on one GPU (replaces MetalSWEngine.shared,
    Sources/MetalSW/MetalSWEngine.swift:8-17)."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0):
        self.lib = abi.load_library()
        h = C.c_void_p()
        _check(self.lib.swb_init(device, mem_budget_bytes, C.byref(h)), "swb_init")
        self.h = h
        self.device = device

    def close(self):
        if self.h:
            self.lib.swb_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- setup
    def upload_reference(self, pac: np.ndarray, n_bases: int):
        pac = np.ascontiguousarray(pac, dtype=np.uint8)
        _check(self.lib.swb_upload_reference(self.h, ptr(pac), n_bases), "swb_upload_reference")

    # ------------------------------------------------------------- batches
    def ext_batch(self, sc: Scoring, bases: np.ndarray, tasks: np.ndarray,
                  out: Optional[np.ndarray] = None) -> np.ndarray:
        assert tasks.dtype == EXT_TASK_DTYPE
        if out is None:
            out = np.zeros(len(tasks), EXT_RESULT_DTYPE)
        assert out.dtype == EXT_RESULT_DTYPE and len(out) >= len(tasks)
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        _check(self.lib.swb_ext_batch(self.h, C.byref(sc), ptr(bases), bases.size,
                                      tasks.ctypes.data, len(tasks), out.ctypes.data),
               "swb_ext_batch")
        return out

    def global_batch(self, sc: Scoring, bases: np.ndarray, tasks: np.ndarray):
        assert tasks.dtype == GLOBAL_TASK_DTYPE
        cap = int((tasks["qlen"].astype(np.int64) + tasks["tlen"]).sum()) + 1
        res = np.zeros(len(tasks), GLOBAL_RESULT_DTYPE)
        cig = np.zeros(cap, np.uint32)
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        _check(self.lib.swb_global_batch(self.h, C.byref(sc), ptr(bases), bases.size,
                                         tasks.ctypes.data, len(tasks), res.ctypes.data,
                                         ptr(cig, C.c_uint32), cap), "swb_global_batch")
        return res, cig

    def local_batch(self, sc: Scoring, bases: np.ndarray, tasks: np.ndarray,
                    out: Optional[np.ndarray] = None) -> np.ndarray:
        assert tasks.dtype == LOCAL_TASK_DTYPE
        if out is None:
            out = np.zeros(len(tasks), LOCAL_RESULT_DTYPE)
        assert out.dtype == LOCAL_RESULT_DTYPE and len(out) >= len(tasks)
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        _check(self.lib.swb_local_batch(self.h, C.byref(sc), ptr(bases), bases.size,
                                        tasks.ctypes.data, len(tasks), out.ctypes.data),
               "swb_local_batch")
        return out

    @staticmethod
    def cigar_caps(tasks: np.ndarray):
        """(cigar_cap, md_cap) that swb_cigar_batch requires for `tasks`:
        sum of (qlen + rlen + 2) words and of (6*(qlen + rlen) + 8) bytes."""
        n = len(tasks)
        s = int(tasks["qlen"].sum(dtype=np.int64)) + int(tasks["rlen"].sum(dtype=np.int64))
        return s + 2 * n + 1, 6 * s + 8 * n + 1

    def cigar_batch_raw(self, sc: Scoring, bases: np.ndarray, tasks: np.ndarray, out=None):
        """CIGARGenerator.generate over CIGAR_TASK_DTYPE tasks -> (CIGAR_RESULT_DTYPE
        array, packed CIGAR words, MD bytes); task k's CIGAR is
        cigar[cigar_off : cigar_off + n_cigar], its MD md[md_off : md_off + md_len].
        out: optional (results, cigar words, MD bytes) arrays to write into, at
        least len(tasks) results and cigar_caps(tasks) long (in pinned memory
        the device writes them directly)."""
        assert tasks.dtype == abi.CIGAR_TASK_DTYPE
        if out is None:
            ccap, mcap = self.cigar_caps(tasks)
            res = np.zeros(len(tasks), abi.CIGAR_RESULT_DTYPE)
            cig = np.empty(ccap, np.uint32)
            md = np.empty(mcap, np.uint8)
        else:
            res, cig, md = out
            assert res.dtype == abi.CIGAR_RESULT_DTYPE and len(res) >= len(tasks)
            assert cig.dtype == np.uint32 and md.dtype == np.uint8
            ccap, mcap = cig.size, md.size
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        if bases.size == 0:
            bases = np.zeros(1, np.uint8)
        _check(self.lib.swb_cigar_batch(self.h, C.byref(sc), ptr(bases), bases.size, tasks.ctypes.data,
                                        len(tasks), res.ctypes.data, ptr(cig, C.c_uint32), ccap,
                                        md.ctypes.data_as(C.c_char_p), mcap), "swb_cigar_batch")
        return res, cig, md

    def cigar_batch(self, sc: Scoring, bases: np.ndarray, tasks: np.ndarray):
        """CIGARGenerator.generate over CIGAR_TASK_DTYPE tasks -> list of dicts
        (cigar, nm, md, score, pos, used_dp)."""
        res, cig, md = self.cigar_batch_raw(sc, bases, tasks)
        raw = md.tobytes()
        out = []
        for r in res:
            o, n = int(r["cigar_off"]), int(r["n_cigar"])
            mo, ml = int(r["md_off"]), int(r["md_len"])
            out.append(dict(cigar=[int(x) for x in cig[o:o + n]], nm=int(r["nm"]), md=raw[mo:mo + ml].decode(),
                            score=int(r["score"]), pos=int(r["pos"]), used_dp=bool(r["used_dp"])))
        return out

    def cigar_generate(self, query_segment, ref_segment, qb, qe, read_len, is_reverse, true_score,
                       initial_w, scoring: Scoring, ref_pos) -> dict:
        """CIGARGenerator.generate (Sources/Alignment/CIGARGenerator.swift:30-42)."""
        q, r = _u8(query_segment), _u8(ref_segment)
        bases = np.concatenate([q, r]) if q.size + r.size else np.zeros(1, np.uint8)
        t = np.zeros(1, abi.CIGAR_TASK_DTYPE)
        t[0] = (0, q.size, q.size, r.size, qb, qe, read_len, int(bool(is_reverse)), true_score, initial_w,
                ref_pos, 0, 0)
        return self.cigar_batch(scoring, bases, t)[0]

    def extend_chains(self, sc: Scoring, bases: np.ndarray, seeds: np.ndarray, chains: np.ndarray,
                      genome_len: int, out=None):
        """ExtensionAligner.extend for every chain (SEED_DTYPE seeds, CHAIN_DTYPE
        chains) against the uploaded forward strand -> (REGION_DTYPE array,
        per-chain region counts, GPU rounds).  Chain c's regions are
        regions[seed_off : seed_off + counts[c]].  out: optional (regions,
        counts) arrays of at least len(seeds) and len(chains) entries to write
        into (in pinned memory the device writes them directly)."""
        assert seeds.dtype == abi.SEED_DTYPE and chains.dtype == abi.CHAIN_DTYPE
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        if bases.size == 0:
            bases = np.zeros(1, np.uint8)
        if out is None:
            out = np.zeros(max(len(seeds), 1), abi.REGION_DTYPE)
            counts = np.zeros(max(len(chains), 1), np.uint32)
        else:
            out, counts = out
            assert out.dtype == abi.REGION_DTYPE and len(out) >= len(seeds)
            assert counts.dtype == np.uint32 and len(counts) >= len(chains)
        rounds = C.c_uint32()
        _check(self.lib.swb_extend_chains(self.h, C.byref(sc), ptr(bases), bases.size, seeds.ctypes.data, len(seeds),
                                          chains.ctypes.data, len(chains), genome_len, out.ctypes.data,
                                          ptr(counts, C.c_uint32), C.byref(rounds)), "swb_extend_chains")
        return out, counts[:len(chains)], rounds.value

    def mate_rescue(self, sc: Scoring, bases: np.ndarray, jobs: np.ndarray, templates: np.ndarray,
                    mate_regions: np.ndarray, stats: np.ndarray, primary: int, contig_offsets: np.ndarray,
                    contig_lengths: np.ndarray, genome_len: int):
        """MateRescue.rescue for every job (RESCUE_JOB_DTYPE) against the uploaded
        forward strand -> (RESCUED_DTYPE array, per-job counts, per-job local
        alignments run).  Job j's regions are out[4*tmpl_off : 4*tmpl_off + counts[j]]."""
        assert jobs.dtype == abi.RESCUE_JOB_DTYPE and stats.dtype == abi.ORIENTATION_DTYPE and len(stats) == 4
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        if bases.size == 0:
            bases = np.zeros(1, np.uint8)
        tp = templates if len(templates) else np.zeros(1, abi.ANCHOR_DTYPE)
        mr = mate_regions if len(mate_regions) else np.zeros(1, abi.ANCHOR_DTYPE)
        offs = np.ascontiguousarray(contig_offsets, np.int64)
        lens = np.ascontiguousarray(contig_lengths, np.int32)
        out = np.zeros(max(4 * len(templates), 1), abi.RESCUED_DTYPE)
        n_out = np.zeros(max(len(jobs), 1), np.uint32)
        n_cand = np.zeros(max(len(jobs), 1), np.uint32)
        _check(self.lib.swb_mate_rescue(self.h, C.byref(sc), ptr(bases), bases.size, jobs.ctypes.data, len(jobs),
                                        tp.ctypes.data, len(templates), mr.ctypes.data, len(mate_regions),
                                        stats.ctypes.data, primary, offs.ctypes.data, lens.ctypes.data, len(offs),
                                        genome_len, out.ctypes.data, ptr(n_out, C.c_uint32),
                                        ptr(n_cand, C.c_uint32)), "swb_mate_rescue")
        return out, n_out[:len(jobs)], n_cand[:len(jobs)]

    def last_batch_stats(self):
        ms, cells = C.c_double(), C.c_uint64()
        _check(self.lib.swb_last_batch_stats(self.h, C.byref(ms), C.byref(cells)), "stats")
        return ms.value, cells.value

    def kernel_launches(self) -> int:
        return int(self.lib.swb_kernel_launches(self.h))

    # ------------------------------------------------------------ profiling
    def profile(self, enable: bool = True):
        _check(self.lib.swb_profile(self.h, int(enable)), "swb_profile")

    def profile_reset(self):
        _check(self.lib.swb_profile_reset(self.h), "swb_profile_reset")

    def profile_read(self) -> dict:
        """{kernel name: (launches, total_ms, cells)} since the last reset."""
        cap = 64
        arr = (abi.KernelStat * cap)()
        n = C.c_int()
        _check(self.lib.swb_profile_read(self.h, arr, cap, C.byref(n)), "swb_profile_read")
        return {arr[k].name.decode(): (arr[k].launches, arr[k].total_ms, arr[k].cells)
                for k in range(min(n.value, cap))}

    def int_alu_peak(self) -> float:
        v = C.c_double()
        _check(self.lib.swb_int_alu_peak(self.h, C.byref(v)), "swb_int_alu_peak")
        return v.value

    def set_ext_bins(self, qmax) -> None:
        """Length classes of the extension bins (ascending query-length bounds)."""
        arr = (C.c_int32 * len(qmax))(*qmax)
        _check(self.lib.swb_set_ext_bins(self.h, arr, len(qmax)), "swb_set_ext_bins")

    def ext_bins(self) -> list:
        arr = (C.c_int32 * 16)()
        n = C.c_int()
        _check(self.lib.swb_get_ext_bins(self.h, arr, 16, C.byref(n)), "swb_get_ext_bins")
        return list(arr[: n.value])

    def tune_ext_bins(self, sc: Scoring, bases: np.ndarray, tasks: np.ndarray) -> dict:
        """Autotune the length classes on a sample batch; the context keeps
        the fastest.  -> {"bins", "ms", "default_ms"}."""
        assert tasks.dtype == EXT_TASK_DTYPE
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        tasks = np.ascontiguousarray(tasks)
        arr = (C.c_int32 * 16)()
        n = C.c_int()
        best, dflt = C.c_float(), C.c_float()
        _check(self.lib.swb_tune_ext_bins(self.h, C.byref(sc), ptr(bases), bases.size, tasks.ctypes.data, len(tasks),
                                          arr, 16, C.byref(n), C.byref(best), C.byref(dflt)), "swb_tune_ext_bins")
        return {"bins": list(arr[: n.value]), "ms": best.value, "default_ms": dflt.value}

    def int16x2_alu_peak(self) -> float:
        """Packed 16-bit (s16x2 DPX add+max) lane operations/s."""
        v = C.c_double()
        _check(self.lib.swb_int16x2_alu_peak(self.h, C.byref(v)), "swb_int16x2_alu_peak")
        return v.value

    def ext_batch_device(self, sc: Scoring, d_bases: int, d_tasks: int, n: int, d_out: int, stream: int = 0):
        """swb_ext_batch_device on device pointers (HBM-resident inputs)."""
        _check(self.lib.swb_ext_batch_device(self.h, C.byref(sc), C.c_void_p(d_bases), C.c_void_p(d_tasks), n,
                                             C.c_void_p(d_out), C.c_void_p(stream)), "swb_ext_batch_device")

    # ------------------------------------------------------- SMEM seeding
    def upload_bwt(self, cp: np.ndarray, count: np.ndarray, length: int, sentinel: int):
        """Keeps an FM index resident (BWT.swift's fields): checkpoints
        (BWT_CHECKPOINT_DTYPE), count[5], length, sentinel."""
        assert cp.dtype == BWT_CHECKPOINT_DTYPE
        cp = np.ascontiguousarray(cp)
        cnt = np.ascontiguousarray(count, dtype=np.int64)
        _check(self.lib.swb_upload_bwt(self.h, cp.ctypes.data, cp.size, cnt.ctypes.data_as(C.POINTER(C.c_int64)),
                                       int(length), int(sentinel)), "swb_upload_bwt")

    def smem_batch(self, bases: np.ndarray, read_off: np.ndarray, read_len: np.ndarray, min_seed_len: int,
                   min_intv: int = 1, cap_per_read: int = 64, split_len: int = 0, split_width: int = 10,
                   out_cap: Optional[int] = None, out=None):
        """SMEMFinder.findAllSMEMs per read on the resident FM index, then (with
        split_len > 0) BWAMemAligner.internalReseed -> (SMEM_DTYPE packed
        SMEMs, n_out, out_off); read r's SMEMs are out[out_off[r] : out_off[r] + n_out[r]].
        out: optional (SMEMs, n_out, out_off) arrays to write into (the SMEM
        array's length is the capacity; in pinned memory the device writes
        them directly)."""
        bases = np.ascontiguousarray(bases, dtype=np.uint8)
        read_off = np.ascontiguousarray(read_off, dtype=np.uint64)
        read_len = np.ascontiguousarray(read_len, dtype=np.int32)
        n = read_off.size
        if out is not None:
            sm, n_out, out_off = out
            assert sm.dtype == SMEM_DTYPE and n_out.dtype == np.uint32 and out_off.dtype == np.uint64
            assert len(n_out) >= max(n, 1) and len(out_off) >= max(n, 1)
            _check(self.lib.swb_smem_batch(self.h, ptr(bases), bases.size, read_off.ctypes.data, read_len.ctypes.data,
                                           n, int(min_seed_len), int(min_intv), int(split_len), int(split_width),
                                           int(cap_per_read), sm.ctypes.data, int(sm.size), n_out.ctypes.data,
                                           out_off.ctypes.data), "swb_smem_batch")
            return sm, n_out[:n], out_off[:n]
        grow = out_cap is None
        if grow:
            out_cap = int(read_len.astype(np.int64).clip(0).sum()) + 16   # usually enough; grown below if not
        n_out = np.zeros(max(n, 1), np.uint32)
        out_off = np.zeros(max(n, 1), np.uint64)
        while True:
            out = np.zeros(max(out_cap, 1), SMEM_DTYPE)
            rc = self.lib.swb_smem_batch(self.h, ptr(bases), bases.size, read_off.ctypes.data, read_len.ctypes.data,
                                         n, int(min_seed_len), int(min_intv), int(split_len), int(split_width),
                                         int(cap_per_read), out.ctypes.data, int(out_cap), n_out.ctypes.data,
                                         out_off.ctypes.data)
            total = int(out_off[n - 1]) + int(n_out[n - 1]) if n else 0
            if grow and rc == abi.SWB_ERR_TOO_LARGE and total > out_cap:
                out_cap = total
                continue
            _check(rc, "swb_smem_batch")
            return out, n_out[:n], out_off[:n]

    def ext_batch_plain_device(self, sc: Scoring, d_bases: int, d_tasks: int, n: int, d_out: int, stream: int = 0):
        """swb_ext_batch_plain_device: the plain one-launch-per-batch kernel (the
        dispatch shape of BandedSWDispatcher.dispatchBatch16), same results."""
        _check(self.lib.swb_ext_batch_plain_device(self.h, C.byref(sc), C.c_void_p(d_bases), C.c_void_p(d_tasks), n,
                                                   C.c_void_p(d_out), C.c_void_p(stream)),
               "swb_ext_batch_plain_device")

    # --------------------------------------------------- single-call forms
    def banded_sw_align(self, query, target, scoring: Scoring, w: int, h0: int,
                        end_bonus: int = 0) -> SWResult:
        q, t = _u8(query), _u8(target)
        out = ExtResult()
        _check(self.lib.swb_banded_sw_align(self.h, ptr(q), q.size, ptr(t), t.size, C.byref(scoring),
                                            w, h0, end_bonus, C.byref(out)), "swb_banded_sw_align")
        return SWResult(*out.as_tuple())

    def global_align(self, query, target, scoring: Scoring, w: int) -> GlobalAlignResult:
        q, t = _u8(query), _u8(target)
        cap = q.size + t.size + 1
        cig = np.zeros(cap, np.uint32)
        n = C.c_int32(cap)
        score = C.c_int32()
        _check(self.lib.swb_global_align(self.h, ptr(q), q.size, ptr(t), t.size, C.byref(scoring), w,
                                         C.byref(score), ptr(cig, C.c_uint32), C.byref(n)),
               "swb_global_align")
        return GlobalAlignResult(score.value, tuple(int(x) for x in cig[: n.value]))

    def local_align(self, query, target, scoring: Scoring,
                    min_sub_score: int = 0) -> Optional[LocalSWResult]:
        q, t = _u8(query), _u8(target)
        out = LocalResult()
        _check(self.lib.swb_local_align(self.h, ptr(q), q.size, ptr(t), t.size, C.byref(scoring),
                                        min_sub_score, C.byref(out)), "swb_local_align")
        return LocalSWResult(*out.as_tuple()) if out.score != 0 else None


_default_lock = threading.Lock()
_default: Optional[Engine] = None


def default_engine() -> Engine:
    """Process-wide engine on device 0 (the MetalSWEngine.shared analogue)."""
    global _default
    with _default_lock:
        if _default is None:
            _default = Engine(0)
        return _default


class BandedSWScalar:
    @staticmethod
    def align(query, target, scoring: Scoring, w: int, h0: int, endBonus: int = 0) -> SWResult:
        return default_engine().banded_sw_align(query, target, scoring, w, h0, endBonus)


class GlobalAligner:
    @staticmethod
    def align(query, target, scoring: Scoring, w: int) -> GlobalAlignResult:
        return default_engine().global_align(query, target, scoring, w)


class LocalSWAligner:
    @staticmethod
    def align(query, target, scoring: Scoring, minSubScore: int = 0) -> Optional[LocalSWResult]:
        return default_engine().local_align(query, target, scoring, minSubScore)
