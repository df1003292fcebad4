"""ctypes mirror of include/swb_cuda.h (the C ABI of libswb_cuda.so).

Struct layouts here must match the header byte for byte; tests check the
sizes against the C compiler's view through ``swb_struct_sizes``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

SWB_OK = 0
SWB_ERR_INVALID_ARG = -1
SWB_ERR_NO_DEVICE = -2
SWB_ERR_CUDA = -3
SWB_ERR_OOM = -4
SWB_ERR_TOO_LARGE = -5
SWB_ERR_NO_REFERENCE = -6
SWB_ERR_TIMEOUT = -7
SWB_ERR_NOT_FOUND = -8
SWB_ERR_KERNEL = -9

SWB_Q_REVERSE = 0x1
SWB_T_REVERSE = 0x2
SWB_T_COMPLEMENT = 0x4
SWB_T_FROM_REF = 0x8
SWB_GLB_RETRY = 0x100


class Scoring(C.Structure):
    """ScoringParameters' SW fields (Sources/BWACore/ScoringParameters.swift:2-28)."""
    _fields_ = [("a", C.c_int32), ("b", C.c_int32),
                ("o_ins", C.c_int32), ("e_ins", C.c_int32),
                ("o_del", C.c_int32), ("e_del", C.c_int32),
                ("zdrop", C.c_int32), ("pen_clip5", C.c_int32), ("pen_clip3", C.c_int32),
                ("band_width", C.c_int32), ("min_seed_len", C.c_int32)]

    @classmethod
    def default(cls, **overrides) -> "Scoring":
        s = cls(a=1, b=4, o_ins=6, e_ins=1, o_del=6, e_del=1, zdrop=100,
                pen_clip5=5, pen_clip3=5, band_width=100, min_seed_len=19)
        for k, v in overrides.items():
            setattr(s, k, int(v))
        return s


class ExtResult(C.Structure):
    """SWResult field order (Sources/BWACore/SWResult.swift:2-24)."""
    _fields_ = [("score", C.c_int32), ("qle", C.c_int32), ("tle", C.c_int32),
                ("gtle", C.c_int32), ("gscore", C.c_int32), ("max_off", C.c_int32)]

    def as_tuple(self):
        return (self.score, self.qle, self.tle, self.gtle, self.gscore, self.max_off)


class ExtTask(C.Structure):
    _fields_ = [("q_off", C.c_uint64), ("t_off", C.c_uint64),
                ("qlen", C.c_int32), ("tlen", C.c_int32),
                ("w", C.c_int32), ("h0", C.c_int32), ("end_bonus", C.c_int32),
                ("flags", C.c_uint32)]


class GlobalTask(C.Structure):
    _fields_ = [("q_off", C.c_uint64), ("t_off", C.c_uint64),
                ("qlen", C.c_int32), ("tlen", C.c_int32),
                ("w", C.c_int32), ("true_score", C.c_int32),
                ("flags", C.c_uint32), ("reserved", C.c_int32)]


class GlobalResult(C.Structure):
    _fields_ = [("score", C.c_int32), ("n_cigar", C.c_int32),
                ("w_used", C.c_int32), ("attempts", C.c_int32),
                ("cigar_off", C.c_uint64)]


class LocalTask(C.Structure):
    _fields_ = [("q_off", C.c_uint64), ("t_off", C.c_uint64),
                ("qlen", C.c_int32), ("tlen", C.c_int32),
                ("min_sub_score", C.c_int32), ("flags", C.c_uint32)]


class LocalResult(C.Structure):
    """LocalSWResult (Sources/Alignment/LocalSWAligner.swift:4-23); score 0 <=> nil."""
    _fields_ = [("score", C.c_int32), ("qb", C.c_int32), ("qe", C.c_int32),
                ("tb", C.c_int32), ("te", C.c_int32), ("score2", C.c_int32)]

    def as_tuple(self):
        return (self.score, self.qb, self.qe, self.tb, self.te, self.score2)


# numpy dtypes with the same layout, for building large task arrays without
# per-element Python work.
EXT_TASK_DTYPE = np.dtype([("q_off", "<u8"), ("t_off", "<u8"), ("qlen", "<i4"), ("tlen", "<i4"),
                           ("w", "<i4"), ("h0", "<i4"), ("end_bonus", "<i4"), ("flags", "<u4")])
EXT_RESULT_DTYPE = np.dtype([("score", "<i4"), ("qle", "<i4"), ("tle", "<i4"),
                             ("gtle", "<i4"), ("gscore", "<i4"), ("max_off", "<i4")])
GLOBAL_TASK_DTYPE = np.dtype([("q_off", "<u8"), ("t_off", "<u8"), ("qlen", "<i4"), ("tlen", "<i4"),
                              ("w", "<i4"), ("true_score", "<i4"), ("flags", "<u4"), ("reserved", "<i4")])
GLOBAL_RESULT_DTYPE = np.dtype([("score", "<i4"), ("n_cigar", "<i4"), ("w_used", "<i4"),
                                ("attempts", "<i4"), ("cigar_off", "<u8")])
LOCAL_TASK_DTYPE = np.dtype([("q_off", "<u8"), ("t_off", "<u8"), ("qlen", "<i4"), ("tlen", "<i4"),
                             ("min_sub_score", "<i4"), ("flags", "<u4")])
LOCAL_RESULT_DTYPE = np.dtype([("score", "<i4"), ("qb", "<i4"), ("qe", "<i4"),
                               ("tb", "<i4"), ("te", "<i4"), ("score2", "<i4")])

SEED_DTYPE = np.dtype([("rbeg", "<i8"), ("qbeg", "<i4"), ("len", "<i4"), ("score", "<i4"), ("reserved", "<i4")])
CHAIN_DTYPE = np.dtype([("read_off", "<u8"), ("read_len", "<i4"), ("rid", "<i4"), ("seed_off", "<u4"),
                        ("n_seeds", "<u4")])
REGION_DTYPE = np.dtype([("rb", "<i8"), ("re", "<i8"), ("qb", "<i4"), ("qe", "<i4"), ("rid", "<i4"),
                         ("score", "<i4"), ("true_score", "<i4"), ("sub", "<i4"), ("sub_n", "<i4"), ("w", "<i4"),
                         ("seed_cov", "<i4"), ("seed_len0", "<i4")])
ORIENTATION_DTYPE = np.dtype([("failed", "<i4"), ("reserved", "<i4"), ("proper_low", "<i8"), ("proper_high", "<i8")])
ANCHOR_DTYPE = np.dtype([("rb", "<i8"), ("rid", "<i4"), ("reserved", "<i4")])
RESCUE_JOB_DTYPE = np.dtype([("mate_off", "<u8"), ("mate_len", "<i4"), ("reserved", "<i4"), ("tmpl_off", "<u4"),
                             ("n_tmpl", "<u4"), ("mreg_off", "<u4"), ("n_mreg", "<u4")])
RESCUED_DTYPE = np.dtype([("rb", "<i8"), ("re", "<i8"), ("qb", "<i4"), ("qe", "<i4"), ("rid", "<i4"), ("score", "<i4"),
                          ("true_score", "<i4"), ("csub", "<i4"), ("seed_cov", "<i4"), ("reserved", "<i4")])
assert ORIENTATION_DTYPE.itemsize == 24 and ANCHOR_DTYPE.itemsize == 16
assert RESCUE_JOB_DTYPE.itemsize == 32 and RESCUED_DTYPE.itemsize == 48
assert SEED_DTYPE.itemsize == 24 and CHAIN_DTYPE.itemsize == 24 and REGION_DTYPE.itemsize == 56
assert EXT_TASK_DTYPE.itemsize == C.sizeof(ExtTask) == 40
assert GLOBAL_TASK_DTYPE.itemsize == C.sizeof(GlobalTask) == 40
assert LOCAL_TASK_DTYPE.itemsize == C.sizeof(LocalTask) == 32
# CheckpointOCC and SMEM (swb_bwt_checkpoint, swb_smem).
BWT_CHECKPOINT_DTYPE = np.dtype([("counts", "<i8", (4,)), ("bits", "<u8", (4,))])
SMEM_DTYPE = np.dtype([("k", "<i8"), ("l", "<i8"), ("qb", "<i4"), ("qe", "<i4")])
assert BWT_CHECKPOINT_DTYPE.itemsize == 64 and SMEM_DTYPE.itemsize == 24
assert GLOBAL_RESULT_DTYPE.itemsize == C.sizeof(GlobalResult) == 24
assert EXT_RESULT_DTYPE.itemsize == C.sizeof(ExtResult) == 24
assert LOCAL_RESULT_DTYPE.itemsize == C.sizeof(LocalResult) == 24

#: Every function include/swb_cuda.h declares (checked against the .so's exports).
EXPORTED_SYMBOLS = (
    "swb_scoring_default", "swb_init", "swb_destroy", "swb_strerror",
    "swb_last_error_message", "swb_upload_reference", "swb_ext_batch",
    "swb_global_batch", "swb_local_batch", "swb_ext_batch_device", "swb_ext_batch_plain_device",
    "swb_banded_sw_align", "swb_global_align", "swb_local_align",
    "swb_kernel_launches", "swb_last_batch_stats", "swb_profile", "swb_profile_reset",
    "swb_profile_read", "swb_int_alu_peak", "swb_int16x2_alu_peak", "swb_set_ext_bins", "swb_get_ext_bins", "swb_tune_ext_bins", "swb_ext_batch_static", "swb_cigar_batch",
    "swb_server_start", "swb_server_submit", "swb_server_poll", "swb_server_wait", "swb_server_resume",
    "swb_server_stats_get", "swb_server_stop", "swb_extend_chains", "swb_mate_rescue",
    "swb_upload_bwt", "swb_smem_batch",
)


class ServerOpts(C.Structure):
    _fields_ = [("arena_bytes", C.c_size_t), ("max_wave_tasks", C.c_size_t), ("plain", C.c_int32),
                ("start_paused", C.c_int32), ("latency_cells", C.c_uint32), ("reserved", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("tasks_completed", C.c_uint64),
                ("waves", C.c_uint64), ("cells", C.c_uint64), ("busy_ms", C.c_double)]

CIGAR_TASK_DTYPE = np.dtype([("q_off", "<u8"), ("t_off", "<u8"), ("qlen", "<i4"), ("rlen", "<i4"),
                             ("qb", "<i4"), ("qe", "<i4"), ("read_len", "<i4"), ("is_reverse", "<i4"),
                             ("true_score", "<i4"), ("initial_w", "<i4"), ("ref_pos", "<i8"),
                             ("flags", "<u4"), ("reserved", "<i4")])
CIGAR_RESULT_DTYPE = np.dtype([("score", "<i4"), ("nm", "<i4"), ("n_cigar", "<i4"), ("md_len", "<i4"),
                               ("pos", "<i8"), ("cigar_off", "<u8"), ("md_off", "<u8"),
                               ("used_dp", "<i4"), ("reserved", "<i4")])
assert CIGAR_TASK_DTYPE.itemsize == 64 and CIGAR_RESULT_DTYPE.itemsize == 48


class KernelStat(C.Structure):
    _fields_ = [("name", C.c_char * 40), ("launches", C.c_uint32), ("total_ms", C.c_double),
                ("cells", C.c_uint64)]

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libswb_cuda.so")


def ptr(a: np.ndarray, ctype=C.c_uint8):
    """Pointer to a contiguous numpy array's data (NULL for None)."""
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ctype))


def declare(lib: C.CDLL) -> C.CDLL:
    """Attach argtypes/restypes for every C-ABI entry point."""
    P = C.POINTER
    u8p, vp = P(C.c_uint8), C.c_void_p
    lib.swb_scoring_default.argtypes = [P(Scoring)]
    lib.swb_scoring_default.restype = None
    lib.swb_init.argtypes = [C.c_int, C.c_size_t, P(vp)]
    lib.swb_init.restype = C.c_int
    lib.swb_destroy.argtypes = [vp]
    lib.swb_destroy.restype = None
    lib.swb_strerror.argtypes = [C.c_int]
    lib.swb_strerror.restype = C.c_char_p
    lib.swb_last_error_message.argtypes = []
    lib.swb_last_error_message.restype = C.c_char_p
    lib.swb_upload_reference.argtypes = [vp, u8p, C.c_uint64]
    lib.swb_upload_reference.restype = C.c_int
    lib.swb_ext_batch.argtypes = [vp, P(Scoring), u8p, C.c_size_t, vp, C.c_size_t, vp]
    lib.swb_ext_batch.restype = C.c_int
    lib.swb_global_batch.argtypes = [vp, P(Scoring), u8p, C.c_size_t, vp, C.c_size_t, vp,
                                     P(C.c_uint32), C.c_size_t]
    lib.swb_global_batch.restype = C.c_int
    lib.swb_local_batch.argtypes = [vp, P(Scoring), u8p, C.c_size_t, vp, C.c_size_t, vp]
    lib.swb_local_batch.restype = C.c_int
    lib.swb_ext_batch_device.argtypes = [vp, P(Scoring), vp, vp, C.c_size_t, vp, vp]
    lib.swb_ext_batch_device.restype = C.c_int
    lib.swb_ext_batch_plain_device.argtypes = [vp, P(Scoring), vp, vp, C.c_size_t, vp, vp]
    lib.swb_ext_batch_plain_device.restype = C.c_int
    lib.swb_upload_bwt.argtypes = [vp, vp, C.c_uint64, P(C.c_int64), C.c_int64, C.c_int64]
    lib.swb_upload_bwt.restype = C.c_int
    lib.swb_smem_batch.argtypes = [vp, vp, C.c_size_t, vp, vp, C.c_size_t, C.c_int32, C.c_int64, C.c_int32,
                                   C.c_int32, C.c_uint32, vp, C.c_size_t, vp, vp]
    lib.swb_smem_batch.restype = C.c_int
    lib.swb_banded_sw_align.argtypes = [vp, u8p, C.c_int32, u8p, C.c_int32, P(Scoring),
                                        C.c_int32, C.c_int32, C.c_int32, P(ExtResult)]
    lib.swb_banded_sw_align.restype = C.c_int
    lib.swb_global_align.argtypes = [vp, u8p, C.c_int32, u8p, C.c_int32, P(Scoring), C.c_int32,
                                     P(C.c_int32), P(C.c_uint32), P(C.c_int32)]
    lib.swb_global_align.restype = C.c_int
    lib.swb_local_align.argtypes = [vp, u8p, C.c_int32, u8p, C.c_int32, P(Scoring), C.c_int32,
                                    P(LocalResult)]
    lib.swb_local_align.restype = C.c_int
    lib.swb_kernel_launches.argtypes = [vp]
    lib.swb_kernel_launches.restype = C.c_uint64
    lib.swb_last_batch_stats.argtypes = [vp, P(C.c_double), P(C.c_uint64)]
    lib.swb_last_batch_stats.restype = C.c_int
    lib.swb_profile.argtypes = [vp, C.c_int]
    lib.swb_profile.restype = C.c_int
    lib.swb_profile_reset.argtypes = [vp]
    lib.swb_profile_reset.restype = C.c_int
    lib.swb_profile_read.argtypes = [vp, P(KernelStat), C.c_int, P(C.c_int)]
    lib.swb_profile_read.restype = C.c_int
    lib.swb_int_alu_peak.argtypes = [vp, P(C.c_double)]
    lib.swb_int_alu_peak.restype = C.c_int
    lib.swb_int16x2_alu_peak.argtypes = [vp, P(C.c_double)]
    lib.swb_int16x2_alu_peak.restype = C.c_int
    lib.swb_set_ext_bins.argtypes = [vp, P(C.c_int32), C.c_int]
    lib.swb_set_ext_bins.restype = C.c_int
    lib.swb_get_ext_bins.argtypes = [vp, P(C.c_int32), C.c_int, P(C.c_int)]
    lib.swb_get_ext_bins.restype = C.c_int
    lib.swb_tune_ext_bins.argtypes = [vp, P(Scoring), vp, C.c_size_t, vp, C.c_size_t, P(C.c_int32), C.c_int,
                                      P(C.c_int), P(C.c_float), P(C.c_float)]
    lib.swb_tune_ext_bins.restype = C.c_int
    lib.swb_ext_batch_static.argtypes = [P(Scoring), vp, vp, vp, C.c_size_t, vp, vp]
    lib.swb_ext_batch_static.restype = C.c_int
    lib.swb_cigar_batch.argtypes = [vp, P(Scoring), u8p, C.c_size_t, vp, C.c_size_t, vp, P(C.c_uint32),
                                    C.c_size_t, C.c_char_p, C.c_size_t]
    lib.swb_cigar_batch.restype = C.c_int
    lib.swb_server_start.argtypes = [vp, P(Scoring), P(ServerOpts), P(vp)]
    lib.swb_server_submit.argtypes = [vp, u8p, C.c_size_t, C.c_uint64, vp, C.c_size_t, vp, P(C.c_uint64)]
    lib.swb_server_poll.argtypes = [vp, C.c_uint64, P(C.c_int), P(C.c_int)]
    lib.swb_server_wait.argtypes = [vp, C.c_uint64, C.c_int, P(C.c_int), P(C.c_uint64), P(C.c_uint64)]
    lib.swb_server_resume.argtypes = [vp]
    lib.swb_server_stats_get.argtypes = [vp, P(ServerStats)]
    lib.swb_server_stop.argtypes = [vp]
    lib.swb_extend_chains.argtypes = [vp, P(Scoring), u8p, C.c_size_t, vp, C.c_size_t, vp, C.c_size_t, C.c_uint64,
                                      vp, P(C.c_uint32), P(C.c_uint32)]
    lib.swb_extend_chains.restype = C.c_int
    lib.swb_mate_rescue.argtypes = [vp, P(Scoring), u8p, C.c_size_t, vp, C.c_size_t, vp, C.c_size_t, vp, C.c_size_t,
                                    vp, C.c_int32, vp, vp, C.c_size_t, C.c_uint64, vp, P(C.c_uint32),
                                    P(C.c_uint32)]
    lib.swb_mate_rescue.restype = C.c_int
    for f in ("swb_server_start", "swb_server_submit", "swb_server_poll", "swb_server_wait", "swb_server_resume",
              "swb_server_stats_get", "swb_server_stop"):
        getattr(lib, f).restype = C.c_int
    return lib


_LIB = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Load the in-tree libswb_cuda.so; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with `python -m swiftbwa_b200.build`")
        _LIB = declare(C.CDLL(path))
    return _LIB
