"""Writes tests/golden/known_answers.json.

Each case transcribes one known-answer test of the reference's Swift test
suite that exercises the Smith-Waterman path: the inputs and the assertions
exactly as the Swift test states them (equality, inequality or nil), with
the test's file:line.  The Swift suite cannot run here (no Swift toolchain),
so these assertions are the pins the C++ oracle and the CUDA kernels are
held to.  Run:  python tests/golden/make_known_answers.py
"""
import json
import os

A, C_, G, T = 0, 1, 2, 3
SRC = "Tests/AlignmentTests/AlignmentTests.swift"


def case(name, line, fn, args, expect, scoring=None):
    return dict(name=name, source=f"{SRC}:{line}", fn=fn, args=args, expect=expect,
                scoring=scoring or {})


ACGTAC = [A, C_, G, T, A, C_]
ACGTACGT = [A, C_, G, T, A, C_, G, T]
ACGTACGTAC = [A, C_, G, T, A, C_, G, T, A, C_]
ZD_Q = [A, C_, G, T, A] + [A] * 100
ZD_T = [A, C_, G, T, A] + [T] * 100

CASES = [
    # ---- BandedSWScalar / BandedSW16 / BandedSW8 (extension kernel) ----
    case("scalar perfect match", 48, "ext", dict(q=ACGTAC, t=ACGTAC, w=10, h0=1),
         [["score", "==", 7]]),
    case("scalar mismatch", 65, "ext", dict(q=[A, C_, G, T], t=[A, C_, A, T], w=10, h0=1),
         [["score", ">", 0]]),
    case("scalar h0 > 0", 82, "ext", dict(q=[A, C_, G], t=[A, C_, G], w=10, h0=5),
         [["score", ">=", 8]]),
    case("SW8 nil for large scores", 98, "sw8", dict(q=[A] * 300, t=[A] * 300, w=10, h0=1),
         [["nil"]]),
    case("SIMD16 agrees with scalar on perfect match", 115, "ext_vs_sw16",
         dict(q=ACGTACGT, t=ACGTACGT, w=10, h0=1), [["score", "==", 9], ["sw16.score", "==", "score"]]),
    case("SW16 globalScore and globalTargetEnd", 140, "ext_vs_sw16",
         dict(q=ACGTAC, t=ACGTAC, w=10, h0=1),
         [["gscore", ">", 0], ["sw16.gscore", "==", "gscore"], ["sw16.gtle", "==", "gtle"]]),
    case("SW16 with h0 > 0 matches scalar", 164, "ext_vs_sw16",
         dict(q=[A, C_, G], t=[A, C_, G], w=10, h0=5), [["score", ">=", 8], ["sw16.score", "==", "score"]]),
    case("SW8 agrees with scalar on short perfect match", 186, "ext_vs_sw8",
         dict(q=ACGTAC, t=ACGTAC, w=10, h0=1), [["sw8", "not_nil"], ["sw8.score", "==", "score"]]),
    case("all three agree on mismatch input", 208, "ext_vs_sw8_sw16",
         dict(q=ACGTACGTAC, t=[A, C_, G, T, T, C_, G, T, A, C_], w=10, h0=1),
         [["score", ">", 0], ["sw16.score", "==", "score"], ["sw8", "not_nil"], ["sw8.score", "==", "score"]]),
    case("z-drop in SW16 with divergent tail", 239, "sw16", dict(q=ZD_Q, t=ZD_T, w=5, h0=1),
         [["score", "==", 6], ["tle", "<", 50]], scoring=dict(zdrop=10)),
    case("z-drop in SW8 with divergent tail", 263, "sw8", dict(q=ZD_Q, t=ZD_T, w=5, h0=1),
         [["not_nil"], ["score", "==", 6], ["tle", "<", 50]], scoring=dict(zdrop=10)),
    # ---- GlobalAligner (NW kernel) ----
    case("NW perfect match", 313, "global", dict(q=ACGTACGTAC, t=ACGTACGTAC, w=10),
         [["cigar", "==", [(10 << 4) | 0]], ["score", "==", 10]]),
    case("NW single mismatch", 331, "global",
         dict(q=ACGTACGTAC, t=[A, C_, G, T, A, T, G, T, A, C_], w=10),
         [["cigar", "==", [(10 << 4) | 0]], ["nm", "==", 1], ["score", "==", 5]]),
    case("NW single insertion", 356, "global", dict(q=[A, C_, G, T, G, A, C_], t=ACGTAC, w=10),
         [["has_op", 1], ["query_bases", "==", 7], ["target_bases", "==", 6]]),
    case("NW single deletion", 391, "global", dict(q=ACGTAC, t=[A, C_, G, T, G, A, C_], w=10),
         [["has_op", 2], ["query_bases", "==", 6], ["target_bases", "==", 7]]),
    case("NW narrow vs wide band", 426, "global_w_pair", dict(q=ACGTACGT, t=ACGTACGT, w1=1, w2=50),
         [["same_score"], ["same_cigar"]]),
    # ---- CIGARGenerator (CIGAR driver) ----
    case("CIGARGenerator no soft-clips", 450, "cigar",
         dict(q=ACGTACGT, r=ACGTACGT, qb=0, qe=8, read_len=8, is_rev=False, true_score=8,
              initial_w=10, ref_pos=0), [["no_op", 4], ["nm", "==", 0]]),
    case("CIGARGenerator soft-clips", 477, "cigar",
         dict(q=[A, C_, G, T, A], r=[A, C_, G, T, A], qb=3, qe=8, read_len=12, is_rev=False,
              true_score=5, initial_w=10, ref_pos=100),
         [["n_ops", "==", 3], ["op", 0, 4, 3], ["op", 2, 4, 4]]),
    case("CIGARGenerator reverse strand clips", 509, "cigar",
         dict(q=[A, C_, G, T, A], r=[A, C_, G, T, A], qb=3, qe=8, read_len=12, is_rev=True,
              true_score=5, initial_w=10, ref_pos=100),
         [["n_ops", "==", 3], ["len", 0, 4], ["len", 2, 3]]),
    case("CIGARGenerator bandwidth retry loop", 537, "cigar",
         dict(q=[A, C_, G, T, G, G, A, C_, G, T], r=ACGTACGT, qb=0, qe=10, read_len=10,
              is_rev=False, true_score=0, initial_w=1, ref_pos=0),
         [["query_bases", "==", 10], ["target_bases", "==", 8]]),
    case("MD perfect match", 574, "cigar",
         dict(q=ACGTACGT, r=ACGTACGT, qb=0, qe=8, read_len=8, is_rev=False, true_score=8,
              initial_w=10, ref_pos=0), [["md", "==", "8"]]),
    case("MD single mismatch", 596, "cigar",
         dict(q=ACGTACGT, r=[A, C_, G, T, T, C_, G, T], qb=0, qe=8, read_len=8, is_rev=False,
              true_score=3, initial_w=10, ref_pos=0), [["md", "==", "4T3"], ["nm", "==", 1]]),
    case("MD deletion", 619, "cigar",
         dict(q=ACGTAC, r=[A, C_, G, T, G, A, C_], qb=0, qe=6, read_len=6, is_rev=False,
              true_score=-1, initial_w=10, ref_pos=0), [["md_contains", "^"]]),
    case("MD insertion", 642, "cigar",
         dict(q=[A, C_, G, T, G, A, C_], r=ACGTAC, qb=0, qe=7, read_len=7, is_rev=False,
              true_score=-1, initial_w=10, ref_pos=0), [["md_not_contains", "^"]]),
    case("MD multiple mismatches", 666, "cigar",
         dict(q=ACGTACGTAC, r=[A, T, G, T, A, C_, G, A, A, C_], qb=0, qe=10, read_len=10,
              is_rev=False, true_score=0, initial_w=10, ref_pos=0),
         [["md", "==", "1T5A2"], ["nm", "==", 2]]),
    # ---- LocalSWAligner (local SW kernel) ----
    case("local perfect match", 715, "local", dict(q=ACGTAC, t=ACGTAC),
         [["not_nil"], ["score", "==", 6], ["qb", "==", 0], ["qe", "==", 5], ["tb", "==", 0], ["te", "==", 5]]),
    case("local embedded", 730, "local", dict(q=[A, C_, G, T], t=[T, T, A, C_, G, T, T, T]),
         [["not_nil"], ["score", "==", 4], ["qb", "==", 0], ["qe", "==", 3], ["tb", "==", 2], ["te", "==", 5]]),
    case("local with mismatch", 746, "local", dict(q=ACGTACGT, t=[A, C_, G, T, T, C_, G, T]),
         [["not_nil"], ["score", ">=", 4]]),
    case("local all-mismatch is nil", 761, "local", dict(q=[A, A, A, A], t=[T, T, T, T]), [["nil"]],
         scoring=dict(a=1, b=4)),
    case("local empty is nil", 774, "local", dict(q=[], t=[A, C_, G]), [["nil"]]),
    # ---- ExtensionAligner.extend (extension driver) ----
    case("extension clips with low penClip", 783, "extend",
         dict(seeds=[[100, 10, 20, 20]], read=[T] * 10 + [A] * 20 + [T] * 10, ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.qb", ">=", 0], ["r0.qe", "<=", 40]],
         scoring=dict(pen_clip5=5, pen_clip3=5)),
    case("extension extends to read boundary with high penClip", 959, "extend",
         dict(seeds=[[100, 5, 20, 20]], read=[A] * 30, ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.qb", "==", 0], ["r0.qe", "==", 30]],
         scoring=dict(pen_clip5=100, pen_clip3=100)),
    case("extension score, seed covers read", 1140, "extend",
         dict(seeds=[[100, 0, 10, 10]], read=[A] * 10, ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.score", "==", 10]]),
    case("extension score, left only", 1170, "extend",
         dict(seeds=[[105, 5, 5, 5]], read=[A] * 10, ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.score", "==", 10]], scoring=dict(pen_clip5=100)),
    case("extension score, right only", 1203, "extend",
         dict(seeds=[[100, 0, 5, 5]], read=[A] * 10, ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.score", "==", 10]], scoring=dict(pen_clip3=100)),
    case("extension score, both sides", 1236, "extend",
         dict(seeds=[[103, 3, 4, 4]], read=[A] * 10, ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.score", "==", 10]],
         scoring=dict(pen_clip5=100, pen_clip3=100)),
    case("sub from covered seed", 1309, "extend",
         dict(seeds=[[100, 0, 30, 30], [110, 10, 20, 20]], read=[A] * 50, ref=[A] * 300),
         [["n_regions", "==", 1], ["r0.sub", "==", 20]], scoring=dict(pen_clip5=100, pen_clip3=100)),
    case("sub below minSeedLength", 1347, "extend",
         dict(seeds=[[100, 0, 30, 30], [105, 5, 10, 10]], read=[A] * 50, ref=[A] * 300),
         [["n_regions", "==", 1], ["r0.sub", "==", 0]], scoring=dict(pen_clip5=100, pen_clip3=100)),
    case("extends through mismatches with high penClip", 1384, "extend",
         dict(seeds=[[105, 5, 10, 10]], read=[A] * 18 + [T] * 2, ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.qe", "==", 20], ["r0.qb", "==", 0]],
         scoring=dict(pen_clip5=100, pen_clip3=100)),
    case("clips mismatching tail with low penClip", 1423, "extend",
         dict(seeds=[[105, 5, 10, 10]], read=[A] * 18 + [T] * 2, ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.qe", "<", 20], ["r0.qb", "==", 0]],
         scoring=dict(pen_clip5=100, pen_clip3=1)),
    case("mismatch in flank", 1460, "extend",
         dict(seeds=[[103, 3, 4, 4]], read=[A] * 9 + [T], ref=[A] * 200),
         [["n_regions", ">=", 1], ["r0.qe", "==", 10], ["r0.qb", "==", 0],
          ["r0.score", "<", 10], ["r0.score", ">", 0]],
         scoring=dict(pen_clip5=100, pen_clip3=100)),
]

# Shapes of the reference's GPU-vs-CPU differential tests
# (Tests/MetalSWTests/*.swift): replayed as CUDA-vs-oracle parity cases.
DIFF_SRC_B = "Tests/MetalSWTests/BandedSW8MetalTests.swift"
DIFF_SRC_L = "Tests/MetalSWTests/LocalSWMetalTests.swift"
_q150 = [i % 4 for i in range(150)]
_t150 = list(_q150)
_t150[50] = (_t150[50] + 1) % 4
_t150[100] = (_t150[100] + 2) % 4
_q32 = [0, 1, 2, 3] * 8
_t32 = list(_q32)
_t32[5] = 3
_t32[15] = 0
_t500 = [i % 4 for i in range(500)]
_t500[200] = (_t500[200] + 1) % 4
_t500[250] = (_t500[250] + 2) % 4
DIFF = [
    dict(kind="ext", source=f"{DIFF_SRC_B}:17", q=ACGTACGTAC, t=ACGTACGTAC, w=100, h0=1, scoring={}),
    dict(kind="ext", source=f"{DIFF_SRC_B}:48", q=ACGTACGT, t=[0, 1, 0, 3, 0, 1, 0, 3], w=100, h0=1, scoring={}),
    dict(kind="ext", source=f"{DIFF_SRC_B}:73", q=ACGTAC, t=ACGTAC, w=100, h0=10, scoring={}),
    dict(kind="ext", source=f"{DIFF_SRC_B}:96", q=[0, 1, 2, 3], t=[0, 1, 2, 3], w=100, h0=1, scoring={}),
    dict(kind="ext", source=f"{DIFF_SRC_B}:96", q=ACGTACGT, t=ACGTACGT, w=100, h0=5, scoring={}),
    dict(kind="ext", source=f"{DIFF_SRC_B}:96", q=[0] * 5, t=[0] * 5, w=100, h0=1, scoring={}),
    dict(kind="ext", source=f"{DIFF_SRC_B}:96", q=ACGTAC, t=[3, 2, 1, 0, 3, 2], w=100, h0=1, scoring={}),
    dict(kind="ext", source=f"{DIFF_SRC_B}:142", q=_q150, t=_t150, w=100, h0=1, scoring={}),
    dict(kind="ext", source=f"{DIFF_SRC_B}:177", q=[0] * 50, t=[0] * 50, w=100, h0=1, scoring=dict(a=10)),
    dict(kind="ext", source=f"{DIFF_SRC_B}:228", q=_q32, t=_t32, w=100, h0=1, scoring=dict(a=8)),
    dict(kind="local", source=f"{DIFF_SRC_L}:11", q=ACGTACGT, t=ACGTACGT, scoring={}),
    dict(kind="local", source=f"{DIFF_SRC_L}:36", q=ACGTAC, t=[3, 3, 0, 1, 2, 3, 0, 1, 3, 3], scoring={}),
    dict(kind="local", source=f"{DIFF_SRC_L}:60", q=[0, 1, 2, 3], t=[0, 1, 2, 3], scoring={}),
    dict(kind="local", source=f"{DIFF_SRC_L}:60", q=ACGTACGT, t=ACGTACGT, scoring={}),
    dict(kind="local", source=f"{DIFF_SRC_L}:60", q=[0] * 5, t=[0] * 5, scoring={}),
    dict(kind="local", source=f"{DIFF_SRC_L}:60", q=[0, 1, 2, 3], t=[3, 2, 1, 0], scoring={}),
    dict(kind="local", source=f"{DIFF_SRC_L}:101", q=_q150, t=_t500, scoring={}),
]

if __name__ == "__main__":
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "known_answers.json"), "w") as f:
        json.dump(dict(known_answers=CASES, differential_shapes=DIFF), f, indent=1)
    print(f"wrote {len(CASES)} known answers and {len(DIFF)} differential shapes")
