"""Evaluates the known-answer fixtures (tests/golden/known_answers.json)
against a backend: the oracle (CPU) or the CUDA library through its C ABI.

A backend is an object with methods ext(q, t, sc, w, h0, end_bonus) -> 6-tuple,
global_(q, t, sc, w) -> (score, cigar), cigar(...) -> dict, local(q, t, sc,
min_sub) -> tuple|None, extend(...) -> regions, sw16/sw8 (oracle only).
"""
import json
import os

from swiftbwa_b200.abi import Scoring

HERE = os.path.dirname(os.path.abspath(__file__))
EXT_FIELDS = ("score", "qle", "tle", "gtle", "gscore", "max_off")
LOCAL_FIELDS = ("score", "qb", "qe", "tb", "te", "score2")


def load():
    with open(os.path.join(HERE, "golden", "known_answers.json")) as f:
        return json.load(f)


def _cmp(a, op, b):
    return {"==": a == b, ">": a > b, ">=": a >= b, "<": a < b, "<=": a <= b}[op]


def _ops(cigar):
    return [(c & 0xF, c >> 4) for c in cigar]


def _bases(cigar):
    qb = tb = 0
    for op, ln in _ops(cigar):
        if op == 0:
            qb += ln
            tb += ln
        elif op == 1:
            qb += ln
        elif op == 2:
            tb += ln
    return qb, tb


def evaluate(case, backend):
    """Returns a list of failure strings (empty = pass).  Cases whose
    function the backend does not provide return None (skipped)."""
    sc = Scoring.default(**case["scoring"])
    a = case["args"]
    fn = case["fn"]
    fails = []
    vals = {}
    if fn in ("ext", "ext_vs_sw16", "ext_vs_sw8", "ext_vs_sw8_sw16"):
        r = backend.ext(a["q"], a["t"], sc, a["w"], a["h0"], 0)
        vals.update(dict(zip(EXT_FIELDS, r)))
        if "sw16" in fn:
            if not hasattr(backend, "sw16"):
                return None
            vals.update({f"sw16.{k}": v for k, v in zip(EXT_FIELDS, backend.sw16(a["q"], a["t"], sc, a["w"], a["h0"]))})
        if "sw8" in fn:
            if not hasattr(backend, "sw8"):
                return None
            r8 = backend.sw8(a["q"], a["t"], sc, a["w"], a["h0"])
            vals["sw8"] = r8
            if r8 is not None:
                vals.update({f"sw8.{k}": v for k, v in zip(EXT_FIELDS, r8)})
    elif fn in ("sw16", "sw8"):
        if not hasattr(backend, fn):
            return None
        r = getattr(backend, fn)(a["q"], a["t"], sc, a["w"], a["h0"])
        vals["_"] = r
        if r is not None:
            vals.update(dict(zip(EXT_FIELDS, r)))
    elif fn == "global":
        score, cigar = backend.global_(a["q"], a["t"], sc, a["w"])
        vals.update(score=score, cigar=cigar, nm=backend.compute_nm(cigar, a["q"], a["t"]))
        vals["query_bases"], vals["target_bases"] = _bases(cigar)
    elif fn == "global_w_pair":
        s1, c1 = backend.global_(a["q"], a["t"], sc, a["w1"])
        s2, c2 = backend.global_(a["q"], a["t"], sc, a["w2"])
        vals.update(same_score=s1 == s2, same_cigar=c1 == c2)
    elif fn == "cigar":
        r = backend.cigar(a["q"], a["r"], a["qb"], a["qe"], a["read_len"], a["is_rev"],
                          a["true_score"], a["initial_w"], sc, a["ref_pos"])
        vals.update(r)
        vals["query_bases"], vals["target_bases"] = _bases(r["cigar"])
        vals["n_ops"] = len(r["cigar"])
    elif fn == "local":
        r = backend.local(a["q"], a["t"], sc, 0)
        vals["_"] = r
        if r is not None:
            vals.update(dict(zip(LOCAL_FIELDS, r)))
    elif fn == "extend":
        if not hasattr(backend, "extend"):
            return None
        regs = backend.extend([tuple(s) for s in a["seeds"]], 0, a["read"], a["ref"], sc)
        vals["n_regions"] = len(regs)
        if regs:
            vals.update({f"r0.{k}": v for k, v in regs[0].items()})
    else:
        raise ValueError(fn)

    for ex in case["expect"]:
        kind = ex[0]
        if kind == "nil":
            ok = vals.get("_") is None
        elif kind == "not_nil":
            ok = vals.get("_", vals.get("score")) is not None
        elif kind in ("same_score", "same_cigar"):
            ok = vals[kind]
        elif kind == "has_op":
            ok = any(op == ex[1] for op, _ in _ops(vals["cigar"]))
        elif kind == "no_op":
            ok = all(op != ex[1] for op, _ in _ops(vals["cigar"]))
        elif kind == "op":
            op, ln = _ops(vals["cigar"])[ex[1]]
            ok = (op, ln) == (ex[2], ex[3])
        elif kind == "len":
            ok = _ops(vals["cigar"])[ex[1]][1] == ex[2]
        elif kind == "md_contains":
            ok = ex[1] in vals["md"]
        elif kind == "md_not_contains":
            ok = ex[1] not in vals["md"]
        elif len(ex) == 2 and ex[1] == "not_nil":
            ok = vals.get(ex[0]) is not None
        else:
            lhs = vals[kind]
            rhs = vals[ex[2]] if isinstance(ex[2], str) and ex[2] in vals else ex[2]
            ok = _cmp(lhs, ex[1], rhs)
        if not ok:
            fails.append(f"{case['name']} ({case['source']}): {ex} with {vals}")
    return fails
