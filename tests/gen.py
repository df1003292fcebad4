"""Seeded random task sets for the parity tests (numpy only).

Each generator returns (bases, tasks[, pac, ref_bases]) in the C ABI's
layout.  Targets are mostly mutated copies of the query so that the
alignments are non-trivial (long matches, gaps, N bases, tandem repeats),
mixed with unrelated random targets, reversed/complemented spans and spans
read from a packed reference.
"""
import numpy as np

from swiftbwa_b200.abi import (EXT_TASK_DTYPE, GLOBAL_TASK_DTYPE, LOCAL_TASK_DTYPE, SWB_GLB_RETRY,
                               SWB_Q_REVERSE, SWB_T_COMPLEMENT, SWB_T_FROM_REF, SWB_T_REVERSE)


def pack_ref(ref: np.ndarray) -> np.ndarray:
    """2-bit .pac layout, first base in bits 7-6 (PackedReference.swift:4-5)."""
    n = len(ref)
    padded = np.zeros((n + 3) // 4 * 4, np.uint8)
    padded[:n] = ref & 3
    p = padded.reshape(-1, 4)
    return ((p[:, 0] << 6) | (p[:, 1] << 4) | (p[:, 2] << 2) | p[:, 3]).astype(np.uint8)


def mutate(rng, seq, sub=0.03, indel=0.01, n_rate=0.005):
    out = []
    i = 0
    L = len(seq)
    while i < L:
        r = rng.random()
        if r < indel / 2:                       # deletion of 1-3 bases
            i += int(rng.integers(1, 4))
            continue
        if r < indel:                           # insertion of 1-3 bases
            out.extend(rng.integers(0, 4, int(rng.integers(1, 4))).tolist())
        b = int(seq[i])
        r2 = rng.random()
        if r2 < sub:
            b = (b + int(rng.integers(1, 4))) % 4
        elif r2 < sub + n_rate:
            b = 4
        out.append(b)
        i += 1
    return np.array(out, np.uint8)


def tandem(rng, n):
    period = int(rng.integers(2, 7))
    unit = rng.integers(0, 4, period)
    return np.resize(unit, n).astype(np.uint8)


def ext_tasks(seed, n, qmax=300, ref_len=0, big_scores=False):
    """Extension tasks in a shared bases buffer (optionally some targets from a packed ref)."""
    rng = np.random.default_rng(seed)
    chunks, tasks = [], np.zeros(n, EXT_TASK_DTYPE)
    off = 0
    ref = rng.integers(0, 4, ref_len).astype(np.uint8) if ref_len else None
    for k in range(n):
        kind = rng.random()
        qlen = int(rng.integers(0, qmax + 1)) if rng.random() < 0.05 else int(rng.integers(1, qmax + 1))
        base = tandem(rng, qlen + 120) if kind < 0.15 else rng.integers(0, 4, qlen + 120).astype(np.uint8)
        q = base[:qlen].copy()
        if rng.random() < 0.3:
            q[rng.random(qlen) < 0.01] = 4
        w = int(rng.choice([1, 2, 5, 10, 20, 50, 100, 150]))
        if kind < 0.75:
            t = mutate(rng, base, sub=rng.choice([0.0, 0.01, 0.03, 0.1]), indel=rng.choice([0.0, 0.005, 0.02]))
            t = t[: qlen + w] if rng.random() < 0.8 else t
        else:
            t = rng.integers(0, 4, int(rng.integers(0, qlen + w + 2))).astype(np.uint8)
        if rng.random() < 0.03:
            t = t[:0]
        flags = 0
        if rng.random() < 0.25:
            flags |= SWB_Q_REVERSE
        if rng.random() < 0.25:
            flags |= SWB_T_REVERSE
        if rng.random() < 0.2:
            flags |= SWB_T_COMPLEMENT
        tlen = len(t)
        q_off = off
        chunks.append(q)
        off += qlen
        if ref is not None and rng.random() < 0.3 and 0 < tlen < ref_len:
            flags |= SWB_T_FROM_REF
            t_off = int(rng.integers(0, ref_len - tlen))
        else:
            t_off = off
            chunks.append(t)
            off += tlen
        h0 = int(rng.integers(0, 120)) if not big_scores else int(rng.integers(30000, 40000))
        if rng.random() < 0.05:
            h0 = int(rng.integers(1, 8))
        tasks[k] = (q_off, t_off, qlen, tlen, w, h0, int(rng.integers(0, 11)), flags)
    bases = np.concatenate(chunks) if chunks else np.zeros(1, np.uint8)
    if bases.size == 0:
        bases = np.zeros(1, np.uint8)
    out = dict(bases=bases, tasks=tasks)
    if ref is not None:
        out.update(pac=pack_ref(ref), ref=ref, ref_bases=ref_len)
    return out


def global_tasks(seed, n, qmax=200, retry=True):
    rng = np.random.default_rng(seed)
    chunks, tasks = [], np.zeros(n, GLOBAL_TASK_DTYPE)
    off = 0
    for k in range(n):
        qlen = int(rng.integers(1, qmax + 1))
        base = tandem(rng, qlen) if rng.random() < 0.15 else rng.integers(0, 4, qlen).astype(np.uint8)
        q = base
        if rng.random() < 0.8:
            t = mutate(rng, base, sub=rng.choice([0.0, 0.02, 0.05]), indel=rng.choice([0.0, 0.01, 0.05]))
        else:
            t = rng.integers(0, 4, int(rng.integers(1, qmax + 1))).astype(np.uint8)
        if len(t) == 0:
            t = np.array([1], np.uint8)
        w = int(rng.choice([1, 2, 3, 5, 10, 30, 100]))
        flags = SWB_GLB_RETRY if (retry and rng.random() < 0.6) else 0
        true_score = int(rng.integers(-10, qlen + 1))
        chunks += [q, t]
        tasks[k] = (off, off + qlen, qlen, len(t), w, true_score, flags, 0)
        off += qlen + len(t)
    return dict(bases=np.concatenate(chunks), tasks=tasks)


def local_tasks(seed, n, qmax=260, tmax=800, ref_len=0):
    rng = np.random.default_rng(seed)
    chunks, tasks = [], np.zeros(n, LOCAL_TASK_DTYPE)
    off = 0
    for k in range(n):
        qlen = int(rng.integers(1, qmax + 1)) if rng.random() < 0.7 else int(rng.choice([150, 100, 250, 16, 17, 32, 33]))
        qlen = min(qlen, qmax)
        q = (tandem(rng, qlen) if rng.random() < 0.15 else rng.integers(0, 4, qlen)).astype(np.uint8)
        if rng.random() < 0.2:
            q[rng.random(qlen) < 0.02] = 4
        tlen = int(rng.integers(1, tmax + 1))
        t = rng.integers(0, 4, tlen).astype(np.uint8)
        if rng.random() < 0.8 and tlen > 10:
            m = mutate(rng, q, sub=rng.choice([0.0, 0.02, 0.05]), indel=rng.choice([0.0, 0.01]))
            pos = int(rng.integers(0, max(1, tlen - len(m) // 2)))
            m = m[: tlen - pos]
            t[pos: pos + len(m)] = np.minimum(m, 3)
            if rng.random() < 0.3:   # a second, weaker copy (exercises score2)
                m2 = mutate(rng, q, sub=0.1, indel=0.02)
                p2 = int(rng.integers(0, max(1, tlen - len(m2) // 2)))
                m2 = m2[: tlen - p2]
                t[p2: p2 + len(m2)] = np.minimum(m2, 3)
        flags = 0
        if rng.random() < 0.2:
            flags |= SWB_Q_REVERSE
        if rng.random() < 0.2:
            flags |= SWB_T_REVERSE
        chunks += [q, t]
        tasks[k] = (off, off + qlen, qlen, tlen, int(rng.choice([19, 0, 5, 30, 300])), flags)
        off += qlen + tlen
    return dict(bases=np.concatenate(chunks), tasks=tasks)


def ext_batch_binned(engine, sc, bases, tasks):
    """Runs tasks through swb_ext_batch_device (HBM-resident inputs): always
    the binned pass -- the host entry sends batches of up to 16384 tasks to
    the one-launch form instead."""
    import torch
    from swiftbwa_b200.abi import EXT_RESULT_DTYPE
    d_b = torch.from_numpy(np.ascontiguousarray(bases)).to("cuda:0")
    d_t = torch.from_numpy(np.ascontiguousarray(tasks).view(np.uint8)).to("cuda:0")
    d_o = torch.full((max(len(tasks), 1) * EXT_RESULT_DTYPE.itemsize,), 0xA5, dtype=torch.uint8, device="cuda:0")
    s = torch.cuda.Stream()
    engine.ext_batch_device(sc, d_b.data_ptr(), d_t.data_ptr(), len(tasks), d_o.data_ptr(), s.cuda_stream)
    s.synchronize()
    return d_o.cpu().numpy().view(EXT_RESULT_DTYPE)[: len(tasks)]
