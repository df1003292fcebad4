"""Pins the C++ oracle against every known answer the reference's own test
suite holds for the Smith-Waterman path (tests/golden/known_answers.json)."""
import pytest

import known


class OracleBackend:
    def __init__(self, o):
        self.o = o

    def ext(self, q, t, sc, w, h0, eb):
        return self.o.banded_sw_scalar(q, t, sc, w, h0, eb)[0]

    def sw16(self, q, t, sc, w, h0):
        return self.o.banded_sw16(q, t, sc, w, h0)

    def sw8(self, q, t, sc, w, h0):
        return self.o.banded_sw8(q, t, sc, w, h0)

    def global_(self, q, t, sc, w):
        return self.o.global_align(q, t, sc, w)[0]

    def compute_nm(self, cigar, q, t):
        return self.o.compute_nm(cigar, q, t)

    def cigar(self, q, r, qb, qe, rl, rev, ts, iw, sc, pos):
        return self.o.cigar_generate(q, r, qb, qe, rl, rev, ts, iw, sc, pos)

    def local(self, q, t, sc, ms):
        return self.o.local_align(q, t, sc, ms)[0]

    def extend(self, seeds, rid, read, ref, sc):
        return self.o.extend(seeds, rid, read, ref, sc)[0]


CASES = known.load()["known_answers"]


@pytest.mark.parametrize("case", CASES, ids=[c["name"] for c in CASES])
def test_known_answer(case, oracle_mod):
    fails = known.evaluate(case, OracleBackend(oracle_mod))
    assert fails is not None
    assert not fails, "\n".join(fails)
