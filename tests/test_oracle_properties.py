"""CPU property tests of the oracles on small generated inputs (hypothesis): the WFA
restatement equals the compiled WFA2-lib in every memory mode, and the selector-summary
restatement equals the compiled selector, with the sketch invariants of the reference
(positions ascending per scale, at most 4 entries per hash, every entry a k-mer of A/C/G/T
whose hash the modulo divides)."""
import collections

import pytest
from hypothesis import HealthCheck, given, settings
from hypothesis import strategies as st

import oracle

SEQ = st.text(alphabet="ACGTNacgt", min_size=0, max_size=120)
DNA = st.text(alphabet="ACGT", min_size=0, max_size=200)
PEN = st.tuples(st.integers(1, 6), st.integers(0, 8), st.integers(1, 3), st.integers(0, 30), st.integers(1, 2))


def _mix(v):
    m = (1 << 64) - 1
    v ^= v >> 30
    v = (v * 0xbf58476d1ce4e5b9) & m
    v ^= v >> 27
    v = (v * 0x94d049bb133111eb) & m
    v ^= v >> 31
    return v


@settings(max_examples=150, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(p=DNA, t=DNA, pen=PEN, mode=st.sampled_from([0, 1, 2]))
def test_wfa_restatement_equals_reference(restatement, reference, p, t, pen, mode):
    a = restatement.wfa_align(p.encode(), t.encode(), *pen, memory_mode=mode)
    b = reference.wfa_align(p.encode(), t.encode(), *pen, memory_mode=mode)
    assert a == b


@settings(max_examples=150, deadline=None, suppress_health_check=[HealthCheck.function_scoped_fixture])
@given(q=SEQ, r=SEQ, mods=st.one_of(st.none(), st.tuples(st.integers(1, 5), st.integers(1, 5), st.integers(1, 5))))
def test_summary_restatement_equals_reference(restatement, reference, q, r, mods):
    if not reference.has_summary:
        pytest.skip("compiled reference without the selector shim")
    a = restatement.sequence_summary(q.encode(), r.encode(), mods)
    b = reference.sequence_summary(q.encode(), r.encode(), mods)
    assert a[0] == b[0]
    for seq, x, y in zip((q, r), a[1], b[1]):
        assert x["sketches"] == y["sketches"] and x["fingerprint"] == y["fingerprint"]
        assert abs(x["normalized_entropy"] - y["normalized_entropy"]) <= 1e-12
        for sc, (k, sk) in enumerate(zip((9, 15, 21), x["sketches"])):
            pos = [p for _, p in sk]
            assert pos == sorted(pos) and len(set(pos)) == len(pos)
            assert max(collections.Counter(h for h, _ in sk).values(), default=0) <= 4
            for h, p in sk:
                kmer = seq[p:p + k].upper()
                assert len(kmer) == k and set(kmer) <= set("ACGT")
                code = 0
                for c in kmer:
                    code = (code << 2) | "ACGT".index(c)
                assert _mix(code) == h
