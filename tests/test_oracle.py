"""CPU: the oracle itself is pinned -- the plain-C restatement against the golden vectors
generated from the compiled reference, and (where oracle/_ref is present) against the
compiled reference live on fresh seeded corpora, for all three SIMD variants."""
import json
import os

import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "ksw2_golden.json")


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)


def _mat(c):
    return c.get("mat") or oracle.anchorwave_matrix(c["mismatch"])


def _codes(s):
    return W.to_codes(s.encode()).tobytes()


def test_restatement_matches_golden(restatement):
    g = _golden()
    bad = []
    for c in g["cases"]:
        flag = c["flag"] | (oracle.KSW_EZ_SINGLETRACK if c["variant"] == 2 else 0)
        r = restatement.ksw_extd2(_codes(c["query"]), _codes(c["target"]), _mat(c), c["q"], c["e"], c["q2"],
                                  c["e2"], w=c["w"], zdrop=c["zdrop"], end_bonus=c["end_bonus"], flag=flag,
                                  block=g["block"])
        exp = c["result"]
        got = {k: getattr(r, k) for k in exp}
        if got != exp:
            bad.append(c["name"])
    assert not bad, f"restatement differs from golden on {bad}"


def test_reference_matches_golden(reference):
    g = _golden()
    if reference.block != g["block"]:
        pytest.skip("host ISA differs from the golden generator's")
    for c in g["cases"][:40]:
        r = reference.ksw_extd2(_codes(c["query"]), _codes(c["target"]), _mat(c), c["q"], c["e"], c["q2"],
                                c["e2"], w=c["w"], zdrop=c["zdrop"], end_bonus=c["end_bonus"], flag=c["flag"],
                                variant=c["variant"])
        assert {k: getattr(r, k) for k in c["result"]} == c["result"], c["name"]


FLAGS = [0, oracle.KSW_EZ_SCORE_ONLY, oracle.KSW_EZ_RIGHT, oracle.KSW_EZ_SEMIGLOBAL_END, oracle.KSW_EZ_EXTZ_ONLY,
         oracle.KSW_EZ_APPROX_MAX, oracle.KSW_EZ_REV_CIGAR, oracle.KSW_EZ_APPROX_MAX | oracle.KSW_EZ_APPROX_DROP]
PEN = [(4, 2, 24, 1), (8, 2, 75, 1), (6, 1, 20, 0), (2, 3, 30, 1), (24, 1, 4, 2)]


@pytest.mark.parametrize("isa", ["avx512", "avx2", "sse"])
def test_restatement_matches_reference_random(restatement, isa):
    try:
        ref = oracle.Reference(isa)
    except FileNotFoundError as e:
        pytest.skip(str(e))
    if isa != "sse" and oracle.ISA_BLOCK[oracle.cpu_isa()] < oracle.ISA_BLOCK[isa]:
        pytest.skip(f"host cannot run {isa}")
    rng = np.random.default_rng(11 + len(isa))
    n = 0
    for it in range(160):
        L = int(rng.integers(1, 500))
        qc, tc = W.divergent_pair(rng, L, 0.01, 0.3, 4.0)
        if rng.random() < 0.2:
            qc = qc.copy()
            qc[rng.integers(0, len(qc), 3)] = 4
        gen = oracle.KSW_EZ_GENERIC_SC if (4 in qc or 4 in tc) else 0
        pen = PEN[it % len(PEN)]
        w = -1 if it % 3 == 0 else int(rng.integers(0, max(2, L // 3)))
        flag = FLAGS[it % len(FLAGS)] | gen
        zdrop = -1 if it % 5 else 60
        mat = oracle.anchorwave_matrix(-4) if it % 7 else [2 if a == b else -4 for a in range(5) for b in range(5)]
        a = restatement.ksw_extd2(qc.tobytes(), tc.tobytes(), mat, *pen, w=w, zdrop=zdrop, flag=flag,
                                  block=ref.block)
        b = ref.ksw_extd2(qc.tobytes(), tc.tobytes(), mat, *pen, w=w, zdrop=zdrop, flag=flag)
        assert a.key() == b.key(), (it, L, w, hex(flag), pen)
        # Singletrack entry of the library's ISA (ksw_extd2_singletrack_sse on the SSE build,
        # which also takes the score-only, semiglobal and extension flags)
        if isa == "sse" or not (flag & (oracle.KSW_EZ_SCORE_ONLY | oracle.KSW_EZ_SEMIGLOBAL_END |
                                         oracle.KSW_EZ_EXTZ_ONLY)):
            a = restatement.ksw_extd2(qc.tobytes(), tc.tobytes(), mat, *pen, w=w, zdrop=zdrop,
                                      flag=flag | oracle.KSW_EZ_SINGLETRACK, block=ref.block)
            b = ref.ksw_extd2(qc.tobytes(), tc.tobytes(), mat, *pen, w=w, zdrop=zdrop, flag=flag, variant=2)
            assert a.key() == b.key(), ("singletrack", it, L, w, hex(flag), pen)
        n += 1
    assert n == 160


def test_restatement_stop_hook_matches_reference(restatement, reference):
    rng = np.random.default_rng(5)
    q, t = W.divergent_pair(rng, 900, 0.05, 0.05, 3.0)
    mat = oracle.anchorwave_matrix(-4)
    for stop_at in (0, 256, 512, 1024, 5000):
        a = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, stop_interval=256, stop_at=stop_at,
                                  block=reference.block)
        b = reference.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, stop_interval=256, stop_at=stop_at)
        assert a.key() == b.key(), stop_at


def test_simd_variants_agree_in_full_mode(reference):
    """Full-mode results are independent of the SIMD width (padding lanes are never read)."""
    rng = np.random.default_rng(3)
    for _ in range(30):
        q, t = W.divergent_pair(rng, int(rng.integers(50, 800)), 0.01, 0.15, 4.0)
        a = reference.ksw_extd2(q.tobytes(), t.tobytes(), oracle.anchorwave_matrix(-4), 4, 2, 24, 1, variant=0)
        b = reference.ksw_extd2(q.tobytes(), t.tobytes(), oracle.anchorwave_matrix(-4), 4, 2, 24, 1, variant=1)
        assert a.key() == b.key()


WFA_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "wfa_golden.json")


def test_wfa_restatement_matches_golden(restatement):
    """The WFA restatement (high memory, Singletrack, medium and low memory) against the
    golden vectors of the compiled WFA2-lib."""
    with open(WFA_GOLDEN) as f:
        g = json.load(f)
    bad = []
    for c in g["cases"]:
        r = restatement.wfa_align(c["target"].encode(), c["query"].encode(), c["x"], c["o1"], c["e1"], c["o2"],
                                  c["e2"], c["singletrack"], memory_mode=c.get("memory_mode", 0))
        if r != (c["result"]["status"], c["result"]["score"], c["result"]["ops"]):
            bad.append(c["name"])
    assert not bad, f"WFA restatement differs from golden on {bad}"
    assert sum(1 for c in g["cases"] if c.get("memory_mode")) >= 24


@pytest.mark.parametrize("memory_mode", [1, 2])
def test_wfa_piggyback_restatement_matches_reference(restatement, reference, memory_mode):
    """Medium / low memory (piggyback traceback) against the compiled WFA2-lib on fresh
    seeded pairs, including tie-heavy penalties and low-complexity sequences."""
    rng = np.random.default_rng(300 + memory_mode)
    pens = [(4, 4, 2, 24, 1), (1, 0, 1, 0, 1), (2, 2, 1, 4, 1), (3, 0, 1, 3, 1)]
    for i in range(120):
        L = int(np.exp(rng.uniform(np.log(1), np.log(2500))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.3, 4.0)
        if i % 5 == 4:  # two-letter alphabet: many equal-score paths
            q, t = q % 2, t % 2
        p, tx = W.to_ascii(t), W.to_ascii(q)
        pen = pens[i % len(pens)]
        exp = reference.wfa_align(p, tx, *pen, memory_mode=memory_mode)
        assert restatement.wfa_align(p, tx, *pen, memory_mode=memory_mode) == exp, (i, len(p), len(tx), pen)
        # the piggyback traceback and the high-memory traceback break ties alike
        assert reference.wfa_align(p, tx, *pen, memory_mode=0) == exp, (i, pen)


SUMMARY_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "summary_golden.json")


def summary_matches(got, exp, entropy_rel=1e-12):
    """A summarizeSequencePair result against a golden record: identity, fingerprints,
    sketch counts and digest, and the fractions (entropy within entropy_rel)."""
    from golden.make_golden import sketch_digest
    ident, sides = got
    if ident != exp["identical"]:
        return False
    for s, e in zip(sides, exp["sides"]):
        if s["fingerprint"] != e["fingerprint"] or [len(k) for k in s["sketches"]] != e["counts"]:
            return False
        if sketch_digest(s) != e["digest"]:
            return False
        if s["ambiguous_fraction"] != e["ambiguous_fraction"]:
            return False
        if s["low_complexity_fraction"] != e["low_complexity_fraction"]:
            return False
        if abs(s["normalized_entropy"] - e["normalized_entropy"]) > entropy_rel * max(1.0, e["normalized_entropy"]):
            return False
    return True


def test_summary_restatement_matches_golden(restatement):
    """The selector's sequence pass restated (summary_oracle.c) against the golden records
    of the compiled selector."""
    with open(SUMMARY_GOLDEN) as f:
        g = json.load(f)
    bad = [c["name"] for c in g["cases"]
           if not summary_matches(restatement.sequence_summary(c["query"].encode(), c["target"].encode()),
                                  c["result"])]
    assert not bad, bad


def test_summary_restatement_matches_reference(restatement, reference):
    if not reference.has_summary:
        pytest.skip("compiled reference without the selector shim")
    rng = np.random.default_rng(61)
    for i in range(40):
        L = int(np.exp(rng.uniform(np.log(1), np.log(20000))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.3, 4.0)
        qa, ta = bytearray(W.to_ascii(q)), bytearray(W.to_ascii(t))
        if i % 3 == 0 and len(qa):
            for j in rng.integers(0, len(qa), 7):
                qa[j] = ord("N")
        if i % 5 == 0:  # low complexity
            qa = bytearray(b"AAAAAAAAAAAAAAAACCCCCCCCCCG" * (len(qa) // 27 + 1))
        mods = None if i % 2 else [int(x) for x in rng.integers(1, 9, 3)]
        a = restatement.sequence_summary(bytes(qa), bytes(ta), mods)
        b = reference.sequence_summary(bytes(qa), bytes(ta), mods)
        assert a[0] == b[0]
        for x, y in zip(a[1], b[1]):
            assert x["sketches"] == y["sketches"] and x["fingerprint"] == y["fingerprint"], i
            assert x["ambiguous_fraction"] == y["ambiguous_fraction"], i
            assert x["low_complexity_fraction"] == y["low_complexity_fraction"], i
            assert abs(x["normalized_entropy"] - y["normalized_entropy"]) <= 1e-12, i


def test_sse_singletrack_restatement_matches_reference(restatement, reference):
    """ksw_extd2_singletrack_sse (the reference's entry 3 on any host) against the restatement
    with 16-byte blocks and the Singletrack flag: end rules, band, and every flag."""
    rng = np.random.default_rng(77)
    flags = [0, oracle.KSW_EZ_SEMIGLOBAL_END, oracle.KSW_EZ_EXTZ_ONLY, oracle.KSW_EZ_REV_CIGAR,
             oracle.KSW_EZ_SCORE_ONLY, oracle.KSW_EZ_APPROX_MAX | oracle.KSW_EZ_APPROX_DROP,
             oracle.KSW_EZ_RIGHT | oracle.KSW_EZ_GENERIC_SC]
    mat = oracle.anchorwave_matrix(-4)
    for it in range(140):
        L = int(np.exp(rng.uniform(np.log(2), np.log(1500))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.25, 4.0)
        flag = flags[it % len(flags)]
        w = -1 if it % 2 == 0 else int(rng.integers(0, max(1, L // 3)))
        zdrop = -1 if it % 3 else 100
        pen = PEN[it % len(PEN)]
        a = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, *pen, w=w, zdrop=zdrop,
                                  flag=flag | oracle.KSW_EZ_SINGLETRACK, block=16)
        b = reference.ksw_extd2(q.tobytes(), t.tobytes(), mat, *pen, w=w, zdrop=zdrop, flag=flag, variant=3)
        assert a.key() == b.key(), (it, L, w, hex(flag), pen)
