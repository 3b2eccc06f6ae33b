"""GPU parity of the selector's sequence pass (aw_sequence_summary_batch) through the C ABI:
sketches (hash, position, order, the 4-per-hash cap), fingerprints and the ambiguous and
low-complexity fractions bit-exact; the normalized entropy within 1e-9 relative (the device
sums the 64-base blocks in double, the reference in long double)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(__file__)
ENTROPY_REL = 1e-9


def _sel():
    from anchorwave_b200 import selector
    return selector


def _same(a, b, ctx):
    assert a[0] == b[0], ctx
    for s, (x, y) in enumerate(zip(a[1], b[1])):
        for sc in range(3):
            assert x["sketches"][sc] == y["sketches"][sc], (ctx, s, sc, len(x["sketches"][sc]), len(y["sketches"][sc]))
        assert x["fingerprint"] == y["fingerprint"], (ctx, s)
        assert x["ambiguous_fraction"] == y["ambiguous_fraction"], (ctx, s)
        assert x["low_complexity_fraction"] == y["low_complexity_fraction"], (ctx, s)
        assert abs(x["normalized_entropy"] - y["normalized_entropy"]) <= ENTROPY_REL * max(1.0, y["normalized_entropy"]), (ctx, s)


def test_summary_golden(gpu):
    from test_oracle import summary_matches
    sel = _sel()
    g = json.load(open(os.path.join(HERE, "golden", "summary_golden.json")))
    qs = [c["query"].encode() for c in g["cases"]]
    ts = [c["target"].encode() for c in g["cases"]]
    res = sel.sequence_summary_batch(qs, ts)
    bad = [c["name"] for c, r in zip(g["cases"], res) if not summary_matches(r, c["result"], ENTROPY_REL)]
    assert not bad, bad


def _pairs(seed, n, lmax=30000):
    rng = np.random.default_rng(seed)
    qs, ts = [], []
    for i in range(n):
        L = int(np.exp(rng.uniform(np.log(1), np.log(lmax))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.25, 4.0)
        qa, ta = bytearray(W.to_ascii(q)), bytearray(W.to_ascii(t))
        if i % 4 == 1 and len(qa):
            for j in rng.integers(0, len(qa), 9):
                qa[j] = ord("N")
        if i % 4 == 2 and len(ta):
            for j in rng.integers(0, len(ta), 50):
                ta[j] = ord(chr(ta[j]).lower())
        if i % 7 == 3:
            qa = bytearray(b"ACGTTTTTTTTTTGGGGGGA" * (len(qa) // 20 + 1))
        if i % 11 == 5:
            ta = bytearray(qa)
        qs.append(bytes(qa))
        ts.append(bytes(ta))
    return qs, ts


def test_summary_batch_vs_oracle(gpu, restatement):
    sel = _sel()
    qs, ts = _pairs(5, 96)
    res = sel.sequence_summary_batch(qs, ts)
    for i, (q, t) in enumerate(zip(qs, ts)):
        _same(res[i], restatement.sequence_summary(q, t), (i, len(q), len(t)))


def test_summary_given_modulos_and_long_low_complexity(gpu, restatement):
    """Caller-given modulos; a 400 kb homopolymer (one k-mer everywhere: the 4-per-hash cap
    across tiles); a 300 kb sequence spanning hundreds of tiles."""
    sel = _sel()
    rng = np.random.default_rng(8)
    big = W.to_ascii(W.random_dna(rng, 300000))
    qs = [b"A" * 400000, big, b"ACGT" * 5000]
    ts = [b"A" * 399000, big[:150000] + b"N" * 10 + big[150010:], b"TTGCA" * 3000]
    mods = [[1, 1, 1], [3, 17, 2], [1, 2, 1]]
    res = sel.sequence_summary_batch(qs, ts, mods)
    for i in range(3):
        _same(res[i], restatement.sequence_summary(qs[i], ts[i], mods[i]), i)
    res2 = sel.sequence_summary_batch(qs, ts)
    for i in range(3):
        _same(res2[i], restatement.sequence_summary(qs[i], ts[i]), ("derived", i))


def test_summary_chunked_equals_whole(gpu):
    """A small candidate budget splits the batch into many chunks; results unchanged."""
    code = ("import sys, json; sys.path.insert(0, %r)\n"
            "from anchorwave_b200 import selector\n"
            "from test_summary_gpu import _pairs\n"
            "qs, ts = _pairs(13, 40)\n"
            "r = selector.sequence_summary_batch(qs, ts)\n"
            "print(json.dumps(r))\n") % os.path.dirname(HERE)
    env = dict(os.environ, PYTHONPATH=os.pathsep.join([os.path.dirname(HERE), HERE]))
    outs = []
    for budget in ("", "5000"):
        e = dict(env)
        if budget:
            e["AW_SUMMARY_CHUNK_CANDIDATES"] = budget
        p = subprocess.run([sys.executable, "-c", code], env=e, capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        outs.append(json.loads(p.stdout.strip().splitlines()[-1]))
    for i, (a, b) in enumerate(zip(outs[0], outs[1])):
        assert a[0] == b[0], i
        for x, y in zip(a[1], b[1]):
            for key in ("fingerprint", "ambiguous_fraction", "low_complexity_fraction", "normalized_entropy"):
                assert x[key] == y[key], (i, key, x[key], y[key])
            assert x["sketches"] == y["sketches"], i


def test_summary_empty_batch_and_invalid(gpu):
    sel = _sel()
    assert sel.sequence_summary_batch([], []) == []
    from anchorwave_b200._lib import AwError
    with pytest.raises(AwError):
        sel.sequence_summary_batch([b"ACGT"], [b"ACGT"], [[0, 1, 1]])
