"""Generates tests/golden/ksw2_golden.json (and wfa_golden.json) from the COMPILED
REFERENCE (oracle/_ref/libawref_<isa>.so, AnchorWave's own KSW2 / WFA2 sources).

Run where the reference tree and oracle/_ref exist:
    make -C oracle && python tests/golden/make_golden.py
The fixtures pin the CPU restatement (oracle/ksw2_oracle.c) and the CUDA path; the GPU
box only reads the JSON, never the reference tree.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from anchorwave_b200 import workloads as W  # noqa: E402

F = oracle
PEN = [(4, 2, 24, 1), (8, 2, 75, 1), (6, 1, 20, 0), (2, 3, 30, 1)]


def res_dict(r: oracle.KswResult):
    return {"max": r.max, "zdropped": r.zdropped, "max_q": r.max_q, "max_t": r.max_t, "mqe": r.mqe,
            "mqe_t": r.mqe_t, "mte": r.mte, "mte_q": r.mte_q, "score": r.score, "n_cigar": r.n_cigar,
            "reach_end": r.reach_end, "stopped": r.stopped, "cigar": r.cigar}


def ksw_cases():
    rng = np.random.default_rng(20261203)
    cases = []

    def add(name, q, t, pen=(4, 2, 24, 1), mm=-4, w=-1, zdrop=-1, end_bonus=0, extra=0, variant=0):
        q = np.asarray(q, dtype=np.uint8)
        t = np.asarray(t, dtype=np.uint8)
        flag = extra | (F.KSW_EZ_GENERIC_SC if (4 in q or 4 in t) else 0)
        cases.append(dict(name=name, query=W.to_ascii(q).decode(), target=W.to_ascii(t).decode(),
                          mismatch=mm, q=pen[0], e=pen[1], q2=pen[2], e2=pen[3], w=w, zdrop=zdrop,
                          end_bonus=end_bonus, flag=flag, variant=variant))

    # plain 5 kb pair (the single-pair workload), full and Singletrack
    q0, t0 = W.plain_pair(0)
    add("plain5kb", q0, t0)
    add("plain5kb-singletrack", q0, t0, variant=2)
    # batched-full-like pairs at small sizes
    for i in range(24):
        L = int(np.exp(rng.uniform(np.log(50), np.log(2500))))
        q, t = W.divergent_pair(rng, L, 0.01, 0.15, 4.0)
        add(f"batched-{i}", q, t, pen=PEN[i % 4])
    # banded (10% band) incl. long indels
    for i in range(10):
        L = int(rng.integers(800, 4000))
        t = W.random_dna(rng, L)
        q = W.mutate(rng, t, 0.03, 0.002, 40.0)
        add(f"banded-{i}", q, t, w=max(1, int(0.1 * min(len(q), len(t)))), pen=PEN[i % 4])
        add(f"banded-singletrack-{i}", q, t, w=max(1, int(0.1 * min(len(q), len(t)))), pen=PEN[i % 4],
            variant=2)
    # flags
    flags = [F.KSW_EZ_SCORE_ONLY, F.KSW_EZ_RIGHT, F.KSW_EZ_SEMIGLOBAL_END, F.KSW_EZ_REV_CIGAR,
             F.KSW_EZ_EXTZ_ONLY, F.KSW_EZ_APPROX_MAX, F.KSW_EZ_APPROX_MAX | F.KSW_EZ_APPROX_DROP]
    for i, fl in enumerate(flags):
        L = int(rng.integers(100, 1500))
        q, t = W.divergent_pair(rng, L, 0.02, 0.2, 4.0)
        add(f"flag-{fl:#x}", q, t, extra=fl, pen=PEN[i % 4])
        add(f"flag-{fl:#x}-band", q, t, extra=fl, w=int(rng.integers(5, 60)), pen=PEN[i % 4])
    # z-drop with a positive match score
    for i in range(4):
        L = int(rng.integers(200, 1200))
        q, t = W.divergent_pair(rng, L, 0.05, 0.3, 4.0)
        cases.append(dict(name=f"zdrop-{i}", query=W.to_ascii(q).decode(), target=W.to_ascii(t).decode(),
                          mat=[2 if a == b else -4 for a in range(5) for b in range(5)], q=4, e=2, q2=24, e2=1,
                          w=-1, zdrop=100, end_bonus=0, flag=F.KSW_EZ_EXTZ_ONLY if i % 2 else 0, variant=0))
    # edge cases
    add("len1-match", [2], [2])
    add("len1-mismatch", [1], [3])
    add("q1", [0], W.random_dna(rng, 300))
    add("t1", W.random_dna(rng, 300), [1])
    add("allN", [4] * 200, [4] * 230)
    qn, tn = W.divergent_pair(rng, 700, 0.05, 0.05, 3.0)
    qn = qn.copy(); qn[rng.integers(0, len(qn), 30)] = 4
    add("with-N", qn, tn)
    add("homopolymer", [0] * 400, [0] * 377)
    unit = W.random_dna(rng, 7)
    add("tandem", np.tile(unit, 60), np.tile(unit, 64))
    tt = W.random_dna(rng, 1500)
    add("long-gap", np.concatenate([tt[:300], tt[900:]]), tt)          # 600 bp deletion > long_thres
    add("long-ins", tt, np.concatenate([tt[:300], tt[900:]]))
    add("q-much-longer", W.random_dna(rng, 2000), W.random_dna(rng, 120))
    add("t-much-longer", W.random_dna(rng, 90), W.random_dna(rng, 2100))
    add("band-too-narrow", np.concatenate([tt[:700], tt[1200:]]), tt, w=100)
    add("band-zero", W.random_dna(rng, 300), W.random_dna(rng, 310), w=0)
    add("early-return", W.random_dna(rng, 50), W.random_dna(rng, 50), mm=-13, pen=(2, 2, 24, 1))
    return cases


def run_ksw(ref: oracle.Reference, c):
    mat = c.get("mat") or oracle.anchorwave_matrix(c["mismatch"])
    q = W.to_codes(c["query"].encode()).tobytes()
    t = W.to_codes(c["target"].encode()).tobytes()
    r = ref.ksw_extd2(q, t, mat, c["q"], c["e"], c["q2"], c["e2"], w=c["w"], zdrop=c["zdrop"],
                      end_bonus=c["end_bonus"], flag=c["flag"], variant=c["variant"])
    return res_dict(r)


def wfa_cases():
    rng = np.random.default_rng(777)
    cases = []
    for i in range(40):
        L = int(np.exp(rng.uniform(np.log(20), np.log(1500))))
        q, t = W.divergent_pair(rng, L, 0.005, 0.08, 4.0)
        cases.append(dict(name=f"wfa-{i}", query=W.to_ascii(q).decode(), target=W.to_ascii(t).decode(),
                          x=4, o1=4, e1=2, o2=24, e2=1, singletrack=bool(i % 3 == 2)))
    tt = W.random_dna(rng, 900)
    edge = [("wfa-gap", W.to_ascii(np.concatenate([tt[:200], tt[500:]])).decode(), W.to_ascii(tt).decode()),
            ("wfa-N", "ACGTNNNNACGT" * 20, "ACGTNNNACGTA" * 20),
            ("wfa-len1", "A", "C"), ("wfa-homopolymer", "A" * 150, "A" * 170),
            ("wfa-empty-query", "", "ACGTACGT"), ("wfa-empty-target", "ACGT", "")]
    for name, q, t in edge:
        for stk in (False, True):
            cases.append(dict(name=name + ("-st" if stk else ""), query=q, target=t, x=4, o1=4, e1=2, o2=24,
                              e2=1, singletrack=stk))
    # medium / low memory (piggyback traceback): long enough pairs that packed CIGARs fill
    # and move into blocks, tie-heavy penalties, and the edge cases
    rng2 = np.random.default_rng(4242)
    pens = [(4, 4, 2, 24, 1), (1, 0, 1, 0, 1), (2, 3, 1, 10, 1), (6, 8, 2, 75, 1)]
    for i in range(24):
        L = int(np.exp(rng2.uniform(np.log(20), np.log(4000))))
        q, t = W.divergent_pair(rng2, L, 0.005, 0.15, 4.0)
        x, o1, e1, o2, e2 = pens[i % len(pens)]
        cases.append(dict(name=f"wfa-mem-{i}", query=W.to_ascii(q).decode(), target=W.to_ascii(t).decode(),
                          x=x, o1=o1, e1=e1, o2=o2, e2=e2, singletrack=False, memory_mode=1 + i % 2))
    for name, q, t in edge:
        for mode in (1, 2):
            cases.append(dict(name=f"{name}-mem{mode}", query=q, target=t, x=4, o1=4, e1=2, o2=24, e2=1,
                              singletrack=bool(mode == 2), memory_mode=mode))
    return cases


def run_wfa(ref: oracle.Reference, c):
    st, score, ops = ref.wfa_align(c["target"].encode(), c["query"].encode(), c["x"], c["o1"], c["e1"], c["o2"],
                                   c["e2"], singletrack=c["singletrack"], memory_mode=c.get("memory_mode", 0))
    return {"status": st, "score": score, "ops": ops}


def summary_cases():
    """Interval pairs for the selector's sequence pass (summarizeSequencePair)."""
    rng = np.random.default_rng(9090)
    cases = []
    for i in range(20):
        L = int(np.exp(rng.uniform(np.log(10), np.log(6000))))
        q, t = W.divergent_pair(rng, L, 0.0, 0.2, 4.0)
        qa, ta = bytearray(W.to_ascii(q)), bytearray(W.to_ascii(t))
        if i % 4 == 1:
            for j in rng.integers(0, max(1, len(qa)), 5):
                if len(qa):
                    qa[j] = ord("N")
        if i % 4 == 2:
            for j in rng.integers(0, max(1, len(ta)), 40):
                if len(ta):
                    ta[j] = ord(chr(ta[j]).lower())  # lowercase counts as the same base
        cases.append(dict(name=f"sum-{i}", query=qa.decode(), target=ta.decode()))
    rnd = W.to_ascii(W.random_dna(rng, 3000)).decode()
    edge = [("sum-empty", "", ""), ("sum-empty-query", "", "ACGTACGTAC"), ("sum-len1", "A", "C"),
            ("sum-len9", "ACGTACGTA", "ACGTACGTA"), ("sum-len21", "ACGTTGCAACGTTGCAACGTA", "ACGTTGCAACGTTGCAACGTT"),
            ("sum-polyA", "A" * 5000, "A" * 4990), ("sum-N-runs", ("ACGTN" * 7 + "NNNN" + "ACGT" * 10) * 20, rnd[:900]),
            ("sum-identical", rnd, rnd), ("sum-dinucleotide", "AC" * 2000, "CA" * 2000),
            ("sum-iupac", "ACGTRYKMSWBDHVN" * 100, "acgtrykmswbdhvn" * 100)]
    for name, q, t in edge:
        cases.append(dict(name=name, query=q, target=t))
    return cases


def sketch_digest(side):
    import hashlib
    h = hashlib.sha256()
    for sk in side["sketches"]:
        for hv, pos in sk:
            h.update(int(hv).to_bytes(8, "little") + int(pos).to_bytes(4, "little"))
    return h.hexdigest()


def run_summary(ref: oracle.Reference, c):
    ident, sides = ref.sequence_summary(c["query"].encode(), c["target"].encode())
    return {"identical": ident,
            "sides": [{"fingerprint": s["fingerprint"], "ambiguous_fraction": s["ambiguous_fraction"],
                       "normalized_entropy": s["normalized_entropy"],
                       "low_complexity_fraction": s["low_complexity_fraction"],
                       "counts": [len(k) for k in s["sketches"]], "digest": sketch_digest(s)} for s in sides]}


def main():
    ref = oracle.Reference()
    ks = ksw_cases()
    for c in ks:
        c["result"] = run_ksw(ref, c)
    with open(os.path.join(HERE, "ksw2_golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "reference_isa": ref.isa, "block": ref.block,
                   "cases": ks}, f, separators=(",", ":"))
    wc = wfa_cases()
    for c in wc:
        c["result"] = run_wfa(ref, c)
    with open(os.path.join(HERE, "wfa_golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "reference_isa": ref.isa, "cases": wc}, f,
                  separators=(",", ":"))
    sc = summary_cases()
    for c in sc:
        c["result"] = run_summary(ref, c)
    with open(os.path.join(HERE, "summary_golden.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": sc}, f, separators=(",", ":"))
    print(f"wrote {len(ks)} KSW2, {len(wc)} WFA and {len(sc)} selector-summary golden cases "
          f"(reference ISA {ref.isa})")


if __name__ == "__main__":
    main()
