"""Seeded synthetic interval pairs with the shapes of the alignment-stage workloads.

The reference measures on B73/Mo17 maize genome intervals, which are not available
here; these generators stand in for them with the lengths, divergences and indel
models of the five workloads (plain 5 kb pair, batched 200 bp-20 kb KSW2 pairs,
batched 100 bp-10 kb WFA pairs, long banded 100 kb-1 Mb pairs, serving trace).

Sequences are returned as uint8 code arrays (A,C,G,T -> 0..3, other -> 4), the
encoding of ``encodeKswSequence`` (src/myImportandFunction/alignSlidingWindow.cpp:645-660).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List

import numpy as np

ASCII = np.frombuffer(b"ACGTN", dtype=np.uint8)
CODE = np.full(256, 4, dtype=np.uint8)
for _i, _c in enumerate(b"ACGT"):
    CODE[_c] = _i
    CODE[_c + 32] = _i  # lower case


def to_ascii(codes: np.ndarray) -> bytes:
    return ASCII[codes].tobytes()


def to_codes(seq: bytes) -> np.ndarray:
    return CODE[np.frombuffer(seq, dtype=np.uint8)]


@dataclass
class PairSet:
    name: str
    queries: List[np.ndarray]
    targets: List[np.ndarray]
    band: List[int]  # KSW2 band width per pair (-1 = full)

    def __len__(self):
        return len(self.queries)

    def cells(self) -> int:
        return int(sum(int(len(q)) * int(len(t)) for q, t in zip(self.queries, self.targets)))


def random_dna(rng: np.random.Generator, n: int) -> np.ndarray:
    return rng.integers(0, 4, size=n, dtype=np.uint8)


def mutate(rng: np.random.Generator, target: np.ndarray, sub_rate: float, indel_rate: float,
           indel_mean: float) -> np.ndarray:
    """Walk the target left to right: per base a substitution (uniform other base) with
    probability sub_rate, an indel start (insertion or deletion, 1/2 each) with
    probability indel_rate, lengths ~ Geometric(mean indel_mean)."""
    n = len(target)
    u = rng.random(n)
    is_sub = u < sub_rate
    is_indel = (u >= sub_rate) & (u < sub_rate + indel_rate)
    out = target.copy()
    subs = np.nonzero(is_sub)[0]
    out[subs] = (out[subs] + rng.integers(1, 4, size=len(subs), dtype=np.uint8)) % 4
    pos = np.nonzero(is_indel)[0]
    if len(pos) == 0:
        return out
    p = 1.0 / max(indel_mean, 1.0)
    lens = rng.geometric(p, size=len(pos))
    ins = rng.random(len(pos)) < 0.5
    pieces = []
    cur = 0
    for i, L, is_ins in zip(pos, lens, ins):
        if i < cur:
            continue
        pieces.append(out[cur:i])
        if is_ins:
            pieces.append(random_dna(rng, int(L)))
            cur = i
        else:
            cur = min(n, i + int(L))
    pieces.append(out[cur:])
    return np.concatenate(pieces) if pieces else out


def plain_pair(seed: int = 0, length: int = 5000):
    """5,000 bp target; query with 5% substitutions, 1% indels (mean 3) and one 500 bp deletion."""
    rng = np.random.default_rng(seed)
    t = random_dna(rng, length)
    qm = mutate(rng, t, 0.05, 0.01, 3.0)
    if len(qm) > 600:
        at = int(rng.integers(50, len(qm) - 550))
        qm = np.concatenate([qm[:at], qm[at + 500:]])
    return qm, t


def plain_set(n: int = 1, seed0: int = 0) -> PairSet:
    qs, ts = [], []
    for s in range(seed0, seed0 + n):
        q, t = plain_pair(s)
        qs.append(q)
        ts.append(t)
    return PairSet("plain-5kb", qs, ts, [-1] * n)


def divergent_pair(rng: np.random.Generator, tlen: int, dmin: float, dmax: float, indel_mean: float):
    d = rng.uniform(dmin, dmax)
    t = random_dna(rng, tlen)
    q = mutate(rng, t, 0.8 * d, 0.2 * d, indel_mean)
    if len(q) == 0:
        q = random_dna(rng, 1)
    return q, t


def batched_full_set(n: int = 4096, seed: int = 1, lmin: int = 200, lmax: int = 20000) -> PairSet:
    """n pairs, target length log-uniform [lmin, lmax], divergence U(1%,15%), 80% substitutions,
    20% indels with geometric lengths of mean 4."""
    rng = np.random.default_rng(seed)
    qs, ts = [], []
    for _ in range(n):
        L = int(math.floor(math.exp(rng.uniform(math.log(lmin), math.log(lmax)))))
        q, t = divergent_pair(rng, max(L, 1), 0.01, 0.15, 4.0)
        qs.append(q)
        ts.append(t)
    return PairSet(f"batched-full-{n}x{lmin}-{lmax}", qs, ts, [-1] * n)


def batched_wfa_set(n: int = 16384, seed: int = 2, lmin: int = 100, lmax: int = 10000) -> PairSet:
    """n pairs, length log-uniform [lmin, lmax], divergence U(0.5%,5%), same 80/20 split."""
    rng = np.random.default_rng(seed)
    qs, ts = [], []
    for _ in range(n):
        L = int(math.floor(math.exp(rng.uniform(math.log(lmin), math.log(lmax)))))
        q, t = divergent_pair(rng, max(L, 1), 0.005, 0.05, 4.0)
        qs.append(q)
        ts.append(t)
    return PairSet(f"batched-wfa-{n}x{lmin}-{lmax}", qs, ts, [-1] * n)


def repeat_query(rng: np.random.Generator, t: np.ndarray, long_indels=(5, 20),
                 long_max: int = 50000, element: int = 5000) -> np.ndarray:
    """Long-interval query: 30% of the length replaced by repeat structure (copies of one
    random element at 85-95% identity, tandem repeats of 2-50 bp units), 3% substitutions,
    5-20 long indels of length U(1, long_max)."""
    L = len(t)
    q = t.copy()
    elem = random_dna(rng, min(element, max(L // 10, 10)))
    budget = int(0.3 * L)
    while budget > 0:
        if rng.random() < 0.5:
            ident = rng.uniform(0.85, 0.95)
            piece = mutate(rng, elem, 1.0 - ident, 0.0, 1.0)
        else:
            unit = random_dna(rng, int(rng.integers(2, 51)))
            piece = np.tile(unit, max(1, int(rng.integers(5, 200))))
        piece = piece[: min(len(piece), budget)]
        at = int(rng.integers(0, max(1, L - len(piece))))
        q[at:at + len(piece)] = piece
        budget -= len(piece)
    q = mutate(rng, q, 0.03, 0.0, 1.0)
    for _ in range(int(rng.integers(long_indels[0], long_indels[1] + 1))):
        ln = int(rng.integers(1, long_max + 1))
        at = int(rng.integers(0, max(1, len(q))))
        if rng.random() < 0.5:
            q = np.concatenate([q[:at], random_dna(rng, ln), q[at:]])
        else:
            q = np.concatenate([q[:at], q[at + ln:]])
        if len(q) == 0:
            q = random_dna(rng, 1)
    return q


def long_banded_set(n: int = 64, seed: int = 3, lmin: int = 100_000, lmax: int = 1_000_000,
                    long_max: int = 50_000, band_frac: float = 0.1) -> PairSet:
    """n long pairs, target length U(lmin, lmax); band = floor(band_frac * min(qlen, tlen))."""
    rng = np.random.default_rng(seed)
    qs, ts, bands = [], [], []
    for _ in range(n):
        L = int(rng.integers(lmin, lmax + 1))
        t = random_dna(rng, L)
        q = repeat_query(rng, t, long_max=long_max, element=min(5000, max(L // 20, 20)))
        qs.append(q)
        ts.append(t)
        bands.append(int(math.floor(band_frac * min(len(q), len(t)))))
    return PairSet(f"long-banded-{n}x{lmin}-{lmax}", qs, ts, bands)


def band_cells(qlen: int, tlen: int, w: int) -> int:
    """Sum over anti-diagonals of the in-band cell count en0-st0+1 (ksw2_extd2_sse.c:147-150),
    up to the first empty band (where the reference stops)."""
    if w < 0 or w > max(qlen, tlen):
        w = max(qlen, tlen)
    r = np.arange(qlen + tlen - 1, dtype=np.int64)
    st = np.maximum(np.maximum(0, r - qlen + 1), (r - w + 1) >> 1)
    en = np.minimum(np.minimum(tlen - 1, r), (r + w) >> 1)
    bad = np.nonzero(st > en)[0]
    if len(bad):
        st, en = st[: bad[0]], en[: bad[0]]
    return int((en - st + 1).sum())


def band_reaches_end(qlen: int, tlen: int, w: int) -> bool:
    """True when no anti-diagonal's band is empty (ksw2_extd2_sse.c:151-154); otherwise the
    reference stops at the first empty one and reports zdropped = 1 with no CIGAR."""
    if w < 0 or w > max(qlen, tlen):
        return True
    r = np.arange(qlen + tlen - 1, dtype=np.int64)
    st = np.maximum(np.maximum(0, r - qlen + 1), (r - w + 1) >> 1)
    en = np.minimum(np.minimum(tlen - 1, r), (r + w) >> 1)
    return bool((st <= en).all())


@dataclass
class Request:
    id: int
    method: int      # 0 KSW2 (full or banded), 1 KSW2 Singletrack, 2 WFA, 3 WFA Singletrack
    band: int
    query: bytes     # ASCII
    target: bytes


def serving_trace(n: int, seed: int = 4, lmin: int = 50, lmax: int = 500_000, repeat_frac: float = 0.1,
                  band_above: int = 20_000) -> List[Request]:
    """Interval requests of the serving workload: length ~ LogNormal(median 2 kb, sigma 1)
    clipped to [lmin, lmax]; divergence and indels as the batched-full workload; repeat_frac of
    them carry long-interval repeat structure.  Engine per request (a stand-in for AnchorWave's
    exact-tier/fallback-tier selector, which stays on the caller's side): low-divergence
    intervals up to 10 kb (d <= 5%, where the wavefront score stays small) go to WFA, intervals
    longer than band_above to banded KSW2 with a 10% band, the rest to full KSW2."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L = int(np.clip(np.exp(rng.normal(math.log(2000), 1.0)), lmin, lmax))
        d = rng.uniform(0.01, 0.15)
        t = random_dna(rng, L)
        if rng.random() < repeat_frac and L >= 200:
            q = repeat_query(rng, t, long_indels=(0, 2), long_max=max(1, L // 20), element=max(20, L // 10))
            d = 1.0
        else:
            q = mutate(rng, t, 0.8 * d, 0.2 * d, 4.0)
            if len(q) == 0:
                q = random_dna(rng, 1)
        method = 2 if (d <= 0.05 and L <= 10_000) else 0
        band = int(0.1 * min(len(q), len(t))) if (method == 0 and max(len(q), len(t)) > band_above) else -1
        out.append(Request(i, method, band, to_ascii(q), to_ascii(t)))
    return out
