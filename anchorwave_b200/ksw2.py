"""Host-side mirror of AnchorWave's KSW2 interface, running on the B200 kernels.

Two layers, both reached through libaw_b200.so's C ABI:

* the minimap2 entry points (minimap2/ksw2.h:91-107, ksw2_singletrack.hpp:17-46):
  :func:`ksw_extd2`, :func:`ksw_extd2_singletrack`, plus the batched form
  :func:`ksw_extd2_batch` and :class:`KswPlan` (device-resident batch);
* the AnchorWave callers that sit on that boundary
  (src/myImportandFunction/alignSlidingWindow.cpp): :func:`minimap2_alignment`
  (:241-332), :func:`alignment_minimap2` (semiglobal end, :334-431),
  :func:`align_sliding_window_minimap2` (banded, :800-890), :func:`ksw2_score_only`
  (:723-796), :func:`align_ksw2_singletrack` / ``_banded`` (:892-1013) and
  :func:`score_gapped_two_piece_affine` (:677-721) -- same names, argument meaning
  (AnchorWave's negative penalties) and error behaviour.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from ._lib import AwError, CertResultC, KswExtz, WindowResultC, check, last_error, lib, libc

KSW_NEG_INF = -0x40000000
KSW_EZ_SCORE_ONLY = 0x01
KSW_EZ_RIGHT = 0x02
KSW_EZ_GENERIC_SC = 0x04
KSW_EZ_APPROX_MAX = 0x08
KSW_EZ_APPROX_DROP = 0x10
KSW_EZ_EXTZ_ONLY = 0x40
KSW_EZ_REV_CIGAR = 0x80
KSW_EZ_SEMIGLOBAL_END = 0x800
KSW_EZ_SINGLETRACK = 0x1000

_ENC = np.full(256, 4, dtype=np.uint8)
for _i, _c in enumerate(b"ACGT"):
    _ENC[_c] = _i
    _ENC[_c + 32] = _i


@dataclass
class KswResult:
    """The comparable ksw_extz_t fields plus the CIGAR (BAM-packed words)."""
    max: int
    zdropped: int
    max_q: int
    max_t: int
    mqe: int
    mqe_t: int
    mte: int
    mte_q: int
    score: int
    n_cigar: int
    reach_end: int
    stopped: int
    cigar: List[int] = field(default_factory=list)

    def key(self):
        return (self.max, self.zdropped, self.max_q, self.max_t, self.mqe, self.mqe_t, self.mte,
                self.mte_q, self.score, self.n_cigar, self.reach_end, self.stopped, tuple(self.cigar))


def _take(ez: KswExtz) -> KswResult:
    cig = list(np.ctypeslib.as_array(ez.cigar, shape=(ez.n_cigar,))) if ez.n_cigar > 0 and ez.cigar else []
    res = KswResult(ez.max, ez.zdropped, ez.max_q, ez.max_t, ez.mqe, ez.mqe_t, ez.mte, ez.mte_q,
                    ez.score, ez.n_cigar, ez.reach_end, ez.stopped, [int(c) for c in cig])
    if ez.cigar:
        libc.free(C.cast(ez.cigar, C.c_void_p))
        ez.cigar = None
        ez.m_cigar = 0
    return res


def _codes(seq) -> np.ndarray:
    if isinstance(seq, np.ndarray):
        return np.ascontiguousarray(seq, dtype=np.uint8)
    if isinstance(seq, str):
        seq = seq.encode()
    return np.frombuffer(bytes(seq), dtype=np.uint8)


def _mat(mat) -> C.Array:
    vals = list(mat)
    return (C.c_int8 * len(vals))(*vals)


def ksw_extd2(query, target, mat, q, e, q2, e2, w=-1, zdrop=-1, end_bonus=0, flag=0, m=5) -> KswResult:
    """One ksw_extd2 call on the GPU (sequences as 0..m-1 codes)."""
    qa, ta = _codes(query), _codes(target)
    ez = KswExtz()
    lib.ksw_extd2_gpu(None, len(qa), qa.ctypes.data, len(ta), ta.ctypes.data, m, _mat(mat), q, e, q2, e2,
                      w, zdrop, end_bonus, flag, C.byref(ez))
    return _take(ez)


def ksw_extd2_singletrack(query, target, mat, q, e, q2, e2, w=-1, zdrop=-1, end_bonus=0, flag=0,
                          m=5) -> KswResult:
    qa, ta = _codes(query), _codes(target)
    ez = KswExtz()
    lib.ksw_extd2_singletrack_gpu(None, len(qa), qa.ctypes.data, len(ta), ta.ctypes.data, m, _mat(mat), q, e,
                                  q2, e2, w, zdrop, end_bonus, flag, C.byref(ez))
    return _take(ez)


def ksw_extd2_singletrack_sse(query, target, mat, q, e, q2, e2, w=-1, zdrop=-1, end_bonus=0, flag=0,
                              m=5) -> KswResult:
    """ksw_extd2_singletrack_sse (minimap2/ksw2_singletrack.cpp:202-626), the Singletrack entry of
    builds without AVX2, on the GPU."""
    qa, ta = _codes(query), _codes(target)
    ez = KswExtz()
    lib.ksw_extd2_singletrack_sse_gpu(None, len(qa), qa.ctypes.data, len(ta), ta.ctypes.data, m, _mat(mat), q, e,
                                      q2, e2, w, zdrop, end_bonus, flag, C.byref(ez))
    return _take(ez)


def _ptr_array(arrs: Sequence[np.ndarray]):
    ptrs = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    return ptrs


def ksw_extd2_batch(queries, targets, mat, q, e, q2, e2, w=None, zdrop=-1, end_bonus=0, flag=0,
                    m=5) -> List[KswResult]:
    """n independent ksw_extd2 calls in one submission (aw_ksw_extd2_batch)."""
    qs = [_codes(x) for x in queries]
    ts = [_codes(x) for x in targets]
    n = len(qs)
    if n == 0:
        return []
    ql = np.array([len(x) for x in qs], dtype=np.int32)
    tl = np.array([len(x) for x in ts], dtype=np.int32)
    wa = None if w is None else np.ascontiguousarray(np.broadcast_to(np.asarray(w, dtype=np.int32), (n,)))
    ez = (KswExtz * n)()
    rc = lib.aw_ksw_extd2_batch(n, ql.ctypes.data, _ptr_array(qs), tl.ctypes.data, _ptr_array(ts),
                                None if wa is None else wa.ctypes.data, m, _mat(mat), q, e, q2, e2, zdrop,
                                end_bonus, flag, ez)
    out = [_take(ez[i]) for i in range(n)]
    check(rc, "aw_ksw_extd2_batch")
    return out


class BatchCall:
    """A prepared aw_ksw_extd2_batch call: argument arrays built once, so timing run() measures
    the C-ABI call itself (host staging, H2D, kernels, D2H, CIGAR buffers in ksw_extz_t)."""

    def __init__(self, queries, targets, mat, q, e, q2, e2, w=None, zdrop=-1, end_bonus=0, flag=0, m=5):
        self.qs = [_codes(x) for x in queries]
        self.ts = [_codes(x) for x in targets]
        self.n = len(self.qs)
        self.ql = np.array([len(x) for x in self.qs], dtype=np.int32)
        self.tl = np.array([len(x) for x in self.ts], dtype=np.int32)
        self.qp, self.tp = _ptr_array(self.qs), _ptr_array(self.ts)
        self.w = None if w is None else np.ascontiguousarray(np.broadcast_to(np.asarray(w, dtype=np.int32), (self.n,)))
        self.args = (m, _mat(mat), q, e, q2, e2, zdrop, end_bonus, flag)
        self.ez = (KswExtz * self.n)()

    def run(self) -> int:
        m, mat, q, e, q2, e2, zdrop, end_bonus, flag = self.args
        rc = lib.aw_ksw_extd2_batch(self.n, self.ql.ctypes.data, self.qp, self.tl.ctypes.data, self.tp,
                                    None if self.w is None else self.w.ctypes.data, m, mat, q, e, q2, e2, zdrop,
                                    end_bonus, flag, self.ez)
        check(rc, "aw_ksw_extd2_batch")
        return rc

    def cigar_words(self) -> int:
        return int(sum(self.ez[i].n_cigar for i in range(self.n)))

    def results(self) -> List[KswResult]:
        """Converts (and releases) the last run's ksw_extz_t array."""
        return [_take(self.ez[i]) for i in range(self.n)]

    def release(self):
        for i in range(self.n):
            if self.ez[i].cigar:
                libc.free(C.cast(self.ez[i].cigar, C.c_void_p))
                self.ez[i].cigar = None
                self.ez[i].m_cigar = 0


class KswPlan:
    """A batch kept resident on the device (aw_ksw_plan_*): upload once, execute many times."""

    def __init__(self, queries, targets, mat, q, e, q2, e2, w=None, zdrop=-1, end_bonus=0, flag=0, m=5):
        self.qs = [_codes(x) for x in queries]
        self.ts = [_codes(x) for x in targets]
        self.n = len(self.qs)
        self.ql = np.array([len(x) for x in self.qs], dtype=np.int32)
        self.tl = np.array([len(x) for x in self.ts], dtype=np.int32)
        self.w = None if w is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(w, dtype=np.int32), (self.n,)))
        self._mat = _mat(mat)
        self.h = lib.aw_ksw_plan_new(self.n, self.ql.ctypes.data, self.tl.ctypes.data,
                                     None if self.w is None else self.w.ctypes.data, m, self._mat, q, e, q2, e2,
                                     zdrop, end_bonus, flag)
        if not self.h:
            raise AwError(f"aw_ksw_plan_new failed: {last_error()}")

    def upload(self):
        check(lib.aw_ksw_plan_upload(self.h, _ptr_array(self.qs), _ptr_array(self.ts)), "aw_ksw_plan_upload")

    def execute(self) -> float:
        ms = C.c_float(0.0)
        check(lib.aw_ksw_plan_execute(self.h, C.byref(ms)), "aw_ksw_plan_execute")
        return ms.value

    def uses_graph(self) -> bool:
        """True when the last execute replayed the plan's CUDA graph."""
        return bool(lib.aw_ksw_plan_graph(self.h))

    def timing(self):
        """(dp_ms, backtrack_ms) of the last execute, CUDA events on the plan's stream."""
        dp, bt = C.c_float(0.0), C.c_float(0.0)
        check(lib.aw_ksw_plan_timing(self.h, C.byref(dp), C.byref(bt)), "aw_ksw_plan_timing")
        return dp.value, bt.value

    def download(self) -> List[KswResult]:
        ez = (KswExtz * self.n)()
        rc = lib.aw_ksw_plan_download(self.h, ez)
        out = [_take(ez[i]) for i in range(self.n)]
        check(rc, "aw_ksw_plan_download")
        return out

    def stats(self):
        cells, tb = C.c_int64(0), C.c_int64(0)
        waves, launches = C.c_int(0), C.c_int(0)
        check(lib.aw_ksw_plan_stats(self.h, C.byref(cells), C.byref(tb), C.byref(waves), C.byref(launches)),
              "aw_ksw_plan_stats")
        return {"cells": cells.value, "tb_bytes": tb.value, "waves": waves.value, "launches": launches.value}

    def routes(self):
        """Pairs per kernel: {"strip": full-matrix strip kernel, "banded": banded strip kernel,
        "exact": exact anti-diagonal kernel}."""
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        check(lib.aw_ksw_plan_routes(self.h, C.byref(a), C.byref(b), C.byref(c)), "aw_ksw_plan_routes")
        return {"strip": a.value, "banded": b.value, "exact": c.value}

    def close(self):
        if self.h:
            lib.aw_ksw_plan_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_traceback_budget(nbytes: int):
    lib.aw_set_traceback_budget(int(nbytes))


def release_thread_buffers():
    """Free the device/pinned buffers this thread's batch calls keep pooled."""
    lib.aw_release_thread_buffers()


def set_deadline(seconds: float = 0.0):
    """Cooperative stop for this thread's KSW2 calls: pairs still running `seconds` from
    now come back with stopped=1 (AnchorWave's ScopedKswDeadline); <= 0 clears it."""
    lib.aw_ksw_set_deadline(float(seconds))


def set_stop_antidiagonal(interval: int = 256, antidiagonal: int = -1):
    """Deterministic stop for this thread: as a ksw2 progress callback that returns 0 at
    the first probed anti-diagonal >= antidiagonal; < 0 clears it."""
    lib.aw_ksw_set_stop_antidiagonal(int(interval), int(antidiagonal))


class deadline:
    """Context manager mirroring ScopedKswDeadline (alignSlidingWindow.cpp:612-638)."""

    def __init__(self, seconds: float):
        self.seconds = seconds

    def __enter__(self):
        set_deadline(self.seconds)
        return self

    def __exit__(self, *exc):
        set_deadline(0.0)
        return False


def set_band_columns(columns: int = 0):
    """Target columns per lane of the banded kernel: 4, 8, or 0 to choose per batch."""
    lib.aw_set_band_columns(int(columns))


def set_full_pair_routing(enabled: bool = True):
    """aw_set_full_pair_routing: critical-path full-matrix pairs on the banded kernel (default)."""
    lib.aw_set_full_pair_routing(1 if enabled else 0)


def set_tuning(large_warps: int = 0, large_tlen_threshold: int = 0):
    lib.aw_set_tuning(int(large_warps), int(large_tlen_threshold))


# ---- AnchorWave callers on the KSW2 boundary -------------------------------------

def anchorwave_matrix(mismatching_penalty: int) -> List[int]:
    """5x5 matrix: match 0, every unequal pair (N included) -|mismatch| (alignSlidingWindow.cpp:245-255)."""
    b = mismatching_penalty if mismatching_penalty < 0 else -mismatching_penalty
    return [0 if i == j else b for i in range(5) for j in range(5)]


def encode(seq: str) -> Tuple[np.ndarray, int]:
    """encodeKswSequence (alignSlidingWindow.cpp:645-660): ACGT -> 0..3, other -> 4 + GENERIC_SC."""
    codes = _ENC[np.frombuffer(seq.encode() if isinstance(seq, str) else bytes(seq), dtype=np.uint8)]
    return codes, (KSW_EZ_GENERIC_SC if (codes == 4).any() else 0)


def decode_cigar(cigar: Sequence[int], dna_q: str, dna_d: str) -> Tuple[str, str, int, int]:
    """CIGAR -> gapped rows (alignSlidingWindow.cpp:307-324): M/=/X copy both, I query only, D target only."""
    aq, ad = [], []
    qp = tp = 0
    for c in cigar:
        ln, op = c >> 4, c & 0xF
        if op in (0, 7, 8):
            aq.append(dna_q[qp:qp + ln]); ad.append(dna_d[tp:tp + ln]); qp += ln; tp += ln
        elif op == 1:
            aq.append(dna_q[qp:qp + ln]); ad.append("-" * ln); qp += ln
        elif op == 2:
            aq.append("-" * ln); ad.append(dna_d[tp:tp + ln]); tp += ln
        else:
            raise ValueError(f"unexpected CIGAR op {op}")
    return "".join(aq), "".join(ad), qp, tp


def score_gapped_two_piece_affine(aln_q: str, aln_d: str, mismatching_penalty: int, open1: int, extend1: int,
                                  open2: int, extend2: int) -> int:
    """scoreGappedTwoPieceAffineAlignment (alignSlidingWindow.cpp:677-721); penalties are negative."""
    if len(aln_q) != len(aln_d):
        raise RuntimeError("KSW2 returned alignment rows with different lengths")
    score = 0
    col = 0
    n = len(aln_q)
    while col < n:
        qg, dg = aln_q[col] == "-", aln_d[col] == "-"
        if qg and dg:
            raise RuntimeError("KSW2 returned an alignment column with two gaps")
        if qg or dg:
            end = col + 1
            while end < n and (aln_q[end] == "-") == qg and (aln_d[end] == "-") != qg:
                end += 1
            ln = end - col
            score += max(open1 + extend1 * ln, open2 + extend2 * ln)
            col = end
            continue
        if aln_q[col] != aln_d[col]:
            score += mismatching_penalty
        col += 1
    return score


def minimap2_alignment(dna_q: str, dna_d: str, matching_score: int, mismatching_penalty: int, open1: int,
                       extend1: int, open2: int, extend2: int) -> Tuple[int, str, str]:
    """minimap2AlignmentWithArena (alignSlidingWindow.cpp:241-332): global KSW2 with CIGAR.
    Returns (ez.score, aligned query, aligned reference)."""
    qs, f1 = encode(dna_q)
    ts, f2 = encode(dna_d)
    res = ksw_extd2(qs, ts, anchorwave_matrix(mismatching_penalty), -open1, -extend1, -open2, -extend2,
                    -1, -1, 0, f1 | f2)
    aq, ad, qp, tp = decode_cigar(res.cigar, dna_q, dna_d)
    assert qp == len(dna_q) and tp == len(dna_d)
    return res.score, aq, ad


def alignment_minimap2(dna_q: str, dna_d: str, matching_score: int, mismatching_penalty: int, open1: int,
                       extend1: int, open2: int, extend2: int) -> Tuple[int, str, str, int, int]:
    """alignmentMinimap2WithArena (alignSlidingWindow.cpp:334-431): traceback from the better end
    (KSW_EZ_SEMIGLOBAL_END).  Returns (score, aln_q, aln_d, endPositionq, endPositiont)."""
    qs, f1 = encode(dna_q)
    ts, f2 = encode(dna_d)
    res = ksw_extd2(qs, ts, anchorwave_matrix(mismatching_penalty), -open1, -extend1, -open2, -extend2,
                    -1, -1, 0, KSW_EZ_SEMIGLOBAL_END | f1 | f2)
    if res.mqe > res.mte:
        end_t, end_q = res.mqe_t + 1, len(dna_q)
    else:
        end_t, end_q = len(dna_d), res.mte_q + 1
    aq, ad, qp, tp = decode_cigar(res.cigar, dna_q, dna_d)
    assert qp == end_q and tp == end_t
    return res.score, aq, ad, end_q, end_t


def align_sliding_window_minimap2(dna_q: str, dna_d: str, sliding_window_size: int, mismatching_penalty: int,
                                  open1: int, extend1: int, open2: int, extend2: int) -> Tuple[int, str, str]:
    """alignSlidingWindow_minimap2 (alignSlidingWindow.cpp:800-890): full (-1) or banded KSW2,
    re-scored with the two-piece objective."""
    qs, f1 = encode(dna_q)
    ts, f2 = encode(dna_d)
    res = ksw_extd2(qs, ts, anchorwave_matrix(mismatching_penalty), -open1, -extend1, -open2, -extend2,
                    int(sliding_window_size), -1, 0, f1 | f2)
    aq, ad, qp, tp = decode_cigar(res.cigar, dna_q, dna_d)
    assert qp == len(dna_q) and tp == len(dna_d)
    return score_gapped_two_piece_affine(aq, ad, mismatching_penalty, open1, extend1, open2, extend2), aq, ad


def ksw2_score_only(dna_q: str, dna_d: str, mismatching_penalty: int, open1: int, extend1: int, open2: int,
                    extend2: int) -> Tuple[int, bool]:
    """ksw2ScoreOnly (alignSlidingWindow.cpp:723-796): (score, stopped)."""
    if not dna_q or not dna_d:
        ln = max(len(dna_q), len(dna_d))
        return max(open1 + extend1 * ln, open2 + extend2 * ln), False
    qs, f1 = encode(dna_q)
    ts, f2 = encode(dna_d)
    res = ksw_extd2(qs, ts, anchorwave_matrix(mismatching_penalty), -open1, -extend1, -open2, -extend2,
                    -1, -1, 0, KSW_EZ_SCORE_ONLY | f1 | f2)
    return res.score, bool(res.stopped)


def align_ksw2_singletrack_banded(dna_q: str, dna_d: str, band_width: int, mismatching_penalty: int,
                                  open1: int, extend1: int, open2: int, extend2: int) -> Tuple[int, str, str, bool]:
    """alignKsw2SingletrackImpl (alignSlidingWindow.cpp:892-990): (score, aln_q, aln_d, stopped).
    Score is KSW_NEG_INF with empty rows when the traceback fails."""
    if not dna_q or not dna_d:
        ln = max(len(dna_q), len(dna_d))
        aq = dna_q if dna_q else "-" * ln
        ad = dna_d if dna_d else "-" * ln
        return max(open1 + extend1 * ln, open2 + extend2 * ln), aq, ad, False
    if band_width < -1:
        raise ValueError("KSW2-Singletrack band width must be -1..INT_MAX")
    qs, f1 = encode(dna_q)
    ts, f2 = encode(dna_d)
    res = ksw_extd2_singletrack(qs, ts, anchorwave_matrix(mismatching_penalty), -open1, -extend1, -open2,
                                -extend2, int(band_width), -1, 0, f1 | f2)
    if res.stopped or res.zdropped:
        return KSW_NEG_INF, "", "", bool(res.stopped)
    try:
        aq, ad, qp, tp = decode_cigar(res.cigar, dna_q, dna_d)
    except ValueError:
        return KSW_NEG_INF, "", "", False
    if qp != len(dna_q) or tp != len(dna_d):
        return KSW_NEG_INF, "", "", False
    return score_gapped_two_piece_affine(aq, ad, mismatching_penalty, open1, extend1, open2, extend2), aq, ad, False


def align_ksw2_singletrack(dna_q: str, dna_d: str, mismatching_penalty: int, open1: int, extend1: int,
                           open2: int, extend2: int):
    """alignKsw2Singletrack (alignSlidingWindow.cpp:992-1003): unbanded Singletrack."""
    return align_ksw2_singletrack_banded(dna_q, dna_d, -1, mismatching_penalty, open1, extend1, open2, extend2)


# ---- score-certified KSW2 (alignSlidingWindow.cpp:1197-1400) -------------------------------

CERT_COMPLETED, CERT_TIME_LIMIT, CERT_NOT_CERTIFIED, CERT_FAILED = "Completed", "TimeLimit", "NotCertified", "Failed"


@dataclass
class CertifiedResult:
    """anchorwave::Ksw2CertifiedResult (alignSlidingWindow.h:38-49) plus the alignment rows,
    which stay empty unless the status is Completed."""
    status: str = CERT_FAILED
    score: int = 0
    optimal_score: int = 0
    final_band_width: int = -1
    traceback_attempts: int = 0
    best_effort_query_alignment: str = ""
    best_effort_reference_alignment: str = ""
    alignment_q: str = ""
    alignment_d: str = ""


def _seq_arrays(seqs):
    """ASCII sequences as (pointer array, lengths, keep-alive buffers) for the C entries."""
    bufs = [C.create_string_buffer(x.encode() if isinstance(x, str) else bytes(x),
                                   len(x) + 1) for x in seqs]
    ptrs = (C.c_void_p * max(1, len(bufs)))(*[C.addressof(b) for b in bufs])
    lens = np.array([len(x) for x in seqs] or [0], dtype=np.int64)
    return ptrs, lens, bufs


_CERT_STATUS = {0: CERT_COMPLETED, 1: CERT_TIME_LIMIT, 2: CERT_NOT_CERTIFIED, 3: CERT_FAILED}


def _text(ptr, n) -> str:
    return C.string_at(ptr, n).decode() if ptr and n > 0 else ""


def align_score_certified_ksw2_batch(pairs, initial_band_width, maximum_band_width,
                                     mismatching_penalty: int, open1: int, extend1: int, open2: int, extend2: int,
                                     maximum_runtime_seconds: float = 0.0,
                                     precomputed_optimal_scores=None) -> List[CertifiedResult]:
    """alignScoreCertifiedKsw2 (alignSlidingWindow.cpp:1197-1400) for many intervals at once,
    through aw_align_score_certified_batch: one score-only batch gives every optimal score,
    then the next band of every interval not yet certified runs as one banded batch, until
    a band's re-scored alignment reaches the optimal score.  Each interval gets the result
    a call of its own would give.  The selector's chained traceback (a selection plan) stays
    on the caller's side.  Penalties are AnchorWave's (negative); maximum_runtime_seconds > 0
    arms the cooperative stop."""
    n = len(pairs)
    if n == 0:
        return []
    qp, ql, qb = _seq_arrays([p[0] for p in pairs])
    rp, rl, rb = _seq_arrays([p[1] for p in pairs])
    pre = None
    if precomputed_optimal_scores is not None:
        pre = np.ascontiguousarray(np.asarray(precomputed_optimal_scores, dtype=np.int64))
    ib = np.broadcast_to(np.asarray(initial_band_width, dtype=np.int64), (n,)).copy()
    mb = np.broadcast_to(np.asarray(maximum_band_width, dtype=np.int64), (n,)).copy()
    out = (CertResultC * n)()
    rc = lib.aw_align_score_certified_batch(n, qp, ql.ctypes.data, rp, rl.ctypes.data, ib.ctypes.data,
                                            mb.ctypes.data, mismatching_penalty, open1, extend1, open2,
                                            extend2, float(maximum_runtime_seconds or 0.0),
                                            pre.ctypes.data if pre is not None else None, out)
    res = []
    for o in out:
        r = CertifiedResult(status=_CERT_STATUS[o.status], score=o.score, optimal_score=o.optimal_score,
                            final_band_width=o.final_band_width, traceback_attempts=o.traceback_attempts,
                            alignment_q=_text(o.alignment_q, o.alignment_len),
                            alignment_d=_text(o.alignment_d, o.alignment_len),
                            best_effort_query_alignment=_text(o.best_effort_q, o.best_effort_len),
                            best_effort_reference_alignment=_text(o.best_effort_d, o.best_effort_len))
        lib.aw_certified_result_free(C.byref(o))
        res.append(r)
    check(rc, "aw_align_score_certified_batch")
    return res


def align_score_certified_ksw2(dna_q: str, dna_d: str, initial_band_width: int, maximum_band_width: int,
                               mismatching_penalty: int, open1: int, extend1: int, open2: int, extend2: int,
                               maximum_runtime_seconds: float = 0.0, precomputed_optimal_score=None) -> CertifiedResult:
    """alignScoreCertifiedKsw2 (alignSlidingWindow.cpp:1197-1400) for one interval."""
    pre = None if precomputed_optimal_score is None else [precomputed_optimal_score]
    return align_score_certified_ksw2_batch([(dna_q, dna_d)], initial_band_width, maximum_band_width,
                                            mismatching_penalty, open1, extend1, open2, extend2,
                                            maximum_runtime_seconds, pre)[0]


# ---- sliding-window semiglobal alignment (alignSlidingWindow.cpp:457-590) ----------------

def align_sliding_window_batch(pairs, sliding_window_size, matching_score: int, mismatching_penalty: int,
                               open1: int, extend1: int, open2: int, extend2: int) -> List[Tuple[int, str, str]]:
    """alignSlidingWindow (alignSlidingWindow.cpp:457-590) for many intervals, through
    aw_align_sliding_window_batch: an interval whose (len_d / W) * (len_q / W) <= 1 gets one
    global alignment; the others advance window by window (W + 1 bases of each sequence,
    semiglobal KSW2 ending at the better of the last row and the last column), and the k-th
    window of every interval still advancing runs in one batched call.  Returns (score of the
    whole alignment under the two-piece objective, aligned query, aligned reference) per
    interval, as a call of its own would."""
    n = len(pairs)
    if n == 0:
        return []
    win = np.broadcast_to(np.asarray(sliding_window_size, dtype=np.int64), (n,)).copy()
    if int(win.max()) > 1073741824:
        raise ValueError("the windows size is too large")
    qp, ql, qb = _seq_arrays([p[0] for p in pairs])
    rp, rl, rb = _seq_arrays([p[1] for p in pairs])
    out = (WindowResultC * n)()
    rc = lib.aw_align_sliding_window_batch(n, qp, ql.ctypes.data, rp, rl.ctypes.data, win.ctypes.data,
                                           matching_score, mismatching_penalty, open1, extend1, open2, extend2, out)
    res = []
    for o in out:
        res.append((o.score, _text(o.alignment_q, o.alignment_len), _text(o.alignment_d, o.alignment_len)))
        lib.aw_window_result_free(C.byref(o))
    if rc != 0:
        raise RuntimeError(f"aw_align_sliding_window_batch failed ({rc}): {last_error()}")
    return res


def align_sliding_window(dna_q: str, dna_d: str, sliding_window_size: int, matching_score: int,
                         mismatching_penalty: int, open1: int, extend1: int, open2: int, extend2: int):
    """alignSlidingWindow (alignSlidingWindow.cpp:457-590) for one interval."""
    return align_sliding_window_batch([(dna_q, dna_d)], sliding_window_size, matching_score, mismatching_penalty,
                                      open1, extend1, open2, extend2)[0]


def cigar_rows_batch(cigars, queries, targets) -> List[Tuple[str, str]]:
    """aw_cigar_rows_batch: the gapped rows (aligned query, aligned reference) of many CIGARs,
    decoded on the device (alignSlidingWindow.cpp:307-324).  queries / targets: str or bytes."""
    n = len(cigars)
    if n == 0:
        return []
    cw = [np.ascontiguousarray(np.asarray(c, dtype=np.uint32)) for c in cigars]
    qb = [q.encode() if isinstance(q, str) else bytes(q) for q in queries]
    tb = [t.encode() if isinstance(t, str) else bytes(t) for t in targets]
    qbufs = [C.create_string_buffer(b, len(b) + 1) for b in qb]
    tbufs = [C.create_string_buffer(b, len(b) + 1) for b in tb]
    cp = (C.c_void_p * n)(*[c.ctypes.data for c in cw])
    qp = (C.c_void_p * n)(*[C.addressof(b) for b in qbufs])
    tp = (C.c_void_p * n)(*[C.addressof(b) for b in tbufs])
    nc = np.array([len(c) for c in cw], dtype=np.int32)
    ql = np.array([len(b) for b in qb], dtype=np.int32)
    tl = np.array([len(b) for b in tb], dtype=np.int32)
    cap = int(ql.sum() + tl.sum()) + 1
    rq, rd = C.create_string_buffer(cap), C.create_string_buffer(cap)
    off = np.zeros(n, dtype=np.int64)
    ln = np.zeros(n, dtype=np.int32)
    check(lib.aw_cigar_rows_batch(n, cp, nc.ctypes.data, qp, ql.ctypes.data, tp, tl.ctypes.data, rq, rd,
                                  off.ctypes.data, ln.ctypes.data, cap), "aw_cigar_rows_batch")
    bq, bd = rq.raw, rd.raw
    return [(bq[o:o + l].decode(), bd[o:o + l].decode()) for o, l in zip(off.tolist(), ln.tolist())]
