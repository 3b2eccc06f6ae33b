"""TEST INFRASTRUCTURE (oracle) -- ctypes front end of the two CPU oracles.

* ``Restatement``: ``liboracle.so`` built from ``ksw2_oracle.c`` / ``wfa_oracle.c`` /
  ``summary_oracle.c``, the plain-C restatement of the reference algorithms (always
  available).
* ``Reference``: ``_ref/libawref_<isa>.so``, AnchorWave's own KSW2 / WFA2 sources
  compiled from the reference tree by ``oracle/Makefile`` (present wherever it was
  built; it travels with the repository snapshot).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline leg may import
this module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional

HERE = os.path.dirname(os.path.abspath(__file__))

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


class KswExtz(C.Structure):
    """ksw_extz_t (minimap2/ksw2.h:40-50)."""
    _fields_ = [("max", C.c_uint32, 31), ("zdropped", C.c_uint32, 1),
                ("max_q", C.c_int), ("max_t", C.c_int), ("mqe", C.c_int), ("mqe_t", C.c_int),
                ("mte", C.c_int), ("mte_q", C.c_int), ("score", C.c_int),
                ("m_cigar", C.c_int), ("n_cigar", C.c_int), ("reach_end", C.c_int),
                ("stopped", C.c_int), ("cigar", C.POINTER(C.c_uint32))]


class SummaryOut(C.Structure):
    """One sequence of summarizeSequencePair (AlignmentAlgorithmSelector.cpp:180-191)."""
    _fields_ = [("fingerprint", C.c_uint64), ("ambiguous_fraction", C.c_double),
                ("normalized_entropy", C.c_double), ("low_complexity_fraction", C.c_double),
                ("count", C.c_int64 * 3)]


def _summary_call(fn, query: bytes, reference: bytes, modulos=None):
    """Runs a summarizeSequencePair front end: returns (identical, [query, reference]) with
    each side {fingerprint, fractions, sketches: [[(hash, pos)...] per k=9, 15, 21]}."""
    import numpy as np
    out = (SummaryOut * 2)()
    ident = C.c_int(0)
    mod = (C.c_uint64 * 3)(*modulos) if modulos is not None else None
    n = fn(query, len(query), reference, len(reference), mod, out, C.byref(ident), None, None, 0)
    h = np.zeros(max(n, 1), dtype=np.uint64)
    p = np.zeros(max(n, 1), dtype=np.uint32)
    fn(query, len(query), reference, len(reference), mod, out, C.byref(ident), h.ctypes.data, p.ctypes.data, n)
    sides, w = [], 0
    for t in range(2):
        sk = []
        for sc in range(3):
            c = int(out[t].count[sc])
            sk.append(list(zip(h[w:w + c].tolist(), p[w:w + c].tolist())))
            w += c
        sides.append({"fingerprint": int(out[t].fingerprint), "ambiguous_fraction": out[t].ambiguous_fraction,
                      "normalized_entropy": out[t].normalized_entropy,
                      "low_complexity_fraction": out[t].low_complexity_fraction, "sketches": sk})
    return bool(ident.value), sides


def _summary_argtypes(fn):
    fn.argtypes = [C.c_char_p, C.c_int64, C.c_char_p, C.c_int64, C.c_void_p, C.c_void_p, C.POINTER(C.c_int),
                   C.c_void_p, C.c_void_p, C.c_int64]
    fn.restype = C.c_int64


@dataclass
class KswResult:
    """All comparable ksw_extz_t fields plus the CIGAR (BAM-packed words)."""
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


def extz_to_result(ez: KswExtz, free_fn) -> KswResult:
    cig = [ez.cigar[i] for i in range(ez.n_cigar)] if ez.n_cigar > 0 and ez.cigar else []
    res = KswResult(ez.max, ez.zdropped, ez.max_q, ez.max_t, ez.mqe, ez.mqe_t, ez.mte, ez.mte_q,
                    ez.score, ez.n_cigar, ez.reach_end, ez.stopped, cig)
    if ez.cigar:
        free_fn(C.cast(ez.cigar, C.c_void_p))
    return res


def _u8(buf: bytes):
    return (C.c_uint8 * max(1, len(buf))).from_buffer_copy(buf if buf else b"\0")


def _i8(vals):
    return (C.c_int8 * len(vals))(*vals)


def cpu_isa() -> str:
    """Best reference ISA this host can run: avx512 / avx2 / sse."""
    flags = set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        pass
    if {"avx512bw", "avx512vl", "avx512cd"} <= flags:
        return "avx512"
    if "avx2" in flags:
        return "avx2"
    return "sse"


ISA_BLOCK = {"avx512": 64, "avx2": 32, "sse": 16}


class Restatement:
    """The plain-C restatement (ksw2_oracle.c, wfa_oracle.c)."""

    def __init__(self, path: Optional[str] = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle liboracle.so`")
        self.lib = C.CDLL(path)
        L = self.lib
        L.oracle_ksw_extd2.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int8,
                                       C.c_void_p, C.c_int8, C.c_int8, C.c_int8, C.c_int8, C.c_int,
                                       C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(KswExtz)]
        L.oracle_free.argtypes = [C.c_void_p]
        assert L.oracle_sizeof_extz() == C.sizeof(KswExtz)
        self.has_wfa = hasattr(L, "oracle_wfa_align")
        if self.has_wfa:
            L.oracle_wfa_align.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int,
                                           C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                           C.c_char_p, C.c_int, C.POINTER(C.c_int)]
            _summary_argtypes(L.oracle_sequence_summary)
            assert L.oracle_sizeof_summary() == C.sizeof(SummaryOut)
            L.oracle_wfa_align_mode.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int,
                                                C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int),
                                                C.c_char_p, C.c_int, C.POINTER(C.c_int)]

    def ksw_extd2(self, query: bytes, target: bytes, mat, q, e, q2, e2, w=-1, zdrop=-1, end_bonus=0,
                  flag=0, block=64, m=5, stop_interval=0, stop_at=-1) -> KswResult:
        ez = KswExtz()
        self.lib.oracle_ksw_extd2(block, len(query), _u8(query), len(target), _u8(target), m, _i8(mat),
                                  q, e, q2, e2, w, zdrop, end_bonus, flag, stop_interval, stop_at,
                                  C.byref(ez))
        return extz_to_result(ez, self.lib.oracle_free)

    def sequence_summary(self, query: bytes, reference: bytes, modulos=None):
        """summarizeSequencePair restated (summary_oracle.c)."""
        return _summary_call(self.lib.oracle_sequence_summary, query, reference, modulos)

    def wfa_align(self, pattern: bytes, text: bytes, x, o1, e1, o2, e2, singletrack=False, memory_mode=0):
        """memory_mode as WFA2-lib's wavefront_memory_t: 0 high, 1 medium, 2 low (piggyback)."""
        score = C.c_int(0)
        nops = C.c_int(0)
        cap = len(pattern) + len(text) + 16
        ops = C.create_string_buffer(cap)
        st = self.lib.oracle_wfa_align_mode(pattern, len(pattern), text, len(text), x, o1, e1, o2, e2,
                                            int(bool(singletrack)), int(memory_mode), C.byref(score), ops, cap,
                                            C.byref(nops))
        return st, score.value, ops.raw[: nops.value].decode() if st == 0 else ""


class Reference:
    """AnchorWave's own compiled KSW2/WFA2 code (oracle/_ref)."""

    def __init__(self, isa: Optional[str] = None):
        isa = isa or cpu_isa()
        path = os.path.join(HERE, "_ref", f"libawref_{isa}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle` where the reference tree exists")
        self.isa = isa
        self.block = ISA_BLOCK[isa]
        self.lib = C.CDLL(path)
        L = self.lib
        L.awref_ksw_extd2.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_int8,
                                      C.c_void_p, C.c_int8, C.c_int8, C.c_int8, C.c_int8, C.c_int,
                                      C.c_int, C.c_int, C.c_int, C.POINTER(KswExtz)]
        L.awref_free.argtypes = [C.c_void_p]
        L.awref_set_progress_stop.argtypes = [C.c_int, C.c_int]
        L.awref_wfa_align.argtypes = [C.c_char_p, C.c_int, C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_char_p,
                                      C.c_int, C.POINTER(C.c_int)]
        L.awref_ksw_batch.restype = C.c_double
        L.awref_ksw_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
        L.awref_wfa_batch.restype = C.c_double
        L.awref_wfa_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.POINTER(C.c_int)]
        assert L.awref_sizeof_extz() == C.sizeof(KswExtz)
        self.has_summary = hasattr(L, "awref_sequence_summary")
        if self.has_summary:
            _summary_argtypes(L.awref_sequence_summary)
            assert L.awref_sizeof_summary() == C.sizeof(SummaryOut)
            L.awref_sequence_summary_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                       C.c_void_p, C.c_void_p, C.c_int]
            L.awref_sequence_summary_batch.restype = C.c_double

    def ksw_extd2(self, query: bytes, target: bytes, mat, q, e, q2, e2, w=-1, zdrop=-1, end_bonus=0,
                  flag=0, m=5, variant=0, stop_interval=0, stop_at=-1) -> KswResult:
        """variant 0: native KSW2 entry, 1: SSE entry, 2: native Singletrack, 3: SSE Singletrack."""
        ez = KswExtz()
        if stop_at >= 0:
            self.lib.awref_set_progress_stop(stop_interval, stop_at)
        try:
            self.lib.awref_ksw_extd2(variant, len(query), _u8(query), len(target), _u8(target), m,
                                     _i8(mat), q, e, q2, e2, w, zdrop, end_bonus, flag, C.byref(ez))
        finally:
            if stop_at >= 0:
                self.lib.awref_clear_progress()
        return extz_to_result(ez, self.lib.awref_free)

    def ksw_batch(self, queries, targets, mat, q, e, q2, e2, w=-1, flag=0, variant=0, nthreads=None,
                  time_budget_s=0.0):
        """Threaded batch over the reference KSW2 entry (the CPU baseline).  Returns a dict with
        per-pair score, n_cigar, result hash (see result_hash), wall seconds and pairs done."""
        import numpy as np
        nthreads = nthreads or os.cpu_count() or 1
        n = len(queries)
        ql = np.array([len(x) for x in queries], dtype=np.int32)
        tl = np.array([len(x) for x in targets], dtype=np.int32)
        qoff = np.zeros(n, dtype=np.int64)
        toff = np.zeros(n, dtype=np.int64)
        if n:
            qoff[1:] = np.cumsum(ql[:-1])
            toff[1:] = np.cumsum(tl[:-1])
        def u8(x):
            return np.frombuffer(x, dtype=np.uint8) if isinstance(x, (bytes, bytearray)) else np.asarray(x, np.uint8)
        qbuf = np.concatenate([u8(x) for x in queries]) if n else np.zeros(1, np.uint8)
        tbuf = np.concatenate([u8(x) for x in targets]) if n else np.zeros(1, np.uint8)
        score = np.zeros(max(n, 1), dtype=np.int32)
        ncig = np.zeros(max(n, 1), dtype=np.int32)
        hsh = np.zeros(max(n, 1), dtype=np.uint64)
        psec = np.zeros(max(n, 1), dtype=np.float64)
        done = C.c_int(0)
        matc = _i8(mat)
        secs = self.lib.awref_ksw_batch(n, ql.ctypes.data, qoff.ctypes.data, qbuf.ctypes.data, tl.ctypes.data,
                                        toff.ctypes.data, tbuf.ctypes.data, matc, q, e, q2, e2, w, flag, variant,
                                        nthreads, time_budget_s, score.ctypes.data, ncig.ctypes.data,
                                        hsh.ctypes.data, psec.ctypes.data, C.byref(done))
        return {"score": score[:n], "n_cigar": ncig[:n], "hash": hsh[:n], "pair_seconds": psec[:n],
                "seconds": secs, "done": done.value, "threads": nthreads}

    def wfa_batch(self, queries, targets, x, o1, e1, o2, e2, singletrack=False, nthreads=None,
                  time_budget_s=0.0, memory_mode=0):
        """Threaded batch over the reference wavefront_align (ASCII sequences)."""
        import numpy as np
        nthreads = nthreads or os.cpu_count() or 1
        n = len(queries)
        ql = np.array([len(x) for x in queries], dtype=np.int32)
        tl = np.array([len(x) for x in targets], dtype=np.int32)
        qoff = np.zeros(n, dtype=np.int64)
        toff = np.zeros(n, dtype=np.int64)
        if n:
            qoff[1:] = np.cumsum(ql[:-1])
            toff[1:] = np.cumsum(tl[:-1])
        qbuf = np.frombuffer(b"".join(queries) or b"\0", dtype=np.uint8).copy()
        tbuf = np.frombuffer(b"".join(targets) or b"\0", dtype=np.uint8).copy()
        score = np.zeros(max(n, 1), dtype=np.int32)
        nops = np.zeros(max(n, 1), dtype=np.int32)
        ooff = np.zeros(max(n, 1), dtype=np.int64)
        if n:
            ooff[1:n] = np.cumsum(ql[:-1].astype(np.int64) + tl[:-1] + 8)
        obuf = np.zeros(int(ooff[n - 1] + ql[-1] + tl[-1] + 8) if n else 1, dtype=np.uint8)
        done = C.c_int(0)
        secs = self.lib.awref_wfa_batch(n, ql.ctypes.data, qoff.ctypes.data, qbuf.ctypes.data, tl.ctypes.data,
                                        toff.ctypes.data, tbuf.ctypes.data, x, o1, e1, o2, e2,
                                        int(bool(singletrack)), int(memory_mode), nthreads, time_budget_s,
                                        score.ctypes.data, nops.ctypes.data, obuf.ctypes.data, ooff.ctypes.data,
                                        C.byref(done))
        return {"score": score[:n], "n_ops": nops[:n], "ops": obuf, "ops_offset": ooff[:n], "seconds": secs,
                "done": done.value, "threads": nthreads}

    def sequence_summary(self, query: bytes, reference: bytes, modulos=None):
        """The compiled selector's summarizeSequencePair (ref_selector_shim.cpp)."""
        return _summary_call(self.lib.awref_sequence_summary, query, reference, modulos)

    def sequence_summary_batch(self, queries, references, nthreads=None):
        """n pairs on the host threads: (seconds, summaries array [n, 2], identical flags)."""
        import numpy as np
        nthreads = nthreads or os.cpu_count() or 1
        n = len(queries)
        qb = [C.create_string_buffer(q, len(q) + 1) for q in queries]
        rb = [C.create_string_buffer(r, len(r) + 1) for r in references]
        qp = (C.c_void_p * n)(*[C.addressof(b) for b in qb])
        rp = (C.c_void_p * n)(*[C.addressof(b) for b in rb])
        ql = np.array([len(q) for q in queries], dtype=np.int64)
        rl = np.array([len(r) for r in references], dtype=np.int64)
        out = (SummaryOut * (2 * n))()
        ident = np.zeros(n, dtype=np.int32)
        secs = self.lib.awref_sequence_summary_batch(n, qp, ql.ctypes.data, rp, rl.ctypes.data, out,
                                                     ident.ctypes.data, nthreads)
        return secs, out, ident

    # ---- AnchorWave's rescue procedures and row decoding (ref_rescue_shim.cpp) -------------
    def _rescue_args(self):
        L = self.lib
        if getattr(self, "_rescue_ready", False):
            return
        vp, i64, i32 = C.c_void_p, C.c_int64, C.c_int
        L.awref_score_certified.argtypes = [C.c_char_p, i64, C.c_char_p, i64, i64, i64, i32, i32, i32, i32, i32,
                                            C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), C.POINTER(i64), vp, vp,
                                            i64, C.POINTER(i64), vp, vp, C.POINTER(i64)]
        L.awref_score_certified.restype = i32
        L.awref_sliding_window.argtypes = [C.c_char_p, i64, C.c_char_p, i64, i64, i32, i32, i32, i32, i32, i32, vp,
                                           vp, i64, C.POINTER(i64)]
        L.awref_sliding_window.restype = i64
        for fn in (L.awref_minimap2_rows,):
            fn.argtypes = [C.c_char_p, i64, C.c_char_p, i64, i32, i32, i32, i32, i32, vp, vp, i64, C.POINTER(i64)]
            fn.restype = i64
        L.awref_banded_rows.argtypes = [C.c_char_p, i64, C.c_char_p, i64, i64, i32, i32, i32, i32, i32, vp, vp, i64,
                                        C.POINTER(i64)]
        L.awref_banded_rows.restype = i64
        self._rescue_ready = True

    def score_certified(self, dq: str, dd: str, initial_band: int, maximum_band: int, pen):
        """alignScoreCertifiedKsw2 (alignSlidingWindow.cpp:1197-1400), no selection plan, no
        deadline: dict with status (0 Completed, 1 TimeLimit, 2 NotCertified, 3 Failed), score,
        optimal_score, final_band_width, traceback_attempts, rows and best-effort rows."""
        self._rescue_args()
        q, d = dq.encode(), dd.encode()
        cap = len(q) + len(d) + 1
        bufs = [C.create_string_buffer(cap) for _ in range(4)]
        v = [C.c_int64(0) for _ in range(6)]
        st = self.lib.awref_score_certified(q, len(q), d, len(d), initial_band, maximum_band, *pen, *[C.byref(x) for x in v[:4]],
                                            bufs[0], bufs[1], cap, C.byref(v[4]), bufs[2], bufs[3], C.byref(v[5]))
        rows = lambda b, n: b.raw[:n].decode() if n > 0 else ""
        return {"status": st, "score": v[0].value, "optimal_score": v[1].value, "final_band_width": v[2].value,
                "traceback_attempts": v[3].value, "alignment_q": rows(bufs[0], v[4].value),
                "alignment_d": rows(bufs[1], v[4].value), "best_effort_q": rows(bufs[2], v[5].value),
                "best_effort_d": rows(bufs[3], v[5].value)}

    def _rows_call(self, fn, q: bytes, d: bytes, *args):
        cap = len(q) + len(d) + 1
        a, b = C.create_string_buffer(cap), C.create_string_buffer(cap)
        n = C.c_int64(0)
        s = fn(q, len(q), d, len(d), *args, a, b, cap, C.byref(n))
        return s, a.raw[:n.value].decode(), b.raw[:n.value].decode()

    def sliding_window(self, dq: str, dd: str, window: int, match: int, pen):
        """alignSlidingWindow (alignSlidingWindow.cpp:457-590): (score, query row, reference row)."""
        self._rescue_args()
        return self._rows_call(self.lib.awref_sliding_window, dq.encode(), dd.encode(), window, match, *pen)

    def minimap2_rows(self, dq: str, dd: str, pen):
        """minimap2AlignmentWithArena (alignSlidingWindow.cpp:241-332): ksw_extd2 of the native ISA
        and its CIGAR decoded into rows (:307-324): (ez.score, query row, reference row)."""
        self._rescue_args()
        return self._rows_call(self.lib.awref_minimap2_rows, dq.encode(), dd.encode(), *pen)

    def banded_rows(self, dq: str, dd: str, band: int, pen):
        """alignSlidingWindow_minimap2 (alignSlidingWindow.cpp:800-890): (re-score, rows)."""
        self._rescue_args()
        return self._rows_call(self.lib.awref_banded_rows, dq.encode(), dd.encode(), band, *pen)

    def wfa_align(self, pattern: bytes, text: bytes, x, o1, e1, o2, e2, singletrack=False, memory_mode=0):
        score = C.c_int(0)
        nops = C.c_int(0)
        cap = len(pattern) + len(text) + 16
        ops = C.create_string_buffer(cap)
        st = self.lib.awref_wfa_align(pattern, len(pattern), text, len(text), x, o1, e1, o2, e2,
                                      int(bool(singletrack)), memory_mode, C.byref(score), ops, cap,
                                      C.byref(nops))
        return st, score.value, ops.raw[: nops.value].decode() if st == 0 else ""


def result_hash(r) -> int:
    """FNV-1a of the comparable ksw_extz_t fields + CIGAR, identical to awref_extz_hash (ref_shim.c)."""
    h = 1469598103934665603
    vals = [r.max, r.zdropped, r.max_q, r.max_t, r.mqe, r.mqe_t, r.mte, r.mte_q, r.score, r.n_cigar,
            r.reach_end, r.stopped] + list(r.cigar)
    for v in vals:
        v &= 0xFFFFFFFF
        for b in range(4):
            h ^= (v >> (8 * b)) & 0xFF
            h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def anchorwave_matrix(mismatch: int):
    """5x5 matrix of alignSlidingWindow.cpp:245-255: match 0, every unequal pair -|mismatch|."""
    b = mismatch if mismatch < 0 else -mismatch
    return [0 if i == j else b for i in range(5) for j in range(5)]
