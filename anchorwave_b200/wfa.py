"""Host-side mirror of AnchorWave's WFA interface on the B200 WFA kernel.

* :class:`WfaAligner` mirrors the WFA2-lib aligner object AnchorWave caches per thread
  (wavefront_aligner_new / wavefront_align / wavefront_aligner_delete, WFA2-lib
  wavefront/wfa.h:129-134, :210-215) with the attributes of
  src/myImportandFunction/WfaAlignment.cpp:143-170 (match 0, positive penalties, no
  heuristic, end to end, full CIGAR) in high memory (optionally Singletrack), medium or
  low memory (WfaAlignment.cpp:461-543: alignWith{Singletrack,Standard,Medium,Low}Wfa).
* :func:`align_with_wfa` mirrors alignWithWfaMode + decodeCigar
  (WfaAlignment.cpp:223-391): reference is the pattern, query the text; 'M'/'X' consume
  both, 'I' the query, 'D' the reference; score is the negated penalty.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Sequence, Tuple

import numpy as np

from ._lib import AwError, WfaAttr, last_error, lib

WF_STATUS_ALG_COMPLETED = 0
WF_STATUS_OOM = -200
WF_STATUS_UNATTAINABLE = -300

# wavefront_memory_t (WFA2-lib wavefront/wavefront_attributes.h:122-127)
WAVEFRONT_MEMORY_HIGH = 0
WAVEFRONT_MEMORY_MED = 1
WAVEFRONT_MEMORY_LOW = 2


def set_wide(width: int = -1, tail_width: int = -1, cluster_ctas: int = 0) -> None:
    """aw_set_wfa_wide: wavefront width from which a high-memory pair leaves its warp for a
    cluster of CTAs (0 = never), the lower width that applies once every pair of the call has
    started, and the CTAs of a cluster (1..8).  Negative widths and cluster_ctas 0 keep the
    setting.  Results are identical under every setting."""
    lib.aw_set_wfa_wide(int(width), int(tail_width), int(cluster_ctas))


def set_long(min_length_sum: int) -> None:
    """aw_set_wfa_long: pairs whose lengths sum to at least this run first on a whole CTA each
    (high memory; 0 = every pair on one warp).  Results are identical under every setting."""
    lib.aw_set_wfa_long(int(min_length_sum))


def positive_penalty(p: int) -> int:
    """AnchorWave passes negative penalties; WFA takes their magnitude (WfaAlignment.cpp:298-302)."""
    return -p if p < 0 else p


class WfaAligner:
    def __init__(self, mismatch: int, gap_opening1: int, gap_extension1: int, gap_opening2: int,
                 gap_extension2: int, singletrack: bool = False, max_memory_abort: int = 0,
                 memory_mode: int = WAVEFRONT_MEMORY_HIGH):
        self.attr = WfaAttr(mismatch, gap_opening1, gap_extension1, gap_opening2, gap_extension2,
                            int(bool(singletrack)), int(memory_mode), int(max_memory_abort))
        self.h = lib.wavefront_aligner_new_gpu(C.byref(self.attr))
        if not self.h:
            raise AwError(f"wavefront_aligner_new_gpu failed: {last_error()}")

    def align(self, pattern: bytes, text: bytes) -> int:
        """wavefront_align(aligner, pattern, |pattern|, text, |text|): returns the WF status."""
        return lib.wavefront_align_gpu(self.h, pattern, len(pattern), text, len(text))

    def cigar(self) -> Tuple[str, int]:
        ops = C.c_char_p()
        n = C.c_int(0)
        score = C.c_int(0)
        lib.wavefront_gpu_cigar(self.h, C.byref(ops), C.byref(n), C.byref(score))
        return (C.string_at(ops, n.value).decode() if n.value else ""), score.value

    def align_batch_raw(self, patterns: Sequence[bytes], texts: Sequence[bytes]):
        """One submission of n alignments without decoding: (status, score, ops offsets, ops
        lengths, ops buffer, device ms, seconds spent in the C call)."""
        import time
        n = len(patterns)
        pbufs = [C.create_string_buffer(p, len(p) + 1) for p in patterns]
        tbufs = [C.create_string_buffer(t, len(t) + 1) for t in texts]
        pp = (C.c_void_p * n)(*[C.addressof(b) for b in pbufs])
        tp = (C.c_void_p * n)(*[C.addressof(b) for b in tbufs])
        pl = np.array([len(p) for p in patterns], dtype=np.int32)
        tl = np.array([len(t) for t in texts], dtype=np.int32)
        status = np.zeros(n, dtype=np.int32)
        score = np.zeros(n, dtype=np.int32)
        offs = np.zeros(n, dtype=np.int64)
        nops = np.zeros(n, dtype=np.int32)
        cap = int(pl.sum() + tl.sum()) + 1
        ops = C.create_string_buffer(cap)
        ms = C.c_float(0.0)
        t0 = time.perf_counter()
        rc = lib.wavefront_align_batch_gpu(self.h, n, pp, pl.ctypes.data, tp, tl.ctypes.data, status.ctypes.data,
                                           score.ctypes.data, offs.ctypes.data, nops.ctypes.data, ops, cap,
                                           C.byref(ms))
        secs = time.perf_counter() - t0
        if rc != 0:
            raise AwError(f"wavefront_align_batch_gpu failed ({rc}): {last_error()}")
        return status, score, offs, nops, ops, ms.value, secs

    def align_batch(self, patterns: Sequence[bytes], texts: Sequence[bytes]):
        """n alignments in one submission: list of (status, score, ops) plus device ms."""
        n = len(patterns)
        if n == 0:
            return [], 0.0
        pbufs = [C.create_string_buffer(p, len(p) + 1) for p in patterns]
        tbufs = [C.create_string_buffer(t, len(t) + 1) for t in texts]
        pp = (C.c_void_p * n)(*[C.addressof(b) for b in pbufs])
        tp = (C.c_void_p * n)(*[C.addressof(b) for b in tbufs])
        pl = np.array([len(p) for p in patterns], dtype=np.int32)
        tl = np.array([len(t) for t in texts], dtype=np.int32)
        status = np.zeros(n, dtype=np.int32)
        score = np.zeros(n, dtype=np.int32)
        offs = np.zeros(n, dtype=np.int64)
        nops = np.zeros(n, dtype=np.int32)
        cap = int(pl.sum() + tl.sum()) + 1
        ops = C.create_string_buffer(cap)
        ms = C.c_float(0.0)
        rc = lib.wavefront_align_batch_gpu(self.h, n, pp, pl.ctypes.data, tp, tl.ctypes.data, status.ctypes.data,
                                           score.ctypes.data, offs.ctypes.data, nops.ctypes.data, ops, cap,
                                           C.byref(ms))
        if rc != 0:
            raise AwError(f"wavefront_align_batch_gpu failed ({rc}): {last_error()}")
        raw = ops.raw
        out = [(int(status[i]), int(score[i]), raw[offs[i]:offs[i] + nops[i]].decode()) for i in range(n)]
        return out, ms.value

    def memory(self) -> Tuple[int, int]:
        """Device bytes the last call's alignments took: (largest single alignment, sum)."""
        mx = C.c_int64(0)
        tot = C.c_int64(0)
        lib.wavefront_gpu_memory(self.h, C.byref(mx), C.byref(tot))
        return mx.value, tot.value

    def launches(self) -> Tuple[int, int, int]:
        """The last call's kernel launches: (all, of which the cluster kernel's, pairs moved to it)."""
        a, b, c = C.c_int(0), C.c_int(0), C.c_int(0)
        lib.wavefront_gpu_last_launches(self.h, C.byref(a), C.byref(b), C.byref(c))
        return a.value, b.value, c.value

    def close(self):
        if self.h:
            lib.wavefront_aligner_delete_gpu(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def decode_cigar(query: str, reference: str, ops: str):
    """decodeCigar (WfaAlignment.cpp:223-268): gapped rows, or None when the CIGAR does not fit."""
    aq, ar = [], []
    qp = rp = 0
    for c in ops:
        if c in "MX":
            if qp >= len(query) or rp >= len(reference):
                return None
            aq.append(query[qp]); ar.append(reference[rp]); qp += 1; rp += 1
        elif c == "I":
            if qp >= len(query):
                return None
            aq.append(query[qp]); ar.append("-"); qp += 1
        elif c == "D":
            if rp >= len(reference):
                return None
            aq.append("-"); ar.append(reference[rp]); rp += 1
        else:
            return None
    if qp != len(query) or rp != len(reference):
        return None
    return "".join(aq), "".join(ar)


def align_with_wfa(query: str, reference: str, mismatching_penalty: int, open1: int, extend1: int, open2: int,
                   extend2: int, singletrack: bool = False, aligner: WfaAligner = None,
                   memory_mode: int = WAVEFRONT_MEMORY_HIGH):
    """alignWithWfaMode (WfaAlignment.cpp:270-391) on the GPU: (status, score, aln_query, aln_reference)."""
    al = aligner or WfaAligner(positive_penalty(mismatching_penalty), positive_penalty(open1),
                               positive_penalty(extend1), positive_penalty(open2), positive_penalty(extend2),
                               singletrack, memory_mode=memory_mode)
    st = al.align(reference.encode(), query.encode())
    if st != WF_STATUS_ALG_COMPLETED:
        return st, 0, "", ""
    ops, score = al.cigar()
    dec = decode_cigar(query, reference, ops)
    if dec is None:
        return WF_STATUS_UNATTAINABLE, 0, "", ""
    return st, score, dec[0], dec[1]


def align_with_medium_wfa(query: str, reference: str, mismatching_penalty: int, open1: int, extend1: int,
                          open2: int, extend2: int, aligner: WfaAligner = None):
    """alignWithMediumWfa (WfaAlignment.cpp:503-522): medium memory, piggyback traceback."""
    return align_with_wfa(query, reference, mismatching_penalty, open1, extend1, open2, extend2, aligner=aligner,
                          memory_mode=WAVEFRONT_MEMORY_MED)


def align_with_low_wfa(query: str, reference: str, mismatching_penalty: int, open1: int, extend1: int,
                       open2: int, extend2: int, aligner: WfaAligner = None):
    """alignWithLowWfa (WfaAlignment.cpp:524-543): low memory, piggyback traceback."""
    return align_with_wfa(query, reference, mismatching_penalty, open1, extend1, open2, extend2, aligner=aligner,
                          memory_mode=WAVEFRONT_MEMORY_LOW)
