"""Host-side mirror of the sequence pass of AnchorWave's alignment selector on the GPU.

:func:`sequence_summary_batch` replaces ``summarizeSequencePair``
(src/myImportandFunction/AlignmentAlgorithmSelector.cpp:730-757) for many interval pairs in
one call through ``aw_sequence_summary_batch``: per sequence the FNV-1a fingerprint, the
ambiguous-base fraction, the normalized 64-base-block entropy, the low-complexity fraction
and the k = 9, 15, 21 sketches, with the sampling modulos of ``makeAlignmentSelectionPlan``
(:1752-1760) unless given.  The rest of the selector (anchor chains, cost models) consumes
these summaries on the host.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from ._lib import AwError, last_error, lib


class SequenceSummary(C.Structure):
    """aw_sequence_summary_t (include/anchorwave_b200.h)."""
    _fields_ = [("fingerprint", C.c_uint64), ("ambiguous_fraction", C.c_double),
                ("normalized_entropy", C.c_double), ("low_complexity_fraction", C.c_double),
                ("sketch_offset", C.c_int64 * 3), ("sketch_count", C.c_int64 * 3)]


def sequence_summary_raw(queries: Sequence[bytes], references: Sequence[bytes], modulos=None, copy=True):
    """One call: (summaries[2n], identical[n], sketch hashes, sketch positions, device ms).
    copy=False returns views of the library's page-locked buffers (valid until the next call
    on this thread)."""
    n = len(queries)
    out = (SequenceSummary * max(2 * n, 1))()
    ident = np.zeros(max(n, 1), dtype=np.int32)
    # pointers straight into the bytes objects (no copies)
    qp = (C.c_char_p * max(n, 1))(*queries)
    rp = (C.c_char_p * max(n, 1))(*references)
    ql = np.array([len(q) for q in queries] or [0], dtype=np.int64)
    rl = np.array([len(r) for r in references] or [0], dtype=np.int64)
    mod = None
    if modulos is not None:
        mod = np.ascontiguousarray(np.asarray(modulos, dtype=np.uint64).reshape(n, 3))
    ms = C.c_float(0.0)
    rc = lib.aw_sequence_summary_batch(n, qp, ql.ctypes.data, rp, rl.ctypes.data,
                                       mod.ctypes.data if mod is not None else None, out, ident.ctypes.data,
                                       C.byref(ms))
    if rc != 0:
        raise AwError(f"aw_sequence_summary_batch failed ({rc}): {last_error()}")
    hp, pp = C.c_void_p(), C.c_void_p()
    total = lib.aw_sequence_summary_sketch_view(C.byref(hp), C.byref(pp))
    if total == 0:
        return out, ident[:n], np.zeros(0, np.uint64), np.zeros(0, np.uint32), ms.value
    h = np.ctypeslib.as_array(C.cast(hp, C.POINTER(C.c_uint64)), shape=(total,))
    p = np.ctypeslib.as_array(C.cast(pp, C.POINTER(C.c_uint32)), shape=(total,))
    if copy:
        h, p = h.copy(), p.copy()
    return out, ident[:n], h, p, ms.value


def sequence_summary_batch(queries: Sequence[bytes], references: Sequence[bytes],
                           modulos=None) -> List[Tuple[bool, list]]:
    """Per pair (identical, [query summary, reference summary]); each summary a dict with
    fingerprint, the three fractions and sketches = [[(hash, position), ...] for k = 9, 15, 21]."""
    out, ident, h, p, _ = sequence_summary_raw(queries, references, modulos)
    res = []
    for i in range(len(queries)):
        sides = []
        for t in range(2):
            s = out[2 * i + t]
            sk = []
            for sc in range(3):
                o, c = int(s.sketch_offset[sc]), int(s.sketch_count[sc])
                sk.append(list(zip(h[o:o + c].tolist(), p[o:o + c].tolist())))
            sides.append({"fingerprint": int(s.fingerprint), "ambiguous_fraction": s.ambiguous_fraction,
                          "normalized_entropy": s.normalized_entropy,
                          "low_complexity_fraction": s.low_complexity_fraction, "sketches": sk})
        res.append((bool(ident[i]), sides))
    return res
