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


def sequence_summary_raw(queries: Sequence[bytes], references: Sequence[bytes], modulos=None):
    """One call: (summaries[2n], identical[n], sketch hashes, sketch positions)."""
    n = len(queries)
    out = (SequenceSummary * max(2 * n, 1))()
    ident = np.zeros(max(n, 1), dtype=np.int32)
    qb = [C.create_string_buffer(q, len(q) + 1) for q in queries]
    rb = [C.create_string_buffer(r, len(r) + 1) for r in references]
    qp = (C.c_void_p * max(n, 1))(*[C.addressof(b) for b in qb])
    rp = (C.c_void_p * max(n, 1))(*[C.addressof(b) for b in rb])
    ql = np.array([len(q) for q in queries] or [0], dtype=np.int64)
    rl = np.array([len(r) for r in references] or [0], dtype=np.int64)
    mod = None
    if modulos is not None:
        mod = np.ascontiguousarray(np.asarray(modulos, dtype=np.uint64).reshape(n, 3))
    rc = lib.aw_sequence_summary_batch(n, qp, ql.ctypes.data, rp, rl.ctypes.data,
                                       mod.ctypes.data if mod is not None else None, out, ident.ctypes.data)
    if rc != 0:
        raise AwError(f"aw_sequence_summary_batch failed ({rc}): {last_error()}")
    total = lib.aw_sequence_summary_sketches(None, None, 0)
    h = np.zeros(max(total, 1), dtype=np.uint64)
    p = np.zeros(max(total, 1), dtype=np.uint32)
    got = lib.aw_sequence_summary_sketches(h.ctypes.data, p.ctypes.data, total)
    if got != total:
        raise AwError(f"aw_sequence_summary_sketches failed ({got}): {last_error()}")
    return out, ident[:n], h[:total], p[:total]


def sequence_summary_batch(queries: Sequence[bytes], references: Sequence[bytes],
                           modulos=None) -> List[Tuple[bool, list]]:
    """Per pair (identical, [query summary, reference summary]); each summary a dict with
    fingerprint, the three fractions and sketches = [[(hash, position), ...] for k = 9, 15, 21]."""
    out, ident, h, p = sequence_summary_raw(queries, references, modulos)
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
