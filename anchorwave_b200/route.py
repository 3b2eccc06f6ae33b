"""Routing front end of the serving loop (frontend/libaw_route.so, frontend/aw_route.h).

AnchorWave's own selector (makeAlignmentSelectionPlan, AlignmentAlgorithmSelector.cpp:1711,
compiled unchanged from its sources) and its executor's first choice on an idle system give
every interval its engine and that engine's parameters, in the form aw_serve_submit_route
takes.  The library is built from the AnchorWave source tree (frontend/Makefile); without it
this module raises on import.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from ._lib import ServeRoute

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "frontend", "libaw_route.so")

# anchorwave::AlignmentCandidate (AlignmentAlgorithmSelector.h:10-20)
CANDIDATES = ["SingletrackWfa", "StandardWfa", "MediumWfa", "LowWfa", "Ksw2Singletrack", "Ksw2ScoreCertified",
              "Ksw2Full", "Ksw2Banded", "SlidingWindow"]
ANCHORWAVE_WINDOW = 100_000  # AnchorWave's default -w (src/controlLayer.cpp:314)
ANCHORWAVE_PENALTIES = (-4, -4, -2, -24, -1)  # mismatch, open1, extend1, open2, extend2


class RouteChoice(C.Structure):
    """aw_route_choice_t."""
    _fields_ = [("route", ServeRoute), ("candidate", C.c_int), ("tier", C.c_int)]


@dataclass
class Route:
    method: int
    band: int
    band_max: int
    window: int
    candidate: str
    tier: int
    predicted_bytes: int = 0


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `make -C anchorwave_b200/frontend REF=<AnchorWave>`")
    lib = C.CDLL(LIB_PATH)
    lib.aw_route_intervals.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                       C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                                       C.POINTER(RouteChoice)]
    lib.aw_route_intervals.restype = C.c_int
    return lib


lib = _load()


def route_intervals(pairs: Sequence[Tuple[bytes, bytes]], window_width: int = ANCHORWAVE_WINDOW,
                    penalties=ANCHORWAVE_PENALTIES, nthreads: int = 0) -> List[Route]:
    """Routes of (query, reference) ASCII pairs: the selector's plan of each interval and the
    engine AnchorWave's executor starts first on an idle system."""
    n = len(pairs)
    if n == 0:
        return []
    qb = [C.create_string_buffer(bytes(q), len(q) + 1) for q, _ in pairs]
    rb = [C.create_string_buffer(bytes(r), len(r) + 1) for _, r in pairs]
    qp = (C.c_void_p * n)(*[C.addressof(b) for b in qb])
    rp = (C.c_void_p * n)(*[C.addressof(b) for b in rb])
    ql = np.array([len(q) for q, _ in pairs], dtype=np.int64)
    rl = np.array([len(r) for _, r in pairs], dtype=np.int64)
    out = (RouteChoice * n)()
    rc = lib.aw_route_intervals(n, qp, ql.ctypes.data, rp, rl.ctypes.data, int(window_width), *penalties,
                                nthreads or os.cpu_count() or 1, out)
    if rc != 0:
        raise ValueError("aw_route_intervals: bad arguments")
    return [Route(o.route.method, o.route.band, o.route.band_max, o.route.window, CANDIDATES[o.candidate], o.tier,
                  o.route.predicted_bytes) for o in out]
