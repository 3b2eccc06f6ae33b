"""Serving loop (continuous batching) in place of AnchorWave's CPU alignment pool.

:class:`AlignmentServer` wraps aw_serve_* (include/anchorwave_b200.h): submit intervals
as the anchor stage emits them (ids consecutive from 0) with the engine the selector chose;
results come back strictly in id order with their submit-to-result latency.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from ._lib import AwError, ServeConfig, ServeResult, ServeRoute, ServeStats, last_error, lib

ROUTE_KSW2 = 0
ROUTE_KSW2_SINGLETRACK = 1
ROUTE_WFA = 2
ROUTE_WFA_SINGLETRACK = 3
ROUTE_WFA_MEDIUM = 4
ROUTE_WFA_LOW = 5
ROUTE_KSW2_CERTIFIED = 6
ROUTE_SLIDING_WINDOW = 7
KSW2_ROUTES = (ROUTE_KSW2, ROUTE_KSW2_SINGLETRACK, ROUTE_KSW2_CERTIFIED, ROUTE_SLIDING_WINDOW)


@dataclass
class ServeRouteSpec:
    """A request's engine and parameters (aw_serve_route_t), as the routing front end returns
    them (anchorwave_b200.route.Route has the same fields)."""
    method: int
    band: int = -1
    band_max: int = -1
    window: int = 0
    predicted_bytes: int = 0


@dataclass
class ServedAlignment:
    id: int
    method: int
    status: int
    latency_s: float
    ksw: Optional[tuple] = None      # ksw_extz_t key (fields + CIGAR), KSW2 routes (the rescue routes:
                                     # their rows as a CIGAR and the re-scored score)
    wfa: Optional[tuple] = None      # (status, score, ops), WFA routes


class AlignmentServer:
    def __init__(self, mat, q, e, q2, e2, wfa_penalties=(4, 4, 2, 24, 1), slots=4, max_batch=256,
                 hbm_budget=0, m=5):
        cfg = ServeConfig()
        cfg.slots, cfg.max_batch, cfg.hbm_budget, cfg.m = slots, max_batch, int(hbm_budget), m
        for i, v in enumerate(mat):
            cfg.mat[i] = v
        cfg.q, cfg.e, cfg.q2, cfg.e2 = q, e, q2, e2
        cfg.wfa_x, cfg.wfa_o1, cfg.wfa_e1, cfg.wfa_o2, cfg.wfa_e2 = wfa_penalties
        self.cfg = cfg
        self.h = lib.aw_serve_open(C.byref(cfg))
        if not self.h:
            raise AwError(f"aw_serve_open failed: {last_error()}")

    def submit(self, rid: int, method: int, query: bytes, target: bytes, band: int = -1, band_max: int = -1,
               window: int = 0, predicted_bytes: int = 0):
        """Enqueue one interval with its engine and that engine's parameters (band: KSW2 band,
        or score-certified KSW2's initial band; band_max: its largest band; window: the
        sliding-window width; predicted_bytes: the selector's memory estimate, 0 = the
        server's own)."""
        rt = ServeRoute(method, band, band_max, window, int(predicted_bytes))
        rc = lib.aw_serve_submit_route(self.h, rid, C.byref(rt), query, len(query), target, len(target))
        if rc != 0:
            raise AwError(f"aw_serve_submit_route failed ({rc}): {last_error()}")

    def poll(self, max_results: int = 1024, wait_ms: int = 0) -> List[ServedAlignment]:
        buf = (ServeResult * max_results)()
        n = lib.aw_serve_poll(self.h, buf, max_results, wait_ms)
        out = []
        for i in range(n):
            r = buf[i]
            item = ServedAlignment(int(r.id), int(r.method), int(r.status), float(r.latency_s))
            if r.method in KSW2_ROUTES:
                ez = r.ez
                # one copy of the CIGAR words (indexing a ctypes pointer word by word costs
                # more than the alignment itself for long intervals)
                cig = (tuple(np.frombuffer(C.string_at(ez.cigar, 4 * ez.n_cigar), dtype=np.uint32).tolist())
                       if ez.n_cigar > 0 and ez.cigar else ())
                item.ksw = (ez.max, ez.zdropped, ez.max_q, ez.max_t, ez.mqe, ez.mqe_t, ez.mte, ez.mte_q, ez.score,
                            ez.n_cigar, ez.reach_end, ez.stopped, cig)
            else:
                ops = C.string_at(r.ops, r.n_ops).decode() if r.n_ops > 0 and r.ops else ""
                item.wfa = (int(r.status), int(r.wfa_score), ops)
            lib.aw_serve_result_free(C.byref(buf[i]))
            out.append(item)
        return out

    def stats(self) -> dict:
        s = ServeStats()
        lib.aw_serve_stats(self.h, C.byref(s))
        return {k: getattr(s, k) for k, _ in ServeStats._fields_}

    def close(self):
        if self.h:
            lib.aw_serve_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
