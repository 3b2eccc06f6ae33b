"""CPU tests of the routing front end (anchorwave_b200/route.py, frontend/libaw_route.so):
AnchorWave's selector, compiled unchanged, gives every interval a route; the front end maps
each selector candidate to the server's route with the plan's parameters, deterministically,
and across a spread of interval shapes more than one engine of each tier is chosen."""
import collections

import numpy as np
import pytest

from anchorwave_b200 import workloads as W

route = pytest.importorskip("anchorwave_b200.route", reason="libaw_route.so not built (needs the AnchorWave tree)")


def _shapes(seed):
    rng = np.random.default_rng(seed)
    pairs = []
    for L, d in [(300, 0.01), (2000, 0.02), (5000, 0.01), (800, 0.15), (3000, 0.12), (12000, 0.10),
                 (40000, 0.05), (9000, 0.01)]:
        for _ in range(3):
            q, t = W.divergent_pair(rng, L, d, d, 4.0)
            pairs.append((W.to_ascii(q), W.to_ascii(t)))
    t = W.random_dna(rng, 150_000)
    q = W.repeat_query(rng, t, long_indels=(2, 3), long_max=20_000)
    pairs.append((W.to_ascii(q), W.to_ascii(t)))
    return pairs


def test_routes_are_deterministic_and_mapped():
    pairs = _shapes(1)
    a = route.route_intervals(pairs, nthreads=4)
    b = route.route_intervals(pairs, nthreads=1)
    assert a == b
    for r in a:
        m = {"SingletrackWfa": 3, "StandardWfa": 2, "MediumWfa": 4, "LowWfa": 5, "Ksw2Singletrack": 1,
             "Ksw2ScoreCertified": 6, "Ksw2Full": 0, "Ksw2Banded": 0, "SlidingWindow": 7}[r.candidate]
        assert r.method == m
        if r.candidate == "Ksw2Banded":
            assert r.band >= 0 and r.tier == 2
        if r.candidate == "SlidingWindow":
            assert r.window > 0 and r.tier == 2
        if r.candidate == "Ksw2ScoreCertified":
            assert 0 <= r.band <= r.band_max
        if r.candidate in ("Ksw2Full", "Ksw2Singletrack") or "Wfa" in r.candidate:
            assert r.tier == 1
    counts = collections.Counter(r.candidate for r in a)
    assert len(counts) >= 2, counts
    # the 150 kb interval is beyond the -w^2 exact envelope: the approximate tier
    assert a[-1].tier == 2
