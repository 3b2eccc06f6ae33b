"""Sliding-window semiglobal alignment (alignSlidingWindow, alignSlidingWindow.cpp:457-590) on
the GPU through aw_align_sliding_window_batch, one interval at a time and batched (window k of
every interval in one call), against the compiled reference's own alignSlidingWindow
(oracle/ref_rescue_shim.cpp) on the same intervals: the score and both rows."""
import numpy as np
import pytest

from anchorwave_b200 import ksw2
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu
PEN = (0, -4, -4, -2, -24, -1)  # matching score, mismatch, gap penalties (AnchorWave's, negative)


def _intervals(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        t = W.random_dna(rng, int(rng.integers(100, 4000)))
        q = W.mutate(rng, t, 0.05, 0.01, 4.0)
        if i % 3 == 0 and len(q) > 600:
            at = int(rng.integers(0, len(q) - 500))
            q = np.concatenate([q[:at], q[at + int(rng.integers(20, 400)):]])
        dq, dd = W.to_ascii(q).decode(), W.to_ascii(t).decode()
        if i % 5 == 2:
            dd = dd[:7] + "N" + dd[8:]
        out.append((dq, dd))
    return out


@pytest.mark.parametrize("win", [150, 400, 2000])
def test_sliding_window_batch_vs_compiled_reference(gpu, reference, win):
    pairs = _intervals(win, 20)
    got = ksw2.align_sliding_window_batch(pairs, win, *PEN)
    for (dq, dd), g in zip(pairs, got):
        exp = reference.sliding_window(dq, dd, win, PEN[0], PEN[1:])
        assert g == exp, (len(dq), len(dd), win)
        assert g[1].replace("-", "") == dq and g[2].replace("-", "") == dd


def test_sliding_window_single_equals_batch(gpu):
    pairs = _intervals(3, 6)
    batch = ksw2.align_sliding_window_batch(pairs, 300, *PEN)
    for (dq, dd), b in zip(pairs, batch):
        assert ksw2.align_sliding_window(dq, dd, 300, *PEN) == b
