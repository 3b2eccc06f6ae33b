"""Full-width KSW2 on the two-cells-per-instruction strip kernel with scoring other than
AnchorWave's default: random substitution matrices over alphabets of 2 to 8 codes (the
kernel's per-lane score profile holds 8 codes), and gap penalties at the edge of the
magnitude bound under which the kernel's 16-bit fields are exact.  Bit-exact against the
oracle restatement: every ksw_extz_t field and the CIGAR."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
RIGHT = 0x02


def _mutated(rng, m, n):
    t = rng.integers(0, m, n).astype(np.uint8)
    q = t.copy()
    sub = rng.random(n) < 0.1
    q[sub] = rng.integers(0, m, int(sub.sum()))
    # a few indels
    for _ in range(int(rng.integers(0, 4))):
        at = int(rng.integers(0, max(1, len(q) - 1)))
        if rng.random() < 0.5:
            q = np.concatenate([q[:at], q[at + int(rng.integers(1, 30)):]])
        else:
            q = np.concatenate([q[:at], rng.integers(0, m, int(rng.integers(1, 30))).astype(np.uint8), q[at:]])
    return (q if len(q) else t[:1].copy()), t


def _matrix(rng, m, lo):
    """mat[0] is the largest entry (the strip kernel's clamp), every entry <= 0."""
    mat = rng.integers(lo, 0, size=(m, m))
    np.fill_diagonal(mat, 0)
    return [int(x) for x in mat.flatten()]


@pytest.mark.parametrize("m", [2, 4, 5, 8])
@pytest.mark.parametrize("flag", [0, RIGHT])
def test_random_matrices(gpu, restatement, m, flag):
    rng = np.random.default_rng(10 * m + flag)
    mat = _matrix(rng, m, -12)
    qs, ts = [], []
    for _ in range(24):
        q, t = _mutated(rng, m, int(rng.integers(1, 1800)))
        qs.append(q)
        ts.append(t)
    res = gpu.ksw_extd2_batch(qs, ts, mat, 4, 2, 24, 1, flag=flag, m=m)
    for q, t, r in zip(qs, ts, res):
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, 4, 2, 24, 1, flag=flag, m=m)
        assert r.key() == o.key(), (m, len(q), len(t))


@pytest.mark.parametrize("pen,lo", [((20, 5, 24, 1), -50), ((30, 3, 33, 0), -34), ((12, 8, 59, 1), -20)])
@pytest.mark.parametrize("flag", [0, RIGHT])
def test_magnitude_edge(gpu, restatement, pen, lo, flag):
    """(q2+e2)+(q+e)+|min score| = 100, the largest magnitude the strip kernel takes (and
    |min score| <= 2(q+e), below which the reference returns at once)."""
    rng = np.random.default_rng(abs(lo) + flag)
    mat = [0 if i == j else lo for i in range(5) for j in range(5)]
    qs, ts = [], []
    for _ in range(16):
        q, t = _mutated(rng, 4, int(rng.integers(50, 2500)))
        qs.append(q)
        ts.append(t)
    res = gpu.ksw_extd2_batch(qs, ts, mat, *pen, flag=flag)
    for q, t, r in zip(qs, ts, res):
        o = restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, *pen, flag=flag)
        assert r.key() == o.key(), (pen, lo, len(q), len(t))
