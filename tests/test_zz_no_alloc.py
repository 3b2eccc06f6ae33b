"""GPU test of aw_ksw_extd2_device_noalloc, the allocation-free KSW2 entry point.

That entry serves callers that cannot allocate device memory at call time (a process
whose device memory is held by its own caching allocator, or a latency-bound loop
that cannot take cudaMalloc's implicit synchronisation): they hand in their own
device buffers and the library's scratch comes from a fixed __device__ array.
The tests call it through the C ABI twice in a row, on pairs of different sizes so
that the second call starts from the scratch contents the first one left behind,
and check every result field and CIGAR word against the existing entry point
ksw_extd2_gpu and against the oracle's restatement (bit-exact, as all KSW2 parity
tests here), for every flag the entry accepts and for the pairs that ksw_extd2
answers without DP.  Around warmed-up calls the device's free memory must not change.
The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu

FIELDS = ("score", "max", "max_q", "max_t", "mqe", "mqe_t", "mte", "mte_q", "n_cigar", "zdropped", "reach_end",
          "stopped")
PEN = (4, 2, 24, 1)


def _noalloc(lib, torch, q, t, mat, pen, flag=0, with_cigar=True):
    dq = torch.from_numpy(np.ascontiguousarray(q).copy() if len(q) else np.zeros(1, np.uint8)).cuda()
    dt = torch.from_numpy(np.ascontiguousarray(t).copy() if len(t) else np.zeros(1, np.uint8)).cuda()
    res = torch.full((12,), -7, dtype=torch.int32, device="cuda")
    cap = len(q) + len(t)
    cig = torch.zeros(max(cap, 1), dtype=torch.int32, device="cuda") if with_cigar else None
    matc = (ctypes.c_int8 * len(mat))(*mat)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.aw_ksw_extd2_device_noalloc(len(q), dq.data_ptr(), len(t), dt.data_ptr(), 5, matc, *pen, flag,
                                         res.data_ptr(), cig.data_ptr() if with_cigar else None, cap, stream)
    torch.cuda.synchronize()
    r = res.cpu().numpy().tolist()
    out = dict(zip(FIELDS, r))
    n = max(0, r[8])
    out["cigar"] = [int(x) & 0xFFFFFFFF for x in cig.cpu().numpy()[:n]] if with_cigar else []
    return rc, out


def _fields(r):
    d = {k: getattr(r, k) for k in FIELDS}
    d["cigar"] = list(r.cigar)
    return d


# flags the entry accepts (the strip kernel's set), each with and without the CIGAR
FLAGS = [0, oracle.KSW_EZ_SCORE_ONLY, oracle.KSW_EZ_RIGHT, oracle.KSW_EZ_GENERIC_SC, oracle.KSW_EZ_REV_CIGAR,
         oracle.KSW_EZ_SEMIGLOBAL_END, oracle.KSW_EZ_RIGHT | oracle.KSW_EZ_REV_CIGAR]


@pytest.mark.parametrize("flag", FLAGS)
def test_noalloc_matches_existing_entry_and_oracle_on_two_calls(gpu, restatement, flag):
    torch = pytest.importorskip("torch")
    from anchorwave_b200 import _lib
    rng = np.random.default_rng(4242 + flag)
    mat = oracle.anchorwave_matrix(-4)
    cases = [W.divergent_pair(rng, 4200, 0.08, 0.08, 4.0), W.divergent_pair(rng, 650, 0.12, 0.12, 4.0)]
    if flag & oracle.KSW_EZ_GENERIC_SC:  # N bases (code 4) on both sides
        cases = [(np.where(rng.random(len(q)) < 0.02, 4, q).astype(np.uint8), t) for q, t in cases]
    score_only = bool(flag & oracle.KSW_EZ_SCORE_ONLY)
    for q, t in cases:  # two calls in a row on the shared scratch array
        rc, got = _noalloc(_lib.lib, torch, q, t, mat, PEN, flag, with_cigar=not score_only)
        assert rc == 0, _lib.last_error()
        exp = _fields(gpu.ksw_extd2(q, t, mat, *PEN, flag=flag))
        assert got == exp
        ora = _fields(restatement.ksw_extd2(q.tobytes(), t.tobytes(), mat, *PEN, flag=flag))
        assert got == ora


def test_noalloc_pairs_answered_without_dp(gpu, restatement):
    torch = pytest.importorskip("torch")
    from anchorwave_b200 import _lib
    mat = oracle.anchorwave_matrix(-4)
    t = np.array([0, 1, 2, 3, 0, 1], np.uint8)
    for q in (np.zeros(0, np.uint8), np.array([2], np.uint8)):
        for tt in (t, np.zeros(0, np.uint8)):
            rc, got = _noalloc(_lib.lib, torch, q, tt, mat, PEN)
            assert rc == 0, _lib.last_error()
            assert got == _fields(restatement.ksw_extd2(q.tobytes(), tt.tobytes(), mat, *PEN))


def test_noalloc_allocates_no_device_memory(gpu):
    torch = pytest.importorskip("torch")
    from anchorwave_b200 import _lib
    rng = np.random.default_rng(99)
    mat = oracle.anchorwave_matrix(-4)
    q, t = W.divergent_pair(rng, 3000, 0.05, 0.05, 4.0)
    dq = torch.from_numpy(q.copy()).cuda()
    dt = torch.from_numpy(t.copy()).cuda()
    res = torch.zeros(12, dtype=torch.int32, device="cuda")
    cig = torch.zeros(len(q) + len(t), dtype=torch.int32, device="cuda")
    matc = (ctypes.c_int8 * len(mat))(*mat)
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        rc = _lib.lib.aw_ksw_extd2_device_noalloc(len(q), dq.data_ptr(), len(t), dt.data_ptr(), 5, matc, *PEN, 0,
                                                  res.data_ptr(), cig.data_ptr(), len(q) + len(t), stream)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()

    call()  # resolves the scratch address and loads the kernels
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        call()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_rejects_pairs_beyond_the_scratch_array(gpu):
    torch = pytest.importorskip("torch")
    from anchorwave_b200 import _lib
    rng = np.random.default_rng(7)
    q, t = W.divergent_pair(rng, 9000, 0.02, 0.02, 4.0)
    rc, _ = _noalloc(_lib.lib, torch, q, t, oracle.anchorwave_matrix(-4), PEN)
    assert rc == -3 and "scratch" in _lib.last_error()


def test_noalloc_refuses_the_deterministic_stop(gpu):
    torch = pytest.importorskip("torch")
    from anchorwave_b200 import _lib
    rng = np.random.default_rng(8)
    q, t = W.divergent_pair(rng, 500, 0.05, 0.05, 4.0)
    _lib.lib.aw_ksw_set_stop_antidiagonal(256, 100)
    try:
        rc, _ = _noalloc(_lib.lib, torch, q, t, oracle.anchorwave_matrix(-4), PEN)
    finally:
        _lib.lib.aw_ksw_set_stop_antidiagonal(0, -1)
    assert rc == -5 and "aw_ksw_set_stop_antidiagonal" in _lib.last_error()
