"""GPU test of aw_ksw_extd2_device_noalloc, the allocation-free KSW2 entry point.

That entry serves callers that cannot allocate device memory at call time (a process
whose device memory is held by its own caching allocator, or a latency-bound loop
that cannot take cudaMalloc's implicit synchronisation): they hand in their own
device buffers and the library's scratch comes from a fixed __device__ array.
The test calls it through the C ABI twice in a row, on pairs of different sizes so
that the second call starts from the scratch contents the first one left behind,
and checks every result field and CIGAR word against the existing entry point
ksw_extd2_gpu (bit-exact, as all KSW2 parity tests here).  The file is named so
that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

import oracle
from anchorwave_b200 import workloads as W

pytestmark = pytest.mark.gpu

FIELDS = ("score", "max", "max_q", "max_t", "mqe", "mqe_t", "mte", "mte_q", "n_cigar", "zdropped", "reach_end",
          "stopped")


def _noalloc(lib, torch, q, t, mat, pen, flag=0):
    dq = torch.from_numpy(q.copy()).cuda()
    dt = torch.from_numpy(t.copy()).cuda()
    res = torch.full((12,), -7, dtype=torch.int32, device="cuda")
    cap = len(q) + len(t)
    cig = torch.zeros(cap, dtype=torch.int32, device="cuda")
    matc = (ctypes.c_int8 * len(mat))(*mat)
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.aw_ksw_extd2_device_noalloc(len(q), dq.data_ptr(), len(t), dt.data_ptr(), 5, matc, *pen, flag,
                                         res.data_ptr(), cig.data_ptr(), cap, stream)
    torch.cuda.synchronize()
    r = res.cpu().numpy().tolist()
    out = dict(zip(FIELDS, r))
    out["cigar"] = [int(x) & 0xFFFFFFFF for x in cig.cpu().numpy()[: max(0, r[8])]]
    return rc, out


def test_noalloc_matches_existing_entry_on_two_calls(gpu):
    torch = pytest.importorskip("torch")
    from anchorwave_b200 import _lib
    rng = np.random.default_rng(4242)
    mat = oracle.anchorwave_matrix(-4)
    pen = (4, 2, 24, 1)
    cases = [W.divergent_pair(rng, 4200, 0.08, 0.08, 4.0), W.divergent_pair(rng, 650, 0.12, 0.12, 4.0)]
    for q, t in cases:  # two calls in a row on the shared scratch array
        rc, got = _noalloc(_lib.lib, torch, q, t, mat, pen)
        assert rc == 0, _lib.last_error()
        ref = gpu.ksw_extd2(q, t, mat, *pen)
        exp = {k: getattr(ref, k) for k in FIELDS}
        exp["cigar"] = list(ref.cigar)
        assert got == exp


def test_noalloc_rejects_pairs_beyond_the_scratch_array(gpu):
    torch = pytest.importorskip("torch")
    from anchorwave_b200 import _lib
    rng = np.random.default_rng(7)
    q, t = W.divergent_pair(rng, 9000, 0.02, 0.02, 4.0)
    rc, _ = _noalloc(_lib.lib, torch, q, t, oracle.anchorwave_matrix(-4), (4, 2, 24, 1))
    assert rc == -3 and "scratch" in _lib.last_error()
