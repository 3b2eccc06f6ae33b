"""CPU: the C-ABI library loads and exports every function and object the include/*.h headers declare;
host-side helpers (workload generators, CIGAR decoding, two-piece rescoring) behave like the
reference's; without a GPU the entry points fail loudly instead of falling back to the CPU."""
import ctypes
import os
import re

import numpy as np

import oracle
from anchorwave_b200 import _lib, ksw2, workloads as W

INCLUDE = os.path.join(os.path.dirname(os.path.dirname(__file__)), "include")
HEADERS = sorted(os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h"))


def header_functions():
    names = set()
    for h in HEADERS:
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        text = "\n".join(ln for ln in text.splitlines() if not ln.lstrip().startswith("typedef"))
        names |= set(re.findall(r"^[A-Za-z_][\w \*]*?\b(\w+)\s*\(", text, flags=re.M))
    return sorted(n for n in names if n not in ("defined",))


def header_data_symbols():
    names = set()
    for h in HEADERS:
        names |= set(re.findall(r"^extern const \w+ (\w+);", open(h).read(), flags=re.M))
    return sorted(names)


def test_header_declares_expected_entry_points():
    names = header_functions()
    for required in ("ksw_extd2_gpu", "ksw_extd2_singletrack_gpu", "aw_ksw_extd2_batch"):
        assert required in names


def test_library_exports_every_header_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in header_functions() + header_data_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    assert "wavefront_aligner_new_wfa2_gpu" in header_functions()
    assert header_data_symbols() == ["wavefront_aligner_attr_default_gpu"]
    assert set(_lib.EXPORTS) <= set(header_functions()) | set(header_data_symbols())


def test_no_cpu_fallback_without_gpu():
    if _lib.lib.aw_device_count() > 0:
        return  # GPU present: covered by the gpu tests
    r = ksw2.ksw_extd2(b"\x00\x01\x02", b"\x00\x01\x03", ksw2.anchorwave_matrix(-4), 4, 2, 24, 1)
    assert r.zdropped == 1 and r.n_cigar == 0
    assert _lib.last_error()


def test_workloads_deterministic_and_shaped():
    a = W.batched_full_set(32, seed=1)
    b = W.batched_full_set(32, seed=1)
    assert all((x == y).all() for x, y in zip(a.queries, b.queries))
    assert all(200 <= len(t) <= 20000 for t in a.targets)
    q, t = W.plain_pair(0)
    assert len(t) == 5000 and 4000 < len(q) < 5000
    assert W.band_cells(100, 100, -1) == 100 * 100


def test_decode_and_rescore_match_reference_semantics(restatement):
    rng = np.random.default_rng(9)
    for _ in range(20):
        qc, tc = W.divergent_pair(rng, int(rng.integers(30, 400)), 0.02, 0.2, 4.0)
        r = restatement.ksw_extd2(qc.tobytes(), tc.tobytes(), oracle.anchorwave_matrix(-4), 4, 2, 24, 1)
        qs, ts = W.to_ascii(qc).decode(), W.to_ascii(tc).decode()
        aq, ad, qp, tp = ksw2.decode_cigar(r.cigar, qs, ts)
        assert qp == len(qs) and tp == len(ts) and len(aq) == len(ad)
        # in full mode the emitted CIGAR's two-piece score is the DP optimum
        assert ksw2.score_gapped_two_piece_affine(aq, ad, -4, -4, -2, -24, -1) == r.score


def test_wfa_attribute_checks_on_the_host():
    """wavefront_aligner_new_gpu rejects what WFA2-lib rejects (wavefront_penalties.c:141-150)
    and the memory modes it does not provide, before touching a device."""
    from anchorwave_b200._lib import WfaAttr
    lib = _lib.lib
    bad = [WfaAttr(0, 4, 2, 24, 1, 0, 0, 0), WfaAttr(4, -1, 2, 24, 1, 0, 0, 0), WfaAttr(4, 4, 0, 24, 1, 0, 0, 0),
           WfaAttr(4, 4, 2, 24, 0, 0, 0, 0), WfaAttr(4, 4, 2, 24, 1, 0, 3, 0), WfaAttr(4, 4, 2, 24, 1, 0, -1, 0)]
    for a in bad:
        assert not lib.wavefront_aligner_new_gpu(ctypes.byref(a))
        assert _lib.last_error()
    assert not lib.wavefront_aligner_new_gpu(ctypes.byref(bad[4]))
    assert "memory_mode" in _lib.last_error()


def test_sequence_summary_argument_checks_on_the_host():
    """aw_sequence_summary_batch validates its arguments before any device work: an empty
    batch succeeds with no entries, NULL arrays and a zero sampling modulo are rejected."""
    lib = _lib.lib
    assert lib.aw_sequence_summary_batch(0, None, None, None, None, None, None, None, None) == 0
    assert lib.aw_sequence_summary_sketches(None, None, 0) == 0
    assert lib.aw_sequence_summary_batch(1, None, None, None, None, None, None, None, None) < 0
    q = (ctypes.c_char_p * 1)(b"ACGT")
    ln = (ctypes.c_int64 * 1)(4)
    out = (ctypes.c_uint8 * 160)()
    ident = (ctypes.c_int * 1)()
    mods = (ctypes.c_uint64 * 3)(0, 1, 1)
    assert lib.aw_sequence_summary_batch(1, q, ln, q, ln, mods, out, ident, None) < 0
    assert "modulo" in _lib.last_error()
    neg = (ctypes.c_int64 * 1)(-1)
    assert lib.aw_sequence_summary_batch(1, q, neg, q, ln, None, out, ident, None) < 0


def test_summary_struct_layouts_agree():
    """aw_sequence_summary_t as the Python mirror and the oracles see it."""
    from anchorwave_b200.selector import SequenceSummary
    assert ctypes.sizeof(SequenceSummary) == 80
    assert ctypes.sizeof(oracle.SummaryOut) == 56
