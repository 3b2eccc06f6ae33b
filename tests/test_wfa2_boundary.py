"""The WFA2-lib-typed boundary of the GPU WFA aligner (include/anchorwave_b200_wfa2.h).

* CPU: the wavefront_aligner_attr_t and cigar_t that the header declares have WFA2-lib's
  memory layout (a program printing sizes and member offsets, compiled once against
  WFA2-lib's own headers in the reference tree and once against the header, must print the
  same), and the entry refuses the attributes it does not provide.
* GPU: oracle/_ref/wfa2_abi_check, a caller written like AnchorWave's WFA adapter
  (WfaAlignment.cpp:143-170: WFA2-lib's wavefront_aligner_attr_default, then its own fields),
  aligns every pair with the compiled WFA2-lib and through the GPU entries with the same
  attribute struct and requires identical status, scores and CIGAR operations.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.environ.get("ANCHORWAVE_REFERENCE") or os.path.join(os.sep, "root", "reference")
CHECK = os.path.join(ROOT, "oracle", "_ref", "wfa2_abi_check")


def _compile(tmp_path, name, src, flags, libs=()):
    exe = str(tmp_path / name)
    r = subprocess.run(["gcc", "-std=gnu99", "-w", "-I", os.path.join(ROOT, "include"), *flags, src, "-o", exe,
                        *libs], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_wfa2_types_have_wfa2_lib_layout(tmp_path):
    if not os.path.isdir(os.path.join(REF, "WFA2-lib")):
        pytest.skip("the reference tree (WFA2-lib headers) is not present")
    src = os.path.join(ROOT, "oracle", "wfa2_layout.c")
    a = _compile(tmp_path, "with_wfa2", src, ["-DAW_WITH_WFA2", "-I", REF, "-I", os.path.join(REF, "WFA2-lib")])
    b = _compile(tmp_path, "mirror", src, [])
    out_a = subprocess.run([a], check=True, capture_output=True, text=True).stdout
    out_b = subprocess.run([b], check=True, capture_output=True, text=True).stdout
    assert out_a == out_b
    assert "sizeof(wavefront_aligner_attr_t)" in out_a


REJECT_SRC = r"""
#include <stdio.h>
#include <string.h>
#include "anchorwave_b200_wfa2.h"
static int expect_null(wavefront_aligner_attr_t a, const char *what) {
    if (wavefront_aligner_new_wfa2_gpu(&a) != NULL) { printf("accepted %s\n", what); return 1; }
    if (!strstr(aw_last_error(), what)) { printf("message for %s: %s\n", what, aw_last_error()); return 1; }
    return 0;
}
int main(void) {
    wavefront_aligner_attr_t base = wavefront_aligner_attr_default_gpu, a;
    int bad = 0;
    if (base.distance_metric != gap_affine || base.heuristic.strategy != wf_heuristic_wfadaptive ||
        base.system.max_memory_abort != UINT64_MAX || base.affine2p_penalties.gap_opening2 != 24 ||
        base.system.min_offsets_per_thread != 500) { printf("defaults\n"); return 1; }
    base.distance_metric = gap_affine_2p, base.heuristic.strategy = wf_heuristic_none;
    a = base; a.distance_metric = gap_affine; bad |= expect_null(a, "distance_metric");
    a = base; a.affine2p_penalties.match = -1; bad |= expect_null(a, "match");
    a = base; a.alignment_form.span = alignment_endsfree; bad |= expect_null(a, "end-to-end");
    a = base; a.alignment_form.extension = true; bad |= expect_null(a, "end-to-end");
    a = base; a.heuristic.strategy = wf_heuristic_xdrop; bad |= expect_null(a, "heuristic");
    a = base; a.memory_mode = wavefront_memory_ultralow; bad |= expect_null(a, "memory_mode");
    a = base; a.mm_allocator = (mm_allocator_t *)&a; bad |= expect_null(a, "mm_allocator");
    if (wavefront_aligner_new_wfa2_gpu(NULL) != NULL) bad = 1;
    return bad;
}
"""


def test_wfa2_entry_refuses_what_it_does_not_provide(tmp_path):
    src = tmp_path / "reject.c"
    src.write_text(REJECT_SRC)
    lib_dir = os.path.join(ROOT, "anchorwave_b200")
    exe = _compile(tmp_path, "reject", str(src), [], ["-L", lib_dir, "-l:libaw_b200.so", f"-Wl,-rpath,{lib_dir}"])
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


def _pairs(tmp_path):
    sys.path.insert(0, ROOT)
    from anchorwave_b200 import workloads as W
    ps = W.batched_wfa_set(96, seed=77, lmin=20, lmax=3000)
    rows = [(W.to_ascii(t).decode(), W.to_ascii(q).decode()) for q, t in zip(ps.queries, ps.targets)]
    rng = np.random.default_rng(5)
    base = W.to_ascii(W.random_dna(rng, 400)).decode()
    rows += [(base, base), ("A", "C"), ("ACGT", "ACGT"), (base, base[:150] + "NNNN" + base[150:]),
             (base[:300], base), ("GATTACA" * 20, "GATACA" * 20)]
    f = tmp_path / "pairs.tsv"
    f.write_text("".join(f"{p}\t{t}\n" for p, t in rows))
    return str(f), len(rows)


@pytest.mark.gpu
@pytest.mark.parametrize("mode,singletrack", [(0, 0), (0, 1), (1, 0), (2, 0)])
def test_wfa2_caller_gets_wfa2_lib_results(gpu, tmp_path, mode, singletrack):
    if not os.path.exists(CHECK):
        pytest.skip("oracle/_ref/wfa2_abi_check is not built (needs the reference tree)")
    path, n = _pairs(tmp_path)
    r = subprocess.run([CHECK, path, str(mode), str(singletrack)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr[-2000:]
    words = r.stdout.split()
    assert words[:4] == ["pairs", str(n), "identical", str(n)]
    assert int(words[5]) >= 2 * n - 8  # two probe calls per completed alignment
