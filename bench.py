"""Benchmark of the batched KSW2 alignment stage on B200 (one JSON line on rank 0).

Workload (default): 4,096 interval pairs, target length log-uniform 200 bp-20 kb, divergence
U(1%,15%) (80% substitutions, 20% indels of geometric length mean 4), AnchorWave scoring
(match 0, mismatch -4, gap 4+2l / 24+l), global ksw_extd2 with CIGAR.  Seeded synthetic
sequences stand in for the reference's B73/Mo17 intervals.

A step = one pass of the hot path over the whole batch: the DP of every pair, the traceback
and the CIGARs.
  * value: inputs already resident in HBM (plan API), CUDA events around K steps on the
    plan's stream; GCUPS = total DP cells / time.
  * e2e: the same batch through the public C-ABI call aw_ksw_extd2_batch with host buffers
    (pinned staging, H2D of the sequences, D2H of results and CIGARs) per step.
  * plain_per_call: the plain per-call GPU form (one ksw_extd2_gpu call per pair) on a
    512-pair sample of the same workload (batched_vs_plain_pairs_per_s compares the two).
  * plain_5kb: the plain single-pair workload as specified (1,000 seeded 5 kb pairs with a
    500 bp deletion, one ksw_extd2_gpu call each, p50/p99), beside the compiled reference's
    per-call latency (single-threaded calls) on the same pairs, results compared.
  * cpu_baseline: AnchorWave's own AVX KSW2 compiled from the reference tree (oracle/_ref),
    all host threads, bounded sample; every pair it finishes is compared field by field
    (ksw_extz_t + CIGAR, through a result hash) with the device-resident results (parity).
  * roofline: the strip kernel is bound by integer issue; it computes two cells per
    instruction in 16-bit fields, so the achieved op rate (DP cells x 47 reference int ops
    per cell / DP-phase CUDA-event time) is set against the packed-field peak measured live
    by aw_int16x2_peak_ops() (the 32-bit peak, aw_int32_peak_ops(), is reported beside it);
    the traceback store stream is reported against HBM bandwidth.
  * serving: a 20,000-request trace (lengths to 500 kb) routed by AnchorWave's own selector,
    through the continuous-batching server under a 150 GB HBM budget (saturated and at 80%
    offered load with p50/p99 latency), beside the plain per-call GPU path on a sample.
  * long_banded: 64 pairs of 100 kb-1 Mb, w = 10%, banded and Singletrack (one execution
    each), every CIGAR checked and re-scored, beside the reference's CPU code on the pairs
    whose host traceback fits a safe share of the host memory.
  * wfa: 16,384 pairs of 100 bp-10 kb (0.5-5%), high memory (standard and Singletrack) and
    medium memory (piggyback), device memory per pair, beside WFA2-lib in the same mode.
  * selector_summary: the selector's sequence pass (k-mer sketches, composition, entropy,
    fingerprints) over the headline pairs, beside the compiled selector.

`--impl reference` times the reference CPU implementation (oracle/_ref) on the same workload,
metric and unit: each step is a time-bounded sample that continues where the previous step
stopped, so the timed steps walk the whole batch.  With torchrun (N>1) every rank aligns its
own batch (weak scaling, no collective on the data path); rank 0 prints the line.

The line ends with `cpu_baseline` (parity included) and a compact `summary` of the
sub-measurements (batched vs plain, p50/p99 latencies, parity counts, WFA and long-pair rates).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

OPS_PER_CELL_CIGAR = 47
OPS_PER_CELL_SCORE = 31
# dram__bytes_read.sum + dram__bytes_write.sum per DP cell of ksw_full_kernel in one ncu
# capture (48-pair case: 3.2 MB read + 1.64 GB written for 1.64e9 cells)
NCU_DRAM_BYTES_PER_CELL = 1.002
METRIC = "batched GCUPS & pairs/s vs plain per-call on 1 B200, bit-exact; p50/p99 latency"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--pairs", type=int, default=4096)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--cpu-budget", type=float, default=15.0, help="seconds of CPU-baseline work")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-sample", type=int, default=512,
                    help="pairs of the batched workload aligned one ksw_extd2_gpu call at a time")
    ap.add_argument("--plain-pairs", type=int, default=1000,
                    help="pairs of the plain 5 kb workload (0 skips it)")
    ap.add_argument("--serve-requests", type=int, default=20000,
                    help="requests of the serving trace (0 skips the serving measurement)")
    ap.add_argument("--no-long-banded", action="store_true", help="skip the long banded/Singletrack sample")
    ap.add_argument("--long-banded-pairs", type=int, default=64)
    ap.add_argument("--long-banded-min", type=int, default=100_000)
    ap.add_argument("--long-banded-max", type=int, default=1_000_000)
    ap.add_argument("--long-banded-indel", type=int, default=50_000, help="longest of the long indels")
    ap.add_argument("--long-banded-budget-gb", type=float, default=0.0,
                    help="traceback budget of the long banded sample in GB (0: the library default); a small "
                         "budget makes its pairs recompute their tracebacks in rounds")
    ap.add_argument("--wfa-pairs", type=int, default=16384, help="pairs of the batched WFA workload (0 skips it)")
    ap.add_argument("--wfa-long-pairs", type=int, default=3,
                    help="single long divergent WFA intervals timed alone (0 skips them)")
    ap.add_argument("--no-selector-summary", action="store_true",
                    help="skip the selector sequence-pass measurement")
    ap.add_argument("--wfa-pool-gb", type=float, default=0.0,
                    help="device wavefront pool of the WFA workload (0: most of the free memory)")
    return ap.parse_args()


def dist_init(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


def barrier(pg):
    if pg is not None:
        import torch
        pg.barrier()
        torch.cuda.synchronize()


def max_over_ranks(pg, v: float) -> float:
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, val in zip(names, p[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload(args, rank):
    from anchorwave_b200 import workloads as W
    return W.batched_full_set(args.pairs, seed=args.seed + rank)


def run_config(ps, world):
    """The config dict of both arms (identical keys and values)."""
    cells = ps.cells()
    return {"workload": ps.name, "pairs": len(ps), "cells": cells,
            "scoring": "match 0, mismatch -4, gap 4+2l/24+l", "form": "ksw_extd2 global with CIGAR",
            "parallelism": f"replicas x{world}",
            "l2": f"each step writes about {cells / 1e9:.0f} GB of traceback (1 B per cell), far above the "
                  f"126 MB L2"}


def sig(x, digits=4):
    """Rounds floats to `digits` significant digits (compact summary)."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}")
    if isinstance(x, dict):
        return {k: sig(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [sig(v, digits) for v in x]
    return x


def run_reference_arm(args):
    # under torchrun rank 0 alone times the reference's CPU code; the others exit without work
    # (no process group: no rank waits on another)
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    try:
        ref = oracle.Reference()
    except FileNotFoundError as e:
        print(json.dumps({"impl": "reference", "unavailable": f"compiled reference missing: {e}"}))
        return 0
    ps = workload(args, 0)
    mat = oracle.anchorwave_matrix(-4)
    import numpy as np
    n = len(ps)
    rng = np.random.default_rng(12345)
    order = rng.permutation(n)
    nthreads = os.cpu_count() or 1
    budget = max(2.0, min(30.0, 60.0 / max(1, args.steps + args.warmup)))
    state = {"start": 0}

    def step():
        # a time-bounded sample that continues where the previous step stopped, so that the
        # steps walk the whole batch in the seeded order
        rot = np.roll(order, -state["start"])
        qs = [ps.queries[i].tobytes() for i in rot]
        ts = [ps.targets[i].tobytes() for i in rot]
        r = ref.ksw_batch(qs, ts, mat, 4, 2, 24, 1, nthreads=nthreads, time_budget_s=budget)
        # pairs handed out before the deadline are all finished by the time the call returns
        finished = [j for j in range(n) if r["hash"][j] != 0][: r["done"]]
        cells = sum(len(qs[j]) * len(ts[j]) for j in finished)
        state["start"] = (state["start"] + len(finished)) % n
        return cells, len(finished), r["seconds"]

    for _ in range(args.warmup):
        step()
    tot_c = tot_p = tot_s = 0.0
    for _ in range(args.steps):
        c, p, s = step()
        tot_c += c
        tot_p += p
        tot_s += s
    gcups = tot_c / tot_s / 1e9
    sample = (f"each step aligns the workload's pairs in seeded order for {budget:.1f} s, continuing where the "
              f"previous step stopped ({int(tot_p)} pairs over the {args.steps} timed steps = "
              f"{tot_p / n:.2f} passes of the {n}-pair batch); ksw_extd2_{ref.isa} from the reference sources")
    line = {"metric": METRIC, "impl": "reference", "value": gcups, "unit": "GCUPS", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int8",
            "data": "synthetic (seeded; stands in for B73/Mo17 intervals)",
            "pairs_per_s": tot_p / tot_s,
            "config": run_config(ps, args.gpus),
            "cpu_baseline": {"value": gcups, "unit": "GCUPS", "cores": nthreads, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": gcups, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# Serving configuration: two workers (each with half of the device budget for its pooled
# traceback arena and wavefront pools) and micro-batches of up to 1,024 requests gave the
# best saturated rate and latency on the trace (more workers split the budget into smaller
# arenas, so the long banded class runs in more waves).
SERVE_SLOTS, SERVE_BATCH = 2, 1024
# offered load of the latency run, as a fraction of the saturated request rate
SERVE_LOAD = 0.8
# the HBM budget of the serving workload (traceback arenas and wavefront pools)
SERVE_HBM_BUDGET = 150 * 10**9


def plain_route_call(rt, q: bytes, t: bytes, mat, aligners):
    """One interval through the single-call form of its routed engine (the plain per-call GPU
    path): ksw_extd2_gpu / ksw_extd2_singletrack_gpu, wavefront_align_gpu, or the rescue
    procedures on one interval.  Returns a comparable result."""
    from anchorwave_b200 import ksw2, wfa
    pen = (-4, -4, -2, -24, -1)
    if rt.method in (0, 1):
        qc, f1 = ksw2.encode(q)
        tc, f2 = ksw2.encode(t)
        fn = ksw2.ksw_extd2_singletrack if rt.method == 1 else ksw2.ksw_extd2
        r = fn(qc, tc, mat, 4, 2, 24, 1, w=rt.band, flag=f1 | f2)
        return (r.score, tuple(r.cigar))
    if rt.method in (2, 3, 4, 5):
        al = aligners.get(rt.method)
        if al is None:
            al = aligners[rt.method] = wfa.WfaAligner(4, 4, 2, 24, 1, singletrack=rt.method == 3,
                                                      memory_mode=max(0, rt.method - 3))
        st = al.align(t, q)
        ops, score = al.cigar() if st == 0 else ("", 0)
        return (st, score, ops)
    if rt.method == 6:
        r = ksw2.align_score_certified_ksw2(q.decode(), t.decode(), rt.band, rt.band_max, *pen)
        return (r.status, r.score)
    return ksw2.align_sliding_window(q.decode(), t.decode(), rt.window, 0, *pen)[0]


def serving_measurement(nreq: int, rank: int, tuning=None, plain_sample: int = 400):
    """Serving trace (lengths log-normal, median 2 kb, sigma 1, clipped to 50 bp-500 kb;
    divergence and indels as the batched workload; 10% with repeat structure).  Every request
    is routed by AnchorWave's own selector (the routing front end: makeAlignmentSelectionPlan
    and the executor's first choice on an idle system) before it is submitted, then the
    continuous-batching server runs the trace under a 150 GB HBM budget: saturated
    throughput with all requests queued at once, then p50/p99 latency with Poisson arrivals
    at 80% of that rate.  Beside it, the plain per-call GPU path (each interval through the
    single-call form of its routed engine) on a seeded sample of the same trace, whose results
    must equal the served ones."""
    import collections

    import numpy as np

    from anchorwave_b200 import ksw2, serve
    from anchorwave_b200 import workloads as W
    try:
        from anchorwave_b200 import route
    except ImportError as e:
        return {"unavailable": f"routing front end missing: {e}"}
    t_all = time.perf_counter()

    def log(msg):
        print(f"[bench serving +{time.perf_counter() - t_all:.1f}s] {msg}", file=sys.stderr, flush=True)

    reqs = W.serving_trace(nreq, seed=4 + rank, lmax=500_000)
    t0 = time.perf_counter()
    routes = route.route_intervals([(r.query, r.target) for r in reqs])
    route_s = time.perf_counter() - t0
    log(f"{len(reqs)} requests generated and routed ({route_s:.1f} s)")
    mix = collections.Counter(rt.candidate for rt in routes)
    cells = sum(len(r.query) * len(r.target) for r in reqs)
    mat = ksw2.anchorwave_matrix(-4)

    cfg = {"slots": SERVE_SLOTS, "max_batch": SERVE_BATCH}

    def run(rate, keep=None):
        rng = np.random.default_rng(99)
        kept = {}
        with serve.AlignmentServer(mat, 4, 2, 24, 1, slots=cfg["slots"], max_batch=cfg["max_batch"],
                                   hbm_budget=SERVE_HBM_BUDGET) as srv:
            t0 = time.perf_counter()

            def producer():
                nxt = t0
                for r, rt in zip(reqs, routes):
                    if rate:
                        nxt += rng.exponential(1.0 / rate)
                        d = nxt - time.perf_counter()
                        if d > 0:
                            time.sleep(d)
                    srv.submit(r.id, rt.method, r.query, r.target, band=rt.band, band_max=rt.band_max,
                               window=rt.window, predicted_bytes=rt.predicted_bytes)

            th = threading.Thread(target=producer)
            th.start()
            got = 0
            while got < len(reqs):
                batch = srv.poll(4096, wait_ms=20)
                got += len(batch)
                if keep is not None:
                    for g in batch:
                        if g.id in keep:
                            kept[g.id] = g
            th.join()
            dt = time.perf_counter() - t0
            st = srv.stats()
        return dt, st, kept

    rng = np.random.default_rng(2024)
    sample = sorted(rng.choice(len(reqs), size=min(plain_sample, len(reqs)), replace=False).tolist())
    # the autotuner picks the worker slots and the micro-batch size for the lowest p99 at 80% of
    # the saturated rate of the default setting, each setting serving the whole trace
    from anchorwave_b200 import autotune
    dt0, _, _ = run(None)
    log(f"default setting saturated: {dt0:.1f} s")
    t_tune = time.perf_counter()
    (cfg["slots"], cfg["max_batch"]), trials = autotune.tune_serving(
        reqs, routes, mat, 4, 2, 24, 1, rate=SERVE_LOAD * len(reqs) / dt0, sample=len(reqs),
        hbm_budget=SERVE_HBM_BUDGET)
    if tuning is not None:
        tuning["serving"] = {"slots": cfg["slots"], "max_batch": cfg["max_batch"], "sample_requests": len(reqs),
                             "seconds": time.perf_counter() - t_tune,
                             "trials": [{k: (round(v, 1) if isinstance(v, float) else v) for k, v in t.items()}
                                        for t in trials]}
    log(f"tuned: {cfg}")
    dt_sat, st_sat, served = run(None, keep=set(sample))
    sat = len(reqs) / dt_sat
    log(f"saturated: {dt_sat:.1f} s")
    dt, st, _ = run(SERVE_LOAD * sat)
    log(f"80% load: {dt:.1f} s")
    # plain per-call GPU path on the sample, and its results against the served ones
    aligners = {}
    plain_s, same = 0.0, True
    for i in sample:
        r, rt = reqs[i], routes[i]
        t1 = time.perf_counter()
        res = plain_route_call(rt, r.query, r.target, mat, aligners)
        dt1 = time.perf_counter() - t1
        plain_s += dt1
        if dt1 > 1.0:
            log(f"plain call {i}: {rt.candidate} {len(r.query)}x{len(r.target)} {dt1:.1f} s")
        g = served[i]
        if rt.method in (0, 1):
            same &= (g.ksw[8], g.ksw[12]) == res
        elif rt.method in (2, 3, 4, 5):
            same &= g.wfa == res
        elif rt.method == 6:
            same &= g.ksw[8] == res[1]
        else:
            same &= g.ksw[8] == res
    for al in aligners.values():
        al.close()
    plain_pps = len(sample) / plain_s
    return {"requests": len(reqs), "cells": cells, "routing": dict(mix), "routing_s": route_s,
            "routed_by": "AnchorWave's makeAlignmentSelectionPlan (compiled unchanged) + the executor's first "
                         "choice on an idle system",
            "saturated_requests_per_s": sat, "saturated_gcups": cells / dt_sat / 1e9,
            "saturated_server_requests_per_s": len(reqs) / st_sat["elapsed_s"] if st_sat["elapsed_s"] else None,
            "offered_requests_per_s": SERVE_LOAD * sat, "load": SERVE_LOAD,
            "requests_per_s": len(reqs) / dt, "gcups": cells / dt / 1e9,
            "latency_ms_p50": 1e3 * st["latency_p50_s"], "latency_ms_p99": 1e3 * st["latency_p99_s"],
            "micro_batches": st["micro_batches"], "slots": cfg["slots"], "max_batch": cfg["max_batch"],
            "hbm_budget": SERVE_HBM_BUDGET,
            "plain_per_call": {"sample": len(sample), "requests_per_s": plain_pps,
                               "served_vs_plain": sat / plain_pps, "results_identical_to_served": bool(same)},
            "trace": "log-normal lengths (median 2 kb, sigma 1) clipped to 50 bp-500 kb, divergence U(1%,15%), 10% "
                     "repeat-rich; routed by AnchorWave's selector; Poisson arrivals at 80% of saturation; "
                     "cells = sum of qlen*tlen"}


def wfa_measurement(npairs: int, rank: int, cpu: bool, pool_gb: float = 0.0):
    """The batched gap-affine-2p WFA workload (lengths log-uniform 100 bp-10 kb, divergence
    0.5-5%, penalties x=4, o1=4, e1=2, o2=24, e2=1), standard and Singletrack in high memory
    and the medium-memory (piggyback) mode: pairs/s on the device and through the C call with
    host buffers, device memory per alignment, and the reference's WFA2 code in the same mode
    on the host cores on the same pairs (status, score and the whole CIGAR operation string of
    every pair the reference finished compared)."""
    import numpy as np

    from anchorwave_b200 import wfa
    from anchorwave_b200 import workloads as W
    ps = W.batched_wfa_set(npairs, seed=2 + rank)
    pats = [W.to_ascii(t) for t in ps.targets]
    txts = [W.to_ascii(q) for q in ps.queries]
    out = {"workload": ps.name, "pairs": len(ps), "matrix_cells": ps.cells()}
    dev = {}
    modes = (("standard", False, 0), ("singletrack", True, 0), ("medium", False, 1))
    for name, stk, mem in modes:
        al = wfa.WfaAligner(4, 4, 2, 24, 1, singletrack=stk, max_memory_abort=int(pool_gb * 2**30),
                            memory_mode=mem)
        al.align_batch_raw(pats[:64], txts[:64])
        runs = [al.align_batch_raw(pats, txts) for _ in range(2)]
        pair_max, total = al.memory()
        al.close()
        st, sc, offs, nops, ops, ms, secs = min(runs, key=lambda r: r[5])
        dev[name] = (st, sc, offs, nops, ops.raw)
        out[name] = {"device_ms": ms, "pairs_per_s": len(ps) / (ms * 1e-3),
                     "e2e_pairs_per_s": len(ps) / min(r[6] for r in runs),
                     "gcups_equivalent": ps.cells() / (ms * 1e-3) / 1e9,
                     "completed": int(np.sum(st == 0)),
                     "device_bytes_per_pair_mean": total / len(ps), "device_bytes_pair_max": pair_max}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        try:
            ref = oracle.Reference()
        except FileNotFoundError as e:
            out["cpu_reference"] = {"unavailable": str(e)}
            return out
        for name, stk, mem in modes:
            # the helper takes (queries, targets) and aligns pattern = target, text = query
            r = ref.wfa_batch(txts, pats, 4, 4, 2, 24, 1, singletrack=stk, time_budget_s=10.0, memory_mode=mem)
            done = [i for i in range(len(ps)) if r["n_ops"][i] > 0]
            st, sc, offs, nops, ops = dev[name]
            rops, roff = r["ops"], r["ops_offset"]
            # status, score and the whole operation string of every pair the reference finished
            same = all(st[i] == 0 and sc[i] == r["score"][i] and nops[i] == r["n_ops"][i] and
                       ops[offs[i]:offs[i] + nops[i]] == rops[roff[i]:roff[i] + nops[i]].tobytes() for i in done)
            cpu_pps = r["done"] / r["seconds"]
            out[name]["cpu_reference"] = {"pairs_per_s": cpu_pps, "threads": r["threads"], "pairs": len(done),
                                          "status_score_cigar_identical": same}
            out[name]["vs_cpu_reference"] = out[name]["pairs_per_s"] / cpu_pps
    return out


# Long divergent intervals of the kind AnchorWave's selector routes to SingletrackWfa
# (interval length, divergence): the latency of one interval alone, the cluster kernel's case.
WFA_LONG_PAIRS = ((12_000, 0.15), (24_000, 0.12), (40_000, 0.08))


def wfa_long_measurement(npairs: int, rank: int, cpu: bool):
    """Single long divergent intervals through the Singletrack WFA (high memory, penalties
    x=4, o1=4, e1=2, o2=24, e2=1), one call each: the device time of the call (a pair whose
    wavefronts outgrow a warp or a CTA moves to the 8-CTA cluster kernel) and, for the first,
    the same call with every pair kept on one warp; beside them the reference's WFA2 code on
    one host thread on the same interval (status, score and operation string compared)."""
    import time

    import numpy as np

    from anchorwave_b200 import wfa
    from anchorwave_b200 import workloads as W
    rng = np.random.default_rng(50 + rank)
    ref = None
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        try:
            ref = oracle.Reference()
        except FileNotFoundError:
            ref = None
    out = []
    for j, (length, d) in enumerate(WFA_LONG_PAIRS[:npairs]):
        q, t = W.divergent_pair(rng, length, d, d, 4.0)
        p_, t_ = W.to_ascii(t), W.to_ascii(q)
        al = wfa.WfaAligner(4, 4, 2, 24, 1, singletrack=True, max_memory_abort=4 << 30)
        al.align_batch([p_], [t_])
        (res,), ms = al.align_batch([p_], [t_])
        moved = al.launches()[2]
        rec = {"length": length, "divergence": d, "status": res[0], "score": res[1], "device_ms": ms,
               "on_cluster_kernel": bool(moved)}
        if j == 0:
            wfa.set_long(0)
            wfa.set_wide(0)
            try:
                _, ms1 = al.align_batch([p_], [t_])
            finally:
                wfa.set_long(1536)
                wfa.set_wide(8192, 1024, 8)
            rec["one_warp_device_ms"] = ms1
        al.close()
        if ref is not None:
            t0 = time.perf_counter()
            r = ref.wfa_align(p_, t_, 4, 4, 2, 24, 1, singletrack=True)
            rs = time.perf_counter() - t0
            rec["cpu_reference"] = {"seconds": rs, "threads": 1, "identical": tuple(r) == tuple(res)}
            rec["vs_cpu_reference"] = rs / (ms * 1e-3)
        out.append(rec)
    return out


def selector_summary_measurement(ps, rank: int, cpu: bool):
    """The selector's sequence pass (summarizeSequencePair: k-mer sketches at k = 9, 15, 21,
    composition, entropy, fingerprints) over the intervals of the headline workload, through
    aw_sequence_summary_batch with host buffers (bases/s of both sequences), and the
    reference's compiled selector on the host threads over the same pairs (fingerprints,
    sketch sizes and fractions compared)."""
    import time

    import numpy as np

    from anchorwave_b200 import selector
    from anchorwave_b200 import workloads as W
    qs = [W.to_ascii(q) for q in ps.queries]
    ts = [W.to_ascii(t) for t in ps.targets]
    bases = sum(len(q) for q in qs) + sum(len(t) for t in ts)
    selector.sequence_summary_raw(qs[:32], ts[:32])
    secs, dev = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        out, ident, h, p, ms = selector.sequence_summary_raw(qs, ts, copy=False)
        secs.append(time.perf_counter() - t0)
        dev.append(ms)
    best = min(secs)
    res = {"pairs": len(qs), "bases": bases, "e2e_bases_per_s": bases / best, "e2e_ms": 1e3 * best,
           "device_ms": min(dev), "device_bases_per_s": bases / (min(dev) * 1e-3),
           "sketch_entries": int(len(h)), "h2d_bytes": bases, "d2h_bytes": int(len(h)) * 12 + len(out) * 80}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        try:
            ref = oracle.Reference()
        except FileNotFoundError as e:
            res["cpu_reference"] = {"unavailable": str(e)}
            return res
        if not ref.has_summary:
            res["cpu_reference"] = {"unavailable": "compiled reference without the selector shim"}
            return res
        rsecs, rout, rident = ref.sequence_summary_batch(qs, ts)
        same = bool(np.array_equal(rident, ident))
        for j in range(2 * len(qs)):
            a, b = out[j], rout[j]
            same &= (a.fingerprint == b.fingerprint and list(a.sketch_count) == list(b.count) and
                     a.ambiguous_fraction == b.ambiguous_fraction and
                     a.low_complexity_fraction == b.low_complexity_fraction and
                     abs(a.normalized_entropy - b.normalized_entropy) <= 1e-9)
        res["cpu_reference"] = {"bases_per_s": bases / rsecs, "seconds": rsecs, "threads": os.cpu_count(),
                                "summaries_identical": same}
        res["vs_cpu_reference"] = res["e2e_bases_per_s"] / (bases / rsecs)
    return res


def cigar_check(res, q, t, mis=4, o1=4, e1=2, o2=24, e2=1):
    """(valid, rescored): the CIGAR consumes the whole query and target, and its two-piece
    affine score (match 0, mismatch -mis, gap min(o1 + l*e1, o2 + l*e2))."""
    import numpy as np
    qp = tp = 0
    sc = 0
    for c in res.cigar:
        ln, op = c >> 4, c & 0xF
        if op == 0:
            sc -= mis * int(np.count_nonzero(q[qp:qp + ln] != t[tp:tp + ln]))
            qp += ln
            tp += ln
        elif op in (1, 2):
            sc -= min(o1 + ln * e1, o2 + ln * e2)
            qp += ln if op == 1 else 0
            tp += ln if op == 2 else 0
        else:
            return False, None
    return qp == len(q) and tp == len(t), sc


def long_banded_measurement(rank: int, cpu: bool, npairs: int = 64, lmin: int = 100_000, lmax: int = 1_000_000,
                            long_max: int = 50_000, budget_gb: float = 0.0, tuning=None):
    """The long-interval banded and Singletrack workload (target length U(lmin, lmax), 30% of
    the query replaced by repeat structure, 3% substitutions, 5-20 long indels of U(1,
    long_max), w = 10% of the shorter length): one execution of the whole set per traceback,
    band GCUPS on the device (pairs whose traceback exceeds the HBM budget recompute it group
    by group; Singletrack pairs beyond the budget are refused like an allocation failure of the
    reference, zdropped = 1, and counted), every CIGAR checked to span both sequences and
    re-scored against ez.score; the reference's own CPU code on the pairs whose host traceback
    fits a safe share of the host memory (one thread per pair), results compared."""
    import numpy as np

    from anchorwave_b200 import ksw2
    from anchorwave_b200 import workloads as W
    ps = W.long_banded_set(npairs, seed=3 + rank, lmin=lmin, lmax=lmax, long_max=long_max)
    mat = ksw2.anchorwave_matrix(-4)
    pair_cells = [W.band_cells(len(q), len(t), w) for q, t, w in zip(ps.queries, ps.targets, ps.band)]
    reach = [W.band_reaches_end(len(q), len(t), w) for q, t, w in zip(ps.queries, ps.targets, ps.band)]
    bcells = sum(pair_cells)
    out = {"workload": ps.name, "pairs": len(ps), "band_cells": bcells,
           "shape": f"target U({lmin // 1000} kb, {lmax // 1000} kb), 30% repeats, 3% substitutions, "
                    f"5-20 long indels of U(1, {long_max // 1000} kb), w = 10% of the shorter length"}
    # kernels loaded before the timed executions
    warm = ksw2.KswPlan(ps.queries[:1], ps.targets[:1], mat, 4, 2, 24, 1, w=[64], flag=0x1000)
    warm.upload()
    warm.execute()
    warm.close()
    # the autotuner picks the banded kernel's columns per lane (4, 8, or the per-batch rule) on the
    # four pairs with the most band cells, score-only: the batch's largest pairs hold most of its
    # cells and run first, together, in its first wave.  Samples of small or random pairs (alone,
    # or with a traceback budget scaled to them) are chain-bound where the whole workload is
    # work-bound, and picked 4 columns, which made the whole workload 20-25% slower than 8.
    from anchorwave_b200 import autotune
    t_tune = time.perf_counter()
    pick = sorted(sorted(range(len(ps)), key=lambda i: -pair_cells[i])[:4])
    cols, trials = autotune.tune_band([ps.queries[i] for i in pick], [ps.targets[i] for i in pick],
                                      [ps.band[i] for i in pick], mat, 4, 2, 24, 1, flag=0x01, sample=len(pick),
                                      reps=1)
    if tuning is not None:
        tuning["band_kernel"] = {"columns_per_lane": cols, "trials_ms": {str(t["columns"]): t["ms"] for t in trials},
                                 "seconds": time.perf_counter() - t_tune, "sample_pairs": len(pick)}
    results = {}
    if budget_gb > 0:
        ksw2.set_traceback_budget(int(budget_gb * 1e9))
        out["traceback_budget_bytes"] = int(budget_gb * 1e9)
    for name, flag in (("banded", 0), ("singletrack", 0x1000)):
        plan = ksw2.KswPlan(ps.queries, ps.targets, mat, 4, 2, 24, 1, w=ps.band, flag=flag)
        plan.upload()
        ms = plan.execute()
        dp, bt = plan.timing()
        st = plan.stats()
        res = plan.download()
        plan.close()
        results[name] = res
        # pairs whose band becomes empty before the end: zdropped, no CIGAR, as the reference
        refused = [i for i, r in enumerate(res) if r.zdropped and r.n_cigar == 0 and reach[i]]
        ran = [i for i in range(len(ps)) if i not in set(refused)]
        rcells = sum(pair_cells[i] for i in ran)
        valid = rescored = 0
        for i in ran:
            if not reach[i]:
                continue
            ok, sc = cigar_check(res[i], ps.queries[i], ps.targets[i])
            valid += ok
            rescored += ok and sc == res[i].score
        out[name] = {"ms": ms, "dp_ms": dp, "traceback_ms": bt, "gcups": rcells / (ms * 1e-3) / 1e9,
                     "pairs_run": len(ran), "band_unreachable": len(ps) - sum(reach),
                     "refused_over_budget": len(refused), "cigars_spanning_both": valid,
                     # a restrictive band may report a frontier score that differs from its CIGAR's
                     # score (the reference re-scores for that reason, alignSlidingWindow.cpp:872-876)
                     "cigars_rescoring_to_score": rescored}
        ksw2.release_thread_buffers()
    ksw2.set_band_columns(0)
    if budget_gb > 0:
        ksw2.set_traceback_budget(0)
    if cpu:
        from concurrent.futures import ThreadPoolExecutor
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        try:
            ref = oracle.Reference()
        except FileNotFoundError as e:
            out["cpu_reference"] = {"unavailable": str(e)}
            return out
        try:
            import psutil
            avail = psutil.virtual_memory().available
        except Exception:
            avail = 16 << 30
        nthreads = os.cpu_count() or 1
        for name, variant, tracks in (("banded", 0, 1), ("singletrack", 2, 2)):
            # the reference's traceback matrix: (qlen + tlen - 1) x (ceil((w+1)/block) + 1) blocks per track
            def host_bytes(i):
                ql, tl, w = len(ps.queries[i]), len(ps.targets[i]), ps.band[i]
                return tracks * (ql + tl) * ((w + 1 + ref.block - 1) // ref.block + 1) * ref.block
            pick, tot = [], 0
            for i in sorted(range(len(ps)), key=host_bytes):
                if len(pick) >= nthreads or tot + host_bytes(i) > min(48 << 30, avail // 4):
                    break
                if results[name][i].zdropped and results[name][i].n_cigar == 0:
                    continue
                pick.append(i)
                tot += host_bytes(i)
            if not pick:
                out[name]["cpu_reference"] = {"unavailable": "no pair's traceback fits the host memory share"}
                continue

            def one(i):
                r = ref.ksw_batch([ps.queries[i].tobytes()], [ps.targets[i].tobytes()], mat, 4, 2, 24, 1,
                                  w=ps.band[i], variant=variant, nthreads=1)
                return int(r["hash"][0])
            t0 = time.perf_counter()
            with ThreadPoolExecutor(len(pick)) as ex:
                hashes = list(ex.map(one, pick))
            secs = time.perf_counter() - t0
            same = all(oracle.result_hash(results[name][i]) == h for i, h in zip(pick, hashes))
            pc = sum(pair_cells[i] for i in pick)
            out[name]["cpu_reference"] = {"pairs": len(pick), "band_cells": pc, "seconds": secs,
                                          "gcups": pc / secs / 1e9, "threads": len(pick), "isa": ref.isa,
                                          "results_identical": same,
                                          "sample": "the pairs with the smallest host traceback, one thread each"}
            out[name]["vs_cpu_reference"] = out[name]["gcups"] / (pc / secs / 1e9)
    return out


def cpu_baseline(ps, budget, res_dev):
    """The compiled reference (native ISA, all host threads) on the workload in seeded random
    order for `budget` seconds; every pair it finishes is compared with the device result
    (all ksw_extz_t fields and the CIGAR, through the shim's result hash)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle
    ref = oracle.Reference()
    rng = np.random.default_rng(54321)
    order = rng.permutation(len(ps))
    qs = [ps.queries[i].tobytes() for i in order]
    ts = [ps.targets[i].tobytes() for i in order]
    nthreads = os.cpu_count() or 1
    r = ref.ksw_batch(qs, ts, oracle.anchorwave_matrix(-4), 4, 2, 24, 1, nthreads=nthreads,
                      time_budget_s=budget)
    done_idx = [i for i in range(len(qs)) if r["hash"][i] != 0]
    cells = sum(len(qs[i]) * len(ts[i]) for i in done_idx)
    bad = [int(order[i]) for i in done_idx if oracle.result_hash(res_dev[order[i]]) != int(r["hash"][i])]
    for i in bad[:5]:
        print(f"[bench] pair {i} differs from the reference", file=sys.stderr)
    return {"value": cells / r["seconds"] / 1e9, "unit": "GCUPS", "cores": nthreads, "kind": "reference",
            "pairs_per_s": len(done_idx) / r["seconds"],
            "parity": {"pairs_checked": len(done_idx), "identical": not bad, "differing": len(bad),
                       "fields": "all ksw_extz_t fields + CIGAR vs the device-resident results"},
            "sample": f"{len(done_idx)} of {len(ps)} pairs in seeded random order within {budget:.0f} s, "
                      f"ksw_extd2_{ref.isa} compiled from the reference sources, {nthreads} threads"}


def plain_measurement(npairs: int, cpu: bool):
    """The plain single-pair workload: seeded 5 kb pairs (5% substitutions, 1% short indels,
    one 500 bp deletion), one ksw_extd2_gpu call per pair (host buffers in, malloc'd CIGAR
    out), per-call latency p50/p99; beside it the compiled reference's per-call latency
    (each call single-threaded, the calls spread over the host threads) on the same pairs,
    and every result compared."""
    import numpy as np

    from anchorwave_b200 import ksw2
    from anchorwave_b200 import workloads as W
    ps = W.plain_set(npairs, seed0=0)
    mat = ksw2.anchorwave_matrix(-4)
    ksw2.ksw_extd2(ps.queries[0], ps.targets[0], mat, 4, 2, 24, 1)
    lat, res = [], []
    for q, t in zip(ps.queries, ps.targets):
        t0 = time.perf_counter()
        res.append(ksw2.ksw_extd2(q, t, mat, 4, 2, 24, 1))
        lat.append(time.perf_counter() - t0)
    cells = ps.cells()
    out = {"workload": ps.name, "pairs": len(ps), "cells": cells, "pairs_per_s": len(ps) / sum(lat),
           "gcups": cells / sum(lat) / 1e9, "latency_ms_p50": 1e3 * float(np.percentile(lat, 50)),
           "latency_ms_p99": 1e3 * float(np.percentile(lat, 99))}
    if cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        try:
            ref = oracle.Reference()
        except FileNotFoundError as e:
            out["cpu_reference"] = {"unavailable": str(e)}
            return out
        r = ref.ksw_batch([q.tobytes() for q in ps.queries], [t.tobytes() for t in ps.targets], mat, 4, 2, 24, 1)
        ps_sec = r["pair_seconds"]
        same = all(oracle.result_hash(g) == int(h) for g, h in zip(res, r["hash"]))
        out["cpu_reference"] = {"latency_ms_p50": 1e3 * float(np.percentile(ps_sec, 50)),
                                "latency_ms_p99": 1e3 * float(np.percentile(ps_sec, 99)),
                                "threads": r["threads"], "isa": ref.isa, "results_identical": same,
                                "pairs_checked": len(ps)}
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference_arm(args)
    rank, world, local, pg = dist_init(args.gpus)
    if world > 1:
        # replicas on N GPUs: the line measures the headline step (and its e2e, plain per-call
        # sample, roofline and clocks) on every rank; the single-GPU sub-measurements and the
        # host-CPU reference legs belong to the 1-GPU line, so that no rank waits minutes at the
        # final barrier for another's extra work
        args.serve_requests = args.plain_pairs = args.wfa_pairs = args.wfa_long_pairs = 0
        args.no_long_banded = args.no_selector_summary = args.no_cpu_baseline = True
    import numpy as np

    from anchorwave_b200 import _lib, ksw2
    ps = workload(args, rank)
    mat = ksw2.anchorwave_matrix(-4)
    cells = ps.cells()
    n = len(ps)

    # the autotuner picks the strip kernel's warps per large pair and the large-pair threshold
    # on a seeded 1,024-pair sample of this workload, before anything is timed
    from anchorwave_b200 import autotune
    t_tune = time.perf_counter()
    (tuned_warps, tuned_thr), _ = autotune.tune(ps.queries, ps.targets, mat, 4, 2, 24, 1, sample=1024, reps=1)
    tuning = {"full_kernel": {"large_warps": tuned_warps, "large_tlen_threshold": tuned_thr,
                              "seconds": time.perf_counter() - t_tune, "sample_pairs": min(1024, n)}}
    plan = ksw2.KswPlan(ps.queries, ps.targets, mat, 4, 2, 24, 1)
    plan.upload()
    st = plan.stats()
    for _ in range(args.warmup):
        plan.execute()
    int_peak = _lib.lib.aw_int32_peak_ops()
    simd_peak = _lib.lib.aw_int16x2_peak_ops()
    sampler = ClockSampler(local)
    sampler.start()
    barrier(pg)
    step_ms, dp_ms, bt_ms = [], [], []
    for _ in range(args.steps):
        step_ms.append(plan.execute())
        d, b = plan.timing()
        dp_ms.append(d)
        bt_ms.append(b)
    barrier(pg)
    clocks = sampler.stop()
    res_dev = plan.download()
    total_ms = max_over_ranks(pg, float(sum(step_ms)))
    ms_per_step = total_ms / args.steps
    value = world * cells / (ms_per_step * 1e-3) / 1e9
    pairs_per_s = world * n / (ms_per_step * 1e-3)
    launches = plan.stats()["launches"]
    plan.close()

    # e2e through the public C-ABI call with host buffers (aw_ksw_extd2_batch): every step
    # stages the sequences into pinned memory, copies them H2D, runs the kernels, copies the
    # results and CIGARs D2H and hands back malloc'd ksw_extz_t CIGARs
    call = ksw2.BatchCall(ps.queries, ps.targets, mat, 4, 2, 24, 1)
    call.run()
    call.release()
    barrier(pg)
    e2e_s = []
    for k in range(args.steps):
        t0 = time.perf_counter()
        call.run()
        e2e_s.append(time.perf_counter() - t0)
        if k + 1 < args.steps:
            call.release()
    barrier(pg)
    e2e_step = max_over_ranks(pg, float(np.mean(e2e_s)))
    cig_words = call.cigar_words()
    res_e2e = call.results()
    diffs = [i for i, (a, b) in enumerate(zip(res_dev, res_e2e)) if a.key() != b.key()]
    identical = not diffs
    for i in diffs[:5]:
        print(f"[bench] pair {i} (qlen {len(ps.queries[i])}, tlen {len(ps.targets[i])}) differs: device-resident "
              f"{res_dev[i].key()[:12]} / e2e {res_e2e[i].key()[:12]}", file=sys.stderr)
    h2d = int(sum(len(q) for q in ps.queries) + sum(len(t) for t in ps.targets) + n * 48 + n * 4)
    d2h = int(n * 48 + cig_words * 4)

    # plain per-call GPU form on a sample of the same workload
    rng = np.random.default_rng(777)
    sample = rng.choice(n, size=min(args.plain_sample, n), replace=False)
    ksw2.ksw_extd2(ps.queries[sample[0]], ps.targets[sample[0]], mat, 4, 2, 24, 1)
    lat, pc_cells, pc_same = [], 0, True
    for i in sample:
        t0 = time.perf_counter()
        r1 = ksw2.ksw_extd2(ps.queries[i], ps.targets[i], mat, 4, 2, 24, 1)
        lat.append(time.perf_counter() - t0)
        pc_same &= r1.key() == res_dev[i].key()
        pc_cells += len(ps.queries[i]) * len(ps.targets[i])
    plain = {"gcups": pc_cells / sum(lat) / 1e9, "pairs_per_s": len(lat) / sum(lat),
             "latency_ms_p50": 1e3 * float(np.percentile(lat, 50)),
             "latency_ms_p99": 1e3 * float(np.percentile(lat, 99)), "sample_pairs": len(lat),
             "results_identical_to_batched": pc_same}
    cpu_on = rank == 0 and not args.no_cpu_baseline
    plain5 = plain_measurement(args.plain_pairs, cpu_on) if args.plain_pairs > 0 else None

    # the batch calls above keep ~100 GB of traceback arena pooled on this thread; give it
    # back before the other workloads size their own device pools
    ksw2.release_thread_buffers()
    serving = serving_measurement(args.serve_requests, rank, tuning) if args.serve_requests > 0 else None
    long_banded = None if args.no_long_banded else long_banded_measurement(
        rank, cpu_on, args.long_banded_pairs, args.long_banded_min, args.long_banded_max, args.long_banded_indel,
        args.long_banded_budget_gb,
        tuning)
    wfa_res = (wfa_measurement(args.wfa_pairs, rank, cpu_on, args.wfa_pool_gb) if args.wfa_pairs > 0 else None)
    wfa_long = wfa_long_measurement(args.wfa_long_pairs, rank, cpu_on) if args.wfa_long_pairs > 0 else None
    summary_res = (None if args.no_selector_summary else selector_summary_measurement(ps, rank, cpu_on))

    if rank != 0:
        barrier(pg)
        pg.destroy_process_group()
        return 0

    hbm_peak, hbm_kind = load_peaks()
    dp_mean = float(np.mean(dp_ms))
    achieved_ops = cells * OPS_PER_CELL_CIGAR / (dp_mean * 1e-3)
    tb_gbs = st["tb_bytes"] / (dp_mean * 1e-3) / 1e9
    batched_vs_plain = pairs_per_s / world / plain["pairs_per_s"]
    line = {
        "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int8",
        "data": "synthetic (seeded; stands in for B73/Mo17 intervals)",
        "pairs_per_s": pairs_per_s,
        "config": run_config(ps, world),
        "plan": {"waves": st["waves"], "traceback_bytes": st["tb_bytes"]},
        "tuning": tuning,
        "latency_ms": {"batch_step_p50": float(np.percentile(step_ms, 50)),
                       "batch_step_p99": float(np.percentile(step_ms, 99)),
                       "serving_p50": serving["latency_ms_p50"] if serving else None,
                       "serving_p99": serving["latency_ms_p99"] if serving else None,
                       "plain_per_call_p50": plain["latency_ms_p50"], "plain_per_call_p99": plain["latency_ms_p99"]},
        "plain_per_call": plain,
        "plain_5kb": plain5,
        "batched_vs_plain_pairs_per_s": batched_vs_plain,
        "phase_ms": {"dp": dp_mean, "traceback": float(np.mean(bt_ms))},
        "roofline": {"bound": "int16x2", "achieved": achieved_ops / 1e12, "peak": simd_peak / 1e12, "unit": "TOPS",
                     "frac": achieved_ops / simd_peak if simd_peak else None,
                     # DRAM bytes of one DP phase: the bytes per DP cell of an ncu capture of
                     # the strip kernel (dram__bytes_read + write, 1.643 GB for 1.64e9 cells
                     # of a 48-pair case, CIGAR mode) scaled by this step's DP cells; the
                     # algorithmic bytes are the 1-byte-per-cell traceback (tb_bytes)
                     "traffic": NCU_DRAM_BYTES_PER_CELL * cells, "traffic_unit": "bytes per DP phase",
                     "traffic_source": "estimate: bytes per DP cell of the CIGAR-mode ncu capture in "
                                       "profiles/ksw_full_kernel_batched_full.md x this step's cells",
                     "algorithmic_bytes": st["tb_bytes"],
                     "peak_source": "aw_int16x2_peak_ops() live microbenchmark (chains of FMA-pipe adds and "
                                    "ALU-pipe SIMD max/min on two 16-bit fields per register, "
                                    "2 field-ops per instruction)",
                     "int32_peak": int_peak / 1e12,
                     "ops_per_cell": OPS_PER_CELL_CIGAR,
                     "hbm_store": {"achieved": tb_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": tb_gbs / hbm_peak,
                                   "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({hbm_kind})"}},
        "e2e": {"value": world * cells / e2e_step / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "pairs_per_s": world * n / e2e_step,
                "results_identical_to_device_path": identical},
        "serving": serving,
        "long_banded": long_banded,
        "wfa": wfa_res,
        "wfa_long_intervals": wfa_long,
        "selector_summary": summary_res,
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
    }
    if not args.no_cpu_baseline:
        try:
            line["cpu_baseline"] = cpu_baseline(ps, args.cpu_budget, res_dev)
        except FileNotFoundError as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    if world > 1:
        line["sub_measurements"] = "on the 1-GPU line (replicas measure the headline step)"
    line["summary"] = compact_summary(line)
    print(json.dumps(line))
    barrier(pg)
    if pg is not None:
        pg.destroy_process_group()
    return 0


def compact_summary(line):
    """The sub-measurements in a few hundred characters, last on the line."""
    def get(d, *ks):
        for k in ks:
            if not isinstance(d, dict):
                return None
            d = d.get(k)
        return d
    out = {"batched_vs_plain_pairs_per_s": line["batched_vs_plain_pairs_per_s"],
           "batched_pairs_per_s": line["pairs_per_s"],
           "plain_mixed": {k: line["plain_per_call"][k] for k in ("pairs_per_s", "latency_ms_p50", "latency_ms_p99",
                                                                 "sample_pairs")}}
    p5 = line.get("plain_5kb")
    if p5:
        out["plain_5kb"] = {"pairs": p5["pairs"], "p50_ms": p5["latency_ms_p50"], "p99_ms": p5["latency_ms_p99"],
                            "ref_p50_ms": get(p5, "cpu_reference", "latency_ms_p50"),
                            "ref_p99_ms": get(p5, "cpu_reference", "latency_ms_p99"),
                            "identical": get(p5, "cpu_reference", "results_identical")}
    par = {"batched_full": get(line, "cpu_baseline", "parity")}
    if par["batched_full"]:
        par["batched_full"] = {k: par["batched_full"][k] for k in ("pairs_checked", "identical")}
    sv = line.get("serving")
    if sv:
        out["serving"] = {k: sv.get(k) for k in ("requests", "saturated_requests_per_s", "requests_per_s",
                                                 "latency_ms_p50", "latency_ms_p99", "load", "routing")}
        if sv.get("plain_per_call"):
            out["serving"]["served_vs_plain"] = sv["plain_per_call"]["served_vs_plain"]
            par["serving_vs_plain"] = sv["plain_per_call"]["results_identical_to_served"]
    lb = line.get("long_banded")
    if lb:
        out["long_banded"] = {"pairs": lb["pairs"], "band_cells": lb["band_cells"]}
        for nm in ("banded", "singletrack"):
            if nm in lb:
                x = lb[nm]
                out["long_banded"][nm] = {"gcups": x.get("gcups"), "s": x["ms"] / 1e3, "run": x["pairs_run"],
                                          "unreachable": x["band_unreachable"],
                                          "refused": x["refused_over_budget"],
                                          "valid": x["cigars_spanning_both"],
                                          "vs_ref": x.get("vs_cpu_reference")}
                par[f"long_{nm}"] = {"pairs_checked": get(x, "cpu_reference", "pairs"),
                                     "identical": get(x, "cpu_reference", "results_identical")}
    wf = line.get("wfa")
    if wf:
        out["wfa"] = {}
        for nm in ("standard", "singletrack", "medium"):
            if nm in wf:
                out["wfa"][nm] = {"pairs_per_s": wf[nm]["pairs_per_s"], "vs_ref": wf[nm].get("vs_cpu_reference")}
                par[f"wfa_{nm}"] = {"pairs_checked": get(wf, nm, "cpu_reference", "pairs"),
                                    "identical": get(wf, nm, "cpu_reference", "status_score_cigar_identical")}
    wl = line.get("wfa_long_intervals")
    if wl:
        out["wfa_long"] = [{"kb": r["length"] // 1000, "ms": r["device_ms"], "vs_ref": r.get("vs_cpu_reference")}
                           for r in wl]
        par["wfa_long"] = all(get(r, "cpu_reference", "identical") for r in wl) if all(
            "cpu_reference" in r for r in wl) else None
    ss = line.get("selector_summary")
    if ss:
        out["selector_pass"] = {"bases_per_s": ss.get("e2e_bases_per_s"), "vs_ref": ss.get("vs_cpu_reference")}
        par["selector_pass"] = get(ss, "cpu_reference", "summaries_identical")
    tn = line.get("tuning") or {}
    out["tuning"] = {"full": [get(tn, "full_kernel", "large_warps"), get(tn, "full_kernel", "large_tlen_threshold")],
                     "band_columns": get(tn, "band_kernel", "columns_per_lane"),
                     "serve": [get(tn, "serving", "slots"), get(tn, "serving", "max_batch")]}
    out["parity"] = par
    return sig(out)


if __name__ == "__main__":
    sys.exit(main())
