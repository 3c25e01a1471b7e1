#!/usr/bin/env python
"""Benchmark: beam-search QPS at recall@10 >= 0.95 on one B200 (per GPU replica).

Workload (the plain float32 path at scale): 1,000,000 base + 10,000 query
vectors, 96-d float32, 256-component Gaussian mixture (centres N(0,1),
per-dimension sigma 0.3), every vector L2-normalised, seed 1 (synthetic,
seeded; stands in for the public datasets). Vamana graph built on the GPU
with R=64, L=128, alpha=1.2, two passes, prefix-doubling batches. Beam search
k=10 from start point 0 with degree_limit=R, limit=n, batch_factor=0.125, at
the smallest beam in the reference's sweep list (check_nn_recall.h:214-216)
whose recall@10 against FP64 brute force is >= 0.95.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one batched beam search over the 10,000 queries. `value` is
device-timed (CUDA events on the launching stream, inputs resident in HBM,
L2 flushed between steps); `e2e` is the same metric through the host-buffer
C-ABI call (pinned host queries in, ids/distances/counters out, copies inside
the timed region). `--impl reference` times the reference's own qsearchAll
(compiled in place, oracle/_ref) on the host cores. Under torchrun every rank
runs an independent replica (no data-path collective); the timed region is
bracketed by barriers and the max over ranks is reported.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BEAMS = [10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 22, 24, 26, 28, 30, 32, 34, 36, 38, 40, 45, 50, 55, 60, 65,
         70, 80, 90, 100, 120, 140, 160, 180, 200]
METRIC = "QPS at recall@10>=0.95 (beam search, 1M x 96-d f32, 10K queries)"
W = dict(n=1_000_000, nq=10_000, d=96, comps=256, seed=1, sigma=0.3, R=64, Lb=128, alpha=1.2, passes=2, k=10,
         bf=0.125)


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


CONFIG = {
    "workload": "plain beam search, 1M x 96-d f32, 10K queries, Vamana R=64 L=128 alpha=1.2 2 passes",
    "n": W["n"], "nq": W["nq"], "d": W["d"], "k": W["k"], "data_seed": W["seed"], "components": W["comps"],
    "graph": "Vamana R=64 L=128 alpha=1.2, two passes, prefix-doubling batches, insertion order "
             "splitmix64(0x5EED5EED5EED + i), start point 0",
    "beam_rule": "smallest beam of the reference's sweep list (check_nn_recall.h:214-216) with recall@10 >= 0.95 "
                 "(checkRecall's ties) against exact FP64 groundtruth",
    "degree_limit": W["R"], "limit": W["n"], "batch_factor": W["bf"],
    "cache_flush": "between timed steps: a 256 MB device write (> L2) on the GPU; the reference's 5M-element "
                   "permutation (check_nn_recall.h:45) on the host",
}


def make_data(gen):
    """The benchmark's base and query vectors from a seeded generator: the product's
    pann_synth_mixture, or the same function in the in-place reference library."""
    base = gen(2, W["n"], W["d"], W["comps"], W["seed"], 0, sigma=W["sigma"], normalize=True)
    q = gen(2, W["nq"], W["d"], W["comps"], W["seed"], 1, sigma=W["sigma"], normalize=True)
    return base, q


def graph_digest(g) -> str:
    """sha1 of the graph's degrees and live neighbour lists (graph.h:138-145 rows, the slots past
    each degree zeroed: the two implementations pad them differently)."""
    import hashlib

    g = np.array(g, dtype=np.uint32, copy=True)
    live = np.arange(g.shape[1] - 1)[None, :] < g[:, :1]
    g[:, 1:][~live] = 0
    return hashlib.sha1(g.tobytes()).hexdigest()


class ClockSampler:
    """SM clock and throttle reasons sampled every 5 ms by a thread (NVML)
    while the timed region runs; no samples (and no `clocks` key) when NVML
    is unavailable."""

    HW_SLOWDOWN, SW_POWER_CAP, HW_THERMAL, SW_THERMAL = 0x8, 0x4, 0x40, 0x20

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []
        self.max_mhz = None
        self._stop = None
        self._thread = None

    def __enter__(self):
        import threading

        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self._stop = threading.Event()

            def poll():
                while not self._stop.is_set():
                    try:
                        mhz = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                        reasons = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((float(mhz), int(reasons)))
                    except Exception:
                        pass
                    self._stop.wait(0.005)

            self._thread = threading.Thread(target=poll, daemon=True)
            self._thread.start()
        except Exception:
            self._thread = None
        return self

    def __exit__(self, *a):
        if self._thread:
            self._stop.set()
            self._thread.join(timeout=2)

    def summary(self):
        if not self.samples:
            return None
        names = {self.HW_SLOWDOWN: "hw_slowdown", self.HW_THERMAL: "hw_thermal_slowdown",
                 self.SW_THERMAL: "sw_thermal_slowdown", self.SW_POWER_CAP: "sw_power_cap"}
        reasons = sorted({n for _, r in self.samples for bit, n in names.items() if r & bit})
        return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "nvml, 5 ms"}


def measured_peak():
    try:
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(mp["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per query of the search kernel from the committed ncu summary (profiles/)."""
    try:
        s = json.load(open(os.path.join(ROOT, "profiles", "search_f32_c1.json")))
        return float(s["dram_bytes_per_query"]), s
    except Exception:
        return None, None


def build_roofline(st, avg_deg, peak, peak_kind):
    """The GPU build against the HBM roofline. Algorithmic bytes: per insertion search the rows
    of the nodes it visits (4 (1 + degree) bytes each, the degree taken as the final graph's mean),
    one point row per distance comparison and the inserted point's own row; one row per robustPrune
    candidate (insertions and re-prunes); the 4R-byte row written per inserted point; 8 bytes per
    reverse-edge pair (the sort of (neighbour, point) pairs)."""
    row = W["d"] * 4
    deg = min(float(W["R"]), avg_deg)
    b = (4.0 * st.visited_total * (1.0 + deg) + st.search_cmps * row + st.inserted * row +
         st.prune_candidates * row + 4.0 * W["R"] * st.inserted + 8.0 * st.edge_pairs)
    achieved = b / st.seconds / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} (hbm_gbs)",
            "algorithmic_bytes": round(b), "seconds_device": round(st.seconds, 3),
            "phase_seconds": {"search": round(st.search_seconds, 3), "prune": round(st.prune_seconds, 3),
                              "reverse": round(st.reverse_seconds, 3)},
            "counters": {"inserted": int(st.inserted), "visited": int(st.visited_total),
                         "search_cmps": int(st.search_cmps), "prune_candidates": int(st.prune_candidates),
                         "edge_pairs": int(st.edge_pairs), "reprunes": int(st.reprunes),
                         "batches": int(st.batches)}}


def max_over_ranks(seconds: float, device) -> float:
    """The slowest rank's time (all ranks take this collective in the same order)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return seconds
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_qps(queries_per_rank: int, steps: int, world: int, slowest_seconds: float) -> float:
    """Whole-job throughput: every rank searches its own replica's queries."""
    return world * queries_per_rank * steps / slowest_seconds


def profile_case(idx, q, beam, args):
    """--case tile:PREC:PARENTS:SCORER (PREC bf16|fp8, SCORER cuda|tc): the tile search alone over the
    1M workload, --warmup + --steps calls at the plain form's beam, for a profiler's launch selection
    (the kernel's own launches only; no JSON metric line)."""
    import parlayann_b200 as P

    kind, prec, parents, scorer = args.case.split(":")
    if kind != "tile":
        raise SystemExit(f"unknown --case {args.case}")
    pr = {"bf16": P.PREC_BF16, "fp8": P.PREC_FP8}[prec]
    sc = {"cuda": P.SCORER_CUDA, "tc": P.SCORER_TENSOR}[scorer]
    idx.set_precision(pr)
    secs = []
    for _ in range(args.warmup + args.steps):
        t = time.time()
        idx.search(q, W["k"], beam, precision=pr, parents=int(parents), scorer=sc)
        secs.append(round(time.time() - t, 5))
    idx.set_precision(P.PREC_F32)
    return {"case": args.case, "beam": beam, "host_seconds_per_call": secs}


def run_ours(args):
    import torch
    import torch.distributed as dist

    import parlayann_b200 as P

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    lib = P.lib()
    base, q = make_data(P.synth_mixture)
    idx = P.Index(base, W["R"])
    t0 = time.time()
    build_dev = None
    build_stats = None
    if args.load_graph:
        idx.load_graph(args.load_graph)
    else:
        bst = idx.build(W["Lb"], W["alpha"], num_passes=W["passes"], batch_factor=W["bf"])
        build_dev = round(bst.seconds, 3)
        build_stats = bst
        if args.save_graph:
            idx.save_graph(args.save_graph)
    build_wall = time.time() - t0
    g = idx.get_graph()
    avg_deg = float(g[:, 0].mean())
    gt, gd = idx.groundtruth(q, 20)
    k = W["k"]
    # smallest beam of the reference's sweep with recall@10 >= 0.95
    beam, recall, sweep, res = None, None, [], None
    for L in ([] if args.beam else BEAMS):
        r = idx.search(q, k, L, batch_factor=W["bf"])
        rec = P.recall_with_ties(r.ids, gt, k, q, base)
        sweep.append((L, round(rec, 4)))
        if rec >= 0.95:
            beam, recall, res = L, rec, r
            break
    if res is None:
        beam = args.beam or BEAMS[-1]
        res = idx.search(q, k, beam, batch_factor=W["bf"])
        recall = P.recall_with_ties(res.ids, gt, k, q, base)
    nq = q.shape[0]
    if args.case:
        return profile_case(idx, q, beam, args)
    mean_vis = float(res.visited.mean())
    mean_cmps = float(res.cmps.mean())
    row_bytes = W["d"] * 4
    bytes_per_query = 4.0 * mean_vis * (1.0 + avg_deg) + mean_cmps * row_bytes + row_bytes

    # device-resident timed loop
    qp = P.QueryParams(k, beam, W["n"], W["R"], W["bf"])
    starts = np.zeros(1, np.uint32)
    dq = torch.from_numpy(q).to(dev)
    d_ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
    d_dists = torch.empty((nq, k), dtype=torch.float32, device=dev)
    d_vis = torch.empty(nq, dtype=torch.int32, device=dev)
    d_cmps = torch.empty(nq, dtype=torch.int32, device=dev)
    d_flags = torch.empty(nq, dtype=torch.int32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # > L2 (126 MB)
    stream = torch.cuda.current_stream(dev)

    def step_device():
        rc = lib.pann_search_device(idx.handle, ctypes.c_void_p(dq.data_ptr()), nq, ctypes.byref(qp),
                                    starts.ctypes.data_as(ctypes.c_void_p), 1, ctypes.c_void_p(d_ids.data_ptr()),
                                    ctypes.c_void_p(d_dists.data_ptr()), ctypes.c_void_p(d_vis.data_ptr()),
                                    ctypes.c_void_p(d_cmps.data_ptr()), ctypes.c_void_p(d_flags.data_ptr()),
                                    ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise P.PannError(rc, lib.pann_last_error().decode())

    for _ in range(args.warmup):
        flush.fill_(1)
        step_device()
    torch.cuda.synchronize()
    assert np.array_equal(d_ids.cpu().numpy().astype(np.uint32), res.ids), "device path differs from host path"
    times = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)  # L2 flush outside the timed span
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step_device()
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1) / 1e3)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t_dev = max_over_ranks(sum(times), dev)
    qps = replica_qps(nq, args.steps, world, t_dev)

    # end-to-end through the host-buffer C-ABI call (pinned buffers, copies timed)
    hq = torch.from_numpy(q).pin_memory()
    h_ids = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    h_d = torch.empty((nq, k), dtype=torch.float32).pin_memory()
    h_v = torch.empty(nq, dtype=torch.int32).pin_memory()
    h_c = torch.empty(nq, dtype=torch.int32).pin_memory()
    h_f = torch.empty(nq, dtype=torch.int32).pin_memory()

    def step_e2e():
        rc = lib.pann_search(idx.handle, ctypes.c_void_p(hq.data_ptr()), nq, ctypes.byref(qp),
                             starts.ctypes.data_as(ctypes.c_void_p), 1, ctypes.c_void_p(h_ids.data_ptr()),
                             ctypes.c_void_p(h_d.data_ptr()), ctypes.c_void_p(h_v.data_ptr()),
                             ctypes.c_void_p(h_c.data_ptr()), ctypes.c_void_p(h_f.data_ptr()))
        if rc != 0:
            raise P.PannError(rc, lib.pann_last_error().decode())

    for _ in range(args.warmup):
        flush.fill_(1)
        torch.cuda.synchronize()
        step_e2e()
    e2e_times = []
    if world > 1:
        dist.barrier()
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t = time.perf_counter()
        step_e2e()
        e2e_times.append(time.perf_counter() - t)
    t_e2e = max_over_ranks(sum(e2e_times), dev)
    assert np.array_equal(h_ids.numpy().astype(np.uint32), res.ids), "e2e path differs"

    peak, peak_kind = measured_peak()
    per_launch_s = t_dev / args.steps
    achieved = bytes_per_query * nq / per_launch_s / 1e9
    traffic_pq, prof = profiled_traffic()
    build_roof = build_roofline(build_stats, avg_deg, peak, peak_kind) if build_stats is not None else None
    line = None
    forms = None
    if rank == 0 and not args.no_forms:
        forms = run_forms(idx, base, q, gt, gd, beam, qps, dev, flush, args)
    if rank == 0:
        cpu = cpu_baseline(base, q, g, beam, res, args) if not args.no_cpu_baseline else None
        line = {
            "metric": METRIC,
            "value": round(qps, 1),
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(1e3 * t_dev / args.steps, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded 256-component Gaussian mixture, L2-normalised)",
            "config": dict(CONFIG, parallelism=f"replicas x{world}"),
            "details": {"beam": beam, "recall_at_10": round(recall, 4), "recall_sweep": sweep,
                        "graph_sha1": graph_digest(g), "mean_degree": round(avg_deg, 3),
                        "build_seconds_device": build_dev, "build_seconds_wall": round(build_wall, 3),
                        "mean_visited": round(mean_vis, 2), "mean_cmps": round(mean_cmps, 2),
                        "flagged_queries": int(res.flags.sum()),
                        "groundtruth": "pann_groundtruth (GPU, FP64 distances, ties by id), 20 per query"},
            "e2e": {"value": round(replica_qps(nq, args.steps, world, t_e2e), 1), "unit": "queries/s",
                    "h2d_bytes_per_step": int(q.nbytes),
                    "d2h_bytes_per_step": int(nq * k * 8 + nq * 12)},
            # per step: the job-order distances, tier 0, the emulation pass beside it, tier 2, the
            # emulation pass after it, the global-table emulation (plus CUB's radix sort of the order)
            "gpu_launches": 6 * args.steps,
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_kind": f"{peak_kind} (hbm_gbs)",
                         "algorithmic_bytes_per_query": round(bytes_per_query, 1),
                         "traffic": (round(traffic_pq * nq / 1e9, 4) if traffic_pq else None),
                         "traffic_unit": "GB per launch (ncu dram read+write, scaled from profiles/)"},
            "cpu_baseline": cpu,
            "build_roofline": build_roof,
        }
        if forms is not None:
            line["forms"] = forms
        c = clk.summary()
        if c:
            line["clocks"] = c
    if world > 1:
        # every collective is behind us (the timed regions' barriers and maxima); rank 0's forms
        # and reference baseline need no other rank, so no rank waits for them
        dist.destroy_process_group()
    idx.close()
    return line


def _timed(step, flush, stream, steps, warmup):
    """Device seconds per step: CUDA events on `stream`, L2 flushed outside each timed span."""
    import torch

    for _ in range(warmup):
        flush.fill_(1)
        step()
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(steps):
        flush.fill_(1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        tot += e0.elapsed_time(e1) / 1e3
    return tot / steps


# (name, precision, parents, scorer): scorer 1 scores the tile search's staged rows on the tensor cores
PRECISION_FORMS = (("bf16", 1, 0, 0), ("fp8", 2, 0, 0), ("bf16_tile2", 1, 2, 0), ("fp8_tile2", 2, 2, 0),
                   ("fp8_tile3", 2, 3, 0), ("bf16_tile2_tc", 1, 2, 1), ("fp8_tile2_tc", 2, 2, 1),
                   ("fp8_tile3_tc", 2, 3, 1))


def scoring_error(idx, base, q, ids, prec, metric):
    """Error of the precision's scores (the ones its traversal ranks candidates by, before the
    exact re-rank) against FP64, on the pairs (query, id): absolute and relative, max and mean."""
    import parlayann_b200 as P

    sub = min(2000, q.shape[0])
    ids = np.ascontiguousarray(ids[:sub], dtype=np.uint32)
    lp = idx.score(q[:sub], ids, prec).astype(np.float64)
    rows = base[ids.ravel().astype(np.int64)].astype(np.float64).reshape(ids.shape + (base.shape[1],))
    q64 = q[:sub].astype(np.float64)[:, None, :]
    d64 = ((rows - q64) ** 2).sum(-1) if metric == P.L2 else -(rows * q64).sum(-1)
    ab = np.abs(lp - d64)
    rel = ab / np.maximum(np.abs(d64), 1e-30)
    return {"pairs": int(ids.size), "abs_max": float(ab.max()), "abs_mean": float(ab.mean()),
            "rel_max": float(rel.max()), "rel_mean": float(rel.mean())}


def precision_forms(idx, base, q, gt, metric, beam, qps_plain, dev, flush, stream, steps, forms=PRECISION_FORMS):
    """Each precision form at its smallest beam with recall@10 >= 0.95: device QPS through a batch
    object (CUDA-graph replay), the speed-up over the plain form, the recall loss at the plain
    form's beam, the error of the precision's own scores against FP64 (before the re-rank, on each
    query's 20 nearest points) and of the reported (re-ranked) distances."""
    import torch

    import parlayann_b200 as P

    lib = P.lib()
    k = W["k"]
    nq = q.shape[0]
    dq = torch.from_numpy(q).to(dev)
    exact_rec_at_beam = P.recall_with_ties(idx.search(q, k, beam).ids, gt, k, q, base, metric)
    out = {}
    for name, prec, parents, scorer in forms:
        idx.set_precision(prec)
        pbeam, prec_rec, pres = None, None, None
        for L in BEAMS:
            if L < beam - 10:
                continue
            r = idx.search(q, k, L, precision=prec, parents=parents, scorer=scorer)
            rec = P.recall_with_ties(r.ids, gt, k, q, base, metric)
            if rec >= 0.95:
                pbeam, prec_rec, pres = L, rec, r
                break
        if pbeam is None:
            continue
        same_beam = idx.search(q, k, beam, precision=prec, parents=parents, scorer=scorer)
        loss = exact_rec_at_beam - P.recall_with_ties(same_beam.ids, gt, k, q, base, metric)
        b = idx.batch(nq, k, pbeam, precision=prec, parents=parents, scorer=scorer)
        d_ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
        d_d = torch.empty((nq, k), dtype=torch.float32, device=dev)
        ks = np.full(nq, k, np.uint32)
        Ls = np.full(nq, pbeam, np.uint32)

        def step_b():
            rc = lib.pann_batch_run(b.handle, ctypes.c_void_p(dq.data_ptr()), nq, ks.ctypes.data_as(ctypes.c_void_p),
                                    Ls.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(d_ids.data_ptr()),
                                    ctypes.c_void_p(d_d.data_ptr()), None, None, None, 1,
                                    ctypes.c_void_p(stream.cuda_stream))
            if rc != 0:
                raise P.PannError(rc, lib.pann_last_error().decode())

        t = _timed(step_b, flush, stream, steps, 3)
        ids_b = d_ids.cpu().numpy().astype(np.uint32)
        assert np.array_equal(ids_b, pres.ids), "batched precision form differs from the plain precision form"
        exact_d = idx.score(q[:2000], pres.ids[:2000])
        rep_err = np.abs(pres.dists[:2000].astype(np.float64) - exact_d) / np.maximum(np.abs(exact_d), 1e-30)
        out[name] = {"beam": pbeam, "parents": parents, "scorer": "tensor cores (tcgen05)" if scorer else "CUDA cores",
                     "recall_at_10": round(prec_rec, 4),
                     "stopped_early": int(((pres.flags & 2) != 0).sum()), "qps_batched_graph": round(nq / t, 1),
                     "speedup_vs_plain": round(nq / t / qps_plain, 3),
                     "recall_loss_at_plain_beam": round(loss, 4),
                     "scoring_error_vs_fp64": scoring_error(idx, base, q, gt[:, :20], prec, metric),
                     "reported_distances_equal_exact_f32": bool(rep_err.max() == 0.0)}
        b.close()
    idx.set_precision(P.PREC_F32)
    return out


def plain_qps(idx, q, beam, dev, flush, stream, steps):
    """Device-timed QPS of the plain (exact) search through pann_search_device."""
    import torch

    import parlayann_b200 as P

    lib = P.lib()
    k = W["k"]
    nq = q.shape[0]
    qp = P.QueryParams(k, beam, idx.n, idx.R, W["bf"])
    starts = np.zeros(1, np.uint32)
    dq = torch.from_numpy(q).to(dev)
    d_ids = torch.empty((nq, k), dtype=torch.int32, device=dev)

    def step():
        rc = lib.pann_search_device(idx.handle, ctypes.c_void_p(dq.data_ptr()), nq, ctypes.byref(qp),
                                    starts.ctypes.data_as(ctypes.c_void_p), 1, ctypes.c_void_p(d_ids.data_ptr()),
                                    None, None, None, None, ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise P.PannError(rc, lib.pann_last_error().decode())

    return nq / _timed(step, flush, stream, steps, 3)


SP_BEAMS = BEAMS + [225, 250, 275, 300, 375, 500, 750, 1000]
SP_LIMITS = [10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26, 28, 30, 35]
SP_BUCKETS = [.1, .2, .3, .4, .5, .6, .7, .75, .8, .85, .9, .93, .95, .97, .98, .99, .995, .999, .9995, .9999, .99995,
              .99999]


def search_and_parse(idx, base, q, gt, dev, flush, stream):
    """The reference's search_and_parse sweep (check_nn_recall.h:184-265) on the GPU: recall@10 and
    device-timed QPS for every beam of its list, for the visit limits 10..35 (beam max(limit, k),
    degree limit min(R, 5 limit)) and for the "best accuracy" point (k = 100, beam 1000, recall of
    the first 10); then, per recall bucket, the fastest configuration whose recall lies in
    [bucket, next bucket] (parse_results.h:189-214)."""
    import torch

    import parlayann_b200 as P

    lib = P.lib()
    k = W["k"]
    nq = q.shape[0]
    starts = np.zeros(1, np.uint32)
    dq = torch.from_numpy(q).to(dev)
    d_ids = torch.empty((nq, 100), dtype=torch.int32, device=dev)
    d_vis = torch.empty(nq, dtype=torch.int32, device=dev)
    d_cmps = torch.empty(nq, dtype=torch.int32, device=dev)

    def check(kk, L, limit, dl):
        qp = P.QueryParams(kk, L, limit, dl, W["bf"])

        def step():
            rc = lib.pann_search_device(idx.handle, ctypes.c_void_p(dq.data_ptr()), nq, ctypes.byref(qp),
                                        starts.ctypes.data_as(ctypes.c_void_p), 1, ctypes.c_void_p(d_ids.data_ptr()),
                                        None, ctypes.c_void_p(d_vis.data_ptr()), ctypes.c_void_p(d_cmps.data_ptr()),
                                        None, ctypes.c_void_p(stream.cuda_stream))
            if rc != 0:
                raise P.PannError(rc, lib.pann_last_error().decode())

        t = _timed(step, flush, stream, 2, 1)
        ids = d_ids.view(-1)[:nq * kk].cpu().numpy().astype(np.uint32).reshape(nq, kk)  # rows of kk ids
        vis = d_vis.cpu().numpy()
        cm = d_cmps.cpu().numpy()
        return {"k": kk, "beam": L, "limit": limit, "degree_limit": dl,
                "recall": round(P.recall_with_ties(ids, gt, k, q, base), 4), "qps": round(nq / t, 1),
                "mean_cmps": round(float(cm.mean()), 1), "mean_visited": round(float(vis.mean()), 2)}

    res = [check(k, L, idx.n, idx.R) for L in SP_BEAMS if L >= k]
    res += [check(k, max(l, k), l, min(idx.R, 5 * l)) for l in SP_LIMITS]
    res.append(check(100, 1000, idx.n, idx.R))
    table = []
    for i, b in enumerate(SP_BUCKETS):
        cands = [r for r in res if r["recall"] >= b]
        if i < len(SP_BUCKETS) - 1 and cands:
            cands = [r for r in cands if r["recall"] <= SP_BUCKETS[i + 1]]
        if cands:
            m = max(cands, key=lambda r: r["qps"])
            table.append({"bucket": b, **m})
    return {"runs": res, "buckets": table}


def run_c2(dev, flush, args, want):
    """The precision form at 10M: 10,000,000 base + 10,000 query vectors, 96-d float32, the same
    generator with 1,024 components, Vamana R=64 L=128 alpha=1.2 two passes built on the GPU with
    the Euclidean distance; searched as a Euclidean index and as a mips index (on L2-normalised
    vectors -q.b orders points as |q - b|^2 does, so the one graph serves both). Per metric: the
    plain form's smallest beam with recall@10 >= 0.95 and its QPS, each precision form next to it."""
    import torch

    import parlayann_b200 as P

    n, nq, d = 10_000_000, 10_000, 96
    t0 = time.time()
    base = P.synth_mixture(P.F32, n, d, 1024, W["seed"], 0, sigma=W["sigma"], normalize=True)
    q = P.synth_mixture(P.F32, nq, d, 1024, W["seed"], 1, sigma=W["sigma"], normalize=True)
    gen_s = time.time() - t0
    stream = torch.cuda.current_stream(dev)
    steps = max(3, min(args.steps, 10))
    idx = P.Index(base, W["R"])
    bst = idx.build(W["Lb"], W["alpha"], num_passes=W["passes"], batch_factor=W["bf"])
    g = idx.get_graph()
    out = {"workload": "10M x 96-d f32 (1024-component mixture, L2-normalised, seed 1), 10K queries, Vamana R=64 "
                       "L=128 alpha=1.2 two passes (GPU build, Euclidean)",
           "build_seconds_device": round(bst.seconds, 3), "mean_degree": round(float(g[:, 0].mean()), 3),
           "generate_seconds_host": round(gen_s, 2)}
    for mname, metric in (("l2", P.L2), ("mips", P.MIPS)):
        if metric == P.L2:
            ix = idx
        else:
            ix = P.Index(base, W["R"], P.MIPS)
            ix.set_graph(g)
        t0 = time.time()
        gt, _ = ix.groundtruth(q, 20)
        gt_s = time.time() - t0
        beam, rec = None, None
        for L in BEAMS:
            r = ix.search(q, W["k"], L, batch_factor=W["bf"])
            rec = P.recall_with_ties(r.ids, gt, W["k"], q, base, metric)
            if rec >= 0.95:
                beam = L
                break
        if beam is None:
            out[mname] = {"failed": "no beam of the sweep reached recall 0.95"}
            continue
        qps = plain_qps(ix, q, beam, dev, flush, stream, steps)
        out[mname] = {"groundtruth_seconds": round(gt_s, 3),
                      "plain": {"beam": beam, "recall_at_10": round(rec, 4), "qps": round(qps, 1)},
                      "precision": precision_forms(ix, base, q, gt, metric, beam, qps, dev, flush, stream, steps)}
        best = max(out[mname]["precision"].values(), key=lambda v: v["qps_batched_graph"], default=None)
        if best:
            out[mname]["best_speedup_vs_plain"] = best["speedup_vs_plain"]
        if metric == P.L2 and "serving" in want:
            out["serving"] = run_serving(ix, q, nq, beam, range_radius(base, q), out[mname]["precision"])
        if ix is not idx:
            ix.close()
    idx.close()
    return out


def run_c3(dev, flush, args):
    """The batched form on a large uint8 index: n base vectors (100,000,000 in the full configuration;
    --c3-n) x 128-d uint8 from the small configuration's generator with 1,024 components, seed 0,
    Vamana R=64 L=128 alpha=1.2 two passes built on the GPU; 100,000 queries with per-query k uniform
    in {1,10,100} and beam uniform in [k, 4k] in one autotuned batch, against one plain launch at the
    largest k and beam; recall@k per k class on the first 1,000 queries against exact (integer)
    groundtruth."""
    import torch

    import parlayann_b200 as P

    n, nq, d = args.c3_n, 100_000, 128
    t0 = time.time()
    base = P.synth_mixture(P.U8, n, d, 1024, 0, 0)
    q = P.synth_mixture(P.U8, nq, d, 1024, 0, 1)
    gen_s = time.time() - t0
    stream = torch.cuda.current_stream(dev)
    idx = P.Index(base, W["R"])
    print(f"c3: generated {n:,} x {d} uint8 in {gen_s:.1f} s; building", file=sys.stderr, flush=True)
    bst = idx.build(W["Lb"], W["alpha"], num_passes=W["passes"], batch_factor=W["bf"])
    print(f"c3: built in {bst.seconds:.1f} s (device)", file=sys.stderr, flush=True)
    dq = torch.from_numpy(q).to(dev)
    out = {"workload": f"{n:,} x 128-d uint8 (1024-component mixture, seed 0), {nq:,} queries, Vamana R=64 L=128 "
                       "alpha=1.2 two passes (GPU build)",
           "n": n, "build_seconds_device": round(bst.seconds, 2), "generate_seconds_host": round(gen_s, 2),
           "resident_bytes": int(n) * (128 + 4 * W["R"])}
    out.update(run_batched_uneven(idx, q, dq, dev, flush, stream, max(3, min(args.steps, 5)), P.lib()))
    sub = 1000
    gt, _ = idx.groundtruth(q[:sub], 100)
    rng = np.random.default_rng(5)
    ks = rng.choice(np.array([1, 10, 100], np.uint32), nq).astype(np.uint32)[:sub]
    Ls = np.array([rng.integers(max(kk, 1), 4 * kk + 1) for kk in ks], np.uint32)
    rec = {}
    for kk in (1, 10, 100):
        sel = np.where(ks == kk)[0]
        hits = 0
        for i in sel:
            r = idx.search(q[i:i + 1], int(kk), int(Ls[i]))
            hits += len(set(r.ids[0].tolist()) & set(gt[i, :kk].tolist()))
        rec[f"recall_at_{kk}"] = round(hits / float(kk * len(sel)), 4) if len(sel) else None
    out["recall_sample"] = {"queries": sub, **rec, "note": "each query at its own k and beam, ids against exact "
                                                              "integer groundtruth"}
    idx.close()
    return out


def run_forms(idx, base, q, gt, gd, beam, qps_plain, dev, flush, args):
    """The precision, batched and serving forms and range search on the same
    index, each next to the plain form: QPS at recall@10 >= 0.95 (device
    timed), recall loss and distance error against FP64 brute force, p50/p99
    latency under open-loop load."""
    import torch

    import parlayann_b200 as P

    lib = P.lib()
    k = W["k"]
    nq = q.shape[0]
    stream = torch.cuda.current_stream(dev)
    starts = np.zeros(1, np.uint32)
    dq = torch.from_numpy(q).to(dev)
    out = {}
    steps = max(3, min(args.steps, 10))

    want = set(args.forms.split(","))
    # ---- precision form (+ batched): smallest beam with recall >= 0.95, device QPS through a batch object
    prec_out = {}
    if "precision" in want or "serving" in want:
        prec_out = precision_forms(idx, base, q, gt, P.L2, beam, qps_plain, dev, flush, stream, steps)
    idx.set_precision(P.PREC_F32)
    if "precision" in want:
        # the reference's own mixed precision: search over one-byte scalar-quantized points, float re-rank of
        # min(k * 100, beam) frontier entries (beam_search_rerank), bit-exact with the reference's code
        idx.set_quantized()
        qbeam, qrec = None, None
        for L in BEAMS:
            if L < beam - 10:
                continue
            rec = P.recall_with_ties(idx.search_quantized(q, k, L).ids, gt, k, q, base)
            if rec >= 0.95:
                qbeam, qrec = L, rec
                break
        if qbeam is not None:
            rq = idx.search_quantized(q, k, qbeam)
            t0 = time.perf_counter()
            for _ in range(3):
                idx.search_quantized(q, k, qbeam)
            t_q = (time.perf_counter() - t0) / 3
            qent = {"beam": qbeam, "rerank_factor": 100, "recall_at_10": round(qrec, 4), "qps_e2e": round(nq / t_q, 1),
                    "slope_offset": list(idx.quant_params())}
            try:
                from oracle import oracle as O

                if O.have_ref() and not args.no_cpu_baseline:
                    ro = O.search_quantized("ref", base, q, idx.get_graph(), k, qbeam)
                    qent["cpu_reference"] = {"qps": round(nq / ro["seconds"], 1),
                                             "cores": int(O.rlib().ref_num_workers()),
                                             "code": "beam_search_rerank over Euclidian_Point<uint8_t>",
                                             "answers_identical": bool(np.array_equal(ro["ids"], rq.ids) and
                                                                       np.array_equal(ro["visited"], rq.visited))}
            except Exception as ex:  # noqa: BLE001
                qent["cpu_reference"] = {"failed": str(ex)}
            out["quantized_rerank"] = qent
    if prec_out:
        out["precision_batched"] = prec_out
    if "batched" in want:
        out["batched_uneven"] = run_batched_uneven(idx, q, dq, dev, flush, stream, steps, lib)
    radius = range_radius(base, q)
    if "range" in want:
        nr = 200
        idx.range_search(q[:nr], 20, radius, P.RANGE_GREEDY)  # warm-up: the expansion tables are allocated
        t0 = time.perf_counter()
        rr = idx.range_search(q[:nr], 20, radius, P.RANGE_GREEDY)
        t_r = time.perf_counter() - t0
        sizes = np.array([len(x) for x in rr["ids"]])
        out["range"] = {"queries": nr, "beam": 20, "type": "greedy", "radius_quantile": 0.01, "radius": radius,
                        "qps_e2e": round(nr / t_r, 1), "mean_answer": float(sizes.mean()),
                        "answer_p50_p99_max": [int(np.percentile(sizes, 50)), int(np.percentile(sizes, 99)),
                                               int(sizes.max())],
                        "answer_ids_per_s": round(float(sizes.sum()) / t_r, 1)}
        # the reference's RangeSearch (compiled in place) on the host cores, same graph and queries
        try:
            from oracle import oracle as O

            if O.have_ref() and not args.no_cpu_baseline:
                g = idx.get_graph()
                nc = 40
                t0 = time.perf_counter()
                ro = O.range_search("ref", base, q[:nc], g, 20, radius, O.RANGE_GREEDY, cap=int(sizes.max() * 4) + 64)
                t_c = time.perf_counter() - t0
                same = all(np.array_equal(a, b) for a, b in zip(ro["ids"], rr["ids"][:nc]))
                out["range"]["cpu_reference"] = {"queries": nc, "qps": round(nc / t_c, 1),
                                                 "cores": int(O.rlib().ref_num_workers()),
                                                 "answers_identical": bool(same)}
        except Exception as ex:  # noqa: BLE001
            out["range"]["cpu_reference"] = {"failed": str(ex)}
        # exact range groundtruth (full scan) and the range recall of check_range_recall.h:44-54
        idx.range_groundtruth(q[:nr], radius)   # warm-up: buffers sized
        t0 = time.perf_counter()
        gt_offs, gt_ids = idx.range_groundtruth(q[:nr], radius)
        t_g = time.perf_counter() - t0
        actual = np.diff(gt_offs).astype(np.float64)
        nz = actual > 0
        rgt = {"queries": nr, "seconds": round(t_g, 4), "qps_e2e": round(nr / t_g, 1),
              "recall_point": round(float(np.mean(sizes[nz] / actual[nz])), 4) if nz.any() else None,
              "recall_cumulative": round(float(sizes.sum() / actual.sum()), 4) if actual.sum() else None}
        try:
            from oracle import oracle as O

            if O.have_ref() and not args.no_cpu_baseline:
                nc = 16
                t0 = time.perf_counter()
                ro, ri = O.range_groundtruth("ref", base, q[:nc], radius)
                t_c = time.perf_counter() - t0
                rgt["cpu_reference"] = {"queries": nc, "qps": round(nc / t_c, 2), "tool": "compute_range_groundtruth",
                                       "answers_identical": bool(np.array_equal(ri, gt_ids[: int(gt_offs[nc])]))}
        except Exception as ex:  # noqa: BLE001
            rgt["cpu_reference"] = {"failed": str(ex)}
        out["range"]["groundtruth"] = rgt
    if "serving" in want and "c2" not in want:
        out["serving"] = run_serving(idx, q, nq, beam, radius, prec_out)
    if "sweep" in want:
        out["search_and_parse"] = search_and_parse(idx, base, q, gt, dev, flush, stream)
    if "c2" in want:
        out["precision_10m"] = run_c2(dev, flush, args, want)
    if "c3" in want:
        out["batched_large_u8"] = run_c3(dev, flush, args)
    return out


def range_radius(base, q):
    """The 1%-quantile of sampled base-query distances (squared L2)."""
    samp = []
    rs = np.random.default_rng(6)
    for i in rs.choice(q.shape[0], 16, replace=False):
        cols = rs.choice(base.shape[0], 4000, replace=False)
        samp.append(((base[cols] - q[i]) ** 2).sum(1))
    return float(np.quantile(np.concatenate(samp), 0.01))


def run_batched_uneven(idx, q, dq, dev, flush, stream, steps, lib, n_index=None):
    """Per-query k in {1,10,100} and beam in [k, 4k] through one batch object
    (autotuned mapping, graph replay), against the plain form in one launch at
    the largest k and beam (what a caller without per-query parameters runs);
    the batch's answers are checked against the plain form run per (k, beam)
    group (untimed)."""
    import torch

    import parlayann_b200 as P

    nq = q.shape[0]
    n_index = n_index or idx.n
    starts = np.zeros(1, np.uint32)
    rng = np.random.default_rng(5)
    ks = rng.choice(np.array([1, 10, 100], np.uint32), nq).astype(np.uint32)
    Ls = np.array([rng.integers(max(kk, 1), 4 * kk + 1) for kk in ks], np.uint32)
    kmax, Lmax = 100, int(Ls.max())
    b = idx.batch(nq, kmax, Lmax, autotune=True)
    d_ids = torch.empty((nq, kmax), dtype=torch.int32, device=dev)
    d_d = torch.empty((nq, kmax), dtype=torch.float32, device=dev)

    def step_u():
        rc = lib.pann_batch_run(b.handle, ctypes.c_void_p(dq.data_ptr()), nq, ks.ctypes.data_as(ctypes.c_void_p),
                                Ls.ctypes.data_as(ctypes.c_void_p), ctypes.c_void_p(d_ids.data_ptr()),
                                ctypes.c_void_p(d_d.data_ptr()), None, None, None, 1,
                                ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise P.PannError(rc, lib.pann_last_error().decode())

    t_b = _timed(step_u, flush, stream, steps, 3)
    ids_u = d_ids.cpu().numpy().astype(np.uint32)
    mapping = b.config()
    b.close()
    # the plain form in one launch at the largest k and beam
    qp = P.QueryParams(kmax, Lmax, n_index, idx.R, W["bf"])
    d_p = torch.empty((nq, kmax), dtype=torch.int32, device=dev)

    def step_plain_max():
        rc = lib.pann_search_device(idx.handle, ctypes.c_void_p(dq.data_ptr()), nq, ctypes.byref(qp),
                                    starts.ctypes.data_as(ctypes.c_void_p), 1, ctypes.c_void_p(d_p.data_ptr()),
                                    None, None, None, None, ctypes.c_void_p(stream.cuda_stream))
        if rc != 0:
            raise P.PannError(rc, lib.pann_last_error().decode())

    t_p = _timed(step_plain_max, flush, stream, steps, 3)
    # bit-exact per query with the plain form at the query's own k and beam (untimed)
    exact = True
    for kk, LL in sorted(set(zip(ks.tolist(), Ls.tolist()))):
        sel = np.where((ks == kk) & (Ls == LL))[0]
        r = idx.search(q[sel], kk, LL, batch_factor=W["bf"])
        exact &= bool(np.array_equal(ids_u[sel, :kk], r.ids))
    return {"queries": nq, "k": "uniform in {1,10,100}", "beam": "uniform in [k, 4k]",
            "qps_batched_graph": round(nq / t_b, 1), "qps_plain_one_launch_at_max_k_and_beam": round(nq / t_p, 1),
            "max_k": kmax, "max_beam": Lmax, "speedup_vs_one_launch": round(t_p / t_b, 3),
            "mapping": mapping, "bit_exact_with_plain": exact}


def run_serving(idx, q, nq, beam, radius, prec_out):
    """Open-loop Poisson arrivals at 5 offered rates, for the plain form and
    for the fastest precision form found above. Each of the 3 slots holds the
    scratch of 4096 queries at k = 100, beam 200 and admits up to 8192 queries a
    batch while their scratch fits (requests at k = 10 and the short beam
    need less per query, so they pack more)."""
    import parlayann_b200 as P

    rng = np.random.default_rng(7)
    rp = P.RangeParams(20, P.RANGE_GREEDY, radius, 0.0, 0)
    forms = [("plain", P.PREC_F32, 0, beam, 0)]
    best = max(prec_out.items(), key=lambda kv: kv[1]["qps_batched_graph"]) if prec_out else None
    if best is not None:
        nm, info = best
        forms.append((nm, P.PREC_BF16 if nm.startswith("bf16") else P.PREC_FP8, info["parents"], info["beam"],
                      1 if nm.endswith("_tc") else 0))
    serving = {}
    for fname, prec, parents, kbeam, scorer in forms:
        if prec != P.PREC_F32:
            idx.set_precision(prec)
        probe = P.Server(idx, max_batch_queries=4096, inflight=1, max_k=100, max_beam=max(200, kbeam),
                         precision=prec, parents=parents, scorer=scorer)
        budget = probe.admission()["scratch_bytes"]
        probe.close()
        srv = P.Server(idx, max_batch_queries=8192, inflight=3, max_k=100, max_beam=max(200, kbeam), precision=prec,
                       parents=parents, scorer=scorer, scratch_bytes=budget)

        def schedule(n, rate_qps, range_frac):
            nqs = rng.integers(1, 257, n)
            kinds = (rng.random(n) < range_frac).astype(np.uint32)
            nqs[kinds == 1] = 1
            kk = rng.choice(np.array([10, 100], np.uint32), n)
            bb = np.where(kk == 10, kbeam, 200).astype(np.uint32)
            gaps = rng.exponential(float(nqs.mean()) / rate_qps, n) if rate_qps else np.zeros(n)
            rows = rng.integers(0, nq - 257, n)
            return np.cumsum(gaps), kinds, nqs, kk, bb, rows

        a, kd, nqs, kk, bb, rows = schedule(400, 0, 0.0)  # capacity: everything at t = 0
        srv.admission(reset=True)
        lat, wall = srv.replay(a, kd, nqs, kk, bb, rows, q, rp)
        cap_qps = float(nqs.sum()) / wall
        adm = srv.admission(reset=True)
        cap_batch = adm["queries"] / max(adm["batches"], 1)
        rates = []
        for frac in (0.2, 0.4, 0.6, 0.8, 0.95):
            rate = frac * cap_qps
            n = int(min(20000, max(200, rate * 2.0 / 128)))
            a, kd, nqs, kk, bb, rows = schedule(n, rate, 0.01)
            lat, wall = srv.replay(a, kd, nqs, kk, bb, rows, q, rp)
            kn, rg = lat[kd == 0], lat[kd == 1]
            adm = srv.admission(reset=True)
            rates.append({"offered_qps": round(rate, 1), "achieved_qps": round(float(nqs.sum()) / wall, 1),
                          "batches": adm["batches"],
                          "queries_per_batch": round(adm["queries"] / max(adm["batches"], 1), 1),
                          "requests": n, "range_requests": int(kd.sum()),
                          "p50_ms": round(1e3 * float(np.percentile(lat, 50)), 3),
                          "p99_ms": round(1e3 * float(np.percentile(lat, 99)), 3),
                          "knn_p50_ms": round(1e3 * float(np.percentile(kn, 50)), 3),
                          "knn_p99_ms": round(1e3 * float(np.percentile(kn, 99)), 3),
                          "range_p50_ms": round(1e3 * float(np.percentile(rg, 50)), 3) if len(rg) else None,
                          "range_p99_ms": round(1e3 * float(np.percentile(rg, 99)), 3) if len(rg) else None})
        srv.close()
        serving[fname] = {"precision": int(prec), "parents": parents, "scorer": scorer, "beam_k10": kbeam,
                          "scratch_bytes_per_slot": budget, "capacity_qps_closed": round(cap_qps, 1),
                          "capacity_queries_per_batch": round(cap_batch, 1), "rates": rates}
    idx.set_precision(P.PREC_F32)
    return {"requests": "1-256 queries, k in {10,100} (beam for recall@10 >= 0.95 / 200), 1% range "
                        "requests (1 query, beam 20, greedy, radius at the 1% distance quantile)",
            "slots": 3, "admission": "by scratch bytes: each slot's arena holds 4096 queries at k=100, beam 200; "
                                     "a batch takes up to 8192 queries while its scratch fits",
            "forms": serving}


def cpu_baseline(base, q, graph, beam, res, args):
    """The reference's qsearchAll (compiled in place) on the host cores, as a
    reported baseline, on the same graph, queries and beam as the GPU line; its
    answers are compared with the GPU's query by query: ids in order, the float
    distance bits, visited counts and distance comparisons."""
    try:
        from oracle import oracle as O

        if not O.have_ref():
            return None
        nq = min(q.shape[0], args.cpu_queries)
        secs, ids, vis, cmps, dists = O.qsearch_time(base, q[:nq], graph, W["k"], beam, batch_factor=W["bf"])
        diff = ((ids != res.ids[:nq]).any(1) | (dists.view(np.uint32) != res.dists[:nq].view(np.uint32)).any(1) |
                (vis != res.visited[:nq]) | (cmps != res.cmps[:nq]))
        return {"value": round(nq / secs, 1), "unit": "queries/s", "cores": int(O.rlib().ref_num_workers()),
                "kind": "reference",
                "sample": f"{nq} of the {q.shape[0]} queries, one qsearchAll pass after a cache flush "
                          f"({secs:.2f} s), same graph and beam {beam}",
                "answers_identical": bool(not diff.any()), "queries_compared": int(nq),
                "queries_differing": int(diff.sum()),
                "compared": "ids in order, float32 distance bits, visited count, distance comparisons"}
    except Exception as ex:  # noqa: BLE001
        return {"value": None, "unit": "queries/s", "cores": 0, "kind": "reference", "sample": f"failed: {ex}"}


def run_reference(args):
    """--impl reference: the reference's own code on the host cores, end to end:
    its build_index builds the graph, its checkRecall (recall with the
    groundtruth's ties, FP64 groundtruth computed on the host) picks the
    smallest beam of its sweep list with recall@10 >= 0.95, and its qsearchAll
    is timed there. Only the in-place reference library is loaded (it also
    generates the data)."""
    rank, world, _ = env_rank()
    if rank != 0:
        return None
    from oracle import oracle as O

    if not O.have_ref():
        return {"impl": "reference", "unavailable": "oracle/_ref/libpann_ref.so was not built (reference checkout absent at build time)"}
    base, q = make_data(O.synth_mixture)
    t0 = time.time()
    graph, _ = O.build_graph("ref", base, W["R"], W["Lb"], W["alpha"], W["passes"], batch_factor=W["bf"])
    build_s = time.time() - t0
    t0 = time.time()
    gt, gd = O.groundtruth_fast(base, q, 20)
    gt_s = time.time() - t0
    k = W["k"]
    nq = min(q.shape[0], args.cpu_queries)
    sweep, beam, rec = [], None, None
    with tempfile.TemporaryDirectory() as tmp:
        gt_path = os.path.join(tmp, "gt.ibin")
        O.write_ibin(gt_path, gt[:nq], gd[:nq])
        for L in ([args.beam] if args.beam else BEAMS):
            r = O.check_recall(base, q[:nq], graph, gt_path, k, L, batch_factor=W["bf"])
            sweep.append((L, round(r["recall"], 4)))
            if r["recall"] >= 0.95 or args.beam:
                beam, rec = L, r
                break
    if beam is None:
        beam, rec = BEAMS[-1], {"recall": sweep[-1][1]}
    for _ in range(args.warmup):
        O.qsearch_time(base, q[:nq], graph, k, beam, batch_factor=W["bf"])
    times = []
    for _ in range(args.steps):
        secs, ids, vis, cmps, _d = O.qsearch_time(base, q[:nq], graph, k, beam, batch_factor=W["bf"])
        times.append(secs)
    t = sum(times)
    qps = nq * args.steps / t
    cores = int(O.rlib().ref_num_workers())
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": round(qps, 1),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(1e3 * t / args.steps, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded 256-component Gaussian mixture, L2-normalised)",
        "config": dict(CONFIG, parallelism=f"replicas x{world}"),
        "details": {"beam": beam, "recall_at_10": round(float(rec["recall"]), 4), "recall_sweep": sweep,
                    "graph_sha1": graph_digest(graph), "build_seconds_cpu": round(build_s, 2),
                    "mean_visited": round(float(vis.mean()), 2), "mean_cmps": round(float(cmps.mean()), 2),
                    "groundtruth": f"FP64 on the host cores (float32 candidate pass + FP64 re-rank, {gt_s:.1f} s), "
                                   "20 per query; recall by the reference's checkRecall",
                    "ranks_run": 1},
        "cpu_baseline": {"value": round(qps, 1), "unit": "queries/s", "cores": cores, "kind": "reference",
                         "sample": f"{nq} queries per step (qsearchAll after a cache flush, check_nn_recall.h:46-59)"},
        "e2e": {"value": round(qps, 1), "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--beam", type=int, default=0, help="fix the beam instead of sweeping for recall 0.95")
    ap.add_argument("--cpu-queries", type=int, default=10000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the precision / batched / range / serving forms")
    ap.add_argument("--forms", default="precision,batched,range,serving,sweep,c2",
                    help="comma list of the forms to run (precision, batched, range, serving, sweep: the "
                         "reference's search_and_parse sweep, and c2: the precision form on a 10M-point index, "
                         "Euclidean and mips)")
    ap.add_argument("--c3-n", type=int, default=100_000_000,
                    help="base vectors of the large uint8 batched-form run (forms c3)")
    ap.add_argument("--case", default="", help="profiling case instead of the benchmark: tile:PREC:PARENTS:SCORER "
                                                "(PREC bf16|fp8, SCORER cuda|tc)")
    ap.add_argument("--save-graph", default="", help="write the built graph (reference file format)")
    ap.add_argument("--load-graph", default="", help="load a graph file instead of building")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    line = run_reference(args) if args.impl == "reference" else run_ours(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
