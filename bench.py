#!/usr/bin/env python
"""ParFlex alignment benchmark (one JSON line on rank 0).

Workload (default, ``--workload prune64``): 64 synthetic chroma pairs,
N ~ U(40000, 60000) frames, M = N x U(0.7, 1.4) (12-d Dirichlet frames,
random monotone warp, 0-10 % unrelated padding per end), L = 2000 tiles,
steps {(1,1),(1,2),(2,1)}, weights {2,3,3}, beta 0.1.  One step aligns all 64
pairs with the chosen exact form: the learned tile proposer picks the tiles,
stage 1 (FP64 DP) runs on those only, stage 2 per pair, and a pair whose
path comes near a pruned tile gets those tiles added or falls back to the
full-tile method.  The reference answer is the plain full-tile FP64 form on
the same pairs (timed as ``plain_fp64_full_tiles``); ``exact_paths`` counts
the pairs whose best cost and path equal its own.

  value     DP cells/s, counting every cell of the full tiling (work the
            proposer avoids counts as throughput), features in HBM
  e2e       the same metric through PrunedBatch.load + run from pinned HOST
            features, paths and costs read back every step
  roofline  the masked run's stage-1 kernel: algorithmic bytes of the kept
            tiles (8 B of cost + 0.25 B of backpointers per cell) / its
            CUDA-event time vs the measured HBM peak, plus its issue roof
  cpu_baseline  the C restatement of the reference (oracle/) on the host
            cores, full tiling, on a block of whole tiles of the first pair
            whose tile count is a multiple of the host threads

Other workloads: ``config1`` (one 30000 x 37001 pair, L = 4000, plain FP64),
``batch256``, ``precision2048`` (FP32 form vs FP64 form), ``config0`` and the
small profiling cases.

Multi-GPU (torchrun, one rank per GPU): every rank aligns its own pairs
(independent replicas, weak scaling, no data-path collective); the time is
the max over ranks.

--impl reference times the reference algorithm's CPU restatement on the
host cores for the same workload (rank 0 only).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from parflexdtw_b200 import workloads as W  # noqa: E402

METRIC = "DP cells/s (ParFlex plain FP64 form, exact-path agreement)"
UNIT = "cells/s"


def tile_cells(N, M, Lb):
    hop = Lb - 1
    n1 = -(-(N - 1) // hop)
    n2 = -(-(M - 1) // hop)
    rows = [min(Lb, N - i * hop) for i in range(n1)]
    cols = [min(Lb, M - j * hop) for j in range(n2)]
    return sum(rows) * sum(cols), n1, n2


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fp:
            d = json.load(fp)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sms, mx, reasons = [], None, set()
        for line in (self.out or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9 or (self.uuid and self.uuid not in f[0]):
                continue
            try:
                sms.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                                "sw_power_cap"), f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sms:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sms), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sms)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reference_arm(args, spec):
    """CPU restatement of the reference on the host cores (rank 0 only)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import build_oracle, oracle
    build_oracle.build()
    threads = os.cpu_count() or 1
    F1, F2 = W.make_pair(spec)
    # the whole pair (every tile), or its first `ref_tile_rows` tile rows
    hop = spec.L - 1
    N, M = F1.shape[1], F2.shape[1]
    rows = F1.shape[1] if args.ref_tile_rows <= 0 else \
        min(F1.shape[1], args.ref_tile_rows * hop + 1)
    C = W.cost_matrix_host(F1[:, :rows], F2)
    cells, n1, n2 = tile_cells(C.shape[0], C.shape[1], spec.L)
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.parflex_full(C, spec.steps, spec.weights, spec.beta, spec.L, threads=threads)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    tot = sum(times)
    v = cells * len(times) / tot
    full_cells, _, _ = tile_cells(N, M, spec.L)
    what = "the whole pair" if rows == N else f"the first {n1} tile rows of the pair"
    sample = (f"{what} ({C.shape[0]} x {C.shape[1]}, {n1 * n2} tiles, {cells} cells) per "
              f"step, all stages")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": config_dict(spec, N, M, full_cells),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_dict(spec, N, M, cells):
    d = spec.describe()
    d.update({"N": N, "M": M, "cells_per_step": cells, "pairs_per_step_per_gpu": 1,
              "l2": "input C larger than L2 (no flush needed)", "parallelism": "replicas"})
    return d


def b200_arm(args, spec):
    import torch
    import torch.distributed as dist

    import parflexdtw_b200 as pf
    from parflexdtw_b200 import _lib

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    # each rank aligns its own pair (seed offset by rank)
    rs = W.PairSpec(spec.name, spec.n, spec.m_core, spec.L, pad_frac=spec.pad_frac,
                    weights=spec.weights, beta=spec.beta, seed=spec.seed + rank)
    F1, F2 = W.make_pair(rs)
    N, M = F1.shape[1], F2.shape[1]
    cells, n1, n2 = tile_cells(N, M, spec.L)
    plan = pf.Plan(N, M, spec.L, spec.steps, spec.weights)
    lib = _lib.load()
    f1d = torch.from_numpy(F1).to(dev)
    f2d = torch.from_numpy(F2).to(dev)
    # the cost matrix resident in HBM, in the plan's tile-skewed layout
    plan.load_features(f1d, f2d)

    def step():
        plan.run(None, spec.beta)

    for _ in range(args.warmup):
        step()
    best, end, found, n = plan.result()
    wp = plan.path(n)

    # --- timed region: device-resident input -------------------------------
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = lib.pfx_kernel_launches()
    with ClockSampler(uuid) as clk:
        e0.record()
        for k in range(args.steps):
            ev[k][0].record()
            plan.stage1()
            ev[k][1].record()
            plan.propagate()
            plan.scan(spec.beta)
            plan.stitch()
        e1.record()
        torch.cuda.synchronize()
    launches = lib.pfx_kernel_launches() - launches0
    ms_total = e0.elapsed_time(e1)
    ms_s1 = sum(a.elapsed_time(b) for a, b in ev) / args.steps
    if ws > 1:
        t = torch.tensor([ms_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / args.steps
    value = cells * ws * args.steps / (ms_total / 1e3)
    best2, end2, _, n2_ = plan.result()
    assert best2 == best and end2 == end, "non-deterministic result across steps"

    # --- e2e through the public API from pinned host features ---------------
    f1p = torch.from_numpy(F1).pin_memory()
    f2p = torch.from_numpy(F2).pin_memory()
    h2d = f1p.numel() * 8 + f2p.numel() * 8

    def e2e_step():
        _, tr = pf.tiled_stage1_from_features(f1p, f2p, steps=spec.steps,
                                              weights=spec.weights, beta=spec.beta, L=spec.L)
        r = pf.run_stage2_from_tiled(tr, beta=spec.beta)
        return r["best_cost"], r["stitched_wp"]

    for _ in range(max(1, min(args.warmup, 2))):
        e2e_step()
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_ms = []
    d2h = 0
    for _ in range(args.e2e_steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        bc, swp = e2e_step()
        b.record()
        torch.cuda.synchronize()
        e2e_ms.append(a.elapsed_time(b))
        d2h = swp.nbytes + 8 * 9  # path + best cost, best_end[7], length
        assert bc == best and np.array_equal(swp.T, wp.T), "e2e result differs"
    e2e_tot = sum(e2e_ms)
    if ws > 1:
        t = torch.tensor([e2e_tot], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_tot = float(t.item())
    e2e_value = cells * ws * len(e2e_ms) / (e2e_tot / 1e3)

    # --- roofline of the stage-1 kernel --------------------------------------
    peak, peak_kind = load_peaks()
    alg_bytes = cells * (8 + 0.25)
    achieved = alg_bytes / (ms_s1 / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "stage1_traffic.txt")
    if os.path.exists(tp):
        kv = {}
        with open(tp) as fp:
            for line in fp:
                if "=" in line and not line.lstrip().startswith("#"):
                    a, b = line.split("=", 1)
                    kv[a.strip()] = b.strip()
        if kv.get("workload") == spec.name:
            traffic = float(kv["bytes_per_launch"])
    roofline = {"bound": "hbm",
                "kernel": "stage 1: k_stage1_cl (largest tiles, 2-CTA clusters) + k_stage1_v3 "
                          "(other tiles, second stream), timed together",
                "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback",
                "stage1_ms_per_launch": ms_s1,
                "alg_bytes_per_cell": 8.25,
                "fp64_dp_cells_per_s": cells / (ms_s1 / 1e3),
                "traffic_source": "profiles/stage1_traffic.txt: dram read+write per cell of "
                                  "k_stage1_cl (8.50 B, profiles/k_stage1_cl_ncu_small.md), "
                                  "scaled by cells",
                "limiter": "the strip pipeline, not HBM: each strip follows the one above "
                           "it; about 226 warp instructions per 64-cell warp-step at 39 % "
                           "issue, FP64 pipe 16 %, the pipeline fill and drain of 32 warps "
                           "per tile the largest stall (profiles/k_stage1_cl_ncu_small.md)"}

    # --- row-major C input: the relayout into the tile-skewed layout --------
    C_dev = pf.cost_matrix_from_features_gpu(F1, F2)
    relayout_ms = []
    for _ in range(3):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        plan.load_cost(C_dev)
        b.record()
        torch.cuda.synchronize()
        relayout_ms.append(a.elapsed_time(b))
    plan.run(None, spec.beta)
    best3, end3, _, n3 = plan.result()
    assert best3 == best and end3 == end, "relayout and fused cost layouts disagree"

    # --- the drop-in call on a host cost matrix (rank 0): parflex(C) with a
    # pageable numpy C, as a caller of the reference passes it; the timed call
    # copies C to the device, relays it into the slabs and runs both stages
    dropin = None
    C = None
    if rank == 0:
        C = C_dev.cpu().numpy()
        bc_d, wp_d = pf.parflex(C, spec.steps, spec.weights, spec.beta, L=spec.L,
                                profile_dir=None)
        dropin_ms = []
        for _ in range(2):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            bc_d, wp_d = pf.parflex(C, spec.steps, spec.weights, spec.beta, L=spec.L,
                                    profile_dir=None)
            b.record()
            torch.cuda.synchronize()
            dropin_ms.append(a.elapsed_time(b))
        assert bc_d == best and np.array_equal(wp_d, wp.T), "drop-in and plan results differ"
        dropin = {"value": cells / (min(dropin_ms) / 1e3), "unit": UNIT,
                  "ms_per_call": min(dropin_ms), "h2d_bytes_per_call": int(C.nbytes),
                  "api": "parflex(C, steps, weights, beta, L) with C a host (pageable) "
                         "float64 numpy array: H2D of C, relayout, stage 1, stage 2"}

    # --- CPU baseline (rank 0): the oracle on the same pair -----------------
    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import build_oracle, oracle
        build_oracle.build()
        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        ref = oracle.parflex_full(C, spec.steps, spec.weights, spec.beta, spec.L,
                                  threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": cells / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"the full pair ({N} x {M}, {n1 * n2} tiles), all stages, once",
               "seconds": dt}
        parity = {"best_cost_equal": bool(ref["best_cost"] == best),
                  "path_equal": bool(np.array_equal(ref["wp"], wp.T)),
                  "path_len": int(wp.shape[0])}
    del C

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": config_dict(spec, N, M, cells),
            "pairs_per_s": ws * args.steps / (ms_total / 1e3),
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": len(e2e_ms),
                    "ms_per_step": e2e_tot / len(e2e_ms),
                    "api": "tiled_stage1_from_features + run_stage2_from_tiled"},
            "gpu_launches": int(launches),
            "relayout_ms": min(relayout_ms),
            "dropin_host_C": dropin,
            "clocks": clk.summary(),
            "parity": parity,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


BATCH_METRIC = "DP cells/s and pairs/s (ParFlex batch, plain FP64 form, exact-path agreement)"


def _batch_sample(pairs, spec, min_cells):
    """Leading pairs of a batch until their tile cells reach min_cells."""
    out, cells = [], 0
    for F1, F2 in pairs:
        n, m = F1.shape[1], F2.shape[1]
        out.append((F1, F2))
        cells += tile_cells(n, m, min(spec.L_choices))[0]
        if cells >= min_cells:
            break
    return out


def _oracle_on_sample(spec, Cs, Ls, threads, repeats=1):
    """Time the oracle (C restatement of the reference) on the cost matrices
    of sample pairs (built outside the timed region)."""
    from oracle import build_oracle, oracle
    build_oracle.build()
    cells = sum(tile_cells(C.shape[0], C.shape[1], Lb)[0] for C, Lb in zip(Cs, Ls))
    refs, times = [], []
    for r in range(repeats):
        t0 = time.perf_counter()
        refs = [oracle.parflex_full(C, spec.steps, spec.weights, spec.beta, Lb, threads=threads)
                for C, Lb in zip(Cs, Ls)]
        times.append(time.perf_counter() - t0)
    return refs, cells, times


def batch_reference_arm(args, spec):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    pairs = W.make_batch(spec)
    sample = _batch_sample(pairs, spec, args.ref_batch_cells)
    Ls = [max(spec.L_choices)] * len(sample)
    times = []
    cells = 0
    Cs = [W.cost_matrix_host(F1, F2) for F1, F2 in sample]
    for s in range(args.warmup + args.steps):
        _, cells, t = _oracle_on_sample(spec, Cs, Ls, threads)
        if s >= args.warmup:
            times.append(t[0])
    tot = sum(times)
    v = cells * len(times) / tot
    total_cells = sum(tile_cells(F1.shape[1], F2.shape[1], max(spec.L_choices))[0]
                      for F1, F2 in pairs)
    line = {
        "impl": "reference", "metric": BATCH_METRIC, "value": v, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(spec.describe(), cells_per_step=total_cells, parallelism="replicas"),
        "pairs_per_s": len(sample) * len(times) / tot,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"the first {len(sample)} pairs of the batch ({cells} tile "
                                   f"cells, L={Ls[0]}) per step, all stages, cost matrix "
                                   f"built outside the timed region"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batch_arm(args, spec):
    import torch
    import torch.distributed as dist

    from parflexdtw_b200 import _lib
    from parflexdtw_b200.autotune import Autotuner
    from parflexdtw_b200.batch import Batch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    lib = _lib.load()
    pairs = W.make_batch(spec, seed_offset=1000 * rank)  # each rank its own batch
    shapes = [(F1.shape[1], F2.shape[1]) for F1, F2 in pairs]
    t0 = time.perf_counter()
    tuner = Autotuner(candidates_L=spec.L_choices)
    Ls, warps = tuner.choose(shapes, spec.steps, spec.weights, spec.d)
    tune_s = time.perf_counter() - t0
    b = Batch(shapes, Ls, spec.steps, spec.weights, spec.d, warps=warps, cost=args.cost)
    cells = b.cells
    b.load(pairs)
    # one direct run with phase events (cost building, stage 1, stage 2)
    b.run(spec.beta, use_graph=False)
    cost_ms, s1_ms, s2_ms = b.timing()
    best0, end0, lens0 = b.results()
    for _ in range(args.warmup):
        b.run(spec.beta)
    torch.cuda.synchronize()

    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = lib.pfx_kernel_launches()
    with ClockSampler(uuid) as clk:
        e0.record()
        for _ in range(args.steps):
            b.run(spec.beta)
        e1.record()
        torch.cuda.synchronize()
    launches = lib.pfx_kernel_launches() - launches0
    ms_total = e0.elapsed_time(e1)
    if ws > 1:
        t = torch.tensor([ms_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_total = float(t.item())
    value = cells * ws * args.steps / (ms_total / 1e3)
    best1, end1, lens1 = b.results()
    assert np.array_equal(best1, best0) and np.array_equal(end1, end0), "non-deterministic"
    paths = b.paths(lens1)

    # e2e: pinned host features in, results and paths out, every step
    pinned = [(torch.from_numpy(F1).pin_memory(), torch.from_numpy(F2).pin_memory())
              for F1, F2 in pairs]
    h2d = sum(a.numel() * 8 + c.numel() * 8 for a, c in pinned)
    d2h = 0
    e2e_ms = []
    for s in range(1 + args.e2e_steps):
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        b.load(pinned)
        b.run(spec.beta)
        bb, ee, ll = b.results()
        pp = b.paths(ll)
        c.record()
        torch.cuda.synchronize()
        if s:
            e2e_ms.append(a.elapsed_time(c))
        d2h = 8 * 9 * b.n + 16 * int(ll.sum())
        assert np.array_equal(bb, best0) and all(np.array_equal(x, y) for x, y in zip(pp, paths))
    e2e_tot = sum(e2e_ms)
    if ws > 1:
        t = torch.tensor([e2e_tot], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_tot = float(t.item())
    e2e_value = cells * ws * len(e2e_ms) / (e2e_tot / 1e3)

    peak, peak_kind = load_peaks()
    achieved = cells * 8.25 / (s1_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": "k_stage1_v3 (tile queue, all pairs of a wave)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": cells * 8.4213,
                "traffic_source": "8.4213 B per cell, measured per launch on the 30000 x 37001 "
                                  "workload (profiles/stage1_traffic.txt); every cell's cost "
                                  "is read once from its slab",
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback",
                "stage1_ms": s1_ms, "cost_build_ms": cost_ms, "stage2_ms": s2_ms,
                "fp64_dp_cells_per_s": cells / (s1_ms / 1e3)}

    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        import parflexdtw_b200 as pf
        sample = _batch_sample(pairs, spec, args.ref_batch_cells)
        # the device's fixed-order FP64 cost, bit-identical to the host
        # restatement (workloads.cost_matrix_det), copied out for the oracle
        Cs = [pf.cost_matrix_from_features_gpu(F1, F2).cpu().numpy() for F1, F2 in sample]
        refs, scells, t = _oracle_on_sample(spec, Cs, Ls[:len(sample)], threads)
        del Cs
        cpu = {"value": scells / t[0], "unit": UNIT, "cores": threads, "kind": "port",
               "pairs_per_s": len(sample) / t[0],
               "sample": f"the first {len(sample)} pairs of the batch ({scells} tile cells, "
                         f"autotuned L), all stages, cost matrix built outside the timing",
               "seconds": t[0]}
        ok_b = all(r["best_cost"] == best0[i] for i, r in enumerate(refs))
        ok_p = all(np.array_equal(r["wp"], paths[i].T) for i, r in enumerate(refs))
        parity = {"pairs_checked": len(refs), "best_cost_equal": bool(ok_b),
                  "path_equal": bool(ok_p)}

    if rank == 0:
        cfg = dict(spec.describe())
        cfg.update({"cells_per_step": cells, "tiles": b.tiles, "waves": b.waves,
                    "warps_per_tile": b.warps, "L_per_pair_counts":
                    {str(x): Ls.count(x) for x in sorted(set(Ls))},
                    "autotune_table": {k: list(v) for k, v in tuner.table.items()},
                    "autotune_seconds": tune_s, "parallelism": "replicas",
                    "graph": "whole batch recorded once, replayed per step",
                    "cost_build": ("inside the stage-1 kernel, tile by tile, one launch"
                                   if b.cost_in_kernel else
                                   "separate cost kernels into slabs, in waves"),
                    "l2": "cost slabs and features larger than L2 (no flush needed)",
                    "input": "features resident in HBM; the timed step builds the cost"})
        line = {
            "metric": BATCH_METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": cfg,
            "pairs_per_s": ws * b.n * args.steps / (ms_total / 1e3),
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": len(e2e_ms),
                    "ms_per_step": e2e_tot / len(e2e_ms),
                    "pairs_per_s": ws * b.n * len(e2e_ms) / (e2e_tot / 1e3),
                    "api": "Batch.load (pinned host features) + run + results + paths"},
            "gpu_launches": int(launches), "clocks": clk.summary(), "parity": parity,
        }
        print(json.dumps(line), flush=True)
    b.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


PREC_METRIC = ("DP cells/s and pairs/s (ParFlex batch, FP32 chosen form: bf16 tensor-core "
               "cost + FP32 DP, against the FP64 plain form)")


def _batch_run_timed(b, beta, steps, warmup, uuid=None):
    """Phase times of one direct run, then `steps` graph replays timed with
    CUDA events (after `warmup`); returns (ms_total, phases, clocks)."""
    import torch
    b.run(beta, use_graph=False)
    phases = b.timing()
    for _ in range(warmup):
        b.run(beta)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = ClockSampler(uuid) if uuid else None
    if clk:
        clk.__enter__()
    e0.record()
    for _ in range(steps):
        b.run(beta)
    e1.record()
    torch.cuda.synchronize()
    if clk:
        clk.__exit__(None, None, None)
    return e0.elapsed_time(e1), phases, (clk.summary() if clk else None)


def precision_reference_arm(args, spec):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    sample = W.make_precision_batch(spec, n_pairs=args.ref_pairs)
    Cs = [W.cost_matrix_host(F1, F2) for F1, F2 in sample]
    times, cells = [], 0
    for s in range(args.warmup + args.steps):
        _, cells, t = _oracle_on_sample(spec, Cs, [spec.L] * len(Cs), threads)
        if s >= args.warmup:
            times.append(t[0])
    tot = sum(times)
    v = cells * len(times) / tot
    line = {
        "impl": "reference", "metric": PREC_METRIC, "value": v, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(spec.describe(), parallelism="replicas"),
        "pairs_per_s": len(Cs) * len(times) / tot,
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"the first {len(Cs)} pairs ({cells} tile cells, L={spec.L}) "
                                   f"per step, FP64 (the reference's arithmetic), all stages, "
                                   f"cost matrix built outside the timed region"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def precision_arm(args, spec):
    import torch
    import torch.distributed as dist

    import parflexdtw_b200 as pf
    from parflexdtw_b200 import _lib
    from parflexdtw_b200 import precision as PR
    from parflexdtw_b200.batch import Batch

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    lib = _lib.load()
    t0 = time.perf_counter()
    pairs = W.make_precision_batch(spec, seed_offset=1000 * rank, n_pairs=args.pairs)
    gen_s = time.perf_counter() - t0
    shapes = [(F1.shape[1], F2.shape[1]) for F1, F2 in pairs]
    n = len(pairs)

    # --- FP32 chosen form -------------------------------------------------
    b32 = Batch(shapes, spec.L, spec.steps, spec.weights, spec.d, precision="fp32")
    cells = b32.cells
    b32.load(pairs)
    if ws > 1:
        dist.barrier()
    launches0 = lib.pfx_kernel_launches()
    ms32, ph32, clk = _batch_run_timed(b32, spec.beta, args.steps, args.warmup, uuid)
    launches = lib.pfx_kernel_launches() - launches0
    if ws > 1:
        t = torch.tensor([ms32], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms32 = float(t.item())
    best32, end32, lens32 = b32.results()
    paths32 = b32.paths(lens32)
    # e2e: pinned host features in, results and paths out, every step
    pinned = [(torch.from_numpy(F1).pin_memory(), torch.from_numpy(F2).pin_memory())
              for F1, F2 in pairs]
    h2d = sum(a.numel() * 8 + c.numel() * 8 for a, c in pinned)
    e2e_ms, d2h = [], 0
    for s in range(1 + args.e2e_steps):
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        b32.load(pinned)
        b32.run(spec.beta)
        bb, ee, ll = b32.results()
        pp = b32.paths(ll)
        c.record()
        torch.cuda.synchronize()
        if s:
            e2e_ms.append(a.elapsed_time(c))
        d2h = 8 * 9 * n + 16 * int(ll.sum())
        assert np.array_equal(bb, best32), "FP32 form not deterministic"
    del pinned
    info32 = {"waves": b32.waves, "tiles": b32.tiles, "warps_per_tile": b32.warps,
              "device_bytes": b32.device_bytes}
    b32.close()
    torch.cuda.empty_cache()

    # --- FP64 plain form on the same pairs ---------------------------------
    b64 = Batch(shapes, spec.L, spec.steps, spec.weights, spec.d, precision="fp64")
    b64.load(pairs)
    ms64, ph64, _ = _batch_run_timed(b64, spec.beta, args.plain_steps, 1)
    if ws > 1:
        t = torch.tensor([ms64], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms64 = float(t.item())
    best64, end64, lens64 = b64.results()
    paths64 = b64.paths(lens64)
    b64.close()
    torch.cuda.empty_cache()

    value32 = cells * ws * args.steps / (ms32 / 1e3)
    value64 = cells * ws * args.plain_steps / (ms64 / 1e3)

    line = None
    if rank == 0:
        t1 = time.perf_counter()
        prec = PR.compare_results(pairs, best32, paths32, best64, paths64, spec.steps,
                                  spec.weights, end32[:, 6], end64[:, 6])
        # cost-matrix error on sample pairs (both forms' slabs)
        cmax, csum, ccnt = 0.0, 0.0, 0
        for F1, F2 in pairs[:args.cerr_pairs]:
            N, M = F1.shape[1], F2.shape[1]
            p32 = pf.Plan(N, M, spec.L, spec.steps, spec.weights, precision="fp32")
            p64 = pf.Plan(N, M, spec.L, spec.steps, spec.weights)
            f1, f2 = torch.from_numpy(F1).to(dev), torch.from_numpy(F2).to(dev)
            p32.load_features(f1, f2)
            p64.load_features(f1, f2)
            mx, sm, ct = PR.cost_error(p32, p64)
            cmax, csum, ccnt = max(cmax, mx), csum + sm, ccnt + ct
            p32.close()
            p64.close()
        prec.update({"C_abs_err_max": cmax, "C_abs_err_mean": csum / max(ccnt, 1),
                     "C_err_pairs": min(args.cerr_pairs, n),
                     "report_seconds": time.perf_counter() - t1})
        cpu = None
        parity = None
        if not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            sample = pairs[:args.ref_pairs]
            Cs = [pf.cost_matrix_from_features_gpu(F1, F2).cpu().numpy() for F1, F2 in sample]
            refs, scells, t = _oracle_on_sample(spec, Cs, [spec.L] * len(Cs), threads)
            cpu = {"value": scells / t[0], "unit": UNIT, "cores": threads, "kind": "port",
                   "pairs_per_s": len(Cs) / t[0],
                   "sample": f"the first {len(Cs)} pairs ({scells} tile cells), FP64, all "
                             f"stages, cost matrix built outside the timing",
                   "seconds": t[0]}
            parity = {"pairs_checked": len(refs),
                      "fp64_plain_best_cost_equal": bool(all(
                          r["best_cost"] == best64[i] for i, r in enumerate(refs))),
                      "fp64_plain_path_equal": bool(all(
                          np.array_equal(r["wp"], paths64[i].T) for i, r in enumerate(refs)))}
            del Cs
        peak, peak_kind = load_peaks()
        s1 = ph32[1]
        roofline = {
            "bound": "hbm", "kernel": "k_stage1_v3<.., float> (FP32 DP, tile queue)",
            "achieved": cells * 4.25 / (s1 / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
            "frac": cells * 4.25 / (s1 / 1e3) / 1e9 / peak,
            "traffic": None, "alg_bytes_per_cell": 4.25,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
            if peak_kind == "measured" else "fallback",
            "stage1_ms": s1, "cost_gemm_ms": ph32[0], "stage2_ms": ph32[2],
            "fp32_dp_cells_per_s": cells / (s1 / 1e3),
            "gemm": {"kernel": "k_gemm_cost_skew (tcgen05 BF16 -> FP32, TMA, skew epilogue)",
                     "bound": "hbm", "alg_bytes_per_cell": 4.0,
                     "achieved_GBps": cells * 4.0 / (ph32[0] / 1e3) / 1e9,
                     "tensor_TFLOPs": 2.0 * spec.d * cells * 1.5 / (ph32[0] / 1e3) / 1e12,
                     "note": "time includes the bf16 feature conversion kernels; FLOPs "
                             "count the 1.5x column overlap the kernel computes"},
        }
        cfg = dict(spec.describe())
        cfg.update({"pairs_run": n, "cells_per_step": cells, "generation_seconds": gen_s,
                    "parallelism": "replicas", "input": "features resident in HBM; the "
                    "timed step builds the cost", "l2": "slabs larger than L2 (no flush "
                    "needed)", "fp32_batch": info32})
        line = {
            "metric": PREC_METRIC, "value": value32, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms32 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16 cost / f32 DP", "data": "synthetic", "config": cfg,
            "pairs_per_s": ws * n * args.steps / (ms32 / 1e3),
            "plain_fp64": {"value": value64, "unit": UNIT, "steps": args.plain_steps,
                           "ms_per_step": ms64 / args.plain_steps,
                           "pairs_per_s": ws * n * args.plain_steps / (ms64 / 1e3),
                           "phases_ms": {"cost": ph64[0], "stage1": ph64[1], "stage2": ph64[2]}},
            "speedup_fp32_over_fp64": value32 / value64,
            "precision": prec,
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": cells * ws * len(e2e_ms) / (sum(e2e_ms) / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "steps": len(e2e_ms), "ms_per_step": sum(e2e_ms) / len(e2e_ms),
                    "api": "Batch.load (pinned host features) + run + results + paths"},
            "gpu_launches": int(launches), "clocks": clk, "parity": parity,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


# BASELINE's metric, measured on the learned-pruning workload: the chosen exact
# form (learned tile pruning + FP64 DP) against the plain full-tile FP64 form;
# cells are counted on the full tiling.
PRUNE_METRIC = "DP cells/s and pairs/s: chosen form vs plain GPU at exact-path agreement"


def _balanced_tile_block(N, M, Lb, threads, rounds):
    """(n1s, n2s): a block of whole L x L tiles at the start of an N x M pair
    whose tile count is a multiple of `threads` (every host thread gets the
    same number of equal tiles) and close to rounds x threads."""
    hop = Lb - 1
    max1, max2 = max((N - 1) // hop, 1), max((M - 1) // hop, 1)
    target = rounds * threads
    best = None
    for a in range(1, max1 + 1):
        for b in range(1, max2 + 1):
            t = a * b
            key = (t % threads != 0, abs(t - target), abs(a - b))
            if best is None or key < best[0]:
                best = (key, a, b)
    return best[1], best[2]


def _prune_cpu_sample(spec, threads, rounds):
    """Cost matrix of a bounded CPU sample of the learned-pruning workload:
    the leading block of whole tiles of its first pair (same generator and
    seed), with a tile count that is a multiple of the host threads, so
    that no thread idles while others work.  Returns (C, cells, text)."""
    Lb = spec.L_choices[0]
    F1, F2 = W.make_batch(W.BatchSpec("x", 1, spec.n_lo, spec.n_hi, pad_frac=spec.pad_frac,
                                      seed=spec.seed))[0]
    N, M = F1.shape[1], F2.shape[1]
    a, b = _balanced_tile_block(N, M, Lb, threads, rounds)
    rows, cols = a * (Lb - 1) + 1, b * (Lb - 1) + 1
    C = W.cost_matrix_host(F1[:, :rows], F2[:, :cols])
    cells = tile_cells(rows, cols, Lb)[0]
    text = (f"the leading {a} x {b} block of whole {Lb} x {Lb} tiles ({a * b} tiles on "
            f"{threads} threads, {rows} x {cols} frames, {cells} cells) of the workload's "
            f"first pair ({N} x {M}), full tiling, FP64, all stages, cost matrix built "
            f"outside the timing")
    return C, cells, text


def prune_reference_arm(args, spec):
    """The C restatement of the reference on the host cores, full tiling (the
    reference has no pruning), on a balanced block of whole tiles of the
    workload's first pair per step."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import build_oracle, oracle
    build_oracle.build()
    threads = os.cpu_count() or 1
    Lb = spec.L_choices[0]
    C, cells, sample = _prune_cpu_sample(spec, threads, args.ref_rounds)
    times = []
    for s_ in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.parflex_full(C, spec.steps, spec.weights, spec.beta, Lb, threads=threads)
        if s_ >= args.warmup:
            times.append(time.perf_counter() - t0)
    tot = sum(times)
    v = cells * len(times) / tot
    line = {
        "impl": "reference", "metric": PRUNE_METRIC, "value": v, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(spec.describe(), parallelism="replicas"),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample + " per step"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _stage1_counters(workload):
    """Per-cell DRAM bytes and warp instructions of the stage-1 kernel, from
    the committed ncu summary (profiles/stage1_counters.txt), for the named
    workload; {} when absent."""
    p = os.path.join(ROOT, "profiles", "stage1_counters.txt")
    out, cur = {}, None
    if not os.path.exists(p):
        return out
    with open(p) as fp:
        for line in fp:
            line = line.split("#", 1)[0].strip()
            if not line or "=" not in line:
                continue
            k, v = (x.strip() for x in line.split("=", 1))
            if k == "workload":
                cur = v
            elif cur == workload:
                try:
                    out[k] = float(v)
                except ValueError:
                    out[k] = v
    return out


def _masked_cells(masks, shapes, Lb):
    """DP cells of the tiles a concatenation of per-pair (n1, n2) masks keeps."""
    hop = Lb - 1
    tot, off = 0, 0
    for N, M in shapes:
        n1, n2 = -(-(N - 1) // hop), -(-(M - 1) // hop)
        rows = np.minimum(Lb, N - np.arange(n1) * hop).astype(np.int64)
        cols = np.minimum(Lb, M - np.arange(n2) * hop).astype(np.int64)
        m = np.asarray(masks[off:off + n1 * n2], bool).reshape(n1, n2)
        tot += int(rows @ m.astype(np.int64) @ cols)
        off += n1 * n2
    return tot


def _masked_slab_bytes(masks, shapes, Lb, elem=8):
    """Bytes the cost kernels write for the kept tiles: per tile its strips x
    skewed steps x 64 rows (span = W + 63 rounded up to 16 steps)."""
    hop = Lb - 1
    tot, off = 0, 0
    for N, M in shapes:
        n1, n2 = -(-(N - 1) // hop), -(-(M - 1) // hop)
        rows = np.minimum(Lb, N - np.arange(n1) * hop).astype(np.int64)
        cols = np.minimum(Lb, M - np.arange(n2) * hop).astype(np.int64)
        strips = -(-rows // 64)
        spans = -(-(cols + 63) // 16) * 16
        m = np.asarray(masks[off:off + n1 * n2], bool).reshape(n1, n2)
        tot += int(strips @ m.astype(np.int64) @ spans) * 64 * elem
        off += n1 * n2
    return tot


def prune_arm(args, spec):
    import torch
    import torch.distributed as dist

    import parflexdtw_b200 as pf
    from parflexdtw_b200 import _lib
    from parflexdtw_b200.batch import Batch
    from parflexdtw_b200.prune import TileProposer

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=900),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    lib = _lib.load()
    Lb = spec.L_choices[0]
    n_pairs = args.pairs or spec.n_pairs
    t0 = time.perf_counter()
    spec_r = W.BatchSpec(spec.name, n_pairs, spec.n_lo, spec.n_hi, pad_frac=spec.pad_frac,
                         seed=spec.seed + 1000 * rank)
    pairs = W.make_batch(spec_r)
    gen_s = time.perf_counter() - t0
    shapes = [(F1.shape[1], F2.shape[1]) for F1, F2 in pairs]
    cells = sum(tile_cells(n, m, Lb)[0] for n, m in shapes)
    net = TileProposer.load()

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def timed(fn, steps):
        gc.collect()  # (automatic collection is off: no pause inside a timed step)
        torch.cuda.synchronize()
        a, b = ev(), ev()
        a.record()
        for _ in range(steps):
            out = fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b), out

    def max_ranks(x):
        if ws == 1:
            return x
        t = torch.tensor([x], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # --- plain form: every tile, FP64, one batch (waves), graph replay --------
    cost_fma = args.cost_def == "fma" and args.cost == "slabs"
    bp = Batch(shapes, Lb, spec.steps, spec.weights, 12, cost=args.cost, warps=args.warps,
               cost_fma=cost_fma)
    bp.load(pairs)
    bp.run(spec.beta, use_graph=False)
    ph_plain = bp.timing()
    best0, end0, lens0 = bp.results()
    paths0 = bp.paths(lens0)
    plain_info = {"waves": bp.waves, "warps_per_tile": bp.warps, "tiles": bp.tiles,
                  "cost_in_stage1": bp.cost_in_kernel}
    for _ in range(max(1, args.warmup - 1)):
        bp.run(spec.beta)
    if ws > 1:
        dist.barrier()
    ms_plain, _ = timed(lambda: bp.run(spec.beta), args.plain_steps)
    ms_plain = max_ranks(ms_plain)
    bp.close()
    del bp
    torch.cuda.empty_cache()

    # --- chosen form: proposer + kept tiles only, FP64 ----------------------
    pb = pf.PrunedBatch(shapes, Lb, spec.steps, spec.weights, 12, proposer=net,
                        cost=args.cost, warps=args.warps, cost_fma=cost_fma)
    pb.load(pairs)
    for _ in range(args.warmup):
        out, info = pb.run(spec.beta)
    if ws > 1:
        dist.barrier()
    launches0 = lib.pfx_kernel_launches()
    with ClockSampler(uuid) as clk:
        ms_pruned, (out, info) = timed(lambda: pb.run(spec.beta), args.steps)
    launches = lib.pfx_kernel_launches() - launches0
    ms_pruned = max_ranks(ms_pruned)
    _, prof = pb.run(spec.beta, profile=True)
    pb_masks = pb.last_masks.cpu().numpy()
    kept_cells = _masked_cells(pb_masks, shapes, Lb)
    agree = sum(int(bc == best0[i] and np.array_equal(wp, paths0[i].T))
                for i, (bc, wp) in enumerate(out))
    # e2e: pinned host features in, results out
    pinned = [(torch.from_numpy(F1).pin_memory(), torch.from_numpy(F2).pin_memory())
              for F1, F2 in pairs]
    h2d = sum(a.numel() * 8 + c.numel() * 8 for a, c in pinned)

    def e2e_step():
        # each pair's upload runs on its proposer stream inside the recorded
        # proposer graph, overlapping the other pairs' proposer passes
        return pb.run(spec.beta, host_pairs=pinned)

    e2e_step()
    ms_e2e, (out2, _) = timed(e2e_step, args.e2e_steps)
    ms_e2e = max_ranks(ms_e2e)
    d2h = sum(wp.nbytes for _, wp in out2) + 8 * 9 * n_pairs
    pb.close()
    del pb
    torch.cuda.empty_cache()

    # --- the same proposer over the FP32 form (BF16 tcgen05 cost GEMM, FP32
    # DP): its full-tile results, then the pruned run against them ----------
    b32 = Batch(shapes, Lb, spec.steps, spec.weights, 12, precision="fp32")
    b32.load(pairs)
    b32.run(spec.beta, use_graph=False)
    best32, _, lens32 = b32.results()
    paths32 = b32.paths(lens32)
    b32.close()
    del b32
    torch.cuda.empty_cache()
    p32 = pf.PrunedBatch(shapes, Lb, spec.steps, spec.weights, 12, proposer=net,
                         precision="fp32")
    p32.load(pairs)
    for _ in range(args.warmup):
        p32.run(spec.beta)
    if ws > 1:
        dist.barrier()
    ms_32, (out32, info32) = timed(lambda: p32.run(spec.beta), args.steps)
    ms_32 = max_ranks(ms_32)
    p32.close()
    del p32
    torch.cuda.empty_cache()
    agree32 = sum(int(bc == best32[i] and np.array_equal(wp, paths32[i].T))
                  for i, (bc, wp) in enumerate(out32))
    agree32_64 = sum(int(np.array_equal(wp, paths0[i].T)) for i, (_, wp) in enumerate(out32))
    rel32 = [abs(bc - best0[i]) / abs(best0[i]) for i, (bc, _) in enumerate(out32)]
    v_32 = cells * ws * args.steps / (ms_32 / 1e3)

    v_pruned = cells * ws * args.steps / (ms_pruned / 1e3)
    v_plain = cells * ws * args.plain_steps / (ms_plain / 1e3)
    clocks = clk.summary()

    # --- roofline of the masked run's stage-1 kernel (kept tiles only) -------
    peak, peak_kind = load_peaks()
    s1_ms = prof["align_ms"]["stage1"]
    ctr = _stage1_counters(spec.name)
    achieved = kept_cells * 8.25 / (s1_ms / 1e3) / 1e9
    roofline = {
        "bound": "hbm", "kernel": "k_stage1_v3<NW, 1, double> (tile queue, kept tiles of all "
                                  "pairs of a wave)",
        "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
        "traffic": kept_cells * ctr["dram_bytes_per_cell"] if "dram_bytes_per_cell" in ctr
        else None,
        "traffic_source": ("ncu dram__bytes_read.sum + dram__bytes_write.sum per DP cell of "
                           "the same kernel on the small case of this workload "
                           "(profiles/stage1_counters.txt), times the kept cells"),
        "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
        if peak_kind == "measured" else "fallback",
        "alg_bytes_per_cell": 8.25, "kept_cells": kept_cells, "stage1_ms": s1_ms,
        "fp64_dp_cells_per_s": kept_cells / (s1_ms / 1e3)}
    # the FP64 cost kernel of the masked run: its slab writes against HBM
    slab_bytes = _masked_slab_bytes(pb_masks, shapes, Lb)
    cost_ms = prof["align_ms"]["cost"]
    roofline["cost_kernel"] = {
        "kernel": "k_cost_skew<12, %s> (FP64 cost into the kept tiles' slabs)"
                  % ("true: FMA chain" if cost_fma else "false: separately rounded"),
        "bound": "hbm", "slab_bytes": slab_bytes, "ms": cost_ms,
        "achieved_GBps": slab_bytes / (cost_ms / 1e3) / 1e9,
        "frac": slab_bytes / (cost_ms / 1e3) / 1e9 / peak,
        "note": "algorithmic bytes = the slab elements written (8 B each, the skewed layout's "
                "zero padding included); the features it reads are L2-resident"}
    if "inst_per_cell" in ctr and clocks.get("sm_mhz"):
        smsp = 4 * torch.cuda.get_device_properties(dev).multi_processor_count
        inst = ctr["inst_per_cell"] * kept_cells / (s1_ms / 1e3)
        issue_peak = smsp * clocks["sm_mhz"] * 1e6
        roofline["issue"] = {
            "achieved_warp_inst_per_s": inst, "peak_warp_inst_per_s": issue_peak,
            "frac": inst / issue_peak, "warp_inst_per_cell": ctr["inst_per_cell"],
            "source": "smsp__inst_executed.sum per DP cell (profiles/stage1_counters.txt); "
                      "peak = one warp instruction per SMSP per cycle at the median SM clock "
                      "sampled during the timed region"}

    # --- CPU baseline (rank 0): the oracle on a balanced sample -------------
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import build_oracle, oracle
        build_oracle.build()
        threads = os.cpu_count() or 1
        C, scells, sample = _prune_cpu_sample(spec, threads, args.ref_rounds)
        ts = []
        for _ in range(args.cpu_repeats):
            t0 = time.perf_counter()
            oracle.parflex_full(C, spec.steps, spec.weights, spec.beta, Lb, threads=threads)
            ts.append(time.perf_counter() - t0)
        del C
        cpu = {"value": scells / statistics.median(ts), "unit": UNIT, "cores": threads,
               "kind": "port", "sample": f"{sample}; median of {len(ts)} runs",
               "seconds": ts}

    if rank == 0:
        line = {
            "metric": PRUNE_METRIC, "value": v_pruned, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_pruned / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": dict(spec.describe(), pairs_run=n_pairs, cells_per_step=cells,
                           generation_seconds=gen_s, parallelism="replicas",
                           input="features resident in HBM; every step builds the cost",
                           cost_build=("inside the stage-1 kernel, tile by tile"
                                       if args.cost == "tile" else
                                       "separate cost kernels into slabs, in waves"),
                           cost_definition=(
                               "1 - sum_f a_f b_f as a fixed-order FP64 FMA chain "
                               "(PFX_BATCH_COST_FMA), both forms" if cost_fma else
                               "1 - sum_f a_f b_f with separately rounded FP64 products and "
                               "sums, both forms"),
                           timing="CUDA events around whole steps (host-side proposer mask "
                                  "read-back and fallback checks included)",
                           l2="cost slabs larger than L2 (no flush needed)"),
            "pairs_per_s": ws * n_pairs * args.steps / (ms_pruned / 1e3),
            "exact_paths": f"{agree}/{n_pairs}",
            "plain_fp64_full_tiles": {
                "value": v_plain, "unit": UNIT, "steps": args.plain_steps,
                "ms_per_step": ms_plain / args.plain_steps,
                "pairs_per_s": ws * n_pairs * args.plain_steps / (ms_plain / 1e3),
                "form": "batched, all tiles, one graph replay", "batch": plain_info,
                "phases_ms": {"cost": ph_plain[0], "stage1": ph_plain[1], "stage2": ph_plain[2]}},
            "speedup_over_plain": v_pruned / v_plain,
            "pruning": dict(info, exact_path_agreement_rate=agree / n_pairs,
                            profiled_phases_ms=prof.get("phases_ms"),
                            profiled_align_ms=prof.get("align_ms"),
                            fallback_rate=info["fallbacks"] / n_pairs,
                            proposer="3 conv layers, 32 channels, bf16 activations, "
                                     "parflexdtw_b200/data/proposer_L2000.npz",
                            threshold=net.threshold, dilation_tiles=1),
            "fp32_pruned": {
                "value": v_32, "unit": UNIT, "ms_per_step": ms_32 / args.steps,
                "speedup_over_plain": v_32 / v_plain,
                "exact_agreement_with_fp32_full_tiles": agree32 / n_pairs,
                "path_agreement_with_fp64_full_tiles": agree32_64 / n_pairs,
                "best_cost_rel_err_vs_fp64": {"max": max(rel32), "mean": float(np.mean(rel32))},
                "skipped_fraction": info32["skipped_fraction"],
                "fallbacks": info32["fallbacks"],
                "form": "same proposer; BF16 tcgen05 cost GEMM, FP32 DP"},
            "roofline": roofline, "cpu_baseline": cpu,
            "e2e": {"value": cells * ws * args.e2e_steps / (ms_e2e / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "steps": args.e2e_steps, "ms_per_step": ms_e2e / args.e2e_steps,
                    "api": "PrunedBatch.run(host_pairs=pinned host features): uploads "
                           "inside the run"},
            "gpu_launches": int(launches), "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


SHARD_METRIC = ("DP cells/s (ParFlex plain FP64 form, one long pair, tiles sharded across "
                "GPUs with one edge exchange)")


def _shard_cpu_sample(spec, threads, rounds):
    """Cost matrix of a bounded CPU sample of the tile-sharded pair: a block
    of whole tiles at its start with a tile count that is a multiple of the
    host threads.  Returns (C, cells, text)."""
    F1, F2 = W.make_pair(spec)
    N, M = F1.shape[1], F2.shape[1]
    a, b = _balanced_tile_block(N, M, spec.L, threads, rounds)
    rows, cols = a * (spec.L - 1) + 1, b * (spec.L - 1) + 1
    C = W.cost_matrix_host(F1[:, :rows], F2[:, :cols])
    cells = tile_cells(rows, cols, spec.L)[0]
    text = (f"the leading {a} x {b} block of whole {spec.L} x {spec.L} tiles ({a * b} tiles on "
            f"{threads} threads, {rows} x {cols} frames, {cells} cells) of the pair "
            f"({N} x {M}), FP64, all stages, cost matrix built outside the timing")
    return C, cells, text


def shard_reference_arm(args, spec):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import build_oracle, oracle
    build_oracle.build()
    threads = os.cpu_count() or 1
    C, cells, sample = _shard_cpu_sample(spec, threads, 2)
    times = []
    for s_ in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.parflex_full(C, spec.steps, spec.weights, spec.beta, spec.L, threads=threads)
        if s_ >= args.warmup:
            times.append(time.perf_counter() - t0)
    tot = sum(times)
    v = cells * len(times) / tot
    line = {
        "impl": "reference", "metric": SHARD_METRIC, "value": v, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(spec.describe(), parallelism="tiles"),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample + " per step"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def shard_arm(args, spec):
    """One long pair, its tiles sharded across the ranks (strong scaling):
    every rank builds the cost and runs stage 1 for its own tile range,
    rank 0 gathers the tile edges (NCCL) and runs stage 2, the crossed
    tiles' backpointers travel to rank 0.  Step time = max over ranks."""
    import torch
    import torch.distributed as dist

    from parflexdtw_b200 import _lib
    from parflexdtw_b200.shard import ShardedPair

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)
    lib = _lib.load()
    F1, F2 = W.make_pair(spec)  # the same pair on every rank
    N, M = F1.shape[1], F2.shape[1]
    cells, n1, n2 = tile_cells(N, M, spec.L)
    f1d, f2d = torch.from_numpy(F1).to(dev), torch.from_numpy(F2).to(dev)
    sp = ShardedPair(N, M, spec.steps, spec.weights, L=spec.L)
    ref = None
    for _ in range(args.warmup):
        ref = sp.run(spec.beta, f1d, f2d)

    def max_ranks(x):
        if ws == 1:
            return x
        t = torch.tensor([x], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    uuid = str(torch.cuda.get_device_properties(dev).uuid)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    local_ms = []
    launches0 = lib.pfx_kernel_launches()
    with ClockSampler(uuid) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            out = sp.run(spec.beta, f1d, f2d, events=True)
            local_ms.append(sp.local_ms())
            if rank == 0:
                assert out[0] == ref[0] and np.array_equal(out[1], ref[1]), "non-deterministic"
        e1.record()
        torch.cuda.synchronize()
    launches = lib.pfx_kernel_launches() - launches0
    ms_total = max_ranks(e0.elapsed_time(e1))
    cost_ms = max_ranks(sum(a for a, _ in local_ms) / args.steps)
    s1_ms = max_ranks(sum(b for _, b in local_ms) / args.steps)

    # e2e: pinned host features in, result out, every step
    f1p, f2p = torch.from_numpy(F1).pin_memory(), torch.from_numpy(F2).pin_memory()
    h2d = f1p.numel() * 8 + f2p.numel() * 8
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    d2h = 0
    for _ in range(args.e2e_steps):
        f1d.copy_(f1p, non_blocking=True)
        f2d.copy_(f2p, non_blocking=True)
        out = sp.run(spec.beta, f1d, f2d)
        if rank == 0:
            d2h = out[1].nbytes + 8
    b.record()
    torch.cuda.synchronize()
    e2e_ms = max_ranks(a.elapsed_time(b))
    own = sp.own_cells
    ex_bytes = sp.edge_exchange_bytes()
    sp.close()

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import build_oracle, oracle
        build_oracle.build()
        threads = os.cpu_count() or 1
        C, scells, sample = _shard_cpu_sample(spec, threads, 2)
        t0 = time.perf_counter()
        oracle.parflex_full(C, spec.steps, spec.weights, spec.beta, spec.L, threads=threads)
        dt = time.perf_counter() - t0
        cpu = {"value": scells / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": sample, "seconds": dt}
        del C
    if rank == 0:
        peak, peak_kind = load_peaks()
        achieved = own * 8.25 / (s1_ms / 1e3) / 1e9
        line = {
            "metric": SHARD_METRIC, "value": cells * args.steps / (ms_total / 1e3), "unit": UNIT,
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_total / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(spec.describe(), N=N, M=M, tiles=n1 * n2, cells_per_step=cells,
                           parallelism=f"tiles over {ws} rank(s)",
                           input="features resident in HBM; every step builds the cost",
                           cost_build="each rank's cost kernel into its tile range's slabs",
                           cost_definition=("1 - sum_f a_f b_f with separately rounded FP64 "
                                            "products and sums"),
                           l2="cost slabs larger than L2 (no flush needed)"),
            "pairs_per_s": args.steps / (ms_total / 1e3),
            "per_rank": {"cost_ms_max": cost_ms, "stage1_ms_max": s1_ms,
                         "rank0_cells": own, "edge_exchange_bytes": ex_bytes},
            "roofline": {"bound": "hbm", "kernel": "k_stage1_v3 (rank 0's tile range)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback",
                         "alg_bytes_per_cell": 8.25},
            "cpu_baseline": cpu,
            "e2e": {"value": cells * args.e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "steps": args.e2e_steps, "ms_per_step": e2e_ms / args.e2e_steps,
                    "api": "ShardedPair.run from features copied from pinned host memory"},
            "gpu_launches": int(launches), "clocks": clk.summary(),
            "note": "N > 1 not measured on hardware here (one GPU per call)",
        }
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    # Python's cyclic garbage collector stays off while the arms run, so that
    # no collection pause lands inside a timed step; reference counting still
    # frees everything that is not in a cycle, and each timed region of the
    # learned-pruning arm starts after an explicit collection.
    gc.disable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="prune64", choices=sorted(W.WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--ref-tile-rows", type=int, default=0,
                    help="single-pair workloads: tile rows the reference arm times "
                         "(0 = the whole pair)")
    ap.add_argument("--ref-batch-cells", type=float, default=3e9,
                    help="batch workloads: tile cells of the leading pairs the CPU times")
    ap.add_argument("--pairs", type=int, default=None,
                    help="precision workload: run only the first PAIRS pairs")
    ap.add_argument("--plain-steps", type=int, default=1,
                    help="precision workload: timed steps of the FP64 plain form")
    ap.add_argument("--cerr-pairs", type=int, default=16,
                    help="precision workload: pairs whose full cost matrices are compared")
    ap.add_argument("--ref-pairs", type=int, default=8,
                    help="precision workload: pairs the CPU oracle times")
    ap.add_argument("--ref-rounds", type=int, default=8,
                    help="learned-pruning workload: tiles per host thread in the CPU sample")
    ap.add_argument("--cpu-repeats", type=int, default=3,
                    help="learned-pruning workload: timed runs of the CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--warps", type=int, default=0, choices=[0, 4, 8, 16],
                    help="learned-pruning workloads: stage-1 warps per tile CTA (0: chosen "
                         "from the tile count)")
    ap.add_argument("--cost-def", default="fma", choices=["fma", "det"],
                    help="learned-pruning workloads: the FP64 cost of both forms as a "
                         "fixed-order FMA chain (fma) or as separately rounded products and "
                         "sums (det, the drop-in path's definition)")
    ap.add_argument("--cost", default="slabs", choices=["slabs", "tile"],
                    help="FP64 batches: build the cost with separate cost kernels into "
                         "slabs, in waves (slabs), or inside the stage-1 kernel, tile by tile, "
                         "in one launch (tile)")
    args = ap.parse_args()
    spec = W.WORKLOADS[args.workload]
    if isinstance(spec, W.ShardSpec):
        (shard_reference_arm if args.impl == "reference" else shard_arm)(args, spec)
        return
    if isinstance(spec, W.PruneSpec):
        (prune_reference_arm if args.impl == "reference" else prune_arm)(args, spec)
        return
    if isinstance(spec, W.PrecisionSpec):
        (precision_reference_arm if args.impl == "reference" else precision_arm)(args, spec)
        return
    batch = isinstance(spec, W.BatchSpec)
    if args.impl == "reference":
        (batch_reference_arm if batch else reference_arm)(args, spec)
    else:
        (batch_arm if batch else b200_arm)(args, spec)


if __name__ == "__main__":
    main()
