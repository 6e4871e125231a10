#!/usr/bin/env python3
"""Benchmark of the DynaMOSP update path on one B200 (or N replicas).

Workload (the road-network configuration): a 1404 x 1404 grid whose edges
are kept with p = 0.70, 1% of the vertices with one diagonal shortcut, the
largest connected component (~1.9M vertices, ~5.4M directed edges); K = 3
objectives with weights U[1,100] (seed 12345); source 0; Pref = (1,1,1);
50,000 changes, 50% insertions, connectivity-safe deletions (seed 777, the
reference generator's uniform mode). Synthetic stand-in for SuiteSparse
roadNet-CA, which is not available here.

One step = one MOSP update: the K SOSP updates (one fused persistent launch)
plus Steps 2-3 (combined graph + its SSSP, a second launch) - the region the
reference reports as gpu_compute_ms. Metric: changed edges (applied inserts
+ deletes) per second of that region. `value` has inputs resident in HBM
(each step restores the initial trees on the device and flushes L2 before its
timed region); `e2e` runs the same update through mosp_update_host with host
buffers (batch application, upload, GPU work, path costs and download inside
the timed region).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload road|powerlaw|batched|serving]

`--workload powerlaw` runs the same measurement on the power-law update
(R-MAT scale 22, edge factor 16, K = 5, log-uniform weights in [1, 10^6],
Pref = (1..5), 100,000 changes aimed at tree edges): the distance-only
fallback with lowest-id parent recovery.

Under torchrun every rank runs the same workload on its own GPU (replicas:
one update does not shard); value = all ranks' changed edges / the slowest
rank's time.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mosp-cuda_b200"))

METRIC = "MOSP update changed-edges/s (K SOSP updates + combined graph + its SSSP)"
UNIT = "changed-edges/s"
WORKLOAD = ("road-network shape: 1404x1404 grid, edges kept p=0.70, 1% diagonal shortcuts, largest "
            "component; K=3 weights U[1,100] seed 12345; source 0; Pref=(1,1,1); 50,000 changes, 50% "
            "insertions, connectivity-safe deletions, seed 777")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--width", type=int, default=1404)
    ap.add_argument("--changes", type=int, default=50000)
    ap.add_argument("--delta", type=int, default=0, help="fixed near-far width (0: default heuristic)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--loop", choices=["auto", "async", "bulk"], default="auto",
                    help="near-far loop of the persistent launches: auto = the autotuner's choice "
                         "(results are the same)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the baselines: the CPU port and the reference's GPU binary")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="skip the reference's GPU binary (oracle/_ref/mosp_ref) beside the CPU baseline")
    ap.add_argument("--verify", action="store_true", help="check the result against the oracle")
    ap.add_argument("--requests", type=int, default=400, help="serving workload: requests per arrival rate")
    ap.add_argument("--rates", default="50,200,1000", help="serving workload: Poisson arrival rates (1/s)")
    ap.add_argument("--workload", choices=["road", "powerlaw", "batched", "serving", "step1"], default="road",
                    help="road: the road-network update (default); powerlaw: the R-MAT scale-22 update with the "
                         "distance-only fallback; batched: 256 grid-road instances in one launch against "
                         "per-instance launches; serving: the resident-graph request loop")
    ap.add_argument("--instances", type=int, default=256, help="batched workload: number of instances")
    ap.add_argument("--rmat-scale", type=int, default=22,
                    help="powerlaw workload: R-MAT scale (22 is the configuration; smaller sizes are for "
                         "profiling captures)")
    ap.add_argument("--rmat-wmax", type=int, default=1_000_000,
                    help="powerlaw workload: largest weight (10^6 is the configuration; a smaller graph needs "
                         "larger weights to take the distance-only fallback)")
    return ap.parse_args()


POWERLAW = ("power-law shape: R-MAT scale 22, edge factor 16, a=0.57 b=0.19 c=0.19, symmetrised, no self-loops "
            "or duplicates; K=5 weights log-uniform in [1,1e6] seed 12345 (distance-only fallback with lowest-id "
            "parent recovery); source 0; Pref=(1,2,3,4,5); 100,000 changes, 30% insertions, 70% deletions aimed "
            "at tree edges (targeted mode, not connectivity-safe), seed 777")


def make_workload(args):
    """(graph, batch, K, Pref or None, description) of the workload."""
    import mosp_b200 as mb
    if getattr(args, "workload", "road") == "powerlaw":
        scale = getattr(args, "rmat_scale", 22)
        wmax = getattr(args, "rmat_wmax", 1_000_000)
        g = mb.HostGraph.rmat(scale, 16, 0.57, 0.19, 0.19, 5, 1, wmax, True, 12345)
        batch = mb.HostBatch.generate(g, 100000, 30.0, "targeted", 0, False, 777, 0, 1, wmax)
        desc = POWERLAW
        if scale != 22 or wmax != 1_000_000:
            desc = desc.replace("R-MAT scale 22", f"R-MAT scale {scale}").replace("[1,1e6]", f"[1,{wmax}]")
        return g, batch, 5, [1, 2, 3, 4, 5], desc
    g = mb.HostGraph.grid_road(args.width, args.width, 0.70, 0.01, 3, 1, 100, 12345)
    batch = mb.HostBatch.generate(g, args.changes, 50.0, "uniform", 0, True, 777, 0, 1, 100)
    return g, batch, 3, None, WORKLOAD


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.path = None
        self.device_index = device_index
        if shutil.which("nvidia-smi") is None:
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                      "-i", str(device_index), "-lms", "200"], stdout=open(self.path, "w"),
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x, pg, device):
    """The largest of every rank's x (every rank calls it in the same
    order); x itself without a process group."""
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(units_per_rank, steps, local_total_ms, world, pg, device):
    """Replicas: every rank processes units_per_rank per step; the job's
    time is the slowest rank's. Returns (units/s of the whole job, that
    time in ms)."""
    total_ms = max_over_ranks(local_total_ms, pg, device)
    return world * units_per_rank * steps / (total_ms / 1000.0), total_ms


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import datetime

    import torch
    import mosp_b200 as mb

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        pg = dist
    g, batch, K, pref, workload = make_workload(args)
    n, src = g.n, 0
    ws = mb.Workspace(timeout_ms=60000)
    ws.enable_timing(True)
    ws.set_async(args.loop != "bulk")
    row, col, w = g.arrays()
    # initial canonical trees of the original graph (GPU engine, from scratch)
    dg0 = mb.DeviceGraph.upload(ws, g)
    d0 = torch.empty((K, n), dtype=torch.int64, device="cuda")
    p0 = torch.empty((K, n), dtype=torch.int32, device="cuda")
    maxw_orig = [int(w[:, k].max()) for k in range(K)]
    for k in range(K):
        ws.sosp_from_scratch(n, g.m, dg0.out_row, dg0.out_col, dg0.out_w_col(k), src,
                             mb.default_delta(g.m, n, int(w[:, k].astype(np.int64).sum())), maxw_orig[k],
                             d0[k], p0[k])
    del dg0
    upd = mb.apply_batch(g, batch)
    ba = batch.arrays()
    changed = int(batch.n_ins + batch.n_del)
    dg = mb.DeviceGraph.upload(ws, upd)
    ch = mb.changed_lists(ba, K)
    cf = torch.from_numpy(np.concatenate([c[0] for c in ch])).cuda()
    ct = torch.from_numpy(np.concatenate([c[1] for c in ch])).cuda()
    off = np.concatenate([[0], np.cumsum([len(c[0]) for c in ch])])
    heads = torch.from_numpy(ba["ins_to"]).cuda()
    maxw = [max(maxw_orig[k], int(ba["ins_w"][:, k].max())) for k in range(K)]
    deltas = [args.delta if args.delta > 0 else mb.default_delta(g.m, n, int(w[:, k].astype(np.int64).sum()))
              for k in range(K)]
    dist_t = torch.empty_like(d0)
    par_t = torch.empty_like(p0)
    cd = torch.empty(n, dtype=torch.int64, device="cuda")
    cp = torch.empty(n, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def step(timed, widths):
        dist_t.copy_(d0)
        par_t.copy_(p0)
        flush.zero_()
        if timed:
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
        stats, cst = ws.update_device(n, upd.m, K, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w,
                                      cf, ct, off, heads, len(ba["ins_to"]), src, widths, maxw, pref, dist_t, par_t,
                                      cd, cp, stream=None)
        if timed:
            e.record(stream)
            e.synchronize()
            return s.elapsed_time(e), ws.last_timing(), stats, cst
        return None

    # widths: the default heuristic (timed for comparison) and the autotuner's
    # choice (the timed steps below), unless --delta fixes them
    for _ in range(max(args.warmup, 0)):
        step(False, deltas)
    default_ms = [step(True, deltas)[0] for _ in range(3)]
    comb_delta = 0
    if args.delta <= 0:
        dist_t.copy_(d0)
        par_t.copy_(p0)
        tuned, comb_delta, _, rounds = ws.autotune_update(n, upd.m, K, dg.out_row, dg.out_col, dg.out_w,
                                                          dg.in_row, dg.in_col, dg.in_w, cf, ct, off, heads,
                                                          len(ba["ins_to"]), src, deltas, maxw, pref, dist_t,
                                                          par_t, cd, cp)
        ws.set_combined_delta(comb_delta)
        ws.set_local_rounds(*rounds)
    else:
        tuned = deltas
        rounds = (0, 2)
    if args.loop != "auto":
        ws.set_async(args.loop == "async")
    grid_ctas, hub_edges, async_on = ws.tuning()
    for _ in range(max(args.warmup, 0)):
        step(False, tuned)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    clocks = ClockSampler(local)
    torch.cuda.synchronize()
    step_ms, upd_ms, comb_ms = [], [], []
    stats = cst = None
    wall0 = time.perf_counter()
    for _ in range(args.steps):
        ms, (um, cm), stats, cst = step(True, tuned)
        step_ms.append(ms)
        upd_ms.append(um)
        comb_ms.append(cm)
    torch.cuda.synchronize()
    wall = time.perf_counter() - wall0
    clock = clocks.stop()
    asy = ws.tuning()[2]
    phases = {"update": ws.last_phases(0), "combined": ws.last_phases(1),
              "update_loop": ws.loop_profile(0, asy), "combined_loop": ws.loop_profile(1, asy)}
    value, total_ms = replica_throughput(changed, args.steps, float(sum(step_ms)), world, pg, "cuda")
    if pg:
        pg.barrier()
    ms_per_step = total_ms / args.steps

    # roofline of the dominant kernel (the fused K-objective update)
    old_d, old_p = d0.cpu().numpy(), p0.cpu().numpy()
    new_d, new_p = dist_t.cpu().numpy(), par_t.cpu().numpy()
    ab = mb.algorithmic_bytes(upd, batch, K, src, old_d, old_p, new_d, new_p, cst.edges)
    restricted = None
    if any(s.packed_parents == 0 for s in stats):
        # the same steps with the input trees declared canonical (they are
        # the library's own): the distance-only objectives recover parents
        # only where the batch reaches; outputs compared with the steps above
        full = (dist_t.clone(), par_t.clone(), cd.clone(), cp.clone())
        engine_full = sum(phases["update"].values())
        ws.set_canonical_trees(True)
        for _ in range(max(args.warmup, 0)):
            step(False, tuned)
        r_ms, r_upd = [], []
        for _ in range(args.steps):
            ms, (um, _), _, _ = step(True, tuned)
            r_ms.append(ms)
            r_upd.append(um)
        engine_r = sum(ws.last_phases(0).values())
        ws.set_canonical_trees(False)
        same = all(torch.equal(a, b) for a, b in zip(full, (dist_t, par_t, cd, cp)))
        restricted = {"value": round(changed / (float(np.mean(r_ms)) / 1000.0), 1), "unit": UNIT,
                      "ms_per_step": round(float(np.mean(r_ms)), 4),
                      "update_ms": round(float(np.mean(r_upd)), 4),
                      "recovery_ms": round(float(np.mean(r_upd)) - engine_r, 4),
                      "full_recovery": {"update_ms": round(float(np.mean(upd_ms)), 4),
                                        "recovery_ms": round(float(np.mean(upd_ms)) - engine_full, 4)},
                      "equal_to_full_recovery": bool(same),
                      "what": "mosp_workspace_set_canonical_trees(ws, 1): the input trees are the library's "
                              "own, so the distance-only parents are recovered only at the vertices the "
                              "batch reaches (recovery_ms = update launch + recovery minus the engine's "
                              "phases)"}
    peak, peak_kind = measured_peak()
    upd_mean = float(np.mean(upd_ms))
    comb_mean = float(np.mean(comb_ms))
    achieved = ab["update"] / (upd_mean / 1000.0) / 1e9
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tfile) and workload == WORKLOAD:  # captured on the road workload
        try:
            traffic = json.load(open(tfile)).get("sosp_update_bytes_per_launch")
        except ValueError:
            traffic = None
    roofline = {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 5), "traffic": traffic,
                "kernel": f"sospEngine<update> (K={K} fused SOSP updates)"
                          + (" + recoverParents" if any(s.packed_parents == 0 for s in stats) else ""),
                "algorithmic_bytes_per_launch": ab["update"], "kernel_ms": round(upd_mean, 4),
                "peak_source": f"{peak_kind} hbm_gbs (MEASURED_PEAKS.json)" if peak_kind == "measured"
                else "fallback 6650 GB/s",
                "combined": {"kernel_ms": round(comb_mean, 4), "algorithmic_bytes_per_launch": ab["combined"],
                             "achieved_gbs": round(ab["combined"] / (comb_mean / 1000.0) / 1e9, 2)}}

    if args.verify:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        exp = orc.expected_update((row, col, w), ba, K, src, pref)
        assert np.array_equal(new_d, exp["dist"]) and np.array_equal(new_p, exp["parent"])
        assert np.array_equal(cd.cpu().numpy(), exp["comb_dist"]) and np.array_equal(cp.cpu().numpy(),
                                                                                      exp["comb_parent"])

    # end to end: host buffers through mosp_update_host
    e2e = None
    if args.e2e_steps > 0:
        # the same widths and local rounds as the device-resident steps, set
        # through the public API
        host_ws = mb.Workspace(timeout_ms=60000)
        host_ws.set_async(async_on)
        host_ws.set_grid(grid_ctas, hub_edges)
        host_ws.set_combined_delta(comb_delta)
        host_ws.set_local_rounds(*rounds)
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        garr = tuple(pin(x) for x in (row, col, w))
        barr = {k: pin(v) for k, v in ba.items() if k != "mask"}
        hd0, hp0 = pin(old_d), pin(old_p)
        KG = w.shape[1]
        outs = (pin(np.empty(K * n, np.int64)), pin(np.empty(K * n, np.int32)), pin(np.empty(n, np.int64)),
                pin(np.empty(n, np.int32)), pin(np.empty(n * KG, np.int64)))
        e2e_delta = tuned[0] if len(set(tuned)) == 1 else 0  # one width for all objectives
        host_ws.update_host(garr, barr, hd0, hp0, K, src, pref=pref, delta=e2e_delta, costs=True,
                            out=outs)  # warm-up
        times = []
        for _ in range(args.e2e_steps):
            t0 = time.perf_counter()
            _, _, _, _, _, tm = host_ws.update_host(garr, barr, hd0, hp0, K, src, pref=pref, delta=e2e_delta,
                                                    costs=True, out=outs)
            times.append(time.perf_counter() - t0)
        e2e_s = max_over_ranks(float(np.mean(times)), pg, "cuda")
        m_upd = upd.m
        # original graph, batch, initial trees and the per-objective change
        # lists in; mask, K trees, the combined tree and the costs out
        h2d = ((n + 1 + g.m) * 4 + g.m * KG * 4 + batch.n_ins * (2 + KG) * 4 + batch.n_del * 2 * 4 + K * n * 12
               + 2 * 4 * sum(len(c[0]) for c in ch))
        d2h = batch.n_ins * 4 + K * n * 12 + n * 12 + n * KG * 8
        e2e = {"value": round(world * changed / e2e_s, 1), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": round(e2e_s * 1000, 3),
               "path": "mosp_update_host (upload, GPU batch apply, GPU update + combined + costs, download)",
               "stages_ms": {k: round(getattr(tm, k), 3) for k in
                             ("apply_batch", "upload", "objectives", "combined", "costs", "download")}}
        host_ws.close()

    cpu = None
    ref_gpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_port(row, col, w, upd, ba, ch, old_d, old_p, K, src, changed, pref)
        if not args.no_reference_gpu:
            ref_gpu = reference_gpu_on(row, col, w, ba, [(old_d[k], old_p[k]) for k in range(K)], K, pref,
                                       changed, local)

    if rank == 0:
        line = {"metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
                "config": shared_config(workload, n, upd.m, K, changed, batch.n_ins, batch.n_del),
                "tuning": {"replicas": world, "delta": tuned, "combined_delta": comb_delta or "default",
                           "local_rounds": {"update": rounds[0], "combined": rounds[1]},
                           "delta_default": deltas,
                           "widths": "autotuned (mosp_autotune_update)" if args.delta <= 0 else "fixed by --delta",
                           "near_far_loop": ("asynchronous" if async_on else "bulk-synchronous")
                           + (" (autotuned)" if args.loop == "auto" else " (forced)"),
                           "grid_ctas": grid_ctas, "hub_row_edges": hub_edges},
                "gpu_compute_ms": round(ms_per_step, 4),
                "default_widths_ms_per_step": round(float(np.mean(default_ms)), 4),
                "roofline": roofline, "cpu_baseline": cpu, "reference_gpu": ref_gpu, "e2e": e2e,
                "restricted_recovery": restricted,
                # update + combined launches, plus the parent-recovery kernel
                # when an objective runs distance-only
                "gpu_launches": (2 + (1 if any(s.packed_parents == 0 for s in stats) else 0)) * args.steps,
                "clocks": clock, "wall_s_timed_loop": round(wall, 4), "phases_ms": phases,
                "stats": {"invalidated": [s.invalidated for s in stats], "iterations": [s.iterations for s in stats],
                          "epochs": [s.epochs for s in stats], "pushes": [s.pushes for s in stats],
                          "jump_rounds": stats[0].jump_rounds, "combined_edges": cst.edges,
                          "combined_iterations": cst.search.iterations, "expanded": ab["expanded"]}}
        print(json.dumps(line), flush=True)
    ws.close()
    if pg:
        pg.destroy_process_group()


def cpu_baseline_port(row, col, w, upd, ba, ch, old_d, old_p, K, src, changed, pref=None):
    """The oracle's restatement of the reference CPU path (sequential update
    per objective, then the host combined graph + Dijkstra), one full
    update, one thread."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    urow, ucol, uw = upd.arrays()
    rrow, rcol, rw = orc.transpose(urow, ucol, uw)
    t0 = time.perf_counter()
    parents = []
    for k in range(K):
        d = old_d[k].copy()
        p = old_p[k].copy()
        n = len(urow) - 1
        lib = orc.olib()
        cf, ct = np.ascontiguousarray(ch[k][0]), np.ascontiguousarray(ch[k][1])
        heads = np.ascontiguousarray(ba["ins_to"], np.int32)
        lib.oracle_sequential_update(n, uw.shape[1], k, src, orc.P(urow), orc.P(ucol), orc.P(uw), orc.P(rrow),
                                     orc.P(rcol), orc.P(rw), len(cf), orc.P(cf), orc.P(ct), len(heads),
                                     orc.P(heads), orc.P(d), orc.P(p))
        parents.append(p)
    crow, ccol, cw = orc.combined_graph(np.stack(parents), len(urow) - 1, K, src, pref)
    orc.dijkstra(crow, ccol, cw, 0, src)
    secs = time.perf_counter() - t0
    return {"value": round(changed / secs, 1), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"one full MOSP update of the workload (K={K} sequential SOSP updates + host combined graph "
                      f"+ Dijkstra), compute only, {secs:.2f} s"}


REF_MOSP = os.path.join(ROOT, "oracle", "_ref", "mosp_ref")


def reference_gpu_on(row, col, w, batch, trees, K, pref, changed, device_index):
    """reference_gpu_leg on the library arm's workload (original graph, batch
    and initial trees written in the reference's formats to a temporary
    directory), beside the CPU baseline."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    if not orc.have_ref() or not os.path.exists(REF_MOSP):
        return {"unavailable": "oracle/_ref was not built (the reference sources were absent at build time)"}
    tmp = tempfile.mkdtemp(prefix="mosp_refgpu_")
    try:
        prefix, changes, init = write_reference_inputs(tmp, row, col, w, batch, trees)
        return reference_gpu_leg(prefix, changes, init, K, pref, changed, device_index=device_index)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def write_reference_inputs(tmp, row, col, w, batch, trees):
    """The workload as the reference's bin/mosp reads it (its own writers, from
    oracle/_ref/libref_cpu.so): <tmp>/graph/graphCsr{RowPtr,ColInd,Values}.txt,
    <tmp>/changes/{insert,delete}.txt and <tmp>/init/obj<k>/{distances
    Original,SSSPTreeOriginal}.txt for the K (distance, parent) trees.
    Returns (graph prefix, changes dir, init dir)."""
    import oracle as orc
    prefix = os.path.join(tmp, "graph", "graphCsr")
    changes, init = os.path.join(tmp, "changes"), os.path.join(tmp, "init")
    os.makedirs(os.path.dirname(prefix), exist_ok=True)
    os.makedirs(changes, exist_ok=True)
    orc.ref_write_csr(prefix, row, col, w)
    orc.ref_write_changes(os.path.join(changes, "insert.txt"), os.path.join(changes, "delete.txt"),
                          np.asarray(w).reshape(len(col), -1).shape[1], batch)
    for k, (d, p) in enumerate(trees):
        os.makedirs(os.path.join(init, f"obj{k}"), exist_ok=True)
        orc.ref_write_tree(os.path.join(init, f"obj{k}", "distancesOriginal.txt"),
                           os.path.join(init, f"obj{k}", "SSSPTreeOriginal.txt"), d, p)
    return prefix, changes, init


def reference_gpu_leg(prefix, changes, init, K, pref, changed, runs=5, device_index=0):
    """The reference's own GPU path on the same B200: its bin/mosp, built from
    its sources for sm_100a (oracle/_ref/mosp_ref), on the files of
    write_reference_inputs, with its default bucket width. One untimed run
    (which also writes the graph's binary cache), then `runs` runs, each its
    own process; the figure is the median of the `RESULT gpu_compute_ms=`
    each prints: the GPU work of the K SOSP updates plus the combined graph
    and its SSSP, the region the reference times (src/mosp.cu:411).
    Clocks are sampled over the runs."""
    import re
    if not os.path.exists(REF_MOSP):
        return {"unavailable": "oracle/_ref/mosp_ref was not built (the reference sources were absent at build time)"}
    cmd = [REF_MOSP, "--graph", prefix, "--changes", changes, "--init", init, "-k", str(K),
           "--cache", prefix + ".cache", "--no-output", "--quiet"]
    if pref is not None:
        cmd += ["--pref", ",".join(str(int(x)) for x in pref)]
    pat = re.compile(r"RESULT gpu_compute_ms=([0-9.]+) end_to_end_ms=([0-9.]+)")
    sampler = ClockSampler(device_index)
    compute, whole = [], []
    failure = None
    for i in range(runs + 1):
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
        except subprocess.TimeoutExpired:
            failure = "mosp_ref ran past 600 s"
            break
        found = pat.search(r.stdout)
        if r.returncode != 0 or found is None:
            tail = (r.stdout + r.stderr).strip().splitlines()[-1:] or [""]
            failure = f"mosp_ref exited {r.returncode}: {tail[0][:200]}"
            break
        if i > 0:
            compute.append(float(found.group(1)))
            whole.append(float(found.group(2)))
    clocks = sampler.stop()
    if failure is not None:
        return {"unavailable": failure}
    ms = float(np.median(compute))
    return {"value": round(changed / (ms / 1000.0), 1), "unit": UNIT, "gpu_compute_ms": round(ms, 3),
            "gpu_compute_ms_runs": compute, "end_to_end_ms_median": round(float(np.median(whole)), 1),
            "runs": len(compute), "clocks": clocks,
            "what": "the reference's bin/mosp built from its sources for sm_100a (oracle/_ref/mosp_ref), default "
                    "bucket width, --no-output; median RESULT gpu_compute_ms (K SOSP updates + combined graph + "
                    "its SSSP); end_to_end_ms includes reading the text inputs"}


# ---------------------------------------------------------------------------
# batched workload: many independent instances in one launch per step
# ---------------------------------------------------------------------------
BATCHED_METRIC = "batched MOSP updates: instances/s (K SOSP updates + combined graph + its SSSP per instance)"


def make_batched_workload(count):
    """Grid-road instances as in the road workload at log-uniform sizes in
    [1,000, 200,000] vertices (seeds 12345*1000+i); per instance a batch of
    1-10% of its edges, 50% insertions, mode drawn from uniform, targeted,
    increase, reweight (seeds 777*1000+i)."""
    import mosp_b200 as mb
    rng = np.random.default_rng(12345)
    modes = ["uniform", "targeted", "increase", "reweight"]
    out = []
    for i in range(count):
        target = float(np.exp(rng.uniform(np.log(1e3), np.log(2e5))))
        side = max(8, int(round(np.sqrt(target))))
        g = mb.HostGraph.grid_road(side, side, 0.70, 0.01, 3, 1, 100, 12345 * 1000 + i)
        mode = modes[int(rng.integers(0, 4))]
        changes = max(2, int(g.m * rng.uniform(0.01, 0.10)))
        try:
            b = mb.HostBatch.generate(g, changes, 50.0, mode, 0, False, 777 * 1000 + i, 0, 1, 100)
        except mb.MospError:
            mode = "uniform"
            b = mb.HostBatch.generate(g, changes, 50.0, mode, 0, False, 777 * 1000 + i, 0, 1, 100)
        out.append((g, b, mode))
    return out


def run_batched(args):
    import torch
    import mosp_b200 as mb
    from mosp_b200 import batched as bt

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    K = 3
    insts = make_batched_workload(args.instances)
    garrs = [g.arrays() for g, _, _ in insts]
    bas = [b.arrays() for _, b, _ in insts]
    row, col, w, off = bt.union_graphs(garrs)
    ub = bt.union_batches(bas, off)
    roots = off[:-1].astype(np.int32)
    ug = mb.HostGraph.from_arrays(row, col, w)
    ubatch = mb.HostBatch.from_arrays(K, ub["ins_from"], ub["ins_to"], ub["ins_w"], ub["del_from"], ub["del_to"])
    upd = mb.apply_batch(ug, ubatch)
    uba = ubatch.arrays()
    N, M = upd.n, upd.m
    changed = int(ubatch.n_ins + ubatch.n_del)

    ws = mb.Workspace(timeout_ms=60000)
    ws.set_sources(roots)
    # initial trees of every instance: one from-scratch launch per objective
    dg0 = mb.DeviceGraph.upload(ws, ug)
    d0 = torch.empty((K, N), dtype=torch.int64, device="cuda")
    p0 = torch.empty((K, N), dtype=torch.int32, device="cuda")
    for k in range(K):
        ws.sosp_from_scratch(N, ug.m, dg0.out_row, dg0.out_col, dg0.out_w_col(k), int(roots[0]),
                             mb.default_delta(ug.m, N, int(w[:, k].sum())), int(w[:, k].max()), d0[k], p0[k])
    del dg0
    dg = mb.DeviceGraph.upload(ws, upd)
    ch = mb.changed_lists(uba, K)
    cf = torch.from_numpy(np.concatenate([c[0] for c in ch])).cuda()
    ct = torch.from_numpy(np.concatenate([c[1] for c in ch])).cuda()
    coff = np.concatenate([[0], np.cumsum([len(c[0]) for c in ch])])
    heads = torch.from_numpy(uba["ins_to"].astype(np.int32)).cuda()
    maxw = [max(int(w[:, k].max()), int(uba["ins_w"][:, k].max())) for k in range(K)]
    base_deltas = [mb.default_delta(ug.m, N, int(w[:, k].sum())) for k in range(K)]
    dist_t, par_t = torch.empty_like(d0), torch.empty_like(p0)
    cd = torch.empty(N, dtype=torch.int64, device="cuda")
    cp = torch.empty(N, dtype=torch.int32, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()
    def default_step():
        ws.update_device(N, M, K, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w, cf, ct, coff,
                         heads, len(uba["ins_to"]), int(roots[0]), base_deltas, maxw, None, dist_t, par_t, cd, cp,
                         want_stats=False)

    dist_t.copy_(d0)
    par_t.copy_(p0)
    tuned, comb_delta, tuned_ms, rounds = ws.autotune_update(N, M, K, dg.out_row, dg.out_col, dg.out_w,
                                                             dg.in_row, dg.in_col, dg.in_w, cf, ct, coff, heads,
                                                             len(uba["ins_to"]), int(roots[0]), base_deltas, maxw,
                                                             None, dist_t, par_t, cd, cp)

    def batched_step():
        ws.update_device(N, M, K, dg.out_row, dg.out_col, dg.out_w, dg.in_row, dg.in_col, dg.in_w, cf, ct, coff,
                         heads, len(uba["ins_to"]), int(roots[0]), tuned, maxw, None, dist_t, par_t, cd, cp,
                         want_stats=False)

    # the plain form: one mosp_update_device per instance on its own graph
    pws = mb.Workspace(timeout_ms=60000)
    plain = []
    for i, (g, b, _) in enumerate(insts):
        ga, ba_i = garrs[i], bas[i]
        u_i = mb.apply_batch(g, b)
        ba_i = b.arrays()
        dgi = mb.DeviceGraph.upload(pws, u_i)
        chi = mb.changed_lists(ba_i, K)
        cfi = torch.from_numpy(np.concatenate([c[0] for c in chi]).astype(np.int32)).cuda()
        cti = torch.from_numpy(np.concatenate([c[1] for c in chi]).astype(np.int32)).cuda()
        offi = np.concatenate([[0], np.cumsum([len(c[0]) for c in chi])])
        hi = torch.from_numpy(ba_i["ins_to"].astype(np.int32)).cuda() if len(ba_i["ins_to"]) else \
            torch.zeros(1, dtype=torch.int32, device="cuda")
        mwi = [max(int(ga[2][:, k].max()), int(ba_i["ins_w"][:, k].max()) if len(ba_i["ins_w"]) else 1)
               for k in range(K)]
        dli = [mb.default_delta(g.m, g.n, int(ga[2][:, k].sum())) for k in range(K)]
        lo, hi_ = int(off[i]), int(off[i + 1])
        d0i = d0[:, lo:hi_].clone()
        p0i = torch.where(p0[:, lo:hi_] >= 0, p0[:, lo:hi_] - lo, p0[:, lo:hi_]).contiguous()
        plain.append(dict(n=u_i.n, m=u_i.m, dg=dgi, cf=cfi, ct=cti, off=offi, heads=hi, nh=len(ba_i["ins_to"]),
                          maxw=mwi, deltas=dli, d0=d0i, p0=p0i, d=torch.empty_like(d0i), p=torch.empty_like(p0i),
                          cd=torch.empty(u_i.n, dtype=torch.int64, device="cuda"),
                          cp=torch.empty(u_i.n, dtype=torch.int32, device="cuda")))

    def plain_step():
        for x in plain:
            dg_i = x["dg"]
            pws.update_device(x["n"], x["m"], K, dg_i.out_row, dg_i.out_col, dg_i.out_w, dg_i.in_row, dg_i.in_col,
                              dg_i.in_w, x["cf"], x["ct"], x["off"], x["heads"], x["nh"], 0, x["deltas"], x["maxw"],
                              None, x["d"], x["p"], x["cd"], x["cp"], want_stats=False)

    def restore(fn):
        # each form restores only its own trees, so both results survive
        if fn is plain_step:
            for x in plain:
                x["d"].copy_(x["d0"])
                x["p"].copy_(x["p0"])
        else:
            dist_t.copy_(d0)
            par_t.copy_(p0)
        flush.zero_()

    def timed(fn):
        restore(fn)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        fn()
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e)

    # the batched form with the default widths and eager launches, then with
    # the tuned widths replayed as a CUDA graph
    for _ in range(max(args.warmup, 0)):
        timed(default_step)
    def_ms = [timed(default_step) for _ in range(max(1, min(args.steps, 3)))]
    ws.set_combined_delta(comb_delta)
    ws.set_local_rounds(*rounds)
    ws.use_graphs(True)
    for _ in range(max(args.warmup, 0)):
        timed(batched_step)
        timed(plain_step)
    clocks = ClockSampler(local)
    bt_ms = [timed(batched_step) for _ in range(args.steps)]
    pl_ms = [timed(plain_step) for _ in range(max(1, min(args.steps, 3)))]
    clock = clocks.stop()
    # the batched results equal the per-instance ones, instance by instance
    same = True
    dd, pp, cdd, cpp = dist_t.cpu().numpy(), par_t.cpu().numpy(), cd.cpu().numpy(), cp.cpu().numpy()
    for i, x in enumerate(plain):
        same &= np.array_equal(bt.split_vertices(dd, off, i), x["d"].cpu().numpy())
        same &= np.array_equal(bt.split_vertices(pp, off, i, parents=True), x["p"].cpu().numpy())
        same &= np.array_equal(bt.split_vertices(cdd, off, i), x["cd"].cpu().numpy())
        same &= np.array_equal(bt.split_vertices(cpp, off, i, parents=True), x["cp"].cpu().numpy())
    b_ms, p_ms = float(np.mean(bt_ms)), float(np.mean(pl_ms))
    if rank == 0:
        line = {"metric": BATCHED_METRIC, "value": round(len(insts) / (b_ms / 1000.0), 2), "unit": "instances/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(b_ms, 4),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                "data": "synthetic",
                "config": {"workload": f"{len(insts)} grid-road instances, n log-uniform in [1e3, 2e5], K=3 "
                                       "U[1,100], per-instance batches of 1-10% of the edges, 50% insertions, "
                                       "modes uniform/targeted/increase/reweight",
                           "instances": len(insts), "vertices": N, "edges": M, "changes_applied": changed,
                           "modes": {mname: sum(1 for _, _, mm in insts if mm == mname)
                                     for mname in ("uniform", "targeted", "increase", "reweight")},
                           "delta_default": base_deltas, "delta_tuned": tuned, "combined_delta_tuned": comb_delta,
                           "local_rounds_tuned": {"update": rounds[0], "combined": rounds[1]},
                           "cuda_graph": True, "l2": "flushed (256 MiB write) before every timed step"},
                "plain": {"value": round(len(insts) / (p_ms / 1000.0), 2), "unit": "instances/s",
                          "ms_per_step": round(p_ms, 3), "steps": len(pl_ms),
                          "form": "one mosp_update_device per instance (default widths), sequential"},
                "batched_default_widths_ms": round(float(np.mean(def_ms)), 4),
                "speedup_vs_plain": round(p_ms / b_ms, 2), "results_equal_plain": bool(same),
                "changed_edges_per_s": round(changed / (b_ms / 1000.0), 1),
                "gpu_launches": 2 * args.steps, "graph_launches": ws.graph_launches(), "clocks": clock}
        print(json.dumps(line), flush=True)
    ws.close()
    pws.close()


# ---------------------------------------------------------------------------
# serving workload: resident graphs, Poisson arrivals of change batches
# ---------------------------------------------------------------------------
SERVING_METRIC = "served MOSP updates: sustained changed-edges/s with p50/p99 latency (arrival -> result on host)"


def make_serving_graphs():
    """8 grid-road graphs of 0.5M-2M vertices and 8 R-MAT graphs of scale
    18-20 (edge factor 16), K = 4, weights U[1,1000] (seeds 12345*1000+i)."""
    import mosp_b200 as mb
    rng = np.random.default_rng(12345)
    graphs = []
    for i in range(8):
        side = int(round(np.sqrt(rng.uniform(0.5e6, 2.0e6) / 0.97)))
        graphs.append(("grid", mb.HostGraph.grid_road(side, side, 0.70, 0.01, 4, 1, 1000, 12345 * 1000 + i)))
    for i, scale in enumerate([18, 18, 18, 19, 19, 19, 20, 20]):
        graphs.append((f"rmat{scale}", mb.HostGraph.rmat(scale, 16, 0.57, 0.19, 0.19, 4, 1, 1000, False,
                                                        12345 * 1000 + 8 + i)))
    return graphs


def run_serving(args):
    import threading

    import mosp_b200 as mb

    world, rank, local = dist_setup(args)
    import torch
    torch.cuda.set_device(local)
    K, pref = 4, [1, 1, 2, 3]
    graphs = make_serving_graphs()
    garrs = [g.arrays() for _, g in graphs]
    rates = [float(x) for x in args.rates.split(",")]
    sources_of = [np.repeat(np.arange(len(r) - 1, dtype=np.int32), np.diff(r)) for r, _, _ in garrs]
    rng = np.random.default_rng(777)
    results = []
    for rate in rates:
        # the request stream: Poisson arrivals, a uniformly chosen graph,
        # batch size log-uniform in [100, 100000]; half the changes insert
        # random vertex pairs (weights U[1,1000]), half delete random edges
        # of the original graph (a deletion of an edge already gone is a
        # no-op)
        count = args.requests
        gaps = rng.exponential(1.0 / rate, count)
        targets = rng.integers(0, len(graphs), count)
        sizes = np.exp(rng.uniform(np.log(100), np.log(100000), count)).astype(int)
        reqs = []
        for j in range(count):
            row, col, _ = garrs[targets[j]]
            src = sources_of[targets[j]]
            n = len(row) - 1
            ni = int(sizes[j]) // 2
            nd = int(sizes[j]) - ni
            pick = rng.integers(0, len(col), nd)
            reqs.append((int(targets[j]), {
                "ins_from": rng.integers(0, n, ni).astype(np.int32), "ins_to": rng.integers(0, n, ni).astype(np.int32),
                "ins_w": rng.integers(1, 1001, (ni, K)).astype(np.int32),
                "del_from": src[pick].astype(np.int32), "del_to": col[pick].astype(np.int32)}))
        changes = sum(len(b["ins_from"]) + len(b["del_from"]) for _, b in reqs)

        def serve(workers, coalesce, paced):
            srv = mb.Server(workers=workers, reserve_bytes=4 << 30, max_coalesce=coalesce)
            ids = [srv.add_graph(ga, K, 0, pref) for ga in garrs]
            # warm-up, not timed: one empty batch per graph (every worker has
            # reserved its workspace for the largest graph by then)
            empty = {"ins_from": np.zeros(0, np.int32), "ins_to": np.zeros(0, np.int32),
                     "ins_w": np.zeros((0, K), np.int32), "del_from": np.zeros(0, np.int32),
                     "del_to": np.zeros(0, np.int32)}
            for gid in ids:
                srv.wait(srv.submit(gid, empty), gid, want_result=False)
            infos = [None] * count
            tickets = [None] * count
            ready = threading.Semaphore(0)

            def waiter():
                for j in range(count):
                    ready.acquire()
                    infos[j] = srv.wait(tickets[j], ids[reqs[j][0]], want_result=False)[2]

            th = threading.Thread(target=waiter)
            th.start()
            t0 = time.perf_counter()
            due = t0
            for j, (gi, b) in enumerate(reqs):
                if paced:
                    due += gaps[j]
                    delay = due - time.perf_counter()
                    if delay > 0:
                        time.sleep(delay)
                tickets[j] = srv.submit(ids[gi], b)
                ready.release()
            th.join()
            wall = time.perf_counter() - t0
            st = srv.stats()
            srv.close()
            return infos, wall, st

        infos, wall, st = serve(workers=2, coalesce=64, paced=True)
        # the plain form: one request per pass, one worker, same per-graph order
        plain, plain_wall, pst = serve(workers=1, coalesce=1, paced=False)
        plain_sum = {(targets[j], plain[j].version): plain[j].checksum for j in range(count)}
        equal = all(plain_sum.get((targets[j], infos[j].version)) == infos[j].checksum for j in range(count))
        lat = np.array([x.latency_us for x in infos]) / 1000.0
        queue = np.array([x.queue_us for x in infos]) / 1000.0
        results.append({"rate_per_s": rate, "requests": count, "changes": int(changes),
                        "p50_ms": round(float(np.percentile(lat, 50)), 3),
                        "p99_ms": round(float(np.percentile(lat, 99)), 3),
                        "mean_queue_ms": round(float(queue.mean()), 3),
                        "offered_s": round(float(gaps.sum()), 3), "wall_s": round(wall, 3),
                        "changed_edges_per_s": round(changes / wall, 1), "passes": st.passes,
                        "max_coalesced": st.max_coalesced, "deferred_admissions": st.deferred,
                        "pass_ms": {"apply": round(st.apply_us / 1000 / max(st.passes, 1), 3),
                                    "engine": round(st.engine_us / 1000 / max(st.passes, 1), 3),
                                    "result": round(st.result_us / 1000 / max(st.passes, 1), 3)},
                        "plain_wall_s": round(plain_wall, 3),
                        "plain_pass_ms": {"apply": round(pst.apply_us / 1000 / max(pst.passes, 1), 3),
                                          "engine": round(pst.engine_us / 1000 / max(pst.passes, 1), 3),
                                          "result": round(pst.result_us / 1000 / max(pst.passes, 1), 3)},
                        "all_equal_plain": bool(equal)})
    if rank == 0:
        top = results[-1]
        line = {"metric": SERVING_METRIC, "value": top["changed_edges_per_s"], "unit": "changed-edges/s",
                "n_gpus": world, "steps": args.requests, "warmup": 0,
                "ms_per_step": round(1000 * top["wall_s"] / top["requests"], 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
                "config": {"workload": "16 resident graphs (8 grid-road 0.5M-2M vertices, 8 R-MAT scale 18-20 ef16), "
                                       "K=4 U[1,1000], Pref=(1,1,2,3); Poisson arrivals, uniform graph choice, "
                                       "batches log-uniform in [100, 100000] changes, 50% insertions of random "
                                       "pairs, 50% deletions of random original edges",
                           "graphs": [{"kind": kind, "n": g.n, "m": g.m} for kind, g in graphs],
                           "workers": 2, "max_coalesce": 64, "reserve_bytes": 4 << 30},
                "rates": results}
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# reference arm: the reference's own CPU implementation of the path
# ---------------------------------------------------------------------------
def shared_config(workload, n, m, K, changed, n_ins, n_del):
    """The `config` of both arms (the same dict for the same workload)."""
    return {"workload": workload, "n": int(n), "m": int(m), "K": int(K), "changes_applied": int(changed),
            "inserts": int(n_ins), "deletes": int(n_del),
            "parallelism": "one process per GPU (replicas); the reference arm: one host thread per call",
            "l2": "library arm: L2 flushed (256 MiB write) before every timed step; reference arm: host only"}


def reference_workload(args):
    """The library arm's workload built from oracle/ alone: the seeded graph
    from oracle/_gen/libworkload.so (the same generator, compiled without the
    library) and the change batch from the reference's own generateChangeBatch
    (oracle/_ref/libref_cpu.so), which the library's generator equals byte for
    byte. Returns (row, col, w, batch dict, K, pref, description)."""
    import oracle as orc
    if getattr(args, "workload", "road") == "powerlaw":
        scale = getattr(args, "rmat_scale", 22)
        wmax = getattr(args, "rmat_wmax", 1_000_000)
        row, col, w = orc.workload_rmat(scale, 16, 0.57, 0.19, 0.19, 5, 1, wmax, True, 12345)
        batch = orc.ref_generate_changes(row, col, w, 100000, 30.0, 1, 0, False, 777, 0, 1, wmax)
        desc = POWERLAW
        if scale != 22 or wmax != 1_000_000:
            desc = desc.replace("R-MAT scale 22", f"R-MAT scale {scale}").replace("[1,1e6]", f"[1,{wmax}]")
        return row, col, w, batch, 5, [1, 2, 3, 4, 5], desc
    row, col, w = orc.workload_grid_road(args.width, args.width, 0.70, 0.01, 3, 1, 100, 12345)
    batch = orc.ref_generate_changes(row, col, w, args.changes, 50.0, 0, 0, True, 777, 0, 1, 100)
    return row, col, w, batch, 3, None, WORKLOAD


def run_reference(args):
    """The reference's CPU path on the library arm's workload, on the host
    cores: per objective the reference's sequentialSOSPUpdate through its own
    file API (text graph, batch and tree in, tree out), the K objectives one
    after another as the reference runs them, then the reference's
    combinedGraphReference + dijkstraCsrGraph on the K trees it wrote. Only
    oracle/ libraries are loaded (the reference compiled from its sources,
    and the workload generator); none of the library's code runs.

    A step is a bounded sample: one objective's update (objective = step mod
    K), so that W + K steps end within minutes; the combined step is timed
    once after them. value = changed edges / (K x mean objective time +
    combined time). The compute-only figures come from the same source
    compiled with two clock reads around its Phases 1-2."""
    world, rank, _ = dist_setup(args)
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    if not orc.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (the reference sources "
                                                              "were absent at build time)"}), flush=True)
        return
    row, col, w, batch, K, pref, workload = reference_workload(args)
    n, src = len(row) - 1, 0
    n_ins, n_del = len(batch["ins_from"]), len(batch["del_from"])
    changed = n_ins + n_del
    urow, ucol, _, _ = orc.ref_apply_batch(row, col, w, batch["ins_from"], batch["ins_to"], batch["ins_w"],
                                           batch["del_from"], batch["del_to"])
    m_upd = len(ucol)
    tmp = tempfile.mkdtemp(prefix="mosp_ref_")
    try:
        trees = [orc.ref_dijkstra(row, col, w, k, src) for k in range(K)]
        prefix, changes, init = write_reference_inputs(tmp, row, col, w, batch, trees)
        ins, dele = os.path.join(changes, "insert.txt"), os.path.join(changes, "delete.txt")

        def objective(k):
            t0 = time.perf_counter()
            ok, compute = orc.ref_sequential_update_timed(prefix,
                                                          os.path.join(init, f"obj{k}", "distancesOriginal.txt"),
                                                          os.path.join(init, f"obj{k}", "SSSPTreeOriginal.txt"),
                                                          ins, dele, k, src, os.path.join(tmp, f"od{k}.txt"),
                                                          os.path.join(tmp, f"ot{k}.txt"))
            whole = time.perf_counter() - t0
            if not ok:
                raise RuntimeError(f"the reference's sequentialSOSPUpdate failed on objective {k}")
            return whole, compute

        for i in range(max(args.warmup, 0)):
            objective(i % K)
        whole, compute = [], []
        for i in range(max(args.steps, 1)):
            a, b = objective(i % K)
            whole.append(a)
            compute.append(b)
        for k in range(K):  # every objective's output tree exists
            if not os.path.exists(os.path.join(tmp, f"ot{k}.txt")):
                objective(k)
        t0 = time.perf_counter()
        parents = np.stack([orc.ref_read_parents(os.path.join(tmp, f"ot{k}.txt"), n) for k in range(K)])
        t1 = time.perf_counter()
        orc.ref_combined_dijkstra(parents, n, K, src, pref)
        t2 = time.perf_counter()
        comb_whole, comb_compute = t2 - t0, t2 - t1
        per_update = K * float(np.mean(whole)) + comb_whole
        per_update_compute = K * float(np.mean(compute)) + comb_compute
        value = changed / per_update

        # labelled variant, not the reference's behaviour: the K objectives
        # in K threads at once (one update, after the timed steps)
        from concurrent.futures import ThreadPoolExecutor
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=K) as pool:
            list(pool.map(objective, range(K)))
        threaded = time.perf_counter() - t0 + comb_whole

        ref_gpu = None if getattr(args, "no_reference_gpu", False) else reference_gpu_leg(prefix, changes, init, K, pref, changed)

        cores = os.cpu_count() or 1
        sample = (f"one objective's reference sequentialSOSPUpdate per step (file API: text graph, batch and tree "
                  f"read, batch applied, update, tree written; objective = step mod {K}), then once the "
                  f"reference's combinedGraphReference + dijkstraCsrGraph on the {K} written trees; one host "
                  f"thread ({cores} cores on the host); value = changed edges / ({K} x mean step + combined)")
        line = {"metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": len(whole),
                "warmup": max(args.warmup, 0), "ms_per_step": round(1000 * float(np.mean(whole)), 2),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
                "data": "synthetic", "impl": "reference",
                "config": shared_config(workload, n, m_upd, K, changed, n_ins, n_del),
                "cpu_baseline": {"value": round(value, 2), "unit": UNIT, "cores": 1, "kind": "reference",
                                 "sample": sample},
                "e2e": {"value": round(value, 2), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "per_update_s": {"file_api": round(per_update, 3), "compute_only": round(per_update_compute, 3),
                                 "objective_file_api": round(float(np.mean(whole)), 3),
                                 "objective_compute_only": round(float(np.mean(compute)), 3),
                                 "combined_file_api": round(comb_whole, 3), "combined_compute": round(comb_compute, 3)},
                "compute_only": {"value": round(changed / per_update_compute, 2), "unit": UNIT,
                                 "what": "the reference's Phases 1-2 per objective (clock reads in a second copy of "
                                         "its source) + combinedGraphReference + dijkstraCsrGraph"},
                "threaded_variant": {"value": round(changed / threaded, 2), "unit": UNIT, "threads": K,
                                     "what": f"not the reference's behaviour: the {K} objectives in {K} threads at "
                                             "once, file API, plus the combined step"},
                "reference_gpu": ref_gpu,
                "host": {"cores": cores}}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def run_step1(args):
    """Step 1 alone (mosp_apply_batch_device: the road workload's batch
    applied to its graph on the GPU), `steps` timed calls after `warmup`:
    the driver of the Step 1 profile captures."""
    import torch
    import mosp_b200 as mb
    g, batch, K, _, workload = make_workload(args)
    ws = mb.Workspace(timeout_ms=60000)
    row, col, w = g.arrays()
    ba = batch.arrays()
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    drow, dcol, dw = t(row), t(col), t(w.reshape(-1))
    ifr, ito, iw = t(ba["ins_from"]), t(ba["ins_to"]), t(ba["ins_w"].reshape(-1))
    dfr, dto = t(ba["del_from"]), t(ba["del_to"])
    cap = g.m + batch.n_ins
    nrow = torch.empty(g.n + 1, dtype=torch.int32, device="cuda")
    ncol = torch.empty(cap, dtype=torch.int32, device="cuda")
    nw = torch.empty(cap * K, dtype=torch.int32, device="cuda")
    mask = torch.empty(max(batch.n_ins, 1), dtype=torch.int32, device="cuda")
    times = []
    for i in range(max(args.warmup, 0) + max(args.steps, 1)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ws.apply_batch_device(g.n, K, g.m, drow, dcol, dw, ifr, ito, iw, dfr, dto, nrow, ncol, nw, mask)
        torch.cuda.synchronize()
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    ms = 1000 * float(np.mean(times))
    print(json.dumps({"metric": "Step 1 (batch application on the GPU) ms", "value": round(ms, 4), "unit": "ms",
                      "higher_is_better": False, "steps": len(times), "warmup": args.warmup,
                      "config": {"workload": workload, "n": g.n, "m": g.m,
                                 "changes": int(batch.n_ins + batch.n_del)}}), flush=True)
    ws.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "step1":
        run_step1(args)
    elif args.workload == "batched":
        run_batched(args)
    elif args.workload == "serving":
        run_serving(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
