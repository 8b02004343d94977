#!/usr/bin/env python3
"""Perft throughput benchmark (leaf nodes/s, bit-exact) on B200.

Default workload: the batched perft of 4096 seeded, stratified playout
positions at depths U[4,6] (one step = one perft_batch over the whole
batch).  Other workloads: --workload start (initial position, depth 5,
repeated), --workload deep (one 20-ply playout with >= 35 moves, depth 8).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): each rank searches its own 4096-position batch (seed
offset by rank); there is no data-path collective, only a barrier and a
max/sum reduction of the timings and counts.

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "perft leaf nodes/s (bit-exact)"
UNIT = "leaf nodes/s"


# ------------------------------------------------------------------ helpers
def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """Samples nvidia-smi clocks/throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(s[1]) for s in self.samples if num(s[1]) is not None]
        mx = [num(s[2]) for s in self.samples if num(s[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if s[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def load_work_figures():
    with open(os.path.join(ROOT, "perft_gpu_b200", "work_figures.json")) as f:
        return json.load(f)["workloads"]


def int32_peak(device):
    """Measured integer-pipe peak (ops/s) from libperft_probe.so."""
    lib = ctypes.CDLL(os.path.join(ROOT, "perft_gpu_b200", "libperft_probe.so"))
    out = (ctypes.c_double * 7)()
    if lib.perft_int32_peak_probe(device, out) != 0:
        return None
    return {"lop3": out[0], "iadd": out[1], "lop3_iadd_shf": out[2], "imad": out[3], "lop3_imad": out[4],
            "imad_hi": out[5], "imad_wide_lop3": out[6]}


def traffic_from_profiles(workload, items_per_launch):
    """DRAM bytes per leaf launch: the ncu-measured bytes per item of a
    captured launch (profiles/leaf_kernel_traffic.json) scaled to this run's
    items per launch (traffic grows with the items processed)."""
    path = os.path.join(ROOT, "profiles", "leaf_kernel_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    per_item = d.get(workload, {}).get("dram_bytes_per_item")
    return per_item * items_per_launch if per_item is not None else None


# ------------------------------------------------------------------ workloads
def make_workload(name, rank, positions=4096):
    from perft_gpu_b200 import workloads as W
    if name == "batch":
        pos, depths = W.batch_positions(n=4096, seed=2026 + rank)
        pos, depths = pos[:positions], depths[:positions]
        cfg = {"workload": f"batch{positions}: {positions} seeded playouts of 8-30 plies, stratified "
                           "(>=10% en passant, >=10% pawn on 7th, >=10% castling), depth U[4,6]",
               "positions": positions, "depths": "U[4,6]", "seed": 2026 + rank}
        return pos, depths, cfg, "batch4096"
    if name == "start":
        pos = np.repeat(W.start_position().reshape(1, 6), 1, axis=0)
        cfg = {"workload": "initial position, depth 5, no transposition table", "positions": 1,
               "depths": "5"}
        return pos, np.array([5], dtype=np.uint8), cfg, "start"
    if name == "deep":
        pos = W.deep_position().reshape(1, 6)
        cfg = {"workload": "one seeded 20-ply playout with >=35 legal moves, depth 8, no TT",
               "positions": 1, "depths": "8"}
        return pos, np.array([8], dtype=np.uint8), cfg, "deep"
    raise SystemExit(f"unknown workload {name}")


# ------------------------------------------------------------------ CPU arms
def cpu_perft_lib():
    """The reference's host perft when it was built (oracle/_ref), else the oracle port."""
    ref = os.path.join(ROOT, "oracle", "_ref", "libperft_ref.so")
    if os.path.exists(ref):
        lib = ctypes.CDLL(ref)
        lib.ref_init()
        fn = lib.ref_perft_batch_mt
        return "reference", fn
    orc = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(orc)
    lib.oracle_init()
    return "port", lib.oracle_perft_batch_mt


def cpu_sample(pos, depths, budget_s, expected=None, threads=None):
    """Runs the CPU perft over a bounded sample of the workload: a seeded
    random order of its positions, taken in groups until budget_s elapses."""
    kind, fn = cpu_perft_lib()
    threads = threads or os.cpu_count() or 1
    order = np.random.default_rng(123).permutation(len(pos))
    done, leaves, t0 = 0, 0, time.perf_counter()
    mismatches = 0
    group = max(1, min(4, len(pos)))  # doubles up to 128: short budgets stop early
    while done < len(pos) and time.perf_counter() - t0 < budget_s:
        idx = order[done:done + group]
        p = np.ascontiguousarray(pos[idx], dtype=np.uint64)
        d = np.ascontiguousarray(depths[idx], dtype=np.uint32)
        out = np.zeros(len(idx), dtype=np.uint64)
        fn(ctypes.c_void_p(p.ctypes.data), ctypes.c_void_p(d.ctypes.data), ctypes.c_uint32(len(idx)),
           ctypes.c_int(threads), ctypes.c_void_p(out.ctypes.data))
        if expected is not None:
            mismatches += int(np.count_nonzero(out != expected[idx]))
        leaves += int(out.sum())
        done += len(idx)
        group = min(group * 2, 128)
    el = time.perf_counter() - t0
    return {"value": leaves / el, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{done} of {len(pos)} positions (seeded order) at their own depths, "
                      f"{leaves} leaves in {el:.1f} s",
            "mismatches_vs_gpu": mismatches if expected is not None else None}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    pos, depths, cfg, _ = make_workload(args.workload, 0, args.positions)
    vals = []
    for _ in range(args.warmup):
        cpu_sample(pos, depths, min(3.0, args.cpu_seconds))
    last = None
    for _ in range(args.steps):
        last = cpu_sample(pos, depths, args.cpu_seconds)
        vals.append(last["value"])
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "ms_per_step": None, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": last["cores"], "kind": last["kind"],
                             "sample": last["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def run_ours(args):
    import torch
    import perft_gpu_b200 as pg
    from perft_gpu_b200.shard import max_sum_over_ranks

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    pos, depths, cfg, wf_key = make_workload(args.workload, rank, args.positions)
    sliders = {"auto": pg.SLIDERS_AUTO, **{v: k for k, v in pg.SLIDER_NAMES.items()}}[args.sliders]
    pg.init(device=local, sliders_expand=sliders, sliders_leaf=sliders,
            arena_bytes=int(args.arena_gb * (1 << 30)))

    n = len(pos)
    d_pos = torch.from_numpy(pos.view(np.int64)).cuda()
    d_out = torch.zeros(n, dtype=torch.int64, device="cuda")

    if args.form == "single":
        # one position per call: the plain one-position-per-launch form
        elem = d_pos.element_size() * 6

        def step_device():
            for i in range(n):
                pg.perft_batch_device(d_pos.data_ptr() + i * elem, depths[i:i + 1], 1,
                                      d_out.data_ptr() + i * d_out.element_size())
    else:
        def step_device():
            pg.perft_batch_device(d_pos.data_ptr(), depths, n, d_out.data_ptr())

    for _ in range(args.warmup):
        step_device()
    counts = d_out.cpu().numpy().view(np.uint64).copy()
    leaves_per_step = int(counts.sum())

    # ---- device-resident timed region
    pg.reset_stats()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        start.record()
        for _ in range(args.steps):
            step_device()
        end.record()
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
    ms = start.elapsed_time(end)
    st = pg.stats()
    again = d_out.cpu().numpy().view(np.uint64)
    stable = bool(np.array_equal(again, counts))

    # ---- end to end through the host-buffer C ABI (H2D + D2H inside)
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    host_pos = np.ascontiguousarray(pos)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e_start.record()
    for _ in range(args.steps):
        if args.form == "single":
            host_out = np.array([pg.perft(host_pos[i], int(depths[i])) for i in range(n)], dtype=np.uint64)
        else:
            host_out = pg.perft_batch(host_pos, depths)
    e_end.record()
    torch.cuda.synchronize()
    e_ms = e_start.elapsed_time(e_end)
    stable = stable and bool(np.array_equal(host_out, counts))

    # ---- reductions over ranks: slowest rank's times, all ranks' leaves
    (ms_max, e_ms_max), (tot,) = max_sum_over_ranks([ms, e_ms], [leaves_per_step], device="cuda")
    total_leaves = tot * args.steps

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return 0

    value = total_leaves / (ms_max / 1e3)
    e2e_value = total_leaves / (e_ms_max / 1e3)

    # ---- roofline of the dominant kernel (count-only leaf tile kernel)
    wf = load_work_figures()[wf_key]
    peaks = int32_peak(local)
    launches = max(1, st["leaf_launches"])
    w_int = 2.0 * (st["leaf_items"] * (wf["c_make"] + wf["c_count"]) + st["leaf_parents"] * wf["c_gen"])
    leaf_s = st["leaf_ms"] / 1e3
    achieved = w_int / leaf_s if leaf_s > 0 else None
    peak = max(peaks.values()) if peaks else None
    roofline = {
        "bound": "int32",
        "kernel": "k_tile<MODE_LEAF> (count-only last ply)",
        "achieved": achieved / 1e12 if achieved else None,
        "peak": peak / 1e12 if peak else None,
        "unit": "Tops/s (32-bit integer ops, reference-algorithm work)",
        "frac": (achieved / peak) if (achieved and peak) else None,
        "peak_source": "of measured: best of the integer instruction mixes timed on this GPU by libperft_probe.so",
        "peak_variants_tops": {k: v / 1e12 for k, v in peaks.items()} if peaks else None,
        "traffic": traffic_from_profiles(wf_key, st["leaf_items"] / launches),
        "traffic_unit": "bytes per leaf launch (ncu bytes/item x items/launch)",
        "work_per_launch_ops": w_int / launches,
        "leaf_launch_ms_avg": st["leaf_ms"] / launches,
        "leaf_share_of_step": (st["leaf_ms"] / ms) if ms > 0 else None,
        "work_figures": {k: wf[k] for k in ("c_count", "c_make", "c_gen")},
    }

    cpu = None
    if ws == 1 and not args.no_cpu:
        cpu = cpu_sample(pos, depths, args.cpu_seconds, expected=counts)

    cfg = dict(cfg)
    cfg.update({"form": "one perft call per position" if args.form == "single" else "one batched call",
                "sliders": {"leaf": pg.SLIDER_NAMES.get(st["sliders_leaf"], "?"),
                            "interior": pg.SLIDER_NAMES.get(st["sliders_expand"], "?"),
                            "chosen_by": args.sliders},
                "l2": "no flush: each step streams multi-GB level buffers through HBM (>> 126 MB L2)",
                "parallelism": f"independent batches, {ws} GPU(s)"})
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": cfg,
        "leaves_per_step": int(tot), "counts_stable": stable,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(pos.nbytes),
                "d2h_bytes_per_step": int(8 * n)},
        "gpu_launches": int(st["leaf_launches"] + st["expand_launches"] + st["other_launches"]),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def run_tt(args):
    """Transposition-table workload: 4 seeded playouts of 12-24 plies at
    depths 9-10 with a 2^30-entry table; parity with the no-table engine is
    checked at depth 8 first."""
    import perft_gpu_b200 as pg
    from perft_gpu_b200 import workloads as W
    pos, depths = W.tt_positions()
    depths = np.minimum(depths, args.max_depth).astype(np.uint8)
    arena = int(args.arena_gb * (1 << 30))
    pd = args.parity_depth
    pg.init(device=0, arena_bytes=arena)
    t0 = time.perf_counter()
    d8_plain = pg.perft_batch(pos, pd)
    t_plain = time.perf_counter() - t0
    pg.init(device=0, arena_bytes=arena, tt_log2_entries=args.tt_log2)
    t0 = time.perf_counter()
    d8_tt = pg.perft_batch(pos, pd)
    t_tt8 = time.perf_counter() - t0
    times, counts = [], None
    for step in range(args.warmup + args.steps):
        pg.tt_clear()
        pg.reset_stats()
        t0 = time.perf_counter()
        counts = pg.perft_batch(pos, depths)
        el = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(el)
    st = pg.stats()
    leaves = int(counts.sum())
    line = {"metric": "perft leaf nodes/s with transposition table (effective, bit-exact)",
            "value": leaves / float(np.mean(times)), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True,
            "dtype": "u64", "data": "synthetic",
            "config": {"workload": "4 seeded playouts of 12-24 plies, TT of 2^%d x 16 B, table cleared each step"
                                   % args.tt_log2, "depths": depths.tolist()},
            "counts": [int(x) for x in counts],
            "parity_depth%d" % pd: {"equal": bool(np.array_equal(d8_plain, d8_tt)), "no_tt_s": t_plain,
                                    "tt_s": t_tt8, "counts": [int(x) for x in d8_plain]},
            "tt": {k: st[k] for k in ("tt_entries", "tt_probes", "tt_hits", "tt_duplicates", "tt_stores")},
            "timing": "host wall clock around the synchronous perft_batch call"}
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """Serving workload: Poisson arrivals of seeded 0-40-ply positions at
    depth U[3,7] through the continuous-batching server; p50/p99 latency is
    submit-to-completion wall time."""
    import perft_gpu_b200 as pg
    from perft_gpu_b200 import workloads as W
    pos, depths, arrivals = W.serving_trace(n=args.queries, rate_qps=args.rate, seed=5)
    pg.init(device=0)
    pg.serve_start(memory_bytes=int(args.serve_memory_gb * (1 << 30)), step_items=args.serve_step_items)
    tickets = [None] * len(pos)
    t_start = time.perf_counter()
    for i in range(len(pos)):
        delay = t_start + arrivals[i] - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        tickets[i] = pg.serve_submit(pos[i], int(depths[i]))
    lat, counts = np.zeros(len(pos)), np.zeros(len(pos), dtype=np.uint64)
    for i, t in enumerate(tickets):
        c, l = pg.serve_wait(t, timeout_s=3600)
        counts[i], lat[i] = c, l
    wall = time.perf_counter() - t_start
    st = pg.serve_stats()
    pg.serve_stop()
    # identity: a seeded sample of the queries, recomputed alone
    sample = np.random.default_rng(1).choice(len(pos), min(256, len(pos)), replace=False)
    alone = pg.perft_batch(pos[sample], depths[sample])
    line = {"metric": "serving queries/s with p50/p99 latency", "value": len(pos) / wall, "unit": "queries/s",
            "n_gpus": 1, "higher_is_better": True, "data": "synthetic", "dtype": "u64",
            "config": {"workload": "Poisson arrivals, seeded 0-40-ply positions, depth U[3,7]",
                       "offered_rate_qps": args.rate, "queries": len(pos),
                       "memory_budget_gb": args.serve_memory_gb or "90% of free arena",
                       "step_items": args.serve_step_items or "server default"},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "max": float(lat.max())},
            "leaf_nodes_per_s": float(counts.sum()) / wall,
            "identical_alone_vs_mix": bool(np.array_equal(alone, counts[sample])),
            "server": {k: st[k] for k in ("iterations", "launches", "memory_peak")}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["batch", "start", "deep", "tt", "serve"], default="batch")
    ap.add_argument("--sliders", choices=["auto", "kogge", "magic", "kogge_fma", "kogge_split", "hybrid"], default="auto")
    ap.add_argument("--positions", type=int, default=4096,
                    help="batch workload: use the first N positions (profiling runs)")
    ap.add_argument("--arena-gb", type=float, default=0.0, help="level-buffer arena (0 = 85%% of free HBM)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--form", choices=["batch", "single"], default="batch",
                    help="batch workload: one batched call, or one call per position")
    ap.add_argument("--tt-log2", type=int, default=30, help="tt workload: table entries (log2)")
    ap.add_argument("--max-depth", type=int, default=10, help="tt workload: cap on the depths")
    ap.add_argument("--parity-depth", type=int, default=8,
                    help="tt workload: depth of the table vs no-table equality check")
    ap.add_argument("--rate", type=float, default=1000.0, help="serve workload: offered queries/s")
    ap.add_argument("--queries", type=int, default=2000, help="serve workload: trace length")
    ap.add_argument("--serve-memory-gb", type=float, default=120.0, help="serve workload: admission budget")
    ap.add_argument("--serve-step-items", type=int, default=0,
                    help="serve workload: items per level per scheduler step (0 = server default)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "tt":
        return run_tt(args)
    if args.workload == "serve":
        return run_serve(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
