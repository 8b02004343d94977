#!/usr/bin/env python3
"""Perft throughput benchmark (leaf nodes/s, bit-exact) on B200.

Default workload: the batched perft of 4096 seeded, stratified playout
positions at depths U[4,6] (one step = one perft_batch over the whole
batch).  Other workloads: --workload start (initial position, depth 5,
repeated), --workload deep (one 20-ply playout with >= 35 moves, depth 8),
--workload tt (4 positions at depths 9-10 with a 2^30-entry table),
--workload serve (Poisson serving trace).

On one GPU the default run also measures the other configurations after the
headline leg and reports them under "configs": the initial position at depth
5, the depth-8 position, the transposition-table positions at depths 9-10,
and the same 4096-position batch run one position per call (the
batched/single ratio).  Counts are checked against the reference's own host
perft (tests/golden/config_counts.json) where it has them.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): each rank searches its own 4096-position batch (seed
offset by rank); there is no data-path collective, only a barrier and a
max/sum reduction of the timings and counts.

The workloads are read from perft_gpu_b200/data/workloads.npz (numpy only),
so the reference arm's process never loads the engine library.

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
WL_PATH = os.path.join(ROOT, "perft_gpu_b200", "data", "workloads.npz")
GOLDEN_PATH = os.path.join(ROOT, "tests", "golden", "config_counts.json")


def stored_workloads():
    """The seeded workloads as plain arrays (numpy only: no engine library)."""
    with np.load(WL_PATH) as z:
        return {k: z[k] for k in z.files}


def reference_counts():
    """Counts of the reference's own host perft on the stored workloads, or None."""
    if not os.path.exists(GOLDEN_PATH):
        return None
    with open(GOLDEN_PATH) as f:
        return json.load(f)


def reference_start_counts():
    """The reference's perft of the initial position by depth (tests/golden/perft_golden.json)."""
    path = os.path.join(ROOT, "tests", "golden", "perft_golden.json")
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        g = json.load(f)
    for e in g["positions"]:
        if e["name"] == "initial_position":
            return {int(k): int(v) for k, v in e["counts"].items()}
    return {}


BATCH_DESC = ("batch{n}: {n} seeded playouts of 8-30 plies, stratified "
              "(>=10% en passant, >=10% pawn on 7th, >=10% castling), depth U[4,6]")


def make_workload(name, rank, positions=4096):
    wl = stored_workloads()
    if name == "batch":
        if rank == 0:
            pos, depths = wl["batch_pos"], wl["batch_depths"]
        else:
            # other ranks' batches (GPU arm under torchrun only): generated
            from perft_gpu_b200 import workloads as W
            pos, depths = W.batch_positions(n=4096, seed=2026 + rank)
        pos, depths = pos[:positions], depths[:positions]
        cfg = {"workload": BATCH_DESC.format(n=positions),
               "positions": positions, "depths": "U[4,6]", "seed": 2026 + rank}
        return pos, depths, cfg, "batch4096"
    if name == "start":
        pos = np.array([[0xFFFF, 0x00FF00000000FF0F, 0x4200000000000042, 0x2C0000000000002C,
                         0x8900000000000089, 0x1000000000000010]], dtype=np.uint64)
        cfg = {"workload": "initial position, depth 5, no transposition table", "positions": 1,
               "depths": "5"}
        return pos, np.array([5], dtype=np.uint8), cfg, "start"
    if name == "deep":
        cfg = {"workload": "one seeded 20-ply playout with >=35 legal moves, depth 8, no TT",
               "positions": 1, "depths": "8"}
        return wl["deep_pos"].reshape(1, 6), np.array([8], dtype=np.uint8), cfg, "deep"
    raise SystemExit(f"unknown workload {name}")


# ------------------------------------------------------------------ CPU arms
def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _cpu_has_x86_64_v3():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return {"avx2", "bmi1", "bmi2", "fma", "movbe", "abm"} <= flags
    except OSError:
        pass
    return False


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_perft_lib():
    """The reference's host perft when it was built (oracle/_ref: the x86-64-v3
    build on hosts with AVX2/BMI2, else the SSE4.2 build), else the oracle port."""
    ref_dir = os.path.join(ROOT, "oracle", "_ref")
    names = (["libperft_ref.so"] if _cpu_has_x86_64_v3() else []) + ["libperft_ref_sse42.so"]
    for name in names:
        path = os.path.join(ref_dir, name)
        if os.path.exists(path):
            lib = ctypes.CDLL(path)
            lib.ref_init()
            return "reference", lib.ref_perft_batch_mt, name
    orc = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(orc):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    lib = ctypes.CDLL(orc)
    lib.oracle_init()
    return "port", lib.oracle_perft_batch_mt, "liboracle.so"


def cpu_sample(pos, depths, budget_s, expected=None, threads=None):
    """Runs the CPU perft over a bounded sample of the workload: a seeded
    random order of its positions, taken in groups until budget_s elapses."""
    kind, fn, libname = cpu_perft_lib()
    threads = threads or host_threads()
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
            "cpu": cpu_model(), "library": f"oracle/_ref/{libname}" if kind == "reference" else f"oracle/{libname}",
            "sample": f"{done} of {len(pos)} positions (seeded order) at their own depths, "
                      f"{leaves} leaves in {el:.1f} s",
            "mismatches_vs_gpu": mismatches if expected is not None else None}


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    pos, depths, cfg, _ = make_workload(args.workload, 0, args.positions)
    # each timed step is a bounded sample; the whole run stays within about
    # three minutes however many steps are asked for
    per_step = min(args.cpu_seconds, max(2.0, 150.0 / max(1, args.steps)))
    vals = []
    for _ in range(args.warmup):
        cpu_sample(pos, depths, min(3.0, per_step))
    last = None
    for _ in range(args.steps):
        last = cpu_sample(pos, depths, per_step)
        vals.append(last["value"])
    v = float(np.mean(vals))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "ms_per_step": None, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": last["cores"], "kind": last["kind"],
                             "cpu": last["cpu"], "library": last["library"], "sample": last["sample"]},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ GPU arm
def single_form_step(pg, d_pos, depths, d_out):
    """The one-position-per-call form: each position is copied into one fixed
    device slot and searched by its own perft_batch_device call (a fixed slot
    lets the engine reuse its per-depth launch graphs; positions of depth 2-5
    take the one-launch small-tree kernel)."""
    import torch
    n = len(depths)
    slot = torch.zeros(6, dtype=torch.int64, device="cuda")
    res = torch.zeros(1, dtype=torch.int64, device="cuda")

    def step():
        for i in range(n):
            slot.copy_(d_pos[i])
            pg.perft_batch_device(slot.data_ptr(), depths[i:i + 1], 1, res.data_ptr())
            d_out[i:i + 1].copy_(res)
    return step


def device_timed(fn, steps, device):
    """Device time (ms) of `steps` calls of fn, between CUDA events on torch's
    current stream (the legacy default stream; the engine's stream is a
    blocking stream, so the events bracket its work), with clocks sampled
    during the region."""
    import torch
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(device) as clk:
        torch.cuda.synchronize()
        s.record()
        for _ in range(steps):
            fn()
        e.record()
        torch.cuda.synchronize()
    return s.elapsed_time(e), clk.summary()


def measure_configs(args, pg, device, d_pos, depths, batch_ms_per_step, golden):
    """The other configurations on this GPU, after the headline leg: the
    initial position at depth 5, the depth-8 position, the 4096-position batch
    one position per call, and (last: it re-creates the engine with a 2^30-entry
    table) the transposition-table positions at depths 9-10."""
    import torch
    wl = stored_workloads()
    out = {}

    # initial position, depth 5, no table: latency-bound, many steps
    start, dstart, _, _ = make_workload("start", 0)
    sp = torch.from_numpy(start.view(np.int64)).cuda()
    so = torch.zeros(1, dtype=torch.int64, device="cuda")
    fn = lambda: pg.perft_batch_device(sp.data_ptr(), dstart, 1, so.data_ptr())  # noqa: E731
    for _ in range(20):
        fn()
    steps = 200
    ms, clk = device_timed(fn, steps, device)
    leaves = int(so.cpu().numpy().view(np.uint64)[0])
    want = reference_start_counts().get(5)
    e_ms, _ = device_timed(lambda: pg.perft(start[0], 5), steps, device)
    out["start_d5"] = {"workload": "initial position, depth 5, no transposition table", "steps": steps,
                       "ms_per_step": ms / steps, "value": leaves * steps / (ms / 1e3), "unit": UNIT,
                       "leaves": leaves, "equals_reference": (leaves == want) if want else None,
                       "e2e": {"value": leaves * steps / (e_ms / 1e3), "unit": UNIT,
                               "h2d_bytes_per_step": 48, "d2h_bytes_per_step": 8},
                       "clocks": clk}

    # one position at depth 8, no table
    dp = torch.from_numpy(wl["deep_pos"].reshape(1, 6).view(np.int64)).cuda()
    do = torch.zeros(1, dtype=torch.int64, device="cuda")
    d8 = np.array([8], dtype=np.uint8)
    fn = lambda: pg.perft_batch_device(dp.data_ptr(), d8, 1, do.data_ptr())  # noqa: E731
    fn()
    steps = 2
    pg.reset_stats()
    ms, clk = device_timed(fn, steps, device)
    st = pg.stats()
    leaves = int(do.cpu().numpy().view(np.uint64)[0])
    want = golden["deep"]["total"] if golden and "deep" in golden else None
    out["deep_d8"] = {"workload": "one seeded 20-ply playout with >=35 legal moves, depth 8, no TT",
                      "steps": steps, "ms_per_step": ms / steps, "value": leaves * steps / (ms / 1e3),
                      "unit": UNIT, "leaves": leaves, "equals_reference": (leaves == want) if want else None,
                      "leaf_share_of_step": st["leaf_ms"] / ms if ms > 0 else None,
                      "chunked_levels": st["chunked_levels"], "clocks": clk}

    # the same 4096-position batch, one position per call
    n = len(depths)
    so = torch.zeros(n, dtype=torch.int64, device="cuda")
    step = single_form_step(pg, d_pos, depths, so)
    ms, clk = device_timed(step, 1, device)
    single = so.cpu().numpy().view(np.uint64)
    want = np.array(golden["batch4096"]["counts"][:n], dtype=np.uint64) if golden else None
    out["batch4096_single"] = {
        "workload": BATCH_DESC.format(n=n) + ", one perft_batch_device call per position (fixed device slot)",
        "steps": 1, "ms_per_step": ms, "value": float(single.sum()) / (ms / 1e3), "unit": UNIT,
        "equals_reference": bool(np.array_equal(single, want)) if want is not None else None,
        "batched_over_single": ms / batch_ms_per_step, "clocks": clk}

    # the same again, one position per call through the host-driven level
    # pipeline: per ply a scan whose total the host reads back, then a tile
    # launch; no captured graph and no small-tree kernel.  This is the shape of
    # the reference's one-position driver (a level loop with a device
    # synchronisation per ply, perft_bb.h:1027-1138).
    saved = {k: os.environ.get(k) for k in ("PERFT_NO_GRAPHS", "PERFT_SMALL_TREE")}
    os.environ.update({"PERFT_NO_GRAPHS": "1", "PERFT_SMALL_TREE": "0"})
    try:
        pg.init(device=device, arena_bytes=int(args.arena_gb * (1 << 30)))
        step = single_form_step(pg, d_pos, depths, so)
        ms2, clk2 = device_timed(step, 1, device)
        levels = so.cpu().numpy().view(np.uint64)
    finally:
        for k, v in saved.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    out["batch4096_single_levels"] = {
        "workload": BATCH_DESC.format(n=n) + ", one perft_batch_device call per position, host-driven level "
                                             "pipeline (no captured graph, no small-tree kernel)",
        "steps": 1, "ms_per_step": ms2, "value": float(levels.sum()) / (ms2 / 1e3), "unit": UNIT,
        "equals_reference": bool(np.array_equal(levels, want)) if want is not None else None,
        "batched_over_single_levels": ms2 / batch_ms_per_step, "clocks": clk2}

    # transposition-table positions at depths 9-10 (2^30 entries), after the
    # depth-8 check without and with the table against the reference
    out["tt_d9_10"] = tt_leg(pg, device, wl, args, golden, timed_steps=1)

    # the 4096-position batch again, through the engine with the 2^30-entry
    # table (cleared first): effective rate, counts against the reference
    so = torch.zeros(n, dtype=torch.int64, device="cuda")
    pg.tt_clear()
    ms, clk = device_timed(lambda: pg.perft_batch_device(d_pos.data_ptr(), depths, n, so.data_ptr()), 1, device)
    got = so.cpu().numpy().view(np.uint64)
    out["batch4096_tt"] = {
        "workload": BATCH_DESC.format(n=n) + ", with a 2^%d-entry table cleared before the step" % args.tt_log2,
        "steps": 1, "ms_per_step": ms, "value": float(got.sum()) / (ms / 1e3),
        "unit": UNIT + " (effective: leaves counted)",
        "equals_reference": bool(np.array_equal(got, want)) if want is not None else None,
        # the same leaves against the plain one-position-per-call form (no table)
        "over_single_plain": out["batch4096_single"]["ms_per_step"] / ms if ms > 0 else None, "clocks": clk}
    return out


def tt_leg(pg, device, wl, args, golden, timed_steps=1, warmup=0):
    """Depths 9-10 of the 4 table positions with a 2^tt_log2-entry table
    (cleared before each step), after checking depth 8 with and without the
    table against the reference's counts."""
    import torch
    pos = wl["tt_pos"]
    depths = np.minimum(wl["tt_depths"], args.max_depth).astype(np.uint8)
    pd = args.parity_depth
    arena = int(args.arena_gb * (1 << 30))
    pg.init(device=device, arena_bytes=arena)
    t0 = time.perf_counter()
    plain = pg.perft_batch(pos, pd)
    t_plain = time.perf_counter() - t0
    pg.init(device=device, arena_bytes=arena, tt_log2_entries=args.tt_log2)
    t0 = time.perf_counter()
    with_tt = pg.perft_batch(pos, pd)
    t_tt = time.perf_counter() - t0
    ref = None
    if golden and "tt" in golden and pd == 8:
        ref = [int(e["total"]) for e in golden["tt"]]
    d_pos = torch.from_numpy(np.ascontiguousarray(pos).view(np.int64)).cuda()
    d_out = torch.zeros(len(pos), dtype=torch.int64, device="cuda")
    fn = lambda: pg.perft_batch_device(d_pos.data_ptr(), depths, len(pos), d_out.data_ptr())  # noqa: E731
    total_ms, clk_all, counts = 0.0, [], None
    for step in range(warmup + timed_steps):
        pg.tt_clear()
        pg.reset_stats()
        ms, clk = device_timed(fn, 1, device)
        if step >= warmup:
            total_ms += ms
            clk_all.append(clk)
        counts = d_out.cpu().numpy().view(np.uint64).copy()
    st = pg.stats()
    leaves = int(counts.sum())
    return {"workload": "4 seeded playouts of 12-24 plies, TT of 2^%d x 16 B, table cleared each step"
                        % args.tt_log2,
            "depths": depths.tolist(), "steps": timed_steps, "ms_per_step": total_ms / timed_steps,
            "value": leaves * timed_steps / (total_ms / 1e3), "unit": UNIT + " (effective: leaves counted)",
            "counts": [int(x) for x in counts],
            "parity_depth%d" % pd: {"no_tt": [int(x) for x in plain], "tt": [int(x) for x in with_tt],
                                    "tt_equals_no_tt": bool(np.array_equal(plain, with_tt)),
                                    "equals_reference": (([int(x) for x in plain] == ref) and
                                                         ([int(x) for x in with_tt] == ref)) if ref else None,
                                    "no_tt_s": t_plain, "tt_s": t_tt},
            "tt": {k: st[k] for k in ("tt_entries", "tt_probes", "tt_hits", "tt_duplicates", "tt_stores")},
            "clocks": clk_all[-1] if clk_all else None}


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
    tuning = [{k: v for k, v in e.items()} for e in pg.tuning()]

    n = len(pos)
    d_pos = torch.from_numpy(pos.view(np.int64)).cuda()
    d_out = torch.zeros(n, dtype=torch.int64, device="cuda")

    if args.form == "single":
        step_device = single_form_step(pg, d_pos, depths, d_out)
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

    golden = reference_counts()
    parity = None
    if golden and args.workload == "batch" and rank == 0 and len(counts) <= len(golden["batch4096"]["counts"]):
        want = np.array(golden["batch4096"]["counts"][:len(counts)], dtype=np.uint64)
        parity = {"positions": int(len(counts)), "equal": int(np.count_nonzero(counts == want)),
                  "reference": "oracle/_ref host perft, every position at its own depth "
                               "(tests/golden/config_counts.json)"}

    configs = None
    if ws == 1 and args.workload == "batch" and args.form == "batch" and not args.no_configs:
        configs = measure_configs(args, pg, local, d_pos, depths, ms_max / args.steps, golden)

    cpu = None
    if ws == 1 and not args.no_cpu:
        cpu = cpu_sample(pos, depths, args.cpu_seconds, expected=counts)

    cfg = dict(cfg)
    cfg.update({"form": "one perft call per position" if args.form == "single" else "one batched call",
                "sliders": {"leaf": pg.SLIDER_NAMES.get(st["sliders_leaf"], "?"),
                            "interior": pg.SLIDER_NAMES.get(st["sliders_expand"], "?"),
                            "chosen_by": args.sliders, "per_depth": tuning},
                "l2": "no flush: each step streams multi-GB level buffers through HBM (>> 126 MB L2)",
                "parallelism": f"independent batches, {ws} GPU(s)"})
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic", "config": cfg,
        "leaves_per_step": int(tot), "counts_stable": stable, "counts_vs_reference": parity,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(pos.nbytes),
                "d2h_bytes_per_step": int(8 * n)},
        "gpu_launches": int(st["leaf_launches"] + st["expand_launches"] + st["other_launches"]
                            + st["small_launches"]),
        "roofline": roofline,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
    }
    if configs is not None:
        line["configs"] = configs
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()
    return 0


def run_tt(args):
    """Transposition-table workload alone: 4 seeded playouts of 12-24 plies
    at depths 9-10 with a 2^30-entry table; parity with the no-table engine
    and with the reference is checked at depth 8 first."""
    import perft_gpu_b200 as pg
    import torch
    torch.cuda.set_device(0)
    r = tt_leg(pg, 0, stored_workloads(), args, reference_counts(), timed_steps=args.steps,
               warmup=args.warmup)
    line = {"metric": "perft leaf nodes/s with transposition table (effective, bit-exact)",
            "value": r["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "dtype": "u64", "data": "synthetic",
            "config": {"workload": r["workload"], "depths": r["depths"]},
            **{k: v for k, v in r.items() if k not in ("workload", "depths", "value", "ms_per_step", "steps")}}
    print(json.dumps(line), flush=True)
    return 0


def run_serve(args):
    """Serving workload: the stored trace of 10,000 seeded 0-40-ply positions
    at depth U[3,7], submitted with Poisson arrivals at each offered rate of
    the sweep through the continuous-batching server (table resident in the
    server when --tt-log2 > 0, cleared between rates).  p50/p99 latency is
    submit-to-completion time.  Every result is checked against the same
    query run alone (the batch engine without a table) and against the other
    rates' results."""
    import perft_gpu_b200 as pg
    import torch
    torch.cuda.set_device(0)
    wl = stored_workloads()
    n = min(args.queries, len(wl["serve_pos"]))
    pos, depths = wl["serve_pos"][:n], wl["serve_depths"][:n]
    rates = [float(x) for x in args.rates.split(",")] if args.rates else [args.rate]
    arena = int(args.arena_gb * (1 << 30))

    pg.init(device=0, arena_bytes=arena)
    t0 = time.perf_counter()
    alone = pg.perft_batch(pos, depths)
    alone_s = time.perf_counter() - t0
    tt_log2 = args.serve_tt_log2
    pg.init(device=0, arena_bytes=arena, tt_log2_entries=tt_log2)
    points = []
    for rate in rates:
        arrivals = np.cumsum(np.random.default_rng(5).exponential(1.0 / rate, size=n))
        if tt_log2:
            pg.tt_clear()
        pg.serve_start(memory_bytes=int(args.serve_memory_gb * (1 << 30)), step_items=args.serve_step_items,
                       use_tt=tt_log2 > 0)
        tickets = [None] * n
        with ClockSampler(0) as clk:
            t_start = time.perf_counter()
            for i in range(n):
                delay = t_start + arrivals[i] - time.perf_counter()
                if delay > 0:
                    time.sleep(delay)
                tickets[i] = pg.serve_submit(pos[i], int(depths[i]))
            lat, counts = np.zeros(n), np.zeros(n, dtype=np.uint64)
            for i, t in enumerate(tickets):
                c, l = pg.serve_wait(t, timeout_s=3600)
                counts[i], lat[i] = c, l
            wall = time.perf_counter() - t_start
        st = pg.serve_stats()
        pg.serve_stop()
        points.append({"offered_qps": rate, "completed_qps": n / wall, "wall_s": wall,
                       "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                                     "max": float(lat.max())},
                       "leaf_nodes_per_s": float(counts.sum()) / wall,
                       "identical_alone_vs_mix": bool(np.array_equal(alone, counts)),
                       "server": {k: st[k] for k in ("iterations", "launches", "memory_peak", "tt_probes", "tt_hits",
                                                     "tt_merged", "tt_stores")},
                       "clocks": clk.summary()})
    line = {"metric": "serving queries/s with p50/p99 latency", "unit": "queries/s", "n_gpus": 1,
            "higher_is_better": True, "data": "synthetic", "dtype": "u64",
            "value": max(p["completed_qps"] for p in points),
            "config": {"workload": "Poisson arrivals of the stored 0-40-ply positions, depth U[3,7]",
                       "queries": n, "memory_budget_gb": args.serve_memory_gb,
                       "transposition_table": f"2^{tt_log2} x 16 B, resident in the server, cleared between rates"
                       if tt_log2 else "none",
                       "step_items": args.serve_step_items or "server default"},
            "alone": {"engine": "perft_batch without a table", "seconds": alone_s,
                      "leaves": int(alone.sum())},
            "sweep": points,
            "timing": "host wall clock (submit to completion per query; whole trace for q/s)"}
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
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other configurations measured after the headline leg")
    ap.add_argument("--form", choices=["batch", "single"], default="batch",
                    help="batch workload: one batched call, or one call per position")
    ap.add_argument("--tt-log2", type=int, default=30, help="tt workload: table entries (log2)")
    ap.add_argument("--max-depth", type=int, default=10, help="tt workload: cap on the depths")
    ap.add_argument("--parity-depth", type=int, default=8,
                    help="tt workload: depth of the table vs no-table equality check")
    ap.add_argument("--rate", type=float, default=1000.0, help="serve workload: offered queries/s")
    ap.add_argument("--rates", default="", help="serve workload: comma-separated offered rates to sweep")
    ap.add_argument("--queries", type=int, default=10000, help="serve workload: trace length")
    ap.add_argument("--serve-tt-log2", type=int, default=30,
                    help="serve workload: table entries (log2) resident in the server; 0 = no table")
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
