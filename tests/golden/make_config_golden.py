"""Generates tests/golden/config_counts.json from the REFERENCE's own host perft.

Run in a container that holds the reference build (``make -C oracle ref``):
    python tests/golden/make_config_golden.py [--threads N]

Counts come from oracle/_ref/libperft_ref.so: the reference's perft_bb
(perft_bb.h:79-101) over its own generateBoards/countMoves, compiled from the
reference sources, run root-split over host threads (ref_perft_batch_mt).
Positions are the stored benchmark workloads (perft_gpu_b200/data/workloads.npz),
so every configuration is pinned at its own size:

  batch4096  perft of each of the 4096 batch positions at its own depth (4-6)
  deep       the depth-8 position: perft(7) of every child (divided perft 8)
  tt         the 4 transposition-table positions: perft(7) of every child
             (divided perft 8); perft(9) and perft(10) are then checked on
             the GPU as sums over the children

Child lists are stored as sorted counts (the reference and the engine emit
moves in different orders) together with their sum.
"""
import argparse
import ctypes
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "libperft_ref.so")
WL = os.path.join(ROOT, "perft_gpu_b200", "data", "workloads.npz")
OUT = os.path.join(HERE, "config_counts.json")


def load_ref():
    lib = ctypes.CDLL(REF)
    lib.ref_children.restype = ctypes.c_uint32
    lib.ref_init()
    return lib


def batch_mt(lib, pos, depths, threads):
    pos = np.ascontiguousarray(np.asarray(pos, dtype=np.uint64).reshape(-1, 6))
    d = np.ascontiguousarray(np.broadcast_to(np.asarray(depths, dtype=np.uint32), (len(pos),)))
    out = np.zeros(len(pos), dtype=np.uint64)
    rc = lib.ref_perft_batch_mt(ctypes.c_void_p(pos.ctypes.data), ctypes.c_void_p(d.ctypes.data),
                                ctypes.c_uint32(len(pos)), ctypes.c_int(threads), ctypes.c_void_p(out.ctypes.data))
    assert rc == 0
    return out


def children(lib, p):
    buf = (ctypes.c_uint64 * (6 * 256))()
    src = (ctypes.c_uint64 * 6)(*[int(x) for x in np.asarray(p, dtype=np.uint64).reshape(6)])
    n = lib.ref_children(src, buf)
    return np.array(list(buf[:6 * n]), dtype=np.uint64).reshape(n, 6)


def divided(lib, p, depth, threads):
    ch = children(lib, p)
    counts = batch_mt(lib, ch, depth - 1, threads)
    return {"depth": depth, "total": int(counts.sum(dtype=np.uint64)),
            "children_sorted": sorted(int(c) for c in counts),
            "pos48": [hex(int(x)) for x in np.asarray(p, dtype=np.uint64).reshape(6)]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    args = ap.parse_args()
    lib = load_ref()
    with np.load(WL) as z:
        wl = {k: z[k] for k in z.files}
    out = {"source": "oracle/_ref/libperft_ref.so (reference perft_bb, perft_bb.h:79-101), "
                     "ref_perft_batch_mt root-split over host threads",
           "script": "tests/golden/make_config_golden.py", "threads": args.threads, "seconds": {}}

    def save():
        with open(OUT, "w") as f:
            json.dump(out, f, indent=1)

    t0 = time.time()
    c = batch_mt(lib, wl["batch_pos"], wl["batch_depths"], args.threads)
    out["batch4096"] = {"depths": "own (batch_depths)", "counts": [int(x) for x in c],
                        "total": int(c.sum(dtype=np.uint64))}
    out["seconds"]["batch4096"] = round(time.time() - t0, 1)
    save()
    print("batch4096", out["batch4096"]["total"], out["seconds"]["batch4096"], "s", flush=True)

    t0 = time.time()
    out["deep"] = divided(lib, wl["deep_pos"][0], 8, args.threads)
    out["seconds"]["deep"] = round(time.time() - t0, 1)
    save()
    print("deep", out["deep"]["total"], out["seconds"]["deep"], "s", flush=True)

    out["tt"] = []
    for i, p in enumerate(wl["tt_pos"]):
        t0 = time.time()
        out["tt"].append(divided(lib, p, 8, args.threads))
        out["seconds"][f"tt{i}"] = round(time.time() - t0, 1)
        save()
        print("tt", i, out["tt"][-1]["total"], out["seconds"][f"tt{i}"], "s", flush=True)


if __name__ == "__main__":
    main()
