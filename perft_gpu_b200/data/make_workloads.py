"""Writes workloads.npz: the seeded benchmark workloads as plain arrays.

The positions come from the generators in perft_gpu_b200/workloads.py (the
engine library's host-side playout code).  Storing them lets a process run a
workload with numpy alone, without loading the engine library: the CPU
reference arm of bench.py reads this file, so its process maps nothing of the
engine.  tests/test_workloads_fixture.py checks that the file still equals
the generators' output.

  python -m perft_gpu_b200.data.make_workloads

Arrays (positions are (n, 6) uint64 in the 48-byte board layout, depths uint8):
  batch_pos, batch_depths   4096 stratified playouts of 8-30 plies, depth U[4,6], seed 2026
  deep_pos                  one 20-ply playout with >= 35 legal moves (depth 8)
  tt_pos, tt_depths         4 playouts of 12-24 plies, depths 9-10
  serve_pos, serve_depths   10,000 playouts of 0-40 plies, depth U[3,7] (serving trace)
"""
import os

import numpy as np

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "workloads.npz")


def generate():
    from perft_gpu_b200 import workloads as W
    batch_pos, batch_depths = W.batch_positions(n=4096, seed=2026)
    tt_pos, tt_depths = W.tt_positions()
    serve_pos, serve_depths, _ = W.serving_trace(n=10000, rate_qps=1000.0, seed=5)
    return {
        "batch_pos": batch_pos.astype(np.uint64), "batch_depths": batch_depths.astype(np.uint8),
        "deep_pos": W.deep_position().astype(np.uint64).reshape(1, 6),
        "tt_pos": tt_pos.astype(np.uint64), "tt_depths": tt_depths.astype(np.uint8),
        "serve_pos": serve_pos.astype(np.uint64), "serve_depths": serve_depths.astype(np.uint8),
    }


def load(path=OUT):
    """The stored workloads (numpy only)."""
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


if __name__ == "__main__":
    np.savez_compressed(OUT, **generate())
    print(OUT, os.path.getsize(OUT), "bytes")
