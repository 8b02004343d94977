"""Test infrastructure: freezes the algorithmic work figures of the perft path.

Runs the op-counting build of the oracle (oracle/opcount, the reference
algorithm restated, with slider lookups charged at the reference's fancy
magic cost) over perft trees of each benchmark workload's positions and
writes the per-call averages to perft_gpu_b200/work_figures.json:

  c_count  64-bit ops per countMoves call   (leaf pass, once per item)
  c_make   64-bit ops per makeMove call     (once per item)
  c_gen    64-bit ops per generateMoves call (once per parent)

bench.py turns them into the integer work of a leaf-kernel launch:
  W = 2 * (items * (c_make + c_count) + parents * c_gen)   32-bit ops
(each 64-bit op counted as two 32-bit integer-pipe operations).

Usage: python oracle/opcount.py
"""
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from perft_gpu_b200 import workloads  # noqa: E402


def measure(positions, depth):
    exe = os.path.join(ROOT, "oracle", "opcount")
    if not os.path.exists(exe):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "opcount"], check=True)
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        f.write(np.ascontiguousarray(positions, dtype=np.uint64).tobytes())
        path = f.name
    try:
        out = subprocess.run([exe, path, str(depth)], check=True, capture_output=True, text=True).stdout
    finally:
        os.unlink(path)
    return json.loads(out)


def main():
    res = {"method": ("op-counting oracle (oracle/opcount_main.cpp): 64-bit and/or/xor/not/shift/"
                      "add/sub/mul/compare/popcount/bitscan per call, slider lookups at the reference "
                      "fancy-magic cost (6 ops); averaged over depth-3 trees of the workload's positions"),
           "workloads": {}}
    pos, _ = workloads.batch_positions()
    sample = pos[np.random.default_rng(1).choice(len(pos), 256, replace=False)]
    res["workloads"]["batch4096"] = measure(sample, 3)
    res["workloads"]["start"] = measure(workloads.start_position().reshape(1, 6), 4)
    deep = workloads.deep_position()
    res["workloads"]["deep"] = measure(deep.reshape(1, 6), 3)
    out = os.path.join(ROOT, "perft_gpu_b200", "work_figures.json")
    with open(out, "w") as f:
        json.dump(res, f, indent=1)
    print(json.dumps(res, indent=1))


if __name__ == "__main__":
    main()
