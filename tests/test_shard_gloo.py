"""Multi-process split on CPU ranks (gloo, world size 2): positions of a
batch and frontier shards of one deep position are dealt across ranks from a
shared cursor on the process group's store, and the sums reduced; every rank
must end with exactly the single-process result, and every unit must be
counted by exactly one rank.  Batch counts come from the oracle; deep counts
come from the product's own perft_deep_shard (host.cpp) linked against the
host stand-in engine (tests/hostapi), so no GPU is needed; the GPU engine
plugs into the same functions through perft_batch / deep."""
import json
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
START = "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1"


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _oracle():
    import sys
    sys.path.insert(0, ROOT)
    from tests._oracle import Oracle
    return Oracle(os.path.join(ROOT, "oracle", "liboracle.so"))


def _midgame(oracle):
    """A position six plies in, reached by a fixed choice of child indices."""
    p = oracle.fen_to_pos(START)
    for k in (11, 5, 16, 9, 3, 20):
        kids = oracle.children(p)
        p = kids[k % len(kids)]
    return p


def _batch(oracle):
    start = oracle.fen_to_pos(START)
    pos = [g for c in oracle.children(start) for g in oracle.children(c)]
    pos += oracle.children(_midgame(oracle))
    pos = np.array(pos, dtype=np.uint64)
    depths = (np.arange(len(pos)) % 3 + 1).astype(np.uint8)
    return pos, depths


def _skewed_batch(oracle):
    """A batch whose cost sits in a few positions: two depth-4 positions among
    many depth-1 ones, so a fixed stride would give one rank most of the work."""
    start = oracle.fen_to_pos(START)
    kids = oracle.children(start)
    pos = np.array([kids[i % len(kids)] for i in range(40)], dtype=np.uint64)
    depths = np.ones(40, dtype=np.uint8)
    depths[[3, 5]] = 4
    return pos, depths


def _hostapi_deep_fn():
    """deep_fn over the real perft_deep_shard of host.cpp, counting with the
    host stand-in engine (tests/hostapi)."""
    import ctypes
    import perft_gpu_b200 as pg
    lib = pg._bind(ctypes.CDLL(os.path.join(ROOT, "tests", "hostapi", "libhostapi.so")))
    lib.hostapi_init()
    calls = []

    def deep_fn(p, depth, split, s, n):
        calls.append((s, n))
        old = pg._lib_handle
        pg._lib_handle = lib
        try:
            return pg.deep(p, depth, split, s, n)
        finally:
            pg._lib_handle = old
    return deep_fn, calls


def _worker(rank, world, port, out_dir):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from datetime import timedelta
    from perft_gpu_b200 import shard

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        oracle = _oracle()
        pos, depths = _batch(oracle)
        seen = []

        def counter(p, d):
            seen.extend(int(x) for x in p[:, 0])
            return [oracle.perft(x, int(k)) for x, k in zip(p, d)]

        taken = []
        batch = shard.perft_batch_sharded(pos, depths, counter=counter, taken=taken)

        spos, sdepths = _skewed_batch(oracle)
        skew_seen = []

        def skew_counter(p, d):
            skew_seen.extend(int(x) for x in d)
            return [oracle.perft(x, int(k)) for x, k in zip(p, d)]

        skew = shard.perft_batch_sharded(spos, sdepths, counter=skew_counter, chunks_per_rank=10)

        mid = _midgame(oracle)
        deep_fn, calls = _hostapi_deep_fn()
        deep_taken = []
        total, div = shard.deep_sharded(mid, 4, 2, deep_fn=deep_fn, taken=deep_taken)
        (tmax, emax), (leaves,) = shard.max_sum_over_ranks([1.0 + rank, 10.0 * rank], [100.0 * (rank + 1)])
        # counts near and past 2^63 / 2^64 in the sum stay exact
        wide = shard._sum_u64(np.array([2**63 + rank, 2**64 - 1 - rank, 2**32 - 1], dtype=np.uint64),
                              dist, None, "cpu")
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"batch": [int(x) for x in batch], "n_counted": len(seen), "total": total, "div": div,
                       "tmax": tmax, "emax": emax, "leaves": leaves, "wide": [str(x) for x in wide],
                       "taken": taken, "skew": [int(x) for x in skew], "skew_depths": skew_seen,
                       "deep_taken": deep_taken, "deep_calls": calls}, f)
    finally:
        dist.destroy_process_group()


def test_strided_deal_covers_once():
    from perft_gpu_b200.shard import strided
    for n in (0, 1, 7, 100):
        for world in (1, 2, 3, 8):
            got = np.sort(np.concatenate([strided(n, r, world) for r in range(world)]))
            assert np.array_equal(got, np.arange(n))
    with pytest.raises(ValueError):
        strided(4, 2, 2)


def test_two_gloo_ranks_match_single_process(tmp_path, oracle):
    from tests.test_host_paths import build_hostapi
    build_hostapi()  # the ranks load it; rebuilt here if its sources changed
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    pos, depths = _batch(oracle)
    want = [oracle.perft(p, int(d)) for p, d in zip(pos, depths)]
    mid = _midgame(oracle)
    want_div = sorted(oracle.perft(c, 3) for c in oracle.children(mid))
    spos, sdepths = _skewed_batch(oracle)
    want_skew = [oracle.perft(p, int(d)) for p, d in zip(spos, sdepths)]
    for r in res:
        assert r["batch"] == want
        assert r["skew"] == want_skew
        assert r["total"] == oracle.perft(mid, 4) == sum(want_div)
        assert sorted(r["div"].values()) == want_div
        assert (r["tmax"], r["emax"], r["leaves"]) == (2.0, 10.0, 300.0)
        assert [int(x) for x in r["wide"]] == [2**64 + 1, 2**65 - 3, 2**33 - 2]
    # each position counted by exactly one rank; every chunk dealt once
    assert sum(r["n_counted"] for r in res) == len(pos)
    assert sorted(res[0]["taken"] + res[1]["taken"]) == list(range(16))
    assert sorted(res[0]["skew_depths"] + res[1]["skew_depths"]) == sorted(int(d) for d in sdepths)
    # deep: shards 0..7 of 8 each searched once, over the real perft_deep_shard
    assert sorted(res[0]["deep_taken"] + res[1]["deep_taken"]) == list(range(8))
    assert sorted(s for r in res for s, n in r["deep_calls"] if n == 8) == list(range(8))


def test_largest_first_chunks():
    """Positions are dealt deepest first: with one position per chunk, the
    first chunks are the expensive ones, whichever rank takes them."""
    from perft_gpu_b200 import shard

    class Store:
        def __init__(self):
            self.v = {}

        def add(self, k, a):
            self.v[k] = self.v.get(k, 0) + a
            return self.v[k]

    depths = np.array([1, 1, 4, 1, 6, 1, 5, 1], dtype=np.uint8)
    pos = np.zeros((8, 6), dtype=np.uint64)
    pos[:, 0] = np.arange(8)
    order = []

    def counter(p, d):
        order.extend(int(x) for x in p[:, 0])
        return np.zeros(len(p), dtype=np.uint64)

    # one process standing in for rank 0 of 2, with a private store: it takes every chunk in order
    orig = shard._world
    shard._world = lambda group: (None, 0, 2)
    try:
        shard.perft_batch_sharded(pos, depths, counter=counter, store=Store(), chunks_per_rank=4)
    finally:
        shard._world = orig
    assert order[:3] == [4, 6, 2]
