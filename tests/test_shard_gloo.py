"""Multi-process split on CPU ranks (gloo, world size 2): positions of a
batch and frontier shards of one deep position are dealt across ranks and the
8-byte sums reduced; every rank must end with exactly the single-process
result.  The counter is the oracle, so no GPU is needed; the GPU engine plugs
into the same functions through perft_batch / deep."""
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

        batch = shard.perft_batch_sharded(pos, depths, counter=counter)

        mid = _midgame(oracle)
        kids = oracle.children(mid)

        def deep_fn(p, depth, split, s, n):
            # stands in for perft_deep_shard: a shard owns every n-th unit
            return None, {f"m{i}": (oracle.perft(c, depth - 1) if i % n == s else 0) for i, c in enumerate(kids)}

        total, div = shard.deep_sharded(mid, 3, 1, deep_fn=deep_fn)
        (tmax, emax), (leaves,) = shard.max_sum_over_ranks([1.0 + rank, 10.0 * rank], [100.0 * (rank + 1)])
        # counts near and past 2^63 / 2^64 in the sum stay exact
        wide = shard._sum_u64(np.array([2**63 + rank, 2**64 - 1 - rank, 2**32 - 1], dtype=np.uint64),
                              dist, None, "cpu")
        with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
            json.dump({"batch": [int(x) for x in batch], "n_counted": len(seen), "total": total, "div": div,
                       "tmax": tmax, "emax": emax, "leaves": leaves, "wide": [str(x) for x in wide]}, f)
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
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.load(open(tmp_path / f"r{r}.json")) for r in range(world)]
    pos, depths = _batch(oracle)
    want = [oracle.perft(p, int(d)) for p, d in zip(pos, depths)]
    mid = _midgame(oracle)
    want_div = [oracle.perft(c, 2) for c in oracle.children(mid)]
    for r in res:
        assert r["batch"] == want
        assert r["total"] == oracle.perft(mid, 3) == sum(want_div)
        assert [r["div"][f"m{i}"] for i in range(len(want_div))] == want_div
        assert (r["tmax"], r["emax"], r["leaves"]) == (2.0, 10.0, 300.0)
        assert [int(x) for x in r["wide"]] == [2**64 + 1, 2**65 - 3, 2**33 - 2]
    # each position counted by exactly one rank
    assert sum(r["n_counted"] for r in res) == len(pos)
    assert abs(res[0]["n_counted"] - res[1]["n_counted"]) <= 1
