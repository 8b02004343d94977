"""Device-driven perft replayed as a CUDA graph: identical counts to the
host-driven path, graph reuse across calls, and the overflow fallback."""
import os

import numpy as np
import pytest

from tests._oracle import pos48_from_hex

pytestmark = pytest.mark.gpu


def _reinit(engine, **env):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        engine.init(device=0, arena_bytes=env.pop("_arena", 4 << 30) if "_arena" in env else 4 << 30)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def test_graph_path_matches_host_path(engine, golden):
    start = next(e for e in golden if e["name"] == "initial_position")
    p = pos48_from_hex(start["pos48"])
    pos = engine.random_playouts(seed=71, n=32, min_plies=2, max_plies=40)
    try:
        _reinit(engine, PERFT_NO_GRAPHS="1")
        host = [engine.perft_batch(pos, d) for d in (2, 3, 4)]
        assert engine.stats()["graph_launches"] == 0
        _reinit(engine, PERFT_NO_GRAPHS="0")
        engine.reset_stats()
        for _ in range(3):  # first call captures, later calls replay
            dd = [engine.perft_batch(pos, d) for d in (2, 3, 4)]
            assert all(np.array_equal(a, b) for a, b in zip(host, dd))
            assert engine.perft(p, 5) == int(start["counts"]["5"])
        st = engine.stats()
        assert st["graph_launches"] >= 9  # the three batches per pass; perft(5) of one position is one launch
        assert st["small_launches"] == 3
    finally:
        engine.init(device=0, arena_bytes=8 << 30)


def test_graph_overflow_falls_back(engine, golden):
    """With the size estimate disabled and a 64 MiB arena, the device plan for
    perft(6) of the initial position overflows; the host path recomputes."""
    start = next(e for e in golden if e["name"] == "initial_position")
    p = pos48_from_hex(start["pos48"])
    old = os.environ.get("PERFT_DD_FORCE")
    os.environ["PERFT_DD_FORCE"] = "1"
    try:
        engine.init(device=0, arena_bytes=64 << 20)
        assert engine.perft(p, 6) == int(start["counts"]["6"])
        assert engine.perft(p, 4) == int(start["counts"]["4"])
    finally:
        if old is None:
            os.environ.pop("PERFT_DD_FORCE", None)
        else:
            os.environ["PERFT_DD_FORCE"] = old
        engine.init(device=0, arena_bytes=8 << 30)


def test_mixed_depth_batch_as_one_graph(engine, oracle):
    """A batch of depths 0-5 runs as one graph (deepest roots start, the
    others join the ply of their remaining depth) and equals the host-driven
    path and the oracle; the host-driven path also shares plies across depth
    groups."""
    pos = engine.random_playouts(seed=72, n=120, min_plies=0, max_plies=40)
    depths = (np.arange(len(pos)) * 7 % 6).astype(np.uint8)  # 0..5, interleaved
    want = oracle.perft_batch_mt(pos, depths)
    try:
        _reinit(engine, PERFT_NO_GRAPHS="1")
        engine.reset_stats()
        host = engine.perft_batch(pos, depths)
        st = engine.stats()
        assert st["graph_launches"] == 0
        assert st["leaf_launches"] == 1  # every depth group in one count-only launch
        assert np.array_equal(host, want)
        _reinit(engine, PERFT_NO_GRAPHS="0")
        engine.reset_stats()
        for _ in range(2):
            assert np.array_equal(engine.perft_batch(pos, depths), want)
        st = engine.stats()
        assert st["graph_launches"] == 2
        assert st["leaf_ms"] > 0 and st["leaf_items"] > 0 and st["leaf_parents"] > 0  # timed inside the graph
        # a depth mix with an empty join level and shallow roots only
        d2 = np.where(depths >= 3, 5, depths % 2).astype(np.uint8)
        assert np.array_equal(engine.perft_batch(pos, d2), oracle.perft_batch_mt(pos, d2))
        d3 = (depths % 2).astype(np.uint8)
        assert np.array_equal(engine.perft_batch(pos, d3), oracle.perft_batch_mt(pos, d3))
    finally:
        engine.init(device=0, arena_bytes=8 << 30)


def test_mixed_depth_graph_overflow_falls_back(engine, oracle):
    """With the size prediction disabled and a 64 MiB arena, the plan for a
    mixed batch whose deepest roots need more overflows part-way (after
    roots have joined); the host-driven path recomputes every count, and the
    same call again goes host-driven at once."""
    import os
    pos = engine.random_playouts(seed=73, n=24, min_plies=4, max_plies=30)
    depths = np.array([6 if i < 2 else 2 + i % 4 for i in range(len(pos))], dtype=np.uint8)
    want = oracle.perft_batch_mt(pos, depths)
    old = os.environ.get("PERFT_DD_FORCE")
    os.environ["PERFT_DD_FORCE"] = "1"
    try:
        engine.init(device=0, arena_bytes=64 << 20)
        for _ in range(2):
            assert np.array_equal(engine.perft_batch(pos, depths), want)
    finally:
        if old is None:
            os.environ.pop("PERFT_DD_FORCE", None)
        else:
            os.environ["PERFT_DD_FORCE"] = old
        engine.init(device=0, arena_bytes=8 << 30)
