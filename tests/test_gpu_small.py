"""One-launch small trees (k_small_tree): a single position of depth 2..5 is
counted in one launch with no level buffers.  Bit-exact against the golden
vectors and the oracle; positions whose depth-5 subtree roots do not fit one
CTA's list fall back to the level pipeline with the same counts."""
import os

import numpy as np
import pytest

from tests._oracle import pos48_from_hex

pytestmark = pytest.mark.gpu


def _reinit(engine, **env):
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        engine.init(device=0, arena_bytes=4 << 30)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def test_golden_positions_in_one_launch(engine, golden):
    engine.reset_stats()
    n = 0
    for e in golden:
        p = pos48_from_hex(e["pos48"])
        for d, c in e["counts"].items():
            if 2 <= int(d) <= 5:
                assert engine.perft(p, int(d)) == int(c), (e["name"], d)
                n += 1
    st = engine.stats()
    assert n > 0 and st["small_launches"] == n
    assert st["leaf_launches"] == 0 and st["graph_launches"] == 0


def test_random_positions_equal_oracle(engine, oracle):
    """Playouts with castling, en passant, promotions, checks and mates, at
    every depth the kernel takes, through the host and the device entry."""
    pos = engine.random_playouts(seed=905, n=48, min_plies=0, max_plies=80)
    for d in (2, 3, 4, 5):
        want = [int(x) for x in oracle.perft_batch_mt(pos, d)]
        got = [engine.perft(p, d) for p in pos]
        assert got == want, d
        dev = [int(engine.perft_batch(p[None, :], d)[0]) for p in pos[:8]]
        assert dev == want[:8], d


def test_many_move_positions(engine, golden, oracle):
    """Positions with the most legal moves: the largest subtree-root lists and
    item windows of more than one pass."""
    pos = engine.random_playouts(seed=906, n=400, min_plies=20, max_plies=60)
    nmoves = np.array([len(engine.legal_moves(p)) for p in pos])
    top = pos[np.argsort(-nmoves)[:6]]
    for d in (3, 4, 5):
        want = [int(x) for x in oracle.perft_batch_mt(top, d)]
        assert [engine.perft(p, d) for p in top] == want, d


def test_list_overflow_falls_back(engine, golden):
    """With room for 64 subtree roots per CTA, perft(5) of the initial
    position (400 roots) does not fit: the level pipeline counts it instead."""
    start = next(e for e in golden if e["name"] == "initial_position")
    p = pos48_from_hex(start["pos48"])
    try:
        _reinit(engine, PERFT_SMALL_LIST_CAP="64")
        engine.reset_stats()
        assert engine.perft(p, 5) == int(start["counts"]["5"])
        assert engine.stats()["small_launches"] == 0
        assert engine.perft(p, 4) == int(start["counts"]["4"])  # depth 4 lists no roots
        assert engine.stats()["small_launches"] == 1
    finally:
        engine.init(device=0, arena_bytes=8 << 30)


def test_disabled_and_enabled_agree(engine, oracle):
    pos = engine.random_playouts(seed=907, n=16, min_plies=4, max_plies=40)
    want = [[int(x) for x in oracle.perft_batch_mt(pos, d)] for d in (2, 5)]
    try:
        _reinit(engine, PERFT_SMALL_TREE="0")
        engine.reset_stats()
        assert [[engine.perft(p, d) for p in pos] for d in (2, 5)] == want
        assert engine.stats()["small_launches"] == 0
    finally:
        engine.init(device=0, arena_bytes=8 << 30)
    engine.reset_stats()
    assert [[engine.perft(p, d) for p in pos] for d in (2, 5)] == want
    assert engine.stats()["small_launches"] == 32


def test_invalid_position_is_refused(engine, golden):
    start = next(e for e in golden if e["name"] == "initial_position")
    p = pos48_from_hex(start["pos48"]).copy()
    p[5] = 0  # no kings
    with pytest.raises(Exception):
        engine.perft(p, 4)
    assert engine.perft(pos48_from_hex(start["pos48"]), 4) == int(start["counts"]["4"])  # still usable
