"""Transposition-table perft: bit-exact against the no-table counts and the
golden vectors, with a warm table, a tiny (heavily overwritten) table, and
same-level duplicates inside a batch."""
import numpy as np
import pytest

from tests._oracle import pos48_from_hex

pytestmark = pytest.mark.gpu


@pytest.fixture
def tt_engine(engine):
    engine.init(device=0, arena_bytes=4 << 30, tt_log2_entries=22)
    yield engine
    engine.init(device=0, arena_bytes=8 << 30)


def _golden(golden, max_leaves=50_000_000):
    items = [(pos48_from_hex(e["pos48"]), int(d), int(c)) for e in golden
             for d, c in e["counts"].items() if int(c) <= max_leaves]
    pos = np.stack([p for p, _, _ in items])
    depths = np.array([d for _, d, _ in items], dtype=np.uint8)
    want = np.array([c for _, _, c in items], dtype=np.uint64)
    return pos, depths, want


def test_tt_matches_golden_cold_and_warm(tt_engine, golden):
    pos, depths, want = _golden(golden)
    tt_engine.tt_clear()
    assert np.array_equal(tt_engine.perft_batch(pos, depths), want)
    tt_engine.reset_stats()
    assert np.array_equal(tt_engine.perft_batch(pos, depths), want)  # warm: answered from the table
    st = tt_engine.stats()
    assert st["tt_entries"] == 1 << 22 and st["tt_hits"] > 0


@pytest.mark.parametrize("small", ["1", "0"], ids=["small_tree", "table_levels"])
def test_tt_single_positions_match_no_tt(tt_engine, oracle, small, monkeypatch):
    """Single positions of depth 2-5 take the one-launch small-tree kernel
    even with a table; with that kernel off they run the table levels."""
    monkeypatch.setenv("PERFT_SMALL_TREE", small)
    tt_engine.init(device=0, arena_bytes=4 << 30, tt_log2_entries=22)
    pos = tt_engine.random_playouts(seed=808, n=40, min_plies=6, max_plies=40)
    tt_engine.reset_stats()
    for d in (2, 3, 4, 5):
        want = oracle.perft_batch_mt(pos[:8], d)
        got = [tt_engine.perft(p, d) for p in pos[:8]]
        assert got == [int(x) for x in want], d
    st = tt_engine.stats()
    assert st["small_launches"] == (32 if small == "1" else 0)
    assert (st["tt_probes"] > 0) == (small == "0")
    depths = np.array([5] * 40, dtype=np.uint8)
    got = tt_engine.perft_batch(pos, depths)
    assert np.array_equal(got, oracle.perft_batch_mt(pos, 5))
    tt_engine.init(device=0, arena_bytes=4 << 30)  # no table
    want = tt_engine.perft_batch(pos, depths)
    assert np.array_equal(got, want)


def test_tt_duplicates_in_batch(tt_engine, golden):
    start = next(e for e in golden if e["name"] == "initial_position")
    p = pos48_from_hex(start["pos48"])
    pos = np.stack([p] * 5)
    tt_engine.tt_clear()
    tt_engine.reset_stats()
    got = tt_engine.perft_batch(pos, np.array([6, 6, 5, 6, 5], dtype=np.uint8))
    assert [int(x) for x in got] == [int(start["counts"]["6"])] * 2 + [int(start["counts"]["5"]),
                                                                        int(start["counts"]["6"]),
                                                                        int(start["counts"]["5"])]
    assert tt_engine.stats()["tt_duplicates"] > 0


def test_tiny_table_stays_exact(engine, golden):
    engine.init(device=0, arena_bytes=2 << 30, tt_log2_entries=10)
    try:
        pos, depths, want = _golden(golden, max_leaves=5_000_000)
        for _ in range(2):
            assert np.array_equal(engine.perft_batch(pos, depths), want)
    finally:
        engine.init(device=0, arena_bytes=8 << 30)


def test_tt_with_chunked_levels(engine, golden):
    engine.init(device=0, arena_bytes=8 << 20, tt_log2_entries=16)
    try:
        start = next(e for e in golden if e["name"] == "initial_position")
        engine.reset_stats()
        assert engine.perft(pos48_from_hex(start["pos48"]), 6) == int(start["counts"]["6"])
        assert engine.stats()["chunked_levels"] > 0
    finally:
        engine.init(device=0, arena_bytes=8 << 30)


def test_slot_key_collisions_stay_exact(engine, golden, oracle):
    """Only 10 bits of the slot key kept: thousands of different positions
    share each table slot and each de-duplication slot, so every hit and
    every merge rests on the independent verification key."""
    import os
    os.environ["PERFT_TT_INDEX_KEY_BITS"] = "10"
    try:
        engine.init(device=0, arena_bytes=2 << 30, tt_log2_entries=16)
        pos, depths, want = _golden(golden, max_leaves=5_000_000)
        engine.reset_stats()
        for _ in range(2):
            assert np.array_equal(engine.perft_batch(pos, depths), want)
        st = engine.stats()
        assert st["tt_hits"] > 0 and st["tt_duplicates"] > 0
        play = engine.random_playouts(seed=41, n=24, min_plies=4, max_plies=30)
        got = engine.perft_batch(play, 4)
        assert [int(x) for x in got] == [oracle.perft(p, 4) for p in play]
    finally:
        os.environ.pop("PERFT_TT_INDEX_KEY_BITS", None)
        engine.init(device=0, arena_bytes=8 << 30)
