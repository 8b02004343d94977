"""GPU parity: the CUDA engine, called through the C ABI, against the oracle.

Bar: bit-exact leaf counts.  Expected values come from the golden fixtures
(generated from the reference's own host perft) and from the clean-room CPU
oracle on seeded positions.
"""
import numpy as np
import pytest

from tests._oracle import pos48_from_hex

pytestmark = pytest.mark.gpu

START_D7 = "7"


def _golden_items(golden, max_leaves=200_000_000):
    for e in golden:
        pos = pos48_from_hex(e["pos48"])
        for d, c in sorted(e["counts"].items(), key=lambda kv: int(kv[0])):
            if c <= max_leaves:
                yield e["name"], pos, int(d), int(c)


def test_golden_counts_single(engine, golden):
    bad = []
    for name, pos, d, c in _golden_items(golden):
        got = engine.perft(pos, d)
        if got != c:
            bad.append((name, d, c, got))
    assert not bad, bad[:10]


def test_golden_counts_batched(engine, golden):
    items = list(_golden_items(golden))
    pos = np.stack([p for _, p, _, _ in items])
    depths = np.array([d for _, _, d, _ in items], dtype=np.uint8)
    want = np.array([c for _, _, _, c in items], dtype=np.uint64)
    got = engine.perft_batch(pos, depths)
    mism = np.nonzero(got != want)[0]
    assert mism.size == 0, [(items[i][0], items[i][2], int(want[i]), int(got[i])) for i in mism[:10]]


def test_golden_divided_depth3(engine, golden):
    for e in golden:
        pos = pos48_from_hex(e["pos48"])
        want = sorted(ch["perft2"] for ch in e["children_perft2"])
        div = engine.divide(pos, 3)
        assert sorted(div.values()) == want, e["name"]


def test_initial_position_depth7(engine, golden):
    start = next(e for e in golden if e["name"] == "initial_position")
    assert engine.perft(pos48_from_hex(start["pos48"]), 7) == int(start["counts"][START_D7])


def test_seeded_playouts_vs_oracle(engine, oracle):
    pos = engine.random_playouts(seed=4242, n=1536, min_plies=0, max_plies=90)
    depths = (np.arange(len(pos)) % 4 + 1).astype(np.uint8)
    got = engine.perft_batch(pos, depths)
    want = oracle.perft_batch_mt(pos, depths)
    mism = np.nonzero(got != want)[0]
    assert mism.size == 0, [(engine.pos_to_fen(pos[i]), int(depths[i]), int(want[i]), int(got[i]))
                            for i in mism[:10]]


def test_stratified_batch_sample_vs_oracle(engine, oracle):
    from perft_gpu_b200 import workloads
    pos, depths = workloads.batch_positions(n=512, seed=77)
    d = np.minimum(depths, 4).astype(np.uint8)
    got = engine.perft_batch(pos, d)
    want = oracle.perft_batch_mt(pos, d)
    assert np.array_equal(got, want)


def test_batch_equals_single(engine):
    pos = engine.random_playouts(seed=99, n=24, min_plies=5, max_plies=40)
    depths = np.array([1 + i % 5 for i in range(24)], dtype=np.uint8)
    batch = engine.perft_batch(pos, depths)
    single = [engine.perft(p, int(d)) for p, d in zip(pos, depths)]
    assert [int(x) for x in batch] == single


def test_depth_zero_and_one(engine, oracle):
    pos = engine.random_playouts(seed=5, n=64, min_plies=0, max_plies=60)
    assert all(x == 1 for x in engine.perft_batch(pos, 0))
    got = engine.perft_batch(pos, 1)
    assert [int(x) for x in got] == [oracle.count(p) for p in pos]


def test_terminal_positions(engine, golden):
    for name in ("stalemate", "back_rank_mate"):
        e = next(x for x in golden if x["name"] == name)
        p = pos48_from_hex(e["pos48"])
        assert [engine.perft(p, d) for d in range(0, 6)] == [1, 0, 0, 0, 0, 0]


def test_empty_batch(engine):
    out = engine.perft_batch(np.zeros((0, 6), dtype=np.uint64), np.zeros(0, dtype=np.uint8))
    assert out.shape == (0,)


def test_invalid_positions_rejected(engine):
    start = engine.fen_to_pos(engine.START_FEN)
    no_king = start.copy()
    no_king[5] = np.uint64(int(start[5]) & ~(1 << 4))  # remove the white king
    with pytest.raises(engine.PerftError) as ei:
        engine.perft(no_king, 3)
    assert ei.value.status == engine.PERFT_ERR_INVALID_ARG
    # the side not to move in check: black to move while the white king is attacked
    bad = engine.fen_to_pos("4k3/8/8/8/8/8/8/r3K3 w - - 0 1")
    bad[1] = np.uint64(int(bad[1]) | (1 << 63))
    with pytest.raises(engine.PerftError):
        engine.perft(bad, 2)
    # the engine stays usable after a rejected call
    assert engine.perft(start, 3) == 8902


def test_divide_sums_to_perft(engine):
    pos = engine.random_playouts(seed=31, n=6, min_plies=10, max_plies=30)
    for p in pos:
        div = engine.divide(p, 4)
        assert sum(div.values()) == engine.perft(p, 4)
        assert sorted(div) == sorted(engine.legal_moves(p))


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4], ids=["kogge", "magic", "kogge_fma", "kogge_split", "hybrid"])
def test_slider_variants(engine, golden, oracle, variant):
    """Every slider variant, on interior and last plies alike, is bit-exact."""
    engine.init(device=0, arena_bytes=2 << 30, sliders_expand=variant, sliders_leaf=variant)
    try:
        st = engine.stats()
        assert st["sliders_leaf"] == variant and st["sliders_expand"] == variant
        items = list(_golden_items(golden, max_leaves=20_000_000))
        pos = np.stack([p for _, p, _, _ in items])
        depths = np.array([d for _, _, d, _ in items], dtype=np.uint8)
        want = np.array([c for _, _, _, c in items], dtype=np.uint64)
        assert np.array_equal(engine.perft_batch(pos, depths), want)
        rnd = engine.random_playouts(seed=600 + variant, n=256, min_plies=0, max_plies=80)
        d = (np.arange(256) % 4 + 1).astype(np.uint8)
        assert np.array_equal(engine.perft_batch(rnd, d), oracle.perft_batch_mt(rnd, d))
    finally:
        engine.init(device=0, arena_bytes=8 << 30)


def test_autotuner_choice_is_reported(engine):
    st = engine.stats()
    assert st["sliders_leaf"] in engine.SLIDER_NAMES and st["sliders_expand"] in engine.SLIDER_NAMES


def test_small_arena_chunks_levels(engine, golden):
    """A 6 MiB arena cannot hold the 197,281-node ply of the initial position:
    the level is split at tile boundaries and expanded depth-first."""
    engine.init(device=0, arena_bytes=6 << 20)
    try:
        engine.reset_stats()
        start = next(e for e in golden if e["name"] == "initial_position")
        p = pos48_from_hex(start["pos48"])
        assert engine.perft(p, 6) == int(start["counts"]["6"])
        assert engine.stats()["chunked_levels"] > 0
    finally:
        engine.init(device=0, arena_bytes=8 << 30)


def test_many_move_positions(engine, oracle):
    """94-170 legal moves per node (and the colour mirrors): single calls,
    one batch and every slider variant against the oracle."""
    from tests._positions import many_moves_with_mirrors
    pos = [engine.fen_to_pos(f) for f in many_moves_with_mirrors()]
    want = {d: [oracle.perft(p, d) for p in pos] for d in (1, 2, 3)}
    for d in (1, 2, 3):
        assert [engine.perft(p, d) for p in pos] == want[d]
        assert [int(x) for x in engine.perft_batch(pos, d)] == want[d]
    for v in range(5):
        engine.init(device=0, arena_bytes=8 << 30, sliders_expand=v, sliders_leaf=v)
        assert [int(x) for x in engine.perft_batch(pos, 3)] == want[3], v
    engine.init(device=0, arena_bytes=8 << 30)
    d4 = engine.perft_batch(pos[:2], 4)
    assert [int(x) for x in d4] == [oracle.perft(p, 4) for p in pos[:2]]


def test_colour_mirror_property(engine):
    """Size-independent property at sizes the oracle cannot reach quickly:
    a position and its colour mirror (ranks reversed, colours and side to
    move swapped) have the same perft, here at depth 5 over 64 playouts."""
    from tests._positions import mirror_fen
    pos = engine.random_playouts(seed=51, n=64, min_plies=6, max_plies=40)
    mir = np.stack([engine.fen_to_pos(mirror_fen(engine.pos_to_fen(p))) for p in pos])
    a = engine.perft_batch(pos, 5)
    b = engine.perft_batch(mir, 5)
    assert np.array_equal(a, b)
    assert int(a.sum()) > 10**9
