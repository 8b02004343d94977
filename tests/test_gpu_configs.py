"""Every benchmark configuration pinned to the reference at its own size.

tests/golden/config_counts.json holds the reference's own host perft
(oracle/_ref, perft_bb.h:79-101) on the stored workloads
(perft_gpu_b200/data/workloads.npz), written by
tests/golden/make_config_golden.py:

  * the 4096-position batch, every position at its own depth (4-6);
  * the depth-8 position, as perft(7) of each child (divided perft 8);
  * the 4 transposition-table positions, as perft(7) of each child.

The GPU engine must reproduce each count bit for bit.  Depths 9 and 10 of the
table positions are beyond a CPU run; there the engine's count with the
table must equal the sum over the position's children of an independent
count: the children's no-table perft(8) for depth 9 (checked against the
reference by the divided-perft-8 pin above, one ply shallower), and the
children's perft(9) with a fresh table and an independent Zobrist key set
for depth 10.
"""
import json
import os

import numpy as np
import pytest

from tests._oracle import ROOT

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(ROOT, "tests", "golden", "config_counts.json")
WL = os.path.join(ROOT, "perft_gpu_b200", "data", "workloads.npz")


@pytest.fixture(scope="module")
def cfg_golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def wl():
    with np.load(WL) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture
def big_engine(engine):
    """The engine with the default arena (85% of free HBM); the session's
    8 GiB configuration is restored afterwards."""
    engine.init(device=0)
    yield engine
    engine.init(device=0, arena_bytes=8 << 30)


def _children(pg, pos):
    return np.stack([pg.apply_move(pos, m) for m in pg.legal_moves(pos)])


@pytest.mark.parametrize("graphs", ["1", "0"], ids=["graph", "host_driven"])
def test_batch4096_every_position_equals_reference(engine, wl, cfg_golden, graphs, monkeypatch):
    """The whole batch as one captured graph (the default when its predicted
    levels fit the arena) and host-driven."""
    monkeypatch.setenv("PERFT_NO_GRAPHS", "0" if graphs == "1" else "1")
    monkeypatch.setenv("PERFT_DD_MAX_GB", "1000")
    engine.init(device=0)
    try:
        want = np.array(cfg_golden["batch4096"]["counts"], dtype=np.uint64)
        engine.reset_stats()
        got = engine.perft_batch(wl["batch_pos"], wl["batch_depths"])
        bad = np.nonzero(got != want)[0]
        assert len(bad) == 0, [(int(i), int(got[i]), int(want[i])) for i in bad[:5]]
        st = engine.stats()
        assert st["leaf_launches"] == 1 and (st["graph_launches"] == 1) == (graphs == "1")
    finally:
        monkeypatch.delenv("PERFT_NO_GRAPHS")
        monkeypatch.delenv("PERFT_DD_MAX_GB")
        engine.init(device=0, arena_bytes=8 << 30)


def test_deep_position_divided_perft8_equals_reference(big_engine, wl, cfg_golden):
    g = cfg_golden["deep"]
    pos = wl["deep_pos"].reshape(6)
    ch = _children(big_engine, pos)
    got = big_engine.perft_batch(ch, 7)
    assert sorted(int(x) for x in got) == g["children_sorted"]
    assert big_engine.perft(pos, 8) == g["total"] == int(got.sum())


@pytest.mark.parametrize("i", range(4))
def test_tt_positions_divided_perft8_equals_reference(big_engine, wl, cfg_golden, i):
    g = cfg_golden["tt"][i]
    pos = wl["tt_pos"][i]
    ch = _children(big_engine, pos)
    got = big_engine.perft_batch(ch, 7)
    assert sorted(int(x) for x in got) == g["children_sorted"]
    assert int(got.sum()) == g["total"]
    # the same depth with the 2^30-entry table, cold
    big_engine.init(device=0, tt_log2_entries=30)
    assert big_engine.perft(pos, 8) == g["total"]


def test_tt_depth9_equals_sum_of_children_without_table(big_engine, wl, cfg_golden):
    """perft(9) with the table = sum over children of no-table perft(8)
    (the smallest depth-9 position of the table workload)."""
    i = int(np.argmin([e["total"] for e in cfg_golden["tt"]]))
    pos = wl["tt_pos"][i]
    ch = _children(big_engine, pos)
    plain = big_engine.perft_batch(ch, 8)
    big_engine.init(device=0, tt_log2_entries=30)
    assert big_engine.perft(pos, 9) == int(plain.sum())


def test_tt_depth10_equals_sum_of_children_with_independent_keys(big_engine, wl, cfg_golden):
    """perft(10) with the table = sum over children of perft(9), each child
    counted with a fresh table and an independent Zobrist key set, so a
    false table hit would have to repeat under unrelated keys."""
    i = int(np.argmin([e["total"] if d == 10 else 1 << 62
                       for e, d in zip(cfg_golden["tt"], wl["tt_depths"])]))
    assert wl["tt_depths"][i] == 10
    pos = wl["tt_pos"][i]
    big_engine.init(device=0, tt_log2_entries=30)
    total = big_engine.perft(pos, 10)
    ch = _children(big_engine, pos)
    big_engine.init(device=0, tt_log2_entries=30, zobrist_seed=0x0DDC0FFEE1234567)
    subs = []
    for c in ch:
        big_engine.tt_clear()
        subs.append(big_engine.perft(c, 9))
    assert total == sum(subs)
