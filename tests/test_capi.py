"""The C-ABI library without a GPU: it loads, exports every entry point that
include/perft_b200.h declares, and its host utilities (FEN, UCI moves,
playouts, features) agree with the oracle.  No compute call needs a GPU here;
GPU-only calls must fail with a status code, not crash."""
import ctypes
import os
import re

import numpy as np
import pytest

import perft_gpu_b200 as pg
from tests._oracle import ROOT, pos48_from_hex

HEADER = os.path.join(ROOT, "include", "perft_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(perft_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    names = _declared()
    lib = ctypes.CDLL(pg.LIB_PATH)
    missing = [n for n in names + ["perft"] if not hasattr(lib, n)]
    assert not missing, missing
    assert len(names) >= 15


def test_probe_library_exports():
    lib = ctypes.CDLL(os.path.join(ROOT, "perft_gpu_b200", "libperft_probe.so"))
    assert hasattr(lib, "perft_int32_peak_probe")


def test_status_strings():
    for code in range(0, -13, -1):
        assert pg._status_string(code) != "unknown status"


def test_fen_roundtrip_and_oracle_parse(oracle, golden):
    for e in golden:
        p = pg.fen_to_pos(e["fen"])
        assert np.array_equal(p, oracle.fen_to_pos(e["fen"])), e["name"]
        assert pg.pos_to_fen(p) == e["fen"], e["name"]


def test_bad_fen_rejected():
    # placement errors, unknown letters, missing kings, pawns on the back rank
    for fen in ("", "not a fen", "8/8/8/8/8/8/8/8 w - - 0 1", "4k3/8/8/8/8/8/8/4K2P w - - 0 1",
                "4k3/8/8/8/8/8/8/4KK2 w - - 0 1"):
        with pytest.raises(pg.PerftError) as ei:
            pg.fen_to_pos(fen)
        assert ei.value.status in (pg.PERFT_ERR_BAD_FEN, pg.PERFT_ERR_INVALID_ARG)


def test_legal_moves_and_apply_vs_oracle(oracle):
    pos = pg.random_playouts(seed=8, n=200, min_plies=0, max_plies=80)
    for p in pos:
        moves = pg.legal_moves(p)
        assert len(moves) == oracle.count(p)
        kids = sorted(tuple(int(x) for x in c) for c in oracle.children(p))
        mine = sorted(tuple(int(x) for x in pg.apply_move(p, m)) for m in moves)
        assert mine == kids


def test_apply_illegal_move():
    start = pg.fen_to_pos(pg.START_FEN)
    with pytest.raises(pg.PerftError) as ei:
        pg.apply_move(start, "e2e5")
    assert ei.value.status == pg.PERFT_ERR_ILLEGAL_MOVE


def test_promotion_and_castling_uci():
    p = pg.fen_to_pos("r3k3/1P6/8/8/8/8/6p1/4K2R w K - 0 1")
    moves = pg.legal_moves(p)
    assert {"b7b8q", "b7b8r", "b7b8b", "b7b8n", "b7a8q"} <= set(moves)
    assert "e1g1" not in moves  # f1 is attacked by the g2 pawn
    c = pg.fen_to_pos("r3k3/1P6/8/8/8/8/8/4K2R w K - 0 1")
    assert "e1g1" in pg.legal_moves(c)
    q = pg.apply_move(c, "e1g1")
    assert pg.pos_to_fen(q).startswith("r3k3/1P6/8/8/8/8/8/5RK1 b -")
    bp = pg.apply_move(pg.fen_to_pos("r3k3/1P6/8/8/8/8/6p1/4K2R b K - 0 1"), "g2h1n")
    assert pg.pos_to_fen(bp).startswith("r3k3/1P6/8/8/8/8/8/4K2n w -")


def test_playouts_deterministic_and_legal(oracle):
    a = pg.random_playouts(seed=123, n=50, min_plies=8, max_plies=30)
    b = pg.random_playouts(seed=123, n=50, min_plies=8, max_plies=30)
    assert np.array_equal(a, b)
    assert all(oracle.count(p) > 0 for p in a)


def test_features():
    ep = pg.fen_to_pos("8/8/8/2k5/3Pp3/8/8/4K3 b - d3 0 1")
    f = pg.features(ep)
    assert f & pg.FEATURE_EP and f & pg.FEATURE_IN_CHECK
    assert pg.features(pg.fen_to_pos(pg.START_FEN)) == pg.FEATURE_CASTLING
    pr = pg.features(pg.fen_to_pos("r3k3/1P6/8/8/8/8/6p1/4K2R w K - 0 1"))
    assert pr & pg.FEATURE_PAWN_ON_7TH and pr & pg.FEATURE_PROMOTION


def test_batch_workload_stratification():
    from perft_gpu_b200 import workloads
    pos, depths = workloads.batch_positions(n=400, seed=3)
    f = np.array([pg.features(p) for p in pos])
    for bit in (pg.FEATURE_EP, pg.FEATURE_PAWN_ON_7TH, pg.FEATURE_CASTLING):
        assert (f & bit != 0).mean() >= 0.10
    assert set(np.unique(depths)) <= {4, 5, 6}
    pos2, depths2 = workloads.batch_positions(n=400, seed=3)
    assert np.array_equal(pos, pos2) and np.array_equal(depths, depths2)


def test_gpu_calls_fail_cleanly_without_engine():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present; covered by the gpu tests")
    with pytest.raises(pg.PerftError) as ei:
        pg.init()
    assert ei.value.status == pg.PERFT_ERR_NO_DEVICE
    with pytest.raises(pg.PerftError) as ei:
        pg.perft(pg.fen_to_pos(pg.START_FEN), 3)
    assert ei.value.status == pg.PERFT_ERR_NOT_INITIALIZED
    fn = pg.lib().perft_batch_noalloc
    fn.restype = ctypes.c_int
    d = np.array([3], dtype=np.uint8)
    rc = fn(ctypes.c_void_p(16), ctypes.c_void_p(d.ctypes.data), 1, ctypes.c_void_p(16), None)
    assert rc == pg.PERFT_ERR_NO_DEVICE
