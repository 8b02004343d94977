"""The callers either side of the batched path, on the GPU: deep perft by host
root split with transposition merging (and its shards), records mode with
resume, and the perft_gpu program (reference CLI and UCI `go perft`).  Every
count must equal the plain engine's and the golden or oracle counts."""
import os
import subprocess

import numpy as np
import pytest

from tests._oracle import ROOT

pytestmark = pytest.mark.gpu

CLI = os.path.join(ROOT, "perft_gpu_b200", "perft_gpu")
# the program runs beside the test process's engine: give it a small arena
ENV = dict(os.environ, PERFT_ARENA_GB="4")


def _by_name(golden, name):
    return next(e for e in golden if e["name"] == name)


@pytest.mark.parametrize("split", [0, 1, 2, 3])
def test_deep_equals_golden(engine, golden, split):
    for e in golden:
        depth = max(int(k) for k in e["counts"])
        depth = min(depth, 6)
        if depth < 1:
            continue
        p = engine.fen_to_pos(e["fen"])
        total, div = engine.deep(p, depth, split)
        assert total == e["counts"][str(depth)], (e["name"], split)
        assert sum(div.values()) == total
        assert set(div) == set(engine.legal_moves(p))


def test_deep_divided_equals_divide(engine):
    pos = engine.random_playouts(seed=31, n=6, min_plies=6, max_plies=24)
    for p in pos:
        total, div = engine.deep(p, 5, 2)
        want = engine.divide(p, 5)
        assert div == want
        assert total == sum(want.values())


def test_deep_start_depth7(engine, golden):
    start = engine.fen_to_pos(engine.START_FEN)
    total, div = engine.deep(start, 7, 3)
    assert total == _by_name(golden, "initial_position")["counts"]["7"] == 3195901860
    assert len(div) == 20


def test_deep_shards_sum_to_whole(engine):
    pos = engine.random_playouts(seed=32, n=3, min_plies=10, max_plies=20)
    for p in pos:
        total, div = engine.deep(p, 6, 2)
        parts = [engine.deep(p, 6, 2, shard=s, n_shards=3) for s in range(3)]
        assert sum(t for t, _ in parts) == total
        for m in div:
            assert sum(d[m] for _, d in parts) == div[m]
        assert all(t > 0 for t, _ in parts)


def test_deep_bad_args(engine):
    start = engine.fen_to_pos(engine.START_FEN)
    for kw in ({"depth": 0}, {"depth": 5, "shard": 2, "n_shards": 2}, {"depth": 5, "n_shards": 0}):
        with pytest.raises(engine.PerftError) as ei:
            engine.deep(start, **kw)
        assert ei.value.status == engine.PERFT_ERR_INVALID_ARG


def _records_file(engine, path, n=40):
    pos = engine.random_playouts(seed=33, n=n, min_plies=4, max_plies=30)
    rng = np.random.default_rng(33)
    occ = rng.integers(1, 10_000, size=n)
    with open(path, "w") as f:
        for p, c in zip(pos, occ):
            f.write(f"{engine.pos_to_fen(p)} {int(c)}\n")
    return pos, occ


def test_records_mode_and_resume(engine, oracle, tmp_path):
    path = str(tmp_path / "records.txt")
    pos, occ = _records_file(engine, path)
    want = oracle.perft_batch_mt(pos, 4)
    assert engine.records(path, 4, batch=16) == len(pos)
    lines = open(path + ".op").read().splitlines()
    src = open(path).read().splitlines()
    assert len(lines) == len(pos)
    for line, s, w, c in zip(lines, src, want, occ):
        head, perft_s, prod_s = line.rsplit(" ", 2)
        assert head == s and int(perft_s) == int(w) and int(prod_s) == int(w) * int(c)
    # interrupted run: keep the first 13 output lines, then resume
    with open(path + ".op", "w") as f:
        f.write("\n".join(lines[:13]) + "\n")
    assert engine.records(path, 4) == len(pos) - 13
    assert open(path + ".op").read().splitlines() == lines
    # nothing left to do
    assert engine.records(path, 4) == 0


def test_records_bad_input(engine, tmp_path):
    with pytest.raises(engine.PerftError) as ei:
        engine.records(str(tmp_path / "missing.txt"), 3)
    assert ei.value.status == engine.PERFT_ERR_NOT_FOUND
    bad = tmp_path / "bad.txt"
    bad.write_text("this is not a fen 12\n")
    with pytest.raises(engine.PerftError) as ei:
        engine.records(str(bad), 3)
    assert ei.value.status == engine.PERFT_ERR_BAD_FEN


def test_cli_perft_lines(golden):
    r = subprocess.run([CLI, "startpos", "6"], capture_output=True, text=True, timeout=300, env=ENV)
    assert r.returncode == 0, r.stderr
    counts = _by_name(golden, "initial_position")["counts"]
    got = {}
    for line in r.stdout.splitlines():
        if line.startswith("Perft("):
            d = int(line[6:8])
            got[d] = int(line.split(":")[1].split(",")[0])
    assert got == {d: counts[str(d)] for d in (3, 4, 5, 6)}


def test_cli_records(tmp_path, engine, oracle):
    path = str(tmp_path / "r.txt")
    pos, occ = _records_file(engine, path, n=10)
    r = subprocess.run([CLI, "--records", path, "3"], capture_output=True, text=True, timeout=300, env=ENV)
    assert r.returncode == 0, r.stderr
    assert "Records done: 10" in r.stdout
    want = oracle.perft_batch_mt(pos, 3)
    got = [int(line.rsplit(" ", 2)[1]) for line in open(path + ".op").read().splitlines()]
    assert got == [int(x) for x in want]


def test_uci_go_perft(engine, oracle):
    script = "position startpos moves e2e4 c7c5 g1f3\ngo perft 4\nquit\n"
    r = subprocess.run([CLI, "--uci"], input=script, capture_output=True, text=True, timeout=300, env=ENV)
    assert r.returncode == 0, r.stderr
    p = engine.position_from_moves(engine.START_FEN, ["e2e4", "c7c5", "g1f3"])
    div = {}
    nodes = None
    for line in r.stdout.splitlines():
        if line.startswith("Nodes searched:"):
            nodes = int(line.split(":")[1])
        elif ": " in line and not line.startswith("info"):
            m, c = line.split(": ")
            div[m] = int(c)
    assert nodes == oracle.perft(p, 4)
    assert div == engine.divide(p, 4)


@pytest.fixture
def stored(engine):
    yield engine
    engine.store_close()


def test_store_resume_skips_finished_subtrees(stored, tmp_path, golden):
    path = str(tmp_path / "deep.store")
    start = stored.fen_to_pos(stored.START_FEN)
    want = _by_name(golden, "initial_position")["counts"]["7"]
    # first run does only half of the frontier (shard 0 of 2), as if stopped midway
    stored.store_open(path)
    half, _ = stored.deep(start, 7, 3, shard=0, n_shards=2)
    first = stored.store_stats()["appended"]
    assert first > 0
    stored.store_close()
    # the resumed run searches only the other half
    stored.store_open(path)
    assert stored.store_stats()["entries"] == first
    total, div = stored.deep(start, 7, 3)
    st = stored.store_stats()
    assert total == want and 0 < half < total
    assert st["hits"] == first and st["appended"] > 0
    stored.store_close()
    # a third run finds everything and launches no leaf kernel
    stored.store_open(path)
    stored.reset_stats()
    again, div2 = stored.deep(start, 7, 3)
    assert again == want and div2 == div
    assert stored.stats()["leaf_launches"] == 0
    assert stored.store_stats()["appended"] == 0


def test_cli_sharded_deep_counts(golden):
    """perft_gpu <fen> <depth> <gpus>: the deep counts split over shard
    processes (all pinned to this GPU here) and summed; divided output from
    depth 7 on, every line equal to the single-process counts."""
    env = dict(ENV, PERFT_DIVIDED_DEPTH="6", PERFT_SHARD_DEVICE="0", PERFT_ARENA_GB="3")
    r = subprocess.run([CLI, "startpos", "7", "3"], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr
    counts = _by_name(golden, "initial_position")["counts"]
    got, div = {}, {}
    for line in r.stdout.splitlines():
        if line.startswith("Perft("):
            got[int(line[6:8])] = int(line.split(":")[1].split(",")[0])
        elif len(line.split()) == 2:
            m, c = line.split()
            div[m] = int(c)
    assert got == {d: counts[str(d)] for d in (3, 4, 5, 6, 7)}
    assert len(div) == 20 and sum(div.values()) == counts["7"]
