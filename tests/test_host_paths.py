"""The host side of the C ABI end to end on the CPU: divided and deep perft
with transposition merging, shards, the result store (also shared by several
processes at once), records mode with resume, and engine failures.  The
library under test is host.cpp linked against a stand-in engine that counts
with the product's move generator compiled for the host
(tests/hostapi/stub_engine.cpp); the oracle checks every count."""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

import perft_gpu_b200 as pg
from tests._oracle import ROOT

API_DIR = os.path.join(ROOT, "tests", "hostapi")
API_LIB = os.path.join(API_DIR, "libhostapi.so")
SOURCES = [os.path.join(API_DIR, "stub_engine.cpp"), os.path.join(ROOT, "perft_gpu_b200", "csrc", "host.cpp"),
           os.path.join(ROOT, "perft_gpu_b200", "csrc", "tables.cpp")]
HEADERS = [os.path.join(ROOT, "perft_gpu_b200", "csrc", "movegen.cuh"), os.path.join(ROOT, "include", "perft_b200.h")]


def build_hostapi():
    if not os.path.exists(API_LIB) or any(os.path.getmtime(s) > os.path.getmtime(API_LIB) for s in SOURCES + HEADERS):
        subprocess.run(["g++", "-O2", "-std=c++20", "-fPIC", "-shared", "-o", API_LIB] + SOURCES, check=True)
    return API_LIB


def bind_hostapi():
    lib = pg._bind(ctypes.CDLL(build_hostapi()))
    lib.hostapi_counters.argtypes = [ctypes.POINTER(ctypes.c_uint64)] * 2
    lib.hostapi_fail_after.argtypes = [ctypes.c_longlong, ctypes.c_int]
    lib.hostapi_scale.argtypes = [ctypes.c_uint64]
    lib.hostapi_init()
    return lib


@pytest.fixture
def api(monkeypatch):
    lib = bind_hostapi()
    monkeypatch.setattr(pg, "_lib_handle", lib)
    lib.hostapi_fail_after(-1, 0)
    lib.hostapi_scale(1)
    lib.hostapi_reset_counters()
    yield lib
    lib.hostapi_fail_after(-1, 0)
    lib.hostapi_scale(1)
    pg.store_close()


def counted(lib):
    b, p = ctypes.c_uint64(), ctypes.c_uint64()
    lib.hostapi_counters(ctypes.byref(b), ctypes.byref(p))
    return b.value, p.value


def positions():
    start = pg.fen_to_pos(pg.START_FEN)
    kiwi = pg.fen_to_pos("r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq - 0 1")
    return [start, kiwi] + list(pg.random_playouts(seed=5, n=4, min_plies=8, max_plies=30))


def test_deep_and_divide_match_oracle(api, oracle):
    for pos in positions():
        for depth, split in ((3, 1), (4, 1), (4, 2)):
            total, div = pg.deep(pos, depth, split)
            assert total == oracle.perft(pos, depth)
            kids = oracle.children(pos)
            assert sorted(div.values()) == sorted(oracle.perft(c, depth - 1) for c in kids)
            assert pg.divide(pos, depth) == div
            boards, paths = pg.deep_frontier(pos, depth, split)
            assert paths == oracle.perft(pos, split + 1) and boards <= paths


def test_shards_split_the_frontier(api):
    pos = positions()[1]
    whole_total, whole = pg.deep(pos, 4, 2)
    boards, _ = pg.deep_frontier(pos, 4, 2)
    for n in (2, 3, 5):
        api.hostapi_reset_counters()
        acc = dict.fromkeys(whole, 0)
        for s in range(n):
            _, div = pg.deep(pos, 4, 2, shard=s, n_shards=n)
            for m, c in div.items():
                acc[m] += c
        assert acc == whole and sum(acc.values()) == whole_total
        assert counted(api)[1] == boards  # every distinct frontier board searched by exactly one shard


def test_store_resume_skips_searched_boards(api, tmp_path):
    path = str(tmp_path / "run.store")
    pos = positions()[0]
    pg.store_open(path)
    total, div = pg.deep(pos, 5, 2)
    boards, _ = pg.deep_frontier(pos, 5, 2)
    st = pg.store_stats()
    assert st["entries"] == boards and st["appended"] == boards and st["hits"] == 0
    pg.store_close()
    assert os.path.getsize(path) == 64 * (1 + boards)
    api.hostapi_reset_counters()
    pg.store_open(path)
    assert pg.deep(pos, 5, 2) == (total, div)
    assert counted(api)[1] == 0
    assert pg.store_stats()["hits"] == boards


_WORKER = r"""
import ctypes, sys
sys.path.insert(0, {root!r})
import perft_gpu_b200 as pg
from tests.test_host_paths import bind_hostapi
pg._lib_handle = bind_hostapi()
shard, n, path = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3]
pg.store_open(path)
for pos in pg.random_playouts(seed=41, n=40, min_plies=6, max_plies=24):
    pg.deep(pos, 4, 1, shard=shard, n_shards=n)
pg.store_close()
"""


def test_store_shared_by_concurrent_shard_processes(api, tmp_path):
    """Four shard processes append to one store file at once (the CLI's
    multi-GPU split with PERFT_STORE): every batch lands whole, and a later
    single-process run finds every board."""
    path = str(tmp_path / "shared.store")
    n = 4
    script = _WORKER.format(root=ROOT)
    procs = [subprocess.Popen([sys.executable, "-c", script, str(s), str(n), path]) for s in range(n)]
    assert [p.wait(timeout=300) for p in procs] == [0] * n
    size = os.path.getsize(path)
    assert size % 64 == 0
    api.hostapi_reset_counters()
    pg.store_open(path)
    entries = pg.store_stats()["entries"]
    assert os.path.getsize(path) == size  # nothing torn or corrupt was cut off
    want_boards = 0
    for pos in pg.random_playouts(seed=41, n=40, min_plies=6, max_plies=24):
        total, _ = pg.deep(pos, 4, 1)
        want_boards += pg.deep_frontier(pos, 4, 1)[0]
    assert counted(api)[1] == 0  # every frontier board was found in the store
    assert size // 64 - 1 >= entries > 0
    assert pg.store_stats()["hits"] == want_boards


def _records(tmp_path, n=12):
    src = tmp_path / "records.txt"
    pos = pg.random_playouts(seed=9, n=n, min_plies=4, max_plies=30)
    occ = [1 + (7 * i) % 13 for i in range(n)]
    with open(src, "w") as f:
        for p, c in zip(pos, occ):
            f.write(f"{pg.pos_to_fen(p)} {c}\n")
    return str(src), pos, occ


def test_records_end_to_end_and_resume(api, tmp_path, oracle):
    src, pos, occ = _records(tmp_path)
    assert pg.records(src, 3, batch=5) == len(pos)
    lines = open(src + ".op").read().splitlines()
    for line, p, c in zip(lines, pos, occ):
        _, perft_s, prod_s = line.rsplit(" ", 2)
        assert int(perft_s) == oracle.perft(p, 3) and int(prod_s) == int(perft_s) * c
    # stopped in the middle of writing line 8: resumes with record 8
    full = open(src + ".op").read()
    cut = full.index(lines[7]) + 20
    with open(src + ".op", "w") as f:
        f.write(full[:cut])
    assert pg.records(src, 3, batch=5) == len(pos) - 7
    assert open(src + ".op").read() == full


def test_engine_failure_stops_records_cleanly(api, tmp_path):
    src, pos, _ = _records(tmp_path)
    api.hostapi_fail_after(1, pg.PERFT_ERR_CUDA)
    with pytest.raises(pg.PerftError) as ei:
        pg.records(src, 2, batch=4)
    assert ei.value.status == pg.PERFT_ERR_CUDA
    assert len(open(src + ".op").read().splitlines()) == 4  # the first batch only
    api.hostapi_fail_after(-1, 0)
    assert pg.records(src, 2, batch=4) == len(pos) - 4
    clean = tmp_path / "clean"
    clean.mkdir()
    src2, _, _ = _records(clean)
    pg.records(src2, 2)
    assert open(src + ".op").read() == open(src2 + ".op").read()


def test_engine_failure_leaves_store_usable(api, tmp_path):
    path = str(tmp_path / "f.store")
    pos = positions()
    pg.store_open(path)
    pg.deep(pos[0], 4, 1)
    api.hostapi_fail_after(0, pg.PERFT_ERR_OUT_OF_MEMORY)
    with pytest.raises(pg.PerftError) as ei:
        pg.deep(pos[1], 4, 1)
    assert ei.value.status == pg.PERFT_ERR_OUT_OF_MEMORY
    api.hostapi_fail_after(-1, 0)
    pg.store_close()
    pg.store_open(path)
    assert pg.store_stats()["entries"] == pg.deep_frontier(pos[0], 4, 1)[0]
    assert pg.deep(pos[1], 4, 1)[0] == pg.deep(pos[1], 4, 1)[0]


def test_deep_argument_checks(api, oracle):
    pos = positions()[0]
    for depth, split, shard, n in ((0, 1, 0, 1), (31, 1, 0, 1), (4, 1, 1, 1), (4, 1, 0, 0)):
        with pytest.raises(pg.PerftError) as ei:
            pg.deep(pos, depth, split, shard=shard, n_shards=n)
        assert ei.value.status == pg.PERFT_ERR_INVALID_ARG
    # a split at or below the depth is clamped to one ply above the leaves
    assert pg.deep(pos, 3, 7) == pg.deep(pos, 3, 2)
    assert pg.deep(pos, 1, 3)[0] == oracle.perft(pos, 1)
    bad = pos.copy()
    bad[5] = 0  # no kings
    with pytest.raises(pg.PerftError) as ei:
        pg.deep(bad, 3, 1)
    assert ei.value.status == pg.PERFT_ERR_INVALID_ARG


# ------------------------------------------------- the perft_gpu program
CLI_HOST = os.path.join(API_DIR, "perft_gpu_host")
CLI_SRC = os.path.join(ROOT, "perft_gpu_b200", "csrc", "cli.cpp")


@pytest.fixture(scope="module")
def cli():
    """cli.cpp linked against the host test library."""
    build_hostapi()
    if not os.path.exists(CLI_HOST) or os.path.getmtime(CLI_HOST) < max(os.path.getmtime(CLI_SRC),
                                                                         os.path.getmtime(API_LIB)):
        subprocess.run(["g++", "-O2", "-std=c++17", "-o", CLI_HOST, CLI_SRC, "-L", API_DIR, "-lhostapi",
                        "-Wl,-rpath,$ORIGIN"], check=True)
    return CLI_HOST


def run_cli(cli, *args, env=None, stdin=None):
    e = {k: v for k, v in os.environ.items() if not k.startswith(("PERFT_", "HOSTAPI_"))}
    e.update(env or {})
    return subprocess.run([cli, *args], capture_output=True, text=True, timeout=120, env=e, input=stdin)


def parse_cli(out):
    totals, div = {}, {}
    for line in out.splitlines():
        if line.startswith("Perft("):
            totals[int(line[6:8])] = int(line.split(":")[1].split(",")[0])
        elif len(line.split()) == 2:
            m, c = line.split()
            div[m] = int(c)
    return totals, div


def test_cli_lines_divided_and_sharded(cli, golden):
    counts = next(e for e in golden if e["name"] == "initial_position")["counts"]
    r = run_cli(cli, "startpos", "5")
    assert r.returncode == 0, r.stderr
    assert parse_cli(r.stdout)[0] == {d: counts[str(d)] for d in (3, 4, 5)}
    outs = []
    for gpus in ("1", "3"):
        r = run_cli(cli, "startpos", "5", gpus, env={"PERFT_DIVIDED_DEPTH": "3"})
        assert r.returncode == 0, r.stderr
        totals, div = parse_cli(r.stdout)
        assert totals == {d: counts[str(d)] for d in (3, 4, 5)}
        assert len(div) == 20 and sum(div.values()) == counts["5"]
        outs.append([line for line in r.stdout.splitlines() if not line.startswith("Perft(")])
    assert outs[0] == outs[1]  # shard processes reproduce the one-process divided lines


def test_cli_shards_share_one_store(cli, api, tmp_path):
    path = str(tmp_path / "cli.store")
    env = {"PERFT_DIVIDED_DEPTH": "3", "PERFT_STORE": path}
    first = run_cli(cli, "startpos", "5", "3", env=env)
    assert first.returncode == 0, first.stderr
    size = os.path.getsize(path)
    again = run_cli(cli, "startpos", "5", "3", env=env)
    assert again.returncode == 0, again.stderr
    assert parse_cli(again.stdout) == parse_cli(first.stdout)
    assert os.path.getsize(path) == size  # the second run found every board and appended nothing
    pg.store_open(path)
    start = pg.fen_to_pos(pg.START_FEN)
    assert pg.store_stats()["entries"] == pg.deep_frontier(start, 4, 1)[0] + pg.deep_frontier(start, 5, 1)[0]


def test_cli_failed_shard_fails_the_run(cli):
    """One shard process whose engine calls fail: the run reports an error
    and exits non-zero instead of printing a partial count."""
    r = run_cli(cli, "startpos", "5", "3", env={"PERFT_DIVIDED_DEPTH": "3", "HOSTAPI_FAIL_DEVICE": "1"})
    assert r.returncode != 0
    assert "shard 1 failed" in r.stderr
    assert "Perft(04)" not in r.stdout and "Perft(05)" not in r.stdout


def test_cli_records_and_uci(cli, tmp_path, oracle):
    src, pos, occ = _records(tmp_path, n=6)
    r = run_cli(cli, "--records", src, "3")
    assert r.returncode == 0, r.stderr
    lines = open(src + ".op").read().splitlines()
    assert [int(line.rsplit(" ", 2)[1]) for line in lines] == [oracle.perft(p, 3) for p in pos]
    script = "uci\nisready\nposition startpos moves e2e4 c7c5 g1f3\ngo perft 3\nquit\n"
    r = run_cli(cli, "--uci", stdin=script)
    assert r.returncode == 0, r.stderr
    p = pg.position_from_moves(pg.START_FEN, ["e2e4", "c7c5", "g1f3"])
    div, nodes = {}, None
    for line in r.stdout.splitlines():
        if line.startswith("Nodes searched:"):
            nodes = int(line.split(":")[1])
        elif ": " in line and not line.startswith("info"):
            m, c = line.split(": ")
            div[m] = int(c)
    assert nodes == oracle.perft(p, 3)
    assert sorted(div.values()) == sorted(oracle.perft(c, 2) for c in oracle.children(p))


U64_MAX = (1 << 64) - 1


def test_totals_beyond_64_bits(api, oracle):
    """Counts scaled so that every per-move subtotal fits 64 bits but the
    total does not: exact subtotals and an exact wide total.  Scaled further,
    a subtotal itself overflows and the call fails with no subtotals."""
    start = pg.fen_to_pos(pg.START_FEN)
    total, div = pg.deep(start, 4, 1)
    k = U64_MAX // max(div.values())
    assert k * total > U64_MAX
    api.hostapi_scale(k)
    wide, wdiv = pg.deep(start, 4, 1)
    assert wdiv == {m: c * k for m, c in div.items()} and wide == k * total
    # every frontier board's count still fits; the largest per-move sum does not
    biggest_board = max(oracle.perft(g, 2) for c in oracle.children(start) for g in oracle.children(c))
    k2 = U64_MAX // biggest_board
    assert max(div.values()) * k2 > U64_MAX
    api.hostapi_scale(k2)
    with pytest.raises(pg.PerftError) as ei:
        pg.deep(start, 4, 1)
    assert ei.value.status == pg.PERFT_ERR_OVERFLOW


def test_cli_prints_wide_totals(cli, golden, oracle):
    counts = next(e for e in golden if e["name"] == "initial_position")["counts"]
    start = pg.fen_to_pos(pg.START_FEN)
    k = U64_MAX // max(oracle.perft(c, 3) for c in oracle.children(start))  # every depth-4 subtotal fits
    for gpus in ("1", "2"):
        r = run_cli(cli, "startpos", "4", gpus, env={"PERFT_DIVIDED_DEPTH": "3", "HOSTAPI_SCALE": str(k)})
        assert r.returncode == 0, r.stderr
        totals, div = parse_cli(r.stdout)
        assert totals == {3: counts["3"] * k, 4: counts["4"] * k}
        assert totals[4] > U64_MAX and sum(div.values()) == totals[4]


def test_cli_uci_edge_cases(cli, oracle):
    kiwi = "r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq - 0 1"
    mate = "rnb1kbnr/pppp1ppp/8/4p3/6Pq/5P2/PPPPP2P/RNBQKBNR w KQkq - 1 3"
    script = "\n".join([
        "ucinewgame",
        f"position fen {kiwi} moves e1g1 a8b8",
        "d",
        "position startpos moves e2e4 e2e5",   # second move illegal: position unchanged
        "d",
        "position fen not/a/fen",
        "go perft 0",
        "flip",
        f"position fen {mate}",
        "go perft 2",
        "quit",
    ]) + "\n"
    r = run_cli(cli, "--uci", stdin=script)
    assert r.returncode == 0, r.stderr
    out = r.stdout.splitlines()
    fens = [line[5:] for line in out if line.startswith("Fen: ")]
    after = pg.position_from_moves(kiwi, ["e1g1", "a8b8"])
    assert fens[0] == pg.pos_to_fen(after)
    assert fens[1] == fens[0]
    assert "info string illegal move e2e5" in out
    assert "info string bad fen" in out
    assert "info string bad depth" in out
    assert "info string unknown command flip" in out
    assert "Nodes searched: 0" in out  # checkmated: no moves, no leaves
    assert oracle.perft(pg.fen_to_pos(mate), 1) == 0


def test_divide_edges(api):
    start = pg.fen_to_pos(pg.START_FEN)
    assert pg.divide(start, 1) == {m: 1 for m in pg.legal_moves(start)}
    for depth in (0, 40):
        with pytest.raises(pg.PerftError) as ei:
            pg.divide(start, depth)
        assert ei.value.status == pg.PERFT_ERR_INVALID_ARG
    mate = pg.fen_to_pos("rnb1kbnr/pppp1ppp/8/4p3/6Pq/5P2/PPPPP2P/RNBQKBNR w KQkq - 1 3")
    assert pg.divide(mate, 3) == {} and pg.deep(mate, 3, 1) == (0, {})


def test_deep_property_random_positions(api, oracle):
    """Seeded random positions, depths, splits and shard counts: the shards'
    subtotals always sum to the oracle's perft, move by move."""
    from hypothesis import HealthCheck, given, settings
    from hypothesis import strategies as st

    @settings(max_examples=40, deadline=None, derandomize=True,
              suppress_health_check=[HealthCheck.function_scoped_fixture])
    @given(seed=st.integers(0, 2**32 - 1), plies=st.integers(0, 60), depth=st.integers(1, 3),
           split=st.integers(0, 3), n=st.integers(1, 4))
    def check(seed, plies, depth, split, n):
        pos = pg.random_playouts(seed=seed, n=1, min_plies=plies, max_plies=plies)[0]
        acc = {}
        for s in range(n):
            _, div = pg.deep(pos, depth, split, shard=s, n_shards=n)
            for m, c in div.items():
                acc[m] = acc.get(m, 0) + c
        assert sum(acc.values()) == oracle.perft(pos, depth)
        assert sorted(acc.values()) == sorted(oracle.perft(c, depth - 1) for c in oracle.children(pos))

    check()
