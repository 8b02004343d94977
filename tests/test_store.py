"""The deep-run result store file without a GPU: header, record format and
check word, torn-tail recovery, and rejection of a foreign file.  Counts added
by deep runs are covered by the gpu tests."""
import struct

import numpy as np

import pytest

import perft_gpu_b200 as pg

M = (1 << 64) - 1
MAGIC = b"PERFTB200STORE1\0"


def _check(words, count, depth):
    h = 0x243F6A8885A308D3 ^ depth
    for x in words:
        h = ((h ^ x) * 0x9E3779B97F4A7C15) & M
    h = ((h ^ count) * 0xD6E8FEB86659FD93) & M
    h ^= h >> 32
    return (h & 0xFFFFFFFF) ^ 0xA5A5A5A5


def _record(words, count, depth, check=None):
    c = _check(words, count, depth) if check is None else check
    return struct.pack("<6QQII", *words, count, depth, c)


@pytest.fixture
def store():
    yield pg
    pg.store_close()


def test_new_file_gets_header(store, tmp_path):
    path = tmp_path / "s.dat"
    store.store_open(str(path))
    assert store.store_stats() == {"entries": 0, "hits": 0, "appended": 0}
    store.store_close()
    data = path.read_bytes()
    assert len(data) == 64 and data[:16] == MAGIC


def test_records_loaded_and_torn_tail_dropped(store, tmp_path):
    start = [int(x) for x in pg.fen_to_pos(pg.START_FEN)]
    start[1] &= (1 << 63) - 1
    good = [_record(start, 4865609, 5), _record(start, 119060324, 6)]
    bad = _record(start, 123, 7, check=0)  # wrong check word
    path = tmp_path / "s.dat"
    path.write_bytes(MAGIC + bytes(48) + b"".join(good) + bad + b"\x01\x02\x03")
    store.store_open(str(path))
    assert store.store_stats()["entries"] == 2
    store.store_close()
    assert path.stat().st_size == 64 + 2 * 64  # truncated after the last good record


def test_foreign_file_rejected(store, tmp_path):
    path = tmp_path / "other.dat"
    path.write_bytes(b"x" * 100)
    with pytest.raises(pg.PerftError) as ei:
        store.store_open(str(path))
    assert ei.value.status == pg.PERFT_ERR_IO
    assert path.read_bytes() == b"x" * 100


def test_memory_store_and_closed_stats(store):
    store.store_open(None)
    assert store.store_stats()["entries"] == 0
    store.store_close()
    with pytest.raises(pg.PerftError):
        store.store_stats()


def test_deep_frontier_merges_transpositions(oracle):
    """The frontier deep perft searches: every move path to 1 + split plies,
    merged into distinct boards.  Paths equal perft at that depth; boards
    equal the distinct positions the oracle reaches (no GPU needed)."""
    start = pg.fen_to_pos(pg.START_FEN)
    mid = pg.random_playouts(seed=77, n=1, min_plies=10, max_plies=10)[0]
    for pos, split in ((start, 1), (start, 2), (mid, 1)):
        boards, paths = pg.deep_frontier(pos, 6, split)
        level = [np.asarray(pos, dtype=np.uint64)]
        for _ in range(split + 1):
            level = [c for p in level for c in oracle.children(p)]
        assert paths == len(level) == oracle.perft(pos, split + 1)
        assert boards == len({tuple(int(x) for x in c) for c in level})
        assert boards <= paths
    boards, paths = pg.deep_frontier(start, 6, 2)
    assert boards < paths  # ply 3 of the initial position already has transpositions
