"""Continuous-batching server: every query's count equals the count of the
same query run alone, whatever else is in flight, and however the levels are
split into steps or queued by the memory budget."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture
def server(engine):
    engine.init(device=0, arena_bytes=6 << 30)
    yield engine
    engine.serve_stop()
    engine.init(device=0, arena_bytes=8 << 30)


def _queries(engine, n, seed, max_depth=5):
    pos = engine.random_playouts(seed=seed, n=n, min_plies=0, max_plies=40)
    rng = np.random.default_rng(seed)
    depths = rng.integers(0, max_depth + 1, size=n).astype(np.uint8)
    return pos, depths


@pytest.mark.parametrize("step_items,memory", [(0, 0), (8192, 0), (1 << 16, 64 << 20)],
                         ids=["default", "tiny_steps", "tight_memory"])
def test_served_counts_equal_alone(server, step_items, memory):
    pos, depths = _queries(server, 300, seed=11)
    alone = server.perft_batch(pos, depths)
    server.serve_start(memory_bytes=memory, step_items=step_items)
    tickets = [server.serve_submit(p, int(d)) for p, d in zip(pos, depths)]
    got = [server.serve_wait(t, timeout_s=120)[0] for t in tickets]
    assert got == [int(x) for x in alone]
    st = server.serve_stats()
    assert st["completed"] == 300 and st["in_flight"] == 0 and st["last_error"] == 0


def test_staggered_arrivals_overlap(server):
    """Queries submitted while others run join them; results stay exact."""
    pos, depths = _queries(server, 120, seed=12, max_depth=6)
    alone = [int(x) for x in server.perft_batch(pos, depths)]
    server.serve_start(step_items=1 << 20)
    results = {}

    def submitter(lo, hi):
        for i in range(lo, hi):
            results[i] = server.serve_submit(pos[i], int(depths[i]))
            time.sleep(0.002)

    threads = [threading.Thread(target=submitter, args=(k * 40, k * 40 + 40)) for k in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    got = [server.serve_wait(results[i], timeout_s=120)[0] for i in range(120)]
    assert got == alone
    assert server.serve_stats()["iterations"] > 1


def test_poll_and_unknown_ticket(server, golden):
    server.serve_start()
    start = server.fen_to_pos(server.START_FEN)
    t = server.serve_submit(start, 6)
    res = None
    for _ in range(20000):
        res = server.serve_poll(t)
        if res is not None:
            break
        time.sleep(0.001)
    assert res is not None and res[0] == 119060324 and res[1] >= 0
    with pytest.raises(server.PerftError) as ei:
        server.serve_poll(t)  # consumed
    assert ei.value.status == server.PERFT_ERR_NOT_FOUND


def test_direct_calls_while_serving(server):
    server.serve_start()
    pos, depths = _queries(server, 50, seed=13)
    tickets = [server.serve_submit(p, int(d)) for p, d in zip(pos, depths)]
    direct = server.perft_batch(pos, depths)  # the arena engine keeps working beside the server
    got = [server.serve_wait(t, timeout_s=120)[0] for t in tickets]
    assert got == [int(x) for x in direct]


@pytest.fixture
def tt_server(engine):
    """The server over an engine with a 2^24-entry table."""
    engine.init(device=0, arena_bytes=6 << 30, tt_log2_entries=24)
    yield engine
    engine.serve_stop()
    engine.init(device=0, arena_bytes=8 << 30)


@pytest.mark.parametrize("step_items,memory", [(0, 0), (8192, 0), (1 << 16, 64 << 20)],
                         ids=["default", "tiny_steps", "tight_memory"])
def test_served_with_table_equal_alone_and_oracle(tt_server, oracle, step_items, memory):
    """With the table resident in the server: every query equals its count
    alone (engine without a table) and the oracle's; identical queries and
    transpositions are answered from the table or merged.  Tiny steps split
    the expansion of a level three plies above the leaves into many child
    levels, which all add into the same parents' sums; a tight budget admits
    queries a few at a time, so new levels join while others wait for their
    child levels."""
    pos, depths = _queries(tt_server, 200, seed=21, max_depth=6)
    pos = np.vstack([pos, pos[:40]])  # repeats: answered from the table
    depths = np.concatenate([depths, depths[:40]])
    want = oracle.perft_batch_mt(pos, depths)
    tt_server.serve_start(memory_bytes=memory, step_items=step_items)
    tickets = [tt_server.serve_submit(p, int(d)) for p, d in zip(pos, depths)]
    got = [tt_server.serve_wait(t, timeout_s=300)[0] for t in tickets]
    assert got == [int(x) for x in want]
    st = tt_server.serve_stats()
    assert st["completed"] == len(pos) and st["last_error"] == 0
    assert st["tt_probes"] > 0 and st["tt_hits"] > 0 and st["tt_merged"] > 0 and st["tt_stores"] > 0
    tt_server.serve_stop()
    # and the same queries without the table in the server
    tt_server.serve_start(memory_bytes=memory, step_items=step_items, use_tt=False)
    tickets = [tt_server.serve_submit(p, int(d)) for p, d in zip(pos, depths)]
    assert [tt_server.serve_wait(t, timeout_s=300)[0] for t in tickets] == got
    assert tt_server.serve_stats()["tt_probes"] == 0


def test_served_with_table_shared_slots(engine, oracle, monkeypatch):
    """A 12-bit slot key: every table and de-duplication slot is shared by
    many different nodes, so counts stay exact only if the verification key
    separates them."""
    monkeypatch.setenv("PERFT_TT_INDEX_KEY_BITS", "12")
    engine.init(device=0, arena_bytes=6 << 30, tt_log2_entries=20)
    try:
        pos, depths = _queries(engine, 120, seed=22, max_depth=5)
        want = oracle.perft_batch_mt(pos, depths)
        engine.serve_start()
        tickets = [engine.serve_submit(p, int(d)) for p, d in zip(pos, depths)]
        got = [engine.serve_wait(t, timeout_s=300)[0] for t in tickets]
        assert got == [int(x) for x in want]
        assert engine.serve_stats()["tt_hits"] > 0
    finally:
        engine.serve_stop()
        monkeypatch.delenv("PERFT_TT_INDEX_KEY_BITS")
        engine.init(device=0, arena_bytes=8 << 30)
