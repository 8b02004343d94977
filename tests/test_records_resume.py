"""Records-mode resume bookkeeping on the host: which records count as
finished, and how a torn output tail is recovered.  Every case here either
has nothing left to search (so no engine is needed) or checks that a call
that does need one fails cleanly after repairing the output."""
import pytest

import perft_gpu_b200 as pg

FENS = [
    "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1 3",
    "r3k2r/p1ppqpb1/bn2pnp1/3PN3/1p2P3/2N2Q1p/PPPBBPPP/R3K2R w KQkq - 0 1 1",
    "8/2p5/3p4/KP5r/1R3p1k/8/4P1P1/8 w - - 0 1 7",
]
DONE = [f"{f} {100 + i} {(100 + i) * int(f.rsplit(' ', 1)[1])}" for i, f in enumerate(FENS)]


def _write(path, text):
    with open(path, "w") as f:
        f.write(text)


def test_all_finished_is_a_no_op(tmp_path):
    src = tmp_path / "r.txt"
    _write(src, "\n".join(FENS[:2]) + "\n\n" + FENS[2] + "\n")  # an empty line is not a record
    op = str(src) + ".op"
    _write(op, "\n".join(DONE) + "\n")
    assert pg.records(str(src), 3) == 0
    assert open(op).read() == "\n".join(DONE) + "\n"


def test_long_output_lines_count_once(tmp_path):
    """A finished line longer than the input-line limit is still one record."""
    src = tmp_path / "r.txt"
    pad = " " * 3000
    _write(src, FENS[0] + "\n" + FENS[1] + "\n")
    op = str(src) + ".op"
    body = f"{FENS[0]}{pad} 1 1\n{FENS[1]} 2 2\n"
    _write(op, body)
    assert pg.records(str(src), 3) == 0
    assert open(op).read() == body


def test_torn_tail_is_cut_and_searched_again(tmp_path):
    src = tmp_path / "r.txt"
    _write(src, "\n".join(FENS) + "\n")
    op = str(src) + ".op"
    _write(op, "\n".join(DONE[:2]) + "\n" + DONE[2][:25])  # stopped in the middle of the third line
    try:
        n = pg.records(str(src), 3)
    except pg.PerftError as e:
        # no engine in this process: the third record cannot be searched, but
        # the torn line is already gone
        assert e.status == pg.PERFT_ERR_NOT_INITIALIZED
        assert open(op).read() == "\n".join(DONE[:2]) + "\n"
        return
    # an engine is up: the third record was searched again and appended whole
    assert n == 1
    lines = open(op).read().splitlines()
    assert lines[:2] == DONE[:2] and len(lines) == 3 and lines[2].startswith(FENS[2] + " ")


def test_torn_tail_only(tmp_path):
    """Output holding only a torn first line: nothing is finished."""
    src = tmp_path / "r.txt"
    _write(src, "")
    op = str(src) + ".op"
    _write(op, DONE[0][:10])
    assert pg.records(str(src), 3) == 0
    assert open(op).read() == ""


def test_missing_input_and_bad_depth(tmp_path):
    with pytest.raises(pg.PerftError) as ei:
        pg.records(str(tmp_path / "missing.txt"), 3)
    assert ei.value.status == pg.PERFT_ERR_NOT_FOUND
    _write(tmp_path / "r.txt", FENS[0] + "\n")
    with pytest.raises(pg.PerftError) as ei:
        pg.records(str(tmp_path / "r.txt"), 21)
    assert ei.value.status == pg.PERFT_ERR_INVALID_ARG
