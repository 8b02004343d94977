"""Generates tests/golden/perft_golden.json from the REFERENCE's own host perft.

Run in a container that holds the reference tree and the reference build
(``make -C oracle``):  python tests/golden/make_golden.py

Counts come from oracle/_ref/libperft_ref.so (the reference's perft_bb,
perft_bb.h:79-101, compiled from the reference sources).  Positions are:
  * the initial position,
  * crafted edge cases written for this project (stalemate, mate, double
    check, en-passant horizontal pin, en-passant check evasion, castling
    through an attacked square, promotions with captures),
  * seeded random playouts (reference move generation), stratified by the
    clean-room oracle's move flags: en passant available, promotion
    available, and unconstrained.
Every position also stores the reference's perft(2) of each child (a
divided perft at depth 3).
"""
import ctypes
import json
import os
import random
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
REF = os.path.join(ROOT, "oracle", "_ref", "libperft_ref.so")
ORC = os.path.join(ROOT, "oracle", "liboracle.so")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "perft_golden.json")

P6 = ctypes.c_uint64 * 6

CRAFTED = {
    "stalemate": "7k/5Q2/6K1/8/8/8/8/8 b - - 0 1",
    "back_rank_mate": "R5k1/5ppp/8/8/8/8/8/6K1 b - - 0 1",
    "double_check": "4k3/8/8/8/8/8/4r3/r3K3 w - - 0 1",
    "ep_horizontal_pin": "8/8/8/K1pP3r/8/8/8/7k w - c6 0 1",
    "ep_evades_pawn_check": "8/8/8/2k5/3Pp3/8/8/4K3 b - d3 0 1",
    "castle_through_attack": "r3k2r/8/8/8/8/5b2/8/R3K2R w KQkq - 0 1",
    "promotions_both_sides": "r3k3/1P6/8/8/8/8/6p1/4K2R w K - 0 1",
    "promotions_black_to_move": "r3k3/1P6/8/8/8/8/6p1/4K2R b K - 0 1",
    "pinned_pieces": "4k3/4r3/8/1b6/8/3N4/4B3/r3K2R w K - 0 1",
    "ep_diagonal_pin": "8/8/8/1k6/2pP4/8/8/5B1K b - d3 0 1",
}


def load():
    ref = ctypes.CDLL(REF)
    orc = ctypes.CDLL(ORC)
    ref.ref_perft.restype = ctypes.c_uint64
    ref.ref_children.restype = ctypes.c_uint32
    ref.ref_count_moves.restype = ctypes.c_uint32
    ref.ref_perft_mt.restype = ctypes.c_uint64
    orc.oracle_generate_moves.restype = ctypes.c_uint32
    ref.ref_init()
    orc.oracle_init()
    return ref, orc


def to_fen(p):
    pawns = p[1] & 0x00FFFFFFFFFFFF00
    rows = []
    for r in range(7, -1, -1):
        row, empty = "", 0
        for f in range(8):
            b = 1 << (r * 8 + f)
            c = ""
            if pawns & b: c = "p"
            elif p[2] & b: c = "n"
            elif p[3] & p[4] & b: c = "q"
            elif p[3] & b: c = "b"
            elif p[4] & b: c = "r"
            elif p[5] & b: c = "k"
            if not c:
                empty += 1
                continue
            if empty:
                row += str(empty)
                empty = 0
            row += c.upper() if p[0] & b else c
        if empty:
            row += str(empty)
        rows.append(row)
    black = (p[1] >> 63) & 1
    cs = "".join(ch for bit, ch in ((1, "K"), (2, "Q"), (4, "k"), (8, "q")) if p[1] & bit) or "-"
    ep = (p[1] >> 4) & 15
    eps = "-" if not ep else "abcdefgh"[ep - 1] + ("3" if black else "6")
    return f"{'/'.join(rows)} {'b' if black else 'w'} {cs} {eps} 0 1"


def move_flags(orc, p):
    mv = (ctypes.c_uint16 * 256)()
    n = orc.oracle_generate_moves(p, mv)
    return [mv[i] >> 12 for i in range(n)]


def walk(ref, rng, plies):
    start = P6()
    ref.ref_fen_to_pos(b"rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1", start)
    p = P6(*start)
    buf = (ctypes.c_uint64 * (6 * 256))()
    for _ in range(plies):
        n = ref.ref_children(p, buf)
        if n == 0:
            return None
        k = rng.randrange(n)
        p = P6(*buf[6 * k:6 * k + 6])
    return p


def main():
    ref, orc = load()
    rng = random.Random(20261203)
    entries = []

    def add(name, p, depths, deep=()):
        counts = {str(d): int(ref.ref_perft(p, d)) for d in depths}
        # deeper counts with the reference's perft root-split over threads
        counts.update({str(d): int(ref.ref_perft_mt(p, d, os.cpu_count() or 1)) for d in deep})
        # divided counts at depth 3 (children from the reference's generateBoards)
        buf = (ctypes.c_uint64 * (6 * 256))()
        n = ref.ref_children(p, buf)
        children = []
        for i in range(n):
            c = P6(*buf[6 * i:6 * i + 6])
            children.append({"fen": to_fen(list(c)), "perft2": int(ref.ref_perft(c, 2))})
        children.sort(key=lambda e: e["fen"])
        entries.append({
            "name": name,
            "fen": to_fen(list(p)),
            "pos48": [f"{int(x):016x}" for x in p],
            "counts": counts,
            "children_perft2": children,
        })
        print(name, counts, file=sys.stderr)

    start = P6()
    ref.ref_fen_to_pos(b"rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1", start)
    add("initial_position", start, range(0, 7), deep=(7,))

    for name, fen in CRAFTED.items():
        p = P6()
        ref.ref_fen_to_pos(fen.encode(), p)
        add(name, p, range(0, 6))

    want = {"ep": 8, "promo": 8, "uniform": 24}
    got = {k: 0 for k in want}
    tries = 0
    while any(got[k] < want[k] for k in want) and tries < 200000:
        tries += 1
        p = walk(ref, rng, rng.randint(4, 60))
        if p is None or ref.ref_count_moves(p) == 0:
            continue
        flags = move_flags(orc, p)
        kind = None
        if 5 in flags and got["ep"] < want["ep"]:
            kind = "ep"
        elif any(f >= 8 for f in flags) and got["promo"] < want["promo"]:
            kind = "promo"
        elif got["uniform"] < want["uniform"] and rng.random() < 0.05:
            kind = "uniform"
        if kind is None:
            continue
        got[kind] += 1
        add(f"playout_{kind}_{got[kind]}", p, range(1, 5), deep=(5,) if got[kind] <= 3 else ())

    with open(OUT, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "source": "reference host perft (oracle/_ref/libperft_ref.so)",
                   "positions": entries}, f, indent=1)
    print(f"wrote {len(entries)} positions to {OUT}", file=sys.stderr)


if __name__ == "__main__":
    main()
