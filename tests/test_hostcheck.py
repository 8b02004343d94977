"""The product's move generator (movegen.cuh), compiled for the host, against
the oracle: legal-move counts, generated children and perft, for every slider
variant.  Runs without a GPU."""
import ctypes
import os
import random
import subprocess

import numpy as np
import pytest

from tests._oracle import P6, ROOT, pos48_from_hex

HC_DIR = os.path.join(ROOT, "tests", "hostcheck")
HC_LIB = os.path.join(HC_DIR, "libhostcheck.so")


@pytest.fixture(scope="module")
def hc():
    src = [os.path.join(HC_DIR, "hostcheck.cpp"), os.path.join(ROOT, "perft_gpu_b200", "csrc", "tables.cpp")]
    hdr = os.path.join(ROOT, "perft_gpu_b200", "csrc", "movegen.cuh")
    if not os.path.exists(HC_LIB) or any(os.path.getmtime(s) > os.path.getmtime(HC_LIB) for s in src + [hdr]):
        subprocess.run(["g++", "-O2", "-std=c++20", "-fPIC", "-shared", "-o", HC_LIB] + src, check=True)
    lib = ctypes.CDLL(HC_LIB)
    lib.hc_count.restype = ctypes.c_uint32
    lib.hc_children.restype = ctypes.c_uint32
    lib.hc_perft.restype = ctypes.c_uint64
    lib.hc_init()
    return lib


def _children(hc, pos, sv):
    buf = (ctypes.c_uint64 * (6 * 256))()
    n = hc.hc_children(P6(*[int(x) for x in pos]), sv, buf)
    return sorted(tuple(buf[6 * i:6 * i + 6]) for i in range(n))


SV_ALL = [0, 1, 2, 3, 4]
SV_IDS = ["kogge", "magic", "kogge_fma", "kogge_split", "hybrid"]


@pytest.mark.parametrize("sv", SV_ALL, ids=SV_IDS)
def test_golden_perft(hc, golden, sv):
    for e in golden:
        p = P6(*[int(h, 16) for h in e["pos48"]])
        for d, c in e["counts"].items():
            if int(c) <= 3_000_000:
                assert hc.hc_perft(p, int(d), sv) == int(c), (e["name"], d)


@pytest.mark.parametrize("sv", SV_ALL, ids=SV_IDS)
def test_counts_and_children_vs_oracle(hc, oracle, sv):
    rng = random.Random(3 + sv)
    start = oracle.fen_to_pos("rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1")
    positions = 0
    for _ in range(120):
        p = start
        for _ in range(rng.randint(0, 80)):
            kids = oracle.children(p)
            assert hc.hc_count(P6(*[int(x) for x in p]), sv) == len(kids)
            assert _children(hc, p, sv) == sorted(tuple(int(x) for x in k) for k in kids)
            positions += 1
            if not kids:
                break
            p = kids[rng.randrange(len(kids))]
    assert positions > 2000


def test_relative_roundtrip(hc, golden):
    out = P6()
    for e in golden:
        p = P6(*[int(h, 16) for h in e["pos48"]])
        hc.hc_roundtrip(p, out)
        assert list(out) == list(p), e["name"]


@pytest.mark.parametrize("sv", SV_ALL, ids=SV_IDS)
def test_stratified_batch_sample_vs_oracle(hc, oracle, sv):
    """The benchmark batch's special-rule strata (legal en-passant captures,
    pawns on the 7th rank, castling rights) through the product's move
    generator on the host: child sets and perft(2) against the oracle."""
    import perft_gpu_b200 as pg
    from perft_gpu_b200 import workloads
    pos, _ = workloads.batch_positions(n=300, seed=17)
    f = np.array([pg.features(p) for p in pos])
    assert (f & pg.FEATURE_EP != 0).sum() >= 30
    for p in pos:
        pp = P6(*[int(x) for x in p])
        kids = oracle.children(p)
        assert hc.hc_count(pp, sv) == len(kids)
        assert _children(hc, p, sv) == sorted(tuple(int(x) for x in k) for k in kids)
        assert hc.hc_perft(pp, 2, sv) == oracle.perft(p, 2)


@pytest.mark.parametrize("sv", SV_ALL, ids=SV_IDS)
def test_mover_bits_children(hc, golden, sv):
    """Moves that carry the mover's planes (the tile kernel's items) give the
    same 16-bit moves in the same order and the same children as plain
    generation with piece lookups in make-move."""
    hc.hc_children_mover.restype = ctypes.c_uint32
    pos = [pos48_from_hex(e["pos48"]) for e in golden]
    rng = random.Random(5)
    buf = (ctypes.c_uint64 * (6 * 256))()
    for p in pos:
        # walk a few plies from each golden position
        for _ in range(12):
            kids = _children(hc, p, sv)
            n = len(kids)
            mv = (ctypes.c_uint16 * 256)()
            m = hc.hc_children_mover(P6(*[int(x) for x in p]), sv, buf, mv)
            assert m == n
            assert sorted(tuple(buf[6 * i:6 * i + 6]) for i in range(m)) == kids
            plain = (ctypes.c_uint64 * (6 * 256))()
            hc.hc_children(P6(*[int(x) for x in p]), sv, plain)
            assert [tuple(buf[6 * i:6 * i + 6]) for i in range(m)] == [tuple(plain[6 * i:6 * i + 6]) for i in range(n)]
            if n == 0:
                break
            p = np.array(kids[rng.randrange(n)], dtype=np.uint64)


def test_mirrored_make_equals_make(hc, golden):
    """Children made from the mirrored parent (the tile kernel's make-move)
    equal make_child's children, in order, on golden positions and seeded
    walks from them (captures, promotions, castling, en passant included)."""
    hc.hc_children_mirrored.restype = ctypes.c_uint32
    rng = random.Random(9)
    buf = (ctypes.c_uint64 * (6 * 256))()
    plain = (ctypes.c_uint64 * (6 * 256))()
    checked = 0
    for e in golden:
        p = pos48_from_hex(e["pos48"])
        for _ in range(16):
            pp = P6(*[int(x) for x in p])
            n = hc.hc_children(pp, 0, plain)
            m = hc.hc_children_mirrored(pp, buf)
            assert m == n
            assert list(buf[:6 * n]) == list(plain[:6 * n]), e["name"]
            checked += n
            if n == 0:
                break
            k = rng.randrange(n)
            p = np.array(list(plain[6 * k:6 * k + 6]), dtype=np.uint64)
    assert checked > 5000


@pytest.mark.parametrize("sv", SV_ALL, ids=SV_IDS)
def test_count_with_known_king_squares(hc, golden, sv):
    """The count with both king squares supplied (from the parent, as the tile
    kernel supplies them; king moves and castling move one) equals the count
    that finds them itself, on golden positions and seeded walks."""
    hc.hc_counts_known_kings.restype = ctypes.c_uint32
    rng = random.Random(13)
    buf = (ctypes.c_uint64 * (6 * 256))()
    for e in golden:
        p = pos48_from_hex(e["pos48"])
        for _ in range(12):
            pp = P6(*[int(x) for x in p])
            assert hc.hc_counts_known_kings(pp, sv) == 0, e["name"]
            n = hc.hc_children(pp, 0, buf)
            if n == 0:
                break
            k = rng.randrange(n)
            p = np.array(list(buf[6 * k:6 * k + 6]), dtype=np.uint64)
