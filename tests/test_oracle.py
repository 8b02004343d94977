"""The oracle pinned against the reference: golden vectors generated from the
reference's own host perft, and (when the reference build exists here) a
direct comparison on seeded playouts and on the reference's known-position
list."""
import ctypes
import json
import os
import random
import re
import subprocess

import numpy as np
import pytest

from tests._oracle import P6, ROOT, pos48_from_hex, reference

# The reference source tree, when this machine has one (the known-position
# test reads its FEN list at test time).
REF_TREE = os.environ.get("PERFT_REFERENCE_DIR", "")


def test_oracle_matches_golden_counts(oracle, golden):
    bad = []
    for e in golden:
        pos = pos48_from_hex(e["pos48"])
        for d, c in e["counts"].items():
            if int(c) > 20_000_000:
                continue
            got = oracle.perft(pos, int(d))
            if got != int(c):
                bad.append((e["name"], d, c, got))
    assert not bad, bad


def test_oracle_matches_golden_divided(oracle, golden):
    for e in golden:
        pos = pos48_from_hex(e["pos48"])
        got = sorted(oracle.perft(c, 2) for c in oracle.children(pos))
        assert got == sorted(ch["perft2"] for ch in e["children_perft2"]), e["name"]


def test_golden_fen_and_board_agree(oracle, golden):
    for e in golden:
        assert np.array_equal(oracle.fen_to_pos(e["fen"]) & np.uint64(~(0xF << 4) & (2**64 - 1)),
                              pos48_from_hex(e["pos48"]) & np.uint64(~(0xF << 4) & (2**64 - 1))), e["name"]


ref = reference()
needs_ref = pytest.mark.skipif(ref is None, reason="reference host perft (oracle/_ref) not built here")


@needs_ref
def test_oracle_vs_reference_seeded_playouts(oracle):
    rng = random.Random(11)
    start = P6()
    ref.ref_fen_to_pos(b"rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1", start)
    buf = (ctypes.c_uint64 * (6 * 256))()
    checked = 0
    for _ in range(150):
        p = P6(*start)
        for _ in range(rng.randint(0, 70)):
            n = ref.ref_children(p, buf)
            if n == 0:
                break
            k = rng.randrange(n)
            p = P6(*buf[6 * k:6 * k + 6])
            d = rng.randint(1, 3)
            arr = np.array(list(p), dtype=np.uint64)
            assert oracle.perft(arr, d) == ref.ref_perft(p, d)
            assert ref.ref_perft_gm(p, d) == ref.ref_perft(p, d)
            checked += 1
    assert checked > 1000


@needs_ref
@pytest.mark.skipif(not (REF_TREE and os.path.exists(os.path.join(REF_TREE, "perft.cu"))),
                    reason="reference tree absent (set PERFT_REFERENCE_DIR)")
def test_oracle_vs_reference_known_positions(oracle):
    """The reference keeps its validation positions as FEN strings in
    perft.cu; read them from the reference tree at test time."""
    src = open(os.path.join(REF_TREE, "perft.cu")).read()
    fens = re.findall(r'readFENString\("([^"]+)"', src)
    assert len(fens) >= 5
    for fen in fens:
        p = P6()
        ref.ref_fen_to_pos(fen.encode(), p)
        mine = oracle.fen_to_pos(fen)
        assert list(mine) == list(p), fen
        for d in (1, 2, 3):
            assert oracle.perft(mine, d) == ref.ref_perft(p, d), (fen, d)


def test_opcount_build_and_work_figures():
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "opcount"], check=True,
                   stdout=subprocess.DEVNULL)
    with open(os.path.join(ROOT, "perft_gpu_b200", "work_figures.json")) as f:
        wf = json.load(f)["workloads"]
    for key in ("batch4096", "start", "deep"):
        for c in ("c_count", "c_make", "c_gen"):
            assert wf[key][c] > 0
    # re-measure the initial position: the frozen figures are reproducible
    import tempfile
    start = np.array([0xFFFF, 0x00FF00000000FF0F, 0x4200000000000042, 0x2C0000000000002C,
                      0x8900000000000089, 0x1000000000000010], dtype=np.uint64)
    with tempfile.NamedTemporaryFile(suffix=".bin", delete=False) as f:
        f.write(start.tobytes())
        path = f.name
    out = subprocess.run([os.path.join(ROOT, "oracle", "opcount"), path, "4"], check=True,
                         capture_output=True, text=True).stdout
    os.unlink(path)
    res = json.loads(out)
    assert res["leaves"] == 197281
    assert abs(res["c_count"] - wf["start"]["c_count"]) < 1e-6


@needs_ref
def test_oracle_vs_reference_many_moves(oracle):
    """Crafted 94-170-move positions and their colour mirrors: the oracle,
    the reference's host perft and the mirror all agree."""
    from tests._positions import MANY_MOVES, mirror_fen
    for fen in MANY_MOVES:
        counts = []
        for f in (fen, mirror_fen(fen)):
            p = P6()
            assert ref.ref_fen_to_pos(f.encode(), p) == 0, f
            arr = np.array(list(p), dtype=np.uint64)
            c = [ref.ref_perft(p, d) for d in (1, 2, 3)]
            assert [oracle.perft(arr, d) for d in (1, 2, 3)] == c, f
            counts.append(c)
        assert counts[0] == counts[1], fen
        assert counts[0][0] >= 94


@needs_ref
def test_oracle_vs_reference_stratified_batch():
    """The benchmark batch's strata, where seeded playouts alone rarely reach
    an en-passant capture (about 0.5% of them): oracle and reference agree on
    perft 1-3 of a 200-position sample."""
    import perft_gpu_b200 as pg
    from perft_gpu_b200 import workloads
    from tests._oracle import Oracle
    oracle = Oracle(os.path.join(ROOT, "oracle", "liboracle.so"))
    pos, _ = workloads.batch_positions(n=200, seed=29)
    ep = 0
    for p in pos:
        ep += (pg.features(p) & pg.FEATURE_EP) != 0
        pp = P6(*[int(x) for x in p])
        for d in (1, 2, 3):
            assert oracle.perft(p, d) == ref.ref_perft(pp, d), ([hex(int(x)) for x in p], d)
    assert ep >= 20
