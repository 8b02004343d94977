"""Test infrastructure: ctypes access to the CPU oracle (oracle/liboracle.so)
and, when it was built, the reference's own host perft (oracle/_ref)."""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libperft_ref.so")

P6 = ctypes.c_uint64 * 6


def _p6(pos):
    a = np.asarray(pos, dtype=np.uint64).reshape(6)
    return P6(*[int(x) for x in a])


class Oracle:
    def __init__(self, path):
        lib = ctypes.CDLL(path)
        lib.oracle_perft.restype = ctypes.c_uint64
        lib.oracle_count_moves.restype = ctypes.c_uint32
        lib.oracle_generate_moves.restype = ctypes.c_uint32
        lib.oracle_divide.restype = ctypes.c_uint32
        lib.oracle_init()
        self.lib = lib

    def perft(self, pos, depth):
        return int(self.lib.oracle_perft(_p6(pos), depth))

    def count(self, pos):
        return int(self.lib.oracle_count_moves(_p6(pos)))

    def moves(self, pos):
        mv = (ctypes.c_uint16 * 256)()
        n = self.lib.oracle_generate_moves(_p6(pos), mv)
        return [mv[i] for i in range(n)]

    def children(self, pos):
        out = []
        for m in self.moves(pos):
            c = _p6(pos)
            self.lib.oracle_make_move(c, m)
            out.append(np.array(list(c), dtype=np.uint64))
        return out

    def fen_to_pos(self, fen):
        p = P6()
        rc = self.lib.oracle_fen_to_pos(fen.encode(), p)
        assert rc == 0, fen
        return np.array(list(p), dtype=np.uint64)

    def perft_batch_mt(self, positions, depths, threads=None):
        pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint64).reshape(-1, 6))
        n = pos.shape[0]
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(depths, dtype=np.uint32), (n,)))
        out = np.zeros(n, dtype=np.uint64)
        rc = self.lib.oracle_perft_batch_mt(ctypes.c_void_p(pos.ctypes.data), ctypes.c_void_p(d.ctypes.data),
                                            n, threads or os.cpu_count() or 1, ctypes.c_void_p(out.ctypes.data))
        assert rc == 0
        return out


def reference():
    """The reference's own host perft, or None when it was not built here."""
    if not os.path.exists(REF_LIB):
        return None
    lib = ctypes.CDLL(REF_LIB)
    lib.ref_perft.restype = ctypes.c_uint64
    lib.ref_perft_gm.restype = ctypes.c_uint64
    lib.ref_count_moves.restype = ctypes.c_uint32
    lib.ref_children.restype = ctypes.c_uint32
    lib.ref_init()
    return lib


def pos48_from_hex(hexes):
    return np.array([int(h, 16) for h in hexes], dtype=np.uint64)
