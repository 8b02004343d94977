"""perft_gpu_b200: Python binding of the B200 perft engine (C ABI in include/perft_b200.h).

The engine itself is C++/CUDA (libperft_b200.so, built in-tree by
``python -m perft_gpu_b200.build``).  This module only marshals arguments:
positions are ``numpy.uint64`` arrays of shape (6,) or (n, 6) in the
reference's HexaBitBoardPosition layout (chess.h:208-230), counts come back
as Python ints / uint64 arrays.

There is no CPU fallback: if the library is missing, importing the binding
raises; if no GPU is present, :func:`init` raises ``PerftError`` with
``PERFT_ERR_NO_DEVICE``.
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable, List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# PERFT_B200_LIB points the binding at another build of the same library
LIB_PATH = os.environ.get("PERFT_B200_LIB") or os.path.join(_HERE, "libperft_b200.so")

PERFT_OK = 0
PERFT_PENDING = 1
PERFT_ERR_INVALID_ARG = -1
PERFT_ERR_NOT_INITIALIZED = -2
PERFT_ERR_CUDA = -3
PERFT_ERR_OUT_OF_MEMORY = -4
PERFT_ERR_INTERNAL = -5
PERFT_ERR_BAD_FEN = -6
PERFT_ERR_NO_DEVICE = -7
PERFT_ERR_ILLEGAL_MOVE = -8
PERFT_ERR_TIMEOUT = -9
PERFT_ERR_NOT_FOUND = -10
PERFT_ERR_IO = -11
PERFT_ERR_OVERFLOW = -12

SLIDERS_AUTO = -1
SLIDERS_KOGGE = 0
SLIDERS_MAGIC = 1
SLIDERS_KOGGE_FMA = 2
SLIDERS_KOGGE_SPLIT = 3
SLIDERS_HYBRID = 4
SLIDER_NAMES = {SLIDERS_KOGGE: "kogge", SLIDERS_MAGIC: "magic", SLIDERS_KOGGE_FMA: "kogge_fma",
                SLIDERS_KOGGE_SPLIT: "kogge_split", SLIDERS_HYBRID: "hybrid"}

START_FEN = "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1"


class PerftError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = _status_string(status)
        super().__init__(f"{what}: {msg} ({status})" if what else f"{msg} ({status})")


class _Pos48(ctypes.Structure):
    _fields_ = [("bb", ctypes.c_uint64 * 6)]


class PerftConfig(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int),
        ("arena_bytes", ctypes.c_uint64),
        ("sliders_expand", ctypes.c_int),
        ("sliders_leaf", ctypes.c_int),
        ("tt_log2_entries", ctypes.c_int),
        ("zobrist_seed", ctypes.c_uint64),
    ]


class PerftStats(ctypes.Structure):
    _fields_ = [
        ("leaf_launches", ctypes.c_uint64),
        ("expand_launches", ctypes.c_uint64),
        ("other_launches", ctypes.c_uint64),
        ("leaf_items", ctypes.c_uint64),
        ("leaf_parents", ctypes.c_uint64),
        ("expand_items", ctypes.c_uint64),
        ("leaf_ms", ctypes.c_double),
        ("expand_ms", ctypes.c_double),
        ("sliders_expand", ctypes.c_int),
        ("sliders_leaf", ctypes.c_int),
        ("arena_bytes", ctypes.c_uint64),
        ("peak_arena_bytes", ctypes.c_uint64),
        ("chunked_levels", ctypes.c_uint32),
        ("tt_entries", ctypes.c_uint64),
        ("tt_probes", ctypes.c_uint64),
        ("tt_hits", ctypes.c_uint64),
        ("tt_duplicates", ctypes.c_uint64),
        ("tt_stores", ctypes.c_uint64),
        ("graph_launches", ctypes.c_uint64),
        ("small_launches", ctypes.c_uint64),
    ]


class ServeConfig(ctypes.Structure):
    _fields_ = [
        ("memory_bytes", ctypes.c_uint64),
        ("step_items", ctypes.c_uint64),
        ("max_in_flight", ctypes.c_uint32),
        ("use_tt", ctypes.c_int32),
    ]


class ServeStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "submitted", "completed", "in_flight", "queued", "iterations", "launches",
        "memory_budget", "memory_reserved", "memory_peak")] + [("last_error", ctypes.c_int)] + [
        (n, ctypes.c_uint64) for n in ("tt_probes", "tt_hits", "tt_merged", "tt_stores")]


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m perft_gpu_b200.build` "
            "(the engine has no CPU fallback)")
    return _bind(ctypes.CDLL(LIB_PATH), require_all=True)


def _bind(lib, require_all: bool = False):
    """Sets the C signatures of include/perft_b200.h on a loaded library.
    Every entry point must exist unless require_all is False (a library
    exporting part of the interface)."""
    P = ctypes.POINTER
    u64p = P(ctypes.c_uint64)
    sig = {
        "perft_config_default": (None, [P(PerftConfig)]),
        "perft_init": (ctypes.c_int, [P(PerftConfig)]),
        "perft_shutdown": (ctypes.c_int, []),
        "perft_status_string": (ctypes.c_char_p, [ctypes.c_int]),
        "perft": (ctypes.c_int, [P(_Pos48), ctypes.c_uint32, u64p]),
        "perft_batch": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]),
        "perft_batch_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32,
                                              ctypes.c_void_p]),
        "perft_divide": (ctypes.c_int, [P(_Pos48), ctypes.c_uint32, ctypes.c_void_p, u64p,
                                        P(ctypes.c_uint32)]),
        "perft_fen_to_pos": (ctypes.c_int, [ctypes.c_char_p, P(_Pos48)]),
        "perft_pos_to_fen": (ctypes.c_int, [P(_Pos48), ctypes.c_char_p, ctypes.c_size_t]),
        "perft_legal_moves_uci": (ctypes.c_int, [P(_Pos48), ctypes.c_char_p, ctypes.c_size_t,
                                                 P(ctypes.c_uint32)]),
        "perft_apply_uci_move": (ctypes.c_int, [P(_Pos48), ctypes.c_char_p]),
        "perft_random_playouts": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                                 ctypes.c_uint32, ctypes.c_void_p]),
        "perft_position_features": (ctypes.c_int, [P(_Pos48), P(ctypes.c_uint32)]),
        "perft_get_stats": (ctypes.c_int, [P(PerftStats)]),
        "perft_get_tuning": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint32, P(ctypes.c_uint32)]),
        "perft_reset_stats": (ctypes.c_int, []),
        "perft_tt_clear": (ctypes.c_int, []),
        "perft_serve_config_default": (None, [P(ServeConfig)]),
        "perft_serve_start": (ctypes.c_int, [P(ServeConfig)]),
        "perft_serve_stop": (ctypes.c_int, []),
        "perft_serve_submit": (ctypes.c_int, [P(_Pos48), ctypes.c_uint32, P(ctypes.c_uint64)]),
        "perft_serve_poll": (ctypes.c_int, [ctypes.c_uint64, P(ctypes.c_uint64), P(ctypes.c_double)]),
        "perft_serve_wait": (ctypes.c_int, [ctypes.c_uint64, ctypes.c_double, P(ctypes.c_uint64),
                                            P(ctypes.c_double)]),
        "perft_serve_get_stats": (ctypes.c_int, [P(ServeStats)]),
        "perft_deep": (ctypes.c_int, [P(_Pos48), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p, u64p,
                                      P(ctypes.c_uint32), u64p]),
        "perft_deep_shard": (ctypes.c_int, [P(_Pos48), ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                            ctypes.c_uint32, ctypes.c_void_p, u64p, P(ctypes.c_uint32), u64p]),
        "perft_result_store_open": (ctypes.c_int, [ctypes.c_char_p]),
        "perft_result_store_close": (ctypes.c_int, []),
        "perft_result_store_stats": (ctypes.c_int, [u64p, u64p, u64p]),
        "perft_deep_frontier": (ctypes.c_int, [P(_Pos48), ctypes.c_uint32, ctypes.c_uint32, u64p, u64p]),
        "perft_records": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint32, ctypes.c_uint32, u64p]),
    }
    for name, (res, args) in sig.items():
        if not require_all and not hasattr(lib, name):
            continue
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


_lib_handle = None


def lib():
    """The loaded ctypes library.  Loaded on first use, so the package (and
    its build module) imports before the library has been built; every
    engine call fails loudly if the library is missing."""
    global _lib_handle
    if _lib_handle is None:
        _lib_handle = _load()
    return _lib_handle


def _status_string(status: int) -> str:
    s = lib().perft_status_string(int(status))
    return s.decode() if s else "unknown"


def _check(rc: int, what: str):
    if rc != PERFT_OK:
        raise PerftError(rc, what)


def _pos(p) -> _Pos48:
    a = np.asarray(p, dtype=np.uint64).reshape(6)
    s = _Pos48()
    for i in range(6):
        s.bb[i] = int(a[i])
    return s


def _arr(s: _Pos48) -> np.ndarray:
    return np.array([s.bb[i] for i in range(6)], dtype=np.uint64)


# --------------------------------------------------------------- engine
def config(device: int = 0, arena_bytes: int = 0, sliders_expand: int = SLIDERS_AUTO,
           sliders_leaf: int = SLIDERS_AUTO, tt_log2_entries: int = 0,
           zobrist_seed: int | None = None) -> PerftConfig:
    cfg = PerftConfig()
    lib().perft_config_default(ctypes.byref(cfg))
    cfg.device = device
    cfg.arena_bytes = arena_bytes
    cfg.sliders_expand = sliders_expand
    cfg.sliders_leaf = sliders_leaf
    cfg.tt_log2_entries = tt_log2_entries
    if zobrist_seed is not None:
        cfg.zobrist_seed = zobrist_seed
    return cfg


def init(device: int = 0, arena_bytes: int = 0, sliders_expand: int = SLIDERS_AUTO,
         sliders_leaf: int = SLIDERS_AUTO, tt_log2_entries: int = 0, zobrist_seed: int | None = None) -> None:
    cfg = config(device, arena_bytes, sliders_expand, sliders_leaf, tt_log2_entries, zobrist_seed)
    _check(lib().perft_init(ctypes.byref(cfg)), "perft_init")


def shutdown() -> None:
    lib().perft_shutdown()


def perft(pos, depth: int) -> int:
    out = ctypes.c_uint64(0)
    p = _pos(pos)
    _check(lib().perft(ctypes.byref(p), int(depth), ctypes.byref(out)), "perft")
    return int(out.value)


def perft_batch(positions, depths) -> np.ndarray:
    pos = np.ascontiguousarray(np.asarray(positions, dtype=np.uint64).reshape(-1, 6))
    n = pos.shape[0]
    d = np.ascontiguousarray(np.broadcast_to(np.asarray(depths, dtype=np.uint8), (n,)))
    out = np.zeros(n, dtype=np.uint64)
    _check(lib().perft_batch(pos.ctypes.data, d.ctypes.data, n, out.ctypes.data), "perft_batch")
    return out


def perft_batch_device(d_pos_ptr: int, depths, n: int, d_out_ptr: int) -> None:
    """Batched perft on device-resident buffers (e.g. torch CUDA tensors' data_ptr())."""
    d = np.ascontiguousarray(np.broadcast_to(np.asarray(depths, dtype=np.uint8), (n,)))
    _check(lib().perft_batch_device(ctypes.c_void_p(d_pos_ptr), d.ctypes.data, n,
                                   ctypes.c_void_p(d_out_ptr)), "perft_batch_device")


def divide(pos, depth: int) -> dict:
    p = _pos(pos)
    moves = (ctypes.c_char * (6 * 256))()
    counts = (ctypes.c_uint64 * 256)()
    n = ctypes.c_uint32(0)
    _check(lib().perft_divide(ctypes.byref(p), int(depth), moves, counts, ctypes.byref(n)), "perft_divide")
    raw = bytes(moves)
    res = {}
    for i in range(n.value):
        mv = raw[6 * i:6 * i + 6].split(b"\0")[0].decode()
        res[mv] = int(counts[i])
    return res


def stats() -> dict:
    s = PerftStats()
    _check(lib().perft_get_stats(ctypes.byref(s)), "perft_get_stats")
    return {name: getattr(s, name) for name, _ in PerftStats._fields_}


class TuneEntry(ctypes.Structure):
    _fields_ = [("leaf", ctypes.c_int), ("remaining", ctypes.c_int), ("sliders", ctypes.c_int),
                ("tile_log2", ctypes.c_int), ("ctas_per_sm", ctypes.c_int), ("calib_ms", ctypes.c_double)]


def tuning() -> list:
    """The launch configuration per (ply kind, remaining depth) in use:
    [{"ply": "leaf"|"interior", "remaining": r, "sliders": name, "tile": items,
      "ctas_per_sm": k (0: all that fit), "calib_ms": ms}, ...]."""
    buf = (TuneEntry * 32)()
    n = ctypes.c_uint32(0)
    _check(lib().perft_get_tuning(ctypes.cast(buf, ctypes.c_void_p), 32, ctypes.byref(n)), "perft_get_tuning")
    return [{"ply": "leaf" if e.leaf else "interior", "remaining": e.remaining,
             "sliders": SLIDER_NAMES.get(e.sliders, "?"), "tile": 1 << e.tile_log2,
             "ctas_per_sm": e.ctas_per_sm, "calib_ms": e.calib_ms} for e in buf[:n.value]]


def reset_stats() -> None:
    lib().perft_reset_stats()


def tt_clear() -> None:
    _check(lib().perft_tt_clear(), "perft_tt_clear")


def deep(pos, depth: int, split_plies: int = 2, shard: int = 0, n_shards: int = 1):
    """(total, {uci move: subtotal}) by host root split with transposition
    merging and GPU batches.  With n_shards > 1 only this shard's frontier
    boards are searched; the shards' results sum to the full count."""
    p = _pos(pos)
    moves = (ctypes.c_char * (6 * 256))()
    counts = (ctypes.c_uint64 * 256)()
    n, total = ctypes.c_uint32(0), ctypes.c_uint64(0)
    rc = lib().perft_deep_shard(ctypes.byref(p), int(depth), int(split_plies), int(shard), int(n_shards), moves,
                                counts, ctypes.byref(n), ctypes.byref(total))
    if rc != PERFT_ERR_OVERFLOW or n.value == 0:  # a total beyond 64 bits: the subtotals are exact, sum them here
        _check(rc, "perft_deep_shard")
    raw = bytes(moves)
    div = {raw[6 * i:6 * i + 6].split(b"\0")[0].decode(): int(counts[i]) for i in range(n.value)}
    return sum(div.values()), div


def deep_frontier(pos, depth: int, split_plies: int = 2):
    """(distinct boards, move paths) of the frontier deep() would search; host only."""
    p = _pos(pos)
    nb, npaths = ctypes.c_uint64(0), ctypes.c_uint64(0)
    _check(lib().perft_deep_frontier(ctypes.byref(p), int(depth), int(split_plies), ctypes.byref(nb),
                                     ctypes.byref(npaths)), "perft_deep_frontier")
    return int(nb.value), int(npaths.value)


def store_open(path: Optional[str] = None) -> None:
    """Opens the deep-run result store (file-backed, or host memory for None)."""
    _check(lib().perft_result_store_open(path.encode() if path else None), "perft_result_store_open")


def store_close() -> None:
    _check(lib().perft_result_store_close(), "perft_result_store_close")


def store_stats() -> dict:
    e, h, a = ctypes.c_uint64(0), ctypes.c_uint64(0), ctypes.c_uint64(0)
    _check(lib().perft_result_store_stats(ctypes.byref(e), ctypes.byref(h), ctypes.byref(a)),
           "perft_result_store_stats")
    return {"entries": int(e.value), "hits": int(h.value), "appended": int(a.value)}


def records(path: str, depth: int, batch: int = 4096) -> int:
    """Records mode; returns the number of records processed by this call."""
    done = ctypes.c_uint64(0)
    _check(lib().perft_records(path.encode(), int(depth), int(batch), ctypes.byref(done)), "perft_records")
    return int(done.value)


# ---------------------------------------------------------------- serving
def serve_start(memory_bytes: int = 0, step_items: int = 0, max_in_flight: int = 0, use_tt: bool = True) -> None:
    """Starts the continuous-batching server (after init).  With use_tt and an
    engine table (init with tt_log2_entries), the server's frontier levels two
    and three plies above the leaves probe, de-duplicate and store into that
    table."""
    cfg = ServeConfig()
    lib().perft_serve_config_default(ctypes.byref(cfg))
    cfg.use_tt = 1 if use_tt else 0
    if memory_bytes:
        cfg.memory_bytes = memory_bytes
    if step_items:
        cfg.step_items = step_items
    if max_in_flight:
        cfg.max_in_flight = max_in_flight
    _check(lib().perft_serve_start(ctypes.byref(cfg)), "perft_serve_start")


def serve_stop() -> None:
    _check(lib().perft_serve_stop(), "perft_serve_stop")


def serve_submit(pos, depth: int) -> int:
    t = ctypes.c_uint64(0)
    p = _pos(pos)
    _check(lib().perft_serve_submit(ctypes.byref(p), int(depth), ctypes.byref(t)), "perft_serve_submit")
    return int(t.value)


def serve_poll(ticket: int):
    """(count, latency_s) when done, None while the query runs."""
    c, lat = ctypes.c_uint64(0), ctypes.c_double(0)
    rc = lib().perft_serve_poll(ticket, ctypes.byref(c), ctypes.byref(lat))
    if rc == PERFT_PENDING:
        return None
    _check(rc, "perft_serve_poll")
    return int(c.value), float(lat.value)


def serve_wait(ticket: int, timeout_s: float = 600.0):
    c, lat = ctypes.c_uint64(0), ctypes.c_double(0)
    _check(lib().perft_serve_wait(ticket, timeout_s, ctypes.byref(c), ctypes.byref(lat)), "perft_serve_wait")
    return int(c.value), float(lat.value)


def serve_stats() -> dict:
    s = ServeStats()
    _check(lib().perft_serve_get_stats(ctypes.byref(s)), "perft_serve_get_stats")
    return {name: getattr(s, name) for name, _ in ServeStats._fields_}


# ------------------------------------------------------- host utilities
def fen_to_pos(fen: str) -> np.ndarray:
    p = _Pos48()
    _check(lib().perft_fen_to_pos(fen.encode(), ctypes.byref(p)), f"fen_to_pos({fen!r})")
    return _arr(p)


def pos_to_fen(pos) -> str:
    buf = ctypes.create_string_buffer(128)
    p = _pos(pos)
    _check(lib().perft_pos_to_fen(ctypes.byref(p), buf, 128), "pos_to_fen")
    return buf.value.decode()


def legal_moves(pos) -> List[str]:
    buf = ctypes.create_string_buffer(6 * 256)
    n = ctypes.c_uint32(0)
    p = _pos(pos)
    _check(lib().perft_legal_moves_uci(ctypes.byref(p), buf, len(buf), ctypes.byref(n)), "legal_moves")
    s = buf.value.decode()
    return s.split() if s else []


def apply_move(pos, uci: str) -> np.ndarray:
    p = _pos(pos)
    _check(lib().perft_apply_uci_move(ctypes.byref(p), uci.encode()), f"apply_move({uci})")
    return _arr(p)


def position_from_moves(fen: str, moves: Iterable[str]) -> np.ndarray:
    pos = fen_to_pos(fen)
    for m in moves:
        pos = apply_move(pos, m)
    return pos


def random_playouts(seed: int, n: int, min_plies: int, max_plies: int) -> np.ndarray:
    out = np.zeros((n, 6), dtype=np.uint64)
    _check(lib().perft_random_playouts(seed, n, min_plies, max_plies, out.ctypes.data), "random_playouts")
    return out


FEATURE_EP = 1
FEATURE_PAWN_ON_7TH = 2
FEATURE_CASTLING = 4
FEATURE_IN_CHECK = 8
FEATURE_PROMOTION = 16


def features(pos) -> int:
    p = _pos(pos)
    f = ctypes.c_uint32(0)
    _check(lib().perft_position_features(ctypes.byref(p), ctypes.byref(f)), "features")
    return int(f.value)


__all__ = [
    "PerftError", "init", "shutdown", "perft", "perft_batch", "perft_batch_device", "divide",
    "stats", "reset_stats", "fen_to_pos", "pos_to_fen", "legal_moves", "apply_move",
    "position_from_moves", "random_playouts", "features", "START_FEN", "LIB_PATH", "lib",
]
