"""Seeded synthetic perft workloads.

The reference measures on hand-picked known positions; these seeded
generators stand in for them with the shapes the benchmark configurations
name (random legal playouts from the initial position, stratified so the
special rules are exercised).  Every generator is deterministic in its seed.

  start_position()         initial position (depth 5: the no-TT start-position run)
  batch_positions(...)     4096 playouts of 8-30 plies, depth U[4,6], stratified:
                           >=10% with a legal en-passant capture, >=10% with a
                           pawn of the side to move on its 7th rank, >=10%
                           keeping a castling right
  deep_position(...)       one 20-ply playout with >= 35 legal moves (depth 8)
  tt_positions(...)        4 playouts of 12-24 plies (depths 9-10, TT runs)
  serving_trace(...)       Poisson arrivals of 0-40-ply positions, depth U[3,7]
"""
from __future__ import annotations

import numpy as np

from . import (FEATURE_CASTLING, FEATURE_EP, FEATURE_PAWN_ON_7TH, START_FEN, features, fen_to_pos,
               legal_moves, random_playouts)


def start_position() -> np.ndarray:
    return fen_to_pos(START_FEN)


def batch_positions(n: int = 4096, seed: int = 2026, min_plies: int = 8, max_plies: int = 30,
                    min_depth: int = 4, max_depth: int = 6, quota: float = 0.10):
    """Stratified batch; returns (positions (n,6) uint64, depths (n,) uint8)."""
    need = int(np.ceil(quota * n))
    pools = {FEATURE_EP: [], FEATURE_PAWN_ON_7TH: [], FEATURE_CASTLING: []}
    general = []
    chunk = 8192
    stream = 0
    while (len(general) < n or any(len(v) < need for v in pools.values())):
        cand = random_playouts(seed * 1000003 + stream, chunk, min_plies, max_plies)
        stream += 1
        for p in cand:
            f = features(p)
            placed = False
            for bit, pool in pools.items():
                if (f & bit) and len(pool) < need:
                    pool.append(p)
                    placed = True
                    break
            if not placed and len(general) < n:
                general.append(p)
        if stream > 200:
            raise RuntimeError("stratified generator did not fill its quotas")
    chosen = [p for pool in pools.values() for p in pool]
    chosen += general[: n - len(chosen)]
    rng = np.random.default_rng(seed)
    order = rng.permutation(n)
    pos = np.stack(chosen)[order].astype(np.uint64)
    depths = rng.integers(min_depth, max_depth + 1, size=n).astype(np.uint8)
    return pos, depths


def deep_position(seed: int = 8, plies: int = 20, min_moves: int = 35) -> np.ndarray:
    stream = 0
    while True:
        cand = random_playouts(seed * 7919 + stream, 256, plies, plies)
        stream += 1
        for p in cand:
            if len(legal_moves(p)) >= min_moves:
                return p


def tt_positions(seed: int = 9, n: int = 4, min_plies: int = 12, max_plies: int = 24):
    pos = random_playouts(seed, n, min_plies, max_plies)
    rng = np.random.default_rng(seed)
    depths = rng.integers(9, 11, size=n).astype(np.uint8)
    return pos, depths


def serving_trace(n: int = 10000, rate_qps: float = 1000.0, seed: int = 5,
                  min_depth: int = 3, max_depth: int = 7):
    """(positions, depths, arrival times in seconds) of a Poisson query trace."""
    pos = random_playouts(seed, n, 0, 40)
    rng = np.random.default_rng(seed)
    depths = rng.integers(min_depth, max_depth + 1, size=n).astype(np.uint8)
    arrivals = np.cumsum(rng.exponential(1.0 / rate_qps, size=n))
    return pos, depths, arrivals
