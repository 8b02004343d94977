"""Multi-GPU split of the perft path: one process per GPU over
torch.distributed, the units (positions of a batch, or the frontier boards of
one deep position) dealt across ranks, and one small sum as the only exchange.

This follows the reference's subtree parallelism (launcher.h:409-583: root
children dealt to one host thread per GPU, the subtotals summed on the host).
There are no cross-GPU loads: every rank searches its own subtrees with its own
engine and transposition table, and the per-position or per-move counts are
summed with one all-reduce (16 bytes each: two 32-bit halves, exact at any
size).

The counting function is a parameter so that the dealing and reduction logic
can run on CPU ranks (gloo) with any counter; by default it is the GPU engine.
"""
import numpy as np


def strided(n: int, rank: int, world: int) -> np.ndarray:
    """Indices of the units rank `rank` of `world` takes: every world-th from
    `rank`.  Costs of neighbouring positions are unrelated, so a stride deals
    them evenly on average."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    return np.arange(rank, n, world, dtype=np.int64)


def _world(group):
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return None, 0, 1
    return dist, dist.get_rank(group), dist.get_world_size(group)


def _sum_u64(values: np.ndarray, dist, group, device) -> list:
    """Element-wise sum over ranks of u64 counts, exact as Python ints at any
    size (a per-move subtotal summed over shards may pass 2^64): each value
    travels as its two 32-bit halves in int64 lanes, whose sums cannot
    overflow for fewer than 2^31 ranks."""
    import torch
    v = np.ascontiguousarray(values, dtype=np.uint64).reshape(-1)
    halves = np.stack([v >> np.uint64(32), v & np.uint64(0xFFFFFFFF)]).astype(np.int64)
    t = torch.from_numpy(halves).to(device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    hi, lo = t.cpu().numpy()
    return [(int(h) << 32) + int(l) for h, l in zip(hi, lo)]


def max_sum_over_ranks(maxes, sums, device="cpu", group=None):
    """(per-entry max over ranks of `maxes`, per-entry sum of `sums`): the
    timing reduction of a multi-rank run (slowest rank's device time, total
    work of all ranks)."""
    import torch
    dist, _, _ = _world(group)
    t = torch.tensor(list(maxes), dtype=torch.float64, device=device)
    s = torch.tensor(list(sums), dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
        dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
    return [float(x) for x in t.cpu()], [float(x) for x in s.cpu()]


def perft_batch_sharded(pos: np.ndarray, depths, counter=None, group=None, device="cpu") -> np.ndarray:
    """perft of every position of a batch, positions dealt across ranks.
    Every rank gets the full result vector.  `counter(pos, depths) -> counts`
    defaults to the GPU engine's perft_batch."""
    if counter is None:
        from . import perft_batch as counter
    dist, rank, world = _world(group)
    pos = np.ascontiguousarray(pos, dtype=np.uint64).reshape(-1, 6)
    depths = np.ascontiguousarray(depths, dtype=np.uint8)
    mine = strided(len(pos), rank, world)
    out = np.zeros(len(pos), dtype=np.uint64)
    if len(mine):
        out[mine] = np.asarray(counter(pos[mine], depths[mine]), dtype=np.uint64)
    # one rank holds each position's count, so every sum fits 64 bits
    return np.array(_sum_u64(out, dist, group, device), dtype=np.uint64)


def deep_sharded(pos, depth: int, split_plies: int = 2, deep_fn=None, group=None, device="cpu"):
    """Deep perft of one position split across ranks: each rank searches every
    world-th distinct frontier board (perft_deep_shard), and the per-root-move
    subtotals are summed over ranks.  Returns (total, {uci move: count}) on
    every rank.  `deep_fn(pos, depth, split_plies, shard, n_shards)` defaults
    to the GPU engine's deep()."""
    if deep_fn is None:
        from . import deep as deep_fn
    dist, rank, world = _world(group)
    _, div = deep_fn(pos, depth, split_plies, rank, world)
    moves = list(div.keys())
    summed = _sum_u64(np.array([div[m] for m in moves], dtype=np.uint64), dist, group, device)
    result = dict(zip(moves, summed))
    return sum(result.values()), result
