"""Multi-GPU split of the perft path: one process per GPU over
torch.distributed, the units (positions of a batch, or the frontier boards of
one deep position) dealt across ranks, and one small sum as the only exchange.

This follows the reference's subtree parallelism (launcher.h:409-583: root
children dealt to one host thread per GPU, the subtotals summed on the host).
There are no cross-GPU loads: every rank searches its own subtrees with its own
engine and transposition table, and the per-position or per-move counts are
summed with one all-reduce (16 bytes each: two 32-bit halves, exact at any
size).

Dealing is dynamic, like the reference's idle GPU thread taking the next root
child: the units are cut into chunks, ordered largest-first by predicted cost,
and each rank takes the next chunk from a shared cursor (an atomic add on the
process group's key-value store) whenever it finishes one.  Subtree sizes of
the positions in a batch spread over orders of magnitude, so a fixed stride
can leave ranks idle while one finishes a run of large positions.  The static
stride (strided) is kept for callers without a store.

The counting function is a parameter so that the dealing and reduction logic
can run on CPU ranks (gloo) with any counter; by default it is the GPU engine.
"""
import itertools

import numpy as np

_deal_ids = itertools.count()


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


def default_store(group=None):
    """The key-value store of the default process group (its rendezvous store)."""
    import torch.distributed as dist
    from torch.distributed import distributed_c10d as c10d
    if not dist.is_initialized():
        return None
    return c10d._get_default_store()


def dealt_chunks(n_chunks: int, store, key: str):
    """Chunk indices this rank takes from the shared cursor `key`, in order,
    until all n_chunks are dealt.  Each store.add returns the cursor after
    this rank's increment, so every index goes to exactly one rank."""
    while True:
        j = int(store.add(key, 1)) - 1
        if j >= n_chunks:
            return
        yield j


def _next_key(tag):
    # every rank makes the same sequence of sharded calls, so the n-th call
    # of every rank uses the same key, and no two calls share one
    return f"perft_gpu_b200/deal/{tag}/{next(_deal_ids)}"


def perft_batch_sharded(pos: np.ndarray, depths, counter=None, group=None, device="cpu", store=None,
                        chunks_per_rank: int = 8, taken=None) -> np.ndarray:
    """perft of every position of a batch, positions dealt across ranks.
    Every rank gets the full result vector.  `counter(pos, depths) -> counts`
    defaults to the GPU engine's perft_batch.

    With more than one rank the positions are ordered by depth, deepest (most
    expensive) first, cut into chunks_per_rank x world chunks, and dealt from
    the store's shared cursor (dynamic); without a store they are dealt by
    stride.  `taken`, if a list, receives the chunk indices this rank took."""
    if counter is None:
        from . import perft_batch as counter
    dist, rank, world = _world(group)
    pos = np.ascontiguousarray(pos, dtype=np.uint64).reshape(-1, 6)
    depths = np.ascontiguousarray(depths, dtype=np.uint8)
    n = len(pos)
    out = np.zeros(n, dtype=np.uint64)
    if world > 1 and store is None:
        store = default_store(group)
    if world == 1 or store is None:
        mine = strided(n, rank, world)
        if len(mine):
            out[mine] = np.asarray(counter(pos[mine], depths[mine]), dtype=np.uint64)
    else:
        order = np.argsort(-depths.astype(np.int64), kind="stable")  # largest first
        n_chunks = max(1, min(n, chunks_per_rank * world))
        bounds = np.linspace(0, n, n_chunks + 1).astype(np.int64)
        for j in dealt_chunks(n_chunks, store, _next_key("batch")):
            idx = order[bounds[j]:bounds[j + 1]]
            if taken is not None:
                taken.append(j)
            if len(idx):
                out[idx] = np.asarray(counter(pos[idx], depths[idx]), dtype=np.uint64)
    # one rank holds each position's count, so every sum fits 64 bits
    return np.array(_sum_u64(out, dist, group, device), dtype=np.uint64)


def deep_sharded(pos, depth: int, split_plies: int = 2, deep_fn=None, group=None, device="cpu", store=None,
                 chunks_per_rank: int = 4, taken=None):
    """Deep perft of one position split across ranks, and the per-root-move
    subtotals summed over ranks.  Returns (total, {uci move: count}) on every
    rank.  `deep_fn(pos, depth, split_plies, shard, n_shards)` defaults to the
    GPU engine's deep() (perft_deep_shard: the frontier boards whose index is
    congruent to shard modulo n_shards).

    With more than one rank and a store, the frontier is cut into
    chunks_per_rank x world shards dealt dynamically from the store's shared
    cursor (the engine keeps the last frontier it built, so a rank's later
    shards do not enumerate it again); otherwise rank r searches shard r of
    world."""
    if deep_fn is None:
        from . import deep as deep_fn
    dist, rank, world = _world(group)
    if world > 1 and store is None:
        store = default_store(group)
    acc = {}
    if world == 1 or store is None:
        _, div = deep_fn(pos, depth, split_plies, rank, world)
        acc = {m: int(c) for m, c in div.items()}
    else:
        n_shards = chunks_per_rank * world
        moves = None
        for j in dealt_chunks(n_shards, store, _next_key("deep")):
            if taken is not None:
                taken.append(j)
            _, div = deep_fn(pos, depth, split_plies, j, n_shards)
            moves = moves or list(div.keys())
            for m, c in div.items():
                acc[m] = acc.get(m, 0) + int(c)
        if moves is None:
            # this rank took no shard: it still needs the move list for the
            # reduction, which every rank makes with the same entries
            _, div = deep_fn(pos, 1, 0, 0, 1)
            acc = {m: 0 for m in div}
    moves = list(acc.keys())
    summed = _sum_u64(np.array([acc[m] for m in moves], dtype=np.uint64), dist, group, device)
    result = dict(zip(moves, summed))
    return sum(result.values()), result
