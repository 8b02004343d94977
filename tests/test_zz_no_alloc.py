"""The allocation-free entry point, perft_batch_noalloc, through the C ABI.

It serves callers that cannot allocate device memory (their HBM is held by
another allocator, or cudaMalloc's device-wide synchronisation is not
acceptable where they run).  Its results must equal the arena entry point's,
call after call, although every call reuses the same static scratch array.

Collected last (file name) so that a failure here leaves every other test
already run; it also passes alone in a fresh process.
"""
import ctypes
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(pg, d_pos, depths, n, d_out, stream=None):
    fn = pg.lib().perft_batch_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    d = np.ascontiguousarray(depths, dtype=np.uint8)
    return fn(d_pos, d.ctypes.data, n, d_out, stream)


def test_noalloc_matches_arena_entry_point_twice():
    import torch
    import perft_gpu_b200 as pg

    pos = pg.random_playouts(seed=2027, n=96, min_plies=2, max_plies=50)
    depths = np.array([i % 5 for i in range(len(pos))], dtype=np.uint8)  # depths 0..4
    start = pg.fen_to_pos(pg.START_FEN)
    pos = np.vstack([pos, start.reshape(1, 6)])
    depths = np.append(depths, np.uint8(5))
    n = len(pos)

    pg.init(device=0, arena_bytes=1 << 30)
    want = pg.perft_batch(pos, depths)  # the existing (arena) entry point

    d_pos = torch.from_numpy(pos.view(np.int64)).cuda()
    d_out = torch.full((n,), -1, dtype=torch.int64, device="cuda")
    after_first = None
    for call in range(2):
        d_out.fill_(-1)  # the entry point must clear its own outputs
        torch.cuda.synchronize()
        rc = _noalloc(pg, d_pos.data_ptr(), depths, n, d_out.data_ptr())
        assert rc == pg.PERFT_OK, (call, rc)
        got = d_out.cpu().numpy().view(np.uint64)
        assert np.array_equal(got, want), (call, np.nonzero(got != want)[0][:5])
        if call == 0:
            after_first = (torch.cuda.memory_allocated(), torch.cuda.memory_reserved(),
                           torch.cuda.mem_get_info()[0])
    # the second call took nothing from this process's allocator
    assert (torch.cuda.memory_allocated(), torch.cuda.memory_reserved()) == after_first[:2]
    # device-wide free memory also counts other processes on a shared GPU, so
    # a change there is reported, not failed
    if torch.cuda.mem_get_info()[0] != after_first[2]:
        warnings.warn("device free memory changed between the two calls (another process?)")


def test_noalloc_refuses_oversized_trees():
    import torch
    import perft_gpu_b200 as pg

    start = pg.fen_to_pos(pg.START_FEN).reshape(1, 6)
    d_pos = torch.from_numpy(start.view(np.int64)).cuda()
    d_out = torch.zeros(1, dtype=torch.int64, device="cuda")
    # depth 7 needs a 4.9M-node ply: far beyond the 32 MiB scratch.  The
    # refusal comes after work was queued on the caller's stream; the call
    # still returns only once that stream has finished.
    side = torch.cuda.Stream()
    rc = _noalloc(pg, d_pos.data_ptr(), np.array([7], dtype=np.uint8), 1, d_out.data_ptr(), side.cuda_stream)
    assert rc == pg.PERFT_ERR_OUT_OF_MEMORY
    assert side.query()
    # and the scratch is still usable afterwards
    rc = _noalloc(pg, d_pos.data_ptr(), np.array([4], dtype=np.uint8), 1, d_out.data_ptr())
    assert rc == pg.PERFT_OK and int(d_out.cpu()[0]) == 197281
