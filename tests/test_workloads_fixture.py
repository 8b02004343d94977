"""The stored benchmark workloads (perft_gpu_b200/data/workloads.npz) equal
what the seeded generators produce today, so the bench's two arms (the GPU
engine and the reference's host perft, which reads only the stored file) and
the reference-count fixture all see the same positions."""
import numpy as np

from perft_gpu_b200.data import make_workloads


def test_stored_workloads_equal_generators():
    stored = make_workloads.load()
    fresh = make_workloads.generate()
    assert set(stored) == set(fresh)
    for k in fresh:
        assert stored[k].dtype == fresh[k].dtype, k
        assert np.array_equal(stored[k], fresh[k]), k


def test_stored_workload_shapes():
    w = make_workloads.load()
    assert w["batch_pos"].shape == (4096, 6) and w["batch_depths"].min() >= 4 and w["batch_depths"].max() <= 6
    assert w["deep_pos"].shape == (1, 6)
    assert w["tt_pos"].shape == (4, 6) and set(w["tt_depths"].tolist()) <= {9, 10}
    assert w["serve_pos"].shape == (10000, 6) and w["serve_depths"].min() >= 3 and w["serve_depths"].max() <= 7
