"""Plane-layout array views (baking_b200/arrays.py), including the empty and single-particle cases
the kernels' C ABI receives."""
import numpy as np
import torch

from baking_b200 import arrays


def test_views_walk_the_planes():
    m = arrays.mat33s(5, device="cpu")
    m.copy_(torch.arange(45.0).reshape(5, 3, 3))
    assert arrays.layout_pitch(m) == 64 and m.stride() == (1, 192, 64)
    np.testing.assert_array_equal(arrays.to_numpy(m), np.arange(45.0).reshape(5, 3, 3))


def test_empty_and_single_arrays_share_a_pitch():
    for n in (0, 1):
        x = arrays.from_numpy(np.zeros((n, 3), np.float32), "f4", "cpu")
        C = arrays.from_numpy(np.zeros((n, 3, 3), np.float32), "f4", "cpu")
        s = arrays.from_numpy(np.zeros(n, np.float32), "f4", "cpu")
        assert arrays.common_pitch(x, C, s) == 64
        assert arrays.to_numpy(C).shape == (n, 3, 3)
