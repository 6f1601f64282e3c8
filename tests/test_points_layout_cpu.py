"""Which point arrays the integration map, carving and frame append read as they are (host logic, no GPU): float32
(n, 3) or (n, 4) rows 3 or 4 floats apart, including the (n, 3) x, y, z view of a float4 frame buffer that
on_frame hands out (the reference hands a vec3 array there, odom.py:657); anything else is refused before a
pointer reaches a kernel."""

import numpy as np
import torch

from livox_warp.gpu import _as_xyz, row_stride


def test_row_stride_of_accepted_layouts():
    buf = torch.zeros((10, 4), dtype=torch.float32)
    assert row_stride(buf) == 4
    assert row_stride(buf[:, :3]) == 4  # on_frame's f_xyz: x, y, z of the float4 rows
    assert row_stride(torch.zeros((10, 3), dtype=torch.float32)) == 3
    assert row_stride(buf[:5, :3]) == 4
    assert row_stride(torch.zeros((1, 3), dtype=torch.float32)) == 3
    assert row_stride(torch.zeros((0, 4), dtype=torch.float32)) == 4


def test_row_stride_refuses_what_the_kernels_cannot_read():
    buf = torch.zeros((10, 8), dtype=torch.float32)
    assert row_stride(buf[:, :3]) == 0  # rows 8 floats apart
    assert row_stride(torch.zeros((10, 4), dtype=torch.float32)[:, 1:]) == 4  # x at column 1: still 4 apart
    assert row_stride(torch.zeros((10, 3), dtype=torch.float64)) == 0
    assert row_stride(torch.zeros((10, 2), dtype=torch.float32)) == 0
    assert row_stride(torch.zeros((3, 10), dtype=torch.float32).t()) == 0  # columns not adjacent
    assert row_stride(torch.zeros(12, dtype=torch.float32)) == 0


def test_as_xyz_refuses_before_any_copy():
    bad = torch.zeros((10, 8), dtype=torch.float32)[:, :3]
    try:
        _as_xyz(bad, torch.device("cpu"))
    except ValueError:
        pass
    else:
        raise AssertionError("a (10, 3) view of rows 8 floats apart was accepted")
    ok = _as_xyz(np.zeros((4, 3), np.float32), torch.device("cpu"))
    assert ok.shape == (4, 3) and row_stride(ok) == 3
