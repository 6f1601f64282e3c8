"""The coarse search's hypothesis scores on the CPU: the exact-sum definition the library computes against the
reference's own float32 sum (k_score_grid, localize.py:55-96), the headings' table, and argument checks that run
before any CUDA call."""

import ctypes
import math

import numpy as np
import pytest

from oracle import oracle


@pytest.fixture(scope="module")
def scene_grid():
    from livox_warp import synth

    sc = synth.box_room(3)
    xyz, nrm = synth.sample_surfaces(sc, 0.03, 0, jitter=0.002)
    planar = np.ones(len(xyz), np.float32)
    og = oracle.PriorGrid(oracle.prior_prepare(xyz, nrm, planar))
    T = synth.free_poses(sc, 1, 3)[0]
    pts = synth.spin_scan(sc, T, 3000, 5)[:1024]
    return sc, og, T, pts


def test_exact_sum_matches_reference_sum(scene_grid):
    """Same poses, same cells: the exact sum and the reference's float32 point-order sum differ by that sum's
    rounding only -- at most n * 2^-24 of the total (the bound for adding n terms in [0, 1] in float32)."""
    sc, og, T, pts = scene_grid
    pos = np.stack(np.meshgrid(np.arange(0.5, 8.0, 0.5), np.arange(0.5, 6.0, 0.5), [1.0, 1.6], indexing="ij"),
                   -1).reshape(-1, 3).astype(np.float32)
    n_yaw = 36
    a = og.score_grid(pts, pos, n_yaw, 0.0, math.radians(10.0), 25.0, 10.0)
    b = og.score_grid(pts, pos, n_yaw, 0.0, math.radians(10.0), 25.0, 10.0, ref=True)
    assert np.array_equal(a == -1.0, b == -1.0) and (a == -1.0).any() and (a > 0).any()
    ok = a >= 0
    assert np.all(np.abs(a[ok] - b[ok]) <= len(pts) * 2.0 ** -24 * np.maximum(b[ok], 1.0))
    assert a.max() <= len(pts)
    lst = og.score_list(pts, np.concatenate([np.repeat(pos[:5], 3, 0), np.tile([[0.1], [1.0], [2.5]], (5, 1))], 1),
                        12.0)
    lst_ref = og.score_list(pts, np.concatenate([np.repeat(pos[:5], 3, 0), np.tile([[0.1], [1.0], [2.5]], (5, 1))],
                                                1), 12.0, ref=True)
    assert np.all(np.abs(lst - lst_ref) <= len(pts) * 2.0 ** -24 * np.maximum(lst_ref, 1.0))


def test_true_pose_scores_near_the_best(scene_grid):
    """Scoring works: the hypothesis at the scan's own position and heading is within a few points of the best."""
    sc, og, T, pts = scene_grid
    yaw = math.atan2(T[1, 0], T[0, 0])
    hyp = np.array([[T[0, 3], T[1, 3], T[2, 3], yaw], [T[0, 3] + 1.0, T[1, 3], T[2, 3], yaw],
                    [T[0, 3], T[1, 3], T[2, 3], yaw + 0.6]], np.float32)
    s = og.score_list(pts, hyp, 12.0)
    assert s[0] > 0.8 * len(pts) and s[0] > s[1] + 100 and s[0] > s[2] + 100


def test_yaw_table_matches_float64_rounding():
    from livox_warp import _lib

    lib = _lib.load(require_cuda=False)
    n, yaw0, dyaw = 180, 0.25, math.radians(2.0)
    c = (ctypes.c_float * n)()
    s = (ctypes.c_float * n)()
    lib.lw_score_yaw_table(n, ctypes.c_float(yaw0), ctypes.c_float(dyaw), c, s)
    yaw = np.float32(yaw0) + np.arange(n, dtype=np.float32) * np.float32(dyaw)
    np.testing.assert_allclose(np.array(c), np.cos(yaw.astype(np.float64)).astype(np.float32), rtol=0, atol=6e-8)
    np.testing.assert_allclose(np.array(s), np.sin(yaw.astype(np.float64)).astype(np.float32), rtol=0, atol=6e-8)


def test_score_arguments_checked_before_cuda():
    from livox_warp import _lib

    lib = _lib.load(require_cuda=False)
    assert lib.lw_score_grid(None, None, 0, None, 0, 1, 1, ctypes.c_float(0), ctypes.c_float(0), ctypes.c_float(25),
                             ctypes.c_float(10), None, None) == _lib.LW_EINVAL
    assert b"lw_score_grid" in lib.lw_last_error()
    assert lib.lw_score_list(None, None, 0, None, 0, ctypes.c_float(12), None, None) == _lib.LW_EINVAL
