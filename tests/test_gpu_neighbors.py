"""Neighbourhood summaries of the visible points (gpu.py:777-905) against the oracle, and the ground labels that
use their normals (perception.py:98-101). Counts, normals and curvature are bit-exact: the sums are fixed point and
the covariance float64 on both sides."""

import numpy as np
import pytest

import common
from oracle import oracle

pytestmark = pytest.mark.gpu


def _cloud(n_frames=6):
    """World points of a few handheld frames in the box room (walls, floor, boxes)."""
    frames = common.handheld_frames(n_frames)
    traj = common.handheld()
    pts = []
    for k, (x, a, t) in enumerate(frames):
        T = common.mid_pose(traj, k)
        pts.append(x.astype(np.float64) @ T[:3, :3].T + T[:3, 3])
    return np.concatenate(pts).astype(np.float32), common.mid_pose(traj, n_frames - 1)[:3, 3]


@pytest.mark.parametrize("radius,normals", [(0.1, True), (0.3, True), (0.2, False)])
def test_neighborhoods_bit_exact(radius, normals):
    from livox_warp import gpu

    xyz, sensor = _cloud()
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    pipe.load_points(xyz)
    n = pipe.count
    assert n == len(xyz)
    pipe.neighborhoods(radius, normals, sensor)
    cnt = pipe.nbr[:n].cpu().numpy()
    ocnt, onrm, ocurv = oracle.neighborhoods(xyz, radius, normals, sensor)
    assert np.array_equal(cnt, ocnt)
    assert cnt.min() >= 1 and np.median(cnt) > 5
    assert 0 < pipe.nb_voxels < n
    assert pipe.normals_valid == normals
    if normals:
        nrm = pipe.nrm[:n].cpu().numpy()
        curv = pipe.curv[:n].cpu().numpy()
        assert np.array_equal(nrm, onrm) and np.array_equal(curv, ocurv)
        assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-5)
        # normals face the sensor and flat surfaces are flat
        assert ((nrm * (sensor - xyz)).sum(1) >= -1e-4).all()
        assert np.median(curv) < 0.1


def test_ground_with_normals_matches_oracle():
    """build(neighbors='normals') then ground(use_normals=True): the labels the oracle gives with the same normals;
    the normals change some labels (a wall's foot inside the ground band is not ground)."""
    from livox_warp import gpu
    from livox_warp.perception import Perception

    xyz, sensor = _cloud()
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    pipe.load_points(xyz)
    n = pipe.count
    pipe.neighborhoods(0.15, True, sensor)
    perc = Perception(pipe)
    kw = dict(cell=0.5, thick=0.15, min_sup=3, thresh=0.2, slope_step=0.3)
    perc.ground(use_normals=True, nz_min=0.7, **kw)
    gnd = pipe.gnd[:n].cpu().numpy()
    nrm = pipe.nrm[:n].cpu().numpy()
    og, oh = oracle.ground(xyz, nrm=nrm, nz_min=0.7, **kw)
    assert np.array_equal(gnd, og) and np.array_equal(pipe.hag[:n].cpu().numpy(), oh)
    plain, _ = oracle.ground(xyz, **kw)
    assert (plain != og).any() and og.sum() < plain.sum()


def test_build_with_neighbors_fills_the_visible_set():
    from livox_warp import gpu

    frames = common.handheld_frames(6)
    traj = common.handheld()
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    view = gpu.make_view(now=0.6, voxel=0.1, map_cap=pipe.map_cap)
    for k, (x, a, t) in enumerate(frames):
        T = common.mid_pose(traj, k).astype(np.float32)
        pipe.set_pose(k, T)
        sx, sa, st, sf = pipe.stage(x, a, t, len(t), 10.0)
        pipe.map_insert(sx, sa, st, sf, len(t), view, 0.1)
    sensor = common.mid_pose(traj, 5)[:3, 3]
    n = pipe.build(view, map_on=True, neighbors="normals", radius=0.3, sensor=sensor)
    assert n > 100 and pipe.normals_valid
    vis = pipe.c_xyz[:n].cpu().numpy()
    ocnt, onrm, ocurv = oracle.neighborhoods(vis, 0.3, True, sensor)
    assert np.array_equal(pipe.nbr[:n].cpu().numpy(), ocnt)
    assert np.array_equal(pipe.nrm[:n].cpu().numpy(), onrm)
    n2 = pipe.build(view, map_on=True)  # a plain build invalidates the normals
    assert n2 == n and not pipe.normals_valid
    with pytest.raises(ValueError):
        pipe.build(view, map_on=True, neighbors="everything")
