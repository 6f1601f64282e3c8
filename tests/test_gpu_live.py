"""The live ring's visible set on the GPU (k_classify_live, gpu.py:637-697, and Pipeline.build's live mode
:1466-1504) against the oracle, bit for bit and in ring order: a ring that has wrapped, points older than the
persistence dropped, odometry on (deskewed by each frame's twist, a frame whose pose slot holds another epoch
not drawn) and off, the crop box, and Motion labels from a carved map's history."""

import numpy as np
import pytest

import common
from oracle import oracle

pytestmark = pytest.mark.gpu

VOXEL = 0.1


def _feed():
    from livox_warp import gpu

    traj = common.handheld()
    frames = common.handheld_frames(16)[10:16]
    pipe = gpu.Pipeline(ring_capacity=1 << 15, map_capacity=1 << 18)
    om = oracle.Map(pipe.map_cap)
    poses = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (oracle.POSE_SLOTS, 1))
    mv = gpu.make_view(now=1.6, voxel=VOXEL, map_cap=pipe.map_cap)
    total = 0
    for j, (x, a, t) in enumerate(frames):
        k = 10 + j
        T = common.mid_pose(traj, k).astype(np.float32)
        twist = np.array([0.03, -0.01, 0.005, 0.01, -0.02, 0.12], np.float32) * (1 + 0.1 * j)
        pipe.set_pose(k, T, twist, epoch=0 if k == 12 else 1)
        poses[k & (oracle.POSE_SLOTS - 1)] = T.reshape(16)
        n = len(t)
        total += n
        sx, sa, st, sf = pipe.stage(x, a, t, n, 10.0)
        pipe.ingest_ring(sx, sa, st, sf, n)
        fid = common.frame_ids(t)
        pipe.map_insert(sx, sa, st, sf, n, mv, VOXEL)
        om.insert(x, a, t, fid, poses, mv, VOXEL)
        pipe.carve(sx, sa, sf, n, VOXEL, every=1)
        om.carve(x, a, fid, poses, VOXEL, every=1)
    assert total > pipe.cap  # the ring has wrapped: ring order is not time order
    return pipe, om


@pytest.mark.parametrize("odo", [10.0, 0.0])
def test_live_build_bit_exact(odo):
    from livox_warp import gpu

    pipe, om = _feed()
    v = gpu.make_view(now=1.6, persist=0.32, voxel=VOXEL, map_cap=pipe.map_cap, inv_frame_dt=odo, epoch=1, dyn_on=1,
                      dyn_settle=0.3, carve_on=1, carve_ratio=0.5, carve_min=1, carve_stale=0.05, crop_on=1,
                      crop_lo=(-50.0, -50.0, -0.5), crop_hi=(50.0, 50.0, 2.2), min_refl=5)
    count = pipe.build(v, map_on=False)
    ring = [pipe.ring_xyz.cpu().numpy(), pipe.ring_attr.cpu().numpy(), pipe.ring_t.cpu().numpy(),
            pipe.ring_frame.cpu().numpy()]
    table = [pipe.poses.cpu().numpy(), pipe.tw.cpu().numpy(), pipe.owner_frame.cpu().numpy(),
             pipe.owner_epoch.cpu().numpy()]
    ox, oa, ot, od = om.live_build(*ring, pipe.filled, *table, v)
    assert count == len(ox) > 1000
    assert np.array_equal(pipe.c_xyz[:count].cpu().numpy(), ox)
    assert np.array_equal(pipe.c_attr[:count].cpu().numpy().view(np.uint32), oa)
    assert np.array_equal(pipe.c_t[:count].cpu().numpy(), ot)
    gd = pipe.c_dyn[:count].cpu().numpy()
    assert np.array_equal(gd, od) and 0 < gd.sum() < count
    frames = np.floor(ot * 10).astype(int)
    # the ring holds the last 2768 points of frame 12 (t >= 1.272), persistence keeps those after 1.28
    assert frames.min() >= 12 and (12 not in frames) == (odo > 0)


def test_live_build_empty_ring():
    from livox_warp import gpu

    pipe = gpu.Pipeline(ring_capacity=1 << 12, map_capacity=1 << 12)
    v = gpu.make_view(now=1.0, voxel=VOXEL, map_cap=pipe.map_cap)
    assert pipe.build(v, map_on=False) == 0
