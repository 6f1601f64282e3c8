"""The reference's Odometry / Pipeline API end to end on the GPU: frames fed through Pipeline.stage ->
Odometry.push exactly as the reference's own test drives it (tests/check_odometry.py:30-51), compared with the
float64 oracle running the same frame state machine, and with the simulated ground truth.
"""

import numpy as np
import pytest
import torch

import common
from oracle import oracle

pytestmark = pytest.mark.gpu

RATE = 100000.0


def _run_gpu(frames, T0, voxel, on_frame=None, **tune):
    from livox_warp import gpu
    from livox_warp.odom import Odometry

    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    odom = Odometry(pipe, reg_slots=1 << 19, frame_cap=1 << 15)
    odom.reg_voxel = voxel
    for k, v in tune.items():
        setattr(odom, k, v)
    odom.reset(T0)
    for k, (x, a, t) in enumerate(frames):
        sx, sa, st, sf = pipe.stage(x, a, t, len(t), 1.0 / odom.frame_dt)
        odom.push(sx, sa, st, len(t), float(t.min()), float(t.max()), on_frame)
    odom.flush(on_frame)
    return pipe, odom


def test_odometry_tracks_ground_truth_and_float64_oracle():
    n = 45
    frames = common.handheld_frames(n)
    traj = common.handheld()
    T0 = common.mid_pose(traj, 0)
    voxel = 0.2
    _, odom = _run_gpu(frames, T0, voxel)
    recs = odom.traj
    assert len(recs) == n
    # the float64 oracle through the same state machine
    p = oracle.Params(reg_voxel=voxel)
    oo = oracle.Odometry(1 << 19, p, T0)
    for k, (x, a, t) in enumerate(frames):
        oo.frame(k, common.raw4(x, t), a)
    err_gt, err_or = [], []
    for (k, tm, T), (ko, tmo, To) in zip(recs, oo.traj):
        assert k == ko and abs(tm - tmo) < 1e-9
        gt = traj.poses(np.array([tm]))[0]
        err_gt.append(oracle.pose_error(gt, T))
        err_or.append(oracle.pose_error(To, T))
    err_gt, err_or = np.array(err_gt), np.array(err_or)
    st = odom.stats
    assert st["frames"] == n and st["keyframes"] >= 8 and st["iters"] > 0
    # ground truth: the reference's own walk gates are rmse < 15 cm, rot rmse < 2 deg (check_odometry.py:96-97)
    assert np.sqrt(np.mean(err_gt[:, 0] ** 2)) < 0.05, err_gt[:, 0].max()
    assert np.sqrt(np.mean(err_gt[:, 1] ** 2)) < 1.0
    # float64 oracle: float32 kernels vs float64 host math over a whole sequence stay within a few mm
    assert err_or[:, 0].max() < 5e-3 and err_or[:, 1].max() < 0.1, err_or.max(axis=0)


def test_on_frame_callback_and_map_insert():
    """on_frame hands the deskewed frame (borrowed device buffers) and its pose; map_insert + carve run on it."""
    from livox_warp import gpu

    frames = common.handheld_frames(14)
    traj = common.handheld()
    T0 = common.mid_pose(traj, 0)
    seen = []
    holder = {}

    def on_frame(k, T, fx, fa, ft, ff, m):
        pipe = holder["pipe"]
        view = gpu.make_view(now=float((k + 1) * 0.1), voxel=0.1, map_cap=pipe.map_cap)
        pipe.map_insert(fx, fa, ft, ff, m, view, 0.1)
        pipe.carve(fx, fa, ff, m, 0.1, every=1)
        seen.append((k, T.copy(), m))

    from livox_warp import gpu as g
    from livox_warp.odom import Odometry

    pipe = g.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    holder["pipe"] = pipe
    odom = Odometry(pipe, reg_slots=1 << 19, frame_cap=1 << 15)
    odom.reg_voxel = 0.2
    odom.reset(T0)
    for x, a, t in frames:
        sx, sa, st, sf = pipe.stage(x, a, t, len(t), 10.0)
        odom.push(sx, sa, st, len(t), float(t.min()), float(t.max()), on_frame)
    assert [s[0] for s in seen] == list(range(13))
    assert all(s[2] == len(frames[s[0]][2]) for s in seen)
    torch.cuda.synchronize()
    occupied = int((pipe.map_keys != -1).sum())
    assert occupied > 1000 and int(pipe.map_stats[0]) == occupied
    # the pose table holds each solved frame's pose for the frame id
    for k, T, _ in seen[-3:]:
        assert np.allclose(pipe.poses[k].cpu().numpy().reshape(4, 4), T, atol=1e-6)
        assert int(pipe.owner_frame[k]) == k


def test_pipeline_rejects_bad_capacity():
    from livox_warp import gpu

    with pytest.raises(ValueError):
        gpu.Pipeline(ring_capacity=1 << 10, map_capacity=1000)


@pytest.mark.parametrize("motion", ["static", "turn"])
def test_odometry_static_and_turn_gates(motion):
    """The reference's odometry gates (check_odometry.py:92-95) on the box room. At rest for 6 s: > 90 % of the
    frames after warm-up registered, rmse < 2 cm, rotation error < 0.2 deg. Turning in place for 15 s from the
    middle of the room: > 90 % registered, over 20 deg turned, rmse < 10 cm. The reference's rotation gate for the
    turn (rmse < 0.5 deg) is set for its own simulated sensor; with the 38-degree rosette each frame turns into
    mostly unseen surfaces and the float64 oracle itself reaches 0.72 deg at this 4 deg/s (1.85 deg at 12 deg/s),
    so here the rotation rmse is held below 1 deg, and the device to the oracle: 5 mm / 0.1 deg over the first 60
    frames, 3 cm / 1 deg over the whole turn."""
    import math

    from livox_warp import synth

    sc = common.room(1)
    if motion == "static":
        T0 = common.config1_pose()
        traj = synth.ConstantVelocity(T0, 1e9, 0.0, 0.0)
        n = 60
    else:
        T0 = common.look_at([4.0, 3.0, 1.4], [8.0, 3.5, 1.0])
        traj = synth.ConstantVelocity(T0, 1.0, 0.0, math.radians(4.0))
        n = 150
    frames = synth.frames(sc, traj, n, RATE, seed=5)
    Ts = traj.poses(np.array([0.05]))[0]
    _, odom = _run_gpu(frames, Ts, 0.2)
    recs = odom.traj
    err_t, err_r, span_r = [], [], []
    for _, tm, T in recs:
        gt = traj.poses(np.array([tm]))[0]
        e = oracle.pose_error(gt, T)
        err_t.append(e[0])
        err_r.append(e[1])
        span_r.append(oracle.pose_error(T0, gt)[1])
    err_t, err_r = np.array(err_t), np.array(err_r)
    # registration evidence after the warm-up: the frames whose registration ran and succeeded
    log = odom.iteration_log()
    n_post = sum(1 for k, _, _ in recs if k >= odom.warmup + 2)
    reg = int((log[:, 0] >= odom.warmup + 2).sum()) / max(1, n_post)
    assert reg > 0.9, reg
    if motion == "static":
        assert np.sqrt(np.mean(err_t ** 2)) < 0.02 and err_r.max() < 0.2, (err_t.max(), err_r.max())
        return
    assert max(span_r) > 20.0
    assert np.sqrt(np.mean(err_t ** 2)) < 0.10 and np.sqrt(np.mean(err_r ** 2)) < 1.0, (err_t.max(), err_r.max())
    oo = oracle.Odometry(1 << 19, oracle.Params(reg_voxel=0.2), Ts)
    for k, (x, a, t) in enumerate(frames):
        oo.frame(k, common.raw4(x, t), a)
    d = np.array([oracle.pose_error(To, T) for (_, _, T), (_, _, To) in zip(recs, oo.traj)])
    assert len(oo.traj) == len(recs)
    # float32 kernels vs float64 host math: within 5 mm / 0.1 deg over the first 60 frames; over the whole turn the
    # two drift apart by ~1.5 cm (each frame registers against a map built from the previous poses)
    assert d[:60, 0].max() < 5e-3 and d[:60, 1].max() < 0.1, d[:60].max(axis=0)
    assert d[:, 0].max() < 0.03 and d[:, 1].max() < 1.0, d.max(axis=0)
