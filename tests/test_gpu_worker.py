"""OdomWorker (slam_worker.py:100-338) on the GPU: the odometry on its own thread and streams gives the same frames,
poses and deskewed points as the direct calls, bit for bit; generations, own-or-drop and configure() as the
reference defines them."""

import time

import numpy as np
import pytest
import torch

import common

pytestmark = pytest.mark.gpu

VOXEL = 0.2


def _direct(frames, T0):
    from livox_warp import gpu
    from livox_warp.odom import Odometry

    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    odom = Odometry(pipe, reg_slots=1 << 19, frame_cap=1 << 15)
    odom.reg_voxel = VOXEL
    odom.reset(T0)
    out = {}

    def on_frame(k, T, fx, fa, ft, ff, m):
        out[k] = (T.copy(), m, fx[:m].clone(), fa[:m].clone())

    for x, a, t in frames:
        sx, sa, st, sf = pipe.stage(x, a, t, len(t), 1.0 / odom.frame_dt)
        odom.push(sx, sa, st, len(t), float(t.min()), float(t.max()), on_frame)
    torch.cuda.synchronize()
    return out


def _collect(w, want, timeout=120.0):
    got = {}
    t0 = time.time()
    while len(got) < want and time.time() - t0 < timeout and w._thread.is_alive():
        for r in w.poll():
            arr = r.arrays()  # empty when the output slots were all taken (own-or-drop): the pose still arrives
            got[r.k] = (r.T, r.m, arr[0].clone() if arr else None, arr[1].clone() if arr else None, r.gen,
                        arr[2].cpu().numpy() if arr else None, arr[3].cpu().numpy() if arr else None)
        torch.cuda.current_stream().synchronize()
        w.release_consumed()
        time.sleep(0.002)
    return got


def test_worker_matches_direct_odometry():
    from livox_warp import gpu
    from livox_warp.slam_worker import OdomWorker

    frames = common.handheld_frames(30)
    T0 = common.mid_pose(common.handheld(), 0)
    want = _direct(frames, T0)
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    w = OdomWorker(pipe, frame_cap=1 << 15, reg_slots=1 << 19, in_slots=64, out_slots=64)
    try:
        w.configure(reg_voxel=VOXEL)
        w.reset(T0)
        for x, a, t in frames:
            sx, sa, st, sf = pipe.stage(x, a, t, len(t), 10.0)
            assert w.submit(sx, sa, st, len(t), float(t.min()), float(t.max()))
        got = _collect(w, len(want))
        st = w.status()
    finally:
        w.close()
    assert sorted(got) == sorted(want) and len(want) == len(frames) - 1  # the last frame is still open
    for k in want:
        T, m, fx, fa = want[k]
        gT, gm, gx, ga, gen, gt, gf = got[k]
        assert np.array_equal(gT, T) and gm == m and gen == 1
        assert torch.equal(gx, fx) and torch.equal(ga, fa)
        # no torn snapshot (check_slam_worker.py:156-163): the frame's points carry its own frame id (or the
        # previous one, for slightly late points) and times within a frame of it
        assert np.isin(gf, [k & 0xFFFF, (k - 1) & 0xFFFF]).all()
        assert ((gt >= (k - 1) * 0.1 - 1e-4) & (gt < (k + 1) * 0.1 + 1e-4)).all()
    assert st["drops"] == {"input_full": 0, "input_own": 0, "output_pool": 0, "stale": 0, "error": 0}, st
    assert st["processed"] == len(frames) and st["frames"] == len(want)


def test_reset_drops_the_old_generation():
    """After reset() nothing of the old generation reaches the caller, and the new generation starts over."""
    from livox_warp import gpu
    from livox_warp.slam_worker import OdomWorker

    frames = common.handheld_frames(12)
    T0 = common.mid_pose(common.handheld(), 0)
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    w = OdomWorker(pipe, frame_cap=1 << 15, reg_slots=1 << 19, in_slots=64)
    try:
        w.configure(reg_voxel=VOXEL)
        w.reset(T0)
        for x, a, t in frames:
            sx, sa, st, sf = pipe.stage(x, a, t, len(t), 10.0)
            w.submit(sx, sa, st, len(t), float(t.min()), float(t.max()))
        w.reset(T0)  # everything above is now stale
        for x, a, t in frames[:6]:
            sx, sa, st, sf = pipe.stage(x, a, t, len(t), 10.0)
            assert w.submit(sx, sa, st, len(t), float(t.min()), float(t.max()))
        got = _collect(w, 5)
        st = w.status()
        gen = w.gen
    finally:
        w.close()
    assert gen == 2 and sorted(got) == list(range(5)) and all(v[4] == gen for v in got.values())
    assert st["drops"]["error"] == 0 and st["drops"]["input_full"] == 0


def test_own_or_drop_and_configure():
    from livox_warp import gpu
    from livox_warp.slam_worker import OdomWorker

    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    w = OdomWorker(pipe, frame_cap=1 << 15, reg_slots=1 << 19, in_slots=2, in_cap=1000)
    try:
        x = torch.zeros((5000, 3), dtype=torch.float32, device="cuda")
        a = torch.zeros(5000, dtype=torch.int32, device="cuda")
        t = torch.zeros(5000, dtype=torch.float32, device="cuda")
        assert not w.submit(x, a, t, 5000, 0.0, 0.05)  # larger than an input slot
        assert w.status()["drops"]["input_own"] == 1
        with pytest.raises(AttributeError):
            w.configure(no_such_knob=1)
        w.configure(max_iter=8)
    finally:
        w.close()
    assert w.odom.max_iter == 8 and not w._thread.is_alive()


def test_restart_clock_keeps_going_on_the_new_clock():
    """A replay loop: the clock restarts at 0; after restart_clock() the frames of the new clock arrive (new
    generation, frame ids from 0 again) and nothing of the old clock does."""
    from livox_warp import gpu
    from livox_warp.slam_worker import OdomWorker

    frames = common.handheld_frames(8)
    T0 = common.mid_pose(common.handheld(), 0)
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 18)
    w = OdomWorker(pipe, frame_cap=1 << 15, reg_slots=1 << 19, in_slots=64)
    try:
        w.configure(reg_voxel=VOXEL)
        w.reset(T0)
        for x, a, t in frames:
            sx, sa, st, sf = pipe.stage(x, a, t, len(t), 10.0)
            assert w.submit(sx, sa, st, len(t), float(t.min()), float(t.max()))
        first = _collect(w, 7)
        w.restart_clock()
        for x, a, t in frames[:5]:
            sx, sa, st, sf = pipe.stage(x, a, t, len(t), 10.0)
            assert w.submit(sx, sa, st, len(t), float(t.min()), float(t.max()))
        second = _collect(w, 4)
        gen, st = w.gen, w.status()
    finally:
        w.close()
    assert sorted(first) == list(range(7)) and all(v[4] == 1 for v in first.values())
    assert gen == 2 and sorted(second) == list(range(4)) and all(v[4] == 2 for v in second.values())
    assert st["drops"]["error"] == 0
