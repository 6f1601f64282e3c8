"""The sequence-odometry configuration on the GPU against the oracle, per frame and at size.

* Per-frame precision, apart from drift: the float64 oracle runs the sequence's frame state machine; at every
  registration it makes, the device registers the same thinned frame from the same start against the same map (a
  device copy of the oracle's registration map, fed the oracle's keyframes -- the insert is bit-exact), and every
  pose lands within 1 mm / 0.01 deg of the oracle's. Drift over a sequence, where the two state machines follow
  their own poses, is a separate number (the benchmark's pose_drift).
* The integration map at size: 200 frames of the sequence through the device odometry with the 0.1 m,
  2^22-slot integration map and carving of every ray; the oracle inserts and carves the same deskewed frames with
  the same poses, and keys, counts, fixed-point sums, first / last times and misses are equal.
"""

import numpy as np
import pytest
import torch

import common
from oracle import oracle

pytestmark = pytest.mark.gpu

FRAME_DT = 0.1


def _sequence(n: int):
    """Frames 0 .. n-1 of the 600-frame sequence (box room, handheld spline <= 1 m/s, <= 60 deg/s)."""
    from livox_warp import synth

    scene = synth.box_room(1)
    traj = synth.Handheld(scene, 31, 62.0)
    return synth.frames(scene, traj, n, 100000.0, 3), traj


def _odom_params(p):
    from livox_warp import _lib

    prm = _lib.OdomParams()
    for name in ("frame_dt", "reg_voxel", "min_range", "max_range", "noise", "alpha", "damping", "velocity_smooth",
                 "degen_thr", "prior_info", "kf_dist", "max_iter", "warmup", "min_points", "min_corr", "ret_mask"):
        setattr(prm, name, getattr(p, name))
    prm.kf_angle_deg, prm.deskew, prm.redeskew, prm.frame_cap = p.kf_angle, 1, 1, 1 << 15
    return prm


def test_every_registration_of_the_sequence_within_1mm_of_float64():
    from livox_warp import kernels

    frames, traj = _sequence(80)
    p = oracle.Params(reg_voxel=0.15)
    prm = _odom_params(p)
    reg = kernels.RegistrationMap(1 << 19)
    gn = kernels.GnScratch()
    errors = []

    class Mirrored(oracle.Odometry):
        def _register(self, xyz4, attr, T_pred):
            ds = oracle.thin(xyz4, attr, np.float32(2.0 / p.reg_voxel), p.min_range, p.max_range, p.ret_mask)
            To, ok, st = oracle.register(ds, T_pred, self.reg, p)
            Tg, ok_g, sg = kernels.icp_solve(torch.from_numpy(ds).cuda(), T_pred, reg, prm, gn)
            assert ok_g == ok
            if ok:
                errors.append((*oracle.pose_error(To, Tg), st["iters"], sg["iters"]))
            return To, ok, st

    T0 = traj.poses(np.array([0.5 * FRAME_DT]))[0]
    oo = Mirrored(1 << 19, p, T0)
    for k, (x, a, t) in enumerate(frames):
        before = oo.map_frames
        T, xyz4, ok = oo.frame(k, common.raw4(x, t), a)
        if oo.map_frames != before:  # the oracle inserted this frame: the device map follows
            reg.insert(torch.from_numpy(np.ascontiguousarray(xyz4)).cuda(),
                       torch.from_numpy(a.view(np.int32)).cuda(), T, p.reg_voxel, p.max_range, p.ret_mask)
    assert reg.as_dict() == oo.reg.as_dict()
    e = np.array(errors)
    assert len(e) >= 50
    assert e[:, 0].max() <= 1e-3 and e[:, 1].max() <= 0.01, e[:, :2].max(axis=0)
    assert (np.abs(e[:, 2] - e[:, 3]) <= 1).all()  # the stop test fires at the same iteration, or one apart


@pytest.mark.parametrize("overlap", [False, True])
def test_integration_map_and_carving_at_size_bit_exact(overlap):
    """200 frames inserted and carved (every ray) into a 2^22-slot map, keys, counts, sums and misses equal to the
    oracle's replay of the same frames at the device's poses; with overlap the insert and carve of each frame run on
    the side stream one frame later, and the map must come out the same."""
    from livox_warp import gpu
    from livox_warp.odom import Odometry

    n = 200
    frames, traj = _sequence(n)
    cap = 1 << 22
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=cap)
    odom = Odometry(pipe, reg_slots=1 << 21, frame_cap=1 << 15)
    odom.reg_voxel = 0.15
    view = gpu.make_view(now=0.0, voxel=0.1, map_cap=cap)
    odom.integrate(view, 0.1, carve_every=1, overlap=overlap)
    odom.reset(traj.poses(np.array([0.5 * FRAME_DT]))[0])
    got = []

    def on_frame(k, T, fx, fa, ft, ff, m):
        got.append((k, T.astype(np.float32), fx[:m].cpu().numpy(), fa[:m].cpu().numpy(), ft[:m].cpu().numpy(),
                    ff[:m].cpu().numpy()))

    for x, a, t in frames:
        sx, sa, st, sf = pipe.stage(x, a, t, len(t), 1.0 / FRAME_DT)
        odom.push(sx, sa, st, len(t), float(t.min()), float(t.max()), on_frame)
    odom.flush(on_frame)
    torch.cuda.synchronize()
    assert len(got) == n
    # the oracle: the same deskewed frames, posed by the device's poses, inserted then carved frame by frame
    om = oracle.Map(cap)
    poses = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (oracle.POSE_SLOTS, 1))
    pipe_view = gpu.make_view(now=0.0, voxel=0.1, map_cap=cap)
    for k, T32, fx, fa, ft, ff in got:
        poses[k & (oracle.POSE_SLOTS - 1)] = T32.reshape(16)
        om.insert(fx, fa.view(np.uint32), ft, ff, poses, pipe_view, 0.1)
        om.carve(fx, fa.view(np.uint32), ff, poses, 0.1, every=1)
    keys = pipe.map_keys.cpu().numpy()
    occ = keys != -1
    assert occ.sum() == (om.keys != -1).sum() > 5000
    g = {int(k): (int(c), tuple(s), float(l), float(f), int(m)) for k, c, s, l, f, m in
         zip(keys[occ], pipe.map_cnt.cpu().numpy()[occ], pipe.map_acc.cpu().numpy()[occ],
             pipe.map_last.cpu().numpy()[occ], pipe.map_first.cpu().numpy()[occ], pipe.map_miss.cpu().numpy()[occ])}
    o = om.as_dict()
    assert g == o
    assert sum(x[4] for x in o.values()) > 10000  # carving did work
