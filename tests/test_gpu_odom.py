"""Odometry kernels on the GPU against the CPU oracle.

Bit exact: deskew, thinning (which points survive, in which order), the registration map's keys, counts and
fixed-point sums. Float tolerances, written per test: the per-voxel records (float64 math rounded to float32:
1e-6 relative), one Gauss-Newton accumulation (float32 on the GPU vs float64 in the oracle: 2e-3 relative on
H and b), and the registered pose against the float64 oracle: <= 1 mm and <= 0.01 deg.
"""

import math

import numpy as np
import pytest
import torch

import common
from oracle import oracle

pytestmark = pytest.mark.gpu

RATE = 100000.0


def test_deskew_bit_exact():
    from livox_warp import kernels

    rng = np.random.default_rng(11)
    n = 20000
    raw = np.concatenate([rng.uniform(-20, 20, (n, 3)), rng.uniform(0.0, 0.1, (n, 1))], axis=1).astype(np.float32)
    tw = np.array([0.05, -0.02, 0.01, 0.01, -0.03, 0.035], np.float32)
    g = kernels.deskew(torch.from_numpy(raw).cuda(), 0.05, 10.0, tw).cpu().numpy()
    o = oracle.deskew(raw, 0.05, 10.0, tw)
    assert np.array_equal(g, o)


def test_deskew_zero_twist_is_identity():
    from livox_warp import kernels

    raw = np.random.default_rng(1).uniform(-5, 5, (1000, 4)).astype(np.float32)
    g = kernels.deskew(torch.from_numpy(raw).cuda(), 0.05, 10.0, np.zeros(6, np.float32)).cpu().numpy()
    assert np.array_equal(g, raw)


@pytest.mark.parametrize("voxel", [0.15, 0.2])
def test_thin_bit_exact(voxel):
    from livox_warp import kernels

    x, a, t = common.handheld_frames(12)[11]
    x4 = common.raw4(x, t)
    a = a.copy()
    a[::17] |= np.uint32(1 << 8)   # some noise-tagged returns
    a[::23] |= np.uint32(2 << 16)  # returns outside the mask
    th = kernels.Thinner(1 << 14)
    inv_v = np.float32(2.0 / voxel)
    g = th(torch.from_numpy(x4).cuda(), torch.from_numpy(a.view(np.int32)).cuda(), float(inv_v), 0.3, 60.0,
           0b0011).cpu().numpy()
    o = oracle.thin(x4, a, inv_v, 0.3, 60.0, 0b0011)
    assert len(g) == len(o) > 200
    assert np.array_equal(g, o)
    # the thinning table is clean for the next frame
    assert int((th.ds_keys != -1).sum()) == 0


def _static_map(voxel, n_frames=10, reg_slots=1 << 18, T0=None):
    """The registration map of n static frames at T0, on the GPU and in the oracle."""
    from livox_warp import kernels

    sc = common.room(1)
    T0 = common.config1_pose() if T0 is None else T0
    from livox_warp import synth

    static = synth.ConstantVelocity(T0, 1e9, 0.0, 0.0)
    frames = synth.frames(sc, static, n_frames, RATE, seed=21)
    reg = kernels.RegistrationMap(reg_slots)
    oreg = oracle.RegMap(reg_slots)
    for x, a, t in frames:
        x4 = common.raw4(x, t)
        reg.insert(torch.from_numpy(x4).cuda(), torch.from_numpy(a.view(np.int32)).cuda(), T0, voxel)
        oreg.insert(x4, a, T0, voxel, 60.0, 0b1111)
    oreg.records(voxel, 0.02, 0.05)
    return reg, oreg, T0, sc


@pytest.mark.parametrize("voxel", [0.2, 0.1])
def test_registration_map_bit_exact(voxel):
    reg, oreg, _, _ = _static_map(voxel)
    g, o = reg.as_dict(), oreg.as_dict()
    assert len(g) == len(o) > 1000
    assert g == o
    assert np.array_equal(reg.stats.cpu().numpy(), oreg.stats)
    # records: float64 math rounded to float32 on both sides (tolerance 1e-6 relative, 1e-6 absolute)
    keys = reg.keys.cpu().numpy()
    rec = reg.rec.cpu().numpy()
    orec = {int(k): r for k, r in zip(oreg.keys, oreg.rec) if k != -1}
    got = np.stack([rec[s] for s in np.nonzero(keys != -1)[0]])
    want = np.stack([orec[int(k)] for k in keys[keys != -1]])
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("voxels", [1, 7])
def test_registration_cap_exact_first_points(voxels):
    """More than 4096 points in a voxel: exactly the first 4096 in point order are summed. With several voxels
    their points interleave at random, so one warp meets several voxels crossing the cap in the same batch."""
    from livox_warp import kernels

    rng = np.random.default_rng(3)
    n = 10000 * voxels
    x4 = np.zeros((n, 4), np.float32)
    centre = np.array([1.02, 1.03, 1.04]) + 0.2 * np.stack([np.arange(voxels), np.arange(voxels) % 2,
                                                            np.zeros(voxels)], 1)
    x4[:, :3] = centre[rng.integers(0, voxels, n)] + rng.uniform(-0.015, 0.015, (n, 3))
    a = np.zeros(n, np.uint32)
    reg = kernels.RegistrationMap(1 << 10)
    oreg = oracle.RegMap(1 << 10)
    for part in (slice(0, 2500 * voxels), slice(2500 * voxels, n)):
        reg.insert(torch.from_numpy(x4[part].copy()).cuda(), torch.from_numpy(a[part].view(np.int32)).cuda(),
                   np.eye(4), 0.2)
        oreg.insert(x4[part], a[part], np.eye(4), 0.2, 60.0, 0b1111)
    assert reg.as_dict() == oreg.as_dict()
    assert sorted(c for c, _, _ in reg.as_dict().values())[-voxels:] == [4096] * voxels


def _test_frame(voxel):
    """The config-1 registration input: a frame taken while moving, thinned, with its start pose."""
    from livox_warp import synth

    sc = common.room(1)
    T0 = common.config1_pose()
    reg, oreg, _, _ = _static_map(voxel, T0=T0)
    # 0.5 m/s forward and 20 deg/s yaw, starting as the static frames end
    mover = synth.ConstantVelocity(T0, 1.0, 0.5, math.radians(20.0))
    x, a, t = synth.scan(sc, mover, 1.0, 1.1, RATE, seed=99)
    x4 = common.raw4(x, t)
    ds = oracle.thin(x4, a, np.float32(2.0 / voxel), 0.3, 60.0, 0b1111)
    T_true = mover.poses(np.array([1.05]))[0]
    return reg, oreg, ds, T0, T_true


def test_icp_accumulate_vs_float64():
    from livox_warp import kernels

    voxel = 0.2
    reg, oreg, ds, T0, _ = _test_frame(voxel)
    gn = kernels.GnScratch()
    for it in (0, 5):
        reach, max_d2, kappa = oracle.schedule(it, voxel)
        g = kernels.icp_accumulate(torch.from_numpy(ds).cuda(), T0, reg, voxel, reach, max_d2, kappa, gn)
        o = oracle.icp_accumulate(ds, T0, oreg, voxel, reach, max_d2, kappa)
        assert abs(g[oracle.ACC_COUNT] - o[oracle.ACC_COUNT]) <= 0.005 * o[oracle.ACC_COUNT]
        H, Ho = oracle.sym6(g[:21]), oracle.sym6(o[:21])
        assert np.linalg.norm(H - Ho) <= 2e-3 * np.linalg.norm(Ho)
        b, bo = g[21:27], o[21:27]
        assert np.linalg.norm(b - bo) <= 2e-3 * np.linalg.norm(bo) + 1e-3 * np.sqrt(np.linalg.norm(Ho))


def test_register_matches_float64_oracle():
    """Config 1: a 10k-point frame registered against a 0.2 m map of 10 static frames, 10 iterations:
    the device solve lands within 1 mm / 0.01 deg of the float64 oracle from the same start."""
    from livox_warp import kernels, _lib

    voxel = 0.2
    reg, oreg, ds, T0, T_true = _test_frame(voxel)
    p = oracle.Params(reg_voxel=voxel, max_iter=10)
    To, ok_o, so = oracle.register(ds, T0, oreg, p)
    prm = _lib.OdomParams()
    for name in ("frame_dt", "reg_voxel", "min_range", "max_range", "noise", "alpha", "damping", "velocity_smooth",
                 "degen_thr", "prior_info", "kf_dist", "max_iter", "warmup", "min_points", "min_corr", "ret_mask"):
        setattr(prm, name, getattr(p, name))
    prm.kf_angle_deg, prm.deskew, prm.redeskew, prm.frame_cap = p.kf_angle, 1, 1, 1 << 14
    gn = kernels.GnScratch()
    Tg, ok_g, sg = kernels.icp_solve(torch.from_numpy(ds).cuda(), T0, reg, prm, gn)
    assert ok_g and ok_o
    dt, dr = oracle.pose_error(To, Tg)
    assert dt <= 1e-3 and dr <= 0.01, (dt, dr, sg, so)
    et, er = oracle.pose_error(T_true, Tg)
    assert et < 0.05 and er < 1.0, (et, er)  # and the registration moved toward the truth (frame not deskewed)
    assert sg["iters"] >= 1 and sg["corr"] > 500


@pytest.mark.parametrize("yaw_deg", [0.0, 1.0])
def test_register_degenerate_corridor_matches_oracle(yaw_deg):
    """A frame from the middle of a 200 m corridor (two walls, floor and ceiling; both ends beyond range):
    sliding along the corridor is unconstrained. With the threshold at 20000 the two weakest directions of the
    surface-normal information (~3.3e3 and ~1.3e4 here; the next is ~2.5e4) fall below it, so every iteration
    takes the degenerate branch (odom.py:436-455): the eigen-decomposition and the step with the weak directions
    held at the prediction. The device solve agrees with the float64 oracle within 1 mm / 0.01 deg, holds the
    same number of directions, and keeps the corridor direction at the prediction. With the prediction also
    turned 1 deg off, the sensor basis the held directions live in (at the current pose, which moves away from the
    prediction over the iterations) must follow the pose as the oracle's does."""
    from livox_warp import kernels, _lib, synth

    voxel = 0.2
    sc = synth.Scene(np.zeros(3), np.array([200.0, 2.4, 2.8]), np.zeros((0, 6)))
    T0 = common.look_at([100.0, 1.2, 1.4], [110.0, 1.6, 1.2])  # looks down the corridor
    static = synth.ConstantVelocity(T0, 1e9, 0.0, 0.0)
    reg = kernels.RegistrationMap(1 << 18)
    oreg = oracle.RegMap(1 << 18)
    for x, a, t in synth.frames(sc, static, 6, RATE, seed=31, noise=0.002):
        x4 = common.raw4(x, t)
        reg.insert(torch.from_numpy(x4).cuda(), torch.from_numpy(a.view(np.int32)).cuda(), T0, voxel)
        oreg.insert(x4, a, T0, voxel, 60.0, 0b1111)
    oreg.records(voxel, 0.02, 0.05)
    x, a, t = synth.scan(sc, static, 0.6, 0.7, RATE, seed=77, noise=0.002)
    ds = oracle.thin(common.raw4(x, t), a, np.float32(2.0 / voxel), 0.3, 60.0, 0b1111)
    Tp = T0.copy()
    Tp[:3, 3] += [0.05, 0.02, -0.01]  # off in every direction, the corridor's one included
    th = np.radians(yaw_deg)
    Tp[:3, :3] = np.array([[np.cos(th), -np.sin(th), 0.0], [np.sin(th), np.cos(th), 0.0], [0.0, 0.0, 1.0]]) @ Tp[:3, :3]
    p = oracle.Params(reg_voxel=voxel, max_iter=10, degen_thr=20000.0)
    To, ok_o, so = oracle.register(ds, Tp, oreg, p)
    prm = _lib.OdomParams()
    for name in ("frame_dt", "reg_voxel", "min_range", "max_range", "noise", "alpha", "damping", "velocity_smooth",
                 "degen_thr", "prior_info", "kf_dist", "max_iter", "warmup", "min_points", "min_corr", "ret_mask"):
        setattr(prm, name, getattr(p, name))
    prm.kf_angle_deg, prm.deskew, prm.redeskew, prm.frame_cap = p.kf_angle, 1, 1, 1 << 14
    Tg, ok_g, sg = kernels.icp_solve(torch.from_numpy(ds).cuda(), Tp, reg, prm, kernels.GnScratch())
    assert ok_g and ok_o
    assert so["degen"] == 2 and sg["degen"] == so["degen"], (sg, so)
    dt, dr = oracle.pose_error(To, Tg)
    assert dt <= 1e-3 and dr <= 0.01, (dt, dr, sg, so)
    if yaw_deg:
        return  # ten iterations do not bring the turned start home along the weak directions
    assert abs(Tg[0, 3] - Tp[0, 3]) < 0.002  # the corridor direction stays at the prediction
    assert abs(Tg[1, 3] - T0[1, 3]) < 0.01 and abs(Tg[2, 3] - T0[2, 3]) < 0.01  # the constrained ones converge
    assert abs(sg["cond"] - so["cond"]) <= 1e-6 + 0.05 * abs(so["cond"])  # float32 sums of H: ~1e-3 relative


@pytest.mark.parametrize("rate", [1.5e6, 0.0])
def test_register_frame_deskews_and_thins_like_the_oracle(rate):
    """The registration launch deskews and thins the frame itself: a 150k-point frame (several points per thread
    of every CTA) with a turning twist leaves f_xyz and ds_xyz bit-exact with the oracle's deskew and thinning,
    the table empty for the next frame (a second, different frame thins exactly too), and an empty frame leaves
    no registration."""
    from livox_warp import gpu, synth
    from livox_warp.odom import Odometry

    voxel = 0.2
    T0, base, moving = synth.single_frame_case(common.room(1), 2, max(rate, RATE), map_frames=3)
    pipe = gpu.Pipeline(ring_capacity=1 << 14, map_capacity=1 << 14)
    odom = Odometry(pipe, reg_slots=1 << 18, frame_cap=1 << 18)
    odom.reg_voxel, odom.max_iter = voxel, 10
    odom.reset(T0)
    oreg = oracle.RegMap(1 << 18)
    for x, a, t in base:
        x4 = common.raw4(x, t)
        oreg.insert(x4, a, T0, voxel, 60.0, 0b1111)
        odom.insert_frame(torch.from_numpy(x4).cuda(), torch.from_numpy(a.view(np.int32)).cuda(), T0)
    tw = np.array([0.05, -0.02, 0.0, 0.0, 0.01, np.radians(2.0)], np.float32)
    if rate == 0.0:
        e = np.zeros((0, 3), np.float32)
        Tg, ok, st = odom.register_frame(e, np.zeros(0, np.uint32), np.zeros(0, np.float32), 1.0, tw, T0)
        assert not ok and st["ds"] == 0 and st["err"] == 0
        assert np.array_equal(Tg, T0)
        return
    for x, a, t, t_mid, _ in moving:
        assert len(t) > 148 * 256 * 3
        x4 = common.raw4(x, t)
        d_o = oracle.deskew(x4, t_mid, 10.0, tw)
        ds = oracle.thin(d_o, a, np.float32(2.0 / voxel), 0.3, 60.0, 0b1111)
        _, _, st = odom.register_frame(x, a, t, t_mid, tw, T0)
        assert st["err"] == 0 and st["ds"] == len(ds)
        assert np.array_equal(odom.f_xyz[:len(t)].cpu().numpy(), d_o)
        assert np.array_equal(odom.ds_xyz[:len(ds)].cpu().numpy(), ds)
    assert bool((odom.ds_keys == -1).all()) and bool((odom._ds_win == np.iinfo(np.int32).max).all())


def test_register_frame_host_frames_queued_without_sync():
    """Host frames queued back to back (sync=False) register as they do one at a time: each call waits until the
    previous launch has read the pinned frame before refilling it, and registration() returns the last frame's
    result from the pinned result buffer."""
    from livox_warp import gpu, synth
    from livox_warp.odom import Odometry

    T0, base, moving = synth.single_frame_case(common.room(1), 3, RATE, map_frames=3)
    pipe = gpu.Pipeline(ring_capacity=1 << 14, map_capacity=1 << 14)
    odom = Odometry(pipe, reg_slots=1 << 18, frame_cap=1 << 15)
    odom.reg_voxel, odom.max_iter = 0.2, 10
    odom.reset(T0)
    for x, a, t in base:
        odom.insert_frame(torch.from_numpy(common.raw4(x, t)).cuda(), torch.from_numpy(a.view(np.int32)).cuda(), T0)
    zero = np.zeros(6, np.float32)
    one_by_one = [odom.register_frame(x, a, t, t_mid, zero, T0) for x, a, t, t_mid, _ in moving]
    for j in range(len(moving)):
        for x, a, t, t_mid, _ in moving[:j + 1]:
            assert odom.register_frame(x, a, t, t_mid, zero, T0, sync=False) is None
        T, ok, st = odom.registration()
        Tj, okj, stj = one_by_one[j]
        assert ok == okj and np.array_equal(T, Tj) and st == stj


def test_register_frame_host_refuses_memory_that_is_not_pinned():
    """lw_register_frame_host reads the frame and writes its result through device pointers of pinned host memory;
    pageable memory is refused before anything is launched, and the next call with pinned buffers registers."""
    import ctypes

    from livox_warp import _lib, gpu, synth
    from livox_warp.odom import Odometry

    T0, base, moving = synth.single_frame_case(common.room(1), 1, RATE, map_frames=2)
    pipe = gpu.Pipeline(ring_capacity=1 << 14, map_capacity=1 << 14)
    odom = Odometry(pipe, reg_slots=1 << 18, frame_cap=1 << 15)
    odom.reg_voxel, odom.max_iter = 0.2, 10
    odom.reset(T0)
    for x, a, t in base:
        odom.insert_frame(torch.from_numpy(common.raw4(x, t)).cuda(), torch.from_numpy(a.view(np.int32)).cuda(), T0)
    x, a, t, t_mid, _ = moving[0]
    m = len(t)
    x3 = np.ascontiguousarray(x[:, :3], np.float32)
    tt = np.ascontiguousarray(t, np.float32)
    aa = np.ascontiguousarray(a, np.uint32)
    out = np.zeros(ctypes.sizeof(_lib.OdomState), np.uint8)
    err = np.zeros(1, np.int32)
    vp = lambda arr: ctypes.c_void_p(arr.ctypes.data)  # noqa: E731
    with pytest.raises(_lib.LwError, match="not pinned"):
        _lib.call("lw_register_frame_host", vp(x3), vp(tt), vp(aa), m, float(t_mid),
                  _lib.f32_array(np.zeros(6, np.float32)), _lib.f64_array(T0.reshape(16)),
                  ctypes.byref(odom.params()), _lib.ptr(odom._state), ctypes.byref(odom.fbuf),
                  ctypes.byref(odom.regmap), ctypes.byref(odom.gn), vp(out), vp(err), odom._sp())
    torch.cuda.synchronize()
    _, ok, st = odom.register_frame(x, a, t, t_mid, np.zeros(6, np.float32), T0)
    assert ok and st["err"] == 0 and st["ds"] > 0


def test_register_frame_single_case_matches_float64_oracle():
    """The single-frame case through Odometry.register_frame (deskew + thinning + Gauss-Newton in one call, from
    host arrays and from device tensors): every one of its 8 seeded frames lands within 1 mm / 0.01 deg of the
    float64 oracle registering the same thinned frame from the same start, and within 3 cm / 1 deg of the truth."""
    from livox_warp import gpu, synth
    from livox_warp.odom import Odometry

    voxel = 0.2
    T0, base, moving = synth.single_frame_case(common.room(1), 8, RATE)
    oreg = oracle.RegMap(1 << 18)
    pipe = gpu.Pipeline(ring_capacity=1 << 14, map_capacity=1 << 14)
    odom = Odometry(pipe, reg_slots=1 << 18, frame_cap=1 << 15)
    odom.reg_voxel, odom.max_iter = voxel, 10
    odom.reset(T0)
    for x, a, t in base:
        x4 = common.raw4(x, t)
        oreg.insert(x4, a, T0, voxel, 60.0, 0b1111)
        odom.insert_frame(torch.from_numpy(x4).cuda(), torch.from_numpy(a.view(np.int32)).cuda(), T0)
    oreg.records(voxel, 0.02, 0.05)
    g, o = odom.reg.as_dict(), oreg.as_dict()
    assert g == o
    p = oracle.Params(reg_voxel=voxel, max_iter=10)
    zero = np.zeros(6, np.float32)
    for j, (x, a, t, t_mid, T_true) in enumerate(moving):
        x4 = common.raw4(x, t)
        ds = oracle.thin(oracle.deskew(x4, t_mid, 10.0, zero), a, np.float32(2.0 / voxel), 0.3, 60.0, 0b1111)
        To, ok_o, so = oracle.register(ds, T0, oreg, p)
        if j % 2:
            Tg, ok_g, sg = odom.register_frame(x, a, t, t_mid, zero, T0)
        else:
            Tg, ok_g, sg = odom.register_frame(torch.from_numpy(x4).cuda(), torch.from_numpy(a.view(np.int32)).cuda(),
                                               None, t_mid, zero, T0)
        assert ok_g and ok_o
        assert sg["ds"] == len(ds) and sg["iters"] == so["iters"], (sg, so)
        assert np.array_equal(odom.ds_xyz[:len(ds)].cpu().numpy(), ds)
        dt, dr = oracle.pose_error(To, Tg)
        assert dt <= 1e-3 and dr <= 0.01, (j, dt, dr)
        et, er = oracle.pose_error(T_true, Tg)
        assert et < 0.03 and er < 1.0, (j, et, er)
