"""The live ring's visible set (k_classify_live, gpu.py:637-697) in the oracle against a numpy restatement of the
reference kernel: which ring slots are drawn (age, keep_raw, the pose slot's owner frame and epoch, the crop box),
in ring order, their deskewed and posed world points (Rodrigues' rotation in float64 here, the oracle's quaternion
form there: within 2e-6 m), attributes, times, and the Motion label against an empty map (nothing settled); and
the reference's live-window gate of smoke_pipeline.py:43-50."""

import numpy as np

from oracle import oracle


def _view(**kw):
    from livox_warp import gpu

    return gpu.make_view(**kw)


def _reference_live(ring_xyz, ring_attr, ring_t, ring_frame, filled, poses, tw, own_f, own_e, v):
    out = []
    for i in range(filled):
        t = np.float32(ring_t[i])
        if v.persist > 0 and np.float32(v.now) - t > np.float32(v.persist):
            continue
        p = ring_xyz[i].astype(np.float32)
        a = int(ring_attr[i])
        r = np.sqrt(np.float32(p[0] * p[0] + p[1] * p[1]) + np.float32(p[2] * p[2]))
        if r < np.float32(v.min_range) or r > np.float32(v.max_range):
            continue
        if (a & 255) < v.min_refl or not (v.noise_mask >> ((a >> 8) & 3)) & 1 or not (v.ret_mask >> ((a >> 16) & 3)) & 1:
            continue
        fid = int(ring_frame[i])
        f = fid & (oracle.POSE_SLOTS - 1)
        if v.inv_frame_dt > 0:
            if own_f[f] != fid or own_e[f] != v.epoch:
                continue
            x = t * np.float32(v.inv_frame_dt)
            s = np.float32(np.float32(x - np.floor(x)) - np.float32(0.5))
            rho, theta = tw[f, :3].astype(np.float32), tw[f, 3:].astype(np.float32)
            rv = (theta * s).astype(np.float64)
            ang = np.linalg.norm(rv)
            q = p.astype(np.float64)
            if ang >= 1e-9:
                k = rv / ang
                q = q * np.cos(ang) + np.cross(k, q) * np.sin(ang) + k * np.dot(k, q) * (1 - np.cos(ang))
            p = (q.astype(np.float32) + rho * s).astype(np.float32)
        T = poses[f].reshape(4, 4).astype(np.float64)
        w = (T[:3, :3] @ p.astype(np.float64) + T[:3, 3]).astype(np.float32)
        if v.crop_on and (np.any(w < np.array(v.crop_lo, np.float32)) or np.any(w > np.array(v.crop_hi, np.float32))):
            continue
        out.append((i, w, a, t))
    return out


def test_live_build_matches_reference_kernel():
    rng = np.random.default_rng(4)
    cap, filled = 4096, 3500
    ring_xyz = rng.uniform(-12, 12, (cap, 3)).astype(np.float32)
    ring_attr = (rng.integers(0, 256, cap) | (rng.integers(0, 3, cap) << 8) | (rng.integers(0, 2, cap) << 16))
    ring_attr = ring_attr.astype(np.uint32)
    ring_t = rng.uniform(0.0, 2.0, cap).astype(np.float32)
    ring_frame = np.floor(ring_t * 10).astype(np.int32)
    S = oracle.POSE_SLOTS
    poses = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (S, 1))
    tw = np.zeros((S, 6), np.float32)
    own_f = np.full(S, -1, np.int32)
    own_e = np.full(S, -1, np.int32)
    for k in range(20):
        a = 0.1 * k
        T = np.eye(4, dtype=np.float32)
        T[:3, :3] = [[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]]
        T[:3, 3] = [0.3 * k, -0.1 * k, 0.05 * k]
        poses[k] = T.reshape(16)
        tw[k] = [0.05, -0.02, 0.01, 0.02, -0.03, 0.3]
        own_f[k] = k
        own_e[k] = 1 if k != 7 else 0  # frame 7's slot holds an old epoch: its points are not drawn
    om = oracle.Map(1 << 12)
    for odo in (0.0, 10.0):
        v = _view(now=2.0, persist=1.5, min_refl=20, noise_mask=0b011, ret_mask=0b01, crop_on=1,
                  crop_lo=(-20.0, -20.0, -6.0), crop_hi=(20.0, 20.0, 6.0), inv_frame_dt=odo, epoch=1, dyn_on=1,
                  voxel=0.1, map_cap=1 << 12, dyn_settle=0.5)
        ox, oa, ot, od = om.live_build(ring_xyz, ring_attr, ring_t, ring_frame, filled, poses, tw, own_f, own_e, v)
        want = _reference_live(ring_xyz, ring_attr, ring_t, ring_frame, filled, poses, tw, own_f, own_e, v)
        assert 100 < len(want) < filled and len(ox) == len(want)
        assert np.array_equal(oa, np.array([w[2] for w in want], np.uint32))
        assert np.array_equal(ot, np.array([w[3] for w in want], np.float32))
        assert np.abs(ox - np.array([w[1] for w in want])).max() <= 2e-6
        assert od.all()  # an empty map: nothing is settled, every drawn point is Motion
    # epoch 0 draws only frame 7 (with odometry on)
    v.epoch = 0
    ox, _, ot, _ = om.live_build(ring_xyz, ring_attr, ring_t, ring_frame, filled, poses, tw, own_f, own_e, v)
    assert len(ox) > 0 and np.all(np.floor(ot * 10) == 7)


def test_live_build_empty_ring():
    om = oracle.Map(1 << 10)
    z = np.zeros((16, 3), np.float32)
    v = _view(now=1.0, voxel=0.1, map_cap=1 << 10)
    S = oracle.POSE_SLOTS
    ox, oa, ot, od = om.live_build(z, np.zeros(16, np.uint32), np.zeros(16, np.float32), np.zeros(16, np.int32), 0,
                                   np.zeros((S, 16), np.float32), np.zeros((S, 6), np.float32), np.zeros(S, np.int32),
                                   np.zeros(S, np.int32), v)
    assert len(ox) == 0


def test_pose_entry_moves_the_live_window():
    """smoke_pipeline.py:43-50: the live set of a static scan with frame 0's pose at identity, then at a yaw of 90
    degrees and a (1, 2, 0) m offset (gpu.mount_matrix): the centroid moves as that pose says, within 5 cm."""
    from livox_warp import gpu, synth

    sc = synth.box_room(1)
    T = np.eye(4)
    T[:3, 3] = [4.0, 3.0, 1.5]
    x = synth.spin_scan(sc, T, 40000, 2)
    n = len(x)
    a = np.full(n, 100, np.uint32)
    t = np.linspace(0.0, 0.4, n).astype(np.float32)
    S = oracle.POSE_SLOTS
    tw = np.zeros((S, 6), np.float32)
    own = np.zeros(S, np.int32)
    om = oracle.Map(1 << 10)
    v = _view(now=0.4, persist=0.5, voxel=0.03, map_cap=1 << 10)
    cents = []
    for M in (np.eye(4, dtype=np.float32), gpu.mount_matrix(0, 0, 90, 1.0, 2.0, 0.0)):
        poses = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (S, 1))
        poses[0] = np.asarray(M, np.float32).reshape(16)
        lx, _, _, _ = om.live_build(x, a, t, np.zeros(n, np.int32), n, poses, tw, own, own, v)
        assert len(lx) > 0.9 * n
        cents.append(lx.astype(np.float64).mean(0))
    c0, c = cents
    assert abs((c[0] - 1.0) + c0[1]) < 0.05 and abs((c[1] - 2.0) - c0[0]) < 0.05


def test_visible_set_sample_and_clock_rebase():
    """The strided sample behind Pipeline.bounds / floor_z (gpu.py:1575-1609) and the clock rebase of the map's
    hit times (k_rebase_clock, gpu.py:330-337), on CPU tensors."""
    import torch

    from livox_warp.gpu import rebase_times, strided_sample

    x = torch.arange(300000, dtype=torch.float32).reshape(-1, 3)  # 100000 rows
    s = strided_sample(x, 100000, 1 << 16)
    assert len(s) == 1 << 16 and torch.equal(s[1], x[1])  # stride 1 (100000 // 65536), first 65536 rows
    s = strided_sample(x, 100000, 1000)
    assert len(s) == 1000 and torch.equal(s[3], x[300])
    s = strided_sample(x, 7, 1 << 16)
    assert len(s) == 7
    keys = torch.tensor([5, -1, 9], dtype=torch.int64)
    first = torch.tensor([10.5, 1.0e30, 3.25], dtype=torch.float32)
    last = torch.tensor([12.0, 0.0, 4.0], dtype=torch.float32)
    rebase_times(keys, first, last, 3.0)
    assert first[0].item() == 7.5 and first[2].item() == 0.25 and first[1].item() > 1e29  # empty slot untouched
    assert last.tolist() == [9.0, 0.0, 1.0]
