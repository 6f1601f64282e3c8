"""Integration map, carving and the map's visible set on the GPU against the CPU oracle: bit exact.

Keys, hit counts, the fixed-point sums, first/last hit times and carving misses are compared as key -> value
maps (slot positions may differ between a parallel and a serial insert under hash collisions; contents may not).
"""

import numpy as np
import pytest
import torch

import common
from oracle import oracle

pytestmark = pytest.mark.gpu

VOXEL = 0.1


def _setup(map_cap=1 << 18):
    from livox_warp import gpu

    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=map_cap)
    om = oracle.Map(map_cap)
    poses = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (oracle.POSE_SLOTS, 1))
    return pipe, om, poses


def _feed(pipe, om, poses, frames, traj, start, view, every=1, carve=True, stride4=False):
    for j, (x, a, t) in enumerate(frames):
        k = start + j
        T = common.mid_pose(traj, k).astype(np.float32)
        pipe.set_pose(k, T)
        poses[k & (oracle.POSE_SLOTS - 1)] = T.reshape(16)
        n = len(t)
        fid = common.frame_ids(t)
        if stride4:
            x4 = common.raw4(x, t)
            sx = torch.from_numpy(x4).cuda()
            sa = torch.from_numpy(a.view(np.int32)).cuda()
            st = torch.from_numpy(t).cuda()
            sf = torch.from_numpy(fid).cuda()
        else:
            sx, sa, st, sf = pipe.stage(x, a, t, n, 10.0)
            assert np.array_equal(sf[:n].cpu().numpy(), fid), "frame ids differ"
        pipe.map_insert(sx, sa, st, sf, n, view, VOXEL)
        om.insert(x if not stride4 else common.raw4(x, t), a, t, fid, poses, view, VOXEL)
        if carve:
            pipe.carve(sx, sa, sf, n, VOXEL, every=every)
            om.carve(x if not stride4 else common.raw4(x, t), a, fid, poses, VOXEL, every=every)


def _gpu_dict(pipe):
    keys = pipe.map_keys.cpu().numpy()
    occ = keys != -1
    cnt, acc = pipe.map_cnt.cpu().numpy()[occ], pipe.map_acc.cpu().numpy()[occ]
    last, first = pipe.map_last.cpu().numpy()[occ], pipe.map_first.cpu().numpy()[occ]
    miss = pipe.map_miss.cpu().numpy()[occ]
    return {int(k): (int(c), tuple(a), float(l), float(f), int(m))
            for k, c, a, l, f, m in zip(keys[occ], cnt, acc, last, first, miss)}


@pytest.mark.parametrize("stride4", [False, True])
def test_map_insert_and_carve_bit_exact(stride4):
    from livox_warp import gpu

    traj = common.handheld()
    frames = common.handheld_frames(16)[10:16]
    pipe, om, poses = _setup()
    view = gpu.make_view(now=1.6, voxel=VOXEL, map_cap=pipe.map_cap)
    _feed(pipe, om, poses, frames, traj, 10, view, every=1, stride4=stride4)
    torch.cuda.synchronize()
    g, o = _gpu_dict(pipe), om.as_dict()
    assert len(g) == len(o) > 300
    assert g == o
    assert np.array_equal(pipe.map_stats.cpu().numpy(), om.stats)
    assert sum(v[4] for v in g.values()) > 0, "no ray pierced anything: the carving test is vacuous"


def test_carve_every_other_ray():
    from livox_warp import gpu

    traj = common.handheld()
    frames = common.handheld_frames(14)[10:14]
    pipe, om, poses = _setup()
    view = gpu.make_view(now=1.4, voxel=VOXEL, map_cap=pipe.map_cap)
    _feed(pipe, om, poses, frames, traj, 10, view, every=2)
    torch.cuda.synchronize()
    assert _gpu_dict(pipe) == om.as_dict()


@pytest.mark.parametrize("voxels", [1, 7])
def test_map_cap_counts_past_4096(voxels):
    """A voxel hit more than 4096 times keeps counting but sums exactly the first 4096 hits in point order. With
    several voxels their hits interleave at random, so one warp meets several voxels crossing the cap at once."""
    from livox_warp import gpu

    pipe, om, poses = _setup(1 << 12)
    rng = np.random.default_rng(5)
    n = 9000 * voxels
    centre = np.array([1.05, 2.05, 0.55]) + 0.1 * np.stack([np.arange(voxels), np.zeros(voxels),
                                                            np.arange(voxels) % 3], 1)
    x = (centre[rng.integers(0, voxels, n)] + rng.uniform(-0.04, 0.04, (n, 3))).astype(np.float32)
    a = rng.integers(0, 256, n).astype(np.uint32)
    t = np.linspace(0.0, 0.09, n).astype(np.float32)
    view = gpu.make_view(now=1.0, voxel=VOXEL, map_cap=pipe.map_cap)
    for half in (slice(0, 3000 * voxels), slice(3000 * voxels, n)):  # the second batch crosses the cap
        xs, as_, ts = x[half], a[half], t[half]
        sx, sa, st, sf = pipe.stage(xs, as_, ts, len(ts), 0.0)
        pipe.map_insert(sx, sa, st, sf, len(ts), view, VOXEL)
        om.insert(xs, as_, ts, np.zeros(len(ts), np.int32), poses, view, VOXEL)
    torch.cuda.synchronize()
    g = _gpu_dict(pipe)
    assert g == om.as_dict()
    assert max(v[0] for v in g.values()) > 4096


def test_map_build_visible_set():
    from livox_warp import gpu

    traj = common.handheld()
    frames = common.handheld_frames(16)[10:16]
    pipe, om, poses = _setup()
    view = gpu.make_view(now=1.6, voxel=VOXEL, map_cap=pipe.map_cap, carve_on=1, carve_ratio=0.5, carve_min=1,
                         carve_stale=0.05, dyn_settle=0.3)
    _feed(pipe, om, poses, frames, traj, 10, view, every=1)
    count = pipe.build(view, map_on=True, min_count=2)
    ox, oa, ot, od = om.build(view, min_count=2)
    assert count == len(ox) > 0
    gx, ga, gt = pipe.export()
    gd = pipe.c_dyn[:count].cpu().numpy()
    # the same set of voxels with the same attributes (order is the slot order of each table)
    g_rows = sorted(zip(map(tuple, gx), ga.tolist(), gt.tolist(), gd.tolist()))
    o_rows = sorted(zip(map(tuple, ox), oa.tolist(), ot.tolist(), od.tolist()))
    assert g_rows == o_rows


def test_map_clear():
    from livox_warp import gpu

    traj = common.handheld()
    frames = common.handheld_frames(12)[10:12]
    pipe, om, poses = _setup()
    view = gpu.make_view(now=1.2, voxel=VOXEL, map_cap=pipe.map_cap)
    _feed(pipe, om, poses, frames, traj, 10, view, carve=False)
    pipe.clear_map()
    torch.cuda.synchronize()
    assert int((pipe.map_keys != -1).sum()) == 0 and int(pipe.map_stats.abs().sum()) == 0
    assert float(pipe.map_first.min()) == float(np.float32(1.0e30))
