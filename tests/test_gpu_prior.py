"""The prior-map builder on the GPU (prior_map.py:57-219) against the oracle: voxel means, colour, intensity and
counts bit for bit and in the same order (first point), whatever the chunking; normals and planarity bit for bit
(fixed-point sums, float64 Jacobi on both sides); and a map built with from_points that a prior grid accepts."""

import numpy as np
import pytest
import torch

from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cloud():
    from livox_warp import synth

    sc = synth.box_room(1)
    xyz = synth.tls_scan(sc, [[2.0, 2.0, 1.5], [5.0, 4.0, 1.2]], seed=0, step_deg=0.5)
    rng = np.random.default_rng(1)
    rgb = rng.integers(0, 256, (len(xyz), 3)).astype(np.float32)
    inten = rng.uniform(0.0, 1.0, len(xyz)).astype(np.float32)
    return sc, xyz, rgb, inten


@pytest.mark.parametrize("chunk", [1 << 25, 50_000])
def test_voxel_downsample_bit_exact(cloud, chunk):
    from livox_warp import prior_map

    _, xyz, rgb, inten = cloud
    assert len(xyz) > 300_000
    gx, gc, gi, gn = prior_map.voxel_downsample(xyz, inten, rgb, 0.02, chunk=chunk, slots_log2=21)
    ox, oc, oi, on = oracle.voxel_downsample(xyz, inten, rgb, 0.02)
    assert len(gx) == len(ox) > 10_000
    assert np.array_equal(gn, on) and np.array_equal(gx, ox)
    assert np.array_equal(gc, oc) and np.array_equal(gi, oi)


def test_voxel_table_device_chunks_and_no_attributes(cloud):
    """Device tensors in uneven chunks through VoxelTable: the same voxels, means and order as one oracle pass."""
    from livox_warp import prior_map

    _, xyz, _, _ = cloud
    table = prior_map.VoxelTable(0.05, slots_log2=20, chunk=1 << 16)
    x = torch.from_numpy(xyz).cuda()
    for a, b in ((0, 1000), (1000, 150_000), (150_000, len(xyz))):
        table.insert(x[a:b])
    gx, gc, gi, gn = table.emit()
    ox, _, _, on = oracle.voxel_downsample(xyz, None, None, 0.05)
    assert np.array_equal(gn.cpu().numpy(), on) and np.array_equal(gx.cpu().numpy(), ox)
    assert not gc.any().item() and not gi.any().item()
    assert table.totals() == (len(ox), 0)
    # a second cloud after clear() starts from nothing
    table.clear()
    table.insert(x[:5000])
    ox2, _, _, on2 = oracle.voxel_downsample(xyz[:5000], None, None, 0.05)
    gx2, _, _, gn2 = table.emit()
    assert np.array_equal(gx2.cpu().numpy(), ox2) and np.array_equal(gn2.cpu().numpy(), on2)


def test_voxel_table_overflow_raises(cloud):
    from livox_warp import prior_map

    _, xyz, _, _ = cloud
    with pytest.raises(RuntimeError, match="voxel table full"):
        prior_map.voxel_downsample(xyz, None, None, 0.02, slots_log2=10)


@pytest.mark.parametrize("voxel,radius", [(0.02, 0.08), (0.05, 0.2)])
def test_normals_bit_exact(cloud, voxel, radius):
    from livox_warp import prior_map

    _, xyz, _, _ = cloud
    vx, _, _, _ = oracle.voxel_downsample(xyz, None, None, voxel)
    gn, gp = prior_map.normals(vx, radius)
    on, op = oracle.normals(vx, radius)
    assert np.array_equal(gn, on) and np.array_equal(gp, op)
    assert (~gn.any(1)).mean() < 0.2 and np.median(gp) > 0.5


def test_from_points_builds_a_prior_grid(cloud):
    """from_points (prior_map.py:358-370) gives the oracle's means, normals and planarity, and the prior grid
    takes its output: the floor's normals are vertical."""
    from livox_warp import prior_map
    from livox_warp.mapgrid import PriorGrid

    sc, xyz, _, _ = cloud
    pm = prior_map.from_points(xyz, voxel=0.02, normal_radius=0.08)
    ox, _, _, on = oracle.voxel_downsample(xyz, None, None, 0.02)
    nrm, pl = oracle.normals(ox, 0.08)
    assert np.array_equal(pm["xyz"], ox) and np.array_equal(pm["count"], on)
    assert np.array_equal(pm["normal"], nrm) and np.array_equal(pm["planarity"], pl)
    floor = (np.abs(pm["xyz"][:, 2] - sc.room_lo[2]) < 0.01) & (pm["planarity"] > 0.5)
    assert floor.sum() > 1000 and np.median(np.abs(pm["normal"][floor, 2])) > 0.99
    grid = PriorGrid(pm)
    assert grid.n == len(ox)


def test_empty_inputs_and_bad_arguments():
    from livox_warp import _lib, prior_map

    gx, gc, gi, gn = prior_map.voxel_downsample(np.zeros((0, 3), np.float32), None, None, 0.05, slots_log2=10)
    assert gx.shape == (0, 3) and gn.shape == (0,)
    nrm, pl = prior_map.normals(np.zeros((0, 3), np.float32), 0.1)
    assert nrm.shape == (0, 3) and pl.shape == (0,)
    x = torch.zeros((16, 3), dtype=torch.float32, device="cuda")
    with pytest.raises(_lib.LwError, match="radius"):
        prior_map.normals_device(x, 0.0)
    with pytest.raises(_lib.LwError, match="radius"):
        prior_map.normals_device(x, 17.0)
    with pytest.raises(ValueError):
        prior_map.normals_device(x[:, :2].contiguous(), 0.1)
    table = prior_map.VoxelTable(0.05, slots_log2=10, chunk=8)
    with pytest.raises(_lib.LwError, match="exceed"):
        _lib.call("lw_vox_insert", table.buf, _lib.ptr(x), 3, None, None, 16, 0, 0.05, _lib.stream_ptr())
    with pytest.raises(_lib.LwError, match="voxel"):
        _lib.call("lw_vox_insert", table.buf, _lib.ptr(x), 3, None, None, 8, 0, 0.0, _lib.stream_ptr())
