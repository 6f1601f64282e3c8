"""The prior-map builder's oracle (prior_map.py:57-219) against a plain numpy restatement of the reference's
definitions: per-voxel means of position, colour and intensity with exact counts (k_vox_insert / k_vox_emit), and a
PCA normal and planarity from every point within the radius (k_normals). The reference ships no fixtures for
these kernels (its prior-map checks need a real scan), so the numpy restatement is the pin: float64 means and
numpy's symmetric eigensolver, the neighbour test in float32 as the kernel writes it."""

import numpy as np
import pytest
from scipy.spatial import cKDTree

from oracle import oracle


@pytest.fixture(scope="module")
def cloud():
    from livox_warp import synth

    sc = synth.box_room(1)
    xyz = synth.tls_scan(sc, [[2.0, 2.0, 1.5], [5.0, 4.0, 1.2]], seed=0, step_deg=1.0)
    rng = np.random.default_rng(1)
    rgb = rng.integers(0, 256, (len(xyz), 3)).astype(np.float32)
    inten = rng.uniform(0.0, 1.0, len(xyz)).astype(np.float32)
    return xyz, rgb, inten


def _voxels_numpy(xyz, voxel, *attrs):
    """Voxel index floor(p * float32(1 / voxel)) in float32, voxels in the order of their first point, float64
    means of every attribute."""
    inv = np.float32(1.0 / np.float64(np.float32(voxel)))
    ijk = np.floor(xyz * inv).astype(np.int64)
    _, first, inverse = np.unique(ijk, axis=0, return_index=True, return_inverse=True)
    inverse = inverse.reshape(-1)
    rank = np.empty(len(first), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(first))
    vid = rank[inverse]
    m = len(first)
    means = []
    for a in (xyz,) + attrs:
        a = np.asarray(a, np.float64).reshape(len(xyz), -1)
        s = np.zeros((m, a.shape[1]))
        np.add.at(s, vid, a)
        means.append(s / np.bincount(vid, minlength=m)[:, None])
    return means, np.bincount(vid, minlength=m)


def test_voxel_means_match_numpy(cloud):
    xyz, rgb, inten = cloud
    ox, oc, oi, on = oracle.voxel_downsample(xyz, inten, rgb, 0.05)
    (mx, mc, mi), mn = _voxels_numpy(xyz, 0.05, rgb, inten)
    assert len(ox) == len(mx) and 0 < len(ox) < len(xyz)
    assert np.array_equal(on, mn) and on.sum() == len(xyz)
    # one float32 rounding of the mean (coordinates below 8 m: half an ulp is 4.8e-7) plus the 2^-35 m sums
    assert np.abs(ox - mx).max() <= 1e-6
    # colour and intensity in 2^-16 units: each term rounds by at most 2^-17
    assert np.abs(oc - mc).max() <= 2e-5 and np.abs(oi - mi[:, 0]).max() <= 2e-5


def test_voxel_means_without_attributes(cloud):
    xyz, _, _ = cloud
    ox, oc, oi, on = oracle.voxel_downsample(xyz, None, None, 0.02)
    (mx,), mn = _voxels_numpy(xyz, 0.02)
    assert np.array_equal(on, mn) and np.abs(ox - mx).max() <= 1e-6
    assert not oc.any() and not oi.any()


def test_voxel_edge_cases():
    ox, oc, oi, on = oracle.voxel_downsample(np.zeros((0, 3), np.float32), None, None, 0.05)
    assert len(ox) == 0 and len(on) == 0
    # negative coordinates floor downwards; a point on a voxel face belongs to the voxel above it
    p = np.array([[-0.01, -0.01, -0.01], [-0.04, -0.02, -0.03], [0.0, 0.0, 0.0], [0.05, 0.0, 0.0]], np.float32)
    ox, _, _, on = oracle.voxel_downsample(p, None, None, 0.05)
    assert on.tolist() == [2, 1, 1]
    assert np.allclose(ox[0], p[:2].astype(np.float64).mean(0), atol=1e-7)


def _normals_numpy(xyz, radius):
    """k_normals (prior_map.py:126-166): neighbours by the float32 test ((dx*dx + dy*dy) + dz*dz) <= r*r, covariance
    in float64, eigenvalues ascending (lo = 0, mid = 1, hi = 2)."""
    r2 = np.float32(radius) * np.float32(radius)
    tree = cKDTree(xyz.astype(np.float64))
    nrm = np.zeros((len(xyz), 3))
    pl = np.zeros(len(xyz))
    for i, cand in enumerate(tree.query_ball_point(xyz.astype(np.float64), float(radius) * 1.001)):
        d = xyz[np.asarray(cand)] - xyz[i]
        dd = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        d = d[dd <= r2].astype(np.float64)
        if len(d) < 4:
            continue
        mu = d.mean(0)
        w, V = np.linalg.eigh(d.T @ d / len(d) - np.outer(mu, mu))
        nrm[i] = V[:, 0] / np.linalg.norm(V[:, 0])
        pl[i] = (w[1] - w[0]) / max(w[2], 1e-12)
    return nrm, pl


@pytest.mark.parametrize("voxel,radius", [(0.03, 0.1), (0.05, 0.2)])
def test_normals_match_numpy(cloud, voxel, radius):
    xyz, _, _ = cloud
    vx, _, _, _ = oracle.voxel_downsample(xyz, None, None, voxel)
    on, op = oracle.normals(vx, radius)
    nn, npl = _normals_numpy(vx, radius)
    zero = ~nn.any(1)
    assert np.array_equal(~on.any(1), zero) and not op[zero].any()
    assert zero.mean() < 0.2
    assert np.abs(op - npl).max() <= 1e-4
    well = ~zero & (npl > 1e-2)  # the smallest eigenvalue is separated: its vector is defined
    assert well.mean() > 0.5
    cos = np.abs((on[well].astype(np.float64) * nn[well]).sum(1))
    assert cos.min() >= 1 - 1e-5
    assert np.allclose(np.linalg.norm(on[~zero], axis=1), 1.0, atol=1e-6)


def test_normals_of_flat_faces():
    """Voxel means of a room's faces: the floor's normals are vertical and its patches planar (above the 0.5 a
    prior grid trusts a normal at; a disc of grid-aligned means is not perfectly round, so l_mid / l_max < 1)."""
    from livox_warp import synth

    sc = synth.box_room(2, n_boxes=0)
    xyz, _ = synth.sample_surfaces(sc, 0.01, 0, jitter=0.001)
    vx, _, _, _ = oracle.voxel_downsample(xyz, None, None, 0.02)
    nrm, pl = oracle.normals(vx, 0.08)
    floor = np.abs(vx[:, 2] - sc.room_lo[2]) < 0.01
    inner = floor & np.all((vx[:, :2] > sc.room_lo[:2] + 0.2) & (vx[:, :2] < sc.room_hi[:2] - 0.2), axis=1)
    assert inner.sum() > 1000
    assert np.abs(nrm[inner, 2]).min() > 0.999 and pl[inner].min() > 0.5 and np.median(pl[inner]) > 0.9


def test_normals_edge_cases():
    nrm, pl = oracle.normals(np.zeros((0, 3), np.float32), 0.1)
    assert nrm.shape == (0, 3) and pl.shape == (0,)
    # three points: fewer than 4 neighbours, zero normal and planarity
    p = np.array([[0, 0, 0], [0.01, 0, 0], [0, 0.01, 0]], np.float32)
    nrm, pl = oracle.normals(p, 0.1)
    assert not nrm.any() and not pl.any()


def test_offset_units_and_arguments_checked_before_cuda():
    """lw_vox_offset_units is host arithmetic; the prior-map and live-ring entry points reject bad arguments before
    any CUDA call, so these run without a GPU."""
    import ctypes

    from livox_warp import _lib

    lib = _lib.load(require_cuda=False)
    # 2^(30 - e) with voxel < 2^e: offsets below half a voxel stay below 2^29 units
    for voxel, e in ((0.02, -5), (0.03125, -4), (0.05, -4), (1.0, 1), (3.0, 2)):
        assert lib.lw_vox_offset_units(voxel) == 2.0 ** (30 - e)
        assert np.float32(voxel) < 2.0 ** e and 0.5 * voxel * 2.0 ** (30 - e) <= 2 ** 29
    fake = ctypes.c_void_p(16)  # never dereferenced: the checks fail first
    vb = _lib.VoxBuf(*([fake] * len(_lib.VoxBuf.PTRS)), 1000, 8)  # not a power of two
    assert lib.lw_vox_insert(vb, fake, 3, None, None, 4, 0, 0.05, None) == _lib.LW_EINVAL
    assert b"power of two" in lib.lw_last_error()
    vb.cap = 1024
    assert lib.lw_vox_insert(vb, fake, 3, None, None, 16, 0, 0.05, None) == _lib.LW_ECAPACITY
    assert lib.lw_vox_insert(vb, fake, 5, None, None, 4, 0, 0.05, None) == _lib.LW_EINVAL
    assert lib.lw_vox_insert(vb, fake, 3, None, None, 4, -1, 0.05, None) == _lib.LW_EINVAL
    assert lib.lw_vox_insert(vb, fake, 3, None, None, 4, 0, 1e-9, None) == _lib.LW_EINVAL
    assert lib.lw_vox_emit(vb, 0.0, 4, None, None, None, None, None) == _lib.LW_EINVAL
    pb = _lib.PcaBuf(*([fake] * len(_lib.PcaBuf.PTRS)), 1024, 512)
    assert lib.lw_normals(fake, 3, 16, 0.0, pb, fake, fake, None) == _lib.LW_EINVAL
    assert b"radius" in lib.lw_last_error()
    assert lib.lw_normals(fake, 3, 16, 17.0, pb, fake, fake, None) == _lib.LW_EINVAL
    assert lib.lw_normals(fake, 3, 600, 0.1, pb, fake, fake, None) == _lib.LW_ECAPACITY  # cap < 2n
    assert lib.lw_normals(fake, 3, 16, 0.1, pb, None, fake, None) == _lib.LW_EINVAL
    empty_map = _lib.Map(*([None] * 9), 1024)
    assert lib.lw_live_build(fake, fake, fake, fake, 16, 16, None, None, empty_map, fake, fake, fake, fake, fake,
                             fake, None) == _lib.LW_EINVAL
    assert b"lw_live_build" in lib.lw_last_error()
