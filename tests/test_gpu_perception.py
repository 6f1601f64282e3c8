"""Ground labels and Euclidean clusters on the GPU against the CPU oracle: bit exact (labels, heights, cluster
ids, counts, centroids, boxes), and the component labels against the reference's own algorithm -- min-label
propagation with pointer jumping (perception.py:142-179), run here in numpy over the same node graph."""

import numpy as np
import pytest
import torch

from oracle import oracle

pytestmark = pytest.mark.gpu


def _office_points(n_frames=2, seed=5):
    """World points of a dual-return scan in the office with walkers (the full-perception configuration)."""
    from livox_warp import synth

    import common

    sc = synth.office(4, walkers=10)
    T0 = common.look_at([6.0, 4.0, 1.4], [14.0, 9.0, 0.6])
    traj = synth.ConstantVelocity(T0, 0.0, 0.5, 0.2)
    pts = []
    for k in range(n_frames):
        x, a, t = synth.scan(sc, traj, k * 0.1, (k + 1) * 0.1, 100000.0, seed, dual=True)
        T = traj.poses(t)
        w = np.einsum("nij,nj->ni", T[:, :3, :3], x.astype(np.float64)) + T[:, :3, 3]
        pts.append(w.astype(np.float32))
    return pts


def _pipe_with(points):
    from livox_warp import gpu

    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 16)
    pipe.load_points(points)
    return pipe


def test_ground_bit_exact_and_grid_restored():
    from livox_warp.perception import Perception

    frames = _office_points(2)
    pipe = _pipe_with(frames[0])
    perc = Perception(pipe, cluster_slots=1 << 18)
    for w in frames:  # the second call checks the grid the first one restored
        pipe.load_points(w)
        perc.ground(cell=0.5, thick=0.15, min_sup=3, thresh=0.2, slope_step=0.3)
        n = pipe.count
        g, h = pipe.gnd[:n].cpu().numpy(), pipe.hag[:n].cpu().numpy()
        og, oh = oracle.ground(w, cell=0.5, thick=0.15, min_sup=3, thresh=0.2, slope_step=0.3)
        assert np.array_equal(g, og)
        assert np.array_equal(h, oh)
        assert 0.1 < g.mean() < 0.9, "the scan should see floor and structure"
    assert float(perc.cell_min.min()) >= 1e29 and int(perc.cell_sup.abs().sum()) == 0


@pytest.mark.parametrize("voxel,connect", [(0.2, 0.35), (0.1, 0.35)])
def test_clusters_bit_exact(voxel, connect):
    from livox_warp.perception import Perception

    w = _office_points(1)[0]
    pipe = _pipe_with(w)
    perc = Perception(pipe, cluster_slots=1 << 18)
    perc.ground(cell=0.5, thick=0.15, min_sup=3, thresh=0.2, slope_step=0.3)
    clusters = perc.cluster(voxel=voxel, connect=connect, min_pts=30, use_ground=True)
    n = pipe.count
    gnd = pipe.gnd[:n].cpu().numpy()
    cid = pipe.cid[:n].cpu().numpy()
    ocid, olabels, oclusters, k_all = oracle.cluster(w, gnd, voxel=voxel, connect=connect, min_pts=30)
    assert perc.cc_converged
    assert len(clusters) == len(oclusters) >= 3
    assert np.array_equal(cid, ocid)
    assert np.array_equal(perc.node_labels(), olabels)
    for c, (cnt, cen, lo, hi) in zip(clusters, oclusters):
        assert c["cnt"] == cnt
        assert np.array_equal(c["cen"].astype(np.float32), cen)
        assert np.array_equal(c["lo"].astype(np.float32), lo) and np.array_equal(c["hi"].astype(np.float32), hi)


def test_components_equal_min_label_propagation():
    """The union-find's labels are the fixed point of the reference's min-label propagation on the same graph."""
    from scipy.spatial import cKDTree

    from livox_warp.perception import Perception

    w = _office_points(1)[0]
    pipe = _pipe_with(w)
    perc = Perception(pipe, cluster_slots=1 << 18)
    perc.cluster(voxel=0.2, connect=0.35, min_pts=30, use_ground=False)
    labels = perc.node_labels()
    m = len(labels)
    cen = perc._t["v_xyz"][:m].cpu().numpy()
    # the graph the reference's radius query walks: node pairs within `connect` (float32 squared distance)
    pairs = np.array(sorted(cKDTree(cen).query_pairs(0.36)), dtype=np.int64).reshape(-1, 2)
    d2 = ((cen[pairs[:, 0]] - cen[pairs[:, 1]]) ** 2).sum(axis=1, dtype=np.float32)
    pairs = pairs[d2 <= np.float32(0.35) * np.float32(0.35)]
    lab = np.arange(m)
    for _ in range(10000):  # k_cc_step (hook to the smallest neighbour label) + k_cc_jump, to convergence
        nb = np.minimum(lab[pairs[:, 0]], lab[pairs[:, 1]])
        new = lab.copy()
        np.minimum.at(new, pairs[:, 0], nb)
        np.minimum.at(new, pairs[:, 1], nb)
        np.minimum.at(new, lab, new)  # hook the ancestor too
        new = new[new]
        if np.array_equal(new, lab):
            break
        lab = new
    assert np.array_equal(lab, labels)
