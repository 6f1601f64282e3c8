"""The oracle against the reference's own kernels.

tests/golden/make_golden.py ran the reference's Warp kernels -- their source, unchanged -- under a serial stand-in
for Warp (tests/golden/warp_shim.py: threads in ascending index order, float32 arithmetic as written) on small
seeded inputs, and stored the inputs with what the kernels produced (tests/golden/ref_*.npz). Here the oracle
(oracle/lw_oracle.cpp, oracle/oracle.py) runs on the same inputs and is held to those outputs:

  * keys, counts, kept points and their order, first / last times, carving misses, visible-set membership,
    Motion labels, ground labels, heights and cluster partitions: bit for bit (hash tables slot for slot);
  * sums, means and covariances: 1e-5 relative -- the reference adds float32 values into float32 sums, the
    oracle keeps exact integer sums and divides once;
  * one Gauss-Newton accumulation (H, b, the surface-normal H, weights, ranges): 2e-5 relative -- float32
    per-point terms in both, summed in float64 by the reference and the oracle alike, with the reference's
    per-point float32 eigen-decomposition against the oracle's float64 one per voxel;
  * deskewed points: within 4 ulps of the point's largest coordinate (the reference rotates with a float32
    quaternion, six roundings deep; the oracle in float64, rounded once);
  * batched localisation: the whole ICP schedule lands within 1e-5 m / 1e-4 deg of the reference's poses, the
    evaluation counts are equal.
"""

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle

GOLD = Path(__file__).resolve().parent / "golden"
FIX_R, FIX_RR, FIX_W = 2.0 ** 32, 2.0 ** 40, 2.0 ** 20


def _load(name):
    return np.load(GOLD / f"{name}.npz")


def _x4(x, t=None):
    x = np.asarray(x, np.float32)
    w = np.zeros((len(x), 4), np.float32)
    w[:, :3] = x
    if t is not None:
        w[:, 3] = t
    return w


def _range4(x):
    """x, y, z and the range sqrt((x x + y y) + z z) in float32, the thinned-point layout."""
    x = np.asarray(x, np.float32)
    r = np.sqrt((x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1]) + x[:, 2] * x[:, 2])
    return np.ascontiguousarray(np.concatenate([x, r[:, None]], 1), dtype=np.float32)


# ---- odometry ----------------------------------------------------------------------------------------------------


def test_thinning_equals_reference_kernel():
    F = _load("ref_odom")
    o = oracle.thin(_x4(F["thin_x"], F["thin_t"]), F["thin_a"], F["thin_inv_v"], 0.3, 60.0, int(F["thin_ret_mask"]))
    assert len(o) == len(F["thin_out"]) > 500
    assert np.array_equal(o[:, :3], F["thin_out"])


def test_deskew_within_float32_rounding_of_reference_kernel():
    F = _load("ref_odom")
    o = oracle.deskew(_x4(F["thin_x"], F["thin_t"]), float(F["deskew_t_mid"]), 10.0, F["deskew_tw"])[:, :3]
    r = F["deskew_out"]
    tol = 4.0 * np.spacing(np.abs(o).max(axis=1, keepdims=True))
    assert (np.abs(o - r) <= tol).all()


def _reg_oracle(F):
    cap = len(F["reg_keys"])
    oreg = oracle.RegMap(cap)
    for x, a, t in zip(F["reg_x"], F["reg_a"], F["reg_t"]):
        oreg.insert(_x4(x, t), a, F["reg_T"], float(F["reg_voxel"]), 60.0, 0b1111)
    return oreg


def test_registration_map_equals_reference_kernel():
    F = _load("ref_odom")
    oreg = _reg_oracle(F)
    # the same voxels in the same slots, the same counts and stats
    assert np.array_equal(oreg.keys, F["reg_keys"])
    assert np.array_equal(oreg.cnt, F["reg_cnt"])
    assert np.array_equal(oreg.stats, F["reg_stats"])
    occ = F["reg_keys"] != -1
    c = F["reg_cnt"][occ].astype(np.float64)[:, None]
    mean_ref = F["reg_sum"][occ].astype(np.float64) / c
    mean_or = oreg.sum[occ] / FIX_R / c
    np.testing.assert_allclose(mean_or, mean_ref, rtol=1e-5, atol=1e-6)
    iu = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]
    outer_ref = np.stack([F["reg_outer"][occ][:, i, j] for i, j in iu], 1).astype(np.float64) / c
    outer_or = oreg.outer[occ] / FIX_RR / c
    np.testing.assert_allclose(outer_or, outer_ref, rtol=1e-5, atol=1e-7)


def test_gauss_newton_accumulation_equals_reference_kernel():
    F = _load("ref_odom")
    oreg = _reg_oracle(F)
    voxel = float(F["reg_voxel"])
    oreg.records(voxel, 0.02, 0.05)
    ds4 = _range4(F["icp_pts"])
    for (it, reach, max_d2, kappa), ref in zip(F["icp_sched"], F["icp_acc"]):
        o = oracle.icp_accumulate(ds4, F["reg_T"], oreg, voxel, int(reach), float(max_d2), float(kappa))
        assert o[oracle.ACC_COUNT] == ref[oracle.ACC_COUNT] > 1000
        for lo, hi in ((0, 21), (21, 27), (32, 53)):  # H, b, the surface-normal H
            assert np.linalg.norm(o[lo:hi] - ref[lo:hi]) <= 2e-5 * np.linalg.norm(ref[lo:hi])
        for k in (oracle.ACC_RMS, oracle.ACC_WEIGHT, oracle.ACC_RANGE):
            assert abs(o[k] - ref[k]) <= 2e-5 * abs(ref[k])


# ---- integration map, carving and the visible set -------------------------------------------------------------


def _view(F):
    from livox_warp import _lib

    vals = list(F["map_view"])
    v = _lib.View()
    for n, ctype in _lib.View._fields_:
        if n in ("crop_lo", "crop_hi"):
            setattr(v, n, [vals.pop(0) for _ in range(3)])
        else:
            x = vals.pop(0)
            setattr(v, n, int(x) if ctype.__name__.startswith("c_int") else float(x))
    return v


@pytest.fixture(scope="module")
def map_run():
    F = _load("ref_map")
    view = _view(F)
    voxel, cap = float(F["map_voxel"]), int(F["map_cap"])
    poses = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (oracle.POSE_SLOTS, 1))
    om = oracle.Map(cap)
    ends = np.cumsum(F["ins_len"])
    starts = ends - F["ins_len"]
    for k, (a, b) in enumerate(zip(starts, ends)):
        poses[k] = F["poses_T0"].astype(np.float32).reshape(16)
        om.insert(F["ins_x"][a:b], F["ins_a"][a:b], F["ins_t"][a:b], F["ins_f"][a:b], poses, view, voxel)
        if k >= 4:
            j = k - 4
            om.carve(F["carve_x"][j], F["carve_a"][j], F["carve_f"][j], poses, voxel, every=int(F["carve_every"][j]),
                     nthreads=1)
    return F, om, view


def test_integration_map_equals_reference_kernel(map_run):
    F, om, _ = map_run
    assert np.array_equal(om.keys, F["keys"])
    assert np.array_equal(om.cnt, F["cnt"])
    assert np.array_equal(om.last, F["last"]) and np.array_equal(om.first, F["first"])
    assert np.array_equal(om.stats, F["stats"])
    occ = F["keys"] != -1
    n = np.minimum(F["cnt"][occ], 4096).astype(np.float64)[:, None]
    np.testing.assert_allclose(om.acc[occ][:, :3] / FIX_W / n, F["acc"][occ][:, :3].astype(np.float64) / n,
                               rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(om.acc[occ][:, 3] / n[:, 0], F["acc"][occ][:, 3] / n[:, 0], rtol=1e-5)


def test_carving_misses_equal_reference_kernel(map_run):
    F, om, _ = map_run
    assert F["miss"].sum() > 1000 and (F["miss"] > 0).sum() > 200
    assert set(F["carve_every"].tolist()) == {1, 2}
    assert np.array_equal(om.miss, F["miss"])


def test_visible_set_and_motion_labels_equal_reference_kernel(map_run):
    F, om, view = map_run
    xyz, attr, t, dyn = om.build(view, 1)
    assert len(xyz) == len(F["cls_slots"]) > 1000
    np.testing.assert_allclose(xyz, F["cls_xyz"], rtol=1e-5, atol=1e-6)
    assert np.array_equal(attr, F["cls_attr"])
    assert np.array_equal(t, F["cls_t"])
    assert np.array_equal(dyn, F["cls_dyn"]) and dyn.sum() > 50


# ---- perception --------------------------------------------------------------------------------------------------


@pytest.mark.parametrize("use_nrm", [0, 1])
def test_ground_equals_reference_kernels(use_nrm):
    F = _load("ref_perception")
    cell, thick, min_sup, thresh, slope, nz_min = F["ground_params"]
    g, h = oracle.ground(F["pts"], cell, thick, int(min_sup), thresh, slope, F["nrm"] if use_nrm else None, nz_min)
    assert np.array_equal(g, F[f"gnd{use_nrm}"]) and 1000 < g.sum() < len(g) - 1000
    assert np.array_equal(h, F[f"hag{use_nrm}"])


def _partition(ids):
    """Points grouped by label, as a set of frozensets (unlabelled points, -1, left out)."""
    groups = {}
    for i, c in enumerate(ids):
        if c >= 0:
            groups.setdefault(int(c), []).append(i)
    return {frozenset(v) for v in groups.values()}


@pytest.mark.parametrize("tag", ["a", "b"])
def test_clusters_equal_reference_kernels(tag):
    F = _load("ref_perception")
    voxel, connect, min_pts = F[f"cl{tag}_params"]
    cid, labels, clusters, k_all = oracle.cluster(F["pts"], F["gnd0"], voxel, connect, int(min_pts))
    assert int(F[f"cl{tag}_converged"]) == 1
    # the same nodes, the same components, the same clusters (the reference numbers them in hash-slot order,
    # the oracle in the order of each cluster's first node: compared as partitions)
    assert len(labels) == len(F[f"cl{tag}_label"])
    ref_cid = F[f"cl{tag}_cid"]
    assert _partition(cid) == _partition(ref_cid)
    assert len(clusters) == len(F[f"cl{tag}_cnt"]) >= 3
    for j, (cnt, cen, lo, hi) in enumerate(clusters):
        members = np.nonzero(cid == j)[0]
        r = int(ref_cid[members[0]])
        assert cnt == F[f"cl{tag}_cnt"][r]
        np.testing.assert_allclose(cen, F[f"cl{tag}_cen"][r], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(lo, F[f"cl{tag}_lo"][r], rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(hi, F[f"cl{tag}_hi"][r], rtol=1e-5, atol=1e-6)


# ---- localisation ------------------------------------------------------------------------------------------------


@pytest.fixture(scope="module")
def loc_grid():
    F = _load("ref_localize")
    prep = {"xyz": F["xyz"], "normal": F["normal"], "planarity": F["planarity"], "start": F["start"],
            "dims": F["dims"], "origin": F["origin"], "cell": float(F["cell"])}
    return F, oracle.PriorGrid(prep)


def test_prior_grid_preparation_equals_reference(loc_grid):
    F, _ = loc_grid
    p = oracle.prior_prepare(F["map_in_xyz"], F["map_in_normal"], F["map_in_planarity"])
    for k in ("xyz", "normal", "planarity", "start", "dims"):
        assert np.array_equal(np.asarray(p[k]), F[k]), k
    np.testing.assert_array_equal(np.asarray(p["origin"], np.float64), F["origin"])


def test_prior_grid_flood_against_reference_kernels(loc_grid):
    """Every cell that holds map points keeps the same seed (k_seed's atomic minimum). The reference floods in
    place, so a cell may read a neighbour already updated in the same pass and its result depends on thread
    timing; the oracle floods double-buffered. Elsewhere the two choose the same seed in >= 99.9 % of the cells,
    and where they differ the seeds lie within 3 mm of the same distance and the distance field within 1 cm."""
    F, g = loc_grid
    seeded = np.diff(F["start"]) > 0
    assert seeded.sum() > 5000 and np.array_equal(g.nn[seeded], F["nn"][seeded])
    diff = np.nonzero(g.nn != F["nn"])[0]
    assert len(diff) <= 1e-3 * len(g.nn)
    nx, ny, _ = F["dims"]
    ix, r = diff % nx, diff // nx
    centre = F["origin"] + (np.stack([ix, r % ny, r // ny], 1) + 0.5) * float(F["cell"])
    x = F["xyz"].astype(np.float64)
    d_or = np.linalg.norm(centre - x[g.nn[diff]], axis=1)
    d_ref = np.linalg.norm(centre - x[F["nn"][diff]], axis=1)
    assert np.abs(d_or - d_ref).max(initial=0.0) <= 3e-3
    assert np.abs(g.df.astype(int) - F["df"].astype(int)).max() <= 1
    assert (g.df != F["df"]).sum() <= 1e-4 * len(g.df)


def test_batched_icp_and_evaluation_equal_reference_kernels(loc_grid):
    F, g = loc_grid
    pts4 = _x4(F["scan"])
    k = len(F["T_start"])
    lo = np.zeros(k, np.int32)
    hi = np.full(k, len(pts4), np.int32)
    sched = [(float(d), int(i)) for d, i in F["schedule"]]
    T, count, run = g.icp(pts4, lo, hi, F["T_start"].copy(), sched)
    assert run == int(F["iters_run"])
    for h in range(k):
        dt, dr = oracle.pose_error(F["T_end"][h], T[h])
        assert dt <= 1e-5 and dr <= 1e-4, (h, dt, dr)
    counts = g.evaluate(pts4, lo, hi, T)
    assert np.array_equal(counts, F["eval_counts"])
