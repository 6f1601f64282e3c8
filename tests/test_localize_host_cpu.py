"""The global search's host stages against the reference's own code (localize.py, run from source on seeded inputs
by tests/golden/make_golden.py into tests/golden/localize_host.npz): rot_to, ScanPrep.up_candidates and
height_profile, GlobalLocalizer._heights, _nms (with _top), _runner_up and _unique. Exact, or to float64 rounding
where an eigensolver is involved."""

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "localize_host.npz"


def _prep(z, k):
    from livox_warp.localize import ScanPrep

    prep = ScanPrep.__new__(ScanPrep)  # the scan given, not prepared: the planes are the fixture's
    prep.pts, prep.normals, prep.max_tilt = z[f"prep{k}_pts"], z[f"prep{k}_normals"], 45.0
    cnt, nrm, off = z[f"prep{k}_plane_cnt"], z[f"prep{k}_plane_n"], z[f"prep{k}_plane_off"]
    starts = np.concatenate([[0], np.cumsum(cnt)])
    prep.planes = [(int(cnt[i]), nrm[i], float(off[i]), np.arange(starts[i], starts[i + 1])) for i in range(len(cnt))]
    return prep


def test_rot_to():
    from livox_warp.localize import rot_to

    z = np.load(GOLDEN)
    for a, b, want in zip(z["rot_a"], z["rot_b"], z["rot_out"]):
        assert np.allclose(rot_to(a, b), want, rtol=0, atol=1e-15)


def test_up_candidates_height_profile_and_heights():
    from livox_warp.localize import GlobalLocalizer

    z = np.load(GOLDEN)
    lvl, _ = np.histogram(np.concatenate([np.full(900, 0.0), np.full(600, 3.9), np.full(300, 0.8)]), bins=300,
                          range=(-1.0, 5.0))

    class Grid:
        levels = (lvl.astype(np.float32), -1.0, 0.02)
        lo = np.array([0.0, 0.0, -0.2])
        hi = np.array([20.0, 10.0, 4.0])

    for k in range(3):
        prep = _prep(z, k)
        ups = prep.up_candidates()
        assert np.allclose(np.array([u[0] for u in ups]), z[f"prep{k}_ups"], rtol=0, atol=1e-12)
        assert [u[1] for u in ups] == z[f"prep{k}_support"].tolist()
        assert np.array_equal(prep.height_profile(ups[0][0], -6.0, 600, 0.02), z[f"prep{k}_hprof"])
        loc = GlobalLocalizer.__new__(GlobalLocalizer)  # the host stages need no device
        loc.grid = Grid
        assert np.array_equal(np.array(loc._heights(prep, ups[0][0]) or []), z[f"prep{k}_heights"])


def test_nms_runner_up_and_unique():
    from livox_warp.localize import GlobalLocalizer

    z = np.load(GOLDEN)
    for j in range(3):
        keep, dist, ang = z[f"nms{j}_args"]
        got = GlobalLocalizer._nms(z["nms_hyps"], z["nms_scores"], int(keep), float(dist), float(ang))
        assert np.array_equal(got, z[f"nms{j}"])
    results = [(float(f), 0.0, 0.0, T, 0, 0.0) for f, T in zip(z["ru_fits"], z["ru_poses"])]
    assert np.array_equal(np.array([GlobalLocalizer._runner_up(results[i:]) for i in range(11)]), z["ru_out"])
    loc = GlobalLocalizer.__new__(GlobalLocalizer)
    assert np.array_equal(np.array([loc._unique(float(p), float(q)) for p, q in z["uq_pairs"]]), z["uq_out"])


def test_localize_end_to_end_with_the_oracle_for_the_device_stages():
    """GlobalLocalizer.localize (localize.py:616-728) as written, with the four device stages answered by the oracle
    (coarse scores and their local maxima, list scores, batched ICP, evaluation) and the scan prepared without
    open3d (ScanPrep: 5 cm means, exact PCA normals, seeded RANSAC planes): a 360-degree scan in the box room,
    in a prior map built from a simulated terrestrial scan, is placed within 2 cm / 0.3 degrees of the truth,
    found unique, with the floor as gravity candidate."""
    import math

    import common
    from livox_warp import synth
    from livox_warp.localize import GlobalLocalizer, ScanPrep, coarse_positions, pose_difference
    from livox_warp.mapgrid import PriorGrid
    from oracle import oracle

    # boxes up to 2.4 m tall in a 9 x 6.5 m room: above 1.5 m a room of low boxes is nearly symmetric under a half
    # turn, and the search rightly calls such an answer ambiguous
    sc = synth.box_room(3, size=(9.0, 6.5, 3.2), n_boxes=25, side=(0.3, 2.4))
    stations = [T[:3, 3] for T in synth.free_poses(sc, 2, 4, z=1.5, margin=0.6)]
    cloud = synth.tls_scan(sc, stations, seed=0, step_deg=0.5)
    vx, _, _, _ = oracle.voxel_downsample(cloud, None, None, 0.02)
    nrm, pl = oracle.normals(vx, 0.08)
    host = PriorGrid.prepare({"xyz": vx, "normal": nrm, "planarity": pl})
    og = oracle.PriorGrid(oracle.prior_prepare(vx, nrm, pl))

    class Grid:
        lo, hi, levels = host["lo"], host["hi"], host["levels"]

    class OracleStages(GlobalLocalizer):
        def __init__(self):
            self.grid, self.seed = Grid, 0

        def _coarse_candidates(self, stream, pts_g, heights, keep=None, pool=20000):
            pos, nx, ny = coarse_positions(Grid.lo, Grid.hi, heights, self.xy_step)
            n_yaw, dyaw = int(round(360.0 / self.yaw_step_deg)), math.radians(self.yaw_step_deg)
            s = og.score_grid(np.asarray(pts_g, np.float32), pos, n_yaw, 0.0, dyaw, self.tau_coarse, self.free_cm)
            shape = (len(heights), nx, ny, n_yaw)
            c = common.rule_local_maxima(s, shape, pool)
            c = c[np.lexsort((c, -s[c]))][:keep]
            return pos, shape, dyaw, c, s[c]

        def _score_list(self, stream, pts, m, hyps, tau):
            return og.score_list(np.asarray(pts, np.float32)[:m], np.asarray(hyps, np.float32), tau)

        def _batch(self, pts, Ts):
            k, n = len(Ts), len(pts)
            pts4 = np.zeros((k * n, 4), np.float32)
            pts4[:, :3] = np.tile(pts, (k, 1))
            lo = np.arange(k) * n
            return pts4, lo, lo + n

        def icp(self, pts, Ts, schedule=None, stream=None):
            from livox_warp.localize import SCHEDULE_ICP

            pts4, lo, hi = self._batch(pts, Ts)
            T, _, _ = og.icp(pts4, lo, hi, np.stack(Ts), schedule or SCHEDULE_ICP)
            return list(T)

        def evaluate(self, pts, Ts, stream=None):
            pts4, lo, hi = self._batch(pts, Ts)
            return og.evaluate(pts4, lo, hi, np.stack(Ts)) / float(len(pts))

    T_true = synth.free_poses(sc, 1, 8, z=1.4, margin=0.6)[0]
    x = synth.spin_scan(sc, T_true, 80000, 21, noise=0.01)
    x = x[np.linalg.norm(x, axis=1) > 0.3]
    prep = ScanPrep(x, normals=oracle.normals)
    T, info = OracleStages().localize(x, prep=prep, log=lambda *a: None)
    dt, dr = pose_difference(T_true, T)
    assert dt < 0.02 and dr < 0.3, (dt, dr, info["inliers"], info["runner_up"])
    assert info["unique"] and info["inliers"] > 0.8 and abs(info["up"][2]) > 0.99


def test_scan_prep_voxel_means_and_ransac_plane():
    """The two steps ScanPrep restates from open3d: voxel means on a grid anchored half a voxel below the points'
    minimum, as open3d anchors it (each voxel's float64 mean, in the order of its first point), and a seeded
    RANSAC plane that finds a noisy plane
    among outliers and returns its least-squares refit and inliers; the same seed gives the same plane."""
    from livox_warp.localize import ransac_plane, voxel_means

    rng = np.random.default_rng(3)
    p = rng.uniform(-1, 1, (5000, 3))
    m = voxel_means(p, 0.25)
    k = np.floor((p - (p.min(0) - 0.125)) / 0.25).astype(np.int64)
    _, first, inv = np.unique(k, axis=0, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")
    want = np.stack([p[inv.reshape(-1) == v].mean(0) for v in order])
    assert np.allclose(m, want, rtol=0, atol=1e-12)
    n = np.array([0.2, -0.1, 1.0]) / np.linalg.norm([0.2, -0.1, 1.0])
    u = np.cross(n, [1.0, 0.0, 0.0])
    u /= np.linalg.norm(u)
    v = np.cross(n, u)
    plane = 0.7 * n + rng.uniform(-2, 2, (3000, 1)) * u + rng.uniform(-2, 2, (3000, 1)) * v
    plane += rng.normal(0, 0.005, plane.shape) * n
    pts = np.concatenate([plane, rng.uniform(-2, 2, (1500, 3))])
    model, inl = ransac_plane(pts, 0.03, 1000, np.random.default_rng(0))
    assert abs(abs(model[:3] @ n) - 1.0) < 1e-4 and abs(abs(model[3]) - 0.7) < 2e-3
    # nearly every plane point, and only the few outliers inside the 3 cm slab (about 1.5 % of 1500)
    assert len(np.intersect1d(inl, np.arange(3000))) > 2990 and len(inl) < 3100
    again, inl2 = ransac_plane(pts, 0.03, 1000, np.random.default_rng(0))
    assert np.array_equal(model, again) and np.array_equal(inl, inl2)
