"""Prior grid and batched localisation ICP on the GPU against the CPU oracle.

The grid (flooded nearest points and distance field) and every nearest-point query are integer results and
must match the oracle bit for bit. The batched ICP is compared pose by pose with the oracle's float64
restatement of GlobalLocalizer._icp (localize.py:517-553): within 1 mm / 0.01 deg, the same iteration count
within one (the stop test moved < 2e-4 can fall either side of an iteration by float rounding), and the
evaluation counts within 0.5 % of the scan.
"""

import math

import numpy as np
import pytest
import torch

import common
from oracle import oracle

pytestmark = pytest.mark.gpu

POSE_TOL_M, POSE_TOL_DEG = 1e-3, 0.01


def _pose_err(A, B):
    d = np.linalg.inv(A) @ B
    ang = math.degrees(math.acos(np.clip((np.trace(d[:3, :3]) - 1) / 2, -1, 1)))
    return float(np.linalg.norm(A[:3, 3] - B[:3, 3])), ang


@pytest.fixture(scope="module")
def room():
    from livox_warp import synth
    from livox_warp.mapgrid import PriorGrid

    sc = synth.box_room(3)
    xyz, nrm = synth.sample_surfaces(sc, 0.02, 0, jitter=0.002)
    planar = np.ones(len(xyz), np.float32)
    planar[::7] = 0.3  # some clutter points: the point-to-point branch
    host = PriorGrid.prepare({"xyz": xyz, "normal": nrm, "planarity": planar})
    grid = PriorGrid(host)
    grid.build()
    og = oracle.PriorGrid(oracle.prior_prepare(xyz, nrm, planar))
    return sc, grid, og


def test_prepare_matches_oracle(room):
    _, grid, og = room
    h = grid._host
    assert np.array_equal(h["xyz"], og.xyz) and np.array_equal(h["start"], og.start)
    assert np.array_equal(h["normal"], og.nrm) and np.array_equal(h["planarity"], og.planar)
    assert np.array_equal(h["origin"], og.prep["origin"]) and np.array_equal(h["dims"], og.dims)


def test_grid_build_bit_exact(room):
    _, grid, og = room
    assert np.array_equal(grid.nn.cpu().numpy(), og.nn)
    assert np.array_equal(grid.df.cpu().numpy(), og.df)
    assert (og.nn >= 0).mean() > 0.3 and (og.df < 255).any()


def test_distances_bit_exact(room):
    sc, grid, og = room
    rng = np.random.default_rng(4)
    # queries near surfaces, in the flooded band and far outside the grid
    q = og.xyz[rng.choice(len(og.xyz), 20000)] + rng.normal(0, 0.08, (20000, 3)).astype(np.float32)
    q = np.concatenate([q, rng.uniform(-5, 15, (5000, 3)).astype(np.float32)]).astype(np.float32)
    T = np.eye(4)
    T[:3, :3] = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    T[:3, 3] = [7.0, -1.0, 0.0]
    Ti = np.linalg.inv(T)
    pts = (q.astype(np.float64) @ Ti[:3, :3].T + Ti[:3, 3]).astype(np.float32)
    dev = torch.from_numpy(pts).cuda()
    out = torch.empty(len(pts), dtype=torch.float32, device="cuda")
    grid.distances(dev, len(pts), T, out)
    got = out.cpu().numpy()
    want = og.distances(pts, T)
    assert np.array_equal(got, want)
    assert (want >= 1e3).any() and (want < 0.05).mean() > 0.3


def _hypotheses(sc, n, seed, trans=0.15, yaw=4.0, sizes=(2000, 20000)):
    from livox_warp import synth

    T_true = synth.free_poses(sc, n, seed, z=1.2, margin=0.5)
    T0 = synth.perturb(T_true, seed + 1, trans, yaw, tilt_deg=1.0)
    rng = np.random.default_rng(seed + 2)
    scans = [synth.spin_scan(sc, T_true[h], int(rng.integers(sizes[0], sizes[1] + 1)), seed + 10 + h)
             for h in range(n)]
    return T_true, T0, scans


def _oracle_batch(og, scans, T0, schedule):
    pts4 = np.zeros((sum(len(s) for s in scans), 4), np.float32)
    hi = np.cumsum([len(s) for s in scans])
    lo = hi - [len(s) for s in scans]
    for s, a in zip(scans, lo):
        pts4[a:a + len(s), :3] = s
    T, count, iters = og.icp(pts4, lo, hi, T0, schedule)
    ev = og.evaluate(pts4, lo, hi, T)
    return T, count, iters, ev


@pytest.mark.parametrize("tile,minb", [(32, 6), (32, 4), (64, 5), (128, 2), (512, 3)])
def test_batch_uneven_scans_match_oracle(room, tile, minb):
    from livox_warp.localize import SCHEDULE_ICP, GlobalLocalizer

    sc, grid, og = room
    T_true, T0, scans = _hypotheses(sc, 12, 40)
    loc = GlobalLocalizer(grid, hyp_cap=64, pts_cap=1 << 19)
    res = loc.register_batch(scans, T0, SCHEDULE_ICP, tile=tile, blocks_per_sm=minb)
    oT, ocount, oiters, oev = _oracle_batch(og, scans, T0, SCHEDULE_ICP)
    assert abs(res.iters - oiters) <= 1
    for h in range(len(scans)):
        dt, da = _pose_err(res.T[h], oT[h])
        assert dt < POSE_TOL_M and da < POSE_TOL_DEG, (h, dt, da)
        n = len(scans[h])
        assert abs(int(res.count[h]) - int(ocount[h])) <= max(2, n // 200), h
        ev = np.rint(res.fit[h] * n).astype(np.int64)
        assert np.all(np.abs(ev - oev[h]) <= max(2, n // 200)), (h, ev, oev[h])
    # the registration itself: the noise-free poses are found
    ok = [(_pose_err(res.T[h], T_true[h])[0] < 0.05) for h in range(len(scans))]
    assert np.mean(ok) >= 0.75


def test_shared_scan_refine_and_starts(room):
    """refine (localize.py:569-612): one shared thinned scan, T0 plus offset starts in the same batch."""
    from livox_warp import synth
    from livox_warp.localize import SCHEDULE_REFINE, GlobalLocalizer, thin_5cm

    sc, grid, og = room
    T_true = synth.free_poses(sc, 1, 77, z=1.3, margin=0.6)[0]
    xyz = synth.spin_scan(sc, T_true, 60000, 78)
    T0 = synth.perturb(T_true[None], 79, 0.08, 2.0)[0]
    loc = GlobalLocalizer(grid, hyp_cap=64, pts_cap=1 << 19)
    starts = [(0.3, 0.0, 0.0), (0.0, -0.3, 0.0, 5.0)]
    T, fit, info = loc.refine(xyz, T0, starts=starts)
    pts = oracle.thin_5cm(xyz)
    assert info["n"] == len(pts)
    assert np.array_equal(thin_5cm(xyz), pts)
    # the oracle refines the same three starts
    c_map = T0[:3, :3] @ pts.mean(axis=0).astype(np.float64) + T0[:3, 3]
    inits = [T0]
    for off in starts:
        Ti = T0.copy()
        off = np.asarray(off, dtype=np.float64)
        if len(off) > 3 and off[3] != 0.0:
            c, s = math.cos(math.radians(off[3])), math.sin(math.radians(off[3]))
            Rz = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
            Ti[:3, :3] = Rz @ Ti[:3, :3]
            Ti[:3, 3] = Rz @ (Ti[:3, 3] - c_map) + c_map
        Ti[:3, 3] += off[:3]
        inits.append(Ti)
    oT, _, _, oev = _oracle_batch(og, [pts] * len(inits), np.stack(inits), SCHEDULE_REFINE)
    ofit = oev / len(pts)
    best = 0
    for i in range(1, len(inits)):
        if ofit[i, 0] > ofit[best, 0] + (0.05 if best == 0 else 0.0):
            best = i
    assert info["switched"] == (best != 0)
    dt, da = _pose_err(T, oT[best])
    assert dt < POSE_TOL_M and da < POSE_TOL_DEG
    assert np.all(np.abs(fit - ofit[best]) <= 0.005)
    assert _pose_err(T, T_true)[0] < 0.03
    start_fit = og.evaluate(np.concatenate([pts, np.zeros((len(pts), 1), np.float32)], 1), [0], [len(pts)], T0[None])
    assert abs(info["fit_start"] - start_fit[0, 0] / len(pts)) < 1e-9


def test_graph_replay_equals_direct_launch(room):
    """A captured launch reading its counts on the device gives the direct launch's results bit for bit, for
    batches of different shapes replayed through the same graph."""
    from livox_warp.localize import SCHEDULE_ICP, GlobalLocalizer

    sc, grid, og = room
    loc = GlobalLocalizer(grid, hyp_cap=64, pts_cap=1 << 19)
    for seed, n in ((50, 10), (60, 6)):
        T_true, T0, scans = _hypotheses(sc, n, seed)
        direct = loc.register_batch(scans, T0, SCHEDULE_ICP, tile=256)
        lo, hi = loc._upload_pts(scans, torch.cuda.current_stream())
        replay = loc.register_graph(lo, hi, SCHEDULE_ICP, tile=256)
        got = replay(lo, hi, T0)
        assert np.array_equal(got.T, direct.T)
        assert np.array_equal(got.count, direct.count) and np.array_equal(got.fit, direct.fit)
        assert got.iters == direct.iters


def test_degenerate_hypotheses_keep_pose(room):
    """A hypothesis with no points, or with fewer than 30 matches, keeps its pose; the others still converge."""
    from livox_warp.localize import SCHEDULE_ICP, GlobalLocalizer

    sc, grid, og = room
    T_true, T0, scans = _hypotheses(sc, 4, 90)
    far = np.eye(4)
    far[:3, 3] = [500.0, 500.0, 500.0]
    scans = scans + [np.zeros((0, 3), np.float32), scans[0][:20]]
    T0 = np.concatenate([T0, far[None], T0[:1]])
    loc = GlobalLocalizer(grid, hyp_cap=64, pts_cap=1 << 19)
    res = loc.register_batch(scans, T0, SCHEDULE_ICP, tile=128)
    assert np.array_equal(res.T[4], far) and np.array_equal(res.T[5], T0[5])
    assert res.count[4] == 0 and res.count[5] <= 20
    oT, _, _, _ = _oracle_batch(og, scans, T0, SCHEDULE_ICP)
    for h in range(4):
        dt, da = _pose_err(res.T[h], oT[h])
        assert dt < POSE_TOL_M and da < POSE_TOL_DEG


def test_argument_errors(room):
    from livox_warp import _lib
    from livox_warp.localize import GlobalLocalizer

    sc, grid, og = room
    loc = GlobalLocalizer(grid, hyp_cap=8, pts_cap=1 << 17)
    with pytest.raises(_lib.LwError):
        loc._launch(1, 1, 100, ((0.1, 2),), torch.cuda.current_stream())  # tile must be a multiple of 32
    with pytest.raises(_lib.LwError):
        loc._launch(1, 1, 256, ((0.1, 200), (0.1, 200)), torch.cuda.current_stream())  # > moved_cap iterations
    with pytest.raises(_lib.LwError):
        loc._launch(1, 1, 256, ((0.1, 2),), torch.cuda.current_stream(), minb=7)  # register budget 2..6
    with pytest.raises(ValueError):
        loc.register_batch([np.zeros((10, 3), np.float32)] * 9, np.tile(np.eye(4), (9, 1, 1)))
    with pytest.raises(RuntimeError):
        loc.refine(np.zeros((50, 3), np.float32), np.eye(4))


def _score_case(sc, seed, n_pts):
    from livox_warp import synth

    T = synth.free_poses(sc, 1, seed)[0]
    pts = synth.spin_scan(sc, T, 3 * n_pts, seed + 1)[:n_pts]
    return T, np.ascontiguousarray(pts, dtype=np.float32)


@pytest.mark.parametrize("n_pts,stride", [(1024, 1), (2500, 1), (1024, "ny"), (700, 5)])
def test_score_grid_bit_exact(room, n_pts, stride):
    """lw_score_grid against the oracle, every (position, heading) bit for bit: positions inside and outside the
    grid and inside surfaces (-1), 36 headings, scans of one and of several shared-memory chunks, each thread
    layout (x neighbours along a warp, plain list order, a stride that does not divide the positions)."""
    from livox_warp.localize import coarse_positions, score_grid

    sc, grid, og = room
    T, pts = _score_case(sc, 7, n_pts)
    pos, nx, ny = coarse_positions(grid.lo - 0.5, grid.hi + 0.5, [0.6, 1.2, 1.8], 0.35)
    n_yaw, yaw0, dyaw = 36, 0.05, math.radians(10.0)
    out = torch.full((len(pos) * n_yaw,), 7.0, dtype=torch.float32, device="cuda")
    score_grid(grid, torch.from_numpy(pts).cuda(), torch.from_numpy(pos).cuda(), n_yaw, yaw0, dyaw, 25.0, 10.0, out,
               pos_stride=ny if stride == "ny" else stride)
    got = out.cpu().numpy()
    want = og.score_grid(pts, pos, n_yaw, yaw0, dyaw, 25.0, 10.0)
    assert np.array_equal(got, want)
    assert (want == -1.0).sum() > 100 and (want > 0.5 * n_pts).any()


def test_score_list_bit_exact(room):
    from livox_warp.localize import score_list

    sc, grid, og = room
    T, pts = _score_case(sc, 11, 2048)
    rng = np.random.default_rng(2)
    yaw = math.atan2(T[1, 0], T[0, 0])
    hyp = np.concatenate([T[:3, 3] + rng.normal(0, 0.3, (5000, 3)), yaw + rng.normal(0, 0.5, (5000, 1))], 1)
    hyp = hyp.astype(np.float32)
    out = torch.empty(len(hyp), dtype=torch.float32, device="cuda")
    score_list(grid, torch.from_numpy(pts).cuda(), torch.from_numpy(hyp).cuda(), 12.0, out)
    got = out.cpu().numpy()
    want = og.score_list(pts, hyp, 12.0)
    assert np.array_equal(got, want)
    true = og.score_list(pts, np.array([[T[0, 3], T[1, 3], T[2, 3], yaw]], np.float32), 12.0)[0]
    assert true > 0.8 * len(pts) and true >= np.quantile(want, 0.99)


def test_coarse_search_finds_the_pose(room):
    """GlobalLocalizer._coarse over the whole room (0.25 m, 2 degrees, three heights): the best hypothesis lies
    within one grid step and two heading steps of the scan's true pose."""
    from livox_warp.localize import GlobalLocalizer

    sc, grid, og = room
    T, pts = _score_case(sc, 13, 1024)
    loc = GlobalLocalizer(grid, hyp_cap=16, pts_cap=1 << 12)
    pos, shape, dyaw, s = loc._coarse(None, pts, [T[2, 3] - 0.1, T[2, 3], T[2, 3] + 0.1])
    assert shape[3] == 180 and len(s) == len(pos) * 180
    best = int(np.argmax(s))
    p, iyaw = pos[best // 180], best % 180
    yaw = math.atan2(T[1, 0], T[0, 0]) % (2 * math.pi)
    dy = abs((iyaw * dyaw - yaw + math.pi) % (2 * math.pi) - math.pi)
    assert np.linalg.norm(p[:2] - T[:2, 3]) <= 0.25 * 1.5 and dy <= 2 * dyaw + 1e-6, (p, T[:3, 3], dy)
    ms = loc._score_list(None, pts, len(pts), np.array([[*p, iyaw * dyaw]], np.float32), loc.tau_mid)
    assert ms[0] == og.score_list(pts, np.array([[*p, iyaw * dyaw]], np.float32), loc.tau_mid)[0]


def test_score_grid_rejects_too_many_headings(room):
    from livox_warp import _lib
    from livox_warp.localize import score_grid

    sc, grid, og = room
    pts = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    pos = torch.zeros((2, 3), dtype=torch.float32, device="cuda")
    out = torch.empty(2 * 2000, dtype=torch.float32, device="cuda")
    with pytest.raises(_lib.LwError, match="n_yaw"):
        score_grid(grid, pts, pos, 2000, 0.0, 0.01, 25.0, 10.0, out)
    with pytest.raises(_lib.LwError, match="pos_stride"):
        score_grid(grid, pts, pos, 4, 0.0, 0.01, 25.0, 10.0, out, pos_stride=0)


def test_coarse_candidates_follow_the_local_maximum_rule(room):
    """lw_score_maxima through GlobalLocalizer._coarse_candidates: every local maximum among the 20000 best scores,
    the same set the reference's rule selects on the full score array, best first."""
    from livox_warp.localize import GlobalLocalizer

    sc, grid, og = room
    T, pts = _score_case(sc, 13, 1024)
    loc = GlobalLocalizer(grid, hyp_cap=16, pts_cap=1 << 12)
    heights = [T[2, 3] - 0.1, T[2, 3], T[2, 3] + 0.1]
    pos, shape, dyaw, s = loc._coarse(None, pts, heights)
    pos2, shape2, dyaw2, idx, val = loc._coarse_candidates(None, pts, heights, keep=1 << 20)
    assert shape2 == shape and np.array_equal(pos2, pos)
    want = common.rule_local_maxima(s, shape, 20000)
    assert len(want) > 10 and set(idx.tolist()) == set(want.tolist())
    assert np.array_equal(val, s[idx]) and np.all(np.diff(val) <= 0)
    top = loc._coarse_candidates(None, pts, heights)[3]
    assert np.array_equal(top, idx[:loc.keep_coarse])


def test_score_empty_inputs(room):
    """No scan points: every free position scores 0 and the rest -1, as the oracle; no positions or hypotheses:
    nothing is written."""
    from livox_warp.localize import coarse_positions, score_grid, score_list

    sc, grid, og = room
    pos, nx, ny = coarse_positions(grid.lo, grid.hi, [1.2], 0.5)
    none = torch.zeros((0, 3), dtype=torch.float32, device="cuda")
    out = torch.full((len(pos) * 8,), 7.0, dtype=torch.float32, device="cuda")
    score_grid(grid, none, torch.from_numpy(pos).cuda(), 8, 0.0, 0.7, 25.0, 10.0, out, pos_stride=ny)
    got = out.cpu().numpy()
    want = og.score_grid(np.zeros((0, 3), np.float32), pos, 8, 0.0, 0.7, 25.0, 10.0)
    assert np.array_equal(got, want) and set(np.unique(got).tolist()) <= {0.0, -1.0} and (got == 0.0).any()
    out.fill_(7.0)
    score_grid(grid, none, torch.zeros((0, 3), dtype=torch.float32, device="cuda"), 8, 0.0, 0.7, 25.0, 10.0, out)
    h = torch.zeros((0, 4), dtype=torch.float32, device="cuda")
    score_list(grid, none, h, 12.0, out)
    assert bool((out == 7.0).all())


def test_global_search_end_to_end_on_the_device():
    """GlobalLocalizer.localize (localize.py:616-728) with every stage on the B200: the prior map built by the
    library from a simulated terrestrial scan (voxel means and normals on the device), the grid flooded on the
    device, the coarse search with its local maxima, the list scores, the batched ICP and the evaluation. A
    360-degree scan is placed within 2 cm / 0.3 deg of the truth and the answer is unique; the same search with
    the oracle answering the device stages (tests/test_localize_host_cpu.py) reaches the same pose within 1 mm."""
    from livox_warp import prior_map, synth
    from livox_warp.localize import Localizer, ScanPrep, pose_difference

    sc = synth.box_room(3, size=(9.0, 6.5, 3.2), n_boxes=25, side=(0.3, 2.4))
    stations = [T[:3, 3] for T in synth.free_poses(sc, 2, 4, z=1.5, margin=0.6)]
    cloud = synth.tls_scan(sc, stations, seed=0, step_deg=0.5)
    pm = prior_map.from_points(cloud, voxel=0.02, normal_radius=0.08)
    loc = Localizer(pm["xyz"], pm["normal"], pm["planarity"])
    T_true = synth.free_poses(sc, 1, 8, z=1.4, margin=0.6)[0]
    x = synth.spin_scan(sc, T_true, 80000, 21, noise=0.01)
    x = x[np.linalg.norm(x, axis=1) > 0.3]
    T, info = loc.search(x, log=lambda *a: None)
    dt, dr = pose_difference(T_true, T)
    assert dt < 0.02 and dr < 0.3, (dt, dr, info["inliers"], info["runner_up"])
    assert info["unique"] and info["inliers"] > 0.8 and abs(info["up"][2]) > 0.99
    assert info["times"]["total"] < 30.0
    # the oracle's stages on the same prepared scan and map
    prep = ScanPrep(x)
    og = oracle.PriorGrid(oracle.prior_prepare(pm["xyz"], pm["normal"], pm["planarity"]))
    pts4 = np.zeros((len(prep.pts), 4), np.float32)
    pts4[:, :3] = prep.pts
    T_o, _, _ = og.icp(pts4, np.zeros(1, np.int32), np.full(1, len(pts4), np.int32), T[None].copy(),
                       ((0.05, 10),))
    do, ro = pose_difference(T_o[0], T)
    assert do < 1e-3 and ro < 0.02, (do, ro)
