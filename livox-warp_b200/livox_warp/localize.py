"""Global localisation in a prior map (localize.py): the search (GlobalLocalizer.localize, Localizer), pose tracking
(refine) and the registration of many pose hypotheses at once (register_batch).

The search keeps the reference's stages: the scan's gravity candidates from its horizontal planes (ScanPrep, here
without open3d: 5 cm voxel means, PCA normals from lw_normals, seeded RANSAC planes), the sensor heights where the
scan's horizontal surfaces line up with the map's, the coarse search with its local maxima on the device, a finer
local grid scored with more points, non-maximum suppression, then the batched ICP and the evaluation.

The reference runs GlobalLocalizer._icp (localize.py:517-553) as 3 launches, a device-to-host copy and a numpy
6x6 solve per iteration, for at most 16 poses over one shared scan. Here the whole schedule -- every iteration
of every stage for every hypothesis, then the evaluation of k_eval_batch (:182-205) -- is one cooperative
launch (lw_loc_icp_batch): each hypothesis may have its own scan of any length, the float64 6x6 solve and the
SE(3) update happen on the device, and the stage stops when no hypothesis moved 2e-4 (:551), exactly as the
reference's host loop decides.

The coarse search's hypothesis scores (k_score_grid / k_score_list, localize.py:55-123) are `score_grid` and
`score_list`: a thread per hypothesis with the scan points in shared memory, the soft count kept as integer sums
(exact, independent of the summation order) and rounded once.

Precision: the residuals and Jacobians run in float32 on points re-centred on the hypothesis' translation; the
tile sums, the normal equations, the Cholesky solve and the poses are float64 (the reference sends float32
poses to the device and solves with numpy in float64).

The launch shape -- points per warp tile (32, 64 or 128) and the register budget (3 to 6 resident 256-thread
CTAs per SM) -- is chosen by `Autotuner`, which times the candidates once per batch shape class and
caches the winner (in memory, and in a JSON file when LW_AUTOTUNE_CACHE names one).
"""

from __future__ import annotations

import ctypes as C
import json
import math
import os
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .mapgrid import PriorGrid

EVAL_RADII = (0.03, 0.05, 0.10)  # a pose's fit: the fractions within these distances (m) of the map, localize.py:47
N_EVAL = len(EVAL_RADII)
SCHEDULE_ICP = ((0.40, 8), (0.20, 8), (0.10, 8), (0.05, 10))  # GlobalLocalizer._icp default, localize.py:517
SCHEDULE_REFINE = ((0.30, 6), (0.12, 8), (0.05, 8))  # GlobalLocalizer.refine default, localize.py:569
ALPHA = 0.05  # along-surface weight of a planar correspondence, localize.py:523
MIN_COUNT = 30  # matches below which a hypothesis keeps its pose, localize.py:538
TILES = (32, 64, 128)  # points per warp tile the autotuner tries
BUDGETS = (3, 4, 5, 6)  # resident CTAs per SM of the register budgets it tries (the library also has 2)
CANDIDATES = tuple((t, m) for t in TILES for m in BUDGETS)


def rotz(a: float) -> np.ndarray:
    """Rotation by a (rad) about z (localize.py:222-224)."""
    c, s = math.cos(a), math.sin(a)
    return np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])


def pose_difference(A: np.ndarray, B: np.ndarray):
    """(translation m, rotation deg) between two 4x4 poses (localize.py:236-240)."""
    d = np.linalg.inv(A) @ B
    ang = math.degrees(math.acos(np.clip((np.trace(d[:3, :3]) - 1) / 2, -1, 1)))
    return float(np.linalg.norm(A[:3, 3] - B[:3, 3])), ang


def rot_to(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Rotation taking unit vector a onto unit vector b (localize.py:211-219)."""
    a, b = a / np.linalg.norm(a), b / np.linalg.norm(b)
    v = np.cross(a, b)
    c = float(np.dot(a, b))
    if np.linalg.norm(v) < 1e-9:
        return np.eye(3) if c > 0 else np.diag([1.0, -1.0, -1.0])
    vx = np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])
    return np.eye(3) + vx + vx @ vx * (1.0 / (1.0 + c))


def voxel_means(xyz: np.ndarray, voxel: float) -> np.ndarray:
    """The mean of the points in each voxel of a grid whose origin is half a voxel below the points' minimum
    (open3d's voxel_down_sample anchors its grid there; the reference's ScanPrep calls it), in the order of each
    voxel's first point (open3d's own order is its hash map's)."""
    p = np.asarray(xyz, dtype=np.float64).reshape(-1, 3)
    if len(p) == 0:
        return p
    k = np.floor((p - (p.min(axis=0) - 0.5 * voxel)) / voxel).astype(np.int64)
    _, first, inv = np.unique(k, axis=0, return_index=True, return_inverse=True)
    inv = inv.reshape(-1)
    rank = np.empty(len(first), np.int64)
    rank[np.argsort(first, kind="stable")] = np.arange(len(first))
    vid = rank[inv]
    out = np.zeros((len(first), 3))
    np.add.at(out, vid, p)
    return out / np.bincount(vid, minlength=len(first))[:, None]


def ransac_plane(pts: np.ndarray, dist: float, iters: int, rng: np.random.Generator):
    """The plane through 3 of the points with the most points within `dist` over `iters` seeded draws, refitted
    to those inliers by least squares (what the reference asks of open3d's segment_plane(dist, 3, iters)):
    (a, b, c, d) with a unit normal, and the inlier indices."""
    n = len(pts)
    tri = rng.integers(0, n, (iters, 3))
    a, b, c = pts[tri[:, 0]], pts[tri[:, 1]], pts[tri[:, 2]]
    nrm = np.cross(b - a, c - a)
    ln = np.linalg.norm(nrm, axis=1)
    good = ln > 1e-12
    nrm[good] /= ln[good, None]
    d = -(nrm * a).sum(axis=1)
    counts = np.full(iters, -1, np.int64)
    ok = np.flatnonzero(good)
    for c0 in range(0, len(ok), 32):  # 32 draws per pass: n x 32 distances at a time
        j = ok[c0:c0 + 32]
        counts[j] = (np.abs(pts @ nrm[j].T + d[j]) <= dist).sum(axis=0)
    if len(ok) == 0:
        return None, np.zeros(0, np.int64)
    best = int(np.argmax(counts))  # the first draw with the most inliers
    inl = np.flatnonzero(np.abs(pts @ nrm[best] + d[best]) <= dist)
    q = pts[inl]
    mu = q.mean(axis=0)
    w, V = np.linalg.eigh((q - mu).T @ (q - mu))
    m = V[:, 0]
    if m @ nrm[best] < 0:
        m = -m
    dd = -float(m @ mu)
    inl = np.flatnonzero(np.abs(pts @ m + dd) <= dist)
    return np.array([m[0], m[1], m[2], dd]), inl


class ScanPrep:
    """Host preparation of a scan in the sensor frame (localize.py:243-316) without open3d: 5 cm voxel means,
    a PCA normal per point from its neighbours within 0.2 m (lw_normals on the device), and up to 8 planes found
    by seeded RANSAC (3 cm, 1000 draws, at least 150 inliers) -> up candidates and the height profile.
    `normals` may supply the normal estimator (a function of (points, radius) returning (normals, planarity))."""

    def __init__(self, xyz: np.ndarray, voxel: float = 0.05, max_tilt_deg: float = 45.0, seed: int = 0,
                 normals=None):
        self.pts = voxel_means(xyz, voxel)
        if normals is None:
            from . import prior_map

            normals = prior_map.normals
        nrm, _ = normals(self.pts.astype(np.float32), 0.2)
        self.normals = np.asarray(nrm, dtype=np.float64)
        self.planes = []  # (inliers, unit normal, offset, inlier indices)
        rng = np.random.default_rng(seed)
        idx = np.arange(len(self.pts))
        for _ in range(8):
            if len(idx) < 300:
                break
            model, inl = ransac_plane(self.pts[idx], 0.03, 1000, rng)
            if model is None or len(inl) < 150:
                break
            self.planes.append((len(inl), model[:3], float(model[3]), idx[inl]))
            keep = np.ones(len(idx), bool)
            keep[inl] = False
            idx = idx[keep]
        self.max_tilt = max_tilt_deg

    def up_candidates(self):
        """[(up unit vector, evidence)] for the scan's gravity direction (the reference's ScanPrep.up_candidates,
        localize.py:275-306): the planes within max_tilt of level are floors or ceilings; taken in RANSAC order,
        each joins the first family whose founding normal lies within 10 degrees of its own (either sign) or founds
        one. A family's evidence is its planes' inlier count. The two best families give a normal each -- the least
        spread direction of their planes' points, each plane's points taken about their own centroid -- in both
        signs, pointing first the way the founding plane did. A scan without such planes gives level, either way
        up."""
        level = [(np.array([0.0, 0.0, 1.0]), 0), (np.array([0.0, 0.0, -1.0]), 0)]
        if not self.planes:
            return level
        normals = np.stack([pl[1] for pl in self.planes])
        inliers = [pl[0] for pl in self.planes]
        flat = np.flatnonzero(np.abs(normals[:, 2]) >= math.cos(math.radians(self.max_tilt)))
        same = math.cos(math.radians(10.0))
        founders: list[np.ndarray] = []
        families: list[list[int]] = []
        for i in flat:
            near = [f for f, n0 in enumerate(founders) if abs(float(normals[i] @ n0)) > same]
            if near:
                families[near[0]].append(int(i))
            else:
                founders.append(normals[i])
                families.append([int(i)])
        evidence = [sum(inliers[i] for i in fam) for fam in families]
        ranked = sorted(range(len(families)), key=lambda f: -evidence[f])[:2]  # stable: earlier family on ties
        out = []
        for f in ranked:
            scatter = sum(self._plane_scatter(i) for i in families[f])
            n = np.linalg.eigh(scatter)[1][:, 0]
            n = n if n @ founders[f] >= 0 else -n
            out.extend([(n, evidence[f]), (-n, evidence[f])])
        return out or level

    def _plane_scatter(self, i: int) -> np.ndarray:
        """Scatter matrix of plane i's inliers about their centroid."""
        q = self.pts[self.planes[i][3]]
        q = q - q.mean(axis=0)
        return q.T @ q

    def height_profile(self, up: np.ndarray, lo: float, n_bins: int, bin_m: float):
        """Histogram of the heights (along up, from the sensor) of the scan's horizontal points (localize.py:308-313)."""
        horiz = np.abs(self.normals @ up) > 0.97
        z = self.pts[horiz] @ up
        h, _ = np.histogram(z, bins=n_bins, range=(lo, lo + n_bins * bin_m))
        return h.astype(np.float32)


def height_candidates(levels: np.ndarray, scan: np.ndarray, z_lo: float, bin_m: float, reach: float, z_range,
                      n_max: int, min_sep: float = 0.08) -> list:
    """Sensor heights at which a scan's height profile (horizontal points binned from -reach to +reach about the
    sensor) lines up with the map's (binned from z_lo), best first: each profile is square-rooted (so a big floor
    does not drown the rest) and smoothed over +-2 bins, their correlation is taken at every relative shift, shifts
    putting the sensor outside z_range are dropped, and the best positive ones are picked greedily at least
    min_sep apart, at most n_max (localize.py:400-424)."""
    taper = np.array([0.25, 0.5, 1.0, 0.5, 0.25], np.float32)
    a = np.convolve(np.sqrt(levels), taper, mode="same")
    b = np.convolve(np.sqrt(scan), taper, mode="same")
    score = np.correlate(a, b, mode="full")  # score[j]: the scan shifted by j - (len(b) - 1) bins
    z = z_lo + (np.arange(len(score)) - (len(b) - 1)) * bin_m + reach
    score = np.where((z >= z_range[0]) & (z <= z_range[1]), score, -1.0)
    picked: list[float] = []
    for j in np.argsort(-score):
        if score[j] <= 0 or len(picked) >= n_max:
            break
        if all(abs(float(z[j]) - q) > min_sep for q in picked):
            picked.append(float(z[j]))
    return picked


def thin_5cm(xyz: np.ndarray) -> np.ndarray:
    """One point per 5 cm voxel, the first in scan order (localize.py:579-581): the same set and order as
    np.unique(axis=0, return_index=True) over the voxel rows, from one packed int64 key per point."""
    pts = np.asarray(xyz, dtype=np.float32)
    if len(pts) == 0:
        return pts.reshape(0, 3)
    k = np.floor(pts / 0.05).astype(np.int64)
    if np.abs(k).max() < (1 << 20):
        key = ((k[:, 0] + (1 << 20)) << 42) | ((k[:, 1] + (1 << 20)) << 21) | (k[:, 2] + (1 << 20))
        _, first = np.unique(key, return_index=True)
    else:
        _, first = np.unique(k, axis=0, return_index=True)
    return pts[np.sort(first)]


def tiling(lo: np.ndarray, hi: np.ndarray, tile: int):
    """Tiles of at most `tile` points that never span two hypotheses: (tile_hyp, tile_lo, hyp_tile)."""
    lo = np.asarray(lo, dtype=np.int64)
    n_h = np.maximum(np.asarray(hi, dtype=np.int64) - lo, 0)
    nt_h = (n_h + tile - 1) // tile
    hyp_tile = np.zeros(len(lo) + 1, np.int64)
    np.cumsum(nt_h, out=hyp_tile[1:])
    nt = int(hyp_tile[-1])
    tile_hyp = np.repeat(np.arange(len(lo), dtype=np.int64), nt_h)
    tile_lo = lo[tile_hyp] + (np.arange(nt, dtype=np.int64) - hyp_tile[tile_hyp]) * tile
    return tile_hyp.astype(np.int32), tile_lo.astype(np.int32), hyp_tile.astype(np.int32)


@dataclass
class BatchResult:
    T: np.ndarray  # (k, 4, 4) refined poses
    fit: np.ndarray  # (k, 3) fractions of each scan within EVAL_RADII of the map
    count: np.ndarray  # (k,) matched points in the last iteration
    iters: int  # iterations run (all stages)
    tile: int  # points per warp tile the launch used
    blocks_per_sm: int = 3  # the register budget the launch used


class Autotuner:
    """Chooses the launch shape (tile, blocks_per_sm) of the batched ICP per batch shape class: each candidate is
    timed once with CUDA events on the caller's stream (the poses restored between trials) and the fastest is
    cached."""

    def __init__(self, path: str | None = None):
        self.path = path if path is not None else os.environ.get("LW_AUTOTUNE_CACHE")
        self.table: dict[str, tuple[int, int]] = {}
        if self.path and os.path.exists(self.path):
            try:
                with open(self.path) as f:
                    self.table = {k: (int(v[0]), int(v[1])) for k, v in json.load(f).items()}
            except (OSError, ValueError, TypeError, IndexError):
                self.table = {}
        self.trials: dict[str, dict[tuple[int, int], float]] = {}

    @staticmethod
    def key(n_hyp: int, n_pts: int, schedule) -> str:
        """Shape class: hypotheses and mean points per hypothesis rounded to powers of two, and the schedule."""
        mean = max(1, n_pts // max(n_hyp, 1))
        sched = ",".join(f"{d:g}x{i}" for d, i in schedule)
        return f"h{1 << max(0, int(n_hyp - 1).bit_length())}-p{1 << max(0, int(mean - 1).bit_length())}-{sched}"

    def choose(self, key: str, run) -> tuple[int, int]:
        """The cached shape for `key`, else time run(shape) -> ms for every candidate and keep the fastest."""
        if key in self.table:
            return self.table[key]
        times = {c: run(c) for c in CANDIDATES}
        best = min(times, key=times.get)
        self.trials[key] = times
        self.table[key] = best
        if self.path:
            try:
                with open(self.path, "w") as f:
                    json.dump(self.table, f, indent=1, sort_keys=True)
            except OSError:
                pass
        return best


class LocBatch:
    """Device buffers of lw_loc_batch sized for hyp_cap hypotheses and pts_cap points, with pinned staging."""

    ITERS_CAP = 256

    def __init__(self, device, hyp_cap: int, pts_cap: int):
        d = torch.device(device)
        self.device = d
        self.hyp_cap, self.pts_cap = int(hyp_cap), int(pts_cap)
        self.tiles_cap = self.pts_cap // TILES[0] + self.hyp_cap
        H, NT = self.hyp_cap, self.tiles_cap
        # int32 inputs, one buffer: dims 2 | scan_end H | hyp_tile H+1 | tile_hyp NT | tile_lo NT
        self.o_end, self.o_ht = 2, 2 + H
        self.o_th = self.o_ht + H + 1
        self.o_tl = self.o_th + NT
        n_in = self.o_tl + NT
        self.ints = torch.zeros(n_in, dtype=torch.int32, device=d)
        self.h_ints = torch.zeros(n_in, dtype=torch.int32).pin_memory()
        # int32 outputs, one buffer: count H | eval 3H | iters_run 1 | err 1
        self.o_ev, self.o_it = H, 4 * H
        self.outs = torch.zeros(4 * H + 2, dtype=torch.int32, device=d)
        self.h_outs = torch.zeros(4 * H + 2, dtype=torch.int32).pin_memory()
        self.pts = torch.zeros((self.pts_cap, 4), dtype=torch.float32, device=d)
        self.h_pts = torch.zeros((self.pts_cap, 4), dtype=torch.float32).pin_memory()
        self.T = torch.zeros((H, 16), dtype=torch.float64, device=d)
        self.h_T = torch.zeros((H, 16), dtype=torch.float64).pin_memory()
        self.tile_part = torch.zeros(NT * 32, dtype=torch.float64, device=d)
        self.moved = torch.zeros(self.ITERS_CAP, dtype=torch.int32, device=d)
        self.next = torch.zeros(self.ITERS_CAP + 1, dtype=torch.int32, device=d)
        self.bar = torch.zeros(2, dtype=torch.int32, device=d)
        self.s = self._struct(dims=False)
        self.s_dims = self._struct(dims=True)

    def _struct(self, dims: bool) -> _lib.LocBatch:
        b = _lib.LocBatch()
        base = self.ints.data_ptr()
        ob = self.outs.data_ptr()
        b.pts = _lib.ptr(self.pts)
        b.scan_end = C.c_void_p(base + 4 * self.o_end)
        b.hyp_tile = C.c_void_p(base + 4 * self.o_ht)
        b.tile_hyp = C.c_void_p(base + 4 * self.o_th)
        b.tile_lo = C.c_void_p(base + 4 * self.o_tl)
        b.T = _lib.ptr(self.T)
        b.tile_part = _lib.ptr(self.tile_part)
        b.moved = _lib.ptr(self.moved)
        b.next = _lib.ptr(self.next)
        b.count = C.c_void_p(ob)
        b.eval = C.c_void_p(ob + 4 * self.o_ev)
        b.iters_run = C.c_void_p(ob + 4 * self.o_it)
        b.err = C.c_void_p(ob + 4 * (self.o_it + 1))
        b.bar = _lib.ptr(self.bar)
        b.dims = C.c_void_p(base) if dims else None
        b.pts_cap = self.pts_cap
        b.moved_cap = self.ITERS_CAP
        b.grid_cap = 1 << 20
        return b

    def stage(self, lo, hi, tile: int, stream):
        """Tile the ranges and copy the index arrays (pinned -> device) on `stream`; returns n_tiles."""
        k = len(lo)
        if k > self.hyp_cap:
            raise ValueError(f"{k} hypotheses exceed the batch's {self.hyp_cap}")
        tile_hyp, tile_lo, hyp_tile = tiling(lo, hi, tile)
        nt = len(tile_hyp)
        if nt > self.tiles_cap:
            raise ValueError(f"{nt} tiles exceed the batch's {self.tiles_cap}")
        h = self.h_ints.numpy()
        h[0], h[1] = k, nt
        h[self.o_end:self.o_end + k] = hi
        h[self.o_ht:self.o_ht + k + 1] = hyp_tile
        h[self.o_th:self.o_th + nt] = tile_hyp
        h[self.o_tl:self.o_tl + nt] = tile_lo
        with torch.cuda.stream(stream):
            for a, n in ((0, 2), (self.o_end, k), (self.o_ht, k + 1), (self.o_th, nt), (self.o_tl, nt)):
                if n:
                    self.ints[a:a + n].copy_(self.h_ints[a:a + n], non_blocking=True)
        return nt


def _f32_rows(x, cols: int, name: str) -> torch.Tensor:
    if not (isinstance(x, torch.Tensor) and x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()
            and x.dim() == 2 and x.shape[1] == cols):
        raise ValueError(f"{name} must be a contiguous [n, {cols}] float32 CUDA tensor")
    return x


def score_grid(grid: PriorGrid, pts: torch.Tensor, pos: torch.Tensor, n_yaw: int, yaw0: float, dyaw: float,
               tau_cm: float, free_cm: float, out: torch.Tensor, stream=None, pos_stride: int = 1):
    """k_score_grid (localize.py:55-96): for every position pos[i] ([n, 3]) and heading yaw0 + j dyaw, the soft
    count of the scan points `pts` ([m, 3], gravity-aligned sensor frame) within tau_cm of the map, into
    out[i * n_yaw + j]; -1 where the sensor would sit outside the grid or within free_cm of a mapped surface.
    pos_stride: positions i and i + pos_stride are x neighbours (ny for coarse_positions' layout); it changes the
    thread layout only."""
    _f32_rows(pts, 3, "pts")
    _f32_rows(pos, 3, "pos")
    if out.dtype != torch.float32 or not out.is_contiguous() or out.numel() < pos.shape[0] * n_yaw:
        raise ValueError("out must hold n_pos * n_yaw float32")
    _lib.call("lw_score_grid", C.byref(grid.struct), _lib.ptr(pts), int(pts.shape[0]), _lib.ptr(pos),
              int(pos.shape[0]), int(pos_stride), int(n_yaw), float(yaw0), float(dyaw), float(tau_cm), float(free_cm),
              _lib.ptr(out), _lib.stream_ptr(stream))


def score_list(grid: PriorGrid, pts: torch.Tensor, hyp: torch.Tensor, tau_cm: float, out: torch.Tensor, stream=None):
    """k_score_list (localize.py:99-123): the same soft count for (x, y, z, yaw) hypotheses `hyp` ([n, 4])."""
    _f32_rows(pts, 3, "pts")
    _f32_rows(hyp, 4, "hyp")
    if out.dtype != torch.float32 or not out.is_contiguous() or out.numel() < hyp.shape[0]:
        raise ValueError("out must hold n float32")
    _lib.call("lw_score_list", C.byref(grid.struct), _lib.ptr(pts), int(pts.shape[0]), _lib.ptr(hyp),
              int(hyp.shape[0]), float(tau_cm), _lib.ptr(out), _lib.stream_ptr(stream))


def coarse_positions(lo, hi, heights, xy_step: float) -> tuple[np.ndarray, int, int]:
    """Every position of the xy grid over [lo, hi] at each height (localize.py:428-432): x outer, y inner, one
    block per height; returns (pos [n, 3] float32, nx, ny)."""
    gx = np.arange(lo[0], hi[0] + 1e-6, xy_step)
    gy = np.arange(lo[1], hi[1] + 1e-6, xy_step)
    X, Y = np.meshgrid(gx, gy, indexing="ij")
    pos = np.concatenate([np.stack([X.ravel(), Y.ravel(), np.full(X.size, z)], 1) for z in heights])
    return pos.astype(np.float32), len(gx), len(gy)


class GlobalLocalizer:
    """Batched ICP against a PriorGrid: refine() is the reference's pose-tracking step (localize.py:569-612);
    register_batch() registers many hypotheses, each with its own scan, in one launch."""

    PTS_CAP = 1 << 17  # scan points after 5 cm thinning, localize.py:322
    ICP_CAP = 16  # poses refine() takes together, localize.py:325
    # coarse search tuning (localize.py:359-364)
    xy_step = 0.25
    yaw_step_deg = 2.0
    tau_coarse = 25.0  # cm
    tau_mid = 12.0
    free_cm = 10.0  # the sensor sits at least this far from any mapped surface
    keep_coarse = 128  # coarse local maxima re-scored on the finer grid (localize.py:367)
    n_heights = 8  # sensor heights tried per gravity candidate (localize.py:358)
    n_coarse_pts = 1024
    n_mid_pts = 2048
    n_icp = ICP_CAP  # medium winners refined by ICP per gravity candidate (localize.py:368)
    # unique: inliers (3 cm) at least accept_inliers, and the best answer elsewhere at least accept_gap lower and
    # below accept_ratio of it (localize.py:369-373)
    accept_inliers = 0.45
    accept_gap = 0.15
    accept_ratio = 0.75

    def __init__(self, grid: PriorGrid, device=None, hyp_cap: int = 1024, pts_cap: int = 1 << 23,
                 tuner: Autotuner | None = None):
        if not grid.ready:
            raise RuntimeError("build() the PriorGrid first")
        self.grid = grid
        self.device = torch.device(device) if device is not None else grid.device
        self.batch = LocBatch(self.device, hyp_cap, max(pts_cap, self.PTS_CAP))
        self.tuner = tuner if tuner is not None else Autotuner()
        self.seed = 0  # refine() draws its subset from a fresh generator with this seed
        self.last_tile = 0
        self.last_candidates = 0
        self._graphs: dict = {}

    # ---- the coarse search's scores ------------------------------------------------------------------

    def _coarse(self, stream, pts_g: np.ndarray, heights):
        """Every free-space position on the xy grid at the given heights x every heading, scored in one launch
        (localize.py:426-448). Returns (pos, (n_heights, nx, ny, n_yaw), dyaw, scores)."""
        g = self.grid
        pos, nx, ny = coarse_positions(g.lo, g.hi, heights, self.xy_step)
        n_yaw = int(round(360.0 / self.yaw_step_deg))
        dyaw = math.radians(self.yaw_step_deg)
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.stream(stream):
            d_pts = torch.from_numpy(np.ascontiguousarray(pts_g, dtype=np.float32)).to(self.device, non_blocking=True)
            d_pos = torch.from_numpy(pos).to(self.device, non_blocking=True)
            out = torch.empty(len(pos) * n_yaw, dtype=torch.float32, device=self.device)
            score_grid(g, d_pts, d_pos, n_yaw, 0.0, dyaw, self.tau_coarse, self.free_cm, out, stream, pos_stride=ny)
            sc = out.cpu().numpy()
        return pos, (len(heights), nx, ny, n_yaw), dyaw, sc

    def _coarse_candidates(self, stream, pts_g: np.ndarray, heights, keep: int | None = None, pool: int = 20000):
        """The coarse search with its local maxima found on the device: the reference's _coarse then
        _local_maxima(sc, shape, keep) (localize.py:426-448, 450-483), but only the candidates cross to the host.
        A candidate scores above zero, no lower than its 26 (x, y, heading) neighbours and at least the pool-th
        best score (the reference looks for maxima among the `pool` best); ties are ordered by index. Returns
        (pos, shape, dyaw, best indices, their scores), best first."""
        g = self.grid
        keep = self.keep_coarse if keep is None else keep
        pos, nx, ny = coarse_positions(g.lo, g.hi, heights, self.xy_step)
        n_yaw = int(round(360.0 / self.yaw_step_deg))
        dyaw = math.radians(self.yaw_step_deg)
        shape = (len(heights), nx, ny, n_yaw)
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        cap = 1 << 16
        with torch.cuda.stream(stream):
            d_pts = torch.from_numpy(np.ascontiguousarray(pts_g, dtype=np.float32)).to(self.device, non_blocking=True)
            d_pos = torch.from_numpy(pos).to(self.device, non_blocking=True)
            n = len(pos) * n_yaw
            out = torch.empty(n, dtype=torch.float32, device=self.device)
            score_grid(g, d_pts, d_pos, n_yaw, 0.0, dyaw, self.tau_coarse, self.free_cm, out, stream, pos_stride=ny)
            thr = torch.topk(out, min(pool, n), sorted=False).values.min()
            idx = torch.empty(cap, dtype=torch.int64, device=self.device)
            val = torch.empty(cap, dtype=torch.float32, device=self.device)
            cnt = torch.zeros(1, dtype=torch.int32, device=self.device)
            _lib.call("lw_score_maxima", _lib.ptr(out), shape[0], nx, ny, n_yaw, float(thr.item()), cap,
                      _lib.ptr(idx), _lib.ptr(val), _lib.ptr(cnt), _lib.stream_ptr(stream))
            k = int(cnt.item())
            if k > cap:
                raise _lib.LwError(f"lw_score_maxima: {k} local maxima exceed {cap}")
            bi, bv = idx[:k].cpu().numpy(), val[:k].cpu().numpy()
        self.last_candidates = k  # local maxima found (and copied to the host) by the last call
        order = np.lexsort((bi, -bv))[:keep]
        return pos, shape, dyaw, bi[order], bv[order]

    # ---- the global search (localize.py:400-424, 476-505, 616-738) -----------------------------------------------

    def _heights(self, prep: ScanPrep, up: np.ndarray):
        """Sensor heights (map z) where the scan's horizontal surfaces line up with the map's, best first, or None
        when the scan shows too few horizontal points (GlobalLocalizer._heights, localize.py:400-424)."""
        levels, z_lo, bin_m = self.grid.levels
        reach = 6.0  # m: the scan's horizontal points are binned within this height of the sensor
        scan = prep.height_profile(up, -reach, int(round(2 * reach / bin_m)), bin_m)
        if scan.sum() < 50:
            return None
        return height_candidates(levels, scan, z_lo, bin_m, reach, (self.grid.lo[2] - 0.5, self.grid.hi[2] + 0.5),
                                 self.n_heights)

    @staticmethod
    def _top(scores: np.ndarray, pool: int = 20000) -> np.ndarray:
        """Indices of the `pool` best scores, best first (localize.py:477-482)."""
        pool = min(pool, len(scores))
        idx = np.argpartition(-scores, pool - 1)[:pool] if pool < len(scores) else np.arange(len(scores))
        return idx[np.argsort(-scores[idx])]

    @staticmethod
    def _nms(hyps: np.ndarray, scores: np.ndarray, keep: int, dist: float, ang_deg: float) -> np.ndarray:
        """Greedy non-maximum suppression over (x, y, z, yaw) hypotheses (localize.py:484-505): walking the best
        scores down (the `_top` pool) until a score is not positive, a hypothesis survives unless an earlier
        survivor lies within `dist` metres and `ang_deg` degrees of heading of it; at most `keep` survive. Their
        indices, best first."""
        ang = math.radians(ang_deg)
        kept = np.empty((0, 4))
        chosen: list[int] = []
        for i in GlobalLocalizer._top(scores):
            if scores[i] <= 0 or len(chosen) >= keep:
                break
            h = hyps[i]
            if len(kept):
                near = np.linalg.norm(kept[:, :3] - h[:3], axis=1) < dist
                turn = np.abs((h[3] - kept[:, 3] + math.pi) % (2 * math.pi) - math.pi) < ang
                if np.any(near & turn):
                    continue
            chosen.append(int(i))
            kept = np.vstack([kept, h[None, :]])
        return np.array(chosen, dtype=np.int64)

    def _unique(self, best: float, alt: float) -> bool:
        return best >= self.accept_inliers and best - alt >= self.accept_gap and alt <= self.accept_ratio * best

    @staticmethod
    def _runner_up(results) -> float:
        """Fit (3 cm inliers) of the best result that is a different answer -- more than 1 m or 15 degrees from the
        best result's pose -- or 0 (localize.py:733-738). `results` is sorted best first."""
        winner = results[0][3]
        elsewhere = (r[0] for r in results[1:] if any(a > b for a, b in zip(pose_difference(winner, r[3]),
                                                                             (1.0, 15.0))))
        return next(elsewhere, 0.0)

    def localize(self, xyz: np.ndarray, stream=None, up_prior: np.ndarray | None = None, log=print, progress=None,
                 prep: ScanPrep | None = None):
        """Sensor-to-map pose (4x4) of a scan given in the sensor frame, and diagnostics (GlobalLocalizer.localize,
        localize.py:616-728). Stages: the scan's gravity candidates; for each, the sensor heights that line the
        scan's horizontal surfaces up with the map's and the coarse search over every free position and heading
        (its local maxima found on the device); then, best candidate first, a finer local grid around each coarse
        maximum scored with more points, non-maximum suppression, the batched ICP and the evaluation -- stopping
        once the best answer is good and unique. up_prior (gravity up in the sensor frame) only orders the
        candidates; progress(text) is called between stages; prep may supply a prepared scan. The same scan always
        gives the same answer (the subsets come from a generator seeded with self.seed)."""
        import time

        times: dict = {}
        t_start = time.perf_counter()
        say = progress or (lambda text: None)
        prep = prep if prep is not None else ScanPrep(xyz)
        scan = self._scan_subsets(prep)
        ups = prep.up_candidates()
        if up_prior is not None:
            toward = np.asarray(up_prior, float) / np.linalg.norm(up_prior)
            ups.sort(key=lambda u: -float(u[0] @ toward))
        times["prep"] = time.perf_counter() - t_start
        t0 = time.perf_counter()
        gravity = [self._coarse_stage(stream, prep, up, support, scan["coarse"], say) for up, support in ups]
        times["coarse"] = time.perf_counter() - t0
        gravity.sort(key=lambda c: -c["best_coarse"])
        results, refined = self._fine_stages(stream, gravity, scan, say, times)
        if not results:
            raise RuntimeError("no hypothesis survived (is the scan inside the map?)")
        best = results[0]
        alt = self._runner_up(results)
        times["total"] = time.perf_counter() - t_start
        n_hyp = sum(c["hypotheses"] for c in gravity)
        winner = gravity[best[4]]
        info = {"inliers": best[0], "inliers5": best[1], "inliers10": best[2], "runner_up": alt,
                "unique": self._unique(best[0], alt), "up": winner["up"], "heights": winner["heights"],
                "gravity_candidates": len(gravity), "refined_candidates": refined, "hypotheses": n_hyp,
                "scan_points": scan["n"], "times": times}
        log(f"  {times['total']:.2f} s (prep {times['prep']:.2f}, coarse {times['coarse']:.2f} for "
            f"{n_hyp / 1e6:.1f}M hypotheses, medium {times['mid']:.2f}, ICP {times['icp']:.2f}; "
            f"{refined}/{len(gravity)} gravity candidates refined): inliers {best[0]:.3f} within 3 cm "
            f"(runner-up elsewhere {alt:.3f})")
        return np.asarray(best[3]), info

    def _scan_subsets(self, prep: ScanPrep) -> dict:
        """The scan's points (at most PTS_CAP), the coarse subset (drawn from one point per 15 cm voxel, so it
        spreads over the scan) and the medium subset, from a generator seeded with self.seed."""
        rng = np.random.default_rng(self.seed)
        pts = prep.pts
        if len(pts) > self.PTS_CAP:
            pts = pts[rng.choice(len(pts), self.PTS_CAP, replace=False)]
        if len(pts) < 200:
            raise RuntimeError(f"scan too sparse to localise ({len(pts)} points after 5 cm thinning)")
        _, first = np.unique(np.floor(pts / 0.15).astype(np.int64), axis=0, return_index=True)
        spread = pts[first]
        coarse = spread[rng.choice(len(spread), min(self.n_coarse_pts, len(spread)), replace=False)]
        mid = pts[rng.choice(len(pts), min(self.n_mid_pts, len(pts)), replace=False)]
        return {"pts32": pts.astype(np.float32), "coarse": coarse, "mid": mid, "n": len(pts)}

    def _coarse_stage(self, stream, prep: ScanPrep, up: np.ndarray, support, coarse_pts: np.ndarray, say) -> dict:
        """One gravity candidate's coarse search: its heights (or every height of the map on the xy step when the
        profiles give none) and the coarse local maxima as (x, y, z, yaw) hypotheses with their scores."""
        say(f"coarse search, up {np.round(up, 2)}")
        Rg = rot_to(up, np.array([0.0, 0.0, 1.0]))  # sensor -> gravity-aligned sensor frame
        heights = self._heights(prep, up) or list(np.arange(self.grid.lo[2], self.grid.hi[2] + 1e-6, self.xy_step))
        pc = coarse_pts @ Rg.T
        pos, shape, dyaw, best, best_sc = self._coarse_candidates(stream, pc, heights, keep=self.keep_coarse)
        n_yaw = shape[3]
        hyps = np.concatenate([pos[best // n_yaw], ((best % n_yaw) * dyaw)[:, None]], 1)
        return {"up": up, "Rg": Rg, "heights": heights, "coarse": hyps, "coarse_score": best_sc,
                "best_coarse": float(best_sc[0]) / len(pc) if len(best) else 0.0, "support": support,
                "hypotheses": len(pos) * n_yaw}

    def _local_window(self) -> np.ndarray:
        """(dx, dy, dz, dyaw) offsets of the finer grid scored around each coarse maximum: +-1 coarse step in x and
        y by quarter steps (two modes a step apart share one coarse maximum), +-4 cm in z, +-one heading step by
        0.5 degrees."""
        off = np.arange(-self.xy_step, self.xy_step + 1e-6, self.xy_step / 4)
        offz = np.array([-0.04, 0.0, 0.04])
        offy = np.radians(np.arange(-self.yaw_step_deg, self.yaw_step_deg + 1e-6, 0.5))
        return np.stack([g.ravel() for g in np.meshgrid(off, off, offz, offy, indexing="ij")], 1)

    def _fine_stages(self, stream, gravity: list, scan: dict, say, times: dict):
        """Medium scores, suppression, ICP and evaluation for each gravity candidate, best first, until the best
        answer is good and unique. Returns (results best first, candidates refined); a result is (inliers 3 cm,
        5 cm, 10 cm, pose, candidate index, medium score)."""
        import time

        times["mid"] = times["icp"] = 0.0
        window = self._local_window()
        results: list = []
        refined = 0
        for ci, c in enumerate(gravity):
            if not len(c["coarse"]):
                continue
            say(f"refining gravity candidate {ci + 1}/{len(gravity)}")
            t0 = time.perf_counter()
            pm = scan["mid"] @ c["Rg"].T
            hyps = (c["coarse"][:, None, :] + window[None, :, :]).reshape(-1, 4)
            ms = self._score_list(stream, pm.astype(np.float32), len(pm), hyps, self.tau_mid)
            best = self._nms(hyps, ms, self.n_icp, 0.1, 1.5)
            times["mid"] += time.perf_counter() - t0
            t0 = time.perf_counter()
            starts = [self._pose_of(hyps[i], c["Rg"]) for i in best]
            Ts = self.icp(scan["pts32"], starts, stream=stream)
            fit = self.evaluate(scan["pts32"], Ts, stream=stream)
            results.extend((float(fit[j, 0]), float(fit[j, 1]), float(fit[j, 2]), Ts[j], ci, float(ms[i]) / len(pm))
                           for j, i in enumerate(best))
            times["icp"] += time.perf_counter() - t0
            refined += 1
            results.sort(key=lambda r: -r[0])
            if self._unique(results[0][0], self._runner_up(results)):
                break
        return results, refined

    @staticmethod
    def _pose_of(h: np.ndarray, Rg: np.ndarray) -> np.ndarray:
        """Sensor-to-map pose of an (x, y, z, yaw) hypothesis in the gravity-aligned frame Rg."""
        T = np.eye(4)
        T[:3, :3] = rotz(h[3]) @ Rg
        T[:3, 3] = h[:3]
        return T

    def _score_list(self, stream, pts, m: int, hyps: np.ndarray, tau: float) -> np.ndarray:
        """The soft counts of (x, y, z, yaw) hypotheses for the first m points of `pts` (localize.py:507-515)."""
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        with torch.cuda.stream(stream):
            d_pts = pts if isinstance(pts, torch.Tensor) else torch.from_numpy(
                np.ascontiguousarray(pts, dtype=np.float32)).to(self.device, non_blocking=True)
            d_pts = d_pts[:m].contiguous()
            d_hyp = torch.from_numpy(np.ascontiguousarray(hyps, dtype=np.float32).reshape(-1, 4)).to(
                self.device, non_blocking=True)
            out = torch.empty(d_hyp.shape[0], dtype=torch.float32, device=self.device)
            score_list(self.grid, d_pts, d_hyp, tau, out, stream)
            return out.cpu().numpy()

    # ---- the launch ------------------------------------------------------------------------------

    def _launch(self, n_hyp: int, n_tiles: int, tile: int, schedule, stream, dims: bool = False, minb: int = 3):
        b = self.batch
        dm = (_lib.f64 * max(1, len(schedule)))(*[float(d) for d, _ in schedule] or [0.0])
        it = (_lib.i32 * max(1, len(schedule)))(*[int(i) for _, i in schedule] or [0])
        _lib.call("lw_loc_icp_batch", C.byref(self.grid.struct), C.byref(b.s_dims if dims else b.s), int(n_hyp),
                  int(n_tiles), int(tile), len(schedule), dm, it, ALPHA, MIN_COUNT, int(minb), 0, _lib.stream_ptr(stream))

    def _put_T(self, Ts, stream):
        b = self.batch
        k = len(Ts)
        b.h_T.numpy()[:k] = np.asarray(Ts, dtype=np.float64).reshape(k, 16)
        with torch.cuda.stream(stream):
            b.T[:k].copy_(b.h_T[:k], non_blocking=True)

    def _get(self, k: int, stream):
        """Copy back poses and counts of k hypotheses (waits for the stream)."""
        b = self.batch
        with torch.cuda.stream(stream):
            b.h_T[:k].copy_(b.T[:k], non_blocking=True)
            b.h_outs.copy_(b.outs, non_blocking=True)
        stream.synchronize()
        o = b.h_outs.numpy()
        if o[b.o_it + 1] != 0:
            raise _lib.LwError(f"lw_loc_icp_batch: a grid barrier gave up (code {int(o[b.o_it + 1])})")
        T = b.h_T.numpy()[:k].reshape(k, 4, 4).copy()
        count = o[:k].copy()
        ev = o[b.o_ev:b.o_ev + 3 * k].reshape(k, 3).copy()
        return T, count, ev, int(o[b.o_it])

    def _run(self, lo, hi, Ts, schedule, stream, tile: int | None = None, minb: int | None = None) -> BatchResult:
        """ICP then evaluation of hypotheses h over points [lo[h], hi[h]) already in the batch's pts. With tile
        None the autotuner picks the launch shape; with tile given, minb None means the default budget (3)."""
        k = len(Ts)
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        lo = np.asarray(lo, dtype=np.int64)
        hi = np.asarray(hi, dtype=np.int64)
        n_pts = int(np.maximum(hi - lo, 0).sum())
        if tile is None:
            key = Autotuner.key(k, n_pts, schedule)

            def trial(shape):
                t, m = shape
                nt = self.batch.stage(lo, hi, t, stream)
                self._put_T(Ts, stream)
                self._launch(k, nt, t, schedule, stream, minb=m)  # warm
                self._put_T(Ts, stream)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                self._launch(k, nt, t, schedule, stream, minb=m)
                e1.record(stream)
                e1.synchronize()
                return e0.elapsed_time(e1)

            tile, minb = self.tuner.choose(key, trial)
        minb = 3 if minb is None else minb
        nt = self.batch.stage(lo, hi, tile, stream)
        self._put_T(Ts, stream)
        self._launch(k, nt, tile, schedule, stream, minb=minb)
        T, count, ev, iters = self._get(k, stream)
        self.last_tile = tile
        n_h = np.maximum(hi - lo, 1).astype(np.float64)
        return BatchResult(T, ev / n_h[:, None], count, iters, tile, minb)

    def _upload_pts(self, parts, stream) -> tuple[np.ndarray, np.ndarray]:
        """Pack point sets (each (n, 3) float32) one after another into the batch's pts; returns (lo, hi)."""
        b = self.batch
        sizes = np.array([len(p) for p in parts], dtype=np.int64)
        hi = np.cumsum(sizes)
        lo = hi - sizes
        total = int(hi[-1]) if len(hi) else 0
        if total > b.pts_cap:
            raise ValueError(f"{total} points exceed the batch's {b.pts_cap}")
        h = b.h_pts.numpy()
        for p, a, n in zip(parts, lo, sizes):
            h[a:a + n, :3] = p
        with torch.cuda.stream(stream):
            b.pts[:total].copy_(b.h_pts[:total], non_blocking=True)
        return lo, hi

    # ---- the reference's API ----------------------------------------------------------------------

    def refine(self, xyz: np.ndarray, T0: np.ndarray, stream=None, schedule=SCHEDULE_REFINE, starts=(),
               switch_margin: float = 0.05):
        """Point-to-plane ICP of a point set against the map from T0 (which maps the points' frame into the
        map), localize.py:569-612. Returns (T, fit, info); fit = the fractions of the thinned points within each
        of EVAL_RADII of the map at T. starts: extra map-frame offsets (x, y, z m[, heading deg about the
        vertical through the points' centre]) refined in the same batch; one wins only if its 3 cm fit beats
        the plain result by switch_margin."""
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        rng = np.random.default_rng(self.seed)
        pts = thin_5cm(xyz)
        if len(pts) > self.PTS_CAP:
            pts = pts[rng.choice(len(pts), self.PTS_CAP, replace=False)]
        n = len(pts)
        if n < 200:
            raise RuntimeError(f"too few points to refine ({n} after 5 cm thinning)")
        T0 = np.asarray(T0, dtype=np.float64)
        inits = [T0]
        c_map = T0[:3, :3] @ pts.mean(axis=0).astype(np.float64) + T0[:3, 3]
        for off in list(starts)[: self.ICP_CAP - 2]:
            Ti = T0.copy()
            off = np.asarray(off, dtype=np.float64)
            if len(off) > 3 and off[3] != 0.0:
                Rz = rotz(math.radians(off[3]))
                Ti[:3, :3] = Rz @ Ti[:3, :3]
                Ti[:3, 3] = Rz @ (Ti[:3, 3] - c_map) + c_map
            Ti[:3, 3] += off[:3]
            inits.append(Ti)
        self._upload_pts([pts], stream)
        k = len(inits)
        res = self._run(np.zeros(k, np.int64), np.full(k, n, np.int64), inits, schedule, stream)
        start = self._run(np.zeros(1, np.int64), np.full(1, n, np.int64), [T0], (), stream, tile=res.tile,
                          minb=res.blocks_per_sm)
        fits = res.fit
        best = 0
        for i in range(1, k):
            if fits[i, 0] > fits[best, 0] + (switch_margin if best == 0 else 0.0):
                best = i
        return res.T[best], fits[best], {"switched": best != 0, "plain_fit": float(fits[0, 0]), "n": n,
                                         "fit_start": float(start.fit[0, 0]), "iters": res.iters}

    def icp(self, pts: np.ndarray, Ts, schedule=SCHEDULE_ICP, stream=None) -> list:
        """GlobalLocalizer._icp (localize.py:517-553) on one shared scan for every pose in Ts."""
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        pts = np.asarray(pts, dtype=np.float32)
        self._upload_pts([pts], stream)
        k = len(Ts)
        res = self._run(np.zeros(k, np.int64), np.full(k, len(pts), np.int64), Ts, schedule, stream)
        return list(res.T)

    def evaluate(self, pts: np.ndarray, Ts, stream=None) -> np.ndarray:
        """GlobalLocalizer._evaluate (localize.py:555-565): fractions of the scan within EVAL_RADII, per pose."""
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        pts = np.asarray(pts, dtype=np.float32)
        self._upload_pts([pts], stream)
        k = len(Ts)
        return self._run(np.zeros(k, np.int64), np.full(k, len(pts), np.int64), Ts, (), stream, tile=256).fit

    # ---- many hypotheses, uneven scans --------------------------------------------------------------

    def register_batch(self, scans, T0s, schedule=SCHEDULE_ICP, stream=None, tile: int | None = None,
                       blocks_per_sm: int | None = None) -> BatchResult:
        """Register hypothesis h's own scan (scans[h], (n_h, 3) float32 in the sensor frame) from T0s[h], all
        in one launch; returns the refined poses, their fits and the matched counts."""
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        if len(scans) != len(T0s):
            raise ValueError("one scan per hypothesis")
        lo, hi = self._upload_pts([np.asarray(s, dtype=np.float32) for s in scans], stream)
        return self._run(lo, hi, T0s, schedule, stream, tile, blocks_per_sm)

    def register_packed(self, pts4: torch.Tensor, lo, hi, T0s, schedule=SCHEDULE_ICP, stream=None,
                        tile: int | None = None, blocks_per_sm: int | None = None) -> BatchResult:
        """register_batch for scans already packed one after another in `pts4` ((N, 4) float32: x, y, z, unused;
        a pinned host tensor is copied asynchronously, a device tensor in place); hypothesis h owns rows
        lo[h] .. hi[h]."""
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        b = self.batch
        n = pts4.shape[0]
        if pts4.dtype != torch.float32 or pts4.dim() != 2 or pts4.shape[1] != 4 or not pts4.is_contiguous():
            raise ValueError("pts4 must be a contiguous (N, 4) float32 tensor")
        if n > b.pts_cap:
            raise ValueError(f"{n} points exceed the batch's {b.pts_cap}")
        lo = np.asarray(lo, dtype=np.int64)
        hi = np.asarray(hi, dtype=np.int64)
        if len(lo) != len(T0s) or len(hi) != len(T0s) or (len(lo) and (lo.min() < 0 or hi.max() > n)):
            raise ValueError("lo / hi must give each hypothesis a row range of pts4")
        with torch.cuda.stream(stream):
            b.pts[:n].copy_(pts4, non_blocking=True)
        return self._run(lo, hi, T0s, schedule, stream, tile, blocks_per_sm)

    def register_graph(self, lo, hi, schedule=SCHEDULE_ICP, tile: int = 256, stream=None, blocks_per_sm: int = 3):
        """A CUDA graph of the batched launch for the staged batch's shape class: the hypothesis and tile counts
        are read on the device (lw_loc_batch.dims), so one capture replays over any batch up to the buffers'
        capacity with that schedule and tile. Returns a callable that stages (lo, hi, T0s) and replays it."""
        stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        key = (tuple(schedule), tile, blocks_per_sm)
        g = self._graphs.get(key)
        b = self.batch
        if g is None:
            nt = b.stage(lo, hi, tile, stream)  # a valid batch in place while capturing
            self._put_T(np.tile(np.eye(4), (len(lo), 1, 1)), stream)
            stream.synchronize()
            g = torch.cuda.CUDAGraph()
            cap = torch.cuda.Stream(self.device)
            cap.wait_stream(stream)
            with torch.cuda.graph(g, stream=cap, capture_error_mode="thread_local"):
                self._launch(b.hyp_cap, b.tiles_cap, tile, schedule, cap, dims=True, minb=blocks_per_sm)
            stream.wait_stream(cap)
            self._graphs[key] = g

        def replay(lo, hi, T0s):
            b.stage(lo, hi, tile, stream)
            self._put_T(T0s, stream)
            with torch.cuda.stream(stream):
                g.replay()
            T, count, ev, iters = self._get(len(T0s), stream)
            n_h = np.maximum(np.asarray(hi) - np.asarray(lo), 1).astype(np.float64)
            return BatchResult(T, ev / n_h[:, None], count, iters, tile, blocks_per_sm)

        return replay


class Localizer:
    """Single-threaded convenience wrapper (localize.py:739-763): builds the prior grid and searches on one
    stream."""

    def __init__(self, map_xyz: np.ndarray, map_normal: np.ndarray, map_planarity: np.ndarray | None = None,
                 device=None, stream=None):
        host = {"xyz": map_xyz, "normal": map_normal}
        if map_planarity is not None:
            host["planarity"] = map_planarity
        self.grid = PriorGrid(host, device)
        self.stream = stream
        self.grid.build(stream)
        self.loc = GlobalLocalizer(self.grid, self.grid.device)

    def search(self, xyz: np.ndarray, log=print, up_prior=None):
        """GlobalLocalizer.localize on this stream: the pose of a sensor-frame scan, and diagnostics."""
        return self.loc.localize(xyz, self.stream, up_prior=up_prior, log=log)

    def refine(self, xyz: np.ndarray, T0: np.ndarray, **kw):
        """GlobalLocalizer.refine on this stream: ICP of a point set from the known pose T0."""
        return self.loc.refine(xyz, T0, self.stream, **kw)

