"""Batched point-to-plane ICP against a prior map (localize.py): pose tracking (refine) and the registration of
many pose hypotheses at once (register_batch).

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
