"""A prior map on the GPU for nearest-point queries: a dense 5 cm grid over the map's extent (mapgrid.py).

Per cell the grid holds
  - `start`: the map points sorted by cell as a prefix array (cell c's points are start[c] .. start[c+1]), so the
    exact nearest map point within one cell of a query is a scan of the 27 cells around it;
  - `nn`: the map point nearest to the cell centre, jump-flooded (steps 8, 4, 2, 1, 1 cells) over a band of
    ~0.8 m, so queries farther from the map still get a nearest point;
  - `df`: that distance in cm as a byte, 255 beyond the band.

Device layout (HBM): each map point is one 16-byte record (x, y, z, planarity) so that a nearest-point scan
gathers one aligned vector per point; nrm packed float32 triples (read only for a matched point); start int32
[ncell+1], nn int32 [ncell], df uint8 [ncell]: n * 28 + ncell * 9 bytes. The build's two scratch arrays (a
uint64 seed and a second int32 flood buffer, ncell * 12 bytes) are freed when build() returns.

Differences from the reference, both in the build: seeds are 64-bit keys (distance mm << 32 | index), so a map
may hold up to 2^31 - 2 points instead of 2^23 - 1 (mapgrid.py:26-30, 223-224); and each flood step reads one
buffer and writes the other, so the flooded seeds do not depend on thread timing (the reference's k_jfa floods
in place, mapgrid.py:128-158).
"""

from __future__ import annotations

import ctypes as C
import time

import numpy as np
import torch

from . import _lib

CELL = 0.05  # grid cell (m), mapgrid.py:24
JFA_STEPS = (8, 4, 2, 1, 1)  # mapgrid.py:31 (the steps lw_prior_grid_build runs)
PLANAR = 0.5  # planarity above which a map point's normal is trusted, mapgrid.py:32
MAX_POINTS = (1 << 31) - 1  # int32 point indices


def horizontal_levels(xyz: np.ndarray, normal: np.ndarray, planarity: np.ndarray, bin_m: float = 0.02):
    """Histogram of the heights of the map's horizontal surfaces (mapgrid.py:197-205): points whose trusted
    normal is near vertical, binned in z. Returns (counts float32, first edge, bin)."""
    nz = np.abs(normal[:, 2].astype(np.float32))
    sel = (nz > 0.97) & (planarity.astype(np.float32) > PLANAR)
    lo, hi = float(xyz[:, 2].min()), float(xyz[:, 2].max())
    edges = np.arange(lo - 0.5, hi + 0.5 + bin_m, bin_m)
    h, _ = np.histogram(xyz[sel, 2], bins=edges)
    return h.astype(np.float32), float(edges[0]), bin_m


class PriorGrid:
    """A prior map on the GPU: points sorted by cell, unit normals, planarity and the grid (mapgrid.py:208-305).

    prepare() is the host work (sorting by cell), build() the GPU work on an explicit stream. After build()
    nothing writes the arrays again, so any stream may read them.
    """

    @staticmethod
    def prepare(host: dict, cell: float = CELL, pad: float = 0.6) -> dict:
        """Host preparation (mapgrid.py:216-243): float32 arrays sorted by grid cell (a stable sort of the flat
        cell index), unit normals, the grid geometry (origin = min - pad, dims = ceil((max + pad - origin) /
        cell)) and the cell prefix array, plus the horizontal levels."""
        if host.get("_prepared"):
            return host
        xyz = np.asarray(host["xyz"], dtype=np.float32)
        n = len(xyz)
        if n >= MAX_POINTS:
            raise ValueError(f"prior map has {n:,} points; the grid indexes at most {MAX_POINTS - 1:,}")
        if n == 0:
            raise ValueError("prior map is empty")
        nrm = np.asarray(host["normal"], dtype=np.float32)
        planar = np.asarray(host["planarity"] if "planarity" in host else np.ones(n), dtype=np.float32)
        lo, hi = xyz.min(0), xyz.max(0)
        origin = (lo - pad).astype(np.float32)
        dims = np.ceil((hi + pad - origin) / cell).astype(np.int64)
        ijk = np.floor((xyz - origin) / cell).astype(np.int64)
        key = (ijk[:, 2] * dims[1] + ijk[:, 1]) * dims[0] + ijk[:, 0]
        order = np.argsort(key, kind="stable")
        ncell = int(np.prod(dims))
        if ncell + 1 >= MAX_POINTS:
            raise ValueError(f"prior grid of {ncell:,} cells exceeds int32 cell indices")
        counts = np.bincount(key, minlength=ncell)
        start = np.zeros(ncell + 1, np.int32)
        np.cumsum(counts, out=start[1:])
        xyz = np.ascontiguousarray(xyz[order])
        nrm = nrm[order]
        nrm = np.ascontiguousarray(nrm / np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-6),
                                   dtype=np.float32)
        planar = np.ascontiguousarray(planar[order])
        return {"_prepared": True, "xyz": xyz, "normal": nrm, "planarity": planar, "lo": lo, "hi": hi,
                "origin": origin, "cell": float(cell), "dims": dims, "start": start,
                "levels": horizontal_levels(xyz, nrm, planar)}

    def __init__(self, host: dict, device=None):
        _lib.load()
        self.device = torch.device(device if device is not None else "cuda")
        host = self.prepare(host)
        self._host = host
        self.n = len(host["xyz"])
        self.lo, self.hi = host["lo"], host["hi"]
        self.dims = np.asarray(host["dims"], dtype=np.int64)
        self.ncell = int(np.prod(self.dims))
        self.origin = np.asarray(host["origin"], dtype=np.float32)
        self.cell = float(host["cell"])
        self.levels = host["levels"]
        d = self.device
        self.xyzp = torch.empty((self.n, 4), dtype=torch.float32, device=d)  # x, y, z, planarity
        self.nrm = torch.empty((self.n, 3), dtype=torch.float32, device=d)
        self.start = torch.empty(self.ncell + 1, dtype=torch.int32, device=d)
        self.nn = torch.empty(self.ncell, dtype=torch.int32, device=d)
        self.df = torch.empty(self.ncell, dtype=torch.uint8, device=d)
        self.ready = False
        self.build_s = 0.0
        self._g = self._struct(None, None)

    def _struct(self, seed, nn2) -> _lib.PriorGrid:
        g = _lib.PriorGrid()
        g.xyz, g.nrm = _lib.ptr(self.xyzp), _lib.ptr(self.nrm)
        g.start, g.nn, g.df = _lib.ptr(self.start), _lib.ptr(self.nn), _lib.ptr(self.df)
        g.seed, g.nn2 = _lib.ptr(seed), _lib.ptr(nn2)
        g.origin = (_lib.f32 * 3)(*[float(v) for v in self.origin])
        g.cell = self.cell
        g.inv_cell = float(np.float32(1.0 / self.cell))
        g.nx, g.ny, g.nz = (int(v) for v in self.dims)
        g.n, g.ncell = self.n, self.ncell
        return g

    @property
    def struct(self) -> _lib.PriorGrid:
        """The lw_prior_grid the localisation launches read."""
        return self._g

    @property
    def xyz(self) -> torch.Tensor:
        """The sorted map points (a view of the (x, y, z, planarity) records)."""
        return self.xyzp[:, :3]

    @property
    def planar(self) -> torch.Tensor:
        return self.xyzp[:, 3]

    def gpu_bytes(self) -> int:
        return self.n * (16 + 12) + (self.ncell + 1) * 4 + self.ncell * (4 + 1)

    def build(self, stream=None):
        """Upload the points and build the grid, every op on `stream`; returns when it is done."""
        t0 = time.perf_counter()
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        h = self._host
        with torch.cuda.stream(s):
            rec = np.empty((self.n, 4), np.float32)
            rec[:, :3] = h["xyz"]
            rec[:, 3] = h["planarity"]
            self.xyzp.copy_(torch.from_numpy(rec))
            self.nrm.copy_(torch.from_numpy(h["normal"]))
            self.start.copy_(torch.from_numpy(h["start"]))
            seed = torch.empty(self.ncell, dtype=torch.int64, device=self.device)
            nn2 = torch.empty(self.ncell, dtype=torch.int32, device=self.device)
            g = self._struct(seed, nn2)
            _lib.call("lw_prior_grid_build", C.byref(g), _lib.stream_ptr(s))
        s.synchronize()
        del seed, nn2
        self.build_s = time.perf_counter() - t0
        self.ready = True

    def distances(self, pts: torch.Tensor, n: int, T_map_from_pts: np.ndarray, out: torch.Tensor, stream=None):
        """Distance to the map of the first n points of `pts` ([*, 3] float32, in a frame that T maps into the
        map) into `out`, 1e3 beyond the band (mapgrid.py:298-305, k_changes_T :173-194)."""
        if n <= 0:
            return
        if pts.dtype != torch.float32 or not pts.is_contiguous() or pts.shape[-1] != 3 or pts.shape[0] < n:
            raise ValueError("pts must be a contiguous [>=n, 3] float32 CUDA tensor")
        if out.dtype != torch.float32 or out.numel() < n:
            raise ValueError("out must hold n float32")
        T = _lib.f64_array(np.asarray(T_map_from_pts, dtype=np.float64).reshape(16))
        _lib.call("lw_prior_distances", C.byref(self._g), _lib.ptr(pts), int(n), T, _lib.ptr(out),
                  _lib.stream_ptr(stream))
