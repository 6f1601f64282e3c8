"""Prior maps from point clouds on the GPU (prior_map.py): voxel means with the mean colour, intensity and point
count, then a PCA normal and a planarity for every mean -- the arrays `mapgrid.PriorGrid` takes.

Same calls as the reference: `voxel_downsample(xyz, intensity, rgb, voxel, device=None, chunk=1 << 25,
slots_log2=27)`, `normals(xyz, radius, device=None)`, `from_points(xyz, voxel=0.02, normal_radius=0.08, device=None,
slots_log2=24, stations=None)` and `load(path)`. `VoxelTable` and `normals_device` are the same steps on torch CUDA
tensors, for a cloud already in device memory; `from_points` keeps the voxel means on the device between the two.

The kernels are the library's `lw_vox_insert` / `lw_vox_emit` (k_vox_insert, k_vox_flag, k_vox_emit,
prior_map.py:57-123) and `lw_normals` (k_normals :126-166). Two differences a caller may notice: the voxels come in
the order of their first point in the input (the reference's come in hash-slot order), and every sum is exact
fixed point, so the results do not change from run to run. E57 conversion (`convert`, `add_stations`, the command
line) reads files with pye57, which this build does not carry; `from_points` is the in-memory equivalent.
"""

from __future__ import annotations

import numpy as np
import torch

from . import _lib

VOXEL_TILE = 1024


def _device(device) -> torch.device:
    d = torch.device(device if device is not None else "cuda")
    if d.type == "cuda" and d.index is None:
        d = torch.device("cuda", torch.cuda.current_device())
    return d


def _rows(t: torch.Tensor, cols: int, name: str) -> torch.Tensor:
    if t.dim() != 2 or t.shape[1] != cols or t.dtype != torch.float32 or not t.is_cuda:
        raise ValueError(f"{name}: expected a float32 CUDA tensor of shape (n, {cols})")
    return t.contiguous()


class VoxelTable:
    """The device voxel table of one cloud (voxel_downsample, prior_map.py:169-203): insert the cloud in chunks of
    at most `chunk` points, then `emit` the per-voxel means. 2^slots_log2 slots of 88 bytes each."""

    def __init__(self, voxel: float, slots_log2: int = 27, chunk: int = 1 << 25, device=None):
        if not voxel > 0:
            raise ValueError("voxel must be positive")
        if not 10 <= slots_log2 <= 30:
            raise ValueError("slots_log2 must lie in [10, 30]")
        self.device = _device(device)
        self.voxel = float(voxel)
        self.chunk = int(chunk)
        cap = 1 << slots_log2
        d = self.device
        self.keys = torch.empty(cap, dtype=torch.int64, device=d)
        self.acc = torch.empty(cap * 8, dtype=torch.int64, device=d)
        self.first = torch.empty(cap, dtype=torch.int64, device=d)
        self.order = torch.empty(cap, dtype=torch.int32, device=d)
        self.slot_of_pt = torch.empty(self.chunk, dtype=torch.int32, device=d)
        self.tiles = torch.empty(self.chunk // VOXEL_TILE + 2, dtype=torch.int32, device=d)
        self.stats = torch.zeros(2, dtype=torch.int64, device=d)
        self.buf = _lib.VoxBuf(*(_lib.ptr(getattr(self, n)) for n in _lib.VoxBuf.PTRS), cap, self.chunk)
        self.points = 0
        self.clear()

    def clear(self, stream=None):
        """Start a new cloud."""
        _lib.call("lw_vox_clear", self.buf, _lib.stream_ptr(stream))
        self.points = 0

    def insert(self, xyz: torch.Tensor, intensity: torch.Tensor | None = None, rgb: torch.Tensor | None = None,
               stream=None):
        """Add points (xyz (n, 3) float32 CUDA; intensity (n,) and rgb (n, 3) optional, zero when absent)."""
        xyz = _rows(xyz, 3, "xyz")
        n = len(xyz)
        if intensity is not None:
            intensity = intensity.reshape(-1).contiguous()
            if intensity.dtype != torch.float32 or len(intensity) != n or not intensity.is_cuda:
                raise ValueError("intensity: expected n float32 CUDA values")
        if rgb is not None:
            rgb = _rows(rgb, 3, "rgb")
            if len(rgb) != n:
                raise ValueError("rgb: expected n rows")
        for a in range(0, n, self.chunk):
            b = min(n, a + self.chunk)
            _lib.call("lw_vox_insert", self.buf, _lib.ptr(xyz[a:b]), 3,
                      _lib.ptr(intensity[a:b] if intensity is not None else None),
                      _lib.ptr(rgb[a:b] if rgb is not None else None), b - a, self.points + a, self.voxel,
                      _lib.stream_ptr(stream))
        self.points += n

    def totals(self) -> tuple[int, int]:
        """(voxels, points dropped because their probe window was full); synchronises."""
        v, drop = self.stats.tolist()
        return int(v), int(drop)

    def emit(self, stream=None, m: int | None = None):
        """The first m voxels (all by default): (xyz (m, 3), rgb (m, 3), intensity (m,), count (m,) int32) CUDA
        tensors, in the order of each voxel's first point."""
        if m is None:
            m, dropped = self.totals()
            if dropped:
                raise RuntimeError(f"voxel table full: {dropped} points dropped; raise slots_log2")
        d = self.device
        xyz = torch.empty((m, 3), dtype=torch.float32, device=d)
        rgb = torch.empty((m, 3), dtype=torch.float32, device=d)
        inten = torch.empty(m, dtype=torch.float32, device=d)
        cnt = torch.empty(m, dtype=torch.int32, device=d)
        _lib.call("lw_vox_emit", self.buf, self.voxel, m, _lib.ptr(xyz), _lib.ptr(rgb), _lib.ptr(inten),
                  _lib.ptr(cnt), _lib.stream_ptr(stream))
        return xyz, rgb, inten, cnt


class NormalBuffers:
    """Scratch of `lw_normals` for up to pt_cap points (the cell table twice as large, rounded to a power of two);
    reused across calls of the same or smaller size."""

    def __init__(self, pt_cap: int, device=None):
        self.device = _device(device)
        self.pt_cap = max(int(pt_cap), 1)
        cap = 1024
        while cap < 2 * self.pt_cap:
            cap *= 2
        d = self.device
        self.keys = torch.empty(cap, dtype=torch.int64, device=d)
        self.cell_cnt = torch.empty(cap, dtype=torch.int32, device=d)
        self.cell_start = torch.empty(cap, dtype=torch.int32, device=d)
        self.slot_of_pt = torch.empty(self.pt_cap, dtype=torch.int32, device=d)
        self.rank_of_pt = torch.empty(self.pt_cap, dtype=torch.int32, device=d)
        self.sorted = torch.empty(self.pt_cap * 4, dtype=torch.float32, device=d)
        self.tiles = torch.empty(cap // VOXEL_TILE + 2, dtype=torch.int32, device=d)
        self.stats = torch.zeros(2, dtype=torch.int32, device=d)
        self.buf = _lib.PcaBuf(*(_lib.ptr(getattr(self, n)) for n in _lib.PcaBuf.PTRS), cap, self.pt_cap)

    def dropped(self) -> int:
        return int(self.stats[1].item())


def normals_device(xyz: torch.Tensor, radius: float, stream=None, bufs: NormalBuffers | None = None):
    """PCA normal and planarity of every point of xyz ((n, 3) float32 CUDA) from its neighbours within `radius`
    (k_normals, prior_map.py:126-166): (normal (n, 3), planarity (n,)) CUDA tensors. Points with fewer than 4
    neighbours (themselves included) get a zero normal and planarity; the normals' sign is the decomposition's."""
    xyz = _rows(xyz, 3, "xyz")
    n = len(xyz)
    if bufs is None or bufs.pt_cap < n:
        bufs = NormalBuffers(n, xyz.device)
    nrm = torch.empty((n, 3), dtype=torch.float32, device=xyz.device)
    pl = torch.empty(n, dtype=torch.float32, device=xyz.device)
    _lib.call("lw_normals", _lib.ptr(xyz), 3, n, float(radius), bufs.buf, _lib.ptr(nrm), _lib.ptr(pl),
              _lib.stream_ptr(stream))
    return nrm, pl


def voxel_downsample(xyz: np.ndarray, intensity: np.ndarray | None, rgb: np.ndarray | None, voxel: float,
                     device=None, chunk: int = 1 << 25, slots_log2: int = 27):
    """Mean position / colour / intensity per voxel of a (huge) host cloud, on the GPU in chunks
    (prior_map.py:169-203). Returns numpy (xyz, rgb, intensity, count) per voxel, in the order of each voxel's
    first point; raises when the table overflows, as the reference does."""
    xyz = np.asarray(xyz, dtype=np.float32).reshape(-1, 3)
    table = VoxelTable(voxel, slots_log2, chunk, device)
    d = table.device
    n = len(xyz)
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        px = torch.from_numpy(np.ascontiguousarray(xyz[a:b])).to(d)
        pi = None if intensity is None else torch.from_numpy(
            np.ascontiguousarray(np.asarray(intensity, np.float32).reshape(-1)[a:b])).to(d)
        pc = None if rgb is None else torch.from_numpy(
            np.ascontiguousarray(np.asarray(rgb, np.float32).reshape(-1, 3)[a:b])).to(d)
        table.insert(px, pi, pc)
    vx, vc, vi, vn = table.emit()
    return vx.cpu().numpy(), vc.cpu().numpy(), vi.cpu().numpy(), vn.cpu().numpy()


def normals(xyz: np.ndarray, radius: float, device=None):
    """PCA normal and planarity of every point of a host cloud (prior_map.py:206-219): numpy (normal, planarity)."""
    d = _device(device)
    x = torch.from_numpy(np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)).to(d)
    nrm, pl = normals_device(x, radius)
    return nrm.cpu().numpy(), pl.cpu().numpy()


def from_points(xyz: np.ndarray, voxel: float = 0.02, normal_radius: float = 0.08, device=None,
                slots_log2: int = 24, stations=None) -> dict:
    """A prior map from a world point cloud (prior_map.py:358-370): voxel means, normals, planarity, counts and
    the stations if given (no colour). The voxel means stay on the device between the two steps."""
    xyz = np.asarray(xyz, dtype=np.float32).reshape(-1, 3)
    table = VoxelTable(voxel, slots_log2, min(1 << 25, max(len(xyz), 1)), device)
    table.insert(torch.from_numpy(np.ascontiguousarray(xyz)).to(table.device))
    vx, _, _, vn = table.emit()
    nrm, pl = normals_device(vx, normal_radius)
    return {"xyz": vx.cpu().numpy(), "normal": nrm.cpu().numpy(), "planarity": pl.cpu().numpy(),
            "count": vn.cpu().numpy(), "voxel": np.float32(voxel), "normal_radius": np.float32(normal_radius),
            "stations": np.zeros((0, 3), np.float32) if stations is None else np.asarray(stations, np.float32)}


def load(path: str) -> dict:
    """A prior-map cache (.npz) as a dict of its arrays (prior_map.py:352-356)."""
    z = np.load(path)
    return {k: z[k] for k in z.files}
