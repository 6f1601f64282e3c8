"""GPU state of one viewer on a B200: pose table, integration voxel map, free-space carving and the map's
visible set -- the `livox_warp.gpu` module of the reference (python/livox_warp/gpu.py), with the Warp kernels
replaced by the sm_100a library `liblivoxb200.so` (include/livox_b200.h).

Same public names and signatures as the reference's Pipeline (gpu.py:1163-1620): stage, ingest_ring,
map_insert, carve, set_pose / set_pose_range / flush_poses, clear_map, build, load_points, export and
export_labels, the View struct and the constants. Buffers are torch CUDA tensors; the library never allocates.

Differences from the reference, all deliberate:
  - map_acc holds exact int64 fixed-point sums (units FIX_W per metre, reflectivity in units of 1) instead of
    float32 sums of undefined order: every run gives the same map, bit for bit (map_centroids() decodes it);
  - the first 4096 hits of a voxel in point order are summed (the reference sums whichever 4096 arrive first);
  - build() compacts either the map's voxels (k_classify_map, slot order) or the live ring's points
    (k_classify_live, ring order); the render-side shading passes are outside this library's scope.
"""

from __future__ import annotations

import ctypes as C
import threading
import time

import numpy as np
import torch

from . import _lib
from ._lib import View  # noqa: F401  (gpu.View of the reference)

POSE_SLOTS = _lib.POSE_SLOTS
POSE_MASK = POSE_SLOTS - 1
MAP_COUNT_CAP = _lib.MAP_CAP
MAX_CLUSTERS = 4096
VOXEL_KEY_BITS = 21
VOXEL_KEY_BIAS = 1 << (VOXEL_KEY_BITS - 1)
VOXEL_KEY_MASK = (1 << VOXEL_KEY_BITS) - 1
HASH_MULTIPLIER = -7046029254386353131  # 0x9E3779B97F4A7C15 as a signed 64-bit value (gpu.py:63-64)
FIX_W = _lib.FIX_W


def voxel_key_ijk(ix, iy, iz):
    """Pack voxel indices into int64 keys (gpu.py:231-239); numpy arrays or ints."""
    ix, iy, iz = (np.asarray(v, dtype=np.int64) for v in (ix, iy, iz))
    b, m = np.int64(VOXEL_KEY_BIAS), np.int64(VOXEL_KEY_MASK)
    return ((ix + b) & m) | (((iy + b) & m) << np.int64(21)) | (((iz + b) & m) << np.int64(42))


def key_to_ijk(keys):
    k = np.asarray(keys, dtype=np.int64)
    m = np.int64(VOXEL_KEY_MASK)
    return ((k & m) - VOXEL_KEY_BIAS, ((k >> 21) & m) - VOXEL_KEY_BIAS, ((k >> 42) & m) - VOXEL_KEY_BIAS)


def mount_matrix(roll: float, pitch: float, yaw: float, x: float, y: float, z: float) -> np.ndarray:
    """Livox extrinsic convention (gpu.py:1113-1123): rotate about x, then y, then z; degrees, metres."""
    r, p, w = np.radians([roll, pitch, yaw])
    cx, sx, cy, sy, cz, sz = np.cos(r), np.sin(r), np.cos(p), np.sin(p), np.cos(w), np.sin(w)
    rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    m = np.eye(4)
    m[:3, :3] = rz @ ry @ rx
    m[:3, 3] = (x, y, z)
    return m.astype(np.float32)


def make_view(now: float = 0.0, persist: float = 0.0, voxel: float = 0.05, map_cap: int = 1 << 20, **kw) -> View:
    """A View with permissive defaults (everything in range, no crop); any field by keyword."""
    v = View()
    v.now, v.persist = float(now), float(persist)
    v.min_range, v.max_range, v.min_refl = 0.1, 500.0, 0
    v.noise_mask, v.ret_mask, v.crop_on = 0b1111, 0b1111, 0
    v.crop_lo, v.crop_hi = (-1e9, -1e9, -1e9), (1e9, 1e9, 1e9)
    v.inv_voxel, v.map_mask = 1.0 / voxel, map_cap - 1
    v.carve_ratio, v.carve_min, v.carve_stale = 2.0, 3, 1.0
    for name, value in kw.items():
        setattr(v, name, value)
    return v


SAMPLE_N = 1 << 16  # points the visible-set statistics sample (gpu.py:1243)


def strided_sample(x: torch.Tensor, count: int, m: int = SAMPLE_N) -> torch.Tensor:
    """Every stride-th of the first `count` rows of x, at most m of them, stride = max(1, count // m)
    (Pipeline._sample_stride and k_gather_*, gpu.py:1029-1049, 1575-1579)."""
    stride = max(1, count // m)
    k = min(m, (count + stride - 1) // stride)
    return x[:count:stride][:k]


def rebase_times(keys: torch.Tensor, first: torch.Tensor, last: torch.Tensor, shift: float):
    """k_rebase_clock (gpu.py:330-337): the occupied voxels' first / last-seen times onto a restarted clock,
    new = old - shift in float32; empty slots keep theirs."""
    occ = keys != -1
    s = torch.tensor(shift, dtype=first.dtype, device=first.device)
    first.copy_(torch.where(occ, first - s, first))
    last.copy_(torch.where(occ, last - s, last))


def row_stride(x: torch.Tensor) -> int:
    """Floats from one point to the next of an (n, 3) or (n, 4) float32 point array; 0 when the kernels cannot
    read it as it is (rows must be 3 or 4 floats apart, at least as wide as a row, columns adjacent)."""
    if x.dtype != torch.float32 or x.dim() != 2 or x.shape[1] not in (3, 4):
        return 0
    if x.shape[0] <= 1:  # a single row's stride is not meaningful
        return int(x.shape[1]) if x.shape[0] == 0 or x.stride(1) == 1 else 0
    s = int(x.stride(0))
    return s if x.stride(1) == 1 and s in (3, 4) and s >= x.shape[1] else 0


def _as_xyz(x, device) -> torch.Tensor:
    """Device float32 points of shape (n, 3) or (n, 4) (x, y, z, anything), contiguous, or the (n, 3) x, y, z
    columns of an (n, 4) buffer (rows 4 floats apart: the frame an on_frame callback is handed)."""
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 3))
    if row_stride(x) == 0:
        raise ValueError("points must be a float32 (n, 3) or (n, 4) array with rows of 3 or 4 floats")
    if x.device.type != "cuda":
        x = x.to(device, non_blocking=True)
        if row_stride(x) == 0:
            x = x.contiguous()
    return x


class Pipeline:
    """GPU state for one viewer: pose table, integration map, per-frame work arrays (gpu.py:1163).

    Threading as the reference: every launch goes to the calling thread's current stream; set_pose and
    set_pose_range only stage host-side edits under a lock and may be called from another thread; flush_poses,
    called by every reader, uploads them.
    """

    def __init__(self, ring_capacity: int = 1 << 23, map_capacity: int = 1 << 23, device=None,
                 nb_capacity: int = 1 << 22):
        _lib.load()
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise ValueError("Pipeline needs a CUDA device (there is no CPU fallback)")
        d = self.device
        self.cap = int(ring_capacity)
        self.map_cap = int(map_capacity)
        for name, cap in (("map_capacity", self.map_cap), ("nb_capacity", int(nb_capacity))):
            if cap <= 0 or cap & (cap - 1):
                raise ValueError(f"{name} must be a power of two, got {cap}")
        self.nb_cap = int(nb_capacity)
        self.work_cap = max(self.cap, self.map_cap)

        # live ring: the points of the last ring_capacity returns, drawn by build(map_on=False)
        self.ring_xyz = torch.zeros((self.cap, 3), dtype=torch.float32, device=d)
        self.ring_attr = torch.zeros(self.cap, dtype=torch.int32, device=d)
        self.ring_t = torch.zeros(self.cap, dtype=torch.float32, device=d)
        self.ring_frame = torch.zeros(self.cap, dtype=torch.int32, device=d)
        self.head = 0
        self.filled = 0

        # pose table: frame id -> sensor-to-world pose and body twist, with owner frame / epoch tags
        self.poses = torch.zeros((POSE_SLOTS, 16), dtype=torch.float32, device=d)
        self.tw = torch.zeros((POSE_SLOTS, 6), dtype=torch.float32, device=d)
        self.owner_frame = torch.full((POSE_SLOTS,), -1, dtype=torch.int32, device=d)
        self.owner_epoch = torch.full((POSE_SLOTS,), -1, dtype=torch.int32, device=d)
        self._pose_host = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (POSE_SLOTS, 1))
        self._tw_host = np.zeros((POSE_SLOTS, 6), np.float32)
        self._own_host = np.full((POSE_SLOTS, 2), -1, np.int32)
        self._pose_dirty: set[int] = set()
        self._pose_lock = threading.Lock()
        self.epoch = 0
        self.pose_table = _lib.PoseTable(_lib.ptr(self.poses).value, _lib.ptr(self.tw).value,
                                         _lib.ptr(self.owner_frame).value, _lib.ptr(self.owner_epoch).value)
        self.set_pose(0, np.eye(4, dtype=np.float32))
        self.flush_poses()

        # integration map
        m = self.map_cap
        self.map_keys = torch.full((m,), -1, dtype=torch.int64, device=d)
        self.map_cnt = torch.zeros(m, dtype=torch.int32, device=d)
        self.map_acc = torch.zeros((m, 4), dtype=torch.int64, device=d)
        self.map_last = torch.zeros(m, dtype=torch.float32, device=d)
        self.map_first = torch.full((m,), 1.0e30, dtype=torch.float32, device=d)
        self.map_miss = torch.zeros(m, dtype=torch.int32, device=d)
        self._map_bcnt = torch.zeros(m, dtype=torch.int32, device=d)
        self._map_lead = torch.full((m,), _lib.INT32_MAX, dtype=torch.int32, device=d)
        self.map_stats = torch.zeros(2, dtype=torch.int32, device=d)
        self.map_struct = _lib.Map(*(_lib.ptr(t).value for t in (
            self.map_keys, self.map_cnt, self.map_acc, self.map_last, self.map_first, self.map_miss, self._map_bcnt,
            self._map_lead, self.map_stats)), m)

        # visible set and per-point labels
        n = self.work_cap
        self.c_xyz = torch.zeros((n, 3), dtype=torch.float32, device=d)
        self.c_attr = torch.zeros(n, dtype=torch.int32, device=d)
        self.c_t = torch.zeros(n, dtype=torch.float32, device=d)
        self.c_dyn = torch.zeros(n, dtype=torch.int32, device=d)
        self.nrm = torch.zeros((n, 3), dtype=torch.float32, device=d)
        self.nbr = torch.zeros(n, dtype=torch.int32, device=d)  # point-weighted neighbour counts
        self.curv = torch.zeros(n, dtype=torch.float32, device=d)
        self._nb = None  # the neighbourhood pass's buffers, made on first use
        self.gnd = torch.zeros(n, dtype=torch.int32, device=d)
        self.hag = torch.zeros(n, dtype=torch.float32, device=d)
        self.cid = torch.full((n,), -1, dtype=torch.int32, device=d)
        self.cl_vel = torch.zeros((MAX_CLUSTERS, 3), dtype=torch.float32, device=d)
        self.cl_tid = torch.full((MAX_CLUSTERS,), -1, dtype=torch.int32, device=d)
        self._slot = torch.zeros(n, dtype=torch.int32, device=d)  # per-point scratch of the insert passes
        self._tiles = torch.zeros(max(m, self.cap) // 1024 + 2, dtype=torch.int32, device=d)
        self.total = torch.zeros(1, dtype=torch.int32, device=d)

        self._stage_cap = 0
        self._stage_xyz = self._stage_attr = self._stage_t = self._stage_frame = None
        self._pin_xyz = self._pin_attr = self._pin_t = None
        self._pin_ev = None
        self.count = 0
        self.normals_valid = False
        self.map_occupied = 0
        self.map_dropped = 0
        self.ms = {"ingest": 0.0, "build": 0.0, "neighbors": 0.0, "shade": 0.0, "carve": 0.0}

    # ---- memory ---------------------------------------------------------------------------------------------

    def gpu_bytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in vars(self).values()
                   if isinstance(t, torch.Tensor) and t.device.type == "cuda")

    def _ensure_stage(self, n: int):
        if n <= self._stage_cap:
            return
        cap = max(n, 1 << 16, self._stage_cap * 2)
        d = self.device
        self._stage_xyz = torch.empty((cap, 3), dtype=torch.float32, device=d)
        self._stage_attr = torch.empty(cap, dtype=torch.int32, device=d)
        self._stage_t = torch.empty(cap, dtype=torch.float32, device=d)
        self._stage_frame = torch.empty(cap, dtype=torch.int32, device=d)
        self._pin_xyz = torch.empty((cap, 3), dtype=torch.float32, pin_memory=True)
        self._pin_attr = torch.empty(cap, dtype=torch.int32, pin_memory=True)
        self._pin_t = torch.empty(cap, dtype=torch.float32, pin_memory=True)
        self._stage_cap = cap

    def clear_live(self):
        self.head = 0
        self.filled = 0

    def clear_map(self):
        _lib.call("lw_map_clear", C_ref(self.map_struct), _lib.stream_ptr())
        self.map_occupied = self.map_dropped = 0

    def rebase_clock(self, shift: float):
        """The live clock restarted (replay loop, sensor reboot): move the map's first / last-seen times onto the new
        clock, new = old - shift, so persistence, Motion labels and ghosts keep working (gpu.py:1368-1372)."""
        rebase_times(self.map_keys, self.map_first, self.map_last, float(shift))

    # ---- poses ----------------------------------------------------------------------------------------------

    def set_pose(self, frame: int, mat: np.ndarray, twist=None, epoch: int = 0):
        """Sensor-to-world matrix and body twist (rho, theta) of one frame id for `epoch`; applied at the next
        flush_poses(), which every reader calls first (gpu.py:1317-1328)."""
        j = frame & POSE_MASK
        m = np.asarray(mat, dtype=np.float32).reshape(16)
        tw = np.zeros(6, np.float32) if twist is None else np.asarray(twist, dtype=np.float32)
        with self._pose_lock:
            self._pose_host[j] = m
            self._tw_host[j] = tw
            self._own_host[j] = (frame, epoch)
            self._pose_dirty.add(j)

    def set_pose_range(self, k0: int, k1: int, mat: np.ndarray, twist=None, epoch: int = 0):
        """The same pose for frames k0 .. k1-1 (gpu.py:1330-1344)."""
        if k1 <= k0:
            return
        k0 = max(k0, k1 - POSE_SLOTS)
        ks = np.arange(k0, k1, dtype=np.int64)
        js = ks & POSE_MASK
        m = np.asarray(mat, dtype=np.float32).reshape(16)
        tw = np.zeros(6, np.float32) if twist is None else np.asarray(twist, dtype=np.float32)
        with self._pose_lock:
            self._pose_host[js] = m
            self._tw_host[js] = tw
            self._own_host[js, 0] = ks.astype(np.int32)
            self._own_host[js, 1] = epoch
            self._pose_dirty.update(js.tolist())

    def flush_poses(self):
        """Upload every pose edited on the host since the last flush (gpu.py:1346-1366)."""
        with self._pose_lock:
            if not self._pose_dirty:
                return
            idx = np.fromiter(self._pose_dirty, dtype=np.int64, count=len(self._pose_dirty))
            self._pose_dirty.clear()
            mats, tws, own = self._pose_host[idx].copy(), self._tw_host[idx].copy(), self._own_host[idx].copy()
        d = self.device
        i = torch.from_numpy(idx).to(d)
        self.poses.index_copy_(0, i, torch.from_numpy(mats).to(d))
        self.tw.index_copy_(0, i, torch.from_numpy(tws).to(d))
        self.owner_frame.index_copy_(0, i, torch.from_numpy(np.ascontiguousarray(own[:, 0])).to(d))
        self.owner_epoch.index_copy_(0, i, torch.from_numpy(np.ascontiguousarray(own[:, 1])).to(d))

    # ---- per batch ------------------------------------------------------------------------------------------

    def stage(self, xyz, attr, t, n: int, inv_frame_dt: float = 0.0):
        """Put a batch on the GPU (or accept device tensors) and compute its frame ids (gpu.py:1376-1401).
        Returns (xyz, attr, t, frame) device tensors valid until the next stage() call."""
        s = torch.cuda.current_stream()
        if isinstance(xyz, np.ndarray):
            if self._pin_ev is not None:
                self._pin_ev.synchronize()  # the previous batch's copy may still read the pinned buffers
            self._ensure_stage(n)
            self._pin_xyz.numpy()[:n] = np.asarray(xyz, dtype=np.float32).reshape(-1, 3)[:n]
            self._pin_attr.numpy()[:n] = np.asarray(attr)[:n].view(np.int32)
            self._pin_t.numpy()[:n] = np.asarray(t, dtype=np.float32)[:n]
            sx, sa, st, sf = self._stage_xyz, self._stage_attr, self._stage_t, self._stage_frame
            # the three copies and the frame ids in one call
            _lib.call("lw_stage_batch", _lib.ptr(self._pin_xyz), _lib.ptr(self._pin_attr), _lib.ptr(self._pin_t), n,
                      _lib.ptr(sx), _lib.ptr(sa), _lib.ptr(st), float(inv_frame_dt), _lib.ptr(sf), _lib.stream_ptr(s))
            if self._pin_ev is None:
                self._pin_ev = torch.cuda.Event()
            self._pin_ev.record(s)
            return sx, sa, st, sf
        else:
            self._ensure_stage(n)
            sx, sa, st = _as_xyz(xyz, self.device), attr, t
        sf = self._stage_frame
        _lib.call("lw_frame_ids", _lib.ptr(st), n, float(inv_frame_dt), _lib.ptr(sf), _lib.stream_ptr(s))
        return sx, sa, st, sf

    def ingest_ring(self, sx, sa, st, sf, n: int):
        """Append staged points to the live ring (gpu.py:1403-1419)."""
        if n <= 0:
            return
        keep = min(n, self.cap)
        off = n - keep
        idx = (torch.arange(keep, device=self.device) + self.head) % self.cap
        self.ring_xyz.index_copy_(0, idx, sx[off:n, :3])
        self.ring_attr.index_copy_(0, idx, sa[off:n].view(torch.int32))
        self.ring_t.index_copy_(0, idx, st[off:n])
        self.ring_frame.index_copy_(0, idx, sf[off:n])
        self.head = (self.head + keep) % self.cap
        self.filled = min(self.filled + keep, self.cap)

    def _scratch(self, n: int) -> torch.Tensor:
        if n > self._slot.numel():
            self._slot = torch.zeros(n, dtype=torch.int32, device=self.device)
        return self._slot

    def map_insert(self, sx, sa, st, sf, n, view: View, voxel: float, n_dev: torch.Tensor | None = None):
        """Accumulate staged points into the integration map through their frames' poses (gpu.py:1421-1434).
        `n` is the point count, or an upper bound when the count lives on the device (`n_dev`)."""
        n = int(n)
        if n <= 0:
            return
        self.flush_poses()
        sx = _as_xyz(sx, self.device)
        _lib.call("lw_map_insert", _lib.ptr(sx), row_stride(sx), _lib.ptr(sa), _lib.ptr(st), _lib.ptr(sf),
                  _lib.ptr(n_dev), n, _lib.ptr(self.poses), C_ref(view), 1.0 / max(voxel, 1e-4),
                  C_ref(self.map_struct), _lib.ptr(self._scratch(n)), _lib.stream_ptr())

    def carve(self, sx, sa, sf, n, voxel: float, every: int = 2, max_range: float = 40.0, max_steps: int = 4096,
              n_dev: torch.Tensor | None = None):
        """Free-space carving: count the map voxels each traced ray pierces (gpu.py:1436-1452)."""
        n = int(n)
        if n <= 0:
            return
        self.flush_poses()
        sx = _as_xyz(sx, self.device)
        _lib.call("lw_carve", _lib.ptr(sx), row_stride(sx), _lib.ptr(sa), _lib.ptr(sf), _lib.ptr(n_dev), n,
                  _lib.ptr(self.poses), max(1, int(every)), 1.0 / max(voxel, 1e-4), float(max_range), int(max_steps),
                  C_ref(self.map_struct), _lib.ptr(self._scratch(n)), _lib.stream_ptr())

    def ingest(self, xyz, attr, t, n: int, view: View, map_on: bool, voxel: float):
        """Stage, ring and map in one call, without odometry (gpu.py:1454-1462)."""
        if n <= 0:
            return
        sx, sa, st, sf = self.stage(xyz, attr, t, n, 0.0)
        self.ingest_ring(sx, sa, st, sf, n)
        if map_on:
            self.map_insert(sx, sa, st, sf, n, view, voxel)

    # ---- per frame ------------------------------------------------------------------------------------------

    def build(self, view: View, map_on: bool = True, min_count: int = 1, neighbors: str = "", radius: float = 0.1,
              sensor=(0.0, 0.0, 0.0)) -> int:
        """Classify + compact the visible set into c_* (gpu.py:1466-1512): with map_on the map's voxels in slot
        order (k_classify_map), else the live ring's points in ring order (k_classify_live)."""
        if neighbors not in ("", "count", "normals"):
            raise ValueError(f"neighbors must be '', 'count' or 'normals', got {neighbors!r}")
        self.flush_poses()
        if map_on:
            _lib.call("lw_map_build", C_ref(self.map_struct), C_ref(view), int(min_count), _lib.ptr(self.c_xyz),
                      _lib.ptr(self.c_attr), _lib.ptr(self.c_t), _lib.ptr(self.c_dyn), _lib.ptr(self._tiles),
                      _lib.ptr(self.total), _lib.stream_ptr())
        else:
            _lib.call("lw_live_build", _lib.ptr(self.ring_xyz), _lib.ptr(self.ring_attr), _lib.ptr(self.ring_t),
                      _lib.ptr(self.ring_frame), self.cap, self.filled, C_ref(self.pose_table), C_ref(view),
                      C_ref(self.map_struct), _lib.ptr(self.c_xyz), _lib.ptr(self.c_attr), _lib.ptr(self.c_t),
                      _lib.ptr(self.c_dyn), _lib.ptr(self._tiles), _lib.ptr(self.total), _lib.stream_ptr())
        host = torch.cat([self.total, self.map_stats]).cpu().numpy()  # the frame's one host sync
        self.count = int(host[0])
        if map_on:
            self.map_occupied, self.map_dropped = int(host[1]), int(host[2])
        self.normals_valid = False
        if neighbors:
            self.neighborhoods(float(radius), neighbors == "normals", sensor)
        return self.count

    def neighborhoods(self, radius: float, want_normals: bool, sensor):
        """Fill nbr (and nrm / curv) for the visible points from a voxel summary a third of `radius` wide
        (gpu.py:1531-1557); build() calls it when asked for neighbours, and it serves load_points() sets too."""
        n = self.count
        if self._nb is None:
            d, cap = self.device, 1 << (2 * self.work_cap - 1).bit_length()
            self._nb_t = {"keys": torch.full((cap,), -1, dtype=torch.int64, device=d),
                          "acc": torch.zeros((cap, 4), dtype=torch.int64, device=d),
                          "vidx": torch.zeros(cap, dtype=torch.int32, device=d),
                          "v_slot": torch.zeros(cap, dtype=torch.int32, device=d),
                          "slot_of_pt": torch.zeros(self.work_cap, dtype=torch.int32, device=d),
                          "v_xyz": torch.zeros((cap, 3), dtype=torch.float32, device=d),
                          "v_w": torch.zeros(cap, dtype=torch.int32, device=d),
                          "v_cnt": torch.zeros(cap, dtype=torch.float32, device=d),
                          "v_nrm": torch.zeros((cap, 3), dtype=torch.float32, device=d),
                          "v_curv": torch.zeros(cap, dtype=torch.float32, device=d),
                          "tiles": torch.zeros(cap // 1024 + 2, dtype=torch.int32, device=d),
                          "m": torch.zeros(1, dtype=torch.int32, device=d)}
            self._nb = _lib.NbrBuf(*(_lib.ptr(self._nb_t[k]).value for k in _lib.NbrBuf.PTRS), cap, self.work_cap)
        t0 = time.perf_counter()
        sen = (C.c_float * 3)(*[float(v) for v in sensor])
        _lib.call("lw_neighborhoods", _lib.ptr(self.c_xyz), 3, None, int(n), float(radius), int(bool(want_normals)),
                  sen, C_ref(self._nb), _lib.ptr(self.nbr), _lib.ptr(self.nrm), _lib.ptr(self.curv),
                  _lib.stream_ptr())
        self.normals_valid = bool(want_normals)
        self.ms["neighbors"] = (time.perf_counter() - t0) * 1e3

    @property
    def nb_voxels(self) -> int:
        """Voxels of the last neighbourhood pass (gpu.py:1547); reading it synchronises the stream."""
        return 0 if self._nb is None else int(self._nb_t["m"].item())

    def load_points(self, xyz: np.ndarray):
        """Make an arbitrary world-frame point set the visible set (gpu.py:1522-1529)."""
        if isinstance(xyz, torch.Tensor):
            n = min(int(xyz.shape[0]), self.work_cap)
            self.c_xyz[:n].copy_(xyz[:n, :3])
        else:
            n = min(len(xyz), self.work_cap)
            self.c_xyz[:n].copy_(torch.from_numpy(np.ascontiguousarray(xyz[:n], dtype=np.float32)))
        self.count = n
        self.normals_valid = False

    def map_centroids(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(keys, centroids, counts) of every occupied map voxel, decoded from the fixed-point sums."""
        keys = self.map_keys.cpu().numpy()
        occ = keys != -1
        cnt = self.map_cnt.cpu().numpy()[occ]
        acc = self.map_acc.cpu().numpy()[occ]
        nsum = np.minimum(cnt, MAP_COUNT_CAP).astype(np.float64)
        cen = (acc[:, :3].astype(np.float64) / (nsum[:, None] * FIX_W)).astype(np.float32)
        return keys[occ], cen, cnt

    def floor_z(self) -> float | None:
        """A low (1st) percentile of the visible z, from a strided sample: where the floor usually is
        (gpu.py:1597-1600)."""
        if self.count == 0:
            return None
        z = strided_sample(self.c_xyz, self.count)[:, 2].cpu().numpy()
        z = z[np.isfinite(z)]
        return float(np.percentile(z, 1.0)) if z.size else None

    def bounds(self, lo_pct: float = 2.0, hi_pct: float = 98.0):
        """Robust (lo, hi) corners of the visible set from a strided sample (gpu.py:1602-1609)."""
        if self.count == 0:
            return None
        pts = strided_sample(self.c_xyz, self.count).cpu().numpy()
        return np.percentile(pts, lo_pct, axis=0), np.percentile(pts, hi_pct, axis=0)

    def export(self):
        n = self.count
        return self.c_xyz[:n].cpu().numpy(), self.c_attr[:n].cpu().numpy().view(np.uint32), self.c_t[:n].cpu().numpy()

    def export_labels(self):
        n = self.count
        return self.gnd[:n].cpu().numpy(), self.cid[:n].cpu().numpy()


def C_ref(struct):
    """ctypes byref of a boundary struct."""
    import ctypes

    return ctypes.byref(struct)
