"""CPU oracle of the livox-warp per-frame hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module, and only as the checker or
the timed CPU baseline; the product (livox-warp_b200/livox_warp) never imports it.

Two layers:
  * liblworacle.so (lw_oracle.cpp): the reference's Warp kernels restated as serial C++ -- keys and hashing,
    deskew, thinning, registration insert and per-voxel records, the ICP accumulation in float64, the
    integration insert, carving and the map's visible set;
  * this file: the host-side float64 Gauss-Newton step of odom.py (_sym6 :390-394, _twist_between :397-401,
    _apply_twist :404-409, _body_twist :412-414, _twist_matrix :417-422, _sensor_basis :425-433,
    _constrained_step :436-455, _register :752-803) and the frame state machine of Odometry
    (_finalize :642-657, _estimate :659-680, _update_velocity :682-694, _is_keyframe :712-717), written with
    numpy and scipy exactly as the reference's host code is -- so the pose oracle is float64 end to end.

The prior-map grid and the batched localisation ICP (mapgrid.py, localize.py) follow at the end of this file:
prepare (mapgrid.py:216-243) in numpy, the kernels in lw_oracle.cpp, the ICP's terms and solve in float64.

Parity of the kernel restatement against the reference is unpinned (NVIDIA Warp is not installed here and the
reference ships no golden vectors for its kernels); the host step is pinned against the reference's own
functions through tests/golden/host_solve.npz (see tests/golden/make_golden.py).
"""

from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path

import numpy as np
from scipy.spatial.transform import Rotation

HERE = Path(__file__).resolve().parent
LIB = HERE / "liblworacle.so"

FIX_R, FIX_RR, FIX_W = 2.0 ** 32, 2.0 ** 40, 2.0 ** 20
POSE_SLOTS = 1 << 16
ACC_H, ACC_B, ACC_COUNT, ACC_ERR, ACC_RMS, ACC_WEIGHT, ACC_RANGE, ACC_HG = 0, 21, 27, 28, 29, 30, 31, 32
WIDE_ITERS = 3
KAPPA_START, KAPPA_DECAY, KAPPA_MIN = 6.0, 0.7, 2.0
STEP_TOL = 1e-4
TIGHT_FRACTION = 0.6
WEAK_COND = 1e-3
REDESKEW_ROT, REDESKEW_TRANS = 2e-3, 5e-3
MAX_FRAME_JUMP = 1.5

_lib = None


class OrGrid(C.Structure):
    _fields_ = [("xyz", C.c_void_p), ("nrm", C.c_void_p), ("planar", C.c_void_p), ("start", C.c_void_p),
                ("nn", C.c_void_p), ("origin", C.c_float * 3), ("cell", C.c_float), ("inv_cell", C.c_float),
                ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("pad_", C.c_int32)]


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        # the OpenMP runtime reads these when the library loads: never spin-wait on a shared host
        os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")
        os.environ.setdefault("GOMP_SPINCOUNT", "0")
        if not LIB.exists():
            import importlib.util
            spec = importlib.util.spec_from_file_location("lw_oracle_build", HERE / "build.py")
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            mod.build()
        _lib = C.CDLL(str(LIB))
        P = C.c_void_p
        i64, i32, f32, f64 = C.c_int64, C.c_int32, C.c_float, C.c_double
        sig = {
            "or_key_ijk": (i64, [i32, i32, i32]),
            "or_slot_hash": (i32, [i64]),
            "or_voxel_keys": (None, [P, i64, f32, P]),
            "or_deskew": (None, [P, i64, f32, f32, P, P]),
            "or_thin": (i64, [P, P, i64, f32, f32, f32, i32, P]),
            "or_reg_insert": (None, [P, P, i64, P, f32, f32, f32, i32, i64, P, P, P, P, P]),
            "or_reg_records": (None, [i64, P, P, P, P, f32, f32, f32, f32, P]),
            "or_icp_accumulate": (None, [P, i64, P, i64, P, P, f64, i32, f64, f64, i32, P]),
            "or_map_insert": (None, [P, i32, P, P, P, i64, P, P, f32, i64, P, P, P, P, P, P]),
            "or_carve": (None, [P, i32, P, P, i64, P, i32, f32, f32, i32, i64, P, P, P, P, i32]),
            "or_map_build": (i64, [i64, P, P, P, P, P, P, P, i32, P, P, P, P]),
            "or_live_build": (i64, [P, P, P, P, i64, i64, P, P, P, P, P, P, P, P, P, P, P, P, P]),
            "or_ground": (None, [P, i32, P, i64, f32, f32, i32, f32, f32, i32, f32, P, P]),
            "or_cluster": (i64, [P, i32, P, i32, i64, f32, f32, f32, i32, P, P, P, P, P, P, P, P]),
            "or_grid_build": (None, [C.POINTER(OrGrid), i64, P, P, i32]),
            "or_nearest": (None, [C.POINTER(OrGrid), P, i64, P, i32]),
            "or_prior_distances": (None, [C.POINTER(OrGrid), P, i64, P, P, i32]),
            "or_loc_icp": (None, [C.POINTER(OrGrid), P, P, P, i32, P, i32, P, P, P, f32, i32, P, P, i32]),
            "or_loc_eval": (None, [C.POINTER(OrGrid), P, P, P, i32, P, P, P, i32]),
            "or_neighborhoods": (None, [P, i32, i64, f32, i32, P, P, P, P, i32]),
            "or_score_grid": (None, [C.POINTER(OrGrid), P, P, i32, P, i64, i32, f32, f32, f32, f32, i32, P, i32]),
            "or_score_list": (None, [C.POINTER(OrGrid), P, P, i32, P, i64, f32, i32, P, i32]),
            "or_voxel_downsample": (i64, [P, i64, P, P, f32, P, P, P, P]),
            "or_normals": (None, [P, i64, f32, P, P, i32]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(_lib, name)
            fn.restype = res
            fn.argtypes = args
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be contiguous"
    return a.ctypes.data_as(C.c_void_p)


def host_cores() -> int:
    """CPUs this process may really use: its affinity set, capped by a cgroup CPU quota when one is set."""
    try:
        n = len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        n = os.cpu_count() or 1
    try:
        quota, period = open("/sys/fs/cgroup/cpu.max").read().split()[:2]
        if quota != "max":
            n = min(n, max(1, int(int(quota) // int(period))))
    except (OSError, ValueError):
        pass
    return max(1, n)


def threads() -> int:
    """OpenMP threads of the oracle: LW_ORACLE_THREADS, else the usable cores (at most 8)."""
    return int(os.environ.get("LW_ORACLE_THREADS", min(host_cores(), 8)))


# ---- kernels ------------------------------------------------------------------------------------------------


def voxel_keys(xyz: np.ndarray, inv: float) -> np.ndarray:
    xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
    out = np.empty(len(xyz), np.int64)
    lib().or_voxel_keys(_p(xyz), len(xyz), inv, _p(out))
    return out


def deskew(raw4: np.ndarray, t_mid: float, inv_dt: float, twist) -> np.ndarray:
    raw4 = np.ascontiguousarray(raw4, dtype=np.float32)
    out = np.empty_like(raw4)
    tw = np.ascontiguousarray(twist, dtype=np.float32)
    lib().or_deskew(_p(raw4), len(raw4), np.float32(t_mid), np.float32(inv_dt), _p(tw), _p(out))
    return out


def thin(xyz4: np.ndarray, attr: np.ndarray, inv_v: float, min_range: float, max_range: float, ret_mask: int):
    xyz4 = np.ascontiguousarray(xyz4, dtype=np.float32)
    attr = np.ascontiguousarray(attr, dtype=np.uint32)
    out = np.empty_like(xyz4)
    n = lib().or_thin(_p(xyz4), _p(attr), len(xyz4), inv_v, min_range, max_range, ret_mask, _p(out))
    return out[:n]


class RegMap:
    """The registration map as the oracle keeps it (same slot layout as the device tables)."""

    def __init__(self, cap: int):
        self.cap = cap
        self.keys = np.full(cap, -1, np.int64)
        self.cnt = np.zeros(cap, np.int32)
        self.sum = np.zeros((cap, 3), np.int64)
        self.outer = np.zeros((cap, 6), np.int64)
        self.stats = np.zeros(2, np.int32)
        self.rec = np.zeros((cap, 20), np.float32)

    def insert(self, xyz4, attr, T, voxel: float, max_range: float, ret_mask: int):
        xyz4 = np.ascontiguousarray(xyz4, dtype=np.float32)
        attr = np.ascontiguousarray(attr, dtype=np.uint32)
        T12 = np.ascontiguousarray(np.asarray(T, np.float64).reshape(4, 4)[:3].astype(np.float32))
        lib().or_reg_insert(_p(xyz4), _p(attr), len(xyz4), _p(T12), np.float32(1.0 / voxel), np.float32(voxel),
                            max_range, ret_mask, self.cap, _p(self.keys), _p(self.cnt), _p(self.sum),
                            _p(self.outer), _p(self.stats))

    def records(self, voxel: float, noise: float, alpha: float):
        tight2 = (TIGHT_FRACTION * voxel / math.sqrt(12.0)) ** 2
        lib().or_reg_records(self.cap, _p(self.keys), _p(self.cnt), _p(self.sum), _p(self.outer), voxel, tight2,
                             noise * noise, alpha, _p(self.rec))
        return self.rec

    def as_dict(self):
        occ = self.keys != -1
        return {int(k): (int(c), tuple(s), tuple(o)) for k, c, s, o in
                zip(self.keys[occ], self.cnt[occ], self.sum[occ], self.outer[occ])}


def icp_accumulate(ds4: np.ndarray, T: np.ndarray, reg: RegMap, voxel: float, reach: int, max_d2: float,
                   kappa: float, nthreads: int | None = None) -> np.ndarray:
    ds4 = np.ascontiguousarray(ds4, dtype=np.float32)
    T = np.ascontiguousarray(np.asarray(T, np.float64).reshape(16))
    out = np.zeros(64)
    lib().or_icp_accumulate(_p(ds4), len(ds4), _p(T), reg.cap, _p(reg.keys), _p(reg.rec), 1.0 / voxel, reach,
                            max_d2, kappa, nthreads or threads(), _p(out))
    return out


# ---- integration map -------------------------------------------------------------------------------------


class Map:
    def __init__(self, cap: int):
        self.cap = cap
        self.keys = np.full(cap, -1, np.int64)
        self.cnt = np.zeros(cap, np.int32)
        self.acc = np.zeros((cap, 4), np.int64)
        self.last = np.zeros(cap, np.float32)
        self.first = np.full(cap, 1.0e30, np.float32)
        self.miss = np.zeros(cap, np.int32)
        self.stats = np.zeros(2, np.int32)

    def insert(self, xyz, attr, t, frame, poses, view, voxel: float):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        stride = xyz.shape[1]
        attr = np.ascontiguousarray(attr, dtype=np.uint32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        frame = np.ascontiguousarray(frame, dtype=np.int32)
        poses = np.ascontiguousarray(poses, dtype=np.float32).reshape(POSE_SLOTS, 16)
        lib().or_map_insert(_p(xyz), stride, _p(attr), _p(t), _p(frame), len(t), _p(poses), C.byref(view),
                            np.float32(1.0 / max(voxel, 1e-4)), self.cap, _p(self.keys), _p(self.cnt), _p(self.acc),
                            _p(self.last), _p(self.first), _p(self.stats))

    def carve(self, xyz, attr, frame, poses, voxel, every=2, max_range=40.0, max_steps=4096, nthreads=None):
        xyz = np.ascontiguousarray(xyz, dtype=np.float32)
        attr = np.ascontiguousarray(attr, dtype=np.uint32)
        frame = np.ascontiguousarray(frame, dtype=np.int32)
        poses = np.ascontiguousarray(poses, dtype=np.float32).reshape(POSE_SLOTS, 16)
        lib().or_carve(_p(xyz), xyz.shape[1], _p(attr), _p(frame), len(frame), _p(poses), max(1, int(every)),
                       np.float32(1.0 / max(voxel, 1e-4)), max_range, max_steps, self.cap, _p(self.keys),
                       _p(self.cnt), _p(self.acc), _p(self.miss), nthreads or threads())

    def build(self, view, min_count: int = 1):
        n = self.cap
        xyz = np.zeros((n, 3), np.float32)
        attr = np.zeros(n, np.uint32)
        t = np.zeros(n, np.float32)
        dyn = np.zeros(n, np.int32)
        k = lib().or_map_build(self.cap, _p(self.keys), _p(self.cnt), _p(self.acc), _p(self.last), _p(self.first),
                               _p(self.miss), C.byref(view), min_count, _p(xyz), _p(attr), _p(t), _p(dyn))
        return xyz[:k], attr[:k], t[:k], dyn[:k]

    def live_build(self, ring_xyz, ring_attr, ring_t, ring_frame, filled, poses, tw, owner_frame, owner_epoch, view):
        """k_classify_live (gpu.py:637-697) over the first `filled` ring slots, in ring order, with this map's
        history for the Motion label: (xyz, attr, t, dyn)."""
        rx = np.ascontiguousarray(ring_xyz, dtype=np.float32).reshape(-1, 3)
        cap = len(rx)
        ra = np.ascontiguousarray(ring_attr).view(np.uint32).reshape(cap)
        rt = np.ascontiguousarray(ring_t, dtype=np.float32).reshape(cap)
        rf = np.ascontiguousarray(ring_frame, dtype=np.int32).reshape(cap)
        ps = np.ascontiguousarray(poses, dtype=np.float32).reshape(POSE_SLOTS, 16)
        tws = np.ascontiguousarray(tw, dtype=np.float32).reshape(POSE_SLOTS, 6)
        of = np.ascontiguousarray(owner_frame, dtype=np.int32).reshape(POSE_SLOTS)
        oe = np.ascontiguousarray(owner_epoch, dtype=np.int32).reshape(POSE_SLOTS)
        xyz = np.zeros((cap, 3), np.float32)
        attr = np.zeros(cap, np.uint32)
        t = np.zeros(cap, np.float32)
        dyn = np.zeros(cap, np.int32)
        k = lib().or_live_build(_p(rx), _p(ra), _p(rt), _p(rf), cap, int(filled), _p(ps), _p(tws), _p(of), _p(oe),
                                C.byref(view), _p(self.keys), _p(self.cnt), _p(self.first), _p(self.miss), _p(xyz),
                                _p(attr), _p(t), _p(dyn))
        return xyz[:k], attr[:k], t[:k], dyn[:k]

    def as_dict(self):
        occ = self.keys != -1
        return {int(k): (int(c), tuple(a), float(l), float(f), int(m)) for k, c, a, l, f, m in
                zip(self.keys[occ], self.cnt[occ], self.acc[occ], self.last[occ], self.first[occ], self.miss[occ])}


# ---- perception ---------------------------------------------------------------------------------------------


def ground(xyz, cell=0.5, thick=0.15, min_sup=3, thresh=0.2, slope_step=0.3, nrm=None, nz_min=0.7):
    """perception.py:29-111: (gnd int32, hag float32) per point."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    n = len(xyz)
    gnd = np.zeros(n, np.int32)
    hag = np.zeros(n, np.float32)
    nrm_a = None if nrm is None else np.ascontiguousarray(nrm, dtype=np.float32)
    lib().or_ground(_p(xyz), xyz.shape[1], None if nrm_a is None else _p(nrm_a), n, cell, thick, min_sup, thresh,
                    slope_step, int(nrm_a is not None), nz_min, _p(gnd), _p(hag))
    return gnd, hag


def neighborhoods(xyz, radius: float, want_normals: bool, sensor=(0.0, 0.0, 0.0)):
    """gpu.py:777-905 as the library defines it (exact voxel sums, neighbours among the 7^3 voxel offsets):
    (count int32 [n], normal [n, 3], curvature [n])."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
    n = len(xyz)
    cnt = np.zeros(n, np.int32)
    nrm = np.zeros((n, 3), np.float32)
    curv = np.zeros(n, np.float32)
    sen = np.ascontiguousarray(sensor, dtype=np.float32)
    lib().or_neighborhoods(_p(xyz), 3, n, float(radius), int(bool(want_normals)), _p(sen), _p(cnt), _p(nrm),
                           _p(curv), threads())
    return cnt, nrm, curv


def voxel_downsample(xyz, intensity=None, rgb=None, voxel: float = 0.02):
    """prior_map.py:57-123, 169-203 as the library defines it (exact fixed-point sums, voxels in the order of their
    first point): (xyz [m, 3], rgb [m, 3], intensity [m], count int32 [m])."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
    n = len(xyz)
    it = None if intensity is None else np.ascontiguousarray(intensity, dtype=np.float32).reshape(n)
    col = None if rgb is None else np.ascontiguousarray(rgb, dtype=np.float32).reshape(n, 3)
    ox = np.zeros((n, 3), np.float32)
    oc = np.zeros((n, 3), np.float32)
    oi = np.zeros(n, np.float32)
    on = np.zeros(n, np.int32)
    m = lib().or_voxel_downsample(_p(xyz), n, None if it is None else _p(it), None if col is None else _p(col),
                                  float(voxel), _p(ox), _p(oc), _p(oi), _p(on))
    return ox[:m], oc[:m], oi[:m], on[:m]


def normals(xyz, radius: float):
    """prior_map.py:126-166 as the library defines it (every point within the radius, fixed-point sums, float64
    Jacobi): (normal [n, 3], planarity [n])."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
    n = len(xyz)
    nrm = np.zeros((n, 3), np.float32)
    pl = np.zeros(n, np.float32)
    lib().or_normals(_p(xyz), n, float(radius), _p(nrm), _p(pl), threads())
    return nrm, pl


def cluster(xyz, gnd=None, voxel=0.1, connect=0.35, min_pts=30, max_out=4096):
    """perception.py:114-271: (cid per point, node labels, clusters [(cnt, cen, lo, hi)], clusters before cap)."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32)
    n = len(xyz)
    g = np.zeros(n, np.int32) if gnd is None else np.ascontiguousarray(gnd, dtype=np.int32)
    cid = np.zeros(n, np.int32)
    labels = np.zeros(max(n, 1), np.int32)
    m = np.zeros(1, np.int64)
    k_all = np.zeros(1, np.int64)
    cnt = np.zeros(max_out, np.float32)
    cen = np.zeros((max_out, 3), np.float32)
    lo = np.zeros((max_out, 3), np.float32)
    hi = np.zeros((max_out, 3), np.float32)
    k = lib().or_cluster(_p(xyz), xyz.shape[1], _p(g), int(gnd is not None), n, voxel, connect, float(min_pts),
                         max_out, _p(cid), _p(labels), _p(m), _p(cnt), _p(cen), _p(lo), _p(hi), _p(k_all))
    clusters = [(float(cnt[j]), cen[j].copy(), lo[j].copy(), hi[j].copy()) for j in range(k)]
    return cid, labels[:int(m[0])], clusters, int(k_all[0])


# ---- the host-side float64 step (odom.py:387-455) -----------------------------------------------------------

_TRIU6 = np.triu_indices(6)


def sym6(upper: np.ndarray) -> np.ndarray:
    H = np.zeros((6, 6))
    H[_TRIU6] = upper
    return H + np.triu(H, 1).T


def twist_between(T_from, T_to):
    M = T_to @ np.linalg.inv(T_from)
    return np.concatenate([M[:3, 3], Rotation.from_matrix(M[:3, :3]).as_rotvec()])


def apply_twist(T, delta):
    Rz = Rotation.from_rotvec(delta[3:]).as_matrix()
    out = T.copy()
    out[:3, :3] = Rz @ T[:3, :3]
    out[:3, 3] = Rz @ T[:3, 3] + delta[:3]
    return out


def body_twist(d):
    return np.concatenate([d[:3, 3], Rotation.from_matrix(d[:3, :3]).as_rotvec()]).astype(np.float32)


def twist_matrix(xi):
    out = np.eye(4)
    out[:3, :3] = Rotation.from_rotvec(np.asarray(xi[3:], dtype=np.float64)).as_matrix()
    out[:3, 3] = xi[:3]
    return out


def sensor_basis(T, L):
    c = T[:3, 3]
    J = np.eye(6)
    J[:3, 3:] = np.array([[0.0, -c[2], c[1]], [c[2], 0.0, -c[0]], [-c[1], c[0], 0.0]])
    B = np.zeros((6, 6))
    B[:3, :3] = B[3:, 3:] = T[:3, :3]
    return J @ B @ np.diag([1.0, 1.0, 1.0, 1.0 / L, 1.0 / L, 1.0 / L])


def constrained_step(A, rhs, Hg, T, L, thr, to_pred):
    J = sensor_basis(T, L)
    lam, V = np.linalg.eigh(J.T @ Hg @ J)
    good = lam >= thr
    if good.all():
        return np.linalg.solve(A, rhs), (lam, V, good)
    Vd = V[:, ~good]
    d0 = Vd @ (Vd.T @ np.linalg.solve(J, to_pred))
    if good.any():
        Vg = V[:, good]
        As = J.T @ A @ J
        d0 = d0 + Vg @ np.linalg.solve(Vg.T @ As @ Vg, Vg.T @ (J.T @ rhs - As @ d0))
    return J @ d0, (lam, V, good)


class Params:
    """Odometry tuning with the reference's defaults (odom.py:499-525)."""

    def __init__(self, **kw):
        self.frame_dt = 0.1
        self.reg_voxel = 0.15
        self.max_iter = 16
        self.warmup = 8
        self.min_points = 200
        self.min_corr = 60
        self.min_range = 0.3
        self.max_range = 60.0
        self.noise = 0.02
        self.ret_mask = 0b1111
        self.alpha = 0.05
        self.damping = 1.0e-3
        self.velocity_smooth = 0.85
        self.degen_thr = 3000.0
        self.prior_info = 2000.0
        self.kf_dist = 0.05
        self.kf_angle = 1.0
        self.deskew = True
        self.redeskew = True
        for k, v in kw.items():
            setattr(self, k, v)


def schedule(it: int, voxel: float):
    """reach, max_d2 and kappa of iteration `it`, rounded to float32 the way the kernels receive them."""
    reach = 2 if it < WIDE_ITERS else 1
    d = np.float32(np.float32(reach) + np.float32(0.5)) * np.float32(voxel)
    max_d2 = float(np.float32(d * d))
    kappa = float(np.float32(max(KAPPA_MIN, KAPPA_START * (KAPPA_DECAY ** it))))
    return reach, max_d2, kappa


def register(ds4: np.ndarray, T_pred: np.ndarray, reg: RegMap, p: Params, nthreads: int | None = None):
    """odom.py:752-803 with the float64 accumulation; returns (T, ok, stats dict)."""
    n_ds = len(ds4)
    stats = {"ds": n_ds}
    if n_ds < p.min_corr:
        return T_pred.copy(), False, stats
    T = T_pred.copy()
    voxel = p.reg_voxel
    iters, corr, rms, cond, n_degen = 0, 0, 0.0, 1.0, 0
    H = np.eye(6)
    for it in range(p.max_iter):
        reach, max_d2, kappa = schedule(it, voxel)
        v = icp_accumulate(ds4, T, reg, voxel, reach, max_d2, kappa, nthreads)
        corr = int(v[ACC_COUNT])
        if corr < p.min_corr:
            break
        H, b, Hg = sym6(v[ACC_H:ACC_H + 21]), v[ACC_B:ACC_B + 6], sym6(v[ACC_HG:ACC_HG + 21])
        L = max(v[ACC_RANGE] / corr, 1.0)
        rms = math.sqrt(max(v[ACC_RMS], 0.0) / max(v[ACC_WEIGHT], 1e-9))
        dg = np.diag(H)
        A = H + np.diag(1e-9 * dg.mean() + p.damping * dg)
        rhs = -b
        xi = twist_between(T, T_pred)
        if p.prior_info > 0.0:
            Ji = np.linalg.inv(sensor_basis(T, L))
            P = p.prior_info * (Ji.T @ Ji)
            A = A + P
            rhs = rhs + P @ xi
        try:
            if p.degen_thr > 0.0:
                delta, (_, _, kept) = constrained_step(A, rhs, Hg, T, L, p.degen_thr, xi)
                n_degen = int((~kept).sum())
            else:
                delta = np.linalg.solve(A, rhs)
        except np.linalg.LinAlgError:
            break
        T = apply_twist(T, delta)
        iters = it + 1
        if np.linalg.norm(delta[:3]) < STEP_TOL and np.linalg.norm(delta[3:]) < STEP_TOL:
            break
    if corr >= p.min_corr:
        dg = np.sqrt(np.maximum(np.diag(H), 1e-12))
        ev = np.linalg.eigvalsh(H / np.outer(dg, dg))
        cond = float(max(ev[0], 0.0) / max(ev[-1], 1e-12))
    stats.update(iters=iters, corr=corr, rms=rms, cond=cond, weak=cond < WEAK_COND or n_degen > 0, degen=n_degen)
    return T, corr >= p.min_corr, stats


class Odometry:
    """The frame pipeline of odom.py:642-727 on the oracle, fed one frame at a time."""

    def __init__(self, reg_slots: int, p: Params, T0=None):
        self.p = p
        self.reg = RegMap(reg_slots)
        self.T = np.eye(4) if T0 is None else np.asarray(T0, np.float64)
        self.T_prev = None
        self.delta = np.eye(4)
        self.xi = np.zeros(6, np.float32)
        self.xi_s = np.zeros(6)
        self.map_frames = 0
        self.T_key = None
        self.traj = []
        self.stats = {}

    def predict(self):
        return self.T @ self.delta

    def _deskew(self, raw4, t_mid, xi):
        return deskew(raw4, np.float32(t_mid), np.float32(1.0 / self.p.frame_dt), xi)

    def _register(self, xyz4, attr, T_pred):
        p = self.p
        ds = thin(xyz4, attr, np.float32(2.0 / p.reg_voxel), p.min_range, p.max_range, p.ret_mask)
        return register(ds, T_pred, self.reg, p)

    def frame(self, k: int, raw4: np.ndarray, attr: np.ndarray):
        """Finalise frame k from its raw points (x, y, z, t); returns (T, xyz4 deskewed, ok)."""
        p = self.p
        m = len(raw4)
        warm = self.map_frames < p.warmup
        t_mid = (k + 0.5) * p.frame_dt
        xi = self.xi if (p.deskew and not warm) else np.zeros(6, np.float32)
        xyz4 = self._deskew(raw4, t_mid, xi) if m > 0 else raw4
        T = self.T if warm else self.predict()
        ok = True
        if m < p.min_points:
            ok = False
        elif not warm:
            T, ok, st = self._register(xyz4, attr, T)
            self.stats.update(st)
            if ok and p.deskew and p.redeskew and self.T_prev is not None:
                xi_new = body_twist(np.linalg.inv(self.T_prev) @ T)
                if (np.linalg.norm(xi_new[3:] - xi[3:]) > REDESKEW_ROT
                        or np.linalg.norm(xi_new[:3] - xi[:3]) > REDESKEW_TRANS):
                    xi = xi_new
                    xyz4 = self._deskew(raw4, t_mid, xi)
                    T, ok, st = self._register(xyz4, attr, T)
                    self.stats.update(st)
        if ok and (warm or self._is_keyframe(T)):
            self.reg.insert(xyz4, attr, T, p.reg_voxel, p.max_range, p.ret_mask)
            self.reg.records(p.reg_voxel, p.noise, p.alpha)
            self.map_frames += 1
            self.T_key = T.copy()
        if self.T_prev is not None and not warm:
            self._update_velocity(np.linalg.inv(self.T_prev) @ T)
        self.T_prev = self.T = T
        self.traj.append((k, t_mid, T.copy()))
        return T, xyz4, ok

    def _is_keyframe(self, T):
        if self.T_key is None:
            return True
        d = np.linalg.inv(self.T_key) @ T
        ang = math.degrees(np.linalg.norm(Rotation.from_matrix(d[:3, :3]).as_rotvec()))
        return np.linalg.norm(d[:3, 3]) >= self.p.kf_dist or ang >= self.p.kf_angle

    def _update_velocity(self, d):
        if np.linalg.norm(d[:3, 3]) < MAX_FRAME_JUMP:
            self.delta = d
            self.xi = body_twist(d)
            if self.p.velocity_smooth > 0.0:
                a = self.p.velocity_smooth
                self.xi_s = a * self.xi_s + (1.0 - a) * self.xi.astype(np.float64)
                self.delta = twist_matrix(self.xi_s)
        else:
            self.delta = np.eye(4)
            self.xi = np.zeros(6, np.float32)
            self.xi_s = np.zeros(6)


def pose_error(A: np.ndarray, B: np.ndarray):
    """(metres, degrees) between two 4x4 poses."""
    d = np.linalg.inv(A) @ B
    return float(np.linalg.norm(d[:3, 3])), float(np.degrees(np.linalg.norm(Rotation.from_matrix(d[:3, :3]).as_rotvec())))


# ---- prior-map grid and batched localisation (mapgrid.py, localize.py) ------------------------------------------

GRID_CELL = 0.05  # mapgrid.py:24
EVAL_RADII = (0.03, 0.05, 0.10)  # localize.py:47


def prior_prepare(xyz, normal, planarity=None, cell: float = GRID_CELL, pad: float = 0.6) -> dict:
    """PriorGrid.prepare (mapgrid.py:216-243): points sorted by cell (stable), unit normals, the cell prefix."""
    xyz = np.asarray(xyz, dtype=np.float32)
    n = len(xyz)
    nrm = np.asarray(normal, dtype=np.float32)
    planar = np.asarray(planarity if planarity is not None else np.ones(n), dtype=np.float32)
    lo, hi = xyz.min(0), xyz.max(0)
    origin = (lo - pad).astype(np.float32)
    dims = np.ceil((hi + pad - origin) / cell).astype(np.int64)
    ijk = np.floor((xyz - origin) / cell).astype(np.int64)
    key = (ijk[:, 2] * dims[1] + ijk[:, 1]) * dims[0] + ijk[:, 0]
    order = np.argsort(key, kind="stable")
    ncell = int(np.prod(dims))
    start = np.zeros(ncell + 1, np.int32)
    np.cumsum(np.bincount(key, minlength=ncell), out=start[1:])
    nrm = nrm[order]
    nrm = np.ascontiguousarray(nrm / np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-6), dtype=np.float32)
    return {"xyz": np.ascontiguousarray(xyz[order]), "normal": nrm, "planarity": np.ascontiguousarray(planar[order]),
            "origin": origin, "cell": float(cell), "dims": dims, "start": start}


class PriorGrid:
    """The grid of a prepared prior map with its flooded nearest points (nn) and distance field (df)."""

    def __init__(self, prep: dict, build: bool = True):
        self.prep = prep
        self.xyz = np.ascontiguousarray(prep["xyz"], dtype=np.float32)
        self.nrm = np.ascontiguousarray(prep["normal"], dtype=np.float32)
        self.planar = np.ascontiguousarray(prep["planarity"], dtype=np.float32)
        self.start = np.ascontiguousarray(prep["start"], dtype=np.int32)
        self.dims = np.asarray(prep["dims"], dtype=np.int64)
        self.ncell = int(np.prod(self.dims))
        self.nn = np.full(self.ncell, -1, np.int32)
        self.df = np.full(self.ncell, 255, np.uint8)
        g = OrGrid()
        g.xyz, g.nrm, g.planar, g.start, g.nn = _p(self.xyz), _p(self.nrm), _p(self.planar), _p(self.start), _p(self.nn)
        g.origin = (C.c_float * 3)(*[float(v) for v in prep["origin"]])
        g.cell = float(prep["cell"])
        g.inv_cell = float(np.float32(1.0 / prep["cell"]))
        g.nx, g.ny, g.nz = (int(d) for d in self.dims)
        self.g = g
        if build:
            lib().or_grid_build(C.byref(g), len(self.xyz), _p(self.nn), _p(self.df), threads())

    def nearest(self, w) -> np.ndarray:
        w = np.ascontiguousarray(w, dtype=np.float32)
        out = np.empty(len(w), np.int32)
        lib().or_nearest(C.byref(self.g), _p(w), len(w), _p(out), threads())
        return out

    def distances(self, pts, T) -> np.ndarray:
        pts = np.ascontiguousarray(pts, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float64)
        out = np.empty(len(pts), np.float32)
        lib().or_prior_distances(C.byref(self.g), _p(pts), len(pts), _p(T), _p(out), threads())
        return out

    def score_grid(self, pts, pos, n_yaw: int, yaw0: float, dyaw: float, tau: float, free_cm: float,
                   ref: bool = False, nthreads: int | None = None) -> np.ndarray:
        """k_score_grid (localize.py:55-96) over every (position, heading): the exact-sum soft count the library
        computes, or with ref the reference's float32 sum in point order (same poses)."""
        pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 3)
        pos = np.ascontiguousarray(pos, dtype=np.float32).reshape(-1, 3)
        out = np.empty(len(pos) * int(n_yaw), np.float32)
        lib().or_score_grid(C.byref(self.g), _p(self.df), _p(pts), len(pts), _p(pos), len(pos), int(n_yaw),
                            float(yaw0), float(dyaw), float(tau), float(free_cm), int(ref), _p(out),
                            nthreads or threads())
        return out

    def score_list(self, pts, hyp, tau: float, ref: bool = False, nthreads: int | None = None) -> np.ndarray:
        """k_score_list (localize.py:99-123) for (x, y, z, yaw) hypotheses."""
        pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 3)
        hyp = np.ascontiguousarray(hyp, dtype=np.float32).reshape(-1, 4)
        out = np.empty(len(hyp), np.float32)
        lib().or_score_list(C.byref(self.g), _p(self.df), _p(pts), len(pts), _p(hyp), len(hyp), float(tau), int(ref),
                            _p(out), nthreads or threads())
        return out

    def icp(self, pts4, lo, hi, T, schedule, alpha=0.05, min_count=30, nthreads=None):
        """GlobalLocalizer._icp (localize.py:517-553) for every hypothesis' own range of pts4: (T, count, iters)."""
        pts4 = np.ascontiguousarray(pts4, dtype=np.float32)
        lo = np.ascontiguousarray(lo, dtype=np.int32)
        hi = np.ascontiguousarray(hi, dtype=np.int32)
        T = np.array(T, dtype=np.float64, order="C").reshape(-1, 4, 4)
        k = len(T)
        max_d2 = np.array([np.float32(d * d) for d, _ in schedule], np.float32)
        c2 = np.array([np.float32((d * 0.5) ** 2) for d, _ in schedule], np.float32)
        iters = np.array([it for _, it in schedule], np.int32)
        count = np.zeros(k, np.int32)
        run = np.zeros(1, np.int32)
        lib().or_loc_icp(C.byref(self.g), _p(pts4), _p(lo), _p(hi), k, _p(T), len(schedule), _p(max_d2), _p(c2),
                         _p(iters), alpha, min_count, _p(count), _p(run), nthreads or threads())
        return T, count, int(run[0])

    def evaluate(self, pts4, lo, hi, T, nthreads=None) -> np.ndarray:
        """k_eval_batch (localize.py:182-205): points within each of EVAL_RADII of the map, per hypothesis."""
        pts4 = np.ascontiguousarray(pts4, dtype=np.float32)
        T = np.ascontiguousarray(np.asarray(T, dtype=np.float64).reshape(-1, 16))
        k = len(T)
        counts = np.zeros((k, 3), np.int32)
        radii = np.array(EVAL_RADII, np.float32)
        lib().or_loc_eval(C.byref(self.g), _p(pts4), _p(np.ascontiguousarray(lo, dtype=np.int32)),
                          _p(np.ascontiguousarray(hi, dtype=np.int32)), k, _p(T), _p(radii), _p(counts),
                          nthreads or threads())
        return counts


def thin_5cm(xyz) -> np.ndarray:
    """One point per 5 cm voxel, the first in scan order (localize.py:579-581)."""
    pts = np.asarray(xyz, dtype=np.float32)
    key = np.floor(pts / 0.05).astype(np.int64)
    _, first = np.unique(key, axis=0, return_index=True)
    return pts[np.sort(first)]


# ---- the learned start-pose network (float64 with the kernels' bf16 rounding points) ------------------------------

NET_P = 1024
NET_NPARAM = 108040
_NET_SEG = (("W1", 0, (64, 3)), ("b1", 192, (64,)), ("W2", 256, (128, 64)), ("b2", 8448, (128,)),
            ("W3", 8576, (256, 128)), ("b3", 41344, (256,)), ("Wh1", 41600, (128, 512)), ("bh1", 107136, (128,)),
            ("Wh2", 107264, (6, 128)), ("bh2", 108032, (6,)))


def bf16r(x) -> np.ndarray:
    """Round float32 values to bf16 (round to nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(a.shape)


def net_params(w_bf16: np.ndarray) -> dict:
    """The bf16 weight vector (as uint16 or float32 values) split into its tensors, float64."""
    w = np.asarray(w_bf16)
    if w.dtype in (np.uint16, np.int16):
        w = (w.astype(np.uint32) << 16).view(np.float32)
    w = w.astype(np.float64)
    return {name: w[o:o + int(np.prod(shape))].reshape(shape) for name, o, shape in _NET_SEG}


def net_forward(w_bf16, sets: np.ndarray, in_scale: float, out_scale) -> dict:
    """Forward pass of n samples: sets (2n, P, >=3). Layer activations rounded to bf16 where the kernels round."""
    p = net_params(w_bf16)
    X = (np.asarray(sets, np.float32)[..., :3] * np.float32(in_scale)).astype(np.float64)
    z1 = X @ p["W1"].T + p["b1"]
    h1 = bf16r(np.maximum(z1, 0.0).astype(np.float32)).astype(np.float64)
    z2 = h1 @ p["W2"].T + p["b2"]
    h2 = bf16r(np.maximum(z2, 0.0).astype(np.float32)).astype(np.float64)
    z3 = np.maximum(h2 @ p["W3"].T + p["b3"], 0.0)
    pooled = z3.max(axis=1)
    argmax = z3.argmax(axis=1)  # first point attaining the maximum
    n = len(sets) // 2
    x = bf16r(pooled.reshape(n, 512).astype(np.float32)).astype(np.float64)
    zh = x @ p["Wh1"].T + p["bh1"]
    hid = bf16r(np.maximum(zh, 0.0).astype(np.float32)).astype(np.float64)
    out = hid @ p["Wh2"].T + p["bh2"]
    step = out * np.asarray(out_scale, np.float64)
    return {"pooled": pooled, "argmax": argmax, "hid": hid, "out": out, "step": step, "x": x, "X": X}


def net_backward(w_bf16, sets: np.ndarray, fwd: dict, target: np.ndarray, w_loss, out_scale) -> tuple:
    """(gradient [NPARAM] with respect to the bf16 weights, loss) of sum_j w_j (out_j - target_j / scale_j)^2 / n,
    through the max by each channel's argmax point only."""
    p = net_params(w_bf16)
    sc = np.asarray(out_scale, np.float64)
    wl = np.asarray(w_loss, np.float64)
    n = len(target)
    diff = fwd["out"] - np.asarray(target, np.float64) / sc
    loss = float((wl * diff * diff).sum() / n)
    dout = 2.0 * wl * diff / n
    g = {k: np.zeros_like(v) for k, v in p.items()}
    g["Wh2"] = dout.T @ fwd["hid"]
    g["bh2"] = dout.sum(0)
    dzh = (dout @ p["Wh2"]) * (fwd["hid"] > 0)
    g["Wh1"] = dzh.T @ fwd["x"]
    g["bh1"] = dzh.sum(0)
    dpool = (dzh @ p["Wh1"]).reshape(2 * n, 256)
    X = fwd["X"]
    for s in range(2 * n):
        for c in range(256):
            if not fwd["pooled"][s, c] > 0.0:
                continue
            gz = dpool[s, c]
            x = X[s, fwd["argmax"][s, c]]
            z1 = x @ p["W1"].T + p["b1"]
            h1 = bf16r(np.maximum(z1, 0.0).astype(np.float32)).astype(np.float64)
            z2 = h1 @ p["W2"].T + p["b2"]
            h2 = bf16r(np.maximum(z2, 0.0).astype(np.float32)).astype(np.float64)
            g["W3"][c] += gz * h2
            g["b3"][c] += gz
            d2 = gz * p["W3"][c] * (z2 > 0)
            g["W2"] += np.outer(d2, h1)
            g["b2"] += d2
            d1 = (d2 @ p["W2"]) * (z1 > 0)
            g["W1"] += np.outer(d1, x)
            g["b1"] += d1
    out = np.zeros(NET_NPARAM)
    for name, o, shape in _NET_SEG:
        out[o:o + int(np.prod(shape))] = g[name].reshape(-1)
    return out, loss
