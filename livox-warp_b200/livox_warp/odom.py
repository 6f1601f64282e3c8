"""LiDAR-only odometry on a B200: the `livox_warp.odom` module of the reference (python/livox_warp/odom.py) with
every per-frame step on the device.

Same algorithm and public API as the reference's Odometry (odom.py:458-803): frames cut by timestamp, deskew
to mid-frame, half-voxel thinning, scan-to-map point-to-distribution Gauss-Newton with a Geman-McClure kernel,
Levenberg-Marquardt damping, a prior toward the prediction and degenerate directions held at it, re-deskew and
re-registration with the solved motion, keyframe insertion into a registration voxel map that keeps per-voxel
sums of the points relative to the voxel centre, and a constant-velocity prediction from a smoothed twist.

What moved: the 6x6 solve (odom.py:772-796), the frame bookkeeping of _finalize / _estimate / _update_velocity
and the pose-table writes run on the GPU (liblivoxb200.so, lw_odom_finalize), so a frame costs no host
round trip. The host keeps only the frame-id bookkeeping of push(), which depends on the batch time span the
caller passes. Reading `T`, `traj`, `stats` or calling on_frame synchronises the stream.
"""

from __future__ import annotations

import ctypes
import math
import time

import numpy as np
import torch

from . import _lib
from .gpu import Pipeline, _as_xyz, row_stride
from .kernels import GnScratch, RegistrationMap

ACC_SLOTS = 64
ACC_H, ACC_B, ACC_COUNT, ACC_ERR, ACC_RMS, ACC_WEIGHT, ACC_RANGE, ACC_HG = (
    _lib.ACC_H, _lib.ACC_B, _lib.ACC_COUNT, _lib.ACC_ERR, _lib.ACC_RMS, _lib.ACC_WEIGHT, _lib.ACC_RANGE, _lib.ACC_HG)
ACC_STRIDE = _lib.ACC_STRIDE
REG_CAP = _lib.REG_CAP
WIDE_ITERS = 3
KAPPA_START, KAPPA_DECAY, KAPPA_MIN = 6.0, 0.7, 2.0
STEP_TOL = 1e-4
TIGHT_FRACTION = 0.6
WEAK_COND = 1e-3
REDESKEW_ROT = 2e-3
REDESKEW_TRANS = 5e-3
MAX_FRAME_JUMP = 1.5
TRAJ_CAP = 1 << 16


def _byref(s):
    return ctypes.byref(s)


class Odometry:
    """Frame cutting, the registration map and scan-to-map ICP on one stream (odom.py:458)."""

    def __init__(self, pipe: Pipeline, device=None, reg_slots: int = 1 << 21, frame_cap: int = 1 << 18,
                 stream: torch.cuda.Stream | None = None):
        _lib.load()
        self.pipe = pipe
        self.device = torch.device(device) if device is not None else pipe.device
        d = self.device
        self.stream = stream if stream is not None else torch.cuda.current_stream(d)
        if reg_slots <= 0 or reg_slots & (reg_slots - 1):
            raise ValueError(f"reg_slots must be a power of two, got {reg_slots}")
        self.reg_cap = reg_slots
        self.reg = RegistrationMap(reg_slots, d)
        self.reg_keys, self.reg_cnt, self.reg_sum, self.reg_outer = self.reg.keys, self.reg.cnt, self.reg.sum, self.reg.outer
        self.reg_rec, self.reg_stats = self.reg.rec, self.reg.stats
        self.regmap = self.reg.struct

        self.frame_cap = frame_cap
        self.ds_cap = 1 << (frame_cap - 1).bit_length()
        self.f_raw = torch.zeros((frame_cap, 4), dtype=torch.float32, device=d)
        self.f_xyz = torch.zeros((frame_cap, 4), dtype=torch.float32, device=d)  # deskewed x, y, z, t
        self.f_attr = torch.zeros(frame_cap, dtype=torch.int32, device=d)
        self.f_t = torch.zeros(frame_cap, dtype=torch.float32, device=d)
        self.f_frame = torch.zeros(frame_cap, dtype=torch.int32, device=d)
        self.f_count = torch.zeros(1, dtype=torch.int32, device=d)
        self.ds_keys = torch.full((self.ds_cap,), -1, dtype=torch.int64, device=d)
        self._ds_win = torch.full((self.ds_cap,), _lib.INT32_MAX, dtype=torch.int32, device=d)
        self._ds_slot = torch.zeros(frame_cap, dtype=torch.int32, device=d)
        self._tiles = torch.zeros(frame_cap // 1024 + 2, dtype=torch.int32, device=d)
        self.ds_xyz = torch.zeros((frame_cap, 4), dtype=torch.float32, device=d)
        self.fbuf = _lib.FrameBuf(*(_lib.ptr(t).value for t in (
            self.f_raw, self.f_xyz, self.f_attr, self.f_t, self.f_frame, self.f_count, self.ds_keys, self._ds_win,
            self._ds_slot, self._tiles, self.ds_xyz)), frame_cap, self.ds_cap)

        self._gn = GnScratch(d)
        self.gn = self._gn.struct
        self._state = torch.zeros(ctypes.sizeof(_lib.OdomState), dtype=torch.uint8, device=d)
        # pinned landing buffers for the state and the registration's error flag: one stream sync per readback
        self._state_host = torch.empty(ctypes.sizeof(_lib.OdomState), dtype=torch.uint8, pin_memory=True)
        self._err_host = torch.empty(1, dtype=torch.int32, pin_memory=True)
        # where a host frame's registration launch writes its result (lw_register_frame_host)
        self._reg_out = torch.empty(ctypes.sizeof(_lib.OdomState), dtype=torch.uint8, pin_memory=True)
        self._reg_err = torch.empty(1, dtype=torch.int32, pin_memory=True)
        self._reg_out_np, self._reg_err_np = self._reg_out.numpy(), self._reg_err.numpy()
        self._out_pending = False
        self._traj = torch.zeros(TRAJ_CAP * ctypes.sizeof(_lib.TrajRec), dtype=torch.uint8, device=d)

        # tuning (odom.py:499-525)
        self.frame_dt = 0.1
        self.reg_voxel = 0.15
        self.max_iter = 16
        self.warmup = 8
        self.max_gap = 20
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
        self.epoch = 0
        self._rec_key = None
        self._integrate = None
        self.side_stream = None  # integration's stream when it overlaps registration (integrate(overlap=True))
        self._snap = None
        self._pending = None
        self._net = None  # (InitNet, lw_net_work, its buffers) when the learned start pose is on
        self._reg_pin = None  # pinned staging of register_frame's host frames, and the event of its last copy
        self._reg_ev = None
        # the frame's point count as the device state holds it (an int32 view into the state buffer)
        off = _lib.OdomState.m.offset
        self._m_dev = self._state[off:off + 4].view(torch.int32)
        self.reset(np.eye(4, dtype=np.float64))

    # ---- parameters ---------------------------------------------------------------------------------------

    def params(self) -> _lib.OdomParams:
        p = _lib.OdomParams()
        p.frame_dt, p.reg_voxel, p.min_range, p.max_range = self.frame_dt, self.reg_voxel, self.min_range, self.max_range
        p.noise, p.alpha, p.damping, p.velocity_smooth = self.noise, self.alpha, self.damping, self.velocity_smooth
        p.degen_thr, p.prior_info, p.kf_dist, p.kf_angle_deg = self.degen_thr, self.prior_info, self.kf_dist, self.kf_angle
        p.max_iter, p.warmup, p.min_points, p.min_corr = self.max_iter, self.warmup, self.min_points, self.min_corr
        p.ret_mask, p.deskew, p.redeskew, p.frame_cap = int(self.ret_mask), int(self.deskew), int(self.redeskew), self.frame_cap
        return p

    def rec_params(self) -> _lib.RecParams:
        rp = _lib.RecParams()
        rp.voxel = self.reg_voxel
        rp.tight2 = (TIGHT_FRACTION * self.reg_voxel / math.sqrt(12.0)) ** 2
        rp.noise2 = self.noise * self.noise
        rp.alpha = self.alpha
        return rp

    def _sync_records(self):
        """The per-voxel records depend on reg_voxel, noise and alpha: recompute them if those changed."""
        key = (self.reg_voxel, self.noise, self.alpha)
        if key != self._rec_key:
            if self._rec_key is not None:
                _lib.call("lw_reg_refresh_all", _byref(self.regmap), _byref(self.rec_params()), self._sp())
            self._rec_key = key

    def _sp(self):
        return _lib.stream_ptr(self.stream)

    # ---- state ----------------------------------------------------------------------------------------------

    def synchronize(self):
        self.stream.synchronize()

    def read_state(self) -> _lib.OdomState:
        """The device state (synchronises the stream)."""
        _lib.call("lw_read_state", _lib.ptr(self._state), None, _lib.ptr(self._state_host), None, self._sp())
        return _lib.OdomState.from_buffer_copy(self._state_host.numpy())

    @staticmethod
    def empty_stats() -> dict:
        return {"frames": 0, "iters": 0, "corr": 0, "ds": 0, "rms": 0.0, "cond": 1.0, "ms": 0.0,
                "weak": False, "map_voxels": 0, "map_full": 0.0, "map_overflow": 0, "skipped": 0, "warm": True,
                "speed": 0.0, "turn": 0.0, "gaps": 0, "degen": 0, "keyframes": 0}

    def reset(self, T0: np.ndarray):
        """Forget the map and the trajectory; the next frame is posed at T0 (odom.py:561-579)."""
        self._issue_pending()
        T0 = np.asarray(T0, dtype=np.float64).reshape(16)
        _lib.call("lw_odom_reset", _lib.f64_array(T0), _lib.ptr(self._state), _byref(self.regmap), 1, self._sp())
        with torch.cuda.stream(self.stream):
            self._gn.err.zero_()  # a registration that gave up stays flagged until the next reset
        _lib.call("lw_frame_reset", _byref(self.fbuf), self._sp())
        self._rec_key = (self.reg_voxel, self.noise, self.alpha)
        self.k_open = None
        self.k_pred = -1
        self._m_ub = 0
        self._gaps = 0
        self._ms = 0.0

    def restart_clock(self):
        """The point timestamps jumped: keep the map and pose, restart frame counting at rest (odom.py:581-589)."""
        self.k_open = None
        self.k_pred = -1
        _lib.call("lw_odom_restart_clock", _lib.ptr(self._state), self._sp())
        _lib.call("lw_frame_reset", _byref(self.fbuf), self._sp())
        self._m_ub = 0

    @property
    def T(self) -> np.ndarray:
        return np.array(self.read_state().T, dtype=np.float64).reshape(4, 4)

    def predict(self) -> np.ndarray:
        st = self.read_state()
        return np.array(st.T).reshape(4, 4) @ np.array(st.delta).reshape(4, 4)

    @property
    def traj(self) -> list:
        """(frame id, mid-frame time, 4x4 pose) of every finalised frame (the last TRAJ_CAP kept)."""
        n = self.read_state().traj_len
        k = min(n, TRAJ_CAP)
        if k == 0:
            return []
        with torch.cuda.stream(self.stream):
            raw = self._traj.cpu().numpy().tobytes()
        recs = (_lib.TrajRec * TRAJ_CAP).from_buffer_copy(raw)
        out = []
        for j in range(n - k, n):
            r = recs[j % TRAJ_CAP]
            out.append((int(r.k), float(r.t_mid), np.array(r.T, dtype=np.float64).reshape(4, 4)))
        return out

    def traj_records(self) -> list:
        """traj plus each frame's (ok, iters, corr)."""
        n = self.read_state().traj_len
        k = min(n, TRAJ_CAP)
        with torch.cuda.stream(self.stream):
            raw = self._traj.cpu().numpy().tobytes()
        recs = (_lib.TrajRec * TRAJ_CAP).from_buffer_copy(raw)
        return [(int(r.k), float(r.t_mid), np.array(r.T).reshape(4, 4), int(r.ok), int(r.iters), int(r.corr))
                for r in (recs[j % TRAJ_CAP] for j in range(n - k, n))]

    @property
    def stats(self) -> dict:
        st = self.read_state()
        with torch.cuda.stream(self.stream):
            rs = self.reg_stats.cpu().numpy()
        xi = np.array(st.xi, dtype=np.float64)
        out = self.empty_stats()
        out.update(frames=st.frames, iters=st.iters, corr=st.corr, ds=st.n_ds, rms=st.rms, cond=st.cond,
                   ms=self._ms, weak=bool(st.weak), map_voxels=int(rs[0]), map_full=int(rs[0]) / self.reg_cap,
                   map_overflow=int(rs[1]), skipped=st.skipped, warm=st.map_frames < self.warmup,
                   speed=float(np.linalg.norm(xi[:3]) / self.frame_dt),
                   turn=float(math.degrees(np.linalg.norm(xi[3:])) / self.frame_dt), gaps=self._gaps,
                   degen=st.degen, keyframes=st.keyframes, err=st.err)
        return out

    # ---- per batch --------------------------------------------------------------------------------------------

    def _poses(self, k0: int, k1: int, mode: int):
        if k1 > k0:
            _lib.call("lw_odom_predict_poses", k0, k1, mode, _lib.ptr(self._state), _byref(self.pipe.pose_table),
                      self.epoch, self._sp())

    def _append(self, sx, sa, st, n, inv_dt, k_min, k_open):
        xyz = _as_xyz(sx if isinstance(sx, torch.Tensor) else torch.as_tensor(sx), self.device)
        _lib.call("lw_frame_append", _lib.ptr(xyz), row_stride(xyz), _lib.ptr(sa), _lib.ptr(st), int(n),
                  float(inv_dt), int(k_min), int(k_open), _byref(self.fbuf), self._sp())
        self._m_ub = min(self._m_ub + int(n), self.frame_cap)

    def _reset_frame(self):
        _lib.call("lw_frame_reset", _byref(self.fbuf), self._sp())
        self._m_ub = 0

    def push(self, sx, sa, st, n: int, t_min: float, t_max: float, on_frame=None):
        """Feed one staged batch. on_frame(k, T, f_xyz, f_attr, f_t, f_frame, m) runs per completed frame with
        the frame's points deskewed to mid-frame (odom.py:596-638). f_xyz is (frame_cap, 4): x, y, z, t.
        Without on_frame no frame synchronises the host."""
        if n <= 0:
            return
        self._sync_records()
        inv_dt = 1.0 / self.frame_dt
        k_lo = int(math.floor(max(t_min, 0.0) * inv_dt))
        k_hi = int(math.floor(max(t_max, 0.0) * inv_dt))
        k_prev = self.k_pred
        if self.k_open is not None and k_hi - self.k_open > self.max_gap:
            # data went missing: close what we have and restart counting from this batch, at rest
            if self._m_ub > 0 and int(self.f_count.cpu()[0]) > 0:
                self._finalize(self.k_open, on_frame)
            self.restart_clock()
            self._gaps += 1
        if self.k_open is None:
            self.k_open = k_lo if k_hi - k_lo <= self.max_gap else k_hi
            self._reset_frame()
            self._poses(self.k_open, self.k_open + 1, 1)  # the current pose with the current twist
            lo = (k_prev + 1) if 0 <= k_prev < self.k_open else k_lo
            if lo < self.k_open:
                self._poses(lo, self.k_open, 3)  # skipped ids held at the current pose, no motion
            self.k_pred = self.k_open
        k0 = max(self.k_pred + 1, self.k_open + 1)
        if k0 <= k_hi:
            self._poses(k0, k_hi + 1, 0)  # every frame id of the batch gets a predicted pose
            self.k_pred = k_hi
        k_min = self.k_open - 1  # a slightly late point joins the open frame; older ones are dropped
        while True:
            self._append(sx, sa, st, n, inv_dt, k_min, self.k_open)
            if k_hi <= self.k_open:
                break
            self._finalize(self.k_open, on_frame)
            self.k_open += 1
            k_min = self.k_open
            self._reset_frame()
            self._poses(self.k_open, self.k_open + 1, 0)
            self.k_pred = max(self.k_pred, self.k_open)

    def integrate(self, view, voxel: float, carve_every: int = 1, max_range: float = 40.0, max_steps: int = 4096,
                  overlap: bool = False):
        """Insert every finalised frame into the pipeline's integration map and carve its rays, on the device,
        straight after registration (what the viewer's on_frame does: app.py:557-563) -- without a host round
        trip. carve_every = 0 inserts without carving; view = None turns it off.

        overlap: run each frame's insert and carve on a second stream (`side_stream`) one frame later, from a copy
        of the frame, while the next frame registers on `stream`. The map then trails the newest pose by one frame
        until flush(); it ends up the same. Work on `stream` that reads the map should first wait for side_stream
        (flush() does that)."""
        self._issue_pending()
        self._integrate = None if view is None else (view, float(voxel), int(carve_every), float(max_range),
                                                     int(max_steps))
        self.side_stream = None
        self._snap = None
        self._pending = None
        if view is not None and overlap:
            d, cap = self.device, self.frame_cap
            self.side_stream = torch.cuda.Stream(d)
            # two copies of the frame buffers: frame k is copied while frame k - 1's copy may still be integrating
            self._snap = [{"xyz": torch.zeros((cap, 4), dtype=torch.float32, device=d),
                           "attr": torch.zeros(cap, dtype=torch.int32, device=d),
                           "t": torch.zeros(cap, dtype=torch.float32, device=d),
                           "frame": torch.zeros(cap, dtype=torch.int32, device=d),
                           "m": torch.zeros(1, dtype=torch.int32, device=d),
                           "copied": torch.cuda.Event(), "done": None, "m_ub": 0} for _ in range(2)]
            self._snap_next = 0

    def _run_integration(self, xyz, attr, t, frame, m_ub: int, m_dev):
        view, voxel, every, max_range, max_steps = self._integrate
        self.pipe.map_insert(xyz, attr, t, frame, m_ub, view, voxel, n_dev=m_dev)
        if every > 0:
            self.pipe.carve(xyz, attr, frame, m_ub, voxel, every, max_range, max_steps, n_dev=m_dev)

    def _issue_pending(self):
        """Start the deferred integration of the last copied frame on the side stream."""
        snap = self._pending
        if snap is None:
            return
        self._pending = None
        side = self.side_stream
        side.wait_event(snap["copied"])
        with torch.cuda.stream(side):
            self._run_integration(snap["xyz"], snap["attr"], snap["t"], snap["frame"], snap["m_ub"], snap["m"])
        snap["done"] = torch.cuda.Event()
        snap["done"].record(side)

    def learned_init(self, net, radius: float = 12.0, nearest: bool = True):
        """Start each frame's registration from the network's proposal (livox_warp.initnet.InitNet) instead of
        the constant-velocity prediction; None turns it off. The network sees the thinned frame and, for each of
        its points, the nearest registration voxel mean (nearest=False: the voxel means within `radius` m),
        both in the predicted sensor frame -- the sets it was trained on."""
        if net is None:
            self._net = None
            return
        d = self.device
        bufs = {"sets": torch.zeros((2, _lib.NET_P, 4), dtype=torch.float32, device=d),
                "pooled": torch.zeros(512, dtype=torch.float32, device=d),
                "argmax": torch.zeros(512, dtype=torch.int32, device=d),
                "hid": torch.zeros(128, dtype=torch.float32, device=d),
                "step": torch.zeros(6, dtype=torch.float32, device=d),
                "err": torch.zeros(1, dtype=torch.int32, device=d),
                "cand": torch.zeros(self.reg_cap, dtype=torch.int32, device=d),
                "tiles": torch.zeros(self.reg_cap // 1024 + 2, dtype=torch.int32, device=d),
                "count": torch.zeros(2, dtype=torch.int32, device=d)}
        work = _lib.NetWork(*(_lib.ptr(bufs[k]).value for k in _lib.NetWork.PTRS), float(radius),
                            float(self.reg_voxel) if nearest else 0.0)
        self._net = (net, work, bufs)

    def register_frame(self, xyz, attr, t, t_mid: float, twist, T_pred: np.ndarray, sync: bool = True):
        """Deskew one frame to t_mid with the body twist (rho, theta) and register it against the map from T_pred:
        the reference's _deskew then _register (odom.py:707-709, 752-803), for a frame handed in directly instead
        of cut from a stream. The map is left as it is (no keyframe insert, no velocity update).

        xyz: (m, 3) sensor points with t (m,) separately, or (m, 4) with t in the last column (t is then
        ignored); attr (m,) uint32. A CUDA tensor (m, 4) float32 is read in place; host arrays are copied into
        pinned memory, which the registration launch reads itself (and where it leaves its result). With sync,
        returns (T, ok, stats) like the reference's _register plus its stats; without, returns None and
        registration() reads the result later."""
        d = self.device
        if isinstance(xyz, torch.Tensor) and xyz.is_cuda:
            m = int(xyz.shape[0])
            raw = xyz if (xyz.dim() == 2 and xyz.shape[1] == 4 and xyz.dtype == torch.float32
                          and xyz.is_contiguous()) else None
            if raw is None:
                raise ValueError("a device frame must be a contiguous (m, 4) float32 tensor (x, y, z, t)")
            at = attr if isinstance(attr, torch.Tensor) else torch.as_tensor(np.asarray(attr).view(np.int32), device=d)
        else:
            x = np.asarray(xyz, np.float32)
            m = len(x)
            if m > self.frame_cap:
                raise ValueError(f"{m} points exceed the frame capacity {self.frame_cap}")
            if self._reg_pin is None or self._reg_pin["x3"].shape[0] < m:
                cap = max(m, 1 << 14)
                self._reg_pin = {"x3": torch.empty((cap, 3), dtype=torch.float32, pin_memory=True),
                                 "t": torch.empty(cap, dtype=torch.float32, pin_memory=True),
                                 "a": torch.empty(cap, dtype=torch.int32, pin_memory=True)}
                # numpy views of the pinned buffers, made once (a tensor's .numpy() costs microseconds per call)
                self._reg_pin.update({k + "_np": self._reg_pin[k].numpy() for k in ("x3", "t", "a")})
            pin = self._reg_pin
            if self._reg_ev is not None:
                self._reg_ev.synchronize()  # the previous launch has read the pinned frame
            # contiguous host copies into pinned memory; the registration launch reads them from there itself and
            # writes its result to pinned memory at its end (one launch, nothing else on the stream)
            pin["a_np"][:m] = np.asarray(attr).view(np.int32)
            pin["x3_np"][:m] = x[:, :3]
            pin["t_np"][:m] = x[:, 3] if x.ndim == 2 and x.shape[1] == 4 else np.asarray(t, np.float32)
            self._sync_records()
            _lib.call("lw_register_frame_host", _lib.ptr(pin["x3"]), _lib.ptr(pin["t"]), _lib.ptr(pin["a"]), m,
                      float(t_mid), _lib.f32_array(np.asarray(twist, np.float32).reshape(6)),
                      _lib.f64_array(np.asarray(T_pred, np.float64).reshape(16)), _byref(self.params()),
                      _lib.ptr(self._state), _byref(self.fbuf), _byref(self.regmap), _byref(self.gn),
                      _lib.ptr(self._reg_out), _lib.ptr(self._reg_err), self._sp())
            if self._reg_ev is None:
                self._reg_ev = torch.cuda.Event()
            self._reg_ev.record(self.stream)
            self._out_pending = True
            return self.registration() if sync else None
        if m > self.frame_cap:
            raise ValueError(f"{m} points exceed the frame capacity {self.frame_cap}")
        self._sync_records()
        _lib.call("lw_register_frame", _lib.ptr(raw), _lib.ptr(at), m, float(t_mid),
                  _lib.f32_array(np.asarray(twist, np.float32).reshape(6)),
                  _lib.f64_array(np.asarray(T_pred, np.float64).reshape(16)), _byref(self.params()),
                  _lib.ptr(self._state), _byref(self.fbuf), _byref(self.regmap), _byref(self.gn), self._sp())
        self._out_pending = False
        return self.registration() if sync else None

    def registration(self):
        """(T, ok, stats) of the last register_frame (synchronises the stream). stats["err"] is non-zero when a
        registration since the last reset gave up (a bounded wait ran out, or a fixed-point sum overflowed)."""
        if self._out_pending:  # a host frame's launch wrote its result to pinned memory
            self._reg_ev.synchronize()
            st = _lib.OdomState.from_buffer_copy(self._reg_out_np)
            err = int(self._reg_err_np[0])
        else:
            _lib.call("lw_read_state", _lib.ptr(self._state), _lib.ptr(self._gn.err), _lib.ptr(self._state_host),
                      _lib.ptr(self._err_host), self._sp())
            st = _lib.OdomState.from_buffer_copy(self._state_host.numpy())
            err = int(self._err_host[0])
        stats = {"ds": st.n_ds, "iters": st.iters, "corr": st.corr, "rms": st.rms, "cond": st.cond,
                 "weak": bool(st.weak), "degen": st.degen, "err": err}
        return np.array(st.T_reg, dtype=np.float64).reshape(4, 4), bool(st.ok), stats

    def insert_frame(self, xyz4: torch.Tensor, attr: torch.Tensor, T: np.ndarray):
        """Add a frame's points (a (m, 4) float32 CUDA tensor), posed by T, to the registration map as a keyframe
        would be (odom.py:719-727): what builds a prior registration map from frames whose poses are known."""
        self._sync_records()
        self.reg.insert(xyz4, attr, T, self.reg_voxel, self.max_range, int(self.ret_mask), self.noise, self.alpha,
                        stream=self.stream)

    def iteration_log(self) -> np.ndarray:
        """(k, iterations of the first registration, iterations of the last) of every logged frame that
        registered."""
        n = self.read_state().traj_len
        k = min(n, TRAJ_CAP)
        with torch.cuda.stream(self.stream):
            raw = self._traj.cpu().numpy().tobytes()
        recs = (_lib.TrajRec * TRAJ_CAP).from_buffer_copy(raw)
        rows = [(int(r.k), int(r.iters_first), int(r.iters)) for r in (recs[j % TRAJ_CAP] for j in range(n - k, n))
                if r.ok and r.iters_first > 0]
        return np.array(rows, dtype=np.int64).reshape(-1, 3)

    def flush(self, on_frame=None):
        """Finalise the open frame now (the end of a recording); with overlapped integration, also integrate the
        last frame and order `stream` after the side stream."""
        if self.k_open is not None and self._m_ub > 0:
            self._finalize(self.k_open, on_frame)
            self.k_open = None
        self._issue_pending()
        if self.side_stream is not None:
            self.stream.wait_stream(self.side_stream)

    def _finalize(self, k: int, on_frame):
        t0 = time.perf_counter()
        self._issue_pending()  # the previous frame's insert and carve run beside this frame's registration
        if self._net is None:
            _lib.call("lw_odom_finalize", int(k), max(self._m_ub, 1), _byref(self.params()), _lib.ptr(self._state),
                      _byref(self.fbuf), _byref(self.regmap), _byref(self.gn), _byref(self.pipe.pose_table),
                      self.epoch, _lib.ptr(self._traj), TRAJ_CAP, self._sp())
        else:
            net, work, _ = self._net
            _lib.call("lw_odom_finalize_net", int(k), max(self._m_ub, 1), _byref(self.params()),
                      _lib.ptr(self._state), _byref(self.fbuf), _byref(self.regmap), _byref(self.gn),
                      _byref(self.pipe.pose_table), self.epoch, _lib.ptr(self._traj), TRAJ_CAP, _byref(net.struct),
                      _byref(work), self._sp())
        if self._integrate is not None:
            m_ub = max(self._m_ub, 1)
            if self._snap is None:
                with torch.cuda.stream(self.stream):
                    self._run_integration(self.f_xyz, self.f_attr, self.f_t, self.f_frame, m_ub, self._m_dev)
            else:
                snap = self._snap[self._snap_next]
                self._snap_next ^= 1
                if snap["done"] is not None:
                    self.stream.wait_event(snap["done"])  # the copy two frames back has been integrated
                with torch.cuda.stream(self.stream):
                    snap["xyz"][:m_ub].copy_(self.f_xyz[:m_ub])
                    snap["attr"][:m_ub].copy_(self.f_attr[:m_ub])
                    snap["t"][:m_ub].copy_(self.f_t[:m_ub])
                    snap["frame"][:m_ub].copy_(self.f_frame[:m_ub])
                    snap["m"].copy_(self._m_dev)
                snap["copied"].record(self.stream)
                snap["m_ub"] = m_ub
                self._pending = snap
        if on_frame is not None:
            st = self.read_state()
            self._ms = (time.perf_counter() - t0) * 1e3
            T = np.array(st.T, dtype=np.float64).reshape(4, 4)
            # f_xyz as the reference hands it (a vec3 per point): the x, y, z columns of the float4 frame buffer
            on_frame(k, T, self.f_xyz[:, :3], self.f_attr, self.f_t, self.f_frame, int(st.m))
