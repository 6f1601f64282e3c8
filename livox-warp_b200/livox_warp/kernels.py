"""The odometry kernels one by one: device tables plus thin wrappers over the C ABI (include/livox_b200.h).

Odometry (odom.py) runs them fused: one lw_odom_finalize per streamed frame, one lw_register_frame per frame handed
in directly. This module exposes each step on its own for callers that compose them differently (the parity
tests, batch tools).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib

TIGHT_FRACTION = 0.6


def _sp(stream=None):
    return _lib.stream_ptr(stream)


class RegistrationMap:
    """The registration voxel map (odom.py:468-474): keys, counts, exact fixed-point sums of (w - centre) and
    their outer products, and the per-voxel record the ICP reads (mean, precisions M and Mg, rms direction)."""

    def __init__(self, slots: int, device="cuda"):
        if slots <= 0 or slots & (slots - 1):
            raise ValueError(f"reg_slots must be a power of two, got {slots}")
        d = torch.device(device)
        self.cap = slots
        self.keys = torch.full((slots,), -1, dtype=torch.int64, device=d)
        self.cnt = torch.zeros(slots, dtype=torch.int32, device=d)
        self.sum = torch.zeros((slots, 3), dtype=torch.int64, device=d)
        self.outer = torch.zeros((slots, 6), dtype=torch.int64, device=d)
        self.rec = torch.zeros((slots, _lib.REC_FLOATS), dtype=torch.float32, device=d)
        self._bcnt = torch.zeros(slots, dtype=torch.int32, device=d)
        self._first = torch.full((slots,), _lib.INT32_MAX, dtype=torch.int32, device=d)
        self.stats = torch.zeros(2, dtype=torch.int32, device=d)
        self.struct = _lib.RegMap(*(_lib.ptr(t).value for t in (
            self.keys, self.cnt, self.sum, self.outer, self.rec, self._bcnt, self._first, self.stats)), slots)
        self._pslot = torch.zeros(1, dtype=torch.int32, device=d)

    def clear(self, stream=None):
        eye = _lib.f64_array(np.eye(4).reshape(16))
        # lw_odom_reset clears the map; a scratch state absorbs the reset of the odometry fields
        st = torch.zeros(ctypes.sizeof(_lib.OdomState), dtype=torch.uint8, device=self.keys.device)
        _lib.call("lw_odom_reset", eye, _lib.ptr(st), ctypes.byref(self.struct), 1, _sp(stream))

    @staticmethod
    def rec_params(voxel: float, noise: float = 0.02, alpha: float = 0.05) -> _lib.RecParams:
        rp = _lib.RecParams()
        rp.voxel = voxel
        rp.tight2 = (TIGHT_FRACTION * voxel / math.sqrt(12.0)) ** 2
        rp.noise2 = noise * noise
        rp.alpha = alpha
        return rp

    def insert(self, xyz4: torch.Tensor, attr: torch.Tensor, T: np.ndarray, voxel: float, max_range: float = 60.0,
               ret_mask: int = 0b1111, noise: float = 0.02, alpha: float = 0.05, n_dev: torch.Tensor | None = None,
               stream=None):
        """Add points (n, 4) posed by T and refresh the touched voxels' records (odom.py:186-230, 719-727)."""
        if (xyz4.dtype != torch.float32 or xyz4.dim() != 2 or xyz4.shape[1] != 4 or not xyz4.is_contiguous()
                or not xyz4.is_cuda):
            raise ValueError("registration map points must be a contiguous float32 (n, 4) CUDA tensor")
        n = int(xyz4.shape[0])
        if n > self._pslot.numel():
            self._pslot = torch.zeros(n, dtype=torch.int32, device=self.keys.device)
        T = _lib.f64_array(np.asarray(T, np.float64).reshape(16))
        _lib.call("lw_reg_insert", _lib.ptr(xyz4), _lib.ptr(attr), _lib.ptr(n_dev), n, T, float(voxel),
                  float(max_range), int(ret_mask), ctypes.byref(self.struct),
                  ctypes.byref(self.rec_params(voxel, noise, alpha)), _lib.ptr(self._pslot), _sp(stream))

    def refresh(self, voxel: float, noise: float = 0.02, alpha: float = 0.05, stream=None):
        _lib.call("lw_reg_refresh_all", ctypes.byref(self.struct), ctypes.byref(self.rec_params(voxel, noise, alpha)),
                  _sp(stream))

    def as_dict(self) -> dict:
        keys = self.keys.cpu().numpy()
        occ = keys != -1
        cnt, s, o = self.cnt.cpu().numpy()[occ], self.sum.cpu().numpy()[occ], self.outer.cpu().numpy()[occ]
        return {int(k): (int(c), tuple(a), tuple(b)) for k, c, a, b in zip(keys[occ], cnt, s, o)}


class GnScratch:
    """Scratch of the Gauss-Newton kernels: per-CTA partials, the grid barrier and its error flag. The struct's
    spin_budget (barrier wait limit, 0 = default) and skip_cta (a CTA that leaves before the first barrier, -1 =
    none) exist for tests of the bounded wait."""

    def __init__(self, device="cuda"):
        d = torch.device(device)
        sms = ctypes.c_int32(0)
        _lib.call("lw_device_sms", ctypes.byref(sms))
        self.grid = int(sms.value)
        self.part = torch.zeros(2 * self.grid * _lib.ACC_STRIDE, dtype=torch.float64, device=d)
        self.bar = torch.zeros(2, dtype=torch.int32, device=d)
        self.err = torch.zeros(1, dtype=torch.int32, device=d)
        self.struct = _lib.GnScratch(_lib.ptr(self.part).value, _lib.ptr(self.bar).value, _lib.ptr(self.err).value,
                                     self.grid, 0, -1, None)
        self.trace = None

    def trace_on(self, on: bool = True):
        """Record the start pose and the pose after each Gauss-Newton iteration (read with poses())."""
        if on and self.trace is None:
            self.trace = torch.zeros(_lib.GN_TRACE * 12, dtype=torch.float64, device=self.part.device)
        self.struct.trace = _lib.ptr(self.trace).value if on else None

    def poses(self, iters: int) -> np.ndarray:
        """The traced poses: (iters + 1, 4, 4), the start first (synchronises)."""
        t = self.trace.cpu().numpy().reshape(_lib.GN_TRACE, 3, 4)[:iters + 1]
        out = np.tile(np.eye(4), (len(t), 1, 1))
        out[:, :3, :] = t
        return out


def deskew(raw4: torch.Tensor, t_mid: float, inv_dt: float, twist, stream=None) -> torch.Tensor:
    """Deskew points (n, 4: x, y, z, t) to mid-frame with the body twist (rho, theta) (odom.py:163-178)."""
    n = int(raw4.shape[0])
    out = torch.empty_like(raw4)
    m = torch.tensor([n], dtype=torch.int32, device=raw4.device)
    _lib.call("lw_deskew", _lib.ptr(raw4), _lib.ptr(out), _lib.ptr(m), n, float(t_mid), float(inv_dt),
              _lib.f32_array(np.asarray(twist, np.float32)), _sp(stream))
    return out


class Thinner:
    """Half-voxel thinning tables for frames of up to `cap` points (odom.py:126-160, 484-488)."""

    def __init__(self, cap: int, device="cuda"):
        d = torch.device(device)
        self.cap = cap
        self.ds_cap = 1 << (cap - 1).bit_length()
        self.f_xyz = torch.zeros((cap, 4), dtype=torch.float32, device=d)
        self.f_attr = torch.zeros(cap, dtype=torch.int32, device=d)
        self.ds_keys = torch.full((self.ds_cap,), -1, dtype=torch.int64, device=d)
        self.ds_win = torch.full((self.ds_cap,), _lib.INT32_MAX, dtype=torch.int32, device=d)
        self.ds_slot = torch.zeros(cap, dtype=torch.int32, device=d)
        self.tiles = torch.zeros(cap // 1024 + 2, dtype=torch.int32, device=d)
        self.ds_xyz = torch.zeros((cap, 4), dtype=torch.float32, device=d)
        self.m = torch.zeros(1, dtype=torch.int32, device=d)
        self.n_ds = torch.zeros(1, dtype=torch.int32, device=d)
        nul = 0
        self.fb = _lib.FrameBuf(nul, _lib.ptr(self.f_xyz).value, _lib.ptr(self.f_attr).value, nul, nul, nul,
                                _lib.ptr(self.ds_keys).value, _lib.ptr(self.ds_win).value,
                                _lib.ptr(self.ds_slot).value, _lib.ptr(self.tiles).value, _lib.ptr(self.ds_xyz).value,
                                cap, self.ds_cap)

    def __call__(self, xyz4: torch.Tensor, attr: torch.Tensor, inv_v: float, min_range: float = 0.3,
                 max_range: float = 60.0, ret_mask: int = 0b1111, stream=None) -> torch.Tensor:
        n = int(xyz4.shape[0])
        if n > self.cap:
            raise ValueError(f"{n} points exceed the thinning capacity {self.cap}")
        self.f_xyz[:n].copy_(xyz4)
        self.f_attr[:n].copy_(attr.view(torch.int32))
        self.m.fill_(n)
        _lib.call("lw_thin", ctypes.byref(self.fb), _lib.ptr(self.m), n, float(inv_v), float(min_range),
                  float(max_range), int(ret_mask), _lib.ptr(self.n_ds), _sp(stream))
        k = int(self.n_ds.cpu()[0])
        return self.ds_xyz[:k]


def icp_accumulate(ds4: torch.Tensor, T: np.ndarray, reg: RegistrationMap, voxel: float, reach: int, max_d2: float,
                   kappa: float, gn: GnScratch, stream=None) -> np.ndarray:
    """One Gauss-Newton accumulation at pose T (odom.py:275-384): the 64 float64 entries of the ACC_* layout."""
    out = torch.zeros(_lib.ACC_STRIDE, dtype=torch.float64, device=ds4.device)
    n = int(ds4.shape[0])
    _lib.call("lw_icp_accumulate", _lib.ptr(ds4), None, n, _lib.f64_array(np.asarray(T, np.float64).reshape(16)),
              ctypes.byref(reg.struct), float(voxel), int(reach), float(max_d2), float(kappa), ctypes.byref(gn.struct),
              _lib.ptr(out), _sp(stream))
    return out.cpu().numpy()


def icp_solve(ds4: torch.Tensor, T_pred: np.ndarray, reg: RegistrationMap, params: _lib.OdomParams, gn: GnScratch,
              stream=None) -> tuple[np.ndarray, bool, dict]:
    """The whole Gauss-Newton registration of odom.py:752-803 on the device, from T_pred (also the prior)."""
    d = ds4.device
    st = _lib.OdomState()
    for i, v in enumerate(np.asarray(T_pred, np.float64).reshape(16)):
        st.T_pred[i] = v
    st.cond = 1.0
    buf = torch.from_numpy(np.frombuffer(bytes(st), dtype=np.uint8).copy()).to(d)
    n = torch.tensor([int(ds4.shape[0])], dtype=torch.int32, device=d)
    _lib.call("lw_icp_solve", _lib.ptr(ds4), _lib.ptr(n), ctypes.byref(params), _lib.ptr(buf), ctypes.byref(reg.struct),
              ctypes.byref(gn.struct), _sp(stream))
    out = _lib.OdomState.from_buffer_copy(buf.cpu().numpy().tobytes())
    T = np.array(out.T_reg, dtype=np.float64).reshape(4, 4)
    stats = {"ds": out.n_ds, "iters": out.iters, "corr": out.corr, "rms": out.rms, "cond": out.cond,
             "weak": bool(out.weak), "degen": out.degen}
    return T, bool(out.ok), stats
