"""Firing-level reader for LVXR recordings (lvxr.py): every firing with its exact time, the empty ones included,
so a real recording can be replayed through the pipeline.

Same interface as the reference: `read_firings(path) -> Firings` with `t`, `xyz`, `refl`, `tag`, `valid`,
`direction`, `dev_type`, `profile`, `interval`, and `Firings.head()` / `.points()`. The decode runs in the library
(`lw_lvxr_decode`, host C++, no GPU needed): datagram walk, time base, record layouts, firing order, as lvxr.py
does it. `Firings.points()` gives the flat (xyz, attr, t, firing) arrays that `Pipeline.stage` takes.
"""

from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, replace

import numpy as np

from . import _lib

PROFILE_STANDARD, PROFILE_MID40_DUAL = 0, 1


@dataclass
class Firings:
    """Every firing of a recording, in time order. R is the most returns any firing carries."""

    t: np.ndarray  # (n,) float64 s since the recording's time base
    xyz: np.ndarray  # (n, R, 3) float32 m, sensor frame; zero where a return slot is empty
    refl: np.ndarray  # (n, R) uint8
    tag: np.ndarray  # (n, R) uint8
    valid: np.ndarray  # (n, R) bool: a return was reported
    direction: np.ndarray  # (n, 3) float32 unit firing direction, NaN where the data gives none
    dev_type: int
    profile: int
    interval: float  # s between firings

    @property
    def returns(self) -> int:
        return self.xyz.shape[1]

    @property
    def misses(self) -> np.ndarray:
        """Firings that returned nothing."""
        return ~self.valid.any(axis=1)

    def head(self, seconds: float) -> Firings:
        """The firings of the first `seconds`."""
        k = self.t < self.t[0] + seconds
        return replace(self, t=self.t[k], xyz=self.xyz[k], refl=self.refl[k], tag=self.tag[k], valid=self.valid[k],
                       direction=self.direction[k])

    def points(self, clean: bool = True, min_range: float = 0.3):
        """The returns as flat time-ordered arrays (xyz, attr, t float64, firing index), attr = reflectivity |
        tag << 8 | return << 16 as the live path packs it; clean keeps the confident returns (tag 0) beyond
        min_range."""
        f, r = np.nonzero(self.valid)
        xyz = self.xyz[f, r]
        tag = self.tag[f, r].astype(np.uint32)
        attr = self.refl[f, r].astype(np.uint32) | (tag << np.uint32(8)) | (r.astype(np.uint32) << np.uint32(16))
        keep = (tag == 0) & (np.linalg.norm(xyz, axis=1) > min_range) if clean else np.ones(len(f), bool)
        sel = np.flatnonzero(keep)
        sel = sel[np.argsort(self.t[f[sel]], kind="stable")]
        return xyz[sel], attr[sel], self.t[f[sel]], f[sel]


def decode(data: bytes) -> Firings:
    """Firings of a recording held in memory."""
    lib = _lib.load(require_cuda=False)
    buf = np.frombuffer(data, np.uint8)
    h = C.c_void_p()
    _lib.check(lib.lw_lvxr_decode(buf.ctypes.data_as(C.c_void_p), len(buf), C.byref(h)), "lw_lvxr_decode")
    try:
        n, R, dev, prof, dt = C.c_int64(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
        _lib.check(lib.lw_lvxr_info(h, C.byref(n), C.byref(R), C.byref(dev), C.byref(prof), C.byref(dt)), "lw_lvxr_info")
        n, R = n.value, R.value
        t = np.empty(n, np.float64)
        xyz = np.empty((n, R, 3), np.float32)
        refl = np.empty((n, R), np.uint8)
        tag = np.empty((n, R), np.uint8)
        valid = np.empty((n, R), np.uint8)
        direction = np.empty((n, 3), np.float32)
        p = [a.ctypes.data_as(C.c_void_p) for a in (t, xyz, refl, tag, valid, direction)]
        _lib.check(lib.lw_lvxr_copy(h, *p), "lw_lvxr_copy")
    finally:
        lib.lw_lvxr_free(h)
    return Firings(t=t, xyz=xyz, refl=refl, tag=tag, valid=valid.astype(bool), direction=direction, dev_type=dev.value,
                   profile=prof.value, interval=dt.value)


def read_firings(path: str | os.PathLike) -> Firings:
    """Every firing of an LVXR recording."""
    with open(path, "rb") as f:
        return decode(f.read())
