"""Shared seeded inputs of the tests: the scenes and scans of the benchmark configurations at test sizes."""

from __future__ import annotations

import functools

import numpy as np

from livox_warp import synth

FRAME_DT = 0.1


@functools.lru_cache(maxsize=None)
def room(seed: int = 1):
    return synth.box_room(seed)


@functools.lru_cache(maxsize=None)
def handheld(seed: int = 2, duration: float = 20.0, scene_seed: int = 1):
    return synth.Handheld(room(scene_seed), seed, duration)


@functools.lru_cache(maxsize=None)
def handheld_frames(n: int, seed: int = 3, traj_seed: int = 2, duration: float = 20.0, rate: float = 100000.0):
    sc = room(1)
    tr = handheld(traj_seed, duration)
    return synth.frames(sc, tr, n, rate, seed)


def frame_ids(t: np.ndarray, inv_dt: float = 10.0) -> np.ndarray:
    """floor(max(t, 0) * inv_dt) in float32, as the frame-id kernel computes it."""
    return np.floor(np.maximum(np.asarray(t, np.float32), np.float32(0)) * np.float32(inv_dt)).astype(np.int32)


def mid_pose(traj, k: int) -> np.ndarray:
    return traj.poses(np.array([(k + 0.5) * FRAME_DT]))[0]


def raw4(xyz, t) -> np.ndarray:
    return np.ascontiguousarray(np.concatenate([xyz, t[:, None]], axis=1).astype(np.float32))


def look_at(p, target) -> np.ndarray:
    """Sensor-to-world pose at p with the sensor's x axis toward target (no roll)."""
    return synth.look_at(p, target)


def config1_pose() -> np.ndarray:
    """The single-frame ICP case's start pose: a corner of the box room, looking across it and slightly down."""
    return look_at([0.8, 0.8, 1.6], [7.0, 5.0, 1.0])


def rule_local_maxima(sc, shape, pool):
    """The local-maximum rule of localize.py:450-475 in numpy over every score at least the pool-th best: positive
    and no lower than any in-range (x, y) / wrapped-heading neighbour at the same height. Unordered; the reference
    takes exactly `pool` candidates, so at a tie on the pool-th score it may leave out some that this keeps
    (tests/test_local_maxima_cpu.py pins the two against each other)."""
    nz, nx, ny, nyaw = shape
    thr = np.partition(sc, len(sc) - pool)[len(sc) - pool] if pool < len(sc) else sc.min()
    cand = np.nonzero((sc > 0) & (sc >= thr))[0]
    iyaw = cand % nyaw
    ip = cand // nyaw
    iy = ip % ny
    ix = (ip // ny) % nx
    iz = ip // (ny * nx)
    best = np.ones(len(cand), bool)
    mine = sc[cand]
    for ox in (-1, 0, 1):
        for oy in (-1, 0, 1):
            for oa in (-1, 0, 1):
                if ox == oy == oa == 0:
                    continue
                jx, jy = ix + ox, iy + oy
                ok = (jx >= 0) & (jx < nx) & (jy >= 0) & (jy < ny)
                j = ((iz * nx + np.clip(jx, 0, nx - 1)) * ny + np.clip(jy, 0, ny - 1)) * nyaw + (iyaw + oa) % nyaw
                best &= ~ok | (sc[j] <= mine)
    return cand[best]
