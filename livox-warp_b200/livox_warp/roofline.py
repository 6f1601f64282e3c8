"""Algorithmic (compulsory) bytes of the per-frame kernels: the numerator of the roofline the benchmark reports.

Each input is read once, each output written once, and each touched table record is read (and written, if
modified) once per launch. The distinct records a launch must touch are counted here on the host with numpy
from the frame's points, its solved pose and the table's occupied keys, per kernel:

  Gauss-Newton registration (one launch = every iteration of a frame), per iteration:
      16 B per thinned point (x, y, z, range)
    +  8 B per distinct neighbour key probed (the union of the (2 reach + 1)^3 neighbourhoods)
    + 16 B per distinct occupied voxel among them (its mean and count)
    + 64 B per distinct voxel a point is matched to (its precision record)
    + 2 * 64 * 8 B per CTA (the float64 partials written and read back)
  and once per launch, for the frame's deskew and thinning that the launch runs before its loop:
      36 B per frame point (x, y, z, t and attr read, the deskewed x, y, z, t written)
    + 40 B per thinned point (x, y, z, range written; its half-voxel's key and index claimed and emptied)
  carving (one launch = one frame's rays):
      20 B per traced ray (x, y, z, attr, frame id)
    + 12 B per distinct voxel the rays visit (key + hit count)
    + 32 B per distinct occupied voxel among them (the fixed-point centroid sums)
    +  4 B per miss counter written (bounded by the occupied visited voxels)
  integration insert (one launch = one batch):
      24 B per point (x, y, z, attr, t, frame id) + 2 * 64 B per distinct voxel touched (key, count, sums, times)

  batched localisation ICP (one launch = every iteration of every hypothesis, then the evaluation), per
  iteration and for the evaluation pass:
      16 B per scan point of every hypothesis (x, y, z, pad)
    +  8 B per distinct grid cell probed (its start pair; the flooded seed is read only where a query has
       no point within one cell and is not counted)
    + 12 B per distinct map point in those cells (its xyz)
    + 16 B per distinct map point matched (its normal and planarity; the ICP iterations only)
    + 2 * 32 * 8 B per tile (the float64 tile partials written and read back)

The counts use the solved pose for every iteration and sample each ray every quarter voxel, so they are
estimates of the compulsory traffic, not measurements: ncu's dram__bytes is the measured counterpart.
"""

from __future__ import annotations

import numpy as np

BIAS = 1 << 20
KMASK = (1 << 21) - 1


def keys_of(ijk: np.ndarray) -> np.ndarray:
    ijk = ijk.astype(np.int64)
    return (((ijk[:, 0] + BIAS) & KMASK) | (((ijk[:, 1] + BIAS) & KMASK) << 21) |
            (((ijk[:, 2] + BIAS) & KMASK) << 42))


def _world(xyz: np.ndarray, T: np.ndarray) -> np.ndarray:
    return xyz[:, :3].astype(np.float64) @ T[:3, :3].T + T[:3, 3]


def thin_host(xyz_sensor: np.ndarray, voxel: float, min_range: float = 0.3, max_range: float = 60.0) -> np.ndarray:
    """First point of every half-voxel (the thinning rule), on the host."""
    r = np.linalg.norm(xyz_sensor[:, :3], axis=1)
    ok = (r >= min_range) & (r <= max_range)
    idx = np.nonzero(ok)[0]
    k = keys_of(np.floor(xyz_sensor[idx, :3] * (2.0 / voxel)).astype(np.int64))
    _, first = np.unique(k, return_index=True)
    return xyz_sensor[idx[np.sort(first)]]


def gn_bytes(ds_sensor: np.ndarray, T: np.ndarray, occupied_keys: np.ndarray, voxel: float, iters: int,
             grid: int, wide_iters: int = 3, frame_points: int = 0) -> float:
    """Compulsory bytes of one registration launch (all its iterations, and the thinning of a frame of
    frame_points points when it has one)."""
    w = _world(ds_sensor, T)
    base = np.floor(w / voxel).astype(np.int64)
    occ = np.sort(occupied_keys)
    total = 0.0
    own = keys_of(base)
    matched = np.unique(own[np.isin(own, occ, assume_unique=False)])
    for reach in (2, 1):
        n_it = min(iters, wide_iters) if reach == 2 else max(iters - wide_iters, 0)
        if n_it == 0:
            continue
        r = np.arange(-reach, reach + 1)
        off = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
        probed = np.unique(keys_of((base[:, None, :] + off[None, :, :]).reshape(-1, 3)))
        v_occ = np.count_nonzero(np.isin(probed, occ))
        per_it = 16 * len(ds_sensor) + 8 * len(probed) + 16 * v_occ + 64 * len(matched) + 2 * grid * 64 * 8
        total += n_it * per_it
    if frame_points:
        total += 36 * frame_points + 40 * len(ds_sensor)
    return float(total)


def carve_bytes(xyz_sensor: np.ndarray, T: np.ndarray, occupied_keys: np.ndarray, voxel: float, every: int = 1,
                max_range: float = 40.0) -> float:
    """Compulsory bytes of one carving launch over a frame's rays."""
    p = xyz_sensor[::every, :3].astype(np.float64)
    w = _world(p, T)
    o = T[:3, 3]
    d = w - o
    L = np.linalg.norm(d, axis=1)
    ok = (L >= 0.05) & (L <= max_range)
    d, L = d[ok] / L[ok, None], L[ok]
    stop = L - np.maximum(3.0 * voxel, 0.03 * L)
    step = voxel / 4.0
    n_s = np.maximum((stop / step).astype(np.int64), 0)
    ray = np.repeat(np.arange(len(L)), n_s)
    t = (np.arange(n_s.sum()) - np.repeat(np.cumsum(n_s) - n_s, n_s) + 0.5) * step
    pts = o + d[ray] * t[:, None]
    visited = np.unique(keys_of(np.floor(pts / voxel).astype(np.int64)))
    occ = np.count_nonzero(np.isin(visited, np.sort(occupied_keys)))
    return float(20 * len(p) + 12 * len(visited) + 32 * occ + 4 * occ)


def map_insert_bytes(xyz_sensor: np.ndarray, T: np.ndarray, voxel: float) -> float:
    w = _world(xyz_sensor, T)
    touched = np.unique(keys_of(np.floor(w / voxel).astype(np.int64)))
    return float(24 * len(w) + 2 * 64 * len(touched))


def loc_bytes(start: np.ndarray, origin: np.ndarray, dims: np.ndarray, cell: float, pts4: np.ndarray,
              lo: np.ndarray, hi: np.ndarray, T: np.ndarray, iters: int, n_tiles: int) -> dict:
    """Compulsory bytes of one batched localisation launch, counted at the final poses T (k, 4, 4)."""
    cells, matched_cells = [], []
    r = np.arange(-1, 2)
    off = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    dims = np.asarray(dims, dtype=np.int64)
    for h in range(len(T)):
        p = pts4[lo[h]:hi[h], :3].astype(np.float64)
        if len(p) == 0:
            continue
        w = p @ T[h, :3, :3].T + T[h, :3, 3]
        ijk = np.floor((w - origin) / cell).astype(np.int64)
        own = ijk
        ok = np.all((own >= 0) & (own < dims), axis=1)
        matched_cells.append(((own[ok, 2] * dims[1] + own[ok, 1]) * dims[0] + own[ok, 0]))
        nb = (ijk[:, None, :] + off[None, :, :]).reshape(-1, 3)
        ok = np.all((nb >= 0) & (nb < dims), axis=1)
        nb = nb[ok]
        cells.append(np.unique((nb[:, 2] * dims[1] + nb[:, 1]) * dims[0] + nb[:, 0]))
    c = np.unique(np.concatenate(cells)) if cells else np.zeros(0, np.int64)
    mc = np.unique(np.concatenate(matched_cells)) if matched_cells else np.zeros(0, np.int64)
    visited = int((start[c + 1] - start[c]).sum())
    matched = int((start[mc + 1] - start[mc]).sum())  # points sharing a cell with a query: the matches' bound
    n_pts = int(np.maximum(np.asarray(hi) - np.asarray(lo), 0).sum())
    per_iter = 16 * n_pts + 8 * len(c) + 12 * visited + 16 * matched + 2 * 32 * 8 * n_tiles
    eval_pass = 16 * n_pts + 8 * len(c) + 12 * visited
    return {"bytes": float(iters * per_iter + eval_pass), "per_iter": float(per_iter), "cells": int(len(c)),
            "visited_points": visited, "matched_points_bound": matched}
