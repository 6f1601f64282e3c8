"""Scene understanding on the visible points on a B200: ground, clusters and tracks -- the `livox_warp.perception`
module of the reference (python/livox_warp/perception.py) with its Warp kernels replaced by liblivoxb200.so.

Same public API as the reference's Perception (perception.py:391-583): ground(), cluster(), track(), the
`clusters` list of dicts (cnt, cen, lo, hi), cc_iters / cc_converged / ms, and pipe.gnd / hag / cid written for
the pipeline's visible points (pipe.c_xyz[:pipe.count]).

Differences, deliberate: the ground grid is cleared once and then restored by each call (no 32 MB fill per call);
the cluster nodes are ordered by their first point, so cluster ids are the same on every run; connected
components come from one union-find pass over a neighbour graph built from the voxel hash, so cc_iters is 1 and
cc_converged is True unless a buffer overflowed.
"""

from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from .gpu import MAX_CLUSTERS, Pipeline

GRID = 2048


class Tracker:
    """Greedy nearest-centroid tracking of clusters over sensor time (the behaviour of perception.py:274-388).

    Every update predicts each track to `now` from its last matched centroid and velocity and matches the closest
    (track, cluster) pairs first, within a gate of gate_base + gate_vel * (distance the track would have moved)
    + gate_ext * (the cluster's box diagonal). A track keeps centroid samples at least `baseline` s apart over the
    last `window` s; its velocity is their least-squares slope, reported as zero unless larger than k_sig times
    its standard error. Tracks unseen for max_age s are dropped; confirmed() lists those followed >= confirm_s.
    """

    def __init__(self, baseline: float = 0.1, window: float = 0.8, k_sig: float = 2.0, max_age: float = 0.8,
                 confirm_s: float = 0.3, gate_base: float = 0.75, gate_vel: float = 0.5, gate_ext: float = 0.25):
        self.baseline, self.window, self.k_sig, self.max_age = baseline, window, k_sig, max_age
        self.confirm_s, self.gate_base, self.gate_vel, self.gate_ext = confirm_s, gate_base, gate_vel, gate_ext
        self.tracks: dict[int, dict] = {}
        self.next_id = 0
        self.last_t = None

    def reset(self):
        self.tracks.clear()
        self.last_t = None

    def _slope(self, samples):
        if len(samples) < 2:
            return np.zeros(3)
        t = np.array([s[0] for s in samples])
        p = np.array([s[1] for s in samples])
        dt = t - t.mean()
        den = float(dt @ dt)
        if den <= 0.0:
            return np.zeros(3)
        dp = p - p.mean(axis=0)
        v = dt @ dp / den
        if len(samples) >= 3:
            resid = dp - np.outer(dt, v)
            stderr = np.sqrt((resid ** 2).sum(axis=0) / (len(samples) - 2) / den)
            if np.linalg.norm(v) < self.k_sig * np.linalg.norm(stderr):
                return np.zeros(3)
        return v

    def _fold(self, tr, c, now):
        if now - tr["samples"][-1][0] >= self.baseline - 1e-3:
            tr["samples"].append((now, c["cen"].copy()))
            tr["samples"] = [s for s in tr["samples"] if s[0] >= now - self.window - 1e-6]
            tr["vel"] = self._slope(tr["samples"])
            tr["n_meas"] += 1
        tr.update(pos=c["cen"].copy(), t=now, seen=now, lo=c["lo"].copy(), hi=c["hi"].copy(), cnt=c["cnt"])

    def update(self, clusters: list, now: float):
        """Returns per cluster its track id (int32) and velocity ((n, 3))."""
        if self.last_t is not None and now < self.last_t - 1e-6:
            self.reset()  # the sensor clock went backwards (a replay restarted)
        self.last_t = now
        ids = list(self.tracks)
        tid = np.full(len(clusters), -1, np.int32)
        vel = np.zeros((len(clusters), 3))
        if ids and clusters:
            age = np.array([max(now - self.tracks[t]["t"], 0.0) for t in ids])
            tv = np.array([self.tracks[t]["vel"] for t in ids])
            pred = np.array([self.tracks[t]["pos"] for t in ids]) + tv * age[:, None]
            cen = np.array([c["cen"] for c in clusters])
            diag = np.array([np.linalg.norm(c["hi"] - c["lo"]) for c in clusters])
            dist = np.linalg.norm(pred[:, None, :] - cen[None, :, :], axis=2)
            gate = self.gate_base + (self.gate_vel * np.linalg.norm(tv, axis=1) * age)[:, None] + self.gate_ext * diag
            taken_t, taken_c = set(), set()
            for flat in np.argsort(dist, axis=None, kind="stable"):
                a, b = divmod(int(flat), len(clusters))
                if a in taken_t or b in taken_c or dist[a, b] > gate[a, b]:
                    continue
                taken_t.add(a)
                taken_c.add(b)
                tr = self.tracks[ids[a]]
                self._fold(tr, clusters[b], now)
                tid[b], vel[b] = ids[a], tr["vel"]
        for t in [t for t, tr in self.tracks.items() if now - tr["seen"] > self.max_age]:
            del self.tracks[t]
        for b, c in enumerate(clusters):
            if tid[b] < 0:
                t = self.next_id
                self.next_id += 1
                self.tracks[t] = {"pos": c["cen"].copy(), "vel": np.zeros(3), "lo": c["lo"].copy(),
                                  "hi": c["hi"].copy(), "cnt": c["cnt"], "t": now, "seen": now, "born": now,
                                  "samples": [(now, c["cen"].copy())], "n_meas": 0}
                tid[b] = t
        return tid, vel

    def confirmed(self):
        return [(t, tr) for t, tr in self.tracks.items()
                if tr["seen"] == self.last_t and tr["n_meas"] >= 1 and tr["seen"] - tr["born"] >= self.confirm_s - 1e-3]


class Perception:
    """Ground labels, clusters and tracks of the pipeline's visible points (perception.py:391)."""

    def __init__(self, pipe: Pipeline, device=None, cluster_slots: int = 1 << 20, edge_factor: int = 64):
        _lib.load()
        self.pipe = pipe
        self.device = torch.device(device) if device is not None else pipe.device
        d = self.device
        if cluster_slots <= 0 or cluster_slots & (cluster_slots - 1):
            raise ValueError(f"cluster_slots must be a power of two, got {cluster_slots}")
        self.cell_min = torch.full((GRID * GRID,), 1.0e30, dtype=torch.float32, device=d)
        self.cell_sup = torch.zeros(GRID * GRID, dtype=torch.int32, device=d)
        n = pipe.work_cap
        c = cluster_slots
        self.cl_cap = c
        mc = MAX_CLUSTERS
        self._t = {
            "keys": torch.full((c,), -1, dtype=torch.int64, device=d),
            "acc": torch.zeros((c, 4), dtype=torch.int64, device=d),
            "first": torch.full((c,), _lib.INT32_MAX, dtype=torch.int32, device=d),
            "vidx": torch.zeros(c, dtype=torch.int32, device=d),
            "slot_of_pt": torch.zeros(n, dtype=torch.int32, device=d),
            "tiles": torch.zeros(n // 1024 + 2, dtype=torch.int32, device=d),
            "node_slot": torch.zeros(n, dtype=torch.int32, device=d),
            "v_xyz": torch.zeros((n, 3), dtype=torch.float32, device=d),
            "v_w": torch.zeros(n, dtype=torch.int32, device=d),
            "edge_off": torch.zeros(n + 1, dtype=torch.int32, device=d),
            "edges": torch.zeros(max(n * edge_factor // 8, 1 << 16), dtype=torch.int32, device=d),
            "label": torch.zeros(n, dtype=torch.int32, device=d),
            "st_sum": torch.zeros((n, 4), dtype=torch.int64, device=d),
            "st_lo": torch.full((n, 3), 1.0e30, dtype=torch.float32, device=d),
            "st_hi": torch.full((n, 3), -1.0e30, dtype=torch.float32, device=d),
            "dense": torch.full((n,), -1, dtype=torch.int32, device=d),
            "out_cnt": torch.zeros(mc, dtype=torch.float32, device=d),
            "out_cen": torch.zeros((mc, 3), dtype=torch.float32, device=d),
            "out_lo": torch.zeros((mc, 3), dtype=torch.float32, device=d),
            "out_hi": torch.zeros((mc, 3), dtype=torch.float32, device=d),
            "m": torch.zeros(1, dtype=torch.int32, device=d),
            "n_clusters": torch.zeros(2, dtype=torch.int32, device=d),
            "err": torch.zeros(1, dtype=torch.int32, device=d),
        }
        t = self._t
        self.cb = _lib.ClusterBuf(*(_lib.ptr(t[k]).value for k in _lib.ClusterBuf.PTRS), c, n, t["edges"].numel())
        self.tracker = Tracker()
        self.clusters: list[dict] = []
        self.cc_iters = 0
        self.cc_max_passes = 256
        self.cc_converged = True
        self.ms = {"ground": 0.0, "clusters": 0.0}

    # ---- ground ------------------------------------------------------------------------------------------------

    def ground(self, *, cell: float = 0.5, thick: float = 0.15, min_sup: int = 3, thresh: float = 0.2,
               slope_step: float = 0.3, use_normals: bool = False, nz_min: float = 0.7, n_dev=None, n_ub=None):
        """Label pipe.gnd / pipe.hag for the visible points (perception.py:458-483)."""
        n = self.pipe.count if n_ub is None else int(n_ub)
        if n == 0:
            return
        t0 = time.perf_counter()
        use_n = bool(use_normals and self.pipe.normals_valid)
        xyz = self.pipe.c_xyz
        _lib.call("lw_ground", _lib.ptr(xyz), xyz.shape[1], _lib.ptr(self.pipe.nrm) if use_n else None,
                  _lib.ptr(n_dev), n, float(cell), float(thick), int(min_sup), float(thresh), float(slope_step),
                  int(use_n), float(nz_min), _lib.ptr(self.cell_min), _lib.ptr(self.cell_sup), _lib.ptr(self.pipe.gnd),
                  _lib.ptr(self.pipe.hag), _lib.stream_ptr())
        self.ms["ground"] = (time.perf_counter() - t0) * 1e3

    # ---- clusters ----------------------------------------------------------------------------------------------

    def cluster(self, voxel: float = 0.1, connect: float = 0.35, min_pts: int = 30, use_ground: bool = True,
                read_back: bool = True):
        """Connected components of the (non-ground) visible points; fills pipe.cid and returns the cluster list
        (perception.py:487-510). With read_back=False nothing is copied to the host (no synchronisation)."""
        n = self.pipe.count
        self.clusters = []
        if n == 0:
            return self.clusters
        t0 = time.perf_counter()
        _lib.call("lw_cluster", _lib.ptr(self.pipe.c_xyz), self.pipe.c_xyz.shape[1], _lib.ptr(self.pipe.gnd),
                  int(use_ground), None, n, float(voxel), float(connect), float(min_pts), MAX_CLUSTERS,
                  ctypes.byref(self.cb), _lib.ptr(self.pipe.cid), _lib.stream_ptr())
        self.cc_iters = 1
        if read_back:
            t = self._t
            head = torch.cat([t["n_clusters"], t["err"]]).cpu().numpy()
            k = int(head[0])
            self.cc_converged = int(head[2]) == 0
            cnt, cen = t["out_cnt"][:k].cpu().numpy(), t["out_cen"][:k].cpu().numpy()
            lo, hi = t["out_lo"][:k].cpu().numpy(), t["out_hi"][:k].cpu().numpy()
            self.clusters = [{"cnt": float(cnt[j]), "cen": cen[j].astype(np.float64), "lo": lo[j].astype(np.float64),
                              "hi": hi[j].astype(np.float64)} for j in range(k)]
        self.ms["clusters"] = (time.perf_counter() - t0) * 1e3
        return self.clusters

    def node_labels(self) -> np.ndarray:
        """Component label (smallest node index) of every node of the last cluster() call."""
        m = int(self._t["m"].cpu()[0])
        return self._t["label"][:m].cpu().numpy()

    # ---- tracks ------------------------------------------------------------------------------------------------

    def track(self, now: float):
        """Associate the last clusters with tracks; upload per-cluster track id and velocity (perception.py:571)."""
        tid, vel = self.tracker.update(self.clusters, now)
        k = min(len(self.clusters), MAX_CLUSTERS)
        v = np.zeros((MAX_CLUSTERS, 3), np.float32)
        ti = np.full(MAX_CLUSTERS, -1, np.int32)
        v[:k], ti[:k] = vel[:k], tid[:k]
        self.pipe.cl_vel.copy_(torch.from_numpy(v))
        self.pipe.cl_tid.copy_(torch.from_numpy(ti))
        return self.tracker.confirmed()
