"""Seeded synthetic LiDAR input: a Mid-40-like rosette traced into analytic scenes (the stand-in for the reference's
Warp ray-casting simulator, python/livox_warp/sources.py, which cannot run without NVIDIA Warp).

Scan pattern. The direction of the return fired at time t is a rose curve r = 0.5 * fov * sin(k * phi) with
fov = 38.4 deg and k = 7/3, phi = ROSE_RATE * t advancing uniformly, and the whole curve turned by a precession
angle psi = PRECESSION_RATE * t so that successive roses fill the field of view (the Mid-40's pattern is
non-repetitive). The rose closes after phi = 3 pi; at ROSE_RATE one closed rose takes 10 ms, and the precession
turns it by the golden angle per rose, so a 0.1 s frame holds ten rotated roses.

Scenes are unions of axis-aligned solid boxes inside an axis-aligned room (an inside-out box), plus vertical
cylinders that may move (walkers). A return is the first hit along the ray, with Gaussian range noise, a
uniform reflectivity 0-255, noise tag 0 and return index 0 (1 for the second return of a dual-return scan).
Sensor axes: x forward (the rosette's centre), y left, z up. Poses are sensor-to-world 4x4 matrices.
Everything is numpy float64 with a seeded PCG64 generator; the returned points are float32.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
from scipy.spatial.transform import Rotation

FOV_DEG = 38.4
ROSE_K = 7.0 / 3.0
ROSE_RATE = 3.0 * math.pi / 0.01          # rad/s of phi: one closed rose per 10 ms
PRECESSION_RATE = 2.399963229728653 / 0.01  # the golden angle per rose


def rosette_dirs(t: np.ndarray) -> np.ndarray:
    """Unit ray directions (sensor frame) for firing times t (s)."""
    t = np.asarray(t, dtype=np.float64)
    phi = ROSE_RATE * t
    psi = PRECESSION_RATE * t
    r = 0.5 * math.radians(FOV_DEG) * np.sin(ROSE_K * phi)  # signed angular radius
    ang = phi + psi
    u, v = r * np.cos(ang), r * np.sin(ang)
    rho = np.abs(r)
    s = np.where(rho > 1e-12, np.sin(rho) / np.maximum(rho, 1e-12), 1.0)
    d = np.stack([np.cos(rho), s * u, s * v], axis=1)
    return d / np.linalg.norm(d, axis=1, keepdims=True)


@dataclass
class Cylinder:
    """A vertical cylinder (a walker) whose axis moves back and forth along a segment at constant speed."""

    p0: np.ndarray      # xy of one end of its path
    p1: np.ndarray      # xy of the other end
    speed: float        # m/s along the path
    radius: float = 0.25
    z0: float = 0.0
    height: float = 1.8
    phase: float = 0.0  # s

    def centre(self, t: np.ndarray) -> np.ndarray:
        L = float(np.linalg.norm(self.p1 - self.p0))
        if L < 1e-9 or self.speed <= 0:
            return np.broadcast_to(self.p0, (np.size(t), 2)).copy()
        s = (np.asarray(t, dtype=np.float64) + self.phase) * self.speed
        u = np.mod(s, 2 * L)
        u = np.where(u > L, 2 * L - u, u) / L  # ping-pong
        return self.p0[None, :] + u[:, None] * (self.p1 - self.p0)[None, :]


@dataclass
class Scene:
    room_lo: np.ndarray
    room_hi: np.ndarray
    boxes: np.ndarray                   # (K, 6) x0, y0, z0, x1, y1, z1 (solid)
    cylinders: list = field(default_factory=list)

    def free(self, p: np.ndarray, margin: float) -> np.ndarray:
        """Points at least `margin` from every box and inside the room by `margin`."""
        p = np.atleast_2d(p)
        ok = np.all((p > self.room_lo + margin) & (p < self.room_hi - margin), axis=1)
        for b in self.boxes:
            inside = np.all((p > b[:3] - margin) & (p < b[3:] + margin), axis=1)
            ok &= ~inside
        return ok


def box_room(seed: int, size=(8.0, 6.0, 3.0), n_boxes: int = 20, side=(0.3, 1.5)) -> Scene:
    """An 8 x 6 x 3 m room with n axis-aligned boxes of 0.3-1.5 m sides standing on the floor."""
    rng = np.random.default_rng(seed)
    lo, hi = np.zeros(3), np.asarray(size, dtype=np.float64)
    boxes = []
    for _ in range(n_boxes):
        s = rng.uniform(side[0], side[1], 3)
        c = rng.uniform(lo[:2] + 0.2, hi[:2] - 0.2)
        b0 = np.array([c[0] - s[0] / 2, c[1] - s[1] / 2, 0.0])
        boxes.append(np.concatenate([np.maximum(b0, lo), np.minimum(b0 + s, hi)]))
    return Scene(lo, hi, np.array(boxes))


def office(seed: int, size=(40.0, 30.0, 3.0), rooms=(4, 3), n_boxes: int = 200, walkers: int = 0,
           walker_speed: float = 1.2) -> Scene:
    """A multi-room office: outer walls, a grid of 0.1 m internal walls with 1 m door gaps, n boxes and walkers."""
    rng = np.random.default_rng(seed)
    lo, hi = np.zeros(3), np.asarray(size, dtype=np.float64)
    H = hi[2]
    walls = []
    th = 0.1
    nx, ny = rooms
    for i in range(1, nx):  # walls of constant x, with one door per room they bound
        x = hi[0] * i / nx
        edges = np.linspace(0, hi[1], ny + 1)
        for j in range(ny):
            d = rng.uniform(edges[j] + 0.8, edges[j + 1] - 1.8)
            walls.append([x - th / 2, edges[j], 0, x + th / 2, d, H])
            walls.append([x - th / 2, d + 1.0, 0, x + th / 2, edges[j + 1], H])
    for j in range(1, ny):
        y = hi[1] * j / ny
        edges = np.linspace(0, hi[0], nx + 1)
        for i in range(nx):
            d = rng.uniform(edges[i] + 0.8, edges[i + 1] - 1.8)
            walls.append([edges[i], y - th / 2, 0, d, y + th / 2, H])
            walls.append([d + 1.0, y - th / 2, 0, edges[i + 1], y + th / 2, H])
    wall_scene = Scene(lo, hi, np.array(walls, dtype=np.float64))
    boxes = list(walls)
    placed, attempts = 0, 0
    while placed < n_boxes:
        attempts += 1
        if attempts > 200000:
            raise RuntimeError("could not place the office boxes")
        s = rng.uniform(0.3, 1.5, 3)
        c = rng.uniform(lo[:2] + 0.5, hi[:2] - 0.5)
        b = np.array([c[0] - s[0] / 2, c[1] - s[1] / 2, 0.0, c[0] + s[0] / 2, c[1] + s[1] / 2, s[2]])
        # keep the doors and a corridor along every wall free (boxes may touch each other)
        mg = 0.7 + 0.5 * s[:2].max()
        if np.any(c - mg < lo[:2]) or np.any(c + mg > hi[:2]):
            continue
        W = wall_scene.boxes
        if np.any(np.all((c[None, :] > W[:, :2] - mg) & (c[None, :] < W[:, 3:5] + mg), axis=1)):
            continue
        boxes.append(b)
        placed += 1
    scene = Scene(lo, hi, np.array(boxes, dtype=np.float64))
    for w in range(walkers):
        for _ in range(20000):
            a = rng.uniform(lo[:2] + 1.0, hi[:2] - 1.0)
            ang = rng.uniform(0, 2 * math.pi)
            b = a + 4.0 * np.array([math.cos(ang), math.sin(ang)])
            seg = np.linspace(0, 1, 20)[:, None] * (b - a) + a
            pts = np.concatenate([seg, np.full((20, 1), 0.9)], axis=1)
            if scene.free(pts, margin=0.4).all():
                scene.cylinders.append(Cylinder(a, b, walker_speed, phase=rng.uniform(0, 10)))
                break
    return scene


# ---- ray casting -----------------------------------------------------------------------------------------


def raycast(o: np.ndarray, d: np.ndarray, scene: Scene, t: np.ndarray, chunk: int = 8192) -> np.ndarray:
    """Distance to the first surface along each ray (inf where none); o, d (n, 3), d unit; t firing times."""
    n = len(o)
    out = np.full(n, np.inf)
    B = scene.boxes
    for a in range(0, n, chunk):
        b = min(n, a + chunk)
        oo, dd = o[a:b], d[a:b]
        inv = 1.0 / np.where(np.abs(dd) < 1e-12, np.copysign(1e-12, dd), dd)
        # the room from inside: the exit distance
        t_room = np.min(np.where(dd > 0, (scene.room_hi - oo) * inv, (scene.room_lo - oo) * inv), axis=1)
        best = t_room
        if len(B):
            t1 = (B[None, :, :3] - oo[:, None, :]) * inv[:, None, :]
            t2 = (B[None, :, 3:] - oo[:, None, :]) * inv[:, None, :]
            tn = np.max(np.minimum(t1, t2), axis=2)
            tf = np.min(np.maximum(t1, t2), axis=2)
            hit = (tn <= tf) & (tn > 1e-6)
            tb = np.where(hit, tn, np.inf).min(axis=1)
            best = np.minimum(best, tb)
        for cyl in scene.cylinders:
            c = cyl.centre(t[a:b])
            ox, oy = oo[:, 0] - c[:, 0], oo[:, 1] - c[:, 1]
            A = dd[:, 0] ** 2 + dd[:, 1] ** 2
            Bq = 2 * (ox * dd[:, 0] + oy * dd[:, 1])
            Cq = ox ** 2 + oy ** 2 - cyl.radius ** 2
            disc = Bq ** 2 - 4 * A * Cq
            ok = (disc >= 0) & (A > 1e-12)
            sq = np.sqrt(np.maximum(disc, 0))
            tc = (-Bq - sq) / np.maximum(2 * A, 1e-12)
            z = oo[:, 2] + tc * dd[:, 2]
            ok &= (tc > 1e-6) & (z >= cyl.z0) & (z <= cyl.z0 + cyl.height)
            best = np.minimum(best, np.where(ok, tc, np.inf))
        out[a:b] = best
    return out


# ---- trajectories -----------------------------------------------------------------------------------------


def _pose(R: np.ndarray, p: np.ndarray) -> np.ndarray:
    T = np.zeros(R.shape[:-2] + (4, 4))
    T[..., :3, :3] = R
    T[..., :3, 3] = p
    T[..., 3, 3] = 1.0
    return T


class ConstantVelocity:
    """At rest at T0 until t_start, then constant body velocity (v forward m/s, yaw rate rad/s)."""

    def __init__(self, T0: np.ndarray, t_start: float, v: float, yaw_rate: float):
        self.T0, self.t_start, self.v, self.w = np.asarray(T0, np.float64), t_start, v, yaw_rate

    def poses(self, t: np.ndarray) -> np.ndarray:
        s = np.maximum(np.asarray(t, np.float64) - self.t_start, 0.0)
        yaw = self.w * s
        # integrate a unicycle: forward speed v along the heading, heading turning at w
        if abs(self.w) > 1e-12:
            dx = self.v / self.w * np.sin(yaw)
            dy = self.v / self.w * (1 - np.cos(yaw))
        else:
            dx, dy = self.v * s, np.zeros_like(s)
        Rz = Rotation.from_euler("z", yaw[:, None]).as_matrix()
        R0 = self.T0[:3, :3]
        R = R0[None] @ Rz
        p = self.T0[:3, 3][None, :] + (R0[None] @ np.stack([dx, dy, np.zeros_like(dx)], axis=1)[..., None])[..., 0]
        return _pose(R, p)


class Handheld:
    """A smooth handheld path: rest for `rest` s, then a Catmull-Rom spline through random free waypoints at a
    cruise speed under v_max, with the sensor turned toward a look-at point drifting around the room's middle
    (yaw rate under w_max, yaw acceleration under a_max), pitched ~10 deg down, with small pitch/roll sway.
    """

    def __init__(self, scene: Scene, seed: int, duration: float, v_max: float = 1.0, w_max_deg: float = 60.0,
                 rest: float = 1.0, height=(1.2, 1.7), margin: float = 0.7, a_max_deg: float = 120.0):
        rng = np.random.default_rng(seed)
        self.rest, self.duration = rest, duration
        pts = []
        while len(pts) < 2 or self._length(pts) < v_max * (duration - rest) * 0.8:
            for _ in range(10000):
                c = rng.uniform(scene.room_lo + margin, scene.room_hi - margin)
                c[2] = rng.uniform(*height)
                if scene.free(c, margin)[0] and (not pts or np.linalg.norm(c - pts[-1]) > 1.0):
                    seg = np.linspace(0, 1, 25)[:, None] * (c - pts[-1]) + pts[-1] if pts else c[None]
                    if scene.free(seg, margin * 0.8).all():
                        pts.append(c)
                        break
            else:
                raise RuntimeError("could not place a waypoint")
            if len(pts) > 400:
                break
        P = np.array(pts)
        P = np.vstack([P[0], P, P[-1]])  # clamp the spline ends
        self.P = P
        # sample the spline densely, arc-length parametrise, time at a speed profile under v_max
        us = np.linspace(0, len(P) - 3, (len(P) - 3) * 200 + 1)
        xyz = self._spline(us)
        # a hand does not turn a corner instantly: where the spline kinks at a waypoint, round it off -- resample
        # every 1 cm of arc length and smooth with a Gaussian of 0.25 m along the path (the ends held)
        seglen = np.linalg.norm(np.diff(xyz, axis=0), axis=1)
        s = np.concatenate([[0.0], np.cumsum(seglen)])
        su = np.arange(0.0, s[-1], 0.01)
        xyz = np.stack([np.interp(su, s, xyz[:, k]) for k in range(3)], 1)
        g = np.exp(-0.5 * (np.arange(-75, 76) / 25.0) ** 2)
        g /= g.sum()
        pad = np.concatenate([np.repeat(xyz[:1], 75, 0), xyz, np.repeat(xyz[-1:], 75, 0)])
        xyz = np.stack([np.convolve(pad[:, k], g, mode="valid") for k in range(3)], 1)
        seglen = np.linalg.norm(np.diff(xyz, axis=0), axis=1)
        s = np.concatenate([[0.0], np.cumsum(seglen)])
        T_move = duration - rest
        v = min(v_max * 0.7, s[-1] / max(T_move * 0.6, 1e-3))  # cruise; the spline's bends stay under v_max
        ramp = 0.8  # s to reach cruise speed, so the first moving frames look like a hand starting to move
        # speed along the path: the cruise speed, slower in bends (sideways acceleration at most a_lat), speeding up
        # and slowing down at most a_lon (the ramp's), from rest at the start
        a_lon, a_lat = v / ramp, 2.5 * max(v_max, 1.0)
        d1 = np.gradient(xyz, s, axis=0)
        d2 = np.gradient(d1, s, axis=0)
        kappa = np.linalg.norm(np.cross(d1, d2), axis=1) / np.maximum(np.linalg.norm(d1, axis=1) ** 3, 1e-12)
        vv = np.minimum(v, np.sqrt(a_lat / np.maximum(kappa, 1e-9)))
        vv[0] = 0.0
        ds = np.diff(s)
        for i in range(1, len(vv)):
            vv[i] = min(vv[i], math.sqrt(vv[i - 1] ** 2 + 2.0 * a_lon * ds[i - 1]))
        for i in range(len(vv) - 2, 0, -1):
            vv[i] = min(vv[i], math.sqrt(vv[i + 1] ** 2 + 2.0 * a_lon * ds[i]))
        t_of_s = np.concatenate([[0.0], np.cumsum(2.0 * ds / np.maximum(vv[1:] + vv[:-1], 1e-6))])

        def s_of(tau):
            return np.interp(np.clip(tau, 0, None), t_of_s, s)
        self._s, self._xyz, self._s_of = s, xyz, s_of
        # yaw: a handheld scan keeps the room in view -- the sensor points from where it is toward a look-at
        # point that drifts around the room's middle, smoothed over 1 s (causal) and rate-limited to w_max, plus
        # a small random sway; a slight downward pitch sees the floor ahead
        self.dt = 0.002
        tt = np.arange(0.0, duration + 1.0, self.dt)
        pos = self._position(tt)
        mid = 0.5 * (scene.room_lo + scene.room_hi)
        half = 0.15 * (scene.room_hi - scene.room_lo)
        lf, lph = rng.uniform(0.02, 0.06, 2), rng.uniform(0, 2 * math.pi, 2)
        centre = np.stack([mid[0] + half[0] * np.sin(2 * math.pi * lf[0] * tt + lph[0]),
                           mid[1] + half[1] * np.sin(2 * math.pi * lf[1] * tt + lph[1])], axis=1)
        # look across the room: through a point near its middle, toward the far side
        away = centre - pos[:, :2]
        near = np.linalg.norm(away, axis=1) < 0.8
        heading = np.arctan2(away[:, 1], away[:, 0])
        for i in range(1, len(heading)):  # right at the middle: keep the last direction
            if near[i]:
                heading[i] = heading[i - 1]
        heading = np.unwrap(heading)
        heading[tt <= rest] = heading[int(np.searchsorted(tt, rest))]  # at rest the sensor holds still
        win = max(1, int(1.0 / self.dt))
        smooth = np.convolve(np.pad(heading, (win - 1, 0), mode="edge"), np.ones(win) / win, mode="valid")
        sway_f, sway_ph = rng.uniform(0.1, 0.3, 2), rng.uniform(0, 2 * math.pi, 2)
        sway = sum(math.radians(8.0) * np.sin(2 * math.pi * f * tt + ph) for f, ph in zip(sway_f, sway_ph))
        want = smooth + sway * (tt > rest)
        # a critically damped follower with the yaw rate capped at w_max and the yaw acceleration at a_max, so
        # turns start and stop the way a hand moves (no step in angular velocity)
        wmax = math.radians(w_max_deg) * 0.95
        amax = math.radians(a_max_deg)
        yaw = np.empty_like(want)
        yaw[0] = want[0]
        rate = 0.0
        k_p = 4.0  # 1/s: how fast the follower closes a heading error
        for i in range(1, len(want)):
            target = np.clip(k_p * (want[i] - yaw[i - 1]), -wmax, wmax)
            rate += np.clip(target - rate, -amax * self.dt, amax * self.dt)
            yaw[i] = yaw[i - 1] + rate * self.dt
        self._yaw = yaw
        self.tilt = rng.uniform(-1, 1, 4) * math.radians(3.0)
        self.pitch0 = math.radians(10.0)

    @staticmethod
    def _length(pts):
        return sum(np.linalg.norm(b - a) for a, b in zip(pts[:-1], pts[1:]))

    def _spline(self, u):
        P = self.P
        i = np.clip(np.floor(u).astype(int), 0, len(P) - 4)
        f = (u - i)[:, None]
        p0, p1, p2, p3 = P[i], P[i + 1], P[i + 2], P[i + 3]
        return 0.5 * ((2 * p1) + (-p0 + p2) * f + (2 * p0 - 5 * p1 + 4 * p2 - p3) * f ** 2 +
                      (-p0 + 3 * p1 - 3 * p2 + p3) * f ** 3)

    def _position(self, t: np.ndarray) -> np.ndarray:
        tau = np.clip(np.asarray(t, np.float64) - self.rest, 0.0, None)
        s = np.minimum(self._s_of(tau), self._s[-1])
        idx = np.clip(np.searchsorted(self._s, s), 1, len(self._s) - 1)
        f = ((s - self._s[idx - 1]) / np.maximum(self._s[idx] - self._s[idx - 1], 1e-12))[:, None]
        return self._xyz[idx - 1] * (1 - f) + self._xyz[idx] * f

    def poses(self, t: np.ndarray) -> np.ndarray:
        t = np.asarray(t, np.float64)
        p = self._position(t)
        yaw = np.interp(t, np.arange(len(self._yaw)) * self.dt, self._yaw)
        tm = np.where(t > self.rest, t - self.rest, 0.0)
        pitch = self.pitch0 + self.tilt[0] * np.sin(0.3 * tm) + self.tilt[1] * np.sin(0.17 * tm)
        roll = self.tilt[2] * np.sin(0.23 * tm) + self.tilt[3] * np.sin(0.11 * tm)
        R = Rotation.from_euler("zyx", np.stack([yaw, pitch, roll], axis=1)).as_matrix()
        return _pose(R, p)


# ---- scans ------------------------------------------------------------------------------------------------


def scan(scene: Scene, traj, t0: float, t1: float, rate: float, seed: int, noise: float = 0.02,
         dual: bool = False, max_range: float = 200.0):
    """Returns fired at `rate` per second over [t0, t1): (xyz float32 (n,3) in each return's own sensor frame,
    attr uint32, t float32). With dual, each ray gives two returns (index 0 and 1) with independent noise."""
    i0 = int(math.ceil(t0 * rate - 1e-9))
    i1 = int(math.ceil(t1 * rate - 1e-9))
    idx = np.arange(i0, i1, dtype=np.int64)
    t = idx / rate
    d = rosette_dirs(t)
    T = traj.poses(t)
    o = T[:, :3, 3]
    dw = (T[:, :3, :3] @ d[..., None])[..., 0]
    rng = np.random.default_rng([seed, i0])
    rng_hit = raycast(o, dw, scene, t)
    ok = np.isfinite(rng_hit) & (rng_hit < max_range)
    n_ret = 2 if dual else 1
    xs, ats, ts = [], [], []
    for r in range(n_ret):
        rr = rng_hit + rng.normal(0.0, noise, len(t))
        refl = rng.integers(0, 256, len(t)).astype(np.uint32)
        xyz = d * rr[:, None]
        attr = refl | (np.uint32(r) << np.uint32(16))
        xs.append(xyz[ok])
        ats.append(attr[ok])
        ts.append(t[ok])
    if dual:
        # interleave the two returns of each ray, in firing order
        xyz = np.stack(xs, axis=1).reshape(-1, 3)
        attr = np.stack(ats, axis=1).reshape(-1)
        tt = np.stack(ts, axis=1).reshape(-1)
    else:
        xyz, attr, tt = xs[0], ats[0], ts[0]
    return xyz.astype(np.float32), attr.astype(np.uint32), tt.astype(np.float32)


def frames(scene: Scene, traj, n_frames: int, rate: float, seed: int, frame_dt: float = 0.1, start: int = 0,
           **kw):
    """Per-frame scans [(xyz, attr, t)] of frames start .. start + n_frames - 1."""
    return [scan(scene, traj, (start + k) * frame_dt, (start + k + 1) * frame_dt, rate, seed, **kw)
            for k in range(n_frames)]


def sample_surfaces(scene: Scene, spacing: float, seed: int, jitter: float = 0.0):
    """Points on every visible face of the scene's room and boxes on a `spacing` grid, with unit normals and a
    planarity of 1 (the prior map of a global-localisation case). Faces inside other boxes are kept."""
    rng = np.random.default_rng(seed)
    pts, nrm = [], []

    def face(origin, u, v, n):
        lu, lv = np.linalg.norm(u), np.linalg.norm(v)
        nu, nv = max(int(lu / spacing), 1), max(int(lv / spacing), 1)
        a, b = np.meshgrid((np.arange(nu) + 0.5) / nu, (np.arange(nv) + 0.5) / nv, indexing="ij")
        p = origin + a.reshape(-1, 1) * u + b.reshape(-1, 1) * v
        if jitter:
            p = p + rng.normal(0, jitter, p.shape)
        pts.append(p)
        nrm.append(np.broadcast_to(n, p.shape))

    lo, hi = scene.room_lo, scene.room_hi
    ex, ey, ez = np.eye(3)
    size = hi - lo
    face(lo, ex * size[0], ey * size[1], ez)                         # floor
    face(lo + ez * size[2], ex * size[0], ey * size[1], -ez)         # ceiling
    face(lo, ex * size[0], ez * size[2], ey)                         # y = lo wall
    face(lo + ey * size[1], ex * size[0], ez * size[2], -ey)
    face(lo, ey * size[1], ez * size[2], ex)
    face(lo + ex * size[0], ey * size[1], ez * size[2], -ex)
    for b in scene.boxes:
        b0, b1 = b[:3], b[3:]
        s = b1 - b0
        face(b0 + ez * s[2], ex * s[0], ey * s[1], ez)
        face(b0, ex * s[0], ez * s[2], -ey)
        face(b0 + ey * s[1], ex * s[0], ez * s[2], ey)
        face(b0, ey * s[1], ez * s[2], -ex)
        face(b0 + ex * s[0], ey * s[1], ez * s[2], ex)
    return np.concatenate(pts).astype(np.float32), np.concatenate(nrm).astype(np.float32)


# ---- global localisation cases -----------------------------------------------------------------------------------


def spin_scan(scene: Scene, T: np.ndarray, n: int, seed: int, noise: float = 0.01, elev_deg=(-7.0, 52.0),
              max_range: float = 40.0) -> np.ndarray:
    """A static 360-degree scan from pose T (sensor to world): n rays with azimuth uniform in [0, 2 pi) and
    elevation uniform in elev_deg (a Mid-360-like field of view), Gaussian range noise; the (m <= n) hits in the
    sensor frame, float32."""
    rng = np.random.default_rng(seed)
    az = rng.uniform(0.0, 2.0 * math.pi, n)
    el = np.radians(rng.uniform(elev_deg[0], elev_deg[1], n))
    d = np.stack([np.cos(el) * np.cos(az), np.cos(el) * np.sin(az), np.sin(el)], axis=1)
    T = np.asarray(T, dtype=np.float64)
    o = np.broadcast_to(T[:3, 3], (n, 3))
    dw = d @ T[:3, :3].T
    r = raycast(np.ascontiguousarray(o), dw, scene, np.zeros(n))
    ok = np.isfinite(r) & (r < max_range)
    rr = r + rng.normal(0.0, noise, n)
    return (d * rr[:, None])[ok].astype(np.float32)


def tls_scan(scene: Scene, stations, seed: int, step_deg: float = 0.2, elevation_deg=(-60.0, 89.0),
             noise: float = 0.002, t: float = 0.0) -> np.ndarray:
    """A terrestrial scanner's capture of the scene (the reference's sources.tls_scan, sources.py:884-899): a
    spherical grid of rays step_deg apart over the elevation range from each station, Gaussian range noise; the
    world points (n, 3) float32 of the rays that hit a surface."""
    rng = np.random.default_rng(seed)
    st = np.asarray(stations, dtype=np.float64).reshape(-1, 3)
    n_az = int(round(360.0 / step_deg))
    n_el = int((elevation_deg[1] - elevation_deg[0]) / step_deg) + 1
    az = np.radians(np.arange(n_az) * step_deg)
    el = np.radians(elevation_deg[0] + np.arange(n_el) * step_deg)
    A, E = np.meshgrid(az, el, indexing="ij")
    d = np.stack([np.cos(E) * np.cos(A), np.cos(E) * np.sin(A), np.sin(E)], axis=-1).reshape(-1, 3)
    out = []
    for o in st:
        oo = np.broadcast_to(o, d.shape)
        r = raycast(np.ascontiguousarray(oo), d, scene, np.full(len(d), t), chunk=1 << 15)
        ok = np.isfinite(r)
        rr = r[ok] + rng.normal(0.0, noise, int(ok.sum()))
        out.append(o + d[ok] * rr[:, None])
    pts = np.concatenate(out) if out else np.zeros((0, 3))
    return pts[np.abs(pts).max(axis=1) < 1.0e3].astype(np.float32)


def free_poses(scene: Scene, n: int, seed: int, z: float = 1.2, margin: float = 0.6, grid: float = 0.0):
    """n sensor poses in free space at height z with yaw uniform in [0, 2 pi): (T (n, 4, 4) sensor to world).
    With grid > 0 the positions lie on that xy grid (distinct cells, drawn without replacement)."""
    rng = np.random.default_rng(seed)
    out = []
    if grid > 0:
        xs = np.arange(scene.room_lo[0] + grid, scene.room_hi[0], grid)
        ys = np.arange(scene.room_lo[1] + grid, scene.room_hi[1], grid)
        P = np.stack(np.meshgrid(xs, ys, indexing="ij"), axis=-1).reshape(-1, 2)
        P = np.concatenate([P, np.full((len(P), 1), z)], axis=1)
        P = P[scene.free(P, margin)]
        if len(P) < n:
            raise RuntimeError(f"only {len(P)} free grid positions for {n} poses")
        P = P[rng.choice(len(P), n, replace=False)]
    else:
        P = np.zeros((0, 3))
        while len(P) < n:
            c = np.concatenate([rng.uniform(scene.room_lo[:2], scene.room_hi[:2], (4 * n, 2)),
                                np.full((4 * n, 1), z)], axis=1)
            P = np.concatenate([P, c[scene.free(c, margin)]])[:n]
    yaw = rng.uniform(0.0, 2.0 * math.pi, n)
    for p, a in zip(P, yaw):
        out.append(_pose(Rotation.from_euler("z", a).as_matrix(), p))
    return np.stack(out)


def perturb(T: np.ndarray, seed: int, trans: float, yaw_deg: float, tilt_deg: float = 0.0) -> np.ndarray:
    """Poses T (n, 4, 4) moved by a uniform xy offset of at most `trans` per axis, a yaw of at most yaw_deg and
    a roll / pitch of at most tilt_deg (a coarse search's quantisation error)."""
    rng = np.random.default_rng(seed)
    T = np.array(T, dtype=np.float64, copy=True)
    n = len(T)
    dxy = rng.uniform(-trans, trans, (n, 2))
    ang = np.radians(np.stack([rng.uniform(-tilt_deg, tilt_deg, n), rng.uniform(-tilt_deg, tilt_deg, n),
                               rng.uniform(-yaw_deg, yaw_deg, n)], axis=1))
    for i in range(n):
        R = Rotation.from_euler("xyz", ang[i]).as_matrix()
        T[i, :3, :3] = R @ T[i, :3, :3]
        T[i, :2, 3] += dxy[i]
    return T


def look_at(p, target) -> np.ndarray:
    """Sensor-to-world pose at p with the sensor's x axis toward target (no roll)."""
    p = np.asarray(p, np.float64)
    d = np.asarray(target, np.float64) - p
    yaw = math.atan2(d[1], d[0])
    pitch = -math.atan2(d[2], np.linalg.norm(d[:2]))
    T = np.eye(4)
    T[:3, :3] = Rotation.from_euler("zyx", [yaw, pitch, 0.0]).as_matrix()
    T[:3, 3] = p
    return T


def single_frame_case(scene: Scene, n_frames: int, rate: float = 100000.0, map_frames: int = 10,
                      v: float = 0.5, yaw_rate_deg: float = 20.0, map_seed: int = 21, seed: int = 100):
    """The single-frame scan-to-map ICP case: a sensor in a corner of the box room, looking across it and slightly
    down, holds still for map_frames frames (they build the map), then moves at v m/s forward while turning at
    yaw_rate_deg deg/s. Returns (T0, map frames [(xyz, attr, t)], moving frames [(xyz, attr, t, t_mid, T_true)]):
    moving frame j is the first 0.1 s of motion of a sensor that starts moving at 1.0 + 0.1 j s, so each is a
    fresh rosette pattern taken while moving, its points in the sensor frame at their own firing times."""
    T0 = look_at([0.8, 0.8, 1.6], [7.0, 5.0, 1.0])
    static = ConstantVelocity(T0, 1e9, 0.0, 0.0)
    base = frames(scene, static, map_frames, rate, map_seed)
    moving = []
    for j in range(n_frames):
        t0 = 0.1 * map_frames + 0.1 * j
        mover = ConstantVelocity(T0, t0, v, math.radians(yaw_rate_deg))
        x, a, t = scan(scene, mover, t0, t0 + 0.1, rate, seed + j)
        moving.append((x, a, t, t0 + 0.05, mover.poses(np.array([t0 + 0.05]))[0]))
    return T0, base, moving
