"""Generate the golden fixtures of tests/golden/ from the reference's own code (run in a container that has the
reference checkout; the fixtures are committed, the GPU tests only read them).

    python tests/golden/make_golden.py /path/to/livox-warp [fixture ...]

The reference's modules import NVIDIA Warp at the top, which is not installed, so they cannot be imported.
Their pure numpy / scipy functions are executed from source instead: this script parses each module with `ast`,
takes the named function definitions (and the module constants they read) verbatim, and runs them in a fresh
namespace on seeded inputs. What they produce pins the CPU oracle's restatement (oracle/oracle.py) and the
device solve:

  host_solve.npz    odom.py _sym6, _twist_between, _apply_twist, _body_twist, _twist_matrix, _sensor_basis,
                    _constrained_step; localize.py _twist_apply, _rotz, pose_difference; gpu.py mount_matrix.
  lvxr.npz          lvxr.py read_firings and Firings.points on seeded synthetic recordings (every record
                    layout, ns and GPS timestamps, clock jumps, IMU / malformed / truncated datagrams, the Mid-40
                    dual-return profile, LVXR1); lvxr.py imports only numpy and is loaded from its file.
  tracker.npz       perception.py Tracker (the class, pure numpy) driven through a seeded scene of static,
                    walking and reappearing objects, updates at 10 Hz and 144 Hz mixed, dropouts, shuffled cluster
                    order and a clock restart: the clusters given, the ids and velocities returned, the confirmed
                    tracks after every update.
  local_maxima.npz  localize.py GlobalLocalizer._local_maxima and _top (the two methods, taken out of the class)
                    on seeded coarse-score arrays with ties, occupied positions and several pool sizes.
  localize_host.npz localize.py _rot_to, ScanPrep.up_candidates / height_profile, GlobalLocalizer._heights, _nms,
                    _top, _runner_up and _unique on seeded inputs (scans with known planes, a map's levels,
                    clustered hypotheses with ties, result lists).
  prior_prepare.npz mapgrid.py PriorGrid.prepare (a static method, taken out of its class) with
                    horizontal_levels and the module constants it reads (CELL, IDX_BITS, MAX_POINTS, PLANAR; the
                    one Warp call among them, wp.constant, is the identity here).
  ref_odom.npz, ref_map.npz, ref_perception.npz, ref_localize.npz
                    the reference's Warp kernels themselves (odom.py, gpu.py, perception.py, mapgrid.py,
                    localize.py), imported unchanged against a serial stand-in for Warp (warp_shim.py) and run on
                    small seeded inputs; kernel_fixtures.py lists the kernels and how each is driven.
"""

from __future__ import annotations

import ast
import sys
from pathlib import Path

import numpy as np
from scipy.spatial.transform import Rotation

HERE = Path(__file__).resolve().parent


def extract(src_path: Path, names: list[str], consts: list[str] = ()) -> dict:
    """Run the named top-level functions / assignments of a module in a namespace with numpy and scipy."""
    tree = ast.parse(src_path.read_text())
    keep = []
    for node in tree.body:
        if isinstance(node, (ast.FunctionDef, ast.ClassDef)) and node.name in names:
            keep.append(node)
        elif isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id in consts for t in node.targets):
            keep.append(node)
    found = {n.name for n in keep if isinstance(n, (ast.FunctionDef, ast.ClassDef))}
    missing = set(names) - found
    if missing:
        raise KeyError(f"{src_path.name}: not found {sorted(missing)}")
    mod = ast.Module(body=keep, type_ignores=[])
    ns = {"np": np, "Rotation": Rotation, "math": __import__("math")}
    exec(compile(mod, str(src_path), "exec"), ns)
    return ns


def extract_methods(src_path: Path, cls: str, names: list[str]) -> type:
    """A class holding only the named methods of `cls` (its other methods and its module's imports are left out)."""
    tree = ast.parse(src_path.read_text())
    node = next(n for n in tree.body if isinstance(n, ast.ClassDef) and n.name == cls)
    body = [m for m in node.body if isinstance(m, ast.FunctionDef) and m.name in names]
    if {m.name for m in body} != set(names):
        raise KeyError(f"{src_path.name}: {cls} lacks {sorted(set(names) - {m.name for m in body})}")
    mod = ast.Module(body=[ast.ClassDef(name=cls, bases=[], keywords=[], body=body, decorator_list=[])],
                     type_ignores=[])
    ns = {"np": np, "math": __import__("math")}
    exec(compile(ast.fix_missing_locations(mod), str(src_path), "exec"), ns)
    return ns[cls]


def random_pose(rng, t_scale=5.0, r_scale=1.0):
    T = np.eye(4)
    T[:3, :3] = Rotation.from_rotvec(rng.normal(0, r_scale, 3)).as_matrix()
    T[:3, 3] = rng.normal(0, t_scale, 3)
    return T


def host_solve(ref: Path) -> dict:
    pkg = ref / "python" / "livox_warp"
    odom = extract(pkg / "odom.py", ["_sym6", "_twist_between", "_apply_twist", "_body_twist", "_twist_matrix",
                                      "_sensor_basis", "_constrained_step"], ["_TRIU6"])
    loc = extract(pkg / "localize.py", ["_twist_apply", "_rotz", "pose_difference"])
    gpu = extract(pkg / "gpu.py", ["mount_matrix"])
    rng = np.random.default_rng(20261203)
    out = {}
    n = 24
    up = rng.normal(0, 1, (n, 21))
    out["sym6_in"], out["sym6_out"] = up, np.stack([odom["_sym6"](u) for u in up])
    A = np.stack([random_pose(rng) for _ in range(n)])
    B = np.stack([A[i] @ random_pose(rng, 0.1, 0.05) for i in range(n)])
    out["tb_from"], out["tb_to"] = A, B
    out["tb_out"] = np.stack([odom["_twist_between"](A[i], B[i]) for i in range(n)])
    d = rng.normal(0, 0.05, (n, 6))
    out["apply_T"], out["apply_delta"] = A, d
    out["apply_out"] = np.stack([odom["_apply_twist"](A[i], d[i]) for i in range(n)])
    out["apply_loc_out"] = np.stack([loc["_twist_apply"](A[i], d[i]) for i in range(n)])
    D = np.stack([random_pose(rng, 0.1, 0.05) for _ in range(n)])
    out["body_in"], out["body_out"] = D, np.stack([odom["_body_twist"](x) for x in D])
    xi = rng.normal(0, 0.05, (n, 6))
    out["twm_in"], out["twm_out"] = xi, np.stack([odom["_twist_matrix"](x) for x in xi])
    L = rng.uniform(1.0, 8.0, n)
    out["sb_T"], out["sb_L"] = A, L
    out["sb_out"] = np.stack([odom["_sensor_basis"](A[i], L[i]) for i in range(n)])
    # constrained steps: normal equations of random point-to-plane problems, some with degenerate directions
    cs_A, cs_rhs, cs_Hg, cs_T, cs_L, cs_thr, cs_pred, cs_out, cs_kept = [], [], [], [], [], [], [], [], []
    for i in range(n):
        J = rng.normal(0, 1, (200, 6))
        if i % 3 == 1:
            J[:, 3] *= 1e-4  # a direction the geometry hardly constrains
        if i % 3 == 2:
            J[:, 0] *= 1e-4
            J[:, 4] *= 1e-4
        H = J.T @ J * (5.0e4 if i % 3 == 0 else 50.0)
        Hg = H * rng.uniform(0.5, 1.0)
        rhs = rng.normal(0, 10, 6)
        T = A[i]
        pred = rng.normal(0, 0.01, 6)
        thr = 3000.0
        dg = np.diag(H)
        Am = H + np.diag(1e-9 * dg.mean() + 1e-3 * dg)
        step, (_, _, kept) = odom["_constrained_step"](Am, rhs, Hg, T, L[i], thr, pred)
        cs_A.append(Am), cs_rhs.append(rhs), cs_Hg.append(Hg), cs_T.append(T), cs_L.append(L[i])
        cs_thr.append(thr), cs_pred.append(pred), cs_out.append(step), cs_kept.append(kept)
    out.update(cs_A=np.stack(cs_A), cs_rhs=np.stack(cs_rhs), cs_Hg=np.stack(cs_Hg), cs_T=np.stack(cs_T),
               cs_L=np.array(cs_L), cs_thr=np.array(cs_thr), cs_pred=np.stack(cs_pred), cs_out=np.stack(cs_out),
               cs_kept=np.stack(cs_kept))
    ang = rng.uniform(-np.pi, np.pi, n)
    out["rotz_in"], out["rotz_out"] = ang, np.stack([loc["_rotz"](a) for a in ang])
    out["pd_out"] = np.array([loc["pose_difference"](A[i], B[i]) for i in range(n)])
    mm = rng.uniform(-30, 30, (n, 6))
    out["mount_in"], out["mount_out"] = mm, np.stack([gpu["mount_matrix"](*m) for m in mm])
    return out


def prior_prepare(ref: Path) -> dict:
    """PriorGrid.prepare on a seeded small map (a few surfaces with jitter, non-unit normals, planarity)."""
    import types

    src = ref / "python" / "livox_warp" / "mapgrid.py"
    tree = ast.parse(src.read_text())
    keep = []
    for node in tree.body:
        if isinstance(node, ast.Assign) and any(isinstance(t, ast.Name) and t.id in ("CELL", "IDX_BITS", "MAX_POINTS",
                                                                                       "PLANAR") for t in node.targets):
            keep.append(node)
        elif isinstance(node, ast.FunctionDef) and node.name == "horizontal_levels":
            keep.append(node)
        elif isinstance(node, ast.ClassDef) and node.name == "PriorGrid":
            for item in node.body:
                if isinstance(item, ast.FunctionDef) and item.name == "prepare":
                    item.decorator_list = []
                    keep.append(item)
    names = {n.name for n in keep if isinstance(n, ast.FunctionDef)}
    if names != {"horizontal_levels", "prepare"}:
        raise KeyError(f"mapgrid.py: found {sorted(names)}")
    ns = {"np": np, "wp": types.SimpleNamespace(constant=lambda v: v)}
    exec(compile(ast.Module(body=keep, type_ignores=[]), str(src), "exec"), ns)
    rng = np.random.default_rng(20261204)
    pts, nrm = [], []
    for _ in range(6):  # patches of planes in a 3 x 2 x 1.5 m box
        c = rng.uniform([0, 0, 0], [3, 2, 1.5])
        u, v = np.linalg.qr(rng.normal(size=(3, 3)))[0][:, :2].T
        ab = rng.uniform(-0.6, 0.6, (900, 2))
        pts.append(c + ab[:, :1] * u + ab[:, 1:] * v + rng.normal(0, 0.003, (900, 3)))
        nrm.append(np.broadcast_to(np.cross(u, v) * rng.uniform(0.5, 2.0), (900, 3)))
    xyz = np.concatenate(pts).astype(np.float32)
    normal = np.concatenate(nrm).astype(np.float32)
    planarity = rng.uniform(0, 1, len(xyz)).astype(np.float32)
    out = ns["prepare"]({"xyz": xyz, "normal": normal, "planarity": planarity})
    lv = out["levels"]
    return {"in_xyz": xyz, "in_normal": normal, "in_planarity": planarity, "xyz": out["xyz"], "normal": out["normal"],
            "planarity": out["planarity"], "origin": out["origin"], "dims": out["dims"], "start": out["start"],
            "lo": out["lo"], "hi": out["hi"], "levels_h": lv[0], "levels_lo": np.float64(lv[1]),
            "levels_bin": np.float64(lv[2])}


# ---- LVXR recordings ---------------------------------------------------------------------------------------------
# Seeded synthetic recordings in the LVXR format (record.rs: `LVXR2\n`, dev_type, profile, then per datagram
# host_ns:u64 len:u16 and the datagram; a datagram is an 18-byte data-packet header -- version, slot, id, rsvd,
# status u32, timestamp type, data type, timestamp u64 -- and its records), decoded by the reference's own reader
# (lvxr.py imports only numpy, so it is loaded from its file).

REC_SIZE = {0: 13, 1: 9, 2: 14, 3: 10, 4: 28, 5: 16, 7: 42, 8: 22}


def _records(rng, dtype: int, n: int) -> bytes:
    """n random records of a data type; about 15 % of the returns empty (all-zero coordinates or depth)."""
    out = bytearray()
    for _ in range(n):
        def cart():
            if rng.uniform() < 0.15:
                return (0).to_bytes(12, "little")
            return b"".join(int(v).to_bytes(4, "little", signed=True) for v in rng.integers(-20000, 20000, 3))

        def sph_depth():
            return int(0 if rng.uniform() < 0.15 else rng.integers(300, 40000)).to_bytes(4, "little")

        refl, tag = int(rng.integers(0, 256)), int(rng.integers(0, 4)) << int(rng.integers(0, 3)) * 2
        if dtype == 0:
            out += cart() + bytes([refl])
        elif dtype == 2:
            out += cart() + bytes([refl, tag])
        elif dtype in (1, 3):
            out += sph_depth() + int(rng.integers(0, 18000)).to_bytes(2, "little")
            out += int(rng.integers(0, 36000)).to_bytes(2, "little") + bytes([refl] + ([tag] if dtype == 3 else []))
        elif dtype in (4, 7):
            for _ in range(2 if dtype == 4 else 3):
                out += cart() + bytes([int(rng.integers(0, 256)), int(rng.integers(0, 4))])
        else:  # 5, 8
            out += int(rng.integers(0, 18000)).to_bytes(2, "little") + int(rng.integers(0, 36000)).to_bytes(2, "little")
            for _ in range(2 if dtype == 5 else 3):
                out += sph_depth() + bytes([int(rng.integers(0, 256)), int(rng.integers(0, 4))])
    assert len(out) == n * REC_SIZE[dtype]
    return bytes(out)


def _datagram(ts_type: int, dtype: int, ts: int, body: bytes, gps=None) -> bytes:
    if gps is not None:  # (hour, microseconds in the hour)
        stamp = bytes([24, 1, 1, gps[0]]) + int(gps[1]).to_bytes(4, "little")
    else:
        stamp = int(ts).to_bytes(8, "little")
    return bytes([5, 0, 0, 0]) + (0).to_bytes(4, "little") + bytes([ts_type, dtype]) + stamp + body


def _frame(dg: bytes, host_ns: int) -> bytes:
    return int(host_ns).to_bytes(8, "little") + len(dg).to_bytes(2, "little") + dg


def lvxr_recordings(seed: int = 11) -> dict:
    rng = np.random.default_rng(seed)
    recs = {}
    # a standard Mid-40 recording: cartesian and spherical packets, an IMU packet, a malformed packet, a forward
    # clock jump, the clock going backwards (a new base), a truncated last datagram
    body, t, host = bytearray(b"LVXR2\n" + bytes([1, 0])), 5_000_000_000, 0
    for k in range(14):
        dtype = 0 if k % 3 else 1
        dg = _datagram(0, dtype, t, _records(rng, dtype, 100))
        if k == 4:
            dg = _datagram(0, 6, t, bytes(24))  # IMU: skipped
        if k == 7:
            dg = dg[:-5]  # malformed: not a whole number of records
        body += _frame(dg, host)
        t += 100 * 10_000 + (2_500_000_000 if k == 9 else 0)
        if k == 11:
            t = 1_000_000_000  # the clock restarted
        host += 1_000_000
    body += _frame(_datagram(0, 0, t, _records(rng, 0, 100)), host)[:-40]  # truncated
    recs["mid40"] = bytes(body)
    # a Horizon (fast device) with the extended, dual and triple types, ns and GPS timestamps
    body, t = bytearray(b"LVXR2\n" + bytes([3, 0])), 7_000_000_000
    for k in range(16):
        dtype = [2, 3, 4, 5, 7, 8][k % 6]
        n_rec = int(rng.integers(20, 96))
        if k % 5 == 4:
            hour, us = 2, 1_000_000 + k * 600_000
            dg = _datagram(3, dtype, 0, _records(rng, dtype, n_rec), gps=(hour, us))
        else:
            dg = _datagram(0, dtype, t, _records(rng, dtype, n_rec))
        body += _frame(dg, k)
        t += n_rec * 4_167
    recs["horizon"] = bytes(body)
    # the Mid-40 dual-return profile: plain records in pairs, 100 per packet; one packet of 98 is rejected
    body, t = bytearray(b"LVXR2\n" + bytes([1, 1])), 3_000_000_000
    for k in range(10):
        dtype = 0 if k % 2 else 1
        dg = _datagram(0, dtype, t, _records(rng, dtype, 98 if k == 6 else 100))
        body += _frame(dg, k)
        t += 50 * 10_000
    recs["dual"] = bytes(body)
    # LVXR1: no profile byte
    body, t = bytearray(b"LVXR1\n" + bytes([1])), 2_000_000_000
    for k in range(4):
        body += _frame(_datagram(0, 0, t, _records(rng, 0, 100)), k)
        t += 100 * 10_000
    recs["v1"] = bytes(body)
    return recs


def lvxr(ref: Path) -> dict:
    import importlib.util
    import tempfile

    spec = importlib.util.spec_from_file_location("ref_lvxr", ref / "python" / "livox_warp" / "lvxr.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ref_lvxr"] = mod  # its dataclasses look their module up
    spec.loader.exec_module(mod)
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, data in lvxr_recordings().items():
            path = Path(tmp) / f"{name}.lvxr"
            path.write_bytes(data)
            f = mod.read_firings(path)
            px, pa, pt, pf = f.points(clean=True, min_range=0.3)
            out.update({f"{name}_bytes": np.frombuffer(data, np.uint8), f"{name}_t": f.t, f"{name}_xyz": f.xyz,
                        f"{name}_refl": f.refl, f"{name}_tag": f.tag, f"{name}_valid": f.valid,
                        f"{name}_direction": f.direction,
                        f"{name}_meta": np.array([f.dev_type, f.profile], np.int64),
                        f"{name}_interval": np.float64(f.interval), f"{name}_pts_xyz": px, f"{name}_pts_attr": pa,
                        f"{name}_pts_t": pt, f"{name}_pts_f": pf})
    return out


def tracker_scene(seed: int = 20261204):
    """(now, clusters) per update: a static object with a wandering centroid, a large static box, a walker at
    1 m/s, a second walker that leaves for longer than max_age and comes back, a pair that cross; updates every
    0.1 s or 1/144 s at random, 10 % cluster dropouts, the clusters in random order, and the clock restarting once."""
    rng = np.random.default_rng(seed)
    times, t = [], 0.0
    while t < 3.2:
        times.append(t)
        t += 0.1 if rng.random() < 0.5 else 1.0 / 144.0
    times += [0.2 + 0.1 * k for k in range(8)]  # the sensor clock restarts (a replay loop)
    objs = [  # (start, velocity, half extent, visible(t))
        (np.array([2.0, 1.0, 0.5]), np.zeros(3), 0.2, lambda t: True),
        (np.array([-4.0, 3.0, 1.0]), np.zeros(3), 1.0, lambda t: True),
        (np.array([-3.0, -2.0, 0.9]), np.array([1.0, 0.3, 0.0]), 0.3, lambda t: True),
        (np.array([4.0, -1.0, 0.9]), np.array([-0.8, 0.0, 0.0]), 0.3, lambda t: t < 1.2 or t > 2.3),
        (np.array([0.0, 4.0, 0.9]), np.array([0.0, -1.2, 0.0]), 0.25, lambda t: True),
        (np.array([-1.0, 1.5, 0.9]), np.array([0.9, 0.0, 0.0]), 0.25, lambda t: True),
    ]
    scene = []
    for now in times:
        cl = []
        for p0, v, h, vis in objs:
            if not vis(now) or rng.random() < 0.1:
                continue
            c = p0 + v * now + rng.normal(0.0, 0.02, 3)
            e = h * (1.0 + 0.2 * rng.random())
            cl.append({"cen": c, "lo": c - e, "hi": c + e, "cnt": int(rng.integers(30, 400))})
        order = rng.permutation(len(cl))
        scene.append((now, [cl[i] for i in order]))
    return scene


def tracker(ref: Path) -> dict:
    ns = extract(ref / "python" / "livox_warp" / "perception.py", ["Tracker"])
    tr = ns["Tracker"]()
    now_l, n_l, cen, lo, hi, cnt, tid, vel, conf, n_conf = [], [], [], [], [], [], [], [], [], []
    for now, cl in tracker_scene():
        ids, v = tr.update(cl, now)
        now_l.append(now)
        n_l.append(len(cl))
        for c in cl:
            cen.append(c["cen"])
            lo.append(c["lo"])
            hi.append(c["hi"])
            cnt.append(c["cnt"])
        tid.extend(int(x) for x in ids)
        vel.extend(v)
        ok = sorted(int(t) for t, _ in tr.confirmed())
        conf.extend(ok)
        n_conf.append(len(ok))
    return {"now": np.array(now_l), "n": np.array(n_l, np.int64), "cen": np.array(cen), "lo": np.array(lo),
            "hi": np.array(hi), "cnt": np.array(cnt, np.int64), "tid": np.array(tid, np.int64),
            "vel": np.array(vel).reshape(-1, 3), "confirmed": np.array(conf, np.int64),
            "n_confirmed": np.array(n_conf, np.int64)}


def local_maxima(ref: Path) -> dict:
    """GlobalLocalizer._local_maxima and _top (localize.py:450-483) on seeded coarse-score arrays: smooth fields
    with several modes, quantised so that equal scores occur, negative (occupied) positions, and pools smaller and
    larger than the array."""
    Loc = extract_methods(ref / "python" / "livox_warp" / "localize.py", "GlobalLocalizer",
                          ["_local_maxima", "_top"])
    rng = np.random.default_rng(20261205)
    out = {}
    cases = [((2, 24, 18, 36), 400, 50), ((3, 30, 20, 60), 20000, 1 << 20), ((1, 9, 7, 12), 5000, 7)]
    for k, (shape, pool, keep) in enumerate(cases):
        nz, nx, ny, nyaw = shape
        x = np.linspace(0, 1, nx)[None, :, None, None]
        y = np.linspace(0, 1, ny)[None, None, :, None]
        a = np.linspace(0, 2 * np.pi, nyaw, endpoint=False)[None, None, None, :]
        field = np.zeros(shape)
        for _ in range(6):
            cx, cy, ca, w = rng.random(), rng.random(), rng.uniform(0, 2 * np.pi), rng.uniform(100, 900)
            field = field + w * np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / 0.02) * np.exp(np.cos(a - ca) - 1)
        field = field + rng.normal(0, 5, shape)
        sc = np.round(field / 4) * 4  # ties
        sc[rng.random(shape) < 0.15] = -1.0  # positions inside the map
        sc = sc.astype(np.float32).ravel()
        loc = Loc()
        loc._top = lambda scores, pool=pool: Loc._top(scores, pool)
        out[f"sc{k}"], out[f"shape{k}"] = sc, np.array(shape, np.int64)
        out[f"pool{k}"], out[f"keep{k}"] = np.int64(pool), np.int64(keep)
        out[f"idx{k}"] = np.asarray(loc._local_maxima(sc, shape, keep), np.int64)
    return out


def localize_host(ref: Path) -> dict:
    """The global search's host stages from localize.py, run from source on seeded inputs: _rot_to; ScanPrep's
    up_candidates and height_profile on scans with known planes (the methods taken out of the class, the open3d
    preparation replaced by the planes given); GlobalLocalizer._heights against a map's horizontal levels, _nms
    with _top, _runner_up and _unique."""
    src = ref / "python" / "livox_warp" / "localize.py"
    ns = extract(src, ["_rot_to", "_rotz", "pose_difference"])
    Prep = extract_methods(src, "ScanPrep", ["up_candidates", "height_profile"])
    Loc = extract_methods(src, "GlobalLocalizer", ["_heights", "_nms", "_top", "_runner_up", "_unique"])
    for name in ("pose_difference",):
        setattr(Loc, name, staticmethod(ns[name]))
    ns_loc = Loc._runner_up.__globals__
    ns_loc.update({"pose_difference": ns["pose_difference"], "GlobalLocalizer": Loc})
    rng = np.random.default_rng(20261206)
    out = {}
    # _rot_to: random pairs, a parallel and an antiparallel one
    a = rng.normal(0, 1, (24, 3))
    b = rng.normal(0, 1, (24, 3))
    b[0], b[1] = 2 * a[0], -3 * a[1]
    out["rot_a"], out["rot_b"] = a, b
    out["rot_out"] = np.stack([ns["_rot_to"](a[i], b[i]) for i in range(len(a))])
    # ScanPrep: a tilted floor, a ceiling, two walls and a second floor level, with the planes as open3d would
    # return them (count, unit normal, offset, indices)
    for k, tilt in enumerate((0.0, 12.0, 170.0)):
        R = Rotation.from_rotvec(np.radians(tilt) * np.array([1.0, 0.4, 0.0]) / np.linalg.norm([1.0, 0.4, 0.0]))
        R = R.as_matrix()
        parts, normals, planes, start = [], [], [], 0
        for n_w, off, cnt in (((0, 0, 1), -1.4, 900), ((0, 0, -1), 2.5, 600), ((1, 0, 0), 3.0, 700),
                              ((0, 1, 0), -2.0, 500), ((0, 0, 1), -0.6, 300), ((0.02, 0, 1), -1.38, 200)):
            n_w = np.asarray(n_w, float) / np.linalg.norm(n_w)
            u = np.cross(n_w, [0.3, 0.5, 0.7])
            u /= np.linalg.norm(u)
            v = np.cross(n_w, u)
            P = (-off) * n_w + rng.uniform(-3, 3, (cnt, 1)) * u + rng.uniform(-3, 3, (cnt, 1)) * v
            P = P + rng.normal(0, 0.005, P.shape)
            P = P @ R.T
            n_s = R @ n_w
            parts.append(P)
            normals.append(np.tile(n_s, (cnt, 1)) * rng.choice([-1, 1], (cnt, 1)))
            planes.append((cnt, n_s, float(off), np.arange(start, start + cnt)))
            start += cnt
        prep = Prep()
        prep.pts = np.concatenate(parts)
        prep.normals = np.concatenate(normals)
        prep.planes = planes
        prep.max_tilt = 45.0
        ups = prep.up_candidates()
        out[f"prep{k}_pts"], out[f"prep{k}_normals"] = prep.pts, prep.normals
        out[f"prep{k}_plane_n"] = np.array([p[1] for p in planes])
        out[f"prep{k}_plane_cnt"] = np.array([p[0] for p in planes], np.int64)
        out[f"prep{k}_plane_off"] = np.array([p[2] for p in planes])
        out[f"prep{k}_ups"] = np.array([u[0] for u in ups])
        out[f"prep{k}_support"] = np.array([u[1] for u in ups], np.int64)
        out[f"prep{k}_hprof"] = prep.height_profile(ups[0][0], -6.0, 600, 0.02)
        # _heights against a map whose horizontal levels are the scan's, lifted by 1.5 m
        lvl, _ = np.histogram(np.concatenate([np.full(900, 0.0), np.full(600, 3.9), np.full(300, 0.8)]),
                              bins=300, range=(-1.0, 5.0))

        class Grid:
            levels = (lvl.astype(np.float32), -1.0, 0.02)
            lo = np.array([0.0, 0.0, -0.2])
            hi = np.array([20.0, 10.0, 4.0])

        loc = Loc()
        loc.grid, loc.n_heights = Grid, 8
        hs = loc._heights(prep, ups[0][0])
        out[f"prep{k}_heights"] = np.array(hs if hs else [], np.float64)
    # _nms with _top: clustered hypotheses, ties, non-positive scores
    hyps = np.concatenate([rng.normal([2, 3, 1.2, 0.5], [0.08, 0.08, 0.02, 0.02], (300, 4)),
                           rng.normal([6, 1, 1.2, 2.5], [0.3, 0.3, 0.05, 0.05], (300, 4))])
    sc = np.round(rng.uniform(-5, 100, len(hyps)))
    out["nms_hyps"], out["nms_scores"] = hyps, sc
    for j, (keep, dist, ang) in enumerate(((16, 0.1, 1.5), (5, 0.3, 10.0), (100, 0.05, 0.5))):
        out[f"nms{j}"] = np.asarray(Loc._nms(hyps, sc, keep, dist, ang), np.int64)
        out[f"nms{j}_args"] = np.array([keep, dist, ang])
    # _runner_up and _unique
    poses = []
    for i in range(12):
        T = np.eye(4)
        T[:3, :3] = ns["_rotz"](rng.uniform(-0.4, 0.4) * (i % 3))
        T[:3, 3] = rng.normal(0, 0.8 * (i % 4), 3)
        poses.append(T)
    fits = np.sort(rng.uniform(0.2, 0.9, 12))[::-1]
    results = [(float(fits[i]), 0.0, 0.0, poses[i], 0, 0.0) for i in range(12)]
    out["ru_poses"], out["ru_fits"] = np.stack(poses), fits
    loc = Loc()
    loc.accept_inliers, loc.accept_gap, loc.accept_ratio = 0.45, 0.15, 0.75
    out["ru_out"] = np.array([Loc._runner_up(results[i:]) for i in range(11)])
    pairs = rng.uniform(0, 1, (40, 2))
    out["uq_pairs"] = pairs
    out["uq_out"] = np.array([loc._unique(float(p), float(q)) for p, q in pairs])
    return out


FIXTURES = {"host_solve": host_solve, "prior_prepare": prior_prepare, "lvxr": lvxr, "tracker": tracker,
            "local_maxima": local_maxima, "localize_host": localize_host}
sys.path.insert(0, str(HERE))
import kernel_fixtures  # noqa: E402 - beside this script

FIXTURES.update(kernel_fixtures.FIXTURES)


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py <reference checkout> [fixture ...]")
    ref = Path(sys.argv[1])
    for name in sys.argv[2:] or list(FIXTURES):  # optionally only the named fixtures
        np.savez_compressed(HERE / f"{name}.npz", **FIXTURES[name](ref))
        print("wrote", HERE / f"{name}.npz")


if __name__ == "__main__":
    main()
