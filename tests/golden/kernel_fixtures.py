"""Fixtures from the reference's own kernels: their unchanged source executed under tests/golden/warp_shim.py (a
serial stand-in for NVIDIA Warp) on small seeded inputs. make_golden.py registers these; the fixtures hold the
inputs and what the reference's kernels produced from them, and tests/test_ref_kernels_cpu.py holds the oracle
(oracle/lw_oracle.cpp, oracle/oracle.py) to them.

  ref_odom.npz        odom.py k_ds_insert (:126-160), k_deskew (:163-178), k_reg_insert (:186-230), k_icp with
                      accumulate / accumulate_h and k_reduce (:233-384).
  ref_map.npz         gpu.py k_map_insert (:373-412), k_carve with local_plane / map_centroid (:415-593, every
                      return and every other one), k_classify_map with transient / ghost / settled_near
                      (:286-299, :596-634, :699-747), in a room with a walker crossing it.
  ref_perception.npz  perception.py k_gnd_min / k_gnd_support / k_gnd_label (:39-111, with and without normals);
                      k_cl_insert (:114-139), gpu.py k_nb_flag / k_total / k_nb_compact (:772, :806-827),
                      k_cc_init / k_cc_step / k_cc_jump (:142-179), k_cc_reset / k_cc_stats / k_cc_flag /
                      k_cc_compact / k_cc_gather (:182-271), driven as Perception._voxelize / _label / _compact
                      drive them (:512-567).
  ref_localize.npz    mapgrid.py PriorGrid.prepare (:216-243) and the grid build k_seed / k_unpack / k_jfa / k_df
                      (:105-170, driven as PriorGrid.build :272-296); localize.py k_icp_batch with nearest_point
                      and k_reduce_batch (:126-179) driven as GlobalLocalizer._icp (:517-553), and k_eval_batch
                      (:182-205).

The host loops that drive the kernels (the label passes, the ICP schedule, the scans between compactions) are
restated here from the reference lines cited at each; everything a kernel computes comes from its source.
"""

from __future__ import annotations

import math
from pathlib import Path
from types import SimpleNamespace

import numpy as np
from scipy.spatial.transform import Rotation

import warp_shim as ws

RATE = 100000.0
POSE_SLOTS = 1 << 16


def _ref(ref: Path):
    return ws.load_reference(Path(ref) / "python" / "livox_warp")


def _synth():
    import sys

    root = Path(__file__).resolve().parents[2]
    for p in (str(root / "livox-warp_b200"),):
        if p not in sys.path:
            sys.path.insert(0, p)
    from livox_warp import synth

    return synth


# ---- odometry ----------------------------------------------------------------------------------------------------


def ref_odom(ref: Path) -> dict:
    R = _ref(ref)
    synth = _synth()
    room = synth.box_room(1)
    out = {}
    # thinning of a handheld frame (sensor frame), some returns noise-tagged or outside the return mask
    tr = synth.Handheld(room, 2, 20.0)
    x, a, t = synth.scan(room, tr, 1.1, 1.2, RATE, 3)
    x, a, t = x[:3000].copy(), a[:3000].copy(), t[:3000].copy()
    a[::17] |= np.uint32(1 << 8)
    a[::23] |= np.uint32(2 << 16)
    voxel = 0.15
    inv_v = np.float32(2.0 / voxel)
    m = len(x)
    keys = np.full(1 << 13, -1, np.int64)
    count = np.zeros(1, np.int32)
    ds = np.zeros((m, 3), np.float32)
    R.odom.k_ds_insert.launch(m, x, a, m, inv_v, 0.3, 60.0, 0b0011, len(keys) - 1, keys, count, ds)
    out.update(thin_x=x, thin_a=a, thin_t=t, thin_inv_v=inv_v, thin_ret_mask=np.int32(0b0011),
               thin_out=ds[:count[0]].copy())
    # deskew of the same frame with a twist
    tw = np.array([0.05, -0.02, 0.01, 0.01, -0.03, 0.035], np.float32)
    dk = np.zeros((m, 3), np.float32)
    R.odom.k_deskew.launch(m, x, t, m, 1.15, 10.0, tw[:3], tw[3:], dk)
    out.update(deskew_tw=tw, deskew_t_mid=np.float64(1.15), deskew_out=dk)
    # the registration map of three static frames at a corner pose, 0.2 m voxels
    T0 = synth.look_at([0.8, 0.8, 1.6], [7.0, 5.0, 1.0])
    static = synth.ConstantVelocity(T0, 1e9, 0.0, 0.0)
    cap = 1 << 14
    rk = np.full(cap, -1, np.int64)
    rsum = np.zeros((cap, 3), np.float32)
    rout = np.zeros((cap, 3, 3), np.float32)
    rcnt = np.zeros(cap, np.int32)
    st = np.zeros(2, np.int32)
    vox = 0.2
    T32 = T0.astype(np.float32)
    xs, as_, ts = [], [], []
    for fx, fa, ft in synth.frames(room, static, 3, RATE, seed=21):
        fx, fa, ft = fx[:2000], fa[:2000], ft[:2000]
        R.odom.k_reg_insert.launch(len(fx), fx, fa, len(fx), T32, np.float32(1.0 / vox), vox, 60.0, 0b1111, cap - 1,
                                   rk, rsum, rout, rcnt, st)
        xs.append(fx), as_.append(fa), ts.append(ft)
    out.update(reg_x=np.stack(xs), reg_a=np.stack(as_), reg_t=np.stack(ts), reg_T=T0, reg_voxel=np.float64(vox),
               reg_keys=rk, reg_sum=rsum, reg_outer=rout, reg_cnt=rcnt, reg_stats=st)
    # one Gauss-Newton accumulation of a moving frame's thinned points at the start pose, wide and narrow
    mover = synth.ConstantVelocity(T0, 1.0, 0.5, math.radians(20.0))
    mx, ma, mt = synth.scan(room, mover, 1.0, 1.1, RATE, seed=99)
    mkeys = np.full(1 << 15, -1, np.int64)
    mcount = np.zeros(1, np.int32)
    mds = np.zeros((len(mx), 3), np.float32)
    R.odom.k_ds_insert.launch(len(mx), mx, ma, len(mx), np.float32(2.0 / vox), 0.3, 60.0, 0b1111, len(mkeys) - 1,
                              mkeys, mcount, mds)
    icp_pts = mds[:min(int(mcount[0]), 1500)].copy()
    n = len(icp_pts)
    tight2 = (0.6 * vox / math.sqrt(12.0)) ** 2
    accs, scheds = [], []
    for it in (0, 5):
        reach = 2 if it < 3 else 1  # odom.py:764-767
        max_d2 = ((reach + 0.5) * vox) ** 2
        kappa = max(2.0, 6.0 * (0.7 ** it))
        acc = np.zeros(64 * 64, np.float64)
        acc_out = np.zeros(64, np.float64)
        R.odom.k_icp.launch(n, icp_pts, n, T32, np.float32(1.0 / vox), vox, cap - 1, rk, rsum, rout, rcnt, reach,
                            max_d2, 0.02 * 0.02, tight2, 0.05, kappa, acc)
        R.odom.k_reduce.launch(64, acc, acc_out)
        accs.append(acc_out)
        scheds.append((it, reach, np.float32(max_d2), np.float32(kappa)))
    out.update(icp_pts=icp_pts, icp_acc=np.stack(accs), icp_sched=np.array(scheds, np.float64))
    return out


# ---- integration map and carving ---------------------------------------------------------------------------------

VIEW_FIELDS = ("now", "persist", "min_range", "max_range", "min_refl", "noise_mask", "ret_mask", "crop_on",
               "crop_lo", "crop_hi", "inv_frame_dt", "epoch", "inv_voxel", "map_mask", "dyn_on", "dyn_settle",
               "carve_on", "carve_ratio", "carve_min", "carve_stale")


def view_array(v: SimpleNamespace) -> np.ndarray:
    """The View's fields as float64, in VIEW_FIELDS order (crop boxes as 3 values each)."""
    vals = []
    for f in VIEW_FIELDS:
        x = getattr(v, f)
        vals.extend(list(x) if f in ("crop_lo", "crop_hi") else [x])
    return np.array(vals, np.float64)


def walker_room(synth):
    """The box room with a walker crossing the sensor's view, and the corner pose looking across the room."""
    room = synth.box_room(1)
    walker = synth.Cylinder(np.array([3.6, 1.4]), np.array([3.6, 4.6]), 1.2, radius=0.25, height=1.8)
    scene = synth.Scene(room.room_lo, room.room_hi, room.boxes, [walker])
    return scene, synth.look_at([0.8, 0.8, 1.6], [7.0, 5.0, 1.0])


def ref_map(ref: Path) -> dict:
    R = _ref(ref)
    synth = _synth()
    scene, T0 = walker_room(synth)
    voxel, cap = 0.1, 1 << 16
    v = SimpleNamespace(now=np.float32(1.3), persist=0.0, min_range=0.1, max_range=500.0, min_refl=0,
                        noise_mask=0b1111, ret_mask=0b1111, crop_on=0, crop_lo=(-1e9, -1e9, -1e9),
                        crop_hi=(1e9, 1e9, 1e9), inv_frame_dt=0.0, epoch=0, inv_voxel=np.float32(1.0 / voxel),
                        map_mask=cap - 1, dyn_on=1, dyn_settle=0.5, carve_on=1, carve_ratio=2.0, carve_min=4,
                        carve_stale=0.3)
    poses = np.tile(np.eye(4, dtype=np.float32), (POSE_SLOTS, 1, 1))
    # a sensor that holds still while the walker crosses; each frame posed by a slightly different pose slot
    static = synth.ConstantVelocity(T0, 1e9, 0.0, 0.0)
    frames = synth.frames(scene, static, 12, RATE, seed=41)
    keys = np.full(cap, -1, np.int64)
    acc = np.zeros((cap, 4), np.float32)
    cnt = np.zeros(cap, np.int32)
    last = np.zeros(cap, np.float32)
    first = np.full(cap, 1e30, np.float32)
    miss = np.zeros(cap, np.int32)
    stats = np.zeros(2, np.int32)
    out = {"map_voxel": np.float64(voxel), "map_cap": np.int64(cap), "map_view": view_array(v)}
    ins_x, ins_a, ins_t, ins_f = [], [], [], []
    carve_x, carve_a, carve_f, carve_every = [], [], [], []
    for k, (x, a, t) in enumerate(frames):
        sel = np.arange(0, len(t), 7)[:1400]  # every 7th return: the whole field of view, fewer points
        x, a, t = x[sel], a[sel], t[sel]
        fid = np.full(len(t), k, np.int32)
        poses[k] = T0.astype(np.float32)
        R.gpu.k_map_insert.launch(len(t), x, a, t, fid, poses, v, np.float32(1.0 / voxel), cap - 1, keys, acc, cnt,
                                  last, first, stats)
        ins_x.append(x), ins_a.append(a), ins_t.append(t), ins_f.append(fid)
        if k >= 4:
            every = 2 if k % 4 == 3 else 1
            cx, ca = x[:500], a[:500]
            cf = fid[:500]
            R.gpu.k_carve.launch((len(cx) + every - 1) // every, cx, ca, cf, poses, len(cx), every,
                                 np.float32(1.0 / voxel), cap - 1, 40.0, 4096, keys, acc, cnt, miss)
            carve_x.append(cx), carve_a.append(ca), carve_f.append(cf), carve_every.append(every)
    out.update(ins_x=np.concatenate(ins_x), ins_a=np.concatenate(ins_a), ins_t=np.concatenate(ins_t),
               ins_f=np.concatenate(ins_f), ins_len=np.array([len(z) for z in ins_t]), poses_T0=T0,
               carve_x=np.stack(carve_x), carve_a=np.stack(carve_a), carve_f=np.stack(carve_f),
               carve_every=np.array(carve_every, np.int32),
               keys=keys, acc=acc, cnt=cnt, last=last, first=first, miss=miss, stats=stats)
    # the visible set of the map (k_classify_map), carving and the Motion label on
    flag = np.zeros(cap, np.int32)
    oxyz = np.zeros((cap, 3), np.float32)
    oattr = np.zeros(cap, np.uint32)
    ot = np.zeros(cap, np.float32)
    odyn = np.zeros(cap, np.int32)
    R.gpu.k_classify_map.launch(cap, keys, acc, cnt, last, first, miss, v, 1, flag, oxyz, oattr, ot, odyn)
    sel = np.nonzero(flag)[0]
    out.update(cls_slots=sel.astype(np.int64), cls_xyz=oxyz[sel], cls_attr=oattr[sel], cls_t=ot[sel],
               cls_dyn=odyn[sel])
    return out


# ---- perception --------------------------------------------------------------------------------------------------


def ref_perception(ref: Path) -> dict:
    R = _ref(ref)
    synth = _synth()
    scene, T0 = walker_room(synth)
    tr = synth.Handheld(synth.box_room(1), 2, 20.0)
    xs = []
    for k in (12, 13, 14):  # three frames of a handheld path, posed by the path, in world coordinates
        x, a, t = synth.scan(scene, tr, 0.1 * k, 0.1 * k + 0.1, RATE, 5)
        T = tr.poses(np.array([0.1 * k + 0.05]))[0]
        xs.append((x[::3].astype(np.float64) @ T[:3, :3].T + T[:3, 3]).astype(np.float32))
    pts = np.concatenate(xs)
    n = len(pts)
    rng = np.random.default_rng(7)
    nrm = rng.normal(0, 1, (n, 3))
    nrm[:, 2] += np.where(pts[:, 2] < 0.3, 4.0, 0.0)  # mostly up near the floor, random elsewhere
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    G = R.perception.GRID
    out = {"pts": pts, "nrm": nrm}
    # ground: perception.py:458-483 (cell_min filled with 1e30, cell_sup zeroed, then the three kernels)
    cell, thick, min_sup, thresh, slope, nz_min = 0.5, 0.15, 3, 0.2, 0.3, 0.7
    for use_nrm in (0, 1):
        cmin = np.full(G * G, 1e30, np.float32)
        csup = np.zeros(G * G, np.int32)
        inv = np.float32(1.0 / cell)
        R.perception.k_gnd_min.launch(n, pts, inv, cmin)
        R.perception.k_gnd_support.launch(n, pts, inv, thick, cmin, csup)
        gnd = np.zeros(n, np.int32)
        hag = np.zeros(n, np.float32)
        R.perception.k_gnd_label.launch(n, pts, nrm, use_nrm, inv, cmin, csup, min_sup, thresh, slope, nz_min, gnd, hag)
        out[f"gnd{use_nrm}"], out[f"hag{use_nrm}"] = gnd, hag
    out["ground_params"] = np.array([cell, thick, min_sup, thresh, slope, nz_min], np.float64)
    # clusters of the non-ground points (perception.py:487-567), twice: 0.2 m / 0.35 m and 0.1 m / 0.15 m
    for tag, (voxel, connect, min_pts) in (("a", (0.2, 0.35, 30)), ("b", (0.1, 0.15, 10))):
        c = 1 << 14
        keys = np.full(c, -1, np.int64)
        acc = np.zeros((c, 4), np.float32)
        slot = np.zeros(n, np.int32)
        R.perception.k_cl_insert.launch(n, pts, out["gnd0"], 1, np.float32(1.0 / max(voxel, 0.01)), c - 1, keys, acc,
                                        slot)
        flag = np.zeros(c, np.int32)
        R.gpu.k_nb_flag.launch(c, keys, flag)
        offs = ws.array_scan_exclusive(flag)  # wp.utils.array_scan(inclusive=False)
        total = np.zeros(1, np.int32)
        R.gpu.k_total.launch(1, flag, offs, c, total)
        m = int(total[0])
        vidx = np.zeros(c, np.int32)
        vxyz = np.zeros((c, 3), np.float32)
        vw = np.zeros(c, np.float32)
        R.gpu.k_nb_compact.launch(c, flag, offs, acc, vidx, vxyz, vw)
        vox = vxyz[:m].copy()
        label = np.zeros(m, np.int32)
        grid = ws.HashGrid(vox)
        R.perception.k_cc_init.launch(m, label)
        changed = np.zeros(1, np.int32)
        passes, converged = 0, False
        while passes < 256:  # _label: 4 x (step + 2 jumps) between reads of `changed` (:527-548)
            changed[0] = 0
            for _ in range(4):
                R.perception.k_cc_step.launch(m, grid, vox, connect, label, changed)
                R.perception.k_cc_jump.launch(m, label)
                R.perception.k_cc_jump.launch(m, label)
                passes += 1
            if changed[0] == 0:
                converged = True
                break
        st_cnt = np.zeros(m, np.float32)
        st_sum = np.zeros((m, 3), np.float32)
        st_lo = np.zeros((m, 3), np.float32)
        st_hi = np.zeros((m, 3), np.float32)
        R.perception.k_cc_reset.launch(m, st_cnt, st_sum, st_lo, st_hi)
        R.perception.k_cc_stats.launch(m, label, vox, vw[:m].copy(), st_cnt, st_sum, st_lo, st_hi)
        cflag = np.zeros(m, np.int32)
        R.perception.k_cc_flag.launch(m, label, st_cnt, float(min_pts), cflag)
        coffs = ws.array_scan_exclusive(cflag)
        ctot = np.zeros(1, np.int32)
        R.gpu.k_total.launch(1, cflag, coffs, m, ctot)
        dense = np.zeros(m, np.int32)
        ocnt = np.zeros(4096, np.float32)
        ocen = np.zeros((4096, 3), np.float32)
        olo = np.zeros((4096, 3), np.float32)
        ohi = np.zeros((4096, 3), np.float32)
        R.perception.k_cc_compact.launch(m, cflag, coffs, st_cnt, st_sum, st_lo, st_hi, 4096, dense, ocnt, ocen, olo,
                                         ohi)
        cid = np.zeros(n, np.int32)
        R.perception.k_cc_gather.launch(n, slot, vidx, label, dense, cid)
        k = min(int(ctot[0]), 4096)
        out.update({f"cl{tag}_params": np.array([voxel, connect, min_pts], np.float64), f"cl{tag}_keys": keys,
                    f"cl{tag}_node_xyz": vox, f"cl{tag}_node_w": vw[:m].copy(), f"cl{tag}_label": label,
                    f"cl{tag}_converged": np.int32(converged), f"cl{tag}_cid": cid, f"cl{tag}_cnt": ocnt[:k].copy(),
                    f"cl{tag}_cen": ocen[:k].copy(), f"cl{tag}_lo": olo[:k].copy(), f"cl{tag}_hi": ohi[:k].copy()})
    return out


# ---- localisation ------------------------------------------------------------------------------------------------


def ref_localize(ref: Path) -> dict:
    R = _ref(ref)
    synth = _synth()
    room = synth.box_room(3, size=(2.4, 2.0, 1.2), n_boxes=3, side=(0.2, 0.5))
    xyz, nrm = synth.sample_surfaces(room, 0.03, seed=1, jitter=0.002)
    rng = np.random.default_rng(5)
    planarity = np.where(rng.uniform(0, 1, len(xyz)) < 0.85, 0.9, 0.2).astype(np.float32)
    prep = R.mapgrid.PriorGrid.prepare({"xyz": xyz, "normal": nrm, "planarity": planarity})
    dims = np.asarray(prep["dims"], np.int64)
    ncell = int(np.prod(dims))
    g = SimpleNamespace(origin=tuple(float(v) for v in prep["origin"]), cell=float(prep["cell"]),
                        inv_cell=float(1.0 / prep["cell"]), nx=int(dims[0]), ny=int(dims[1]), nz=int(dims[2]))
    mx = np.ascontiguousarray(prep["xyz"], np.float32)
    mn = np.ascontiguousarray(prep["normal"], np.float32)
    mp = np.ascontiguousarray(prep["planarity"], np.float32)
    start = np.ascontiguousarray(prep["start"], np.int32)
    # PriorGrid.build (mapgrid.py:272-296)
    nn = np.full(ncell, R.mapgrid.EMPTY, np.int32)
    R.mapgrid.k_seed.launch(len(mx), mx, g, nn)
    R.mapgrid.k_unpack.launch(ncell, nn)
    seeds = nn.copy()
    for step in R.mapgrid.JFA_STEPS:
        R.mapgrid.k_jfa.launch(ncell, nn, mx, g, int(step))
    df = np.zeros(ncell, np.uint8)
    R.mapgrid.k_df.launch(ncell, nn, mx, g, df)
    out = {"map_in_xyz": xyz, "map_in_normal": nrm, "map_in_planarity": planarity, "xyz": mx, "normal": mn,
           "planarity": mp, "start": start, "origin": np.asarray(prep["origin"], np.float64), "dims": dims,
           "cell": np.float64(prep["cell"]), "seeds": seeds, "nn": nn, "df": df}
    # four hypotheses near the scan's true pose, one shared scan (GlobalLocalizer._icp, localize.py:517-553)
    T_true = np.eye(4)
    T_true[:3, :3] = Rotation.from_euler("z", 0.7).as_matrix()
    T_true[:3, 3] = (1.1, 0.9, 0.7)
    pts = synth.spin_scan(room, T_true, 700, seed=9, noise=0.003)
    k = 4
    Ts = []
    for h in range(k):
        T = T_true.copy()
        a = rng.uniform(-3.0, 3.0) * math.pi / 180.0
        T[:3, :3] = Rotation.from_euler("z", a).as_matrix() @ T[:3, :3]
        T[:3, 3] += rng.uniform(-0.06, 0.06, 3) * (1, 1, 0.3)
        Ts.append(T)
    T_start = np.stack(Ts)
    schedule = ((0.20, 4), (0.10, 4), (0.05, 6))
    twist_apply = R.localize._twist_apply
    n_pts = len(pts)
    acc_first = None
    iters_run = 0
    for dmax, iters in schedule:
        c2 = (dmax * 0.5) ** 2
        for _ in range(iters):
            Tf = np.stack([T.astype(np.float32) for T in Ts])
            acc = np.zeros(k * 64 * 64, np.float64)
            R.localize.k_icp_batch.launch(k * n_pts, pts, n_pts, Tf, g, start, nn, mx, mn, mp, dmax * dmax, c2, 0.05,
                                          acc)
            v = np.zeros(k * 64, np.float64)
            R.localize.k_reduce_batch.launch(k * 64, acc, k, v)
            v = v.reshape(k, 64)
            if acc_first is None:
                acc_first = v.copy()
            iters_run += 1
            moved = 0.0
            for h in range(k):
                if v[h, 27] < 30:
                    continue
                H = np.zeros((6, 6))
                H[np.triu_indices(6)] = v[h, :21]
                H += np.triu(H, 1).T
                b = v[h, 21:27]
                A = H + np.diag(1e-3 * np.diag(H) + 1e-9)
                try:
                    delta = np.linalg.solve(A, -b)
                except np.linalg.LinAlgError:
                    continue
                Ts[h] = twist_apply(Ts[h], delta)
                moved = max(moved, float(np.linalg.norm(delta[:3])), float(np.linalg.norm(delta[3:])) * 5.0)
            if moved < 2e-4:
                break
    T_end = np.stack(Ts)
    counts = np.zeros(k * 3, np.int32)
    radii = ws.vec3(*R.localize.EVAL_RADII)
    R.localize.k_eval_batch.launch(k * n_pts, pts, n_pts, np.stack([T.astype(np.float32) for T in Ts]), g, start, nn,
                                   mx, radii, counts)
    out.update(scan=pts, T_true=T_true, T_start=T_start, T_end=T_end, acc_first=acc_first,
               schedule=np.array(schedule, np.float64), iters_run=np.int32(iters_run), eval_counts=counts.reshape(k, 3))
    return out


FIXTURES = {"ref_odom": ref_odom, "ref_map": ref_map, "ref_perception": ref_perception, "ref_localize": ref_localize}
