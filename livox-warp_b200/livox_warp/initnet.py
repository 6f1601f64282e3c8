"""A learned start pose for the odometry's registration: a point-set network trained on the GPU by this library's own
bf16 forward (tensor cores) and backward kernels (lw_net_*), and the tools that make its training pairs.

The reference's odometry starts every frame from a constant-velocity prediction (odom.py:591-592). Here that
prediction stays the input frame and the fallback: the network sees LW_NET_P points of the thinned frame and, for
each, the nearest registration-map voxel mean around the prediction (or, in patch mode, the voxel means within a
radius), both in the predicted sensor frame, and proposes a
step (tx, ty, tz, rx, ry, rz) with T = T_pred * [R(r), t]; the Gauss-Newton registration then starts from, and
anchors its prior at, that pose (Odometry.learned_init).

Training pairs (make_pairs): a sequence is registered by the plain odometry; its converged poses are the
labels. The registration map is then rebuilt frame by frame from those poses, and before frame k is inserted
its point sets are cut around Gaussian-perturbed copies of its converged pose, the perturbation being the
target -- so a frame never sees itself in its map patch, as at run time.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch
from scipy.spatial.transform import Rotation

from . import _lib
from .kernels import RegistrationMap

P = _lib.NET_P
OFF = _lib.NET_OFF
NPARAM = _lib.NET_NPARAM
OUT_SCALE = (0.05, 0.05, 0.05, 0.03, 0.03, 0.03)  # m, rad: the step's expected size per component


def step_between(T_from: np.ndarray, T_to: np.ndarray) -> np.ndarray:
    """The step s with T_to = T_from * [R(s_r), s_t] (translation in T_from's frame)."""
    R0 = T_from[:3, :3]
    t = R0.T @ (T_to[:3, 3] - T_from[:3, 3])
    r = Rotation.from_matrix(R0.T @ T_to[:3, :3]).as_rotvec()
    return np.concatenate([t, r])


def apply_step(T: np.ndarray, s: np.ndarray) -> np.ndarray:
    out = np.eye(4)
    out[:3, :3] = T[:3, :3] @ Rotation.from_rotvec(s[3:]).as_matrix()
    out[:3, 3] = T[:3, 3] + T[:3, :3] @ s[:3]
    return out


class InitNet:
    """Parameters (float32 masters, bf16 copy, Adam moments), forward / backward / Adam through the C ABI."""

    def __init__(self, device=None, seed: int = 0, in_scale: float = 0.125, out_scale=OUT_SCALE,
                 batch_cap: int = 256):
        _lib.load()
        self.device = torch.device(device if device is not None else "cuda")
        d = self.device
        self.master = torch.zeros(NPARAM, dtype=torch.float32, device=d)
        self.w = torch.zeros(NPARAM, dtype=torch.int16, device=d)
        self.grad = torch.zeros(NPARAM, dtype=torch.float32, device=d)
        self.adam_m = torch.zeros(NPARAM, dtype=torch.float32, device=d)
        self.adam_v = torch.zeros(NPARAM, dtype=torch.float32, device=d)
        self.out_scale = torch.tensor(out_scale, dtype=torch.float32, device=d)
        self.in_scale = float(in_scale)
        self.struct = _lib.InitNet(*(_lib.ptr(t).value for t in (self.master, self.w, self.grad, self.adam_m,
                                                                  self.adam_v, self.out_scale)), self.in_scale, 0)
        self.t = 0
        self.batch_cap = 0
        self._alloc(batch_cap)
        _lib.call("lw_net_init", ctypes.byref(self.struct), ctypes.c_uint64(seed), _lib.stream_ptr())

    def _alloc(self, n: int):
        if n <= self.batch_cap:
            return
        d = self.device
        K = 2 * n * 256
        f = lambda *shape: torch.zeros(*shape, dtype=torch.float32, device=d)  # noqa: E731
        self._scr = {"dz3": f(K), "h2g": torch.zeros(K * 128, dtype=torch.int16, device=d), "d2t": f(128 * K),
                     "h1t": f(65 * K), "d1t": f(64 * K), "xt": f(4 * K), "dzh": f(n * 128), "dout": f(n * 6),
                     "dpool": f(n * 512), "part": f(64 * 8448), "loss": f(n)}
        self.scr = _lib.NetScratch(*(_lib.ptr(self._scr[k]).value for k in _lib.NetScratch.PTRS), n, 0)
        self._fwd = {"pooled": f(n * 512), "argmax": torch.zeros(n * 512, dtype=torch.int32, device=d),
                     "hid": f(n * 128), "step": f(n * 6), "err": torch.zeros(1, dtype=torch.int32, device=d)}
        self.batch_cap = n

    # ---- passes -------------------------------------------------------------------------------------------

    def forward(self, sets: torch.Tensor, n: int, stream=None) -> dict:
        """sets: (2n, P, 4) float32 CUDA tensor (frame set 2s, map set 2s+1). Returns views of the outputs."""
        if sets.dtype != torch.float32 or not sets.is_contiguous() or sets.shape[0] < 2 * n or sets.shape[1:] != (P, 4):
            raise ValueError(f"sets must be a contiguous ({2 * n}, {P}, 4) float32 tensor")
        self._alloc(n)
        o = self._fwd
        _lib.call("lw_net_forward", ctypes.byref(self.struct), _lib.ptr(sets), int(n), _lib.ptr(o["pooled"]),
                  _lib.ptr(o["argmax"]), _lib.ptr(o["hid"]), _lib.ptr(o["step"]), _lib.ptr(o["err"]),
                  _lib.stream_ptr(stream))
        return {"pooled": o["pooled"][:n * 512], "argmax": o["argmax"][:n * 512], "hid": o["hid"][:n * 128],
                "step": o["step"][:n * 6].view(n, 6), "err": o["err"]}

    def backward(self, sets: torch.Tensor, n: int, fwd: dict, target: torch.Tensor, w_loss=None, stream=None):
        """Gradient of the weighted squared step error into self.grad; returns the per-sample losses."""
        wl = torch.as_tensor(w_loss if w_loss is not None else np.ones(6), dtype=torch.float32, device=self.device)
        target = target.to(self.device, torch.float32).contiguous()
        _lib.call("lw_net_backward", ctypes.byref(self.struct), _lib.ptr(sets), int(n), _lib.ptr(fwd["pooled"]),
                  _lib.ptr(fwd["argmax"]), _lib.ptr(fwd["hid"]), _lib.ptr(fwd["step"]), _lib.ptr(target),
                  _lib.ptr(wl), ctypes.byref(self.scr), _lib.stream_ptr(stream))
        return self._scr["loss"][:n]

    def adam(self, lr: float, beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8, weight_decay: float = 0.0,
             stream=None):
        self.t += 1
        _lib.call("lw_net_adam", ctypes.byref(self.struct), int(self.t), float(lr), float(beta1), float(beta2),
                  float(eps), float(weight_decay), _lib.stream_ptr(stream))

    def predict(self, sets: torch.Tensor, n: int) -> np.ndarray:
        return self.forward(sets, n)["step"].cpu().numpy().astype(np.float64)

    # ---- training -----------------------------------------------------------------------------------------

    def fit(self, sets: torch.Tensor, targets: torch.Tensor, epochs: int = 30, batch: int = 256, lr: float = 1e-3,
            lr_end: float = 1e-5, seed: int = 0, val_frac: float = 0.05, log=None) -> dict:
        """Adam over shuffled mini-batches with a cosine learning-rate decay; the last val_frac of the pairs is
        held out. Returns the loss history (train per epoch, validation per epoch)."""
        N = targets.shape[0]
        n_val = max(1, int(N * val_frac))
        n_tr = N - n_val
        g = torch.Generator(device="cpu")
        g.manual_seed(seed)
        hist = {"train": [], "val": []}
        steps = epochs * (n_tr // batch)
        k = 0
        sets_p = sets.view(N, 2, P, 4)
        for ep in range(epochs):
            perm = torch.randperm(n_tr, generator=g).to(self.device)
            tot = torch.zeros((), dtype=torch.float32, device=self.device)
            for b0 in range(0, n_tr - batch + 1, batch):
                idx = perm[b0:b0 + batch]
                xs = sets_p.index_select(0, idx).view(2 * batch, P, 4)
                ys = targets.index_select(0, idx)
                fwd = self.forward(xs, batch)
                tot += self.backward(xs, batch, fwd, ys).sum()
                lr_k = lr_end + 0.5 * (lr - lr_end) * (1.0 + math.cos(math.pi * k / max(steps, 1)))
                self.adam(lr_k)
                k += 1
            hist["train"].append(float(tot) / max(1, n_tr // batch))
            hist["val"].append(self.evaluate(sets_p[n_tr:].reshape(2 * n_val, P, 4), targets[n_tr:]))
            if log:
                log(f"epoch {ep}: train {hist['train'][-1]:.4f} val {hist['val'][-1]:.4f}")
        return hist

    def evaluate(self, sets: torch.Tensor, targets: torch.Tensor, batch: int = 256) -> float:
        """Mean loss (unit weights) over the pairs, forward only."""
        N = targets.shape[0]
        tot = 0.0
        sc = self.out_scale
        for b0 in range(0, N, batch):
            n = min(batch, N - b0)
            out = self.forward(sets[2 * b0:2 * (b0 + n)].contiguous(), n)["step"]
            tot += float((((out - targets[b0:b0 + n]) / sc) ** 2).sum())
        return tot / N

    def state_dict(self) -> dict:
        return {"master": self.master.cpu().numpy().copy(), "out_scale": self.out_scale.cpu().numpy().copy(),
                "in_scale": self.in_scale}

    def load_state_dict(self, sd: dict):
        self.master.copy_(torch.from_numpy(np.asarray(sd["master"], np.float32)))
        self.out_scale.copy_(torch.from_numpy(np.asarray(sd["out_scale"], np.float32)))
        self.in_scale = float(sd["in_scale"])
        self.struct.in_scale = self.in_scale
        self.adam_m.zero_()
        self.adam_v.zero_()
        self.t = 0
        # the bf16 copy: one Adam call with lr 0 rewrites it from the masters
        self.grad.zero_()
        self.adam(0.0)
        self.t = 0


# ---- training pairs -------------------------------------------------------------------------------------------


def frame_sets(ds: torch.Tensor, n_ds: torch.Tensor, reg: RegistrationMap, T: torch.Tensor, radius: float,
               out: torch.Tensor, scratch: dict, voxel: float = 0.0, stream=None):
    """lw_net_sets: the frame's and the map's point sets at the device pose T (16 float64) into out ((2, P, 4)).
    voxel > 0: the map set is each frame point's nearest registration voxel mean; else the patch within radius."""
    _lib.call("lw_net_sets", _lib.ptr(ds), _lib.ptr(n_ds), ctypes.byref(reg.struct), _lib.ptr(T), float(radius),
              float(voxel), _lib.ptr(out), _lib.ptr(scratch.get("cand")), _lib.ptr(scratch.get("tiles")),
              _lib.ptr(scratch["count"]), _lib.stream_ptr(stream))


def make_pairs(frames, odom, T0: np.ndarray, per_frame: int, sigma, seed: int, radius: float = 12.0,
               nearest: bool = True, frame_dt: float = 0.1, warm: int = 10, reg_slots: int = 1 << 21, accept=None,
               log=None):
    """Register the sequence `frames` [(xyz, attr, t)] with the plain odometry `odom` (reset to T0 here), then
    rebuild the registration map from its converged poses and cut `per_frame` perturbed pairs per frame before
    inserting it. accept(k, T) may veto a frame (e.g. a sanity check of the converged pose); a vetoed frame
    gives no pairs and is not inserted. Returns (sets (2N, P, 4) device, targets (N, 6) device, info)."""
    d = odom.device
    odom.reset(T0)
    odom.learned_init(None)
    ds_list, n_list = [], []

    def keep(k, T, f_xyz, f_attr, f_t, f_frame, m):
        st = odom.read_state()
        n = int(st.n_ds)
        if st.ok and st.run_reg and n >= 200:
            # the frame's float4 rows (x, y, z, t), which the registration map's insert reads
            ds_list.append((k, odom.ds_xyz[:n].clone(), np.array(st.T, dtype=np.float64).reshape(4, 4),
                            odom.f_xyz[:m].clone(), f_attr[:m].clone()))

    pipe = odom.pipe
    for k, (x, a, t) in enumerate(frames):
        sx, sa, st_, sf = pipe.stage(x, a, t, len(t), 1.0 / frame_dt)
        odom.push(sx, sa, st_, len(t), float(t.min()), float(t.max()), on_frame=keep)
    odom.flush(on_frame=keep)
    # replay: the map of frames < k, pairs of frame k, then frame k's insert at its converged pose
    reg = RegistrationMap(reg_slots, d)
    rng = np.random.default_rng(seed)
    N = len(ds_list) * per_frame
    sets = torch.zeros((2 * N, P, 4), dtype=torch.float32, device=d)
    targets = np.zeros((N, 6), np.float64)
    scratch = {"cand": torch.zeros(reg_slots, dtype=torch.int32, device=d),
               "tiles": torch.zeros(reg_slots // 1024 + 2, dtype=torch.int32, device=d),
               "count": torch.zeros(2, dtype=torch.int32, device=d)}
    Ts = np.zeros((N, 16), np.float64)
    sig = np.asarray(sigma, np.float64)
    j = 0
    vetoed = 0
    for i, (k, ds, T, fx, fa) in enumerate(ds_list):
        if accept is not None and not accept(k, T):
            vetoed += 1
            continue
        n_ds = torch.tensor([ds.shape[0]], dtype=torch.int32, device=d)
        if i >= warm:
            for _ in range(per_frame):
                s = rng.normal(0.0, 1.0, 6) * sig
                T_init = _perturbed(T, s)
                targets[j] = step_between(T_init, T)
                Ts[j] = T_init.reshape(16)
                j += 1
            Td = torch.from_numpy(Ts[j - per_frame:j].copy()).to(d)
            for q in range(per_frame):
                frame_sets(ds, n_ds, reg, Td[q], radius, sets[2 * (j - per_frame + q):2 * (j - per_frame + q) + 2],
                           scratch, odom.reg_voxel if nearest else 0.0)
        reg.insert(fx, fa, T, odom.reg_voxel, odom.max_range, odom.ret_mask, odom.noise, odom.alpha)
    sets = sets[:2 * j]
    tg = torch.from_numpy(targets[:j]).to(d, torch.float32)
    if log:
        log(f"pairs: {j} from {len(ds_list)} registered frames")
    return sets, tg, {"frames": len(ds_list) - vetoed, "vetoed": vetoed, "pairs": j}


def _perturbed(T: np.ndarray, s: np.ndarray) -> np.ndarray:
    """T_init with T = T_init * [R(s_r), s_t]."""
    R = T[:3, :3] @ Rotation.from_rotvec(s[3:]).as_matrix().T
    out = np.eye(4)
    out[:3, :3] = R
    out[:3, 3] = T[:3, 3] - R @ s[:3]
    return out


# ---- frame by frame: training pairs and the evaluation on paths the registration is judged on ----------------


def iterations_to(poses: np.ndarray, target: np.ndarray, tol_m: float = 1e-3, tol_deg: float = 0.01) -> int:
    """The first Gauss-Newton iteration from which a registration's traced poses (start first) all stay within
    tol_m / tol_deg of `target`; len(poses) when they never settle there."""
    def close(T):
        d = np.linalg.inv(target) @ T
        ang = math.degrees(np.linalg.norm(Rotation.from_matrix(d[:3, :3]).as_rotvec()))
        return np.linalg.norm(d[:3, 3]) <= tol_m and ang <= tol_deg

    ok = [close(T) for T in poses]
    first = len(poses)
    for i in range(len(poses) - 1, -1, -1):
        if not ok[i]:
            break
        first = i
    return first


def pose_gap(A: np.ndarray, B: np.ndarray) -> tuple:
    """(metres, degrees) from pose A to pose B."""
    d = np.linalg.inv(A) @ B
    return float(np.linalg.norm(d[:3, 3])), float(math.degrees(np.linalg.norm(Rotation.from_matrix(d[:3, :3]).as_rotvec())))


class FrameByFrame:
    """A path's frames registered one at a time against a registration map of the frames before them, inserted at
    their true poses: each frame from the constant-velocity prediction (the motion between the two previous true
    poses carried on; deskewed with it), from the network's proposal made at that prediction, and from its true
    pose -- the converged registration that judges the other two. Both starts see the same map and the same
    deskewed, thinned frame, so what differs is only where the registration starts (and anchors its prior).

    Drives Odometry.register_frame with its Gauss-Newton trace on; `radius` / `nearest` choose the network's map
    set as in Odometry.learned_init."""

    def __init__(self, odom, radius: float = 12.0, nearest: bool = True):
        self.odom = odom
        self.radius, self.nearest = radius, nearest
        d = odom.device
        self.scratch = {"cand": torch.zeros(odom.reg_cap, dtype=torch.int32, device=d),
                        "tiles": torch.zeros(odom.reg_cap // 1024 + 2, dtype=torch.int32, device=d),
                        "count": torch.zeros(2, dtype=torch.int32, device=d)}
        odom._gn.trace_on(True)

    def _register(self, raw4, attr, t_mid, twist, T):
        Tr, ok, st = self.odom.register_frame(raw4, attr, None, t_mid, twist, T)
        return Tr, ok, st, self.odom._gn.poses(st["iters"])

    def sets_at(self, T: np.ndarray, out: torch.Tensor):
        """The network's two point sets for the frame last thinned by register_frame, at pose T, into out."""
        o = self.odom
        off = _lib.OdomState.n_ds.offset
        n_ds = o._state[off:off + 4].view(torch.int32)
        Td = torch.from_numpy(np.asarray(T, np.float64).reshape(16).copy()).to(o.device)
        frame_sets(o.ds_xyz, n_ds, o.reg, Td, self.radius, out, self.scratch,
                   o.reg_voxel if self.nearest else 0.0, o.stream)

    def run(self, frames, truth, net=None, warm: int = 10, per_frame: int = 0, sigma=None, seed: int = 0,
            tol_m: float = 1e-3, tol_deg: float = 0.01):
        """Frames [(xyz, attr, t)] of a path and truth(t) -> 4x4 poses. The first `warm` frames only build the map.
        Without per_frame: each later frame is registered from both starts (the network's: `net`'s proposal, or
        the prediction itself when net is None) and a row of results is kept. With per_frame > 0: training pairs
        instead -- the prediction and per_frame - 1 Gaussian perturbations (sigma) of the converged pose, each with
        its point sets and its step to the converged pose. Returns (rows, sets, targets)."""
        o = self.odom
        dt = o.frame_dt
        rng = np.random.default_rng(seed)
        rows, sets, targets = [], [], []
        zero = np.zeros(6, np.float32)
        o.reset(np.eye(4))
        for k, (x, a, t) in enumerate(frames):
            t_mid = (k + 0.5) * dt
            T_true = truth(np.array([t_mid]))[0]
            raw4 = torch.from_numpy(np.ascontiguousarray(np.concatenate([x, t[:, None]], 1), dtype=np.float32))
            raw4 = raw4.to(o.device)
            at = torch.from_numpy(np.asarray(a).view(np.int32)).to(o.device)
            if k < max(warm, 2):
                o.register_frame(raw4, at, None, t_mid, zero, T_true, sync=False)  # deskew only; map at the truth
                o.insert_frame(o.f_xyz[:len(t)], at, T_true)
                continue
            T1, T2 = truth(np.array([t_mid - dt, t_mid - 2 * dt]))
            delta = np.linalg.inv(T2) @ T1
            T_cv = T1 @ delta
            tw = np.concatenate([delta[:3, 3], Rotation.from_matrix(delta[:3, :3]).as_rotvec()]).astype(np.float32)
            T_star, ok_s, _, _ = self._register(raw4, at, t_mid, tw, T_true)  # the judge
            if per_frame > 0:
                if ok_s:
                    starts = [T_cv] + [_perturbed(T_star, rng.normal(0.0, 1.0, 6) * np.asarray(sigma))
                                       for _ in range(per_frame - 1)]
                    buf = torch.zeros((2 * len(starts), P, 4), dtype=torch.float32, device=o.device)
                    for q, T0 in enumerate(starts):
                        self.sets_at(T0, buf[2 * q:2 * q + 2])
                        targets.append(step_between(T0, T_star))
                    sets.append(buf)
            else:
                T_a, ok_a, st_a, tr_a = self._register(raw4, at, t_mid, tw, T_cv)
                buf = torch.zeros((2, P, 4), dtype=torch.float32, device=o.device)
                self.sets_at(T_cv, buf)
                step = net.predict(buf, 1)[0] if net is not None else np.zeros(6)
                T_l = apply_step(T_cv, step)
                T_b, ok_b, st_b, tr_b = self._register(raw4, at, t_mid, tw, T_l)
                rows.append({"k": k, "ok": bool(ok_s and ok_a and ok_b),
                             "start_cv": pose_gap(T_star, T_cv), "start_net": pose_gap(T_star, T_l),
                             "final_cv": pose_gap(T_star, T_a), "final_net": pose_gap(T_star, T_b),
                             "truth_judge": pose_gap(T_true, T_star),
                             "iters_cv": int(st_a["iters"]), "iters_net": int(st_b["iters"]),
                             "to_acc_cv": iterations_to(tr_a, T_star, tol_m, tol_deg),
                             "to_acc_net": iterations_to(tr_b, T_star, tol_m, tol_deg),
                             "to_own_cv": iterations_to(tr_a, T_a, tol_m, tol_deg),
                             "to_own_net": iterations_to(tr_b, T_b, tol_m, tol_deg)})
            o.insert_frame(o.f_xyz[:len(t)], at, T_true)
        if per_frame > 0:
            return rows, (torch.cat(sets) if sets else None), torch.tensor(np.array(targets), dtype=torch.float32,
                                                                          device=o.device)
        return rows, None, None
