#!/usr/bin/env python
"""Benchmark of the per-frame SLAM hot path on B200.

Default workload (`--workload single`, the single-frame scan-to-map ICP configuration): a seeded 8 x 6 x 3 m box
room with 20 boxes and a Mid-40-like rosette (r = 0.5 fov sin(7/3 phi), fov 38.4 deg) at 100k points/s; the
registration map (0.2 m voxels, 2^21 slots) is built from 10 frames of a sensor holding still in a corner, then
the sensor moves at 0.5 m/s forward and 20 deg/s yaw. A step registers one 10k-point frame taken in the first
0.1 s of that motion: deskew with the constant-velocity prediction (a sensor that was at rest: its pose and a
zero twist), half-voxel thinning, and at most 10 Gauss-Newton iterations with the float64 6x6 solve on the device
(Odometry.register_frame, the reference's _deskew + _register, odom.py:707-709, 752-803). Eight seeded frames are
cycled. The line reports frames/s and points/s, each distinct frame's pose against the float64 oracle registering
the same thinned frame from the same start (the metric's <= 1 mm / 0.01 deg) and against the truth.

  value  frames/s with the frames already resident in HBM, device time (CUDA events per step), L2 flushed
         between steps by a 256 MB write outside the timed events;
  e2e    the same through the public API from host (numpy) buffers: pinned H2D of each frame, the result read
         back (D2H) every frame, CUDA events around all steps;
  roofline  the dominant kernel's algorithmic bytes / its live average launch time vs the measured HBM peak;
  cpu_baseline  the CPU oracle (a C++ / numpy restatement of the reference's kernels and host solve, OpenMP)
         on a bounded sample of the same frames.

`--workload sequence` measures sequence odometry: the same room and rosette along a smooth handheld trajectory (a
spline through random waypoints, <= 1 m/s and <= 60 deg/s, after 1 s at rest). Each step is one frame through the
whole path: frame cut, deskew, half-voxel thinning, scan-to-map Gauss-Newton, re-deskew, keyframe insert into the
0.15 m registration map, velocity update, then insertion of the frame into the 0.1 m integration map (2^22 slots)
and free-space carving of every ray; the timed frames start after the at-rest second and the ramp to cruise speed.

`--impl reference` times the reference's CPU implementation of the path instead: NVIDIA Warp (the reference's
only runtime) is not installed, so that arm runs the CPU restatement, on every host core.
`--workload frame` measures the full perception frame: a dual-return rosette (100k rays/s, two returns each: ~20k
points per frame) on a handheld path through a seeded 40 x 30 x 3 m office with 10 walkers (r 0.25 m, h 1.8 m,
1.2 m/s); per frame deskew + Gauss-Newton ICP + keyframe insert, integration-map insert and carving of every ray
(walker ghosts), the map's visible set, the 0.5 m ground grid (slope allowance 0.3) and clusters of the non-ground
points at 0.2 m voxels (connect 0.35 m, 30 points), read back to the host; latency p50 / p99 per frame.

`--workload learned` measures the learned start pose: fast handheld paths in the box room (<= 2 m/s, <= 120 deg/s),
every frame registered against a map of the frames before it (inserted at their true poses) three times -- from
the constant-velocity prediction, from the network's proposal made at that prediction, and from the true pose
(the converged registration that judges the other two). The network is trained on the GPU by the library's bf16
kernels on ~48k pairs from 8 paths (each frame's prediction and 9 perturbations of its converged pose); 3 held-out
600-frame paths compare the Gauss-Newton iterations each start needs to reach the converged pose within
1 mm / 0.01 deg, and their final errors.

`--workload localize` measures the batched global localisation instead: a 20.3M-point prior map sampled every
15 mm on the surfaces of a seeded 40 x 30 x 3 m office (walls with doors, 200 boxes), 256 hypotheses, each with
its own static 360-degree scan of U[2k, 20k] points taken at a free pose (z = 1.2 m, yaw uniform), started from
that pose snapped to a 0.5 m xy grid and a 5 deg heading grid; one step = one batched registration of all 256
(the schedule (0.40, 8), (0.20, 8), (0.10, 8), (0.05, 10)) plus the evaluation, in one graph-replayed launch.

`--workload coarse` measures the coarse global search (localize.py:426-448): the office prior map at 30 mm, one
1024-point scan subset, every free position on a 0.25 m xy grid at 8 heights x 180 headings (28M hypotheses) scored
by the distance-field soft count in one launch; hypotheses/s, with e2e through GlobalLocalizer._coarse_candidates
(the local maxima found on the device, only the candidates read back).

`--workload prior` measures the prior-map builder (prior_map.py:57-219, from_points :358-370): the office's surfaces
sampled every 10 mm with 2 mm jitter (45.7M points, a building-scale terrestrial scan), voxel means at 20 mm in a
2^27-slot table (chunks of 2^25 points) and a PCA normal and planarity per mean from its neighbours within 80 mm;
input points/s, with e2e through prior_map.from_points from host arrays to host arrays.

Multi-GPU: the path does not shard (each frame registers against the map of the frames before it), so
`--gpus N` runs N independent replicas, one per GPU, and `value` sums their frames.
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT), str(ROOT / "livox-warp_b200")]

RATE = 100000.0
FRAME_DT = 0.1
REG_VOXEL = 0.15
MAP_VOXEL = 0.1
MAP_SLOTS = 1 << 22
REG_SLOTS = 1 << 21
FRAME_CAP = 1 << 18
ROOM_SEED = 1   # the box room
PATH_SEED = 31  # the handheld path (a sequence the float64 oracle tracks for the whole 60 s)
SCAN_SEED = 3
L2_FLUSH_BYTES = 256 << 20
SEQ_DURATION = 62.1  # s: the handheld path of the 600-frame sequence (the float64 oracle tracks all of it)
SOAK_S = 0.6  # s of untimed steps after a short timed region, so the clock sampler sees the load
SEQ_SOAK_FRAMES = 600  # sequence frames generated after the timed ones, for the clock soak
SEQ_MAX_FRAMES = 620
SEQ_SKIP = 20  # sequence frames never timed: 1 s at rest and the 1 s ramp to cruise speed
LOC_SEED = 1          # the office
LOC_SPACING = 0.015   # prior-map sample spacing: 20.3M points on the office's surfaces
LOC_HYP = 256
LOC_PTS = (2000, 20000)
LOC_Z = 1.2
LOC_POSE_SEED = 11
FRAME_SCENE_SEED = 4   # the office with walkers
FRAME_PATH_SEED = 5
FRAME_RAYS = 100000.0  # rays/s; two returns each


# ---- workload --------------------------------------------------------------------------------------------------


def _gen_chunk(args):
    duration, k0, k1 = args
    from livox_warp import synth

    scene = synth.box_room(ROOM_SEED)
    traj = synth.Handheld(scene, PATH_SEED, duration)
    return synth.frames(scene, traj, k1 - k0, RATE, SCAN_SEED, start=k0)


def workload(n_frames: int, procs: int | None = None):
    """The frames 0 .. n_frames-1 of the sequence (generated in a spawn pool before any CUDA call)."""
    from livox_warp import synth

    duration = SEQ_DURATION  # the path of the 600-frame sequence, whatever n_frames
    procs = procs or min(8, os.cpu_count() or 1)
    step = max(1, math.ceil(n_frames / (procs * 4)))
    chunks = [(duration, k, min(k + step, n_frames)) for k in range(0, n_frames, step)]
    if procs > 1 and len(chunks) > 1:
        with mp.get_context("spawn").Pool(procs) as pool:
            parts = pool.map(_gen_chunk, chunks)
    else:
        parts = [_gen_chunk(c) for c in chunks]
    frames = [f for p in parts for f in p]
    scene = synth.box_room(ROOM_SEED)
    traj = synth.Handheld(scene, PATH_SEED, duration)
    return frames, traj


# ---- clocks --------------------------------------------------------------------------------------------------


class Clocks:
    """nvidia-smi samples of the SM clock and the throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def start(self):
        """Start sampling; returns once the sampler has written its first row (or after 3 s)."""
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
            return
        t_end = time.time() + 3.0
        while time.time() < t_end and os.path.getsize(self.path) == 0:
            time.sleep(0.02)
        self.skip = sum(1 for _ in open(self.path))  # rows written before the timed region (idle clocks)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        for i, line in enumerate(open(self.path)):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9 and i >= getattr(self, "skip", 0):
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = np.array([float(r[1]) for r in rows if r[1].replace(".", "").isdigit()] or [0.0])
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in rows for j in range(4) if r[5 + j].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows)}


# ---- the device arm ----------------------------------------------------------------------------------------------


def make_engine(device, overlap: bool = True):
    from livox_warp import gpu
    from livox_warp.odom import Odometry

    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=MAP_SLOTS, device=device)
    odom = Odometry(pipe, reg_slots=REG_SLOTS, frame_cap=FRAME_CAP)
    odom.reg_voxel = REG_VOXEL
    view = gpu.make_view(now=0.0, voxel=MAP_VOXEL, map_cap=MAP_SLOTS)
    # each frame's insert and carve run on a second stream beside the next frame's registration
    odom.integrate(view, MAP_VOXEL, carve_every=1, overlap=overlap)
    return pipe, odom


def run_device(frames, traj, warmup: int, steps: int, device, clocks: "Clocks | None"):
    import torch

    from livox_warp import _lib

    pipe, odom = make_engine(device)
    T0 = traj.poses(np.array([0.5 * FRAME_DT]))[0]
    odom.reset(T0)
    dev = [(torch.from_numpy(x).to(device), torch.from_numpy(a.view(np.int32)).to(device),
            torch.from_numpy(t).to(device), len(t), float(t.min()), float(t.max())) for x, a, t in frames]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)

    def step(k):
        sx, sa, st, n, t0, t1 = dev[k]
        sf = pipe._stage_frame if pipe._stage_frame is not None and pipe._stage_frame.numel() >= n else None
        if sf is None:
            pipe._ensure_stage(n)
            sf = pipe._stage_frame
        _lib.call("lw_frame_ids", _lib.ptr(st), n, float(1.0 / FRAME_DT), _lib.ptr(sf), _lib.stream_ptr())
        odom.push(sx, sa, st, n, t0, t1)
        if odom.side_stream is not None:
            stream.wait_stream(odom.side_stream)  # the step's end event covers the insert and carve it started

    for k in range(warmup):
        step(k)
    torch.cuda.synchronize(device)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    _lib.prof_reset()
    _lib.prof_enable(True)
    _lib.launches(reset=True)
    if clocks:
        clocks.start()
    torch.cuda.synchronize(device)
    for j in range(steps):
        flush.fill_(float(j))  # L2 flush, outside the step's events
        evs[j][0].record(stream)
        step(warmup + j)
        evs[j][1].record(stream)
    torch.cuda.synchronize(device)
    launches = _lib.launches()
    _lib.prof_enable(False)
    step_ms = np.array([a.elapsed_time(b) for a, b in evs])
    names = ("gn", "carve", "map_insert", "thin", "reg_insert", "frame_append", "control")
    prof = {n: _lib.prof_read(n) for n in names}
    clk = None
    if clocks:
        # the sequence goes on, untimed, so the clock sampler (100 ms period) sees this load for SOAK_S more
        k, t_soak = warmup + steps, time.time() + SOAK_S
        while time.time() < t_soak and k < len(dev):
            step(k)
            k += 1
            if k % 20 == 0:
                torch.cuda.synchronize(device)
        torch.cuda.synchronize(device)
        clk = clocks.stop()
        clk["window"] = f"the timed frames and {k - warmup - steps} more frames of the sequence"
    odom.flush()
    torch.cuda.synchronize(device)
    return {"step_ms": step_ms, "prof": prof, "launches": launches, "clocks": clk, "odom": odom, "pipe": pipe}


def run_e2e(frames, traj, warmup: int, steps: int, device):
    """Through the public API from host buffers: stage (pinned H2D), push, pose read back every frame."""
    import torch

    pipe, odom = make_engine(device)
    odom.reset(traj.poses(np.array([0.5 * FRAME_DT]))[0])
    pose_host = torch.empty(16, dtype=torch.float64, pin_memory=True)
    stream = torch.cuda.current_stream(device)

    def step(k):
        x, a, t = frames[k]
        sx, sa, st, sf = pipe.stage(x, a, t, len(t), 1.0 / FRAME_DT)
        odom.push(sx, sa, st, len(t), float(t.min()), float(t.max()))
        pose_host.copy_(odom._state[:128].view(torch.float64), non_blocking=True)
        stream.synchronize()  # the caller consumes the frame's pose
        return pose_host.numpy()

    for k in range(warmup):
        step(k)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for j in range(steps):
        step(warmup + j)
    if odom.side_stream is not None:
        stream.wait_stream(odom.side_stream)  # the last frames' insert and carve inside the timed region
    e1.record(stream)
    torch.cuda.synchronize(device)
    ms = e0.elapsed_time(e1)
    n_pts = np.mean([len(frames[warmup + j][2]) for j in range(steps)])
    return {"ms": ms, "h2d": int(round(n_pts * 20)), "d2h": 128}


def roofline(res, frames, traj, warmup, steps, peak):
    """The dominant kernel's achieved GB/s: algorithmic bytes per launch / live average launch time."""
    from livox_warp import roofline as rl

    prof = res["prof"]
    name = max(prof, key=lambda n: prof[n][0])
    ms, cnt = prof[name]
    odom, pipe = res["odom"], res["pipe"]
    recs = {r[0]: r for r in odom.traj_records()}
    reg_keys = odom.reg_keys.cpu().numpy()
    reg_keys = reg_keys[reg_keys != -1]
    map_keys = pipe.map_keys.cpu().numpy()
    map_keys = map_keys[map_keys != -1]
    sample = list(range(warmup, warmup + steps, max(1, steps // 12)))
    per_launch = []
    for k in sample:
        if k not in recs:
            continue
        _, _, T, ok, iters, corr = recs[k]
        x = frames[k][0]
        if name == "gn":
            ds = rl.thin_host(x, REG_VOXEL)
            per_launch.append(rl.gn_bytes(ds, T, reg_keys, REG_VOXEL, max(iters, 1), odom._gn.grid,
                                          frame_points=len(x)))
        elif name == "carve":
            per_launch.append(rl.carve_bytes(x, T, map_keys, MAP_VOXEL))
        else:
            per_launch.append(rl.map_insert_bytes(x, T, MAP_VOXEL))
    if name == "gn":
        launches_per_frame = 2  # the first registration and the (usually gated-off) re-registration
        bytes_per_launch = float(np.mean(per_launch)) / launches_per_frame
    else:
        bytes_per_launch = float(np.mean(per_launch))
    avg_ms = ms / max(cnt, 1)
    achieved = bytes_per_launch / (avg_ms * 1e-3) / 1e9
    traffic = SEQ_TRAFFIC.get(name)
    return {"kernel": name, "bound": "hbm", "achieved": round(achieved, 3), "peak": peak["hbm_gbs"], "unit": "GB/s",
            "frac": round(achieved / peak["hbm_gbs"], 5), "traffic": traffic,
            "traffic_source": SEQ_TRAFFIC_SRC if traffic else None,
            "peak_source": peak["source"], "avg_launch_us": round(avg_ms * 1e3, 2), "launches": int(cnt),
            "algorithmic_bytes_per_launch": int(bytes_per_launch),
            "kernel_ms_share": {n: round(prof[n][0] / max(sum(v[0] for v in prof.values()), 1e-9), 4) for n in prof}}


def pose_drift(odom, traj, oracle_poses: dict) -> dict:
    """Registered poses against the simulated ground truth (every frame) and against the float64 oracle run on
    the frames the CPU baseline processed."""
    from scipy.spatial.transform import Rotation

    def pose_error(A, B):
        d = np.linalg.inv(A) @ B
        return float(np.linalg.norm(d[:3, 3])), float(np.degrees(np.linalg.norm(Rotation.from_matrix(d[:3, :3]).as_rotvec())))

    recs = odom.traj
    gt = [pose_error(traj.poses(np.array([tm]))[0], T) for k, tm, T in recs]
    orc = [pose_error(oracle_poses[k], T) for k, tm, T in recs if k in oracle_poses]
    g = np.array(gt)
    o = np.array(orc) if orc else np.zeros((1, 2))
    return {"frames": len(recs), "gt_rmse_m": round(float(np.sqrt((g[:, 0] ** 2).mean())), 4),
            "gt_max_m": round(float(g[:, 0].max()), 4), "gt_rot_rmse_deg": round(float(np.sqrt((g[:, 1] ** 2).mean())), 3),
            "vs_fp64_oracle_frames": len(orc), "vs_fp64_oracle_max_m": round(float(o[:, 0].max()), 6),
            "vs_fp64_oracle_max_deg": round(float(o[:, 1].max()), 5)}


# DRAM bytes (read + write) per launch from one ncu capture of the sequence (profiles/k_gn_k_carve_sequence.md,
# rounded as summarised there) and of the coarse search (profiles/k_score_grid_office_coarse.md)
SEQ_TRAFFIC = {"gn": 2_186_752, "carve": 6_774_848}  # gn: thinning + iterations (mean of two full launches); carve: setup + walk
SEQ_TRAFFIC_SRC = "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/k_gn_k_carve_sequence.md"
SINGLE_TRAFFIC = {"gn": 1_387_776}  # ncu, one timed launch of the single-frame case (1,387,520 B read, 256 written)
SINGLE_TRAFFIC_SRC = "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/k_gn_single_frame.md"
COARSE_TRAFFIC = 42_780_928 + 71_592_448
COARSE_TRAFFIC_SRC = "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/k_score_grid_office_coarse.md"


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d.get("bf16_tflops", 1590.0)),
                "bf16_tflops_sustained": float(d.get("bf16_tflops_sustained", d.get("bf16_tflops", 1400.0))),
                "source": "measured (MEASURED_PEAKS.json)"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0,
            "source": "fallback 6.65 TB/s, 1.59 PFLOP/s"}


# ---- replicas ---------------------------------------------------------------------------------------------------


def max_over_ranks(x: float, device) -> float:
    """The largest of every rank's x (a device time): the job takes as long as its slowest replica. One
    all-reduce on `device` (a CUDA tensor for NCCL, a CPU one for gloo); x itself with one process."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(units_per_rank: int, world: int, ms_max: float) -> float:
    """Whole-job throughput of `world` replicas that each processed units_per_rank in at most ms_max."""
    return world * units_per_rank / (ms_max * 1e-3)


# ---- the CPU arms ------------------------------------------------------------------------------------------------


def cpu_pipeline(frames, traj, warmup: int, budget_s: float, max_frames: int, threads: int):
    """The oracle's frame pipeline (odometry + integration insert + carving) over frames 0..; the first `warmup`
    frames untimed, then frames until max_frames or budget_s of CPU time. Returns (frames timed, seconds)."""
    os.environ["LW_ORACLE_THREADS"] = str(threads)
    from oracle import oracle

    p = oracle.Params(reg_voxel=REG_VOXEL)
    T0 = traj.poses(np.array([0.5 * FRAME_DT]))[0]
    od = oracle.Odometry(REG_SLOTS, p, T0)
    om = oracle.Map(MAP_SLOTS)
    poses = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (oracle.POSE_SLOTS, 1))
    view = _oracle_view(oracle)
    timed, t_total = 0, 0.0
    poses_out = {}
    for k, (x, a, t) in enumerate(frames):
        t0 = time.perf_counter()
        raw = np.ascontiguousarray(np.concatenate([x, t[:, None]], 1), dtype=np.float32)
        T, xyz4, ok = od.frame(k, raw, a)
        poses[k & (oracle.POSE_SLOTS - 1)] = T.astype(np.float32).reshape(16)
        fid = np.full(len(t), k, np.int32)
        om.insert(xyz4, a, t, fid, poses, view, MAP_VOXEL)
        om.carve(xyz4, a, fid, poses, MAP_VOXEL, every=1, nthreads=threads)
        dt = time.perf_counter() - t0
        poses_out[k] = T
        if k >= warmup:
            timed += 1
            t_total += dt
            if timed >= max_frames or t_total >= budget_s:
                break
    return timed, t_total, poses_out


def _oracle_view(oracle):
    from livox_warp import _lib

    v = _lib.View()
    v.now, v.persist, v.min_range, v.max_range = 0.0, 0.0, 0.1, 500.0
    v.min_refl, v.noise_mask, v.ret_mask, v.crop_on = 0, 0b1111, 0b1111, 0
    v.crop_lo, v.crop_hi = (-1e9, -1e9, -1e9), (1e9, 1e9, 1e9)
    v.inv_voxel, v.map_mask = 1.0 / MAP_VOXEL, MAP_SLOTS - 1
    return v


# ---- learned start pose ------------------------------------------------------------------------------------------

LEARN_TRAIN_SEEDS = tuple(range(101, 109))  # 8 paths x 600 frames, 10 pairs per frame
LEARN_EVAL_SEEDS = (201, 202, 203)
LEARN_FRAMES = 600
LEARN_V, LEARN_W = 2.0, 120.0  # path limits: <= 2 m/s (cruise 1.4 m/s), <= 120 deg/s
LEARN_SIGMA = (0.015, 0.015, 0.015, 0.006, 0.006, 0.006)  # m, rad: perturbations of the converged pose for training


def _learn_chunk(args):
    from livox_warp import synth

    seed, n, k0, k1 = args
    scene = synth.box_room(ROOM_SEED)
    traj = synth.Handheld(scene, seed, n * FRAME_DT + 2.0, v_max=LEARN_V, w_max_deg=LEARN_W, a_max_deg=2 * LEARN_W)
    return synth.frames(scene, traj, k1 - k0, RATE, SCAN_SEED + seed, start=k0)


def learn_sequences(seeds, n_frames: int, procs: int | None = None):
    """{seed: (frames, trajectory)} of fast handheld paths in the box room (generated before any CUDA call)."""
    from livox_warp import synth

    procs = procs or min(16, os.cpu_count() or 1)
    step = max(1, math.ceil(n_frames / 8))
    jobs = [(sd, n_frames, k, min(k + step, n_frames)) for sd in seeds for k in range(0, n_frames, step)]
    with mp.get_context("spawn").Pool(procs) as pool:
        parts = pool.map(_learn_chunk, jobs)
    out = {}
    scene = synth.box_room(ROOM_SEED)
    for (sd, _, _, _), part in zip(jobs, parts):
        out.setdefault(sd, []).extend(part)
    return {sd: (fr, synth.Handheld(scene, sd, n_frames * FRAME_DT + 2.0, v_max=LEARN_V, w_max_deg=LEARN_W,
                                    a_max_deg=2 * LEARN_W)) for sd, fr in out.items()}


def run_learned(a, rank: int, world: int, local: int):
    """The learned start pose against the constant-velocity one, frame by frame (initnet.FrameByFrame)."""
    import torch

    from livox_warp import _lib, gpu
    from livox_warp.initnet import FrameByFrame, InitNet
    from livox_warp.odom import Odometry

    seqs = learn_sequences(LEARN_TRAIN_SEEDS + LEARN_EVAL_SEEDS, LEARN_FRAMES)
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 16, device=device)
    odom = Odometry(pipe, reg_slots=REG_SLOTS, frame_cap=FRAME_CAP)
    odom.reg_voxel = REG_VOXEL
    fbf = FrameByFrame(odom, nearest=True)
    t0 = time.perf_counter()
    all_sets, all_tg = [], []
    for sd in LEARN_TRAIN_SEEDS:
        frames, traj = seqs[sd]
        _, sets, tg = fbf.run(frames, traj.poses, per_frame=10, sigma=LEARN_SIGMA, seed=sd)
        all_sets.append(sets)
        all_tg.append(tg)
    sets = torch.cat(all_sets)
    tg = torch.cat(all_tg)
    del all_sets, all_tg
    n_pairs = int(tg.shape[0])
    gen_s = time.perf_counter() - t0
    perm = torch.randperm(n_pairs, generator=torch.Generator().manual_seed(0)).to(device)
    sets = sets.view(n_pairs, 2, -1, 4).index_select(0, perm).view(2 * n_pairs, -1, 4)
    tg = tg.index_select(0, perm)
    net = InitNet(device, seed=0, batch_cap=256)
    torch.cuda.synchronize(device)
    clocks = Clocks(local)
    clocks.start()
    _lib.prof_reset()
    _lib.prof_enable(True)
    t1 = time.perf_counter()
    hist = net.fit(sets, tg, epochs=a.learn_epochs, batch=256, lr=1e-3, val_frac=0.05)
    torch.cuda.synchronize(device)
    train_s = time.perf_counter() - t1
    _lib.prof_enable(False)
    clk = clocks.stop()
    clk["window"] = "the network's training"
    fwd_ms, fwd_n = _lib.prof_read("net_forward")
    # a CPU sample of the same training step: the float64 oracle's forward and backward of a few pairs
    from oracle import oracle as _o

    w_host = net.w.cpu().numpy().view(np.uint16)
    sc = net.out_scale.cpu().numpy()
    n_cpu, cpu_s = 0, 0.0
    sample = sets.view(n_pairs, 2, -1, 4)[:64].cpu().numpy()
    tgt = tg[:64].cpu().numpy()
    t_cpu = time.perf_counter()
    while n_cpu < len(sample) and time.perf_counter() - t_cpu < 10.0:
        f = _o.net_forward(w_host, sample[n_cpu:n_cpu + 1].reshape(2, -1, 4), net.in_scale, sc)
        _o.net_backward(w_host, sample[n_cpu:n_cpu + 1].reshape(2, -1, 4), f, tgt[n_cpu:n_cpu + 1], np.ones(6), sc)
        n_cpu += 1
    cpu_s = time.perf_counter() - t_cpu
    del sets
    rows = []
    _lib.launches(reset=True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for sd in LEARN_EVAL_SEEDS:
        frames, traj = seqs[sd]
        r, _, _ = fbf.run(frames, traj.poses, net=net)
        rows.extend(dict(x, seed=sd) for x in r)
    e1.record()
    torch.cuda.synchronize(device)
    eval_ms = e0.elapsed_time(e1)
    launches = _lib.launches()
    if rank != 0:
        return
    ok = [r for r in rows if r["ok"]]

    def mean(key):
        return float(np.mean([r[key] for r in ok]))

    def pct(key, i, q):
        return float(np.percentile([r[key][i] for r in ok], q))

    to_cv, to_net = mean("to_acc_cv"), mean("to_acc_net")
    line = {"metric": "mean Gauss-Newton iterations to reach the converged pose (1 mm / 0.01 deg): constant-velocity "
                      "start / learned start",
            "value": round(to_cv / max(to_net, 1e-9), 4), "unit": "x fewer iterations", "n_gpus": world,
            "steps": len(ok), "warmup": 0, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 network (fp32 accumulate), f32/f64 registration", "data": "synthetic",
            "config": {"workload": f"learned start pose: box room 8x6x3 m, 20 boxes, handheld paths <= {LEARN_V} m/s "
                                   f"(cruise {0.7 * LEARN_V:.1f}), <= {LEARN_W} deg/s; each frame registered against the "
                                   "map of the frames before it (at their true poses) from the constant-velocity "
                                   "prediction and from the network's proposal; the registration from the true pose "
                                   "is the judge",
                       "train_paths": len(LEARN_TRAIN_SEEDS), "eval_paths": len(LEARN_EVAL_SEEDS),
                       "frames_per_path": LEARN_FRAMES, "pairs": n_pairs, "sigma": LEARN_SIGMA,
                       "epochs": a.learn_epochs, "batch": 256, "max_iter": odom.max_iter},
            "iterations_to_converged": {"constant_velocity": round(to_cv, 3), "learned": round(to_net, 3)},
            "iterations_to_own_final": {"constant_velocity": round(mean("to_own_cv"), 3),
                                        "learned": round(mean("to_own_net"), 3)},
            "iterations_to_stop_test": {"constant_velocity": round(mean("iters_cv"), 3),
                                        "learned": round(mean("iters_net"), 3)},
            "start_error_vs_converged": {"constant_velocity_p50_m_deg": [round(pct("start_cv", 0, 50), 4),
                                                                         round(pct("start_cv", 1, 50), 3)],
                                         "learned_p50_m_deg": [round(pct("start_net", 0, 50), 4),
                                                               round(pct("start_net", 1, 50), 3)]},
            "final_error_vs_converged": {"constant_velocity_p95_m_deg": [round(pct("final_cv", 0, 95), 5),
                                                                         round(pct("final_cv", 1, 95), 4)],
                                         "learned_p95_m_deg": [round(pct("final_net", 0, 95), 5),
                                                               round(pct("final_net", 1, 95), 4)]},
            "judge_vs_truth_p50_m_deg": [round(pct("truth_judge", 0, 50), 4), round(pct("truth_judge", 1, 50), 3)],
            "frames_evaluated": len(ok), "frames_failed": len(rows) - len(ok),
            "train_loss": [round(x, 4) for x in hist["train"][::max(1, len(hist["train"]) // 10)]],
            "val_loss": [round(x, 4) for x in hist["val"][::max(1, len(hist["val"]) // 10)]],
            "pair_gen_s": round(gen_s, 2), "train_s": round(train_s, 2),
            "train_pairs_per_s": round(n_pairs * a.learn_epochs / max(train_s, 1e-9), 1)}
    peak = measured_peak()
    flops = 256 * 2 * 2 * _lib.NET_P * (3 * 64 + 64 * 128 + 128 * 256)  # one training batch's two point sets
    achieved = flops / (fwd_ms / max(fwd_n, 1) * 1e-3) / 1e12
    line["roofline"] = {"kernel": "net_forward (k_net_mlp + k_net_head, batch 256)", "bound": "tensor",
                        "achieved": round(achieved, 2), "peak": peak["bf16_tflops"], "unit": "TFLOP/s",
                        "frac": round(achieved / peak["bf16_tflops"], 5), "traffic": None,
                        "peak_source": peak["source"] + " bf16 burst", "launches": int(fwd_n),
                        "avg_launch_us": round(fwd_ms / max(fwd_n, 1) * 1e3, 2),
                        "flops_per_launch": flops}
    line["cpu_baseline"] = {"value": round(n_cpu / max(cpu_s, 1e-9), 3), "unit": "training pairs/s",
                            "cores": 1, "kind": "port",
                            "sample": f"{n_cpu} pairs through the float64 oracle's network forward and backward "
                                      f"({cpu_s:.1f} s); the device trains {line['train_pairs_per_s']} pairs/s"}
    line["e2e"] = {"value": line["value"], "unit": line["unit"],
                   "h2d_bytes_per_step": int(np.mean([len(f[2]) for sd in LEARN_EVAL_SEEDS for f in seqs[sd][0]]) * 20),
                   "d2h_bytes_per_step": 3 * 976 + 3 * 12 * 8 * 17,
                   "note": "measured through Odometry.register_frame from host frames (each frame copied to the "
                           f"device and three registrations read back); evaluation {eval_ms / 1e3:.1f} s"}
    line["gpu_launches"] = int(launches)
    line["clocks"] = clk
    print(json.dumps(line))


# ---- full perception frame --------------------------------------------------------------------------------------


def _frame_chunk(args):
    from livox_warp import synth

    duration, k0, k1 = args
    scene = synth.office(FRAME_SCENE_SEED, walkers=10)
    traj = synth.Handheld(scene, FRAME_PATH_SEED, duration)
    return synth.frames(scene, traj, k1 - k0, FRAME_RAYS, SCAN_SEED, start=k0, dual=True)


def frame_workload(n_frames: int, procs: int | None = None):
    from livox_warp import synth

    duration = n_frames * FRAME_DT + 2.0
    procs = procs or min(8, os.cpu_count() or 1)
    step = max(1, math.ceil(n_frames / (procs * 4)))
    chunks = [(duration, k, min(k + step, n_frames)) for k in range(0, n_frames, step)]
    with mp.get_context("spawn").Pool(procs) as pool:
        parts = pool.map(_frame_chunk, chunks)
    scene = synth.office(FRAME_SCENE_SEED, walkers=10)
    return [f for p in parts for f in p], synth.Handheld(scene, FRAME_PATH_SEED, duration)


FRAME_GROUND = dict(cell=0.5, thick=0.15, min_sup=3, thresh=0.2, slope_step=0.3)
FRAME_CLUSTER = dict(voxel=0.2, connect=0.35, min_pts=30)


def cpu_frame_pipeline(frames, traj, warmup: int, budget_s: float, max_frames: int, threads: int):
    """The oracle's full frame (odometry, insert, carve, visible set, ground, clusters); frames after `warmup`
    are timed until max_frames or budget_s. Returns (frames timed, seconds)."""
    os.environ["LW_ORACLE_THREADS"] = str(threads)
    from oracle import oracle

    p = oracle.Params(reg_voxel=REG_VOXEL)
    od = oracle.Odometry(REG_SLOTS, p, traj.poses(np.array([0.5 * FRAME_DT]))[0])
    om = oracle.Map(MAP_SLOTS)
    poses = np.tile(np.eye(4, dtype=np.float32).reshape(1, 16), (oracle.POSE_SLOTS, 1))
    view = _oracle_view(oracle)
    view.carve_on = 1
    timed, total = 0, 0.0
    for k, (x, a, t) in enumerate(frames):
        t0 = time.perf_counter()
        raw = np.ascontiguousarray(np.concatenate([x, t[:, None]], 1), dtype=np.float32)
        T, xyz4, ok = od.frame(k, raw, a)
        poses[k & (oracle.POSE_SLOTS - 1)] = T.astype(np.float32).reshape(16)
        fid = np.full(len(t), k, np.int32)
        om.insert(xyz4, a, t, fid, poses, view, MAP_VOXEL)
        om.carve(xyz4, a, fid, poses, MAP_VOXEL, every=1, nthreads=threads)
        view.now = (k + 1) * FRAME_DT
        vis = om.build(view)[0]
        gnd, _ = oracle.ground(vis, **FRAME_GROUND)
        oracle.cluster(vis, gnd, **FRAME_CLUSTER)
        dt = time.perf_counter() - t0
        if k >= warmup:
            timed += 1
            total += dt
            if timed >= max_frames or total >= budget_s:
                break
    return timed, total


def run_frame(a, rank: int, world: int, local: int):
    n_frames = a.warmup + a.steps + 1
    frames, traj = frame_workload(n_frames)
    metric = "full perception frame latency p50 (stage + odometry + insert + carve + visible set + ground + clusters)"
    config = {"workload": "full perception frame: office 40x30x3 m, 10 walkers (r 0.25 m, h 1.8 m, 1.2 m/s), "
                          "dual-return rosette 100k rays/s (~20k pts/frame), handheld path, reg voxel 0.15 m, map voxel "
                          "0.1 m (2^22 slots) with carving, ground 0.5 m slope 0.3, clusters 0.2 m connect 0.35 m",
              "frames": n_frames, "points_per_frame": int(np.mean([len(f[2]) for f in frames])),
              "l2": "not flushed: each frame's latency is measured as the pipeline runs",
              "parallelism": f"replicas x{a.gpus}"}
    if a.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as _o

        threads = _o.host_cores()
        timed, secs = cpu_frame_pipeline(frames, traj, a.warmup, max(20.0, min(120.0, 0.2 * a.steps)), a.steps,
                                         threads)
        ms = 1e3 * secs / max(timed, 1)
        print(json.dumps({"impl": "reference", "metric": metric, "value": round(ms, 3), "unit": "ms",
                          "n_gpus": a.gpus, "steps": timed, "warmup": a.warmup, "ms_per_step": round(ms, 3),
                          "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
                          "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": round(ms, 3), "unit": "ms", "cores": threads, "kind": "port",
                                           "sample": f"{timed} frames after {a.warmup} untimed, CPU restatement"},
                          "e2e": {"value": round(ms, 3), "unit": "ms", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    import torch

    from livox_warp import _lib, gpu
    from livox_warp.odom import Odometry
    from livox_warp.perception import Perception

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=MAP_SLOTS, device=device)
    odom = Odometry(pipe, reg_slots=REG_SLOTS, frame_cap=FRAME_CAP)
    odom.reg_voxel = REG_VOXEL
    view = gpu.make_view(now=0.0, voxel=MAP_VOXEL, map_cap=MAP_SLOTS, carve_on=1)
    odom.integrate(view, MAP_VOXEL, carve_every=1)
    perc = Perception(pipe, cluster_slots=1 << 20)
    odom.reset(traj.poses(np.array([0.5 * FRAME_DT]))[0])
    stream = torch.cuda.current_stream(device)
    lat_host, lat_dev, n_clusters = [], [], []

    def step(k):
        x, at, t = frames[k]
        sx, sa, st, sf = pipe.stage(x, at, t, len(t), 1.0 / FRAME_DT)
        odom.push(sx, sa, st, len(t), float(t.min()), float(t.max()))  # completes frame k - 1
        view.now = (k + 1) * FRAME_DT
        pipe.build(view, map_on=True)
        perc.ground(**FRAME_GROUND)
        return perc.cluster(**FRAME_CLUSTER)  # read back to the host

    for k in range(a.warmup):
        step(k)
    torch.cuda.synchronize(device)
    clocks = Clocks(local)
    clocks.start()
    _lib.launches(reset=True)
    _lib.prof_reset()
    _lib.prof_enable(True)
    h2d = d2h = 0
    for j in range(a.steps):
        k = a.warmup + j
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        cl = step(k)
        e1.record(stream)
        e1.synchronize()
        lat_host.append((time.perf_counter() - t0) * 1e3)
        lat_dev.append(e0.elapsed_time(e1))
        n_clusters.append(len(cl))
        h2d += len(frames[k][2]) * 20
        d2h += 12 + len(cl) * 40 + 12
    clk = clocks.stop()
    launches = _lib.launches()
    _lib.prof_enable(False)
    prof = {n: _lib.prof_read(n) for n in ("gn", "carve", "map_insert", "thin", "reg_insert", "frame_append", "control",
                                           "map_build", "ground", "cluster")}
    if rank != 0:
        return
    # parity of the last frame's labels: the oracle's ground and clusters on the same visible set
    from oracle import oracle as _o

    n = pipe.count
    vis = pipe.c_xyz[:n].cpu().numpy()
    og, _ = _o.ground(vis, **FRAME_GROUND)
    ocid, _, ocl, _ = _o.cluster(vis, og, **FRAME_CLUSTER)
    gnd_ok = bool(np.array_equal(pipe.gnd[:n].cpu().numpy(), og))
    cid_ok = bool(np.array_equal(pipe.cid[:n].cpu().numpy(), ocid)) and len(ocl) == len(cl)
    threads = _o.host_cores()
    timed, secs = cpu_frame_pipeline(frames, traj, a.warmup, a.cpu_budget, max(3, min(40, a.steps)), threads)
    lh, ld = np.array(lat_host), np.array(lat_dev)
    recs = odom.traj
    from livox_warp.localize import pose_difference

    gt = np.array([pose_difference(traj.poses(np.array([tm]))[0], T) for _, tm, T in recs])
    top = {n: prof[n] for n in ("gn", "carve", "map_insert")}  # the kernels roofline() has byte counts for
    roof = roofline({"prof": top, "odom": odom, "pipe": pipe}, frames, traj, a.warmup, a.steps, measured_peak())
    total_ms = sum(v[0] for v in prof.values())
    roof["kernel_ms_share"] = {n: round(v[0] / max(total_ms, 1e-9), 4) for n, v in prof.items()}
    roof["traffic"], roof["traffic_source"] = None, None  # the ncu traffic figures are the sequence's
    line = {"metric": metric, "value": round(float(np.percentile(lh, 50)), 4), "unit": "ms", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(float(lh.mean()), 4),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 solve)",
            "data": "synthetic", "config": config,
            "latency_ms": {"p50": round(float(np.percentile(lh, 50)), 4), "p99": round(float(np.percentile(lh, 99)), 4),
                           "max": round(float(lh.max()), 4), "device_p50": round(float(np.percentile(ld, 50)), 4),
                           "device_p99": round(float(np.percentile(ld, 99)), 4)},
            "frames_per_s": round(1e3 * a.steps / float(lh.sum()), 3),
            "visible_points_last": int(n), "clusters_mean": round(float(np.mean(n_clusters)), 2),
            "labels_bit_exact_last_frame": {"gnd": gnd_ok, "cid": cid_ok},
            "pose_vs_gt": {"rmse_m": round(float(np.sqrt((gt[:, 0] ** 2).mean())), 4),
                           "max_m": round(float(gt[:, 0].max()), 4), "max_deg": round(float(gt[:, 1].max()), 3)},
            "roofline": roof,
            "cpu_baseline": {"value": round(1e3 * secs / max(timed, 1), 3), "unit": "ms", "cores": threads,
                             "kind": "port", "sample": f"{timed} frames of the same sequence through the CPU oracle "
                                                       f"(odometry, insert, carve, visible set, ground, clusters)"},
            "e2e": {"value": round(float(np.percentile(lh, 50)), 4), "unit": "ms",
                    "h2d_bytes_per_step": int(h2d / a.steps), "d2h_bytes_per_step": int(d2h / a.steps)},
            "gpu_launches": int(launches), "clocks": clk}
    print(json.dumps(line))


# ---- single-frame scan-to-map ICP (the headline configuration) --------------------------------------------------

SINGLE_VOXEL = 0.2    # registration voxel of the single-frame case
SINGLE_ITERS = 10     # Gauss-Newton iterations at most
SINGLE_FRAMES = 8     # distinct seeded frames, cycled over the timed steps
SINGLE_REG_SLOTS = 1 << 21  # the reference's default registration table (odom.py:461)


def single_workload():
    from livox_warp import synth

    return synth.single_frame_case(synth.box_room(ROOM_SEED), SINGLE_FRAMES, RATE)


def _single_oracle_params(_o):
    return _o.Params(reg_voxel=SINGLE_VOXEL, max_iter=SINGLE_ITERS)


def single_oracle(w, threads: int, budget_s: float, max_frames: int):
    """The float64 oracle on the single-frame case: the map of the static frames, then deskew + thinning +
    registration of moving frames in turn (cycling) until budget_s of CPU time or max_frames. Returns (frames
    timed, seconds, {j: T} for every distinct frame registered, {j: stats})."""
    os.environ["LW_ORACLE_THREADS"] = str(threads)
    from oracle import oracle as _o

    T0, base, moving = w
    oreg = _o.RegMap(SINGLE_REG_SLOTS)
    for x, a, t in base:
        oreg.insert(np.ascontiguousarray(np.concatenate([x, t[:, None]], 1), dtype=np.float32), a, T0, SINGLE_VOXEL,
                    60.0, 0b1111)
    oreg.records(SINGLE_VOXEL, 0.02, 0.05)
    p = _single_oracle_params(_o)
    timed, secs, poses, stats = 0, 0.0, {}, {}
    while timed < max_frames and (secs < budget_s or len(poses) < len(moving)):
        j = timed % len(moving)
        x, a, t, t_mid, _ = moving[j]
        t0 = time.perf_counter()
        raw = np.ascontiguousarray(np.concatenate([x, t[:, None]], 1), dtype=np.float32)
        d = _o.deskew(raw, t_mid, 1.0 / FRAME_DT, np.zeros(6, np.float32))
        ds = _o.thin(d, a, np.float32(2.0 / SINGLE_VOXEL), p.min_range, p.max_range, p.ret_mask)
        T, ok, st = _o.register(ds, T0, oreg, p, nthreads=threads)
        secs += time.perf_counter() - t0
        timed += 1
        poses[j], stats[j] = T, st
    return timed, secs, poses, stats


def run_single(a, rank: int, world: int, local: int):
    w = single_workload()  # before any CUDA call
    T0, base, moving = w
    pts = int(np.mean([len(f[2]) for f in moving]))
    metric = "single-frame scan-to-map ICP frames/s (deskew + thinning + <=10 Gauss-Newton iterations, f64 solve)"
    config = {"workload": "single-frame scan-to-map ICP: box room 8x6x3 m, 20 boxes, rosette 100k pts/s "
                          f"(~{pts} pts/frame), map of {len(base)} static frames at 0.2 m voxels (2^21 slots), "
                          "sensor 0.5 m/s + 20 deg/s, constant-velocity start (the rest pose and zero twist of a "
                          f"sensor that just started moving), <= {SINGLE_ITERS} Gauss-Newton iterations; "
                          f"{len(moving)} seeded frames cycled",
              "points_per_frame": pts, "frames_distinct": len(moving),
              "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{a.gpus}"}
    if a.impl == "reference":
        if rank != 0:
            return
        from oracle import oracle as _o

        threads = _o.host_cores()
        single_oracle(w, threads, 0.0, a.warmup)  # untimed warm-up registrations
        timed, secs, _, _ = single_oracle(w, threads, 15.0, 1 << 30)
        v = timed / secs
        print(json.dumps({"impl": "reference", "metric": metric, "value": round(v, 3), "unit": "frames/s",
                          "n_gpus": a.gpus, "steps": timed, "warmup": a.warmup,
                          "ms_per_step": round(1e3 * secs / max(timed, 1), 3), "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
                          "config": config,
                          "cpu_baseline": {"value": round(v, 3), "unit": "frames/s", "cores": threads, "kind": "port",
                                           "sample": f"{timed} registrations of the same frames; NVIDIA Warp (the "
                                                     "reference runtime) is not installed, so this is the CPU "
                                                     "restatement of its kernels (C++/OpenMP) with the float64 "
                                                     "host solve"},
                          "e2e": {"value": round(v, 3), "unit": "frames/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    import torch
    import torch.distributed as dist

    from livox_warp import _lib, gpu
    from livox_warp.odom import Odometry

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)
    pipe = gpu.Pipeline(ring_capacity=1 << 16, map_capacity=1 << 16, device=device)
    odom = Odometry(pipe, reg_slots=SINGLE_REG_SLOTS, frame_cap=1 << 15)
    odom.reg_voxel, odom.max_iter = SINGLE_VOXEL, SINGLE_ITERS
    odom.reset(T0)
    for x, at, t in base:
        x4 = torch.from_numpy(np.ascontiguousarray(np.concatenate([x, t[:, None]], 1), dtype=np.float32)).to(device)
        odom.insert_frame(x4, torch.from_numpy(at.view(np.int32)).to(device), T0)
    dev = [(torch.from_numpy(np.ascontiguousarray(np.concatenate([x, t[:, None]], 1), dtype=np.float32)).to(device),
            torch.from_numpy(at.view(np.int32)).to(device), t_mid) for x, at, t, t_mid, _ in moving]
    zero = np.zeros(6, np.float32)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    stream = torch.cuda.current_stream(device)

    def step(k):
        x4, at, t_mid = dev[k % len(dev)]
        odom.register_frame(x4, at, None, t_mid, zero, T0, sync=False)

    for k in range(a.warmup):
        step(k)
    torch.cuda.synchronize(device)
    if world > 1:
        dist.barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    clocks = Clocks(local)
    _lib.prof_reset()
    _lib.prof_enable(True)
    _lib.launches(reset=True)
    clocks.start()
    torch.cuda.synchronize(device)
    for j in range(a.steps):
        flush.fill_(float(j))  # L2 flush, outside the step's events
        evs[j][0].record(stream)
        step(a.warmup + j)
        evs[j][1].record(stream)
    torch.cuda.synchronize(device)
    launches = _lib.launches()
    _lib.prof_enable(False)
    gn_ms, gn_cnt = _lib.prof_read("gn")
    # the timed steps last milliseconds, less than the sampler's 100 ms period: the same steps go on, untimed,
    # for SOAK_S more so that the clock samples see this load
    t_soak = time.time() + SOAK_S
    j = 0
    while time.time() < t_soak:
        for _ in range(20):
            flush.fill_(float(j))
            step(j)
            j += 1
        torch.cuda.synchronize(device)
    clk = clocks.stop()
    clk["window"] = f"the timed steps and {SOAK_S} s more of the same steps"
    step_ms = np.array([e0.elapsed_time(e1) for e0, e1 in evs])
    ms_total = max_over_ranks(float(step_ms.sum()), device)
    value = replica_rate(a.steps, world, ms_total)
    # every distinct frame once more, with its result read back: the poses the oracle checks
    res = []
    for j in range(len(dev)):
        step(j)
        res.append(odom.registration())
    # end to end through the public API: host arrays copied to pinned memory, read by the launch over the bus, and
    # the result read back every step
    for k in range(a.warmup):
        x, at, t, t_mid, _ = moving[k % len(moving)]
        odom.register_frame(x, at, t, t_mid, zero, T0)
    torch.cuda.synchronize(device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for j in range(a.steps):
        x, at, t, t_mid, _ = moving[(a.warmup + j) % len(moving)]
        odom.register_frame(x, at, t, t_mid, zero, T0)
    e1.record(stream)
    torch.cuda.synchronize(device)
    e_ms = max_over_ranks(e0.elapsed_time(e1), device)
    import ctypes as _ct

    e2e = {"value": round(replica_rate(a.steps, world, e_ms), 3), "unit": "frames/s",
           "h2d_bytes_per_step": pts * 20, "d2h_bytes_per_step": _ct.sizeof(_lib.OdomState)}
    reg_keys = odom.reg_keys.cpu().numpy()
    reg_keys = reg_keys[reg_keys != -1]
    grid = odom._gn.grid
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    from livox_warp import roofline as rl
    from oracle import oracle as _o

    threads = _o.host_cores()
    timed, secs, opose, ostats = single_oracle(w, threads, min(a.cpu_budget, 15.0), 1 << 30)
    err = np.array([_o.pose_error(opose[j], res[j][0]) for j in range(len(moving))])
    gt = np.array([_o.pose_error(moving[j][4], res[j][0]) for j in range(len(moving))])
    iters = np.array([res[j][2]["iters"] for j in range(len(moving))])
    per_launch = []
    for j, (x, at, t, t_mid, _) in enumerate(moving):
        ds = rl.thin_host(x, SINGLE_VOXEL)
        per_launch.append(rl.gn_bytes(ds, res[j][0], reg_keys, SINGLE_VOXEL, max(int(iters[j]), 1), grid,
                                      frame_points=len(x)))
    avg_ms = gn_ms / max(gn_cnt, 1)
    achieved = float(np.mean(per_launch)) / (avg_ms * 1e-3) / 1e9
    peak = measured_peak()
    traffic = SINGLE_TRAFFIC.get("gn")
    roof = {"kernel": "gn", "bound": "hbm", "achieved": round(achieved, 3), "peak": peak["hbm_gbs"], "unit": "GB/s",
            "frac": round(achieved / peak["hbm_gbs"], 5), "traffic": traffic,
            "traffic_source": SINGLE_TRAFFIC_SRC if traffic else None, "peak_source": peak["source"],
            "avg_launch_us": round(avg_ms * 1e3, 2), "launches": int(gn_cnt),
            "algorithmic_bytes_per_launch": int(np.mean(per_launch)),
            "kernel_ms_share": {"gn": round(gn_ms / max(float(step_ms.sum()), 1e-9), 4)}}
    line = {"metric": metric, "value": round(value, 3), "unit": "frames/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms_total / a.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 solve)", "data": "synthetic",
            "config": config, "points_per_s": round(value * pts, 1),
            "step_ms_p50_p99": [round(float(np.percentile(step_ms, 50)), 4),
                                round(float(np.percentile(step_ms, 99)), 4)],
            "pose_error_vs_fp64": {"frames": len(moving), "max_m": round(float(err[:, 0].max()), 7),
                                   "max_deg": round(float(err[:, 1].max()), 6),
                                   "bound": "1 mm / 0.01 deg", "within_bound": bool((err[:, 0] <= 1e-3).all() and
                                                                                   (err[:, 1] <= 0.01).all())},
            "pose_error_vs_truth": {"max_m": round(float(gt[:, 0].max()), 5), "max_deg": round(float(gt[:, 1].max()), 4)},
            "gn_iterations": {"mean": round(float(iters.mean()), 2),
                              "oracle_mean": round(float(np.mean([ostats[j]["iters"] for j in ostats])), 2)},
            "roofline": roof,
            "cpu_baseline": {"value": round(timed / secs, 3), "unit": "frames/s", "cores": threads, "kind": "port",
                             "sample": f"{timed} registrations of the same frames through the CPU oracle (C++/OpenMP "
                                       f"accumulation, numpy float64 solve), {secs:.1f} s"},
            "e2e": e2e, "gpu_launches": int(launches), "clocks": clk}
    print(json.dumps(line))


# ---- batched global localisation -----------------------------------------------------------------------------------


def _loc_scans(args):
    from livox_warp import synth

    T, sizes, seeds = args
    scene = synth.office(LOC_SEED)
    return [synth.spin_scan(scene, T[i], int(sizes[i]), int(seeds[i])) for i in range(len(T))]


def loc_workload(n_hyp: int = LOC_HYP, spacing: float = LOC_SPACING, procs: int | None = None):
    """Prior map, packed scans (N, 4), per-hypothesis row ranges, true and initial poses (before any CUDA call)."""
    from livox_warp import synth

    scene = synth.office(LOC_SEED)
    xyz, nrm = synth.sample_surfaces(scene, spacing, LOC_SEED, jitter=0.002)
    T_true = synth.free_poses(scene, LOC_HYP, LOC_POSE_SEED, z=LOC_Z, margin=0.6)[:n_hyp]
    rng = np.random.default_rng(LOC_POSE_SEED + 1)
    sizes = rng.integers(LOC_PTS[0], LOC_PTS[1] + 1, LOC_HYP)[:n_hyp]
    seeds = 1000 + np.arange(n_hyp)
    procs = procs or min(8, os.cpu_count() or 1)
    parts = np.array_split(np.arange(n_hyp), procs * 2)
    jobs = [(T_true[p], sizes[p], seeds[p]) for p in parts if len(p)]
    with mp.get_context("spawn").Pool(procs) as pool:
        scans = [s for chunk in pool.map(_loc_scans, jobs) for s in chunk]
    n = np.array([len(x) for x in scans], dtype=np.int64)
    hi = np.cumsum(n)
    lo = hi - n
    pts4 = np.zeros((int(hi[-1]), 4), np.float32)
    for x, a in zip(scans, lo):
        pts4[a:a + len(x), :3] = x
    # the hypotheses: the true pose snapped to a 0.5 m xy grid and a 5 deg heading grid (a coarse search's cells)
    T0 = T_true.copy()
    yaw = np.arctan2(T_true[:, 1, 0], T_true[:, 0, 0])
    yq = np.round(np.degrees(yaw) / 5.0) * np.radians(5.0)
    for h in range(n_hyp):
        c, s_ = math.cos(yq[h]), math.sin(yq[h])
        T0[h, :3, :3] = np.array([[c, -s_, 0.0], [s_, c, 0.0], [0.0, 0.0, 1.0]])
        T0[h, :2, 3] = np.round(T_true[h, :2, 3] / 0.5) * 0.5
    return {"xyz": xyz, "nrm": nrm, "pts4": pts4, "lo": lo, "hi": hi, "T_true": T_true, "T0": T0}


def _loc_success(T, T_true):
    from livox_warp.localize import pose_difference

    err = np.array([pose_difference(T_true[h], T[h]) for h in range(len(T))])
    ok = (err[:, 0] < 0.1) & (err[:, 1] < 1.0)
    return float(ok.mean()), err


def loc_oracle(og, w, idx, threads):
    """The oracle's batched ICP + evaluation of hypotheses idx: (T, count, iters, eval, seconds)."""
    from livox_warp.localize import SCHEDULE_ICP

    os.environ["LW_ORACLE_THREADS"] = str(threads)
    n = w["hi"][idx] - w["lo"][idx]
    hi = np.cumsum(n)
    lo = hi - n
    pts4 = np.concatenate([w["pts4"][w["lo"][h]:w["hi"][h]] for h in idx])
    t0 = time.perf_counter()
    T, count, iters = og.icp(pts4, lo, hi, w["T0"][idx], SCHEDULE_ICP, nthreads=threads)
    ev = og.evaluate(pts4, lo, hi, T, nthreads=threads)
    return T, count, iters, ev, time.perf_counter() - t0


def run_localize(a, rank: int, world: int, local: int):
    from oracle import oracle as _o

    w = loc_workload(a.loc_hyp, a.loc_spacing)
    K = len(w["T0"])
    metric = "batched global localisation hypotheses/s (point-to-plane ICP schedule + evaluation)"
    config = {"workload": f"global localisation: office 40x30x3 m (walls, doors, 200 boxes), prior map "
                          f"{len(w['xyz']):,} pts at {a.loc_spacing * 1e3:.0f} mm with normals, {K} hypotheses "
                          f"(xy on a 0.5 m grid, yaw on 5 deg, z {LOC_Z} m) each with its own 360-degree scan of "
                          f"U[{LOC_PTS[0]}, {LOC_PTS[1]}] pts",
              "map_points": int(len(w["xyz"])), "hypotheses": K, "scan_points_total": int(len(w["pts4"])),
              "schedule": "(0.40,8),(0.20,8),(0.10,8),(0.05,10)", "l2": "flushed between steps (256 MB write)",
              "parallelism": f"replicas x{a.gpus}"}
    if a.impl == "reference":
        if rank != 0:
            return
        threads = _o.host_cores()
        og = _o.PriorGrid(_o.prior_prepare(w["xyz"], w["nrm"]))
        k = min(K, max(threads, 8))
        T, count, iters, ev, secs = loc_oracle(og, w, np.arange(k), threads)
        v = k / secs
        line = {"impl": "reference", "metric": metric, "value": round(v, 3), "unit": "hypotheses/s",
                "n_gpus": a.gpus, "steps": 1, "warmup": 0, "ms_per_step": round(1e3 * secs, 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": round(v, 3), "unit": "hypotheses/s", "cores": threads, "kind": "port",
                                 "sample": f"the first {k} hypotheses as one batch through the CPU restatement "
                                           "(NVIDIA Warp is not installed)"},
                "e2e": {"value": round(v, 3), "unit": "hypotheses/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return
    import torch

    from livox_warp import _lib
    from livox_warp import roofline as rl
    from livox_warp.localize import SCHEDULE_ICP, GlobalLocalizer
    from livox_warp.mapgrid import PriorGrid

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    grid = PriorGrid({"xyz": w["xyz"], "normal": w["nrm"]}, device)
    prep_s = time.perf_counter() - t0
    grid.build()
    n_all = len(w["pts4"])
    loc = GlobalLocalizer(grid, device, hyp_cap=K, pts_cap=n_all)
    stream = torch.cuda.current_stream(device)
    pinned = torch.from_numpy(w["pts4"]).pin_memory()
    # autotune (tile per CTA) through the public call, then capture the launch in a graph
    res = loc.register_packed(pinned, w["lo"], w["hi"], w["T0"])
    tile, minb = res.tile, res.blocks_per_sm
    replay = loc.register_graph(w["lo"], w["hi"], SCHEDULE_ICP, tile, blocks_per_sm=minb)
    b = loc.batch
    T0_dev = torch.from_numpy(w["T0"].reshape(K, 16).copy()).to(device)
    b.pts[:n_all].copy_(pinned.to(device))
    b.stage(w["lo"], w["hi"], tile, stream)
    g = loc._graphs[(tuple(SCHEDULE_ICP), tile, minb)]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)

    def dev_step():
        b.T[:K].copy_(T0_dev)
        g.replay()

    for _ in range(a.warmup):
        dev_step()
    torch.cuda.synchronize(device)
    clocks = Clocks(local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    clocks.start()
    torch.cuda.synchronize(device)
    for j in range(a.steps):
        flush.fill_(float(j))
        evs[j][0].record(stream)
        dev_step()
        evs[j][1].record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    step_ms = np.array([x.elapsed_time(y) for x, y in evs])
    T_dev = b.T[:K].cpu().numpy().reshape(K, 4, 4)
    iters = int(b.outs[b.o_it].item())
    ms_total = float(step_ms.sum())
    value = world * a.steps * K / (ms_total * 1e-3)
    # e2e: from pinned host scans through register_packed (H2D of scans, tiles and poses; D2H of poses and fits)
    for _ in range(3):
        loc.register_packed(pinned, w["lo"], w["hi"], w["T0"], tile=tile, blocks_per_sm=minb)
    torch.cuda.synchronize(device)
    e_steps = max(3, min(a.steps, 20))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e_steps):
        r = loc.register_packed(pinned, w["lo"], w["hi"], w["T0"], tile=tile, blocks_per_sm=minb)
    e1.record(stream)
    torch.cuda.synchronize(device)
    e_ms = e0.elapsed_time(e1)
    nt = int(b.h_ints[1])
    h2d = n_all * 16 + K * 128 + 4 * (2 + K + K + 1 + 2 * nt)
    d2h = K * 128 + 4 * (4 * K + 2)
    # the timed region replays the captured graph (k_loc_reset + k_loc_icp) once per step; graph replays do not
    # pass through the library's host-side launch counter
    launches = 2 * a.steps
    if rank != 0:
        return
    success, err = _loc_success(r.T, w["T_true"])
    assert np.array_equal(r.T, T_dev), "graph replay and the public call disagree"
    # roofline of k_loc_icp: algorithmic bytes / the measured step time (the step is that one launch)
    peak = measured_peak()
    lb = rl.loc_bytes(grid._host["start"], grid.origin, grid.dims, grid.cell, w["pts4"], w["lo"], w["hi"], T_dev,
                      iters, nt)
    avg_ms = ms_total / a.steps
    ach = lb["bytes"] / (avg_ms * 1e-3) / 1e9
    roof = {"kernel": "k_loc_icp", "bound": "hbm", "achieved": round(ach, 3), "peak": peak["hbm_gbs"],
            "unit": "GB/s", "frac": round(ach / peak["hbm_gbs"], 5), "traffic": None,
            "peak_source": peak["source"], "avg_launch_us": round(avg_ms * 1e3, 2), "iterations": iters,
            "algorithmic_bytes_per_launch": int(lb["bytes"]), "distinct_cells": lb["cells"],
            "distinct_map_points": lb["visited_points"], "tile": tile,
            "blocks_per_sm": minb, "autotune_ms": {f"{t}x{m}": round(v, 3) for (t, m), v in
                                                   next(iter(loc.tuner.trials.values()), {}).items()}}
    # parity and the CPU baseline: the first 16 hypotheses as one batch, GPU and oracle
    threads = _o.host_cores()
    # the oracle's grid over the same prepared arrays; its flooded seeds are the device's, which the parity
    # tests hold bit-exact to the oracle's own flood (flooding 43M cells on the host would take a minute)
    og = _o.PriorGrid(grid._host, build=False)
    og.nn[:] = grid.nn.cpu().numpy()
    idx = np.arange(min(16, K))
    oT, ocount, oiters, oev, secs = loc_oracle(og, w, idx, threads)
    n16 = w["hi"][idx] - w["lo"][idx]
    hi16 = np.cumsum(n16)
    lo16 = hi16 - n16
    p16 = torch.from_numpy(np.concatenate([w["pts4"][w["lo"][h]:w["hi"][h]] for h in idx])).pin_memory()
    g16 = loc.register_packed(p16, lo16, hi16, w["T0"][idx], tile=tile, blocks_per_sm=minb)
    from livox_warp.localize import pose_difference

    pd = np.array([pose_difference(oT[h], g16.T[h]) for h in range(len(idx))])
    line = {"metric": metric, "value": round(value, 3), "unit": "hypotheses/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(avg_ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 tile sums, solve and poses)",
            "data": "synthetic", "config": config,
            "success_rate": round(success, 4), "pose_err_median_m": round(float(np.median(err[:, 0])), 4),
            "pose_err_median_deg": round(float(np.median(err[:, 1])), 4),
            "step_ms_p50_p99": [round(float(np.percentile(step_ms, 50)), 4),
                                round(float(np.percentile(step_ms, 99)), 4)],
            "roofline": roof,
            "cpu_baseline": {"value": round(len(idx) / secs, 3), "unit": "hypotheses/s", "cores": threads,
                             "kind": "port",
                             "sample": f"the first {len(idx)} hypotheses as one batch through the CPU oracle "
                                       f"(C++/OpenMP, float64 terms), {secs:.1f} s"},
            "vs_fp64_oracle": {"hypotheses": len(idx), "max_m": round(float(pd[:, 0].max()), 7),
                               "max_deg": round(float(pd[:, 1].max()), 6), "iters_gpu": g16.iters,
                               "iters_oracle": oiters},
            "e2e": {"value": round(world * e_steps * K / (e_ms * 1e-3), 3), "unit": "hypotheses/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            "gpu_launches": int(launches), "graph": True, "clocks": clk, "prepare_s": round(prep_s, 2),
            "grid_build_s": round(grid.build_s, 3)}
    print(json.dumps(line))


# ---- coarse hypothesis scoring (k_score_grid) --------------------------------------------------------------------

COARSE_SPACING = 0.03  # prior-map sample spacing (m): the scores read only the grid's distance field
COARSE_PTS = 1024      # scan points per hypothesis (localize.py:365, n_coarse_pts)
COARSE_HEIGHTS = 8     # sensor heights per gravity candidate (localize.py:361)


def coarse_workload():
    """The office prior map, one 360-degree scan from a free pose and its 1024-point subset (one point per 15 cm
    voxel first, as localize.py:635-638 spreads it), and 8 sensor heights around the true one."""
    from livox_warp import synth

    scene = synth.office(LOC_SEED)
    xyz, nrm = synth.sample_surfaces(scene, COARSE_SPACING, LOC_SEED, jitter=0.002)
    T = synth.free_poses(scene, 1, LOC_POSE_SEED, z=LOC_Z, margin=0.6)[0]
    scan = synth.spin_scan(scene, T, 60000, LOC_POSE_SEED + 7)
    rng = np.random.default_rng(0)
    _, first = np.unique(np.floor(scan / 0.15).astype(np.int64), axis=0, return_index=True)
    spread = scan[np.sort(first)]
    pts = spread[rng.choice(len(spread), min(COARSE_PTS, len(spread)), replace=False)].astype(np.float32)
    heights = [round(float(T[2, 3]) + 0.08 * k, 3) for k in range(-3, COARSE_HEIGHTS - 3)]
    return {"xyz": xyz, "nrm": nrm, "T": T, "pts": pts, "heights": heights}


def run_coarse(a, rank: int, world: int, local: int):
    from oracle import oracle as _o

    w = coarse_workload()
    metric = "coarse global-search hypotheses/s (distance-field soft count of 1024 scan points per hypothesis)"
    n_yaw, dyaw, tau, free_cm, step = 180, math.radians(2.0), 25.0, 10.0, 0.25
    config = {"workload": f"coarse global search: office 40x30x3 m prior map ({len(w['xyz']):,} pts at "
                          f"{COARSE_SPACING * 1e3:.0f} mm, 5 cm grid), every free position on a {step} m xy grid x "
                          f"{COARSE_HEIGHTS} heights x {n_yaw} headings, {len(w['pts'])} scan points each, "
                          f"tau {tau:.0f} cm, free {free_cm:.0f} cm (localize.py:426-448)",
              "scan_points": int(len(w["pts"])), "headings": n_yaw, "heights": COARSE_HEIGHTS,
              "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{a.gpus}"}
    if a.impl == "reference":
        if rank != 0:
            return
        from livox_warp.localize import coarse_positions
        from livox_warp.mapgrid import PriorGrid

        threads = _o.host_cores()
        prep = PriorGrid.prepare({"xyz": w["xyz"], "normal": w["nrm"]})  # host numpy
        og = _o.PriorGrid(prep)
        pos, nx, ny = coarse_positions(prep["lo"], prep["hi"], w["heights"], step)
        sample = pos[::97]
        t0 = time.perf_counter()
        og.score_grid(w["pts"], sample, n_yaw, 0.0, dyaw, tau, free_cm, ref=True, nthreads=threads)
        secs = time.perf_counter() - t0
        v = len(sample) * n_yaw / secs
        print(json.dumps({"impl": "reference", "metric": metric, "value": round(v, 3), "unit": "hypotheses/s",
                          "n_gpus": a.gpus, "steps": 1, "warmup": 0, "ms_per_step": round(1e3 * secs, 3),
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": round(v, 3), "unit": "hypotheses/s", "cores": threads,
                                           "kind": "port", "sample": f"every 97th position ({len(sample)}) x "
                                                                     f"{n_yaw} headings through the CPU restatement"},
                          "e2e": {"value": round(v, 3), "unit": "hypotheses/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    import torch

    from livox_warp import _lib
    from livox_warp.localize import GlobalLocalizer, coarse_positions, score_grid
    from livox_warp.mapgrid import PriorGrid

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    grid = PriorGrid({"xyz": w["xyz"], "normal": w["nrm"]}, device)
    grid.build()
    loc = GlobalLocalizer(grid, device, hyp_cap=16, pts_cap=1 << 12)
    pos, nx, ny = coarse_positions(grid.lo, grid.hi, w["heights"], step)
    n_hyp = len(pos) * n_yaw
    stream = torch.cuda.current_stream(device)
    d_pts = torch.from_numpy(w["pts"]).to(device)
    d_pos = torch.from_numpy(pos).to(device)
    out = torch.empty(n_hyp, dtype=torch.float32, device=device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)

    def dev_step():
        score_grid(grid, d_pts, d_pos, n_yaw, 0.0, dyaw, tau, free_cm, out, stream, pos_stride=ny)

    for _ in range(a.warmup):
        dev_step()
    torch.cuda.synchronize(device)
    clocks = Clocks(local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    _lib.launches(reset=True)
    clocks.start()
    torch.cuda.synchronize(device)
    for j in range(a.steps):
        flush.fill_(float(j))
        evs[j][0].record(stream)
        dev_step()
        evs[j][1].record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    launches = _lib.launches()
    step_ms = np.array([x.elapsed_time(y) for x, y in evs])
    ms_total = max_over_ranks(float(step_ms.sum()), device)
    value = replica_rate(a.steps * n_hyp, world, ms_total)
    sc = out.cpu().numpy()
    # e2e through the public calls from the host scan: _coarse_candidates (scores and local maxima on the device,
    # the candidates back) and _coarse (every score back to the host, as the reference's _coarse returns them)
    for _ in range(2):
        loc._coarse(stream, w["pts"], w["heights"])
        loc._coarse_candidates(stream, w["pts"], w["heights"])
    torch.cuda.synchronize(device)
    e_steps = max(3, min(a.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e_steps):
        _, _, _, cand, cand_sc = loc._coarse_candidates(stream, w["pts"], w["heights"])
    e_s = max_over_ranks(time.perf_counter() - t0, device)
    t0 = time.perf_counter()
    for _ in range(e_steps):
        pos_e, shape, _, sc_e = loc._coarse(stream, w["pts"], w["heights"])
    e_all_s = max_over_ranks(time.perf_counter() - t0, device)
    if rank != 0:
        return
    assert np.array_equal(sc_e, sc), "the public call and the timed launches disagree"
    assert np.array_equal(cand_sc, sc[cand]) and int(cand[0]) == int(np.argmax(sc)), "candidates disagree"
    # parity on a sample of positions, and the CPU baseline on it (the oracle's grid over the same prepared
    # arrays; the distance field is the device's, which the parity tests hold bit-exact to the oracle's flood)
    threads = _o.host_cores()
    og = _o.PriorGrid(grid._host, build=False)
    og.df[:] = grid.df.cpu().numpy()
    sample = np.arange(0, len(pos), 97)
    t0 = time.perf_counter()
    want = og.score_grid(w["pts"], pos[sample], n_yaw, 0.0, dyaw, tau, free_cm, nthreads=threads)
    secs = time.perf_counter() - t0
    got = sc.reshape(len(pos), n_yaw)[sample].reshape(-1)
    best = int(np.argmax(sc))
    bp, by = pos[best // n_yaw], (best % n_yaw) * dyaw
    T = w["T"]
    yaw = math.atan2(T[1, 0], T[0, 0]) % (2 * math.pi)
    avg_ms = ms_total / a.steps
    # the unique bytes a launch must move: the distance field, the scan, the positions and every score
    ubytes = int(grid.ncell + 12 * len(w["pts"]) + 12 * len(pos) + 4 * n_hyp)
    peak = measured_peak()
    ach = ubytes / (avg_ms * 1e-3) / 1e9
    roof = {"kernel": "k_score_grid", "bound": "hbm", "achieved": round(ach, 3), "peak": peak["hbm_gbs"],
            "unit": "GB/s", "frac": round(ach / peak["hbm_gbs"], 5), "traffic": COARSE_TRAFFIC,
            "traffic_source": COARSE_TRAFFIC_SRC, "peak_source": peak["source"],
            "avg_launch_us": round(avg_ms * 1e3, 2), "algorithmic_bytes_per_launch": ubytes,
            "byte_gathers_per_launch": int(n_hyp * len(w["pts"])),
            "gathers_per_s": round(n_hyp * len(w["pts"]) / (avg_ms * 1e-3), 1),
            "limiter": "one 1-byte distance-field gather per (hypothesis, point), served from L1 / L2 (the 5 cm "
                       "field fits in L2); HBM moves only the unique bytes"}
    line = {"metric": metric, "value": round(value, 3), "unit": "hypotheses/s", "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(avg_ms, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 poses, int32 sums", "data": "synthetic",
            "config": config, "hypotheses_per_step": int(n_hyp),
            "best_vs_true": {"xy_m": round(float(np.linalg.norm(bp[:2] - T[:2, 3])), 4),
                             "z_m": round(float(abs(bp[2] - T[2, 3])), 4),
                             "yaw_deg": round(math.degrees(abs((by - yaw + math.pi) % (2 * math.pi) - math.pi)), 3)},
            "bit_exact_vs_oracle_sample": bool(np.array_equal(got, want)),
            "step_ms_p50_p99": [round(float(np.percentile(step_ms, 50)), 4),
                                round(float(np.percentile(step_ms, 99)), 4)],
            "roofline": roof,
            "cpu_baseline": {"value": round(len(sample) * n_yaw / secs, 3), "unit": "hypotheses/s",
                             "cores": threads, "kind": "port",
                             "sample": f"every 97th position ({len(sample)}) x {n_yaw} headings through the CPU "
                                       f"oracle (C++/OpenMP), {secs:.1f} s"},
            "e2e": {"value": round(world * e_steps * n_hyp / e_s, 3), "unit": "hypotheses/s",
                    "h2d_bytes_per_step": int(12 * len(w["pts"]) + 12 * len(pos)),
                    "d2h_bytes_per_step": int(4 + 12 * loc.last_candidates),
                    "path": "GlobalLocalizer._coarse_candidates: scores and local maxima on the device"},
            "e2e_all_scores": {"value": round(world * e_steps * n_hyp / e_all_s, 3), "unit": "hypotheses/s",
                               "d2h_bytes_per_step": int(4 * n_hyp),
                               "path": "GlobalLocalizer._coarse: every score back to the host"},
            "gpu_launches": int(launches), "clocks": clk}
    print(json.dumps(line))


PRIOR_SPACING, PRIOR_VOXEL, PRIOR_RADIUS, PRIOR_SLOTS = 0.01, 0.02, 0.08, 27


def prior_workload():
    """The office's surfaces every 10 mm with 2 mm jitter: a building-scale terrestrial scan's density."""
    from livox_warp import synth

    xyz, _ = synth.sample_surfaces(synth.office(LOC_SEED), PRIOR_SPACING, LOC_SEED, jitter=0.002)
    return np.ascontiguousarray(xyz, dtype=np.float32)


def run_prior(a, rank: int, world: int, local: int):
    from oracle import oracle as _o

    xyz = prior_workload()
    n = len(xyz)
    metric = "prior-map build input points/s (voxel means + PCA normals and planarity)"
    config = {"workload": f"prior map from a cloud: office 40x30x3 m surfaces every {PRIOR_SPACING * 1e3:.0f} mm "
                          f"({n:,} pts), voxel {PRIOR_VOXEL * 1e3:.0f} mm (2^{PRIOR_SLOTS} slots, chunks of 2^25), "
                          f"normal radius {PRIOR_RADIUS * 1e3:.0f} mm (prior_map.py:57-219)",
              "points": int(n), "l2": "inputs larger than L2, and flushed between steps (256 MB write)",
              "parallelism": f"replicas x{a.gpus}"}
    threads = _o.host_cores()

    def cpu_run():
        t0 = time.perf_counter()
        vx, _, _, vn = _o.voxel_downsample(xyz, None, None, PRIOR_VOXEL)
        t1 = time.perf_counter()
        nrm, pl = _o.normals(vx, PRIOR_RADIUS)
        return vx, vn, nrm, pl, t1 - t0, time.perf_counter() - t1

    if a.impl == "reference":
        if rank != 0:
            return
        _, _, _, _, sv, sn = cpu_run()
        secs = sv + sn
        v = n / secs
        print(json.dumps({"impl": "reference", "metric": metric, "value": round(v, 1), "unit": "points/s",
                          "n_gpus": a.gpus, "steps": 1, "warmup": 0, "ms_per_step": round(1e3 * secs, 3),
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                          "data": "synthetic", "config": config,
                          "cpu_baseline": {"value": round(v, 1), "unit": "points/s", "cores": threads,
                                           "kind": "port", "sample": f"the whole cloud once through the CPU "
                                                                     f"restatement (voxels 1 thread {sv:.1f} s, "
                                                                     f"normals {threads} threads {sn:.1f} s)"},
                          "e2e": {"value": round(v, 1), "unit": "points/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return
    import torch

    from livox_warp import _lib, prior_map

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    stream = torch.cuda.current_stream(device)
    x_dev = torch.from_numpy(xyz).to(device)
    table = prior_map.VoxelTable(PRIOR_VOXEL, PRIOR_SLOTS, 1 << 25, device)
    table.insert(x_dev)
    m, dropped = table.totals()
    assert dropped == 0
    bufs = prior_map.NormalBuffers(m, device)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=device)
    out = {}

    def dev_step():
        table.clear(stream)
        table.insert(x_dev, stream=stream)
        vx, _, _, vn = table.emit(stream, m=m)
        nrm, pl = prior_map.normals_device(vx, PRIOR_RADIUS, stream, bufs)
        out.update(vx=vx, vn=vn, nrm=nrm, pl=pl)

    for _ in range(a.warmup):
        dev_step()
    torch.cuda.synchronize(device)
    clocks = Clocks(local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    _lib.launches(reset=True)
    _lib.prof_reset()
    _lib.prof_enable(True)
    clocks.start()
    torch.cuda.synchronize(device)
    for j in range(a.steps):
        flush.fill_(float(j))
        evs[j][0].record(stream)
        dev_step()
        evs[j][1].record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    launches = _lib.launches()
    kern = {k: _lib.prof_read(k) for k in ("lw_vox_insert", "lw_vox_emit", "lw_normals")}
    _lib.prof_enable(False)
    assert table.totals() == (m, 0)
    step_ms = np.array([x.elapsed_time(y) for x, y in evs])
    ms_total = max_over_ranks(float(step_ms.sum()), device)
    value = replica_rate(a.steps * n, world, ms_total)
    # e2e: the public call from host arrays to host arrays (upload, build, both kernels, read back)
    for _ in range(2):
        prior_map.from_points(xyz, PRIOR_VOXEL, PRIOR_RADIUS, device, slots_log2=PRIOR_SLOTS)
    torch.cuda.synchronize(device)
    e_steps = max(3, min(a.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e_steps):
        pm = prior_map.from_points(xyz, PRIOR_VOXEL, PRIOR_RADIUS, device, slots_log2=PRIOR_SLOTS)
    e_s = max_over_ranks(time.perf_counter() - t0, device)
    if rank != 0:
        return
    vx, vn = out["vx"].cpu().numpy(), out["vn"].cpu().numpy()
    nrm, pl = out["nrm"].cpu().numpy(), out["pl"].cpu().numpy()
    ox, on, onrm, opl, sv, sn = cpu_run()
    exact = bool(np.array_equal(vx, ox) and np.array_equal(vn, on) and np.array_equal(nrm, onrm)
                 and np.array_equal(pl, opl) and np.array_equal(pm["xyz"], ox) and np.array_equal(pm["normal"], onrm))
    avg_ms = ms_total / a.steps
    ins_ms, nrm_ms = kern["lw_vox_insert"][0] / a.steps, kern["lw_normals"][0] / a.steps
    # the insert's algorithmic bytes: each point read once (12 B) and its slot written and read back twice (4 B
    # x 3), each voxel's table line (keys 8, sums 64, first 8) written once and read by the emit, the order entry
    peak = measured_peak()
    ins_bytes = int(n * (12 + 12) + m * (80 + 80 + 4))
    ach = ins_bytes / (ins_ms * 1e-3) / 1e9
    roof = {"kernel": "lw_vox_insert (k_vox_insert + first-point compaction)", "bound": "hbm",
            "achieved": round(ach, 3), "peak": peak["hbm_gbs"], "unit": "GB/s", "frac": round(ach / peak["hbm_gbs"], 5),
            "traffic": None, "peak_source": peak["source"], "algorithmic_bytes_per_launch": ins_bytes,
            "avg_ms": round(ins_ms, 4),
            "limiter": "five int64 atomics per point on its voxel's line (about four points share a 20 mm voxel)"}
    line = {"metric": metric, "value": round(value, 1), "unit": "points/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(avg_ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 in, int64 fixed-point sums, f64 PCA", "data": "synthetic",
            "config": config, "voxels": int(m),
            "kernel_ms": {"lw_vox_insert": round(ins_ms, 4), "lw_vox_emit": round(kern["lw_vox_emit"][0] / a.steps, 4),
                          "lw_normals": round(nrm_ms, 4)},
            "normals_points_per_s": round(m / (nrm_ms * 1e-3), 1),
            "bit_exact_vs_oracle": exact, "roofline": roof,
            "cpu_baseline": {"value": round(n / (sv + sn), 1), "unit": "points/s", "cores": threads, "kind": "port",
                             "sample": f"the whole cloud once through the CPU oracle (voxels 1 thread {sv:.1f} s, "
                                       f"normals {threads} threads {sn:.1f} s)"},
            "e2e": {"value": round(world * e_steps * n / e_s, 1), "unit": "points/s",
                    "h2d_bytes_per_step": int(12 * n), "d2h_bytes_per_step": int(m * (12 + 12 + 4 + 4)),
                    "path": "prior_map.from_points(host xyz) -> host xyz, normal, planarity, count"},
            "gpu_launches": int(launches), "clocks": clk}
    print(json.dumps(line))


# ---- main -------------------------------------------------------------------------------------------------------


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=580)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--cpu-budget", type=float, default=20.0, help="seconds of CPU work for the CPU baseline")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", choices=("single", "sequence", "localize", "frame", "learned", "coarse", "prior"),
                    default="single")
    ap.add_argument("--learn-epochs", type=int, default=40, help="learned: training epochs")
    ap.add_argument("--loc-hyp", type=int, default=256, help="localize: hypotheses (a smaller profiling case)")
    ap.add_argument("--loc-spacing", type=float, default=0.015, help="localize: prior-map sample spacing (m)")
    a = ap.parse_args()
    if a.warmup < 3:
        ap.error("--warmup must be >= 3")

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.workload == "single":
        run_single(a, rank, world, local)
        return
    if a.workload == "localize":
        run_localize(a, rank, world, local)
        return
    if a.workload == "frame":
        run_frame(a, rank, world, local)
        return
    if a.workload == "learned":
        run_learned(a, rank, world, local)
        return
    if a.workload == "coarse":
        run_coarse(a, rank, world, local)
        return
    if a.workload == "prior":
        run_prior(a, rank, world, local)
        return
    # the at-rest second and the first second of motion (the ramp to cruise speed) are never timed
    skip = max(a.warmup, SEQ_SKIP)
    n_frames = skip + a.steps + 1
    n_gen = min(max(n_frames + SEQ_SOAK_FRAMES, n_frames), SEQ_MAX_FRAMES)  # frames after the timed ones: the clock soak
    metric = "ICP sequence odometry frames/s (deskew + GN ICP + keyframe insert + map insert + carve)"
    config = {"workload": "sequence odometry: box room 8x6x3 m, 20 boxes, rosette 100k pts/s (~10k pts/frame), "
                          "handheld spline <=1 m/s <=60 deg/s, reg voxel 0.15 m (2^21 slots), "
                          "integration voxel 0.1 m (2^22 slots), carve every ray",
              "frames": n_frames, "timed_frames": [skip, skip + a.steps - 1], "points_per_frame": None,
              "l2": "flushed between steps (256 MB write)",
              "parallelism": f"replicas x{a.gpus}"}

    if a.impl == "reference":
        if rank != 0:
            return
        frames, traj = workload(n_frames)
        config["points_per_frame"] = int(np.mean([len(f[2]) for f in frames]))
        from oracle import oracle as _o

        threads = _o.host_cores()
        budget = max(30.0, min(150.0, 0.25 * a.steps))
        timed, secs, _ = cpu_pipeline(frames, traj, skip, budget, a.steps, threads)
        v = timed / secs
        line = {"impl": "reference", "metric": metric, "value": round(v, 3), "unit": "frames/s", "n_gpus": a.gpus,
                "steps": timed, "warmup": a.warmup, "ms_per_step": round(1e3 * secs / max(timed, 1), 3),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64",
                "data": "synthetic", "config": config,
                "cpu_baseline": {"value": round(v, 3), "unit": "frames/s", "cores": threads, "kind": "port",
                                 "sample": f"frames {skip}..{skip + timed - 1} of the sequence after "
                                           f"{skip} untimed frames; NVIDIA Warp (the reference runtime) is not "
                                           "installed, so this is the CPU restatement of its kernels and host "
                                           "solve"},
                "e2e": {"value": round(v, 3), "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    frames, traj = workload(n_gen)  # before any CUDA call (spawn pool)
    config["points_per_frame"] = int(np.mean([len(f[2]) for f in frames]))
    import torch
    import torch.distributed as dist

    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=device)
    clocks = Clocks(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(device)
    res = run_device(frames, traj, skip, a.steps, device, clocks)
    ms_total = max_over_ranks(float(res["step_ms"].sum()), device)
    value = replica_rate(a.steps, world, ms_total)
    e2e = None
    if not a.no_e2e:
        e = run_e2e(frames, traj, skip, a.steps, device)
        e_ms = max_over_ranks(e["ms"], device)
        e2e = {"value": round(replica_rate(a.steps, world, e_ms), 3), "unit": "frames/s",
               "h2d_bytes_per_step": e["h2d"], "d2h_bytes_per_step": e["d2h"]}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    roof = roofline(res, frames, traj, skip, a.steps, measured_peak())
    from oracle import oracle as _o

    threads = _o.host_cores()
    n_cpu = max(3, min(60, a.steps))
    timed, secs, opose = cpu_pipeline(frames, traj, skip, a.cpu_budget, n_cpu, threads)
    pts = config["points_per_frame"]
    drift = pose_drift(res["odom"], traj, opose)
    line = {"metric": metric, "value": round(value, 3), "unit": "frames/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms_total / a.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 solve)", "data": "synthetic",
            "config": config, "points_per_s": round(value * pts, 1),
            "step_ms_p50_p99": [round(float(np.percentile(res["step_ms"], 50)), 4),
                                round(float(np.percentile(res["step_ms"], 99)), 4)],
            "roofline": roof,
            "cpu_baseline": {"value": round(timed / secs, 3), "unit": "frames/s", "cores": threads, "kind": "port",
                             "sample": f"{timed} frames ({skip}..{skip + timed - 1}) of the same sequence "
                                       f"through the CPU oracle (C++/OpenMP kernels + numpy float64 solve), "
                                       f"{secs:.1f} s"},
            "e2e": e2e, "gpu_launches": int(res["launches"]), "clocks": res["clocks"], "pose_drift": drift}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
