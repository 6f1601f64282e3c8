"""ctypes binding of liblivoxb200.so, the sm_100a C ABI declared in include/livox_b200.h.

The structs below mirror the header field for field. Every call passes raw device pointers (torch CUDA tensors'
data_ptr()) and the CUDA stream; a non-zero status raises LwError with the library's message. There is no CPU
fallback: importing this module without the built library, or calling into it without a CUDA device, raises.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

import torch

LIB_PATH = Path(__file__).resolve().parent / "liblivoxb200.so"

LW_OK, LW_EINVAL, LW_ECAPACITY, LW_ETIMEOUT, LW_ECUDA = 0, -1, -2, -3, -4
FIX_R, FIX_RR, FIX_W = 2.0 ** 32, 2.0 ** 40, 2.0 ** 20
VOX_FIX_ATTR = 2.0 ** 16
REG_CAP = MAP_CAP = 4096
ACC_STRIDE = 64
GN_TRACE = 17  # poses a Gauss-Newton trace holds (LW_GN_TRACE)
REC_FLOATS = 20
POSE_SLOTS = 1 << 16
ACC_H, ACC_B, ACC_COUNT, ACC_ERR, ACC_RMS, ACC_WEIGHT, ACC_RANGE, ACC_HG = 0, 21, 27, 28, 29, 30, 31, 32
INT32_MAX = 0x7FFFFFFF


class LwError(RuntimeError):
    """A status other than LW_OK from the CUDA library."""


P = C.c_void_p
i32, i64, f32, f64 = C.c_int32, C.c_int64, C.c_float, C.c_double


class RegMap(C.Structure):
    _fields_ = [("keys", P), ("cnt", P), ("sum", P), ("outer", P), ("rec", P), ("bcnt", P), ("first", P),
                ("stats", P), ("cap", i64)]


class RecParams(C.Structure):
    _fields_ = [("voxel", f32), ("tight2", f32), ("noise2", f32), ("alpha", f32)]


class OdomParams(C.Structure):
    _fields_ = [(n, f64) for n in ("frame_dt", "reg_voxel", "min_range", "max_range", "noise", "alpha", "damping",
                                    "velocity_smooth", "degen_thr", "prior_info", "kf_dist", "kf_angle_deg")] + \
               [(n, i32) for n in ("max_iter", "warmup", "min_points", "min_corr", "ret_mask", "deskew", "redeskew",
                                    "frame_cap")]


class OdomState(C.Structure):
    _fields_ = [("T", f64 * 16), ("T_prev", f64 * 16), ("T_key", f64 * 16), ("delta", f64 * 16), ("xi_s", f64 * 6),
                ("T_pred", f64 * 16), ("T_reg", f64 * 16), ("t_mid", f64), ("rms", f64), ("cond", f64),
                ("xi", f32 * 6), ("xi_used", f32 * 6)] + \
               [(n, i32) for n in ("has_prev", "has_key", "map_frames", "frame_k", "m", "n_ds", "warm", "ok",
                                    "run_reg", "do_insert", "redo", "err", "iters", "corr", "degen", "weak", "frames",
                                    "skipped", "keyframes", "traj_len", "iters_first", "pad_")]


class TrajRec(C.Structure):
    _fields_ = [("T", f64 * 16), ("t_mid", f64), ("k", i32), ("ok", i32), ("iters", i32), ("corr", i32),
                ("iters_first", i32), ("pad_", i32)]


class FrameBuf(C.Structure):
    _fields_ = [("f_raw", P), ("f_xyz", P), ("f_attr", P), ("f_t", P), ("f_frame", P), ("count", P), ("ds_keys", P),
                ("ds_win", P), ("ds_slot", P), ("tiles", P), ("ds_xyz", P), ("cap", i64), ("ds_cap", i64)]


class GnScratch(C.Structure):
    _fields_ = [("part", P), ("bar", P), ("err", P), ("grid", i32), ("spin_budget", i32), ("skip_cta", i32),
                ("trace", P)]


class PoseTable(C.Structure):
    _fields_ = [("poses", P), ("tw", P), ("owner_frame", P), ("owner_epoch", P)]


class Map(C.Structure):
    _fields_ = [("keys", P), ("cnt", P), ("acc", P), ("last", P), ("first", P), ("miss", P), ("bcnt", P),
                ("lead", P), ("stats", P), ("cap", i64)]


class ClusterBuf(C.Structure):
    PTRS = ("keys", "acc", "first", "vidx", "slot_of_pt", "tiles", "node_slot", "v_xyz", "v_w", "edge_off", "edges",
            "label", "st_sum", "st_lo", "st_hi", "dense", "out_cnt", "out_cen", "out_lo", "out_hi", "m", "n_clusters",
            "err")
    _fields_ = [(n, P) for n in PTRS] + [("cap", i64), ("pt_cap", i64), ("edge_cap", i64)]


class NbrBuf(C.Structure):
    PTRS = ("keys", "acc", "vidx", "v_slot", "slot_of_pt", "v_xyz", "v_w", "v_cnt", "v_nrm", "v_curv", "tiles", "m")
    _fields_ = [(n, P) for n in PTRS] + [("cap", i64), ("pt_cap", i64)]


class VoxBuf(C.Structure):
    PTRS = ("keys", "acc", "first", "order", "slot_of_pt", "tiles", "stats")
    _fields_ = [(n, P) for n in PTRS] + [("cap", i64), ("pt_cap", i64)]


class PcaBuf(C.Structure):
    PTRS = ("keys", "cell_cnt", "cell_start", "slot_of_pt", "rank_of_pt", "sorted", "tiles", "stats")
    _fields_ = [(n, P) for n in PTRS] + [("cap", i64), ("pt_cap", i64)]


class PriorGrid(C.Structure):
    """mapgrid.Grid (mapgrid.py:35-43) plus the map arrays the grid kernels read."""

    _fields_ = [("xyz", P), ("nrm", P), ("start", P), ("nn", P), ("df", P), ("seed", P), ("nn2", P),
                ("origin", f32 * 3), ("cell", f32), ("inv_cell", f32), ("nx", i32), ("ny", i32), ("nz", i32),
                ("pad_", i32), ("n", i64), ("ncell", i64)]


class LocBatch(C.Structure):
    PTRS = ("pts", "scan_end", "tile_hyp", "tile_lo", "hyp_tile", "T", "tile_part", "moved", "next", "count", "eval",
            "bar", "err", "iters_run", "dims")
    _fields_ = [(n, P) for n in PTRS] + [("pts_cap", i64), ("moved_cap", i32), ("grid_cap", i32)]


SCORE_MAX_YAW = 1024  # headings lw_score_grid takes per launch (LW_SCORE_MAX_YAW)
NET_P = 1024
NET_OFF = {"W1": 0, "B1": 192, "W2": 256, "B2": 8448, "W3": 8576, "B3": 41344, "WH1": 41600, "BH1": 107136,
           "WH2": 107264, "BH2": 108032}
NET_NPARAM = 108040


class InitNet(C.Structure):
    _fields_ = [("master", P), ("w", P), ("grad", P), ("adam_m", P), ("adam_v", P), ("out_scale", P),
                ("in_scale", f32), ("pad_", i32)]


class NetScratch(C.Structure):
    PTRS = ("dz3", "h2g", "d2t", "h1t", "d1t", "xt", "dzh", "dout", "dpool", "part", "loss")
    _fields_ = [(n, P) for n in PTRS] + [("n_cap", i32), ("pad_", i32)]


class NetWork(C.Structure):
    PTRS = ("sets", "pooled", "argmax", "hid", "step", "err", "cand", "tiles", "count")
    _fields_ = [(n, P) for n in PTRS] + [("radius", f32), ("voxel", f32)]


class View(C.Structure):
    """gpu.View (gpu.py:76-98): the filters and labels the map kernels read."""

    _fields_ = [("now", f32), ("persist", f32), ("min_range", f32), ("max_range", f32), ("min_refl", i32),
                ("noise_mask", i32), ("ret_mask", i32), ("crop_on", i32), ("crop_lo", f32 * 3), ("crop_hi", f32 * 3),
                ("inv_frame_dt", f32), ("epoch", i32), ("inv_voxel", f32), ("map_mask", i32), ("dyn_on", i32),
                ("dyn_settle", f32), ("carve_on", i32), ("carve_ratio", f32), ("carve_min", i32),
                ("carve_stale", f32)]

    def __setattr__(self, name, value):
        if name in ("crop_lo", "crop_hi"):
            value = (f32 * 3)(*[float(x) for x in value])
        super().__setattr__(name, value)


# (name, restype, argtypes) of every exported entry point
_SIGS = {
    "lw_version": (C.c_char_p, []),
    "lw_last_error": (C.c_char_p, []),
    "lw_device_sms": (i32, [C.POINTER(i32)]),
    "lw_prof_enable": (i32, [i32]),
    "lw_prof_read": (i32, [C.c_char_p, C.POINTER(f64), C.POINTER(i64)]),
    "lw_prof_reset": (i32, []),
    "lw_launches": (i64, [i32]),
    "lw_frame_append": (i32, [P, i32, P, P, i64, f64, i32, i32, C.POINTER(FrameBuf), P]),
    "lw_frame_reset": (i32, [C.POINTER(FrameBuf), P]),
    "lw_odom_finalize": (i32, [i32, i64, C.POINTER(OdomParams), P, C.POINTER(FrameBuf), C.POINTER(RegMap),
                               C.POINTER(GnScratch), C.POINTER(PoseTable), i32, P, i64, P]),
    "lw_odom_predict_poses": (i32, [i32, i32, i32, P, C.POINTER(PoseTable), i32, P]),
    "lw_odom_reset": (i32, [C.POINTER(f64), P, C.POINTER(RegMap), i32, P]),
    "lw_odom_restart_clock": (i32, [P, P]),
    "lw_deskew": (i32, [P, P, P, i64, f64, f64, C.POINTER(f32), P]),
    "lw_thin": (i32, [C.POINTER(FrameBuf), P, i64, f64, f64, f64, i32, P, P]),
    "lw_thin_noalloc": (i32, [P, P, i64, f64, f64, f64, i32, P, P, P]),
    "lw_reg_insert": (i32, [P, P, P, i64, C.POINTER(f64), f64, f64, i32, C.POINTER(RegMap), C.POINTER(RecParams),
                              P, P]),
    "lw_reg_refresh_all": (i32, [C.POINTER(RegMap), C.POINTER(RecParams), P]),
    "lw_icp_accumulate": (i32, [P, P, i64, C.POINTER(f64), C.POINTER(RegMap), f32, i32, f32, f32,
                                C.POINTER(GnScratch), P, P]),
    "lw_icp_solve": (i32, [P, P, C.POINTER(OdomParams), P, C.POINTER(RegMap), C.POINTER(GnScratch), P]),
    "lw_read_state": (i32, [P, P, P, P, P]),
    "lw_stage_batch": (i32, [P, P, P, i64, P, P, P, f32, P, P]),
    "lw_register_frame": (i32, [P, P, i64, f64, C.POINTER(f32), C.POINTER(f64), C.POINTER(OdomParams), P,
                                C.POINTER(FrameBuf), C.POINTER(RegMap), C.POINTER(GnScratch), P]),
    "lw_register_frame_host": (i32, [P, P, P, i64, f64, C.POINTER(f32), C.POINTER(f64), C.POINTER(OdomParams), P,
                                     C.POINTER(FrameBuf), C.POINTER(RegMap), C.POINTER(GnScratch), P, P, P]),
    "lw_map_insert": (i32, [P, i32, P, P, P, P, i64, P, C.POINTER(View), f32, C.POINTER(Map), P, P]),
    "lw_carve": (i32, [P, i32, P, P, P, i64, P, i32, f32, f32, i32, C.POINTER(Map), P, P]),
    "lw_map_build": (i32, [C.POINTER(Map), C.POINTER(View), i32, P, P, P, P, P, P, P]),
    "lw_map_clear": (i32, [C.POINTER(Map), P]),
    "lw_live_build": (i32, [P, P, P, P, i64, i64, C.POINTER(PoseTable), C.POINTER(View), C.POINTER(Map), P, P, P, P,
                            P, P, P]),
    "lw_frame_ids": (i32, [P, i64, f32, P, P]),
    "lw_ground": (i32, [P, i32, P, P, i64, f32, f32, i32, f32, f32, i32, f32, P, P, P, P, P]),
    "lw_cluster": (i32, [P, i32, P, i32, P, i64, f32, f32, f32, i32, C.POINTER(ClusterBuf), P, P]),
    "lw_neighborhoods": (i32, [P, i32, P, i64, f32, i32, P, C.POINTER(NbrBuf), P, P, P, P]),
    "lw_vox_offset_units": (f64, [f32]),
    "lw_vox_clear": (i32, [C.POINTER(VoxBuf), P]),
    "lw_vox_insert": (i32, [C.POINTER(VoxBuf), P, i32, P, P, i64, i64, f32, P]),
    "lw_vox_emit": (i32, [C.POINTER(VoxBuf), f32, i64, P, P, P, P, P]),
    "lw_normals": (i32, [P, i32, i64, f32, C.POINTER(PcaBuf), P, P, P]),
    "lw_lvxr_decode": (i32, [P, i64, C.POINTER(P)]),
    "lw_lvxr_info": (i32, [P, C.POINTER(i64), C.POINTER(i32), C.POINTER(i32), C.POINTER(i32), C.POINTER(f64)]),
    "lw_lvxr_copy": (i32, [P, P, P, P, P, P, P]),
    "lw_lvxr_free": (None, [P]),
    "lw_prior_grid_build": (i32, [C.POINTER(PriorGrid), P]),
    "lw_net_init": (i32, [C.POINTER(InitNet), C.c_uint64, P]),
    "lw_net_forward": (i32, [C.POINTER(InitNet), P, i32, P, P, P, P, P, P]),
    "lw_net_backward": (i32, [C.POINTER(InitNet), P, i32, P, P, P, P, P, P, C.POINTER(NetScratch), P]),
    "lw_net_adam": (i32, [C.POINTER(InitNet), i32, f32, f32, f32, f32, f32, P]),
    "lw_net_sets": (i32, [P, P, C.POINTER(RegMap), P, f32, f32, P, P, P, P, P]),
    "lw_odom_finalize_net": (i32, [i32, i64, C.POINTER(OdomParams), P, C.POINTER(FrameBuf), C.POINTER(RegMap),
                                   C.POINTER(GnScratch), C.POINTER(PoseTable), i32, P, i64, C.POINTER(InitNet),
                                   C.POINTER(NetWork), P]),
    "lw_prior_distances": (i32, [C.POINTER(PriorGrid), P, i64, C.POINTER(f64), P, P]),
    "lw_score_grid": (i32, [C.POINTER(PriorGrid), P, i32, P, i64, i64, i32, f32, f32, f32, f32, P, P]),
    "lw_score_list": (i32, [C.POINTER(PriorGrid), P, i32, P, i64, f32, P, P]),
    "lw_score_yaw_table": (None, [i32, f32, f32, P, P]),
    "lw_score_maxima": (i32, [P, i32, i32, i32, i32, f32, i32, P, P, P, P]),
    "lw_loc_icp_batch": (i32, [C.POINTER(PriorGrid), C.POINTER(LocBatch), i32, i32, i32, i32, C.POINTER(f64),
                               C.POINTER(i32), f32, i32, i32, i32, P]),
}

_lib = None


def exported_names() -> list[str]:
    return list(_SIGS)


def load(require_cuda: bool = True) -> C.CDLL:
    """Load the library (once). Raises if it is missing, or if require_cuda and no CUDA device is present."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is missing: build it with `python livox-warp_b200/csrc/build.py` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    if require_cuda and not torch.cuda.is_available():
        raise RuntimeError("livox_warp needs a CUDA device (sm_100a); there is no CPU fallback")
    return lib


def check(status: int, what: str = ""):
    if status != LW_OK:
        msg = _lib.lw_last_error().decode(errors="replace") if _lib is not None else ""
        raise LwError(f"{what or 'livox_warp'}: status {status}: {msg}")


def call(name: str, *args):
    lib = load()
    check(getattr(lib, name)(*args), name)


def ptr(t: torch.Tensor | None):
    """Device pointer of a tensor (None -> NULL)."""
    return None if t is None else C.c_void_p(t.data_ptr())


def stream_ptr(stream=None) -> C.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def f64_array(values) -> C.Array:
    a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
    return (f64 * a.size).from_buffer_copy(a)


def f32_array(values) -> C.Array:
    a = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
    return (f32 * a.size).from_buffer_copy(a)


def prof_enable(on: bool = True):
    call("lw_prof_enable", int(on))


def prof_read(name: str) -> tuple[float, int]:
    """(summed ms, launches) of the named launches since the last reset (waits for them)."""
    ms, cnt = f64(0.0), i64(0)
    call("lw_prof_read", name.encode(), C.byref(ms), C.byref(cnt))
    return ms.value, cnt.value


def prof_reset():
    call("lw_prof_reset")


def launches(reset: bool = False) -> int:
    """Kernels launched by the library since the last reset."""
    return int(load().lw_launches(int(reset)))
