"""The C ABI library (no GPU needed): it loads, and exports exactly the entry points include/livox_b200.h
declares, with the Python binding covering every one of them."""

import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "livox_b200.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(lw_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "lw_odom_finalize" in names and "lw_map_insert" in names and "lw_carve" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from livox_warp import _lib

    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_every_declared_symbol():
    from livox_warp import _lib

    assert sorted(_lib.exported_names()) == declared_functions()


def test_struct_layouts_match_header(tmp_path):
    """Every ctypes mirror has the size and field offsets the C compiler gives the header's struct."""
    import shutil
    import subprocess

    from livox_warp import _lib

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    mirrors = {"lw_regmap": _lib.RegMap, "lw_rec_params": _lib.RecParams, "lw_odom_params": _lib.OdomParams,
               "lw_odom_state": _lib.OdomState, "lw_traj_rec": _lib.TrajRec, "lw_frame_buf": _lib.FrameBuf,
               "lw_gn_scratch": _lib.GnScratch, "lw_pose_table": _lib.PoseTable, "lw_map": _lib.Map,
               "lw_view": _lib.View, "lw_cluster_buf": _lib.ClusterBuf, "lw_nbr_buf": _lib.NbrBuf, "lw_prior_grid": _lib.PriorGrid,
               "lw_vox_buf": _lib.VoxBuf, "lw_pca_buf": _lib.PcaBuf,
               "lw_loc_batch": _lib.LocBatch, "lw_initnet": _lib.InitNet, "lw_net_scratch": _lib.NetScratch,
               "lw_net_work": _lib.NetWork}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in mirrors.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname} {fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            a, b, v = line.split()
            got[(a, b)] = int(v)
    for cname, py in mirrors.items():
        assert got[(cname, "size")] == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert got[(cname, fname)] == getattr(py, fname).offset, (cname, fname)


def test_version_and_error_without_gpu():
    from livox_warp import _lib

    lib = _lib.load(require_cuda=False)
    assert b"sm_100a" in lib.lw_version()
    # a bad argument is rejected on the host before any CUDA call
    assert lib.lw_map_clear(None, None) == _lib.LW_EINVAL
    assert b"lw_map_clear" in lib.lw_last_error()


def test_no_cpu_fallback():
    """Without CUDA the package refuses to run instead of falling back to the CPU."""
    import torch
    from livox_warp import _lib

    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    saved = _lib._lib
    _lib._lib = None
    try:
        with pytest.raises(RuntimeError, match="no CPU fallback"):
            _lib.load(require_cuda=True)
    finally:
        _lib._lib = saved


def test_noalloc_thinning_refuses_misaligned_points_without_a_gpu():
    """lw_thin_noalloc reads and writes float4 points: a pointer off a 16-byte boundary is refused with LW_EINVAL
    before any device work (so this runs without a GPU; the pointers are never dereferenced)."""
    from livox_warp import _lib

    lib = _lib.load(require_cuda=False)
    good, bad = 0x10000, 0x10004
    for xyz, out in ((bad, good), (good, bad)):
        rc = lib.lw_thin_noalloc(ctypes.c_void_p(xyz), ctypes.c_void_p(good), 100, 10.0, 0.3, 60.0, 15,
                                 ctypes.c_void_p(out), ctypes.c_void_p(good), None)
        assert rc == _lib.LW_EINVAL
        assert b"16-byte" in lib.lw_last_error()


def test_register_frame_host_refuses_bad_arguments_without_a_gpu():
    """lw_register_frame_host checks its arguments before it asks CUDA for anything: a null buffer is LW_EINVAL and
    a frame above the frame buffer's capacity LW_ECAPACITY (so this runs without a GPU; no pointer is used)."""
    from livox_warp import _lib

    lib = _lib.load(require_cuda=False)
    dummy = ctypes.c_void_p(0x10000)
    tw = _lib.f32_array(np.zeros(6, np.float32))
    T = _lib.f64_array(np.eye(4).reshape(16))
    prm = _lib.OdomParams()
    fb = _lib.FrameBuf()
    fb.cap = 16
    reg = _lib.RegMap()
    gn = _lib.GnScratch()

    def call(xyz3, m):
        return lib.lw_register_frame_host(xyz3, dummy, dummy, m, 0.0, tw, T, ctypes.byref(prm), dummy,
                                          ctypes.byref(fb), ctypes.byref(reg), ctypes.byref(gn), dummy, dummy, None)

    assert call(None, 8) == _lib.LW_EINVAL
    assert b"null" in lib.lw_last_error()
    assert call(dummy, 32) == _lib.LW_ECAPACITY
    assert b"capacity" in lib.lw_last_error()
    assert call(dummy, -1) == _lib.LW_ECAPACITY
