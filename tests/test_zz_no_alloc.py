"""The thinning entry point for callers that cannot allocate device memory (lw_thin_noalloc).

Such callers -- a real-time sensor thread, or a host whose device memory is fixed at start-up -- must not call
cudaMalloc on the frame path, so this entry point keeps its tables in a file-scope device array and takes only
the caller's points and output buffer. Its result must equal the allocating entry point's (lw_thin) exactly,
on two calls in a row (the shared array keeps the last call's contents), and a call above its fixed maximum of
65536 points must be refused. This file is collected last, so a failure here leaves every other test run.
"""

import ctypes

import numpy as np
import pytest
import torch

import common
from oracle import oracle

pytestmark = pytest.mark.gpu


def _noalloc(x4: torch.Tensor, a: torch.Tensor, inv_v: float, ret_mask: int, m: int | None = None):
    from livox_warp import _lib

    lib = _lib.load()
    m = int(x4.shape[0]) if m is None else m
    out = torch.zeros((max(m, 1), 4), dtype=torch.float32, device=x4.device)
    n_ds = torch.full((1,), -1, dtype=torch.int32, device=x4.device)
    rc = lib.lw_thin_noalloc(_lib.ptr(x4), _lib.ptr(a), m, inv_v, 0.3, 60.0, ret_mask, _lib.ptr(out), _lib.ptr(n_ds),
                             _lib.stream_ptr())
    _lib.check(rc, "lw_thin_noalloc")
    k = int(n_ds.cpu()[0])
    return out[:k].cpu().numpy()


def test_noalloc_thinning_matches_lw_thin_twice():
    from livox_warp import kernels

    voxel = 0.15
    inv_v = float(np.float32(2.0 / voxel))
    th = kernels.Thinner(1 << 15)
    frames = common.handheld_frames(14)
    for x, a, t in (frames[12], frames[13]):  # two calls in a row on the shared array
        a = a.copy()
        a[::29] |= np.uint32(1 << 8)  # some noise-tagged returns
        x4 = torch.from_numpy(common.raw4(x, t)).cuda()
        at = torch.from_numpy(a.view(np.int32)).cuda()
        want = th(x4, at, inv_v, 0.3, 60.0, 0b1111).cpu().numpy()
        got = _noalloc(x4, at, inv_v, 0b1111)
        assert len(got) == len(want) > 100
        assert np.array_equal(got, want)
        # and the oracle's thinning of the same points
        assert np.array_equal(got, oracle.thin(common.raw4(x, t), a, np.float32(inv_v), 0.3, 60.0, 0b1111))


def test_noalloc_empty_and_full_frames():
    """No points (only the count is written), then 65536 points -- the fixed maximum, tiled from handheld frames so
    the 131072-slot table is half full -- against the oracle, twice in a row."""
    voxel = 0.15
    inv_v = float(np.float32(2.0 / voxel))
    one = torch.zeros((1, 4), dtype=torch.float32, device="cuda")
    assert len(_noalloc(one, torch.zeros(1, dtype=torch.int32, device="cuda"), inv_v, 0b1111, m=0)) == 0
    frames = common.handheld_frames(20)
    xs = np.concatenate([common.raw4(x, t) for x, a, t in frames[10:20]])[:65536]
    at = np.concatenate([a for x, a, t in frames[10:20]])[:65536]
    assert len(xs) == 65536
    x4 = torch.from_numpy(np.ascontiguousarray(xs)).cuda()
    a4 = torch.from_numpy(at.view(np.int32)).cuda()
    want = oracle.thin(xs, at, np.float32(inv_v), 0.3, 60.0, 0b1111)
    for _ in range(2):
        got = _noalloc(x4, a4, inv_v, 0b1111)
        assert len(got) == len(want) > 10000
        assert np.array_equal(got, want)


def test_noalloc_refuses_more_than_its_maximum():
    from livox_warp import _lib

    lib = _lib.load()
    x4 = torch.zeros((70000, 4), dtype=torch.float32, device="cuda")
    a = torch.zeros(70000, dtype=torch.int32, device="cuda")
    out = torch.zeros_like(x4)
    n_ds = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.lw_thin_noalloc(_lib.ptr(x4), _lib.ptr(a), 70000, 10.0, 0.3, 60.0, 15, _lib.ptr(out), _lib.ptr(n_ds),
                             _lib.stream_ptr())
    assert rc == _lib.LW_ECAPACITY
    assert b"65536" in lib.lw_last_error()
