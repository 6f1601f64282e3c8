"""Failure detection on the GPU without a fault: the persistent Gauss-Newton kernel's grid barrier is a bounded
wait. A test makes one CTA leave before the first barrier (the scratch's skip_cta, a flag nothing else sets) with a
short wait limit: the other CTAs give up, the launch ends, the host reads the error, and the next registration on
the same context runs normally. No trap, no fault, no unbounded wait."""

import time

import numpy as np
import pytest
import torch

import common
from oracle import oracle

pytestmark = pytest.mark.gpu


def _case():
    from livox_warp import gpu, synth
    from livox_warp.odom import Odometry

    voxel = 0.2
    T0, base, moving = synth.single_frame_case(common.room(1), 1)
    pipe = gpu.Pipeline(ring_capacity=1 << 14, map_capacity=1 << 14)
    odom = Odometry(pipe, reg_slots=1 << 18, frame_cap=1 << 15)
    odom.reg_voxel, odom.max_iter = voxel, 10
    odom.reset(T0)
    oreg = oracle.RegMap(1 << 18)
    for x, a, t in base:
        x4 = common.raw4(x, t)
        odom.insert_frame(torch.from_numpy(x4).cuda(), torch.from_numpy(a.view(np.int32)).cuda(), T0)
        oreg.insert(x4, a, T0, voxel, 60.0, 0b1111)
    oreg.records(voxel, 0.02, 0.05)
    return odom, oreg, T0, moving[0], voxel


def test_barrier_wait_runs_out_and_the_context_stays_usable():
    odom, oreg, T0, (x, a, t, t_mid, _), voxel = _case()
    zero = np.zeros(6, np.float32)
    gn = odom._gn
    gn.struct.spin_budget = 2000   # ~0.5 ms of polls instead of seconds
    gn.struct.skip_cta = gn.grid - 1
    t0 = time.perf_counter()
    _, ok, st = odom.register_frame(x, a, t, t_mid, zero, T0)
    waited = time.perf_counter() - t0
    assert st["err"] == 1 and not ok
    assert waited < 2.0  # the short limit, not the default one
    # the failed launch left the barrier words zero on its way out (and the thinning table empty); clear the sticky
    # flag as reset() does and register normally
    gn.struct.spin_budget, gn.struct.skip_cta = 0, -1
    gn.err.zero_()
    Tg, ok, st = odom.register_frame(x, a, t, t_mid, zero, T0)
    assert ok and st["err"] == 0
    ds = oracle.thin(oracle.deskew(common.raw4(x, t), t_mid, 10.0, zero), a, np.float32(2.0 / voxel), 0.3, 60.0,
                     0b1111)
    To, ok_o, _ = oracle.register(ds, T0, oreg, oracle.Params(reg_voxel=voxel, max_iter=10))
    dt, dr = oracle.pose_error(To, Tg)
    assert ok_o and dt <= 1e-3 and dr <= 0.01


def test_every_cta_but_one_gives_up_in_turn():
    """Whichever CTA is missing, the launch ends with the error set (CTA 0 included, which sets up the start state
    and clears the accumulators before the first barrier)."""
    odom, _, T0, (x, a, t, t_mid, _), _ = _case()
    zero = np.zeros(6, np.float32)
    gn = odom._gn
    gn.struct.spin_budget = 2000
    for skip in (0, gn.grid // 2):
        gn.err.zero_()
        gn.struct.skip_cta = skip
        _, ok, st = odom.register_frame(x, a, t, t_mid, zero, T0)
        assert st["err"] == 1 and not ok
    gn.struct.skip_cta, gn.struct.spin_budget = -1, 0
    gn.err.zero_()
    _, ok, st = odom.register_frame(x, a, t, t_mid, zero, T0)
    assert ok and st["err"] == 0


def test_launches_that_give_up_leave_the_thinning_table_empty():
    """A launch that gives up at its first barrier has claimed the frame's thinning slots already: each CTA empties
    the slots its points claimed on the way out. After three such launches the same frame registers as the oracle
    does, with the oracle's thinned point count, so no slot was left behind."""
    odom, oreg, T0, (x, a, t, t_mid, _), voxel = _case()
    zero = np.zeros(6, np.float32)
    gn = odom._gn
    gn.struct.spin_budget = 2000
    for skip in (1, gn.grid // 3, gn.grid - 2):
        gn.err.zero_()
        gn.struct.skip_cta = skip
        _, ok, st = odom.register_frame(x, a, t, t_mid, zero, T0)
        assert st["err"] == 1 and not ok
    gn.struct.skip_cta, gn.struct.spin_budget = -1, 0
    gn.err.zero_()
    Tg, ok, st = odom.register_frame(x, a, t, t_mid, zero, T0)
    assert ok and st["err"] == 0
    ds = oracle.thin(oracle.deskew(common.raw4(x, t), t_mid, 10.0, zero), a, np.float32(2.0 / voxel), 0.3, 60.0,
                     0b1111)
    assert st["ds"] == len(ds)
    To, ok_o, _ = oracle.register(ds, T0, oreg, oracle.Params(reg_voxel=voxel, max_iter=10))
    dt, dr = oracle.pose_error(To, Tg)
    assert ok_o and dt <= 1e-3 and dr <= 0.01
