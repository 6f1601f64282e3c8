"""The CPU oracle's float64 host math against golden vectors produced by the reference's own functions
(odom.py :390-455, localize.py :222-240, gpu.py :1113-1123, executed from the reference source by
tests/golden/make_golden.py). Tolerance: 1e-12 absolute on poses and twists, 1e-9 relative on the steps."""

from pathlib import Path

import numpy as np
import pytest

from oracle import oracle

G = np.load(Path(__file__).resolve().parent / "golden" / "host_solve.npz")


def test_sym6():
    for u, want in zip(G["sym6_in"], G["sym6_out"]):
        assert np.array_equal(oracle.sym6(u), want)


def test_twist_between_and_apply():
    for a, b, want in zip(G["tb_from"], G["tb_to"], G["tb_out"]):
        np.testing.assert_allclose(oracle.twist_between(a, b), want, atol=1e-12)
    for T, d, want, want_loc in zip(G["apply_T"], G["apply_delta"], G["apply_out"], G["apply_loc_out"]):
        np.testing.assert_allclose(oracle.apply_twist(T, d), want, atol=1e-12)
        np.testing.assert_allclose(oracle.apply_twist(T, d), want_loc, atol=1e-12)


def test_body_twist_and_twist_matrix():
    for D, want in zip(G["body_in"], G["body_out"]):
        got = oracle.body_twist(D)
        assert got.dtype == np.float32 and np.array_equal(got, want)
    for xi, want in zip(G["twm_in"], G["twm_out"]):
        np.testing.assert_allclose(oracle.twist_matrix(xi), want, atol=1e-12)


def test_sensor_basis():
    for T, L, want in zip(G["sb_T"], G["sb_L"], G["sb_out"]):
        np.testing.assert_allclose(oracle.sensor_basis(T, L), want, atol=1e-12)


def test_constrained_step():
    for i in range(len(G["cs_out"])):
        step, (_, _, kept) = oracle.constrained_step(G["cs_A"][i], G["cs_rhs"][i], G["cs_Hg"][i], G["cs_T"][i],
                                                     G["cs_L"][i], G["cs_thr"][i], G["cs_pred"][i])
        assert np.array_equal(kept, G["cs_kept"][i])
        np.testing.assert_allclose(step, G["cs_out"][i], rtol=1e-9, atol=1e-12)
    # the fixtures exercise all three branches: all directions kept, some frozen
    kept = G["cs_kept"]
    assert kept.all(axis=1).any() and (~kept.all(axis=1)).any()


def test_pose_difference_and_mount():
    for A, B, want in zip(G["tb_from"], G["tb_to"], G["pd_out"]):
        d = oracle.pose_error(A, B)
        # pose_difference reports the translation between the two positions and the relative angle
        assert abs(np.degrees(np.linalg.norm(
            __import__("scipy.spatial.transform", fromlist=["Rotation"]).Rotation.from_matrix(
                (np.linalg.inv(A) @ B)[:3, :3]).as_rotvec())) - want[1]) < 1e-6
        assert abs(np.linalg.norm(A[:3, 3] - B[:3, 3]) - want[0]) < 1e-12
        assert d[1] == pytest.approx(want[1], abs=1e-6)
    from livox_warp import gpu

    for m, want in zip(G["mount_in"], G["mount_out"]):
        assert np.array_equal(gpu.mount_matrix(*m), want)


def test_prior_prepare_matches_reference():
    """PriorGrid.prepare (mapgrid.py:216-243) as the reference computes it, bit for bit: the product's host
    preparation and the oracle's restatement against tests/golden/prior_prepare.npz."""
    from livox_warp.mapgrid import PriorGrid

    P = np.load(Path(__file__).resolve().parent / "golden" / "prior_prepare.npz")
    host = {"xyz": P["in_xyz"], "normal": P["in_normal"], "planarity": P["in_planarity"]}
    got = PriorGrid.prepare(host)
    for k in ("xyz", "normal", "planarity", "origin", "dims", "start", "lo", "hi"):
        assert np.array_equal(np.asarray(got[k]), P[k]), k
    h, lo, b = got["levels"]
    assert np.array_equal(h, P["levels_h"]) and lo == float(P["levels_lo"]) and b == float(P["levels_bin"])
    o = oracle.prior_prepare(P["in_xyz"], P["in_normal"], P["in_planarity"])
    for k in ("xyz", "normal", "planarity", "origin", "dims", "start"):
        assert np.array_equal(np.asarray(o[k]), P[k]), k
