"""The reference's behavioural gates for the perception path, restated on this repository's synthetic scenes and
evaluated on the CPU oracle (the GPU is held bit-exact to it by the -m gpu tests): ground labels and heights
(check_perception.py:182-183), connected components on long structures (:276-284) and the tracker's static noise
and speed (:262-263)."""

import math

import numpy as np
import pytest

from oracle import oracle


def _crate_scan():
    """A static downward-looking scan of a 10 x 8 x 3 m room with a 1.2 x 0.8 x 0.5 m crate on the floor."""
    from livox_warp import synth

    crate = np.array([[4.0, 3.0, 0.0, 5.2, 3.8, 0.5]])
    sc = synth.Scene(np.zeros(3), np.array([10.0, 8.0, 3.0]), crate)
    T = np.eye(4)
    T[:3, 3] = [2.5, 3.4, 1.6]
    pts = synth.spin_scan(sc, T, 120000, 3, noise=0.01, elev_deg=(-70.0, 10.0))
    return (pts.astype(np.float64) + T[:3, 3]).astype(np.float32), crate[0]


def test_ground_gates():
    """Floor recall > 95 %, the crate top < 5 % and walls / objects < 2 % labelled ground; the crate top reads its
    height above the floor within 0.1 m and the floor within 5 cm (check_perception.py:182-183)."""
    xyz, c = _crate_scan()
    gnd, hag = oracle.ground(xyz, cell=0.5, thick=0.15, min_sup=3, thresh=0.2, slope_step=0.3)
    floor = xyz[:, 2] < 0.1
    inset = 0.1
    top = (np.all(xyz[:, :2] > c[:2] + inset, axis=1) & np.all(xyz[:, :2] < c[3:5] - inset, axis=1)
           & (xyz[:, 2] > c[5] - inset))
    walls = (xyz[:, 2] > 0.4) & ~top
    assert floor.sum() > 10000 and top.sum() > 200 and walls.sum() > 10000
    assert gnd[floor].mean() > 0.95
    assert gnd[top].mean() < 0.05
    assert gnd[walls].mean() < 0.02
    assert abs(float(np.median(hag[top])) - c[5]) < 0.1
    assert float(np.median(np.abs(hag[floor]))) < 0.05


@pytest.mark.parametrize("label,pts,vox,conn", [
    ("60 x 3 m wall", np.stack(np.meshgrid(np.arange(-30, 30, 0.05), np.arange(-1.5, 1.5, 0.05)), -1).reshape(-1, 2),
     0.1, 0.35),
    ("60 m rail", np.stack([np.arange(-30, 30, 0.02), np.zeros(3000)], -1), 0.05, 0.1),
])
def test_components_on_long_structures(label, pts, vox, conn):
    """One component along 60 m: the union-find needs no iteration cap to connect it (check_perception.py:276-284)."""
    p3 = np.zeros((len(pts), 3), np.float32)
    p3[:, 0], p3[:, 1], p3[:, 2] = 20.0, pts[:, 0], pts[:, 1]
    cid, _, clusters, _ = oracle.cluster(p3, None, voxel=vox, connect=conn, min_pts=10)
    assert len(clusters) == 1, label
    assert (cid >= 0).all()


def test_tracker_static_noise_and_speed():
    """Static clusters whose centroids wander by a few cm read as still (90th percentile speed < 0.1 m/s, < 3 %
    above 0.15 m/s); a cluster walking at 1.2 m/s reads its speed within 25 % (check_perception.py:262-263)."""
    from livox_warp.perception import Tracker

    rng = np.random.default_rng(7)
    tr = Tracker()
    static = [np.array([2.0, 1.0, 0.5]), np.array([6.0, -2.0, 0.4]), np.array([-3.0, 4.0, 0.6])]
    walker0, v = np.array([0.0, -5.0, 0.9]), np.array([0.0, 1.2, 0.0])
    st_speed, w_speed = [], []
    for i in range(60):  # 10 Hz for 6 s
        now = 0.1 * i
        cl = []
        for c in static + [walker0 + v * now]:
            cen = c + rng.normal(0, 0.02, 3)
            cl.append({"cen": cen, "lo": cen - 0.3, "hi": cen + 0.3, "cnt": 200})
        tid, vel = tr.update(cl, now)
        if i >= 10:
            st_speed += [float(np.linalg.norm(vel[k])) for k in range(3)]
            w_speed.append(float(np.linalg.norm(vel[3])))
    st = np.array(st_speed)
    assert np.percentile(st, 90) < 0.1 and (st > 0.15).mean() < 0.03
    assert abs(np.median(w_speed) - 1.2) < 0.25 * 1.2
    assert len({int(t) for t in tid}) == 4  # four tracks, one per cluster
