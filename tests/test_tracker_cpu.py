"""The host tracker (perception.py:274-388) against the reference's own Tracker class, run from its source on a
seeded scene by tests/golden/make_golden.py (tests/golden/tracker.npz): static, walking, crossing and reappearing
objects, 10 Hz and 144 Hz updates mixed, dropouts, shuffled cluster order and a clock restart. Track ids and the
confirmed set must be identical after every update, velocities equal to float64 rounding."""

from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "tracker.npz"


def test_tracker_matches_reference_class():
    from livox_warp.perception import Tracker

    z = np.load(GOLDEN)
    tr = Tracker()
    a = c = 0
    moving = 0
    for k, now in enumerate(z["now"]):
        n = int(z["n"][k])
        cl = [{"cen": z["cen"][a + i].copy(), "lo": z["lo"][a + i].copy(), "hi": z["hi"][a + i].copy(),
               "cnt": int(z["cnt"][a + i])} for i in range(n)]
        ids, vel = tr.update(cl, float(now))
        assert ids.tolist() == z["tid"][a:a + n].tolist(), f"update {k}: track ids differ"
        assert np.allclose(vel, z["vel"][a:a + n], rtol=0, atol=1e-12), f"update {k}: velocities differ"
        moving += int((np.linalg.norm(vel, axis=1) > 0.5).sum())
        m = int(z["n_confirmed"][k])
        assert sorted(t for t, _ in tr.confirmed()) == z["confirmed"][c:c + m].tolist(), f"update {k}: confirmed"
        a += n
        c += m
    assert a == len(z["tid"]) and c == len(z["confirmed"])
    assert moving > 50  # the walkers are tracked with their speed, not only the static objects
