"""The coarse search's local-maximum rule, which the GPU test holds lw_score_maxima to (every score at least the
pool-th best that is positive and no lower than its 26 (x, y, heading) neighbours), against the reference's own
GlobalLocalizer._local_maxima and _top (localize.py:450-483), run from source on seeded score arrays with ties
by tests/golden/make_golden.py (tests/golden/local_maxima.npz). The reference takes exactly `pool` candidates
(an unstable partition), so where the pool-th score is tied it may keep fewer of the tied ones; every other
candidate is the same, and so is the order of the scores."""

from pathlib import Path

import numpy as np

import common

GOLDEN = Path(__file__).resolve().parent / "golden" / "local_maxima.npz"


def test_rule_matches_reference_local_maxima():
    z = np.load(GOLDEN)
    k = 0
    while f"sc{k}" in z.files:
        sc, shape = z[f"sc{k}"], tuple(int(x) for x in z[f"shape{k}"])
        pool, keep, want = int(z[f"pool{k}"]), int(z[f"keep{k}"]), z[f"idx{k}"]
        got = common.rule_local_maxima(sc, shape, pool)
        got = got[np.lexsort((got, -sc[got]))]  # best first, ties by index (lw_score_maxima's order)
        thr = np.sort(sc)[::-1][min(pool, len(sc)) - 1]
        assert set(want.tolist()) <= set(got.tolist())
        extra = np.setdiff1d(got, want)
        assert np.all(sc[extra] == thr) or len(want) == keep, (k, sc[extra], thr)
        assert np.array_equal(sc[got[:len(want)]], sc[want]), k  # the same scores in the same order
        assert len(want) > 3
        k += 1
    assert k == 3
