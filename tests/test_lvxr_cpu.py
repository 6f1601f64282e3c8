"""LVXR recordings decoded by the library against the reference's own reader (lvxr.py read_firings and
Firings.points, run by tests/golden/make_golden.py on seeded synthetic recordings: every record layout, ns and GPS
timestamps, a forward clock jump and a restart, IMU / malformed / truncated datagrams, the Mid-40 dual-return
profile, LVXR1). Times, reflectivity, tags, validity and the firing order are exact; cartesian coordinates are
exact; spherical ones come from float32 sin / cos, which numpy's vectorised float32 routines round differently from
the C library's in about one value in ten -- within 4 float32 ulps (rtol 5e-7)."""

from pathlib import Path

import numpy as np
import pytest

G = np.load(Path(__file__).resolve().parent / "golden" / "lvxr.npz")
NAMES = ("mid40", "horizon", "dual", "v1")


@pytest.mark.parametrize("name", NAMES)
def test_decode_matches_reference_reader(name):
    from livox_warp import lvxr

    f = lvxr.decode(G[f"{name}_bytes"].tobytes())
    assert (f.dev_type, f.profile) == tuple(G[f"{name}_meta"]) and f.interval == float(G[f"{name}_interval"])
    assert f.xyz.shape == G[f"{name}_xyz"].shape and f.returns == G[f"{name}_xyz"].shape[1]
    assert np.array_equal(f.t, G[f"{name}_t"])
    assert np.array_equal(f.refl, G[f"{name}_refl"]) and np.array_equal(f.tag, G[f"{name}_tag"])
    assert np.array_equal(f.valid, G[f"{name}_valid"])
    np.testing.assert_allclose(f.xyz, G[f"{name}_xyz"], rtol=5e-7, atol=0)
    want_dir = G[f"{name}_direction"]
    assert np.array_equal(np.isnan(f.direction), np.isnan(want_dir))
    ok = ~np.isnan(want_dir)
    np.testing.assert_allclose(f.direction[ok], want_dir[ok], rtol=5e-7, atol=1e-7)
    assert (f.xyz == G[f"{name}_xyz"]).mean() > 0.8  # most of it bit-identical (every cartesian return)
    px, pa, pt, pf = f.points(clean=True, min_range=0.3)
    assert np.array_equal(pa, G[f"{name}_pts_attr"]) and np.array_equal(pt, G[f"{name}_pts_t"])
    assert np.array_equal(pf, G[f"{name}_pts_f"])
    np.testing.assert_allclose(px, G[f"{name}_pts_xyz"], rtol=5e-7, atol=0)


def test_decode_edge_cases(tmp_path):
    from livox_warp import _lib, lvxr

    with pytest.raises(_lib.LwError, match="not an LVXR"):
        lvxr.decode(b"PCAP\n....")
    with pytest.raises(_lib.LwError, match="no point packets"):
        lvxr.decode(b"LVXR2\n" + bytes([1, 0]))
    data = G["v1_bytes"].tobytes()
    p = tmp_path / "rec.lvxr"
    p.write_bytes(data)
    f = lvxr.read_firings(p)
    assert len(f.t) == 400 and f.misses.sum() == (~G["v1_valid"].any(axis=1)).sum()
    h = f.head(0.002)
    assert len(h.t) == int((f.t < f.t[0] + 0.002).sum()) and h.xyz.shape[1:] == f.xyz.shape[1:]
