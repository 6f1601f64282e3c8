"""The learned start-pose network on the GPU against the CPU oracle (float64 with the kernels' bf16 rounding points).

Forward: the tensor-core layers accumulate in float32 in an order of their own, so pooled values agree with the
float64 oracle to float32 rounding; a bf16 rounding of an activation can fall the other way when its float32 and
float64 values straddle a rounding boundary, and an argmax can move when two points tie to that precision, so a
small fraction of channels may differ. Tolerances: pooled within 1e-3 of the largest value for >= 99 % of the
channels, argmax equal for >= 98 %, the step within 2e-3 of its scale. Backward: every parameter tensor's
gradient within 2 % relative (Frobenius) of the oracle's.
"""

import numpy as np
import pytest
import torch

from oracle import oracle

pytestmark = pytest.mark.gpu


def _sets(n, seed):
    """2n point sets shaped like the real ones: points on a few random planes, a few metres out."""
    rng = np.random.default_rng(seed)
    out = np.zeros((2 * n, 1024, 4), np.float32)
    for s in range(2 * n):
        pts = []
        for _ in range(4):
            c = rng.uniform(-6, 6, 3)
            u, v = np.linalg.qr(rng.normal(size=(3, 3)))[0][:, :2].T
            ab = rng.uniform(-2, 2, (256, 2))
            pts.append(c + ab[:, :1] * u + ab[:, 1:] * v)
        out[s, :, :3] = np.concatenate(pts)
    return out


@pytest.fixture(scope="module")
def net():
    from livox_warp.initnet import InitNet

    return InitNet(seed=7, batch_cap=16)


def _w(net):
    return net.w.cpu().numpy().view(np.uint16)


def test_forward_matches_oracle(net):
    n = 4
    sets = _sets(n, 1)
    dev = torch.from_numpy(sets).cuda()
    f = net.forward(dev, n)
    pooled = f["pooled"].cpu().numpy().reshape(2 * n, 256)
    argmax = f["argmax"].cpu().numpy().reshape(2 * n, 256)
    step = f["step"].cpu().numpy()
    assert int(f["err"].cpu()[0]) == 0
    o = oracle.net_forward(_w(net), sets, net.in_scale, net.out_scale.cpu().numpy())
    scale = np.abs(o["pooled"]).max()
    close = np.abs(pooled - o["pooled"]) <= 1e-3 * scale
    assert close.mean() >= 0.99, close.mean()
    assert (argmax == o["argmax"]).mean() >= 0.98
    assert (pooled > 0).mean() > 0.3, "most channels should be active"
    sc = net.out_scale.cpu().numpy()
    assert np.all(np.abs(step - o["step"]) <= 2e-3 * sc)


def test_forward_training_batch(net):
    """The training batch's shape (256 pairs: 512 CTAs, about 3.5 waves on 148 SMs): the first and last pairs
    against the oracle, and every pair equal to the same pair run in a small batch (the CTAs are independent)."""
    n = 256
    sets = _sets(n, 5)
    dev = torch.from_numpy(sets).cuda()
    for _ in range(2):
        f = net.forward(dev, n)
        pooled = f["pooled"].cpu().numpy().reshape(2 * n, 256)
        assert int(f["err"].cpu()[0]) == 0
    pick = [0, n - 1]
    idx = np.array([[2 * q, 2 * q + 1] for q in pick]).reshape(-1)
    o = oracle.net_forward(_w(net), sets[idx], net.in_scale, net.out_scale.cpu().numpy())
    scale = np.abs(o["pooled"]).max()
    assert (np.abs(pooled[idx] - o["pooled"]) <= 1e-3 * scale).mean() >= 0.99
    small = net.forward(torch.from_numpy(np.ascontiguousarray(sets[idx])).cuda(), len(pick))
    assert np.array_equal(small["pooled"].cpu().numpy().reshape(-1, 256), pooled[idx])


def test_backward_matches_oracle(net):
    n = 4
    sets = _sets(n, 2)
    dev = torch.from_numpy(sets).cuda()
    rng = np.random.default_rng(3)
    target = (rng.normal(0, 1, (n, 6)) * net.out_scale.cpu().numpy()).astype(np.float32)
    wl = np.array([1, 1, 1, 2, 2, 2], np.float32)
    f = net.forward(dev, n)
    loss = net.backward(dev, n, f, torch.from_numpy(target), wl).sum().item()
    g = net.grad.cpu().numpy().astype(np.float64)
    o = oracle.net_forward(_w(net), sets, net.in_scale, net.out_scale.cpu().numpy())
    og, oloss = oracle.net_backward(_w(net), sets, o, target, wl, net.out_scale.cpu().numpy())
    assert abs(loss - oloss) <= 1e-3 * max(oloss, 1e-6)
    for name, off, shape in oracle._NET_SEG:
        m = int(np.prod(shape))
        a, b = g[off:off + m], og[off:off + m]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12)
        assert err < 2e-2, (name, err)


def test_adam_moves_masters_and_refreshes_bf16(net):
    from livox_warp.initnet import InitNet

    m = InitNet(seed=11, batch_cap=4)
    before = m.master.clone()
    m.grad.fill_(1.0)
    m.adam(1e-2)
    d = (m.master - before).cpu().numpy()
    assert np.allclose(d[:108038], -1e-2, atol=1e-6)  # first Adam step: -lr * sign(g)
    w = m.w.cpu().numpy().view(np.uint16)
    assert np.array_equal(w[:108038], oracle.bf16r(m.master.cpu().numpy()[:108038]).view(np.uint32)[:] >> 16)


def test_training_reduces_loss():
    """Training on the GPU learns: one scene seen from poses displaced by random steps (the map set is the frame
    set moved by the step, plus noise); the held-out loss falls well below where it starts."""
    from livox_warp.initnet import InitNet, apply_step

    N = 4096
    rng = np.random.default_rng(5)
    base = _sets(1, 9)[0, :, :3]
    sc = np.array([0.05, 0.05, 0.05, 0.03, 0.03, 0.03])
    steps = rng.normal(0, 1, (N, 6)) * sc
    sets = np.zeros((2 * N, 1024, 4), np.float32)
    for i in range(N):
        sets[2 * i, :, :3] = base
        Ti = np.linalg.inv(apply_step(np.eye(4), steps[i]))
        sets[2 * i + 1, :, :3] = base @ Ti[:3, :3].T + Ti[:3, 3] + rng.normal(0, 0.01, (1024, 3))
    net = InitNet(seed=1, batch_cap=128)
    hist = net.fit(torch.from_numpy(sets).cuda(), torch.from_numpy(steps.astype(np.float32)).cuda(), epochs=12,
                   batch=128, lr=1e-3)
    assert hist["val"][-1] < 0.5 * hist["val"][0], hist


def test_sets_match_numpy():
    """lw_net_sets: frame points at an even stride, map voxel means within the radius in slot order at an even
    stride, in the pose's frame."""
    from livox_warp import _lib, synth
    from livox_warp.initnet import frame_sets
    from livox_warp.kernels import RegistrationMap

    import common

    sc = synth.box_room(2)
    T = common.look_at([2.0, 2.0, 1.4], [6.0, 4.0, 1.0])
    traj = synth.ConstantVelocity(T, 0.0, 0.0, 0.0)
    x, a, t = synth.scan(sc, traj, 0.0, 0.3, 100000.0, 4)
    reg = RegistrationMap(1 << 16, "cuda")
    xyz4 = torch.from_numpy(np.concatenate([x, np.zeros((len(x), 1), np.float32)], 1)).cuda()
    reg.insert(xyz4, torch.from_numpy(a.view(np.int32)).cuda(), T, 0.15)
    ds = torch.from_numpy(np.concatenate([x[:5000], np.ones((5000, 1), np.float32)], 1)).cuda()
    n_ds = torch.tensor([5000], dtype=torch.int32, device="cuda")
    Tq = T.copy()
    Tq[:3, 3] += [0.3, -0.2, 0.1]
    Td = torch.from_numpy(Tq.reshape(16)).cuda()
    out = torch.zeros((2, 1024, 4), dtype=torch.float32, device="cuda")
    scratch = {"cand": torch.zeros(1 << 16, dtype=torch.int32, device="cuda"),
               "tiles": torch.zeros(66, dtype=torch.int32, device="cuda"),
               "count": torch.zeros(2, dtype=torch.int32, device="cuda")}
    frame_sets(ds, n_ds, reg, Td, 3.0, out, scratch, voxel=0.0)
    got = out.cpu().numpy()
    idx = (np.arange(1024) * 5000) // 1024
    assert np.array_equal(got[0, :, :3], x[idx])
    keys = reg.keys.cpu().numpy()
    rec = reg.rec.cpu().numpy().reshape(-1, _lib.REC_FLOATS)
    occ = (keys != -1) & (rec[:, 3] > 0)
    d2 = ((rec[:, :3] - Tq[:3, 3].astype(np.float32)) ** 2).sum(1)
    cand = np.nonzero(occ & (d2 <= np.float32(9.0)))[0]
    assert int(scratch["count"].cpu()[1]) == len(cand) > 50
    sel = cand[(np.arange(1024) * len(cand)) // 1024]
    want = (rec[sel, :3].astype(np.float64) - Tq[:3, 3]) @ Tq[:3, :3]
    assert np.allclose(got[1, :, :3], want, atol=1e-5)

    # nearest mode: each frame point's nearest voxel mean among the 27 voxels around it
    out2 = torch.zeros((2, 1024, 4), dtype=torch.float32, device="cuda")
    frame_sets(ds, n_ds, reg, Td, 0.0, out2, {"count": scratch["count"]}, voxel=0.15)
    got2 = out2.cpu().numpy()
    assert np.array_equal(got2[0], got[0])
    from livox_warp.gpu import key_to_ijk

    ijk = np.stack(key_to_ijk(keys[occ]), axis=1)
    means = rec[occ, :3]
    lut = {tuple(v): i for i, v in enumerate(ijk)}
    w = x[idx].astype(np.float64) @ Tq[:3, :3].T + Tq[:3, 3]
    c = np.floor(w.astype(np.float32) * np.float32(1.0 / 0.15)).astype(np.int64)
    hits = 0
    for i in range(1024):
        best, bd = None, np.inf
        for d in np.stack(np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1], indexing="ij"), -1).reshape(-1, 3):
            j = lut.get(tuple(c[i] + d))
            if j is None:
                continue
            e = means[j] - w[i].astype(np.float32)
            d2 = float((e * e).sum())
            if d2 < bd:
                bd, best = d2, j
        want_i = x[idx[i]] if best is None else (means[best].astype(np.float64) - Tq[:3, 3]) @ Tq[:3, :3]
        hits += best is not None
        assert np.allclose(got2[1, i, :3], want_i, atol=1e-4), i
    assert hits > 500
