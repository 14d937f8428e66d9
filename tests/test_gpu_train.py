"""The learned part on the GPU: training-data generator against the oracle,
hand-written gradients against finite differences of the oracle's loss, and
what a trained network gains over the method without it."""
import ctypes as C

import numpy as np
import pytest

from oracle import orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _sphere_volume(res=64):
    import internship_b200 as mr
    from internship_b200 import scenes
    dens = scenes.sphere_density(res)
    v = mr.VolumeRender(res)
    v.SetDatas(dens)
    v.Update()
    return v, dens


def test_train_points_match_oracle(torch):
    from internship_b200 import _lib
    v, dens = _sphere_volume()
    n_rays, cap = 4000, 20000
    pos = torch.empty(cap, 3, device="cuda")
    dirs = torch.empty(cap, 3, device="cuda")
    cnt = C.c_int32()
    _lib.check(_lib.load().mr_train_points(v.handle, 16.0, 0.857, 3, n_rays, cap, _ptr(pos), _ptr(dirs), C.byref(cnt),
                                           None))
    n = cnt.value
    gp, gd = pos[:n].cpu().numpy(), dirs[:n].cpu().numpy()
    rp, rd = orc.train_points(dens, v.max_density, 16.0, 0.857, 3, n_rays, cap)
    assert n > 500 and abs(n - len(rp)) <= max(3, 0.01 * len(rp))
    # same set of points (order differs: the GPU compacts with an atomic counter)
    key = lambda p: np.round(p * 1e4).astype(np.int64)
    gs = {tuple(k) for k in np.concatenate([key(gp), key(gd)], 1)}
    hit = sum(tuple(k) in gs for k in np.concatenate([key(rp), key(rd)], 1))
    assert hit >= 0.97 * len(rp)
    assert np.all(np.abs(gp) <= 0.5 + 1.0 / 128 + 1e-6)
    np.testing.assert_allclose(np.linalg.norm(gd, axis=1), 1.0, atol=1e-5)
    v.close()


def test_train_labels_match_oracle(torch):
    from internship_b200 import _lib
    v, dens = _sphere_volume()
    rp, rd = orc.train_points(dens, v.max_density, 16.0, 0.857, 5, 600, 200)
    n, spp = len(rp), 32
    L = np.array([0.3, 0.8, -0.5], np.float32)
    L /= np.linalg.norm(L)
    sums = torch.zeros(n, device="cuda", dtype=torch.float64)
    dp, dd = torch.from_numpy(rp).cuda(), torch.from_numpy(rd).cuda()  # kept alive across the launch
    _lib.check(_lib.load().mr_train_labels(v.handle, _ptr(dp), _ptr(dd), n, _lib.f3(L), 16.0, 0.857, 0.95, 64, spp, 9,
                                           _ptr(sums), None))
    gpu = sums.cpu().numpy() / spp
    ref = orc.get_samples(dens, v.max_density, rp, rd, np.tile(L, (n, 1)), np.full(n, 16.0, np.float32),
                          np.full(n, 0.857, np.float32), np.full(n, 0.95, np.float32), 64, spp, 9)
    assert (ref > 0).mean() > 0.5
    rel = np.abs(gpu - ref) / (np.abs(ref) + 1e-4)
    # identical streams: most labels agree to float rounding; a path whose
    # accept/reject flips on an ulp difference changes one of 32 samples
    assert np.median(rel) < 1e-3
    assert abs(gpu.mean() - ref.mean()) < 0.02 * ref.mean()
    v.close()


def test_train_frames_match_oracle(torch):
    from internship_b200 import _lib
    rng = np.random.default_rng(2)
    d = rng.normal(size=(300, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    L = np.array([0.0, 1.0, 0.0], np.float32)
    fr = torch.empty(300, 12, device="cuda")
    dd = torch.from_numpy(d).cuda()
    _lib.check(_lib.load().mr_train_frames(_ptr(dd), 300, _lib.f3(L), 4, _ptr(fr), None))
    np.testing.assert_allclose(fr.cpu().numpy(), orc.train_frames(d, L, 4), rtol=1e-5, atol=1e-6)


def _rows(n, seed):
    """Synthetic rows with the value ranges of real descriptors."""
    rng = np.random.default_rng(seed)
    desc = np.concatenate([rng.uniform(0, 1.5, (n, 192)), rng.uniform(0, 1, (n, 192)),
                           rng.uniform(0, 2, (n, 192))], 1).astype(np.float32)
    srp = ((0.95 / 1.001) ** 4)
    aux = np.stack([rng.uniform(0.7, 0.9, n), rng.uniform(0, np.pi, n), np.full(n, srp), np.full(n, srp),
                    np.full(n, srp)], 1).astype(np.float32)
    label = rng.uniform(0.01, 2.0, n).astype(np.float32)
    return desc, aux, label


def test_gradient_matches_oracle_finite_differences(torch):
    from internship_b200.train import Trainer
    from internship_b200.weights import active_random_weights, layout
    w = active_random_weights(1)
    desc, aux, label = _rows(64, 7)
    tr = Trainer(w)
    dd, da, dl = (torch.from_numpy(x).cuda() for x in (desc, aux, label))
    g, loss = tr.gradient(dd, da, dl)
    tr.close()
    assert loss == pytest.approx(orc.train_loss(w, desc, aux, label), rel=1e-4)
    # one random entry of every weight array, plus the largest gradients
    rng = np.random.default_rng(0)
    idx, off = [], 0
    for _, n in layout():
        idx.append(off + int(rng.integers(n)))
        off += n
    idx += list(np.argsort(-np.abs(g))[:60])
    eps = 1e-3
    ok = 0
    gmax = float(np.abs(g).max())
    assert gmax > 0
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (orc.train_loss(wp, desc, aux, label) - orc.train_loss(wm, desc, aux, label)) / (2 * eps)
        ok += abs(g[i] - fd) <= 2e-3 * gmax + 0.05 * abs(fd)
    # ReLU kinks within eps of a row's pre-activation spoil a few differences
    assert ok >= 0.9 * len(idx), (ok, len(idx))


def test_training_gain_over_no_network(torch):
    """Train on generated data; on held-out rows the trained network's error
    in X = log(1 + L/srp) must be well below the method without the network
    (single scattering only, X = 0) and below the untrained network."""
    from internship_b200 import train
    cfgs = train.scene_configs(2, seed=3, resolutions=(64,), alpha_range=(16.0, 48.0))
    desc, aux, label = train.generate(cfgs, 6000, spp=128, max_bounces=128, seed=1)
    n = len(label)
    assert n > 8000
    perm = torch.randperm(n, device="cuda", generator=torch.Generator(device="cuda").manual_seed(0))
    hold, trn = perm[:1500], perm[1500:]
    w0 = train.initial_weights(1)
    w, hist = train.fit(desc[trn], aux[trn], label[trn], w0, epochs=25, batch=1024, lr=1e-3)
    print("loss per epoch", [round(h, 5) for h in hist])
    T = train.targets(aux[hold], label[hold])
    dh, ah = desc[hold].contiguous(), aux[hold].contiguous()
    rmse = float(torch.sqrt(torch.mean((train.predict_x(w, dh, ah) - T) ** 2)))
    rmse_init = float(torch.sqrt(torch.mean((train.predict_x(w0, dh, ah) - T) ** 2)))
    rmse_none = float(torch.sqrt(torch.mean(T ** 2)))
    print("held-out rmse: trained %.4f, untrained %.4f, no network %.4f" % (rmse, rmse_init, rmse_none))
    assert hist[-1] < 0.5 * hist[0]
    assert rmse < 0.5 * rmse_none, (rmse, rmse_none)
    assert rmse < 0.5 * rmse_init, (rmse, rmse_init)


def test_bf16_gradient_close_to_fp32(torch):
    """MR_PREC_BF16 training: the head's products on the tensor cores with BF16
    operands. Its gradient, against the fp32 kernel's on the same rows (which
    the finite-difference test pins), differs by BF16 rounding only."""
    from internship_b200.train import Trainer
    from internship_b200.weights import active_random_weights, layout
    w = active_random_weights(1)
    desc, aux, label = _rows(4096, 7)
    dd, da, dl = (torch.from_numpy(x).cuda() for x in (desc, aux, label))
    res = {}
    for prec in ("fp32", "bf16"):
        tr = Trainer(w, prec)
        res[prec] = tr.gradient(dd, da, dl)
        tr.close()
    (g32, l32), (g16, l16) = res["fp32"], res["bf16"]
    assert l16 == pytest.approx(l32, rel=5e-3)
    cos = float(np.dot(g32, g16) / (np.linalg.norm(g32) * np.linalg.norm(g16)))
    assert cos > 0.9999, cos
    assert np.linalg.norm(g32 - g16) < 0.01 * np.linalg.norm(g32)
    off = 0
    for name, n in layout():
        a, b = g32[off:off + n], g16[off:off + n]
        if np.linalg.norm(a) > 1e-3 * np.linalg.norm(g32):
            assert np.linalg.norm(a - b) < 0.03 * np.linalg.norm(a), name
        off += n


def test_bf16_training_gain_over_no_network(torch):
    """The same gain test as for fp32 training, with the BF16 tensor-core head."""
    from internship_b200 import train
    cfgs = train.scene_configs(2, seed=3, resolutions=(64,), alpha_range=(16.0, 48.0))
    desc, aux, label = train.generate(cfgs, 6000, spp=128, max_bounces=128, seed=1)
    n = len(label)
    perm = torch.randperm(n, device="cuda", generator=torch.Generator(device="cuda").manual_seed(0))
    hold, trn = perm[:1500], perm[1500:]
    w0 = train.initial_weights(1)
    w, hist = train.fit(desc[trn], aux[trn], label[trn], w0, epochs=25, batch=1024, lr=1e-3, precision="bf16")
    T = train.targets(aux[hold], label[hold])
    dh, ah = desc[hold].contiguous(), aux[hold].contiguous()
    rmse = float(torch.sqrt(torch.mean((train.predict_x(w, dh, ah) - T) ** 2)))
    rmse_none = float(torch.sqrt(torch.mean(T ** 2)))
    print("BF16 training, held-out rmse: trained %.4f, no network %.4f" % (rmse, rmse_none))
    assert hist[-1] < 0.5 * hist[0]
    assert rmse < 0.5 * rmse_none, (rmse, rmse_none)
