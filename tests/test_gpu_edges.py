"""Edge cases of the render path on the GPU: an empty volume, a one-pixel and
a ragged odd-sized frame, paths with no bounce allowed, a batch that mixes an
empty volume with a full one, and network row counts that end inside a
128-row tile."""
import ctypes as C

import numpy as np
import pytest

from oracle import orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mr():
    import torch
    assert torch.cuda.is_available()
    import internship_b200 as m
    return m


def _volume(mr, dens):
    v = mr.VolumeRender(dens.shape[0])
    v.SetDatas(dens)
    v.Update()
    return v


def _render(v, p, net=None):
    from internship_b200 import _lib
    out = np.zeros(p.width * p.height * 3, np.float32)
    _lib.check(_lib.load().mr_render_host(v.handle, net, C.byref(p), out.ctypes.data))
    return out.reshape(p.height, p.width, 3)


@pytest.mark.parametrize("rt", ["pt", "mrpnn"])
def test_empty_volume_shows_the_environment(mr, rt):
    """Density zero everywhere: no collision anywhere, every ray escapes and
    sees the constant environment colour (SkyBox without a map)."""
    from internship_b200 import _lib, scenes
    from internship_b200.weights import active_random_weights
    v = _volume(mr, np.zeros((32, 32, 32), np.float32))
    env = (0.2, 0.3, 0.4)
    if rt == "pt":
        p = scenes.make_params(16, 12, 4)
        net = None
    else:
        v.SetWeights(active_random_weights(1), mr.builtin_stencil())
        p = scenes.make_params(16, 12, 1, rt=_lib.RT_MRPNN)
        net = v.network.handle
    p.env_color = _lib.f3(env)
    img = _render(v, p, net)
    np.testing.assert_allclose(img, np.broadcast_to(np.array(env, np.float32), img.shape), rtol=1e-6, atol=1e-7)
    v.close()


def test_zero_bounces(mr):
    """max_bounces 0: a ray that enters the volume contributes nothing; one
    that misses it sees the environment."""
    from internship_b200 import _lib, scenes
    dens, p = scenes.sphere_scene(24, 24, 2)
    p.max_bounces = 0
    p.env_color = _lib.f3((1.0, 1.0, 1.0))
    v = _volume(mr, dens)
    img = _render(v, p)
    s, _, _ = orc.render_pt(dens, v.max_density, p)
    ref = (s / p.spp).reshape(img.shape)
    # each of the 2 samples of a pixel contributes 0 (entered) or 1 (missed)
    assert set(np.unique(ref)) <= {0.0, 0.5, 1.0} and (ref == 0).any() and (ref == 1).any()
    # the same jittered rays: only a ray grazing the box edge may decide differently
    assert np.sum(np.abs(img - ref).max(axis=2) > 1e-6) <= 2
    v.close()


@pytest.mark.parametrize("w,h", [(1, 1), (7, 3), (3, 7)])
def test_tiny_and_ragged_frames_match_oracle(mr, w, h):
    """One-pixel and odd-sized frames through both render types, against the
    oracle on the same streams."""
    from internship_b200 import _lib, scenes
    from internship_b200.weights import active_random_weights
    dens = scenes.sphere_density(64)
    v = _volume(mr, dens)
    p = scenes.make_params(w, h, 64)
    gpu = _render(v, p).ravel()
    s, s2, _ = orc.render_pt(dens, v.max_density, p)
    ref = (s / p.spp).astype(np.float32)
    # the same streams: equal but where a rounding difference flips a Woodcock
    # decision, which changes one of the pixel's 64 paths
    se = np.sqrt(2 * np.maximum(s2 / p.spp - (s / p.spp) ** 2, 0) / p.spp)
    assert np.all(np.abs(gpu - ref) <= 4 * se + 1e-4)
    w8, st = active_random_weights(1), mr.builtin_stencil()
    v.SetWeights(w8, st)
    p = scenes.make_params(w, h, 1, rt=_lib.RT_MRPNN)
    gpu = _render(v, p, v.network.handle).ravel()
    gm = np.concatenate([v.read(_lib.READ_MIP, k) for k in range(9)])
    tr = np.concatenate([v.read(_lib.READ_TR, k) for k in range(8)])
    ref = orc.render_neural(dens, v.max_density, gm, tr, v.read(_lib.READ_HGLUT), w8, st, p)
    close = np.abs(gpu - ref) <= 1e-3 * (np.abs(ref) + 1e-3) + 1e-6
    assert close.mean() >= 0.9 or (gpu.size < 10 and close.sum() >= gpu.size - 1)
    v.close()


def test_batch_with_an_empty_volume(mr):
    """A batch whose first job sees an empty volume and whose second sees the
    sphere: the empty job's frame is the environment, the other matches its
    single render."""
    import torch
    from internship_b200 import _lib, scenes
    from internship_b200.weights import active_random_weights
    L = _lib.load()
    ve = _volume(mr, np.zeros((32, 32, 32), np.float32))
    vs = _volume(mr, scenes.sphere_density(64))
    w, st = active_random_weights(1), mr.builtin_stencil()
    net = mr.Network(w, st)
    jobs = []
    for v, (W, H) in ((ve, (20, 10)), (vs, (24, 16))):
        p = scenes.make_params(W, H, 1, rt=_lib.RT_MRPNN, precision=_lib.PREC_BF16)
        p.env_color = _lib.f3((0.25, 0.5, 0.75))
        jobs.append((v, p, torch.empty(W * H * 3, device="cuda")))
    b = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b)))
    for v, p, o in jobs:
        _lib.check(L.mr_batch_add(b, v.handle, C.byref(p), C.c_void_p(o.data_ptr())))
    stream = torch.cuda.Stream()
    sp = C.c_void_p(stream.cuda_stream)
    _lib.check(L.mr_batch_prepare(b, net.handle, 256, sp))
    _lib.check(L.mr_batch_render(b, net.handle, sp))
    stream.synchronize()
    empty = jobs[0][2].cpu().numpy().reshape(-1, 3)
    np.testing.assert_allclose(empty, np.broadcast_to(np.array([0.25, 0.5, 0.75], np.float32), empty.shape),
                               rtol=1e-6)
    v, p, o = jobs[1]
    single = np.zeros(p.width * p.height * 3, np.float32)
    _lib.check(L.mr_render_host(v.handle, net.handle, C.byref(p), single.ctypes.data))
    # separately compiled kernels of the same source: fp32 contraction may differ in a few values
    np.testing.assert_allclose(o.cpu().numpy(), single, rtol=5e-6, atol=1e-7)
    _lib.check(L.mr_batch_destroy(b))
    net.close()
    ve.close()
    vs.close()


@pytest.mark.parametrize("n", [1, 127, 129, 383])
def test_predict_ragged_row_counts(mr, n):
    """mr_radiance_predict on row counts that leave a partial 128-row tile:
    fp32 against the oracle's network, BF16 and FP8 close to fp32, and no
    write past row n."""
    import torch
    from internship_b200 import _lib
    from internship_b200.weights import active_random_weights
    rng = np.random.default_rng(n)
    desc = np.zeros((n, 576), np.float32)
    desc[:, :192] = rng.uniform(0.05, 3, (n, 192))
    desc[:, 192:384] = rng.uniform(0, 1, (n, 192))
    desc[:, 384:] = rng.uniform(0.05, 3, (n, 192))
    aux = np.zeros((n, 5), np.float32)
    aux[:, 0], aux[:, 1], aux[:, 2:5] = 0.857, rng.uniform(0, 3, n), 0.96
    w = active_random_weights(1)
    net = mr.Network(w, mr.builtin_stencil())
    dd, da = torch.from_numpy(desc).cuda(), torch.from_numpy(aux).cuda()
    ref = orc.predict(w, desc, aux)
    outs = {}
    for name, prec in (("fp32", _lib.PREC_FP32), ("bf16", _lib.PREC_BF16), ("fp8", _lib.PREC_FP8)):
        out = torch.full((n + 64, 3), -7.0, device="cuda")  # sentinel rows after the last
        _lib.check(_lib.load().mr_radiance_predict(net.handle, prec, C.c_void_p(dd.data_ptr()),
                                                   C.c_void_p(da.data_ptr()), n, C.c_void_p(out.data_ptr()), None))
        torch.cuda.synchronize()
        o = out.cpu().numpy()
        assert np.all(o[n:] == -7.0), name
        outs[name] = o[:n]
    np.testing.assert_allclose(outs["fp32"], ref, rtol=1e-4, atol=1e-6)
    # on X = log(1 + L / srp), with the tensor-core tests' bounds (BF16: 8-bit
    # mantissas through ~30 layers; E4M3: 3-bit)
    x32 = np.log1p(outs["fp32"] / 0.96)
    db = np.abs(np.log1p(outs["bf16"] / 0.96) - x32)
    d8 = np.abs(np.log1p(outs["fp8"] / 0.96) - x32) / np.maximum(x32, 1e-3)
    assert np.all(np.isfinite(outs["bf16"])) and np.all(np.isfinite(outs["fp8"]))
    assert db.max() < 0.3 and (n < 10 or np.median(db) < 0.05)
    assert n < 10 or np.median(d8) < 0.08
    net.close()
