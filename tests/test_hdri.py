"""Environment light (SetHDRI, SkyBox and the neural render's env / light
choice: core/hdr_loader.h:249, core/render.cuh:57-61, core/volume.cu:417-432,
1426-1458): the .hdr reader against the format's restatement and the
reference's own loader, and the CUDA renders against the oracle and the
reference's offline Render."""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import golden
from oracle import hdr_np, orc, ref_py
from internship_b200 import volume as V


def _sky_image(w=48, h=24, seed=3):
    """A smooth sky with a bright sun: (h, w, 3)."""
    rng = np.random.default_rng(seed)
    v = (np.arange(h) + 0.5) / h
    u = (np.arange(w) + 0.5) / w
    U, Vv = np.meshgrid(u, v)
    base = np.stack([0.3 + 0.5 * (1 - Vv), 0.4 + 0.4 * (1 - Vv), 0.8 + 0.2 * np.cos(2 * np.pi * U)], -1)
    sun = 40.0 * np.exp(-(((U - 0.3) / 0.05) ** 2 + ((Vv - 0.3) / 0.08) ** 2))
    img = base + sun[..., None] * np.array([1.0, 0.9, 0.7])
    return (img * rng.uniform(0.9, 1.1, img.shape)).astype(np.float32)


@pytest.mark.parametrize("rle", [True, False])
def test_hdr_reader_matches_format(tmp_path, rle):
    img = _sky_image()
    p = str(tmp_path / ("sky_rle.hdr" if rle else "sky_flat.hdr"))
    rgbe = hdr_np.write(p, img, rle=rle)
    ours = V.read_hdr(p)
    assert ours.shape == (24, 48, 4)
    np.testing.assert_array_equal(ours, hdr_np.decode(rgbe))
    # RGBE shares one exponent per pixel: each channel within 1/128 of the pixel's largest
    assert np.all(np.abs(ours[..., :3] - img) <= img.max(-1, keepdims=True) / 128)


@pytest.mark.parametrize("rle", [True, False])
def test_hdr_reader_matches_reference_loader(tmp_path, rle):
    """load_hdr_float4 of the reference, run on the same file."""
    if not os.path.exists(ref_py.VOL_SO):
        pytest.skip("oracle/_ref not built")
    img = _sky_image(40, 20, seed=7)
    p = str(tmp_path / "sky.hdr")
    hdr_np.write(p, img, rle=rle)
    np.testing.assert_array_equal(V.read_hdr(p), ref_py.RefVolume().load_hdr(p))


def test_hdr_reader_rejects_bad_files(tmp_path):
    from internship_b200 import _lib
    cases = {"not_radiance.hdr": b"P6\n1 1\n255\n\x00\x00\x00",
             "no_res.hdr": b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n",
             "truncated.hdr": b"#?RADIANCE\n\n-Y 4 +X 4\n\x01\x02\x03"}
    for name, data in cases.items():
        p = str(tmp_path / name)
        open(p, "wb").write(data)
        with pytest.raises(_lib.MRError):
            V.read_hdr(p)


def _setup(mr, tmp_path, res=48):
    from internship_b200 import scenes
    dens = scenes.sphere_density(res)
    v = mr.VolumeRender(res)
    v.SetDatas(dens)
    v.Update()
    p = str(tmp_path / "sky.hdr")
    hdr_np.write(p, _sky_image())
    v.SetHDRI(p)
    env = V.read_hdr(p)
    return v, dens, env


@pytest.mark.gpu
def test_delta_tracking_with_hdri_matches_oracle(tmp_path):
    """Escaped rays see the map (SkyBox): GPU delta tracking against the
    oracle on the same Philox streams, with the map set on both."""
    import internship_b200 as mr
    from internship_b200 import _lib, scenes
    v, dens, env = _setup(mr, tmp_path)
    p = scenes.make_params(24, 20, 32, alpha=16.0)
    p.env_color = _lib.f3((1.5, 1.5, 1.5))
    out = np.zeros(24 * 20 * 3, np.float32)
    _lib.check(_lib.load().mr_render_host(v.handle, None, C.byref(p), out.ctypes.data))
    orc.set_env(env)
    try:
        s, s2, _ = orc.render_pt(dens, v.max_density, p)
    finally:
        orc.set_env(None)
    ref = s / p.spp
    assert ref.mean() > 0.1  # the sky dominates the image
    close = np.abs(out - ref) <= 1e-4 * (np.abs(ref) + 1e-3)
    assert close.mean() > 0.9
    var = np.maximum(s2 / p.spp - ref ** 2, 0)
    assert np.all(np.abs(out - ref) <= 6 * np.sqrt(2 * var / p.spp) + 1e-5)
    v.close()


@pytest.mark.gpu
def test_neural_render_with_hdri_matches_oracle(tmp_path):
    """Neural passes with a map: sky pixels are SkyBox(dir); each pass takes
    the light the oracle's restatement of the env / light choice picks, with
    the transmittance pyramid of that light."""
    import internship_b200 as mr
    from internship_b200 import _lib, scenes
    from internship_b200.weights import active_random_weights
    v, dens, env = _setup(mr, tmp_path)
    w = active_random_weights(1)
    st = mr.builtin_stencil()
    v.SetWeights(w, st)
    md, mips, _ = orc.build_mips(dens)
    orc.set_env(env)
    picked_env = 0
    try:
        for k in range(6):
            p = scenes.make_params(16, 16, 1, rt=_lib.RT_MRPNN, alpha=16.0, sample_offset=k)
            p.env_color = _lib.f3((1.0, 1.0, 1.0))
            out = np.zeros(16 * 16 * 3, np.float32)
            _lib.check(_lib.load().mr_render_host(v.handle, v.network.handle, C.byref(p), out.ctypes.data))
            q = orc.RenderParams.from_buffer_copy(p)
            ld, lc = orc.select_env_light(q)
            picked_env += int(not np.allclose(ld, [p.light_dir.x, p.light_dir.y, p.light_dir.z]))
            q.light_dir.x, q.light_dir.y, q.light_dir.z = (float(c) for c in ld)
            q.light_color.x, q.light_color.y, q.light_color.z = (float(c) for c in lc)
            # the oracle with the tables of the chosen light
            tr = orc.build_tr(mips, q.alpha, ld / np.linalg.norm(ld))
            lut = orc.build_hglut(q.g, q.seed)
            ref = orc.render_neural(dens, md, mips, tr, lut, w, st, q)
            close = np.abs(out - ref) <= 2e-3 * (np.abs(ref) + 1e-3) + 1e-6
            assert close.mean() > 0.85, (k, close.mean())
    finally:
        orc.set_env(None)
    assert picked_env >= 1  # some passes took the light from the map
    v.close()


@pytest.mark.gpu
def test_delta_tracking_with_hdri_matches_reference():
    """The sphere scene under a map, against the reference's offline Render
    with SetHDRI on the same .hdr file (tests/golden/ref_hdri.npz)."""
    import internship_b200 as mr
    import torch
    from internship_b200 import _lib, scenes
    d = golden("ref_hdri.npz")
    W, H, spp = int(d["width"]), int(d["height"]), int(d["spp"])
    dens = scenes.sphere_density(128)
    v = mr.VolumeRender(128)
    v.SetDatas(dens)
    v.Update()
    v.SetHDRI(hdr_np.decode(d["rgbe"]))
    p = scenes.make_params(W, H, 1024, alpha=float(d["alpha"]), seed=9)
    p.env_color = _lib.f3((float(d["env_exp"]),) * 3)
    n = W * H * 3
    s = torch.zeros(n, dtype=torch.float64, device="cuda")
    s2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    _lib.check(_lib.load().mr_render_accumulate_f64(v.handle, C.byref(p), C.c_void_p(s.data_ptr()),
                                                   C.c_void_p(s2.data_ptr()), None))
    mean = (s / 1024).cpu().numpy()
    var = np.maximum((s2 / 1024).cpu().numpy() - mean ** 2, 0)
    ref = d["image"]
    se = np.sqrt(var / 1024 + var / spp) + 1e-4 * np.abs(ref) + 1e-6
    z = (mean - ref) / se
    assert np.mean(np.abs(z) > 4) < 0.01, np.mean(np.abs(z) > 4)
    assert abs(mean.mean() - ref.mean()) < 4 * np.sqrt((var / 1024 + var / spp).sum()) / var.size + 2e-3 * ref.mean()
    v.close()
