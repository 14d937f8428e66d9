"""CPU tests of the oracle: known-answer vectors, the reference's own math
(tests/golden/ref_math.npz from core/vector.cu) and the fixtures produced by
the reference's device code (tests/golden/ref_*.npz)."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden, reference_file
from oracle import cloud_np, orc, ref_py
from internship_b200 import scenes


def test_philox_known_answers():
    # Random123 published KAT vectors for philox4x32_10.
    assert list(orc.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(orc.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(orc.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0])) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_uniform_stream_layout():
    u = orc.uniforms(7, 3, 5, 1, 9)
    for k in range(9):
        w = orc.philox([3, 5, k // 4, 1], [7, 0])
        assert u[k] == np.float32(((int(w[k % 4]) >> 9) + 0.5) * 2.0 ** -23)
    assert (u > 0).all() and (u < 1).all()


def test_python_philox_matches():
    assert scenes.philox4x32_10([1, 2, 3, 4], [5, 6]) == list(orc.philox([1, 2, 3, 4], [5, 6]))


def test_reference_math_golden():
    d = golden("ref_math.npz")
    a, o = d["inputs"], d["outputs"]
    L = orc.lib()
    for k in range(0, len(a), 7):
        c, g, s, e0 = (float(x) for x in a[k, :4])
        p = np.ascontiguousarray(a[k, 5:8])
        v = np.ascontiguousarray(o[k, 2:5])
        assert L.orc_hg(c, g) == pytest.approx(float(o[k, 0]), rel=1e-6)
        assert L.orc_hg_sample_cos(s, g) == pytest.approx(float(o[k, 1]), rel=1e-6, abs=1e-7)
        dd = np.zeros(3, np.float32)
        L.orc_hg_sample_dir(s, e0, v, g, dd)
        np.testing.assert_allclose(dd, o[k, 5:8], atol=2e-6)
        assert L.orc_ray_box_offset(p, v) == o[k, 8]
        assert L.orc_ray_box_distance(p, v) == o[k, 9]


def test_stencil_layout_golden():
    st = golden("ref_math.npz")["stencil"]
    L = orc.lib()
    for i in range(193):
        off, mip, ty, li = C.c_float(), C.c_int(), C.c_int(), C.c_int()
        L.orc_stencil_info(i, C.byref(off), C.byref(mip), C.byref(ty), C.byref(li))
        assert (off.value, mip.value, ty.value, li.value) == tuple(st[i].tolist())


def _np_trilinear_border(d, uv):
    res = d.shape[0]
    p = np.asarray(uv, np.float64) * res - 0.5
    f = np.floor(p)
    w = p - f
    x, y, z = f.astype(int)
    acc = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                i, j, k = x + dx, y + dy, z + dz
                v = d[i, j, k] if (0 <= i < res and 0 <= j < res and 0 <= k < res) else 0.0
                acc += v * (w[0] if dx else 1 - w[0]) * (w[1] if dy else 1 - w[1]) * (w[2] if dz else 1 - w[2])
    return acc


def test_trilinear_border_matches_numpy():
    rng = np.random.default_rng(0)
    d = rng.uniform(0, 1, (9, 9, 9)).astype(np.float32)
    L = orc.lib()
    for _ in range(200):
        uv = rng.uniform(-0.2, 1.2, 3).astype(np.float32)
        assert L.orc_sample_border(d.ravel(), 9, uv) == pytest.approx(_np_trilinear_border(d, uv), abs=2e-6)


def test_mip_pyramid_properties():
    rng = np.random.default_rng(1)
    d = rng.uniform(0, 2, (32, 32, 32)).astype(np.float32)
    md, mips, var = orc.build_mips(d)
    assert md == pytest.approx(float(d.max()))
    lv = [mips[sum(orc.MIP_SIZES[:k]):sum(orc.MIP_SIZES[:k + 1])].reshape((256 >> k,) * 3) for k in range(9)]
    vv = [var[sum(orc.MIP_SIZES[:k]):sum(orc.MIP_SIZES[:k + 1])].reshape((256 >> k,) * 3) for k in range(9)]
    for k in range(8):
        box = lv[k].reshape(128 >> k, 2, 128 >> k, 2, 128 >> k, 2)
        np.testing.assert_allclose(lv[k + 1], box.mean(axis=(1, 3, 5)), rtol=1e-5, atol=1e-6)
        np.testing.assert_allclose(vv[k + 1], np.maximum(0, (box ** 2).mean(axis=(1, 3, 5)) - box.mean(axis=(1, 3, 5)) ** 2),
                                   rtol=1e-3, atol=1e-5)
    assert (var >= 0).all()
    # mip0 samples the density at the 256^3 texel centres
    for idx in [(0, 0, 0), (100, 37, 200), (255, 255, 255)]:
        uv = (np.array(idx) + 0.5) / 256
        assert lv[0][idx] == pytest.approx(_np_trilinear_border(d, uv), abs=1e-5)


def test_tr_uniform_medium_known_answer():
    # Uniform density 1: along +x the transmittance of TR level k at an
    # interior voxel is exp(-alpha/1.73^(k+1) * (0.5 - x)).
    d = np.ones((64, 64, 64), np.float32)
    md, mips, var = orc.build_mips(d)
    alpha = 4.0
    tr = orc.build_tr(mips, alpha, np.array([1, 0, 0], np.float32))
    for k in (0, 1, 2):
        r = 128 >> k
        lvl = tr[sum(orc.TR_SIZES[:k]):sum(orc.TR_SIZES[:k + 1])].reshape(r, r, r)
        for x in (r // 8, r // 4, r // 2):
            px = (x + 0.5) / r - 0.5
            expect = np.exp(-alpha / 1.73 ** (k + 1) * (0.5 - px))
            # the last half texel before the exit blends with the zero border
            assert lvl[x, r // 2, r // 2] == pytest.approx(expect, rel=0.03)


def test_hglut_small_cone_is_phase_function():
    g = 0.857
    lut = orc.build_hglut(g, 0).reshape(512, 512)
    L = orc.lib()
    for i in (40, 200, 300, 450, 500):
        c = (i + 0.5) / 512 * 2 - 1
        assert lut[0, i] == pytest.approx(L.orc_hg(c, g), rel=0.02)
    assert (lut > 0).all()


def test_cloud_numpy_matches_definition_statistics():
    c = cloud_np.cloud(32, 3)
    assert c.min() >= 0 and c.max() <= 1
    assert 0.05 < (c > 0).mean() < 0.6


# ---- pins against the reference's own device code ---------------------------------

def test_network_matches_reference_xavier():
    d = golden("ref_network.npz")
    from internship_b200.weights import active_random_weights
    wx = active_random_weights(1)
    desc = ref_py.raw_to_desc(d["raw"], d["frames"], d["light"], d["g"])
    fr = d["frames"]
    gamma = np.arccos(np.clip((fr[:, 0:3] * fr[:, 9:12]).sum(1, dtype=np.float32), -1, 1)).astype(np.float32)
    for sr, key in ((d["scatterrate"], "out_xavier"), (d["scatterrate3"], "out_xavier3")):
        srp = ((sr * sr) * (sr * sr)).astype(np.float32)
        aux = np.zeros((len(desc), 5), np.float32)
        aux[:, 0], aux[:, 1], aux[:, 2:5] = d["g"], gamma, srp
        out = orc.predict(wx, desc, aux)
        ref = d[key]
        assert (ref > 0).mean() > 0.9
        np.testing.assert_allclose(out, ref, rtol=1e-4, atol=1e-6)


def test_network_matches_reference_weights():
    from internship_b200 import weights as W
    blob = W.load_nnweight_header(reference_file("core/NNWeight.cuh"))
    d = golden("ref_network.npz")
    desc = ref_py.raw_to_desc(d["raw"], d["frames"], d["light"], d["g"])
    fr = d["frames"]
    gamma = np.arccos(np.clip((fr[:, 0:3] * fr[:, 9:12]).sum(1, dtype=np.float32), -1, 1)).astype(np.float32)
    sr = d["scatterrate"]
    aux = np.zeros((len(desc), 5), np.float32)
    aux[:, 0], aux[:, 1], aux[:, 2:5] = d["g"], gamma, (sr * sr) * (sr * sr)
    out = orc.predict(blob, desc, aux)
    np.testing.assert_allclose(out, d["out_refw"], rtol=1e-4, atol=1e-6)


def _sphere_tables():
    dens = scenes.sphere_density(128)
    md, mips, var = orc.build_mips(dens)
    p = scenes.make_params(32, 32, 1)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    tr = orc.build_tr(mips, p.alpha, L)
    lut = orc.build_hglut(p.g, 0)
    return dens, md, mips, tr, lut, p, L


def test_delta_tracking_matches_reference_statistically():
    d = golden("ref_pt_sphere.npz")
    n_ref = int(d["spp"])
    ref_mean = d["sum"] / n_ref
    ref_var = np.maximum(d["sumsq"] / n_ref - ref_mean ** 2, 0)
    dens = scenes.sphere_density(128)
    md = float(dens.max())
    p = scenes.make_params(32, 32, 256)
    s, s2, _ = orc.render_pt(dens, md, p)
    mean = s / 256
    var = np.maximum(s2 / 256 - mean ** 2, 0)
    se = np.sqrt(ref_var / n_ref + var / 256) + 1e-6
    z = (mean - ref_mean) / se
    # per-pixel z-scores: Gaussian-like, no pixel far out
    assert np.abs(z).max() < 6.0
    assert np.mean(np.abs(z) > 3) < 0.01
    # image mean within a 4-sigma bound
    tot_se = np.sqrt((ref_var / n_ref + var / 256).sum()) / ref_mean.size
    assert abs(mean.mean() - ref_mean.mean()) < 4 * tot_se + 1e-6


def test_gather_network_matches_reference():
    from internship_b200 import weights as W
    stencil = W.load_stencil_source(reference_file("core/vector.cu"))
    blob = W.load_nnweight_header(reference_file("core/NNWeight.cuh"))
    d = golden("ref_gather.npz")
    dens, md, mips, tr, lut, p, L = _sphere_tables()
    desc, aux = orc.gather(mips, tr, lut, stencil, d["pos"], d["frames"], d["alpha"], d["g"],
                           np.array([0.99] * 3, np.float32), d["light"])
    out = orc.predict(blob, desc, aux)
    ref = d["out"]
    assert (ref > 0).mean() > 0.5
    # The reference reads through hardware texture filtering (8-bit
    # interpolation weights); the oracle interpolates in fp32.
    diff = np.abs(out - ref)
    err = diff / (np.abs(ref) + 1e-3)
    assert np.median(err) < 2e-3
    # every output within 5 % of the reference's, or 1e-4 absolute where the
    # radiance itself is a few 1e-4 and the 8-bit weights dominate
    assert np.all((diff < 5e-2 * np.abs(ref)) | (diff < 1e-4)), err.max()


def test_neural_render_matches_reference_statistically():
    from internship_b200 import weights as W
    stencil = W.load_stencil_source(reference_file("core/vector.cu"))
    blob = W.load_nnweight_header(reference_file("core/NNWeight.cuh"))
    d = golden("ref_nn_sphere.npz")
    n_ref = int(d["spp"])
    ref_mean = d["sum"] / n_ref
    ref_var = np.maximum(d["sumsq"] / n_ref - ref_mean ** 2, 0)
    dens, md, mips, tr, lut, p, L = _sphere_tables()
    p.render_type = 2
    K = 96
    acc = np.zeros(32 * 32 * 3)
    acc2 = np.zeros(32 * 32 * 3)
    for k in range(K):
        p.sample_offset = k
        o = orc.render_neural(dens, md, mips, tr, lut, blob, stencil, p).astype(np.float64)
        acc += o
        acc2 += o * o
    mean = acc / K
    var = np.maximum(acc2 / K - mean ** 2, 0)
    # heavy-tailed per-pass values: pool the variance over the image for the bound
    se = np.sqrt(ref_var / n_ref + var / K + (ref_var.mean() / n_ref + var.mean() / K))
    z = (mean - ref_mean) / (se + 1e-6)
    assert np.mean(np.abs(z) > 3) < 0.01
    tot_se = np.sqrt((ref_var / n_ref + var / K).sum()) / ref_mean.size
    assert abs(mean.mean() - ref_mean.mean()) < 4 * tot_se
    assert ref_mean.mean() > 0


def test_oracle_training_points_frames_and_loss():
    from internship_b200 import scenes
    from internship_b200.weights import active_random_weights
    dens = scenes.sphere_density(48)
    md, _, _ = orc.build_mips(dens)
    p1, d1 = orc.train_points(dens, md, 16.0, 0.857, 3, 1500, 10000)
    p2, d2 = orc.train_points(dens, md, 16.0, 0.857, 3, 1500, 10000)
    assert len(p1) > 100
    np.testing.assert_array_equal(p1, p2)  # one stream per ray: deterministic
    assert np.all(np.abs(p1) <= 0.5 + 1.0 / 128 + 1e-6)
    # samples lie where the medium is: inside the sphere of radius 0.25 (+ jitter)
    assert np.all(np.linalg.norm(p1, axis=1) < 0.25 + 0.02)
    fr = orc.train_frames(d1[:50], np.array([0, 0, 1], np.float32), 1)
    X, Y, Z = fr[:, 0:3], fr[:, 3:6], fr[:, 6:9]
    np.testing.assert_allclose(X, d1[:50] / np.linalg.norm(d1[:50], axis=1, keepdims=True), atol=1e-6)
    np.testing.assert_allclose(np.sum(X * Y, 1), 0, atol=1e-5)
    np.testing.assert_allclose(np.cross(Y, X), Z, atol=1e-5)
    rng = np.random.default_rng(0)
    desc = rng.uniform(0, 1, (8, 576)).astype(np.float32)
    aux = np.tile(np.array([0.85, 1.0, 0.9, 0.9, 0.9], np.float32), (8, 1))
    w = active_random_weights(1)
    out = orc.predict(w, desc, aux)
    X0 = np.log1p(out[:, 0] / 0.9)
    # loss against the network's own output is ~0; against shifted labels it is the shift squared
    assert orc.train_loss(w, desc, aux, out[:, 0]) < 1e-9
    lab = (np.expm1(X0 + 0.5) * 0.9).astype(np.float32)
    assert orc.train_loss(w, desc, aux, lab) == pytest.approx(0.25, rel=1e-3)
