"""The rest of VolumeRender's surface in the Python mirror (core/volume.hpp:96-145):
host-side table samplers (DensityAtUV / DensityAtPosition / TrAtPosition /
VarianceAtUV, core/volume.cu:675-722,1495-1576), GetSamples, the interactive
Render overload and SetSurfaceIOR."""
import numpy as np
import pytest

from oracle import orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def vol():
    import torch
    assert torch.cuda.is_available()
    import internship_b200 as mr
    rng = np.random.default_rng(4)
    d = rng.uniform(0, 1, (32, 32, 32)).astype(np.float32)
    v = mr.VolumeRender(32)
    v.SetDatas(d)
    v.Update()
    yield v, d
    v.close()


def _trilinear(data, uv, clamp):
    res = data.shape[0]
    p = np.asarray(uv, np.float64) * res - 0.5
    f = np.floor(p).astype(int)
    w = p - f
    acc = 0.0
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                i, j, k = f[0] + dx, f[1] + dy, f[2] + dz
                if clamp:
                    i, j, k = (min(max(a, 0), res - 1) for a in (i, j, k))
                ok = 0 <= i < res and 0 <= j < res and 0 <= k < res
                val = max(float(data[i, j, k]), 0.0) if ok else 0.0
                acc += val * (w[0] if dx else 1 - w[0]) * (w[1] if dy else 1 - w[1]) * (w[2] if dz else 1 - w[2])
    return acc


def test_density_at_uv_and_position(vol):
    v, d = vol
    _, mips, _ = orc.build_mips(d)
    rng = np.random.default_rng(0)
    for mip in (0, 2, 5):
        r = 256 >> mip
        off = sum(orc.MIP_SIZES[:mip])
        lvl = mips[off:off + r ** 3].reshape(r, r, r)
        for _ in range(20):
            uv = rng.uniform(-0.05, 1.05, 3).astype(np.float32)
            assert float(v.DensityAtUV(mip, uv[None])[0]) == pytest.approx(_trilinear(lvl, uv, False), abs=2e-5)
            assert float(v.DensityAtPosition(mip, (uv - 0.5)[None])[0]) == pytest.approx(
                _trilinear(lvl, uv, False), abs=2e-5)
    uv = np.array([[0.3, 0.6, 0.45]], np.float32)
    blend = 0.25 * v.DensityAtUV(2, uv) + 0.75 * v.DensityAtUV(3, uv)
    np.testing.assert_allclose(v.DensityAtUV(2.75, uv), blend, rtol=1e-6)


def test_variance_at_uv_as_the_reference_reads_it(vol):
    v, d = vol
    _, _, var = orc.build_mips(d)
    rng = np.random.default_rng(1)
    mip, r = 3, 32
    off = sum(orc.MIP_SIZES[:mip])
    flat = var[off:off + r ** 3]
    for _ in range(20):
        uv = rng.uniform(0, 1, 3).astype(np.float32)
        p = uv * r
        x0, y0, z0 = (int(a) for a in p)
        x1, y1, z1 = (min(a + 1, r - 1) for a in (x0, y0, z0))
        fx, fy, fz = p[0] - x0, p[1] - y0, p[2] - z0

        def g(x, y, z):
            return float(flat[(z * r + y) * r + x])
        c0 = (g(x0, y0, z0) * (1 - fx) + g(x1, y0, z0) * fx) * (1 - fy) + (g(x0, y1, z0) * (1 - fx) + g(x1, y1, z0) * fx) * fy
        c1 = (g(x0, y0, z1) * (1 - fx) + g(x1, y0, z1) * fx) * (1 - fy) + (g(x0, y1, z1) * (1 - fx) + g(x1, y1, z1) * fx) * fy
        ref = c0 * (1 - fz) + c1 * fz
        assert float(v.VarianceAtUV(mip, uv[None])[0]) == pytest.approx(ref, rel=1e-3, abs=1e-5)
    assert float(v.VarianceAtUV(9, np.zeros((1, 3), np.float32))[0]) == 0.0


def test_tr_at_position(vol):
    v, d = vol
    L = np.array([0.3, 0.8, -0.52], np.float32)
    L /= np.linalg.norm(L)
    v.Update_TR(L, 24.0)
    from internship_b200 import _lib
    lvl = v.read(_lib.READ_TR, 1).reshape(64, 64, 64)
    inside = np.array([[0.1, -0.2, 0.3]], np.float32)
    assert float(v.TrAtPosition(1, inside, L)[0]) == pytest.approx(_trilinear(lvl, inside[0] + 0.5, True), abs=1e-5)
    # outside: the volume entry towards the light, or 1 where that ray misses
    from internship_b200.scenes import ray_box_offset_np
    below, up = np.array([0.0, -0.9, 0.0], np.float32), np.array([0.0, 1.0, 0.0], np.float32)
    entry = below + up * np.float32(ray_box_offset_np(below, up)) + np.float32(0.5)
    assert float(v.TrAtPosition(1, below[None], up)[0]) == pytest.approx(_trilinear(lvl, entry, True), abs=1e-5)
    # RayBoxOffset misses only when the ray's slab intervals do not overlap (a
    # ray beside the box); one that starts above it and points away still
    # gets offset 0, as in the reference
    miss = np.array([[0.9, 0.9, 0.0]], np.float32)
    assert ray_box_offset_np(miss[0], up) < 0
    assert float(v.TrAtPosition(1, miss, up)[0]) == 1.0


def test_get_samples_matches_oracle(vol):
    v, d = vol
    rng = np.random.default_rng(2)
    pos = rng.uniform(-0.3, 0.3, (16, 3)).astype(np.float32)
    dirs = rng.normal(size=(16, 3)).astype(np.float32)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    L = np.array([0.0, 1.0, 0.0], np.float32)
    got = v.GetSamples(pos, dirs, L, 8.0, 0.8, 0.95, multiScatter=64, spp=512, seed=3)
    ref = orc.get_samples(d, v.max_density, pos, dirs, np.tile(L, (16, 1)), np.full(16, 8.0, np.float32),
                          np.full(16, 0.8, np.float32), np.full(16, 0.95, np.float32), 64, 512, seed=3)
    assert got.shape == (16,)
    # the same Philox streams: equal but where a rounding difference flips a decision
    assert np.mean(np.abs(got - ref) <= 1e-3 * np.abs(ref) + 1e-6) > 0.8


def test_render_interactive_wrapper(vol):
    import torch
    v, d = vol
    from internship_b200 import scenes
    W, H = 24, 16
    acc = torch.zeros(W * H * 3, device="cuda")
    hist = torch.zeros(W * H * 33, device="cuda")
    bgra = torch.zeros(W * H, dtype=torch.int32, device="cuda")
    ori, up, right = scenes.camera_vectors(np.array([0.0, 0.0, 2.5]), 40.0)
    v.SetCheckboard(False)
    for frame in range(3):
        v.RenderInteractive(acc, hist, bgra, (W, H), ori, up, right, (0.0, 1.0, 0.0), alpha=8.0, multiScatter=16,
                            randseed=frame, toneType=2, denoise=True)
    torch.cuda.synchronize()
    px = bgra.cpu().numpy().view(np.uint32)
    assert np.all(px >> 24 == 255)
    h = hist.cpu().numpy().reshape(-1, 33)
    assert np.all(h[:, 30] == 3)  # three frames in every pixel's histogram


def test_set_surface_ior(vol):
    v, _ = vol
    from internship_b200 import _lib
    v.SetSurfaceIOR(1.33)
    v.SetSurfaceIOR(-1.0)
    with pytest.raises(_lib.MRError):
        _lib.check(_lib.load().mr_volume_set_surface_ior(None, 1.0))
