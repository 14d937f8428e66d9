"""The exact sampler's two forms: fp32 trilinear / bilinear filters over texel
loads (used where nothing may be allocated) and over texture gathers (tld4,
the default form). Gathers return the 2 x 2 footprint's texels unfiltered, so
the two forms agree bit for bit; the one documented exception is a subnormal
texel, which the texture unit reads as 0."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
R = 32  # MR_SAMPLER_SELFTEST_RES


def _run(table, uv):
    from internship_b200 import _lib
    n = uv.shape[0]
    out = np.zeros((n, 6), np.float32)
    _lib.check(_lib.load().mr_sampler_selftest(n, table.ctypes.data, np.ascontiguousarray(uv).ctypes.data,
                                               out.ctypes.data))
    return out


def _points(rng, n):
    uv = rng.uniform(-0.15, 1.15, (n, 3)).astype(np.float32)
    # texel centres, texel edges and the table border exactly
    g = (np.arange(-1, R + 2, dtype=np.float32) + 0.5) / R
    e = np.arange(-1, R + 2, dtype=np.float32) / R
    k = len(g)
    uv[:k, 0] = g
    uv[k:2 * k, 1] = e
    uv[2 * k:3 * k, 2] = g
    return uv


def _tri_ref(t, uv, border):
    """float64 trilinear filter of the x-major table t (R^3), texture space."""
    T = t.reshape(R, R, R).astype(np.float64)
    p = uv.astype(np.float64) * R - 0.5
    f = np.floor(p)
    w = p - f
    i = f.astype(np.int64)
    out = np.zeros(len(uv))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                x, y, z = i[:, 0] + dx, i[:, 1] + dy, i[:, 2] + dz
                if border:
                    ok = (x >= 0) & (x < R) & (y >= 0) & (y < R) & (z >= 0) & (z < R)
                    v = np.where(ok, T[np.clip(x, 0, R - 1), np.clip(y, 0, R - 1), np.clip(z, 0, R - 1)], 0.0)
                else:
                    v = T[np.clip(x, 0, R - 1), np.clip(y, 0, R - 1), np.clip(z, 0, R - 1)]
                wt = (w[:, 0] if dx else 1 - w[:, 0]) * (w[:, 1] if dy else 1 - w[:, 1]) * (w[:, 2] if dz else 1 - w[:, 2])
                out += wt * v
    return out


def test_gather_form_matches_load_form_bitwise():
    rng = np.random.default_rng(7)
    table = (rng.random(R ** 3, dtype=np.float32) * 4.0).astype(np.float32)
    table[rng.random(R ** 3) < 0.2] = 0.0
    uv = _points(rng, 20000)
    out = _run(table, uv)
    for a, b in ((0, 1), (2, 3), (4, 5)):
        np.testing.assert_array_equal(out[:, b], out[:, a])
    # and both are the trilinear filter of the table (border 0 / clamp)
    np.testing.assert_allclose(out[:, 0], _tri_ref(table, uv, True), rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(out[:, 2], _tri_ref(table, uv, False), rtol=1e-5, atol=1e-5)


def test_gather_form_reads_subnormal_texels_as_zero():
    rng = np.random.default_rng(8)
    table = np.full(R ** 3, np.float32(1e-40), np.float32)  # subnormal everywhere
    uv = rng.uniform(0.1, 0.9, (256, 3)).astype(np.float32)
    out = _run(table, uv)
    assert (out[:, 0] > 0).all() and (out[:, 2] > 0).all()  # loads keep them
    assert (out[:, 1] == 0).all() and (out[:, 3] == 0).all()  # gathers flush them
