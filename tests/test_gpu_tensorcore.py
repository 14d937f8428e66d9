"""GPU tests of the tcgen05 tensor-core network path (BF16 operands, FP32
accumulation) against plain matrix products and the FP32 oracle network."""
import ctypes as C

import numpy as np
import pytest

from oracle import orc, ref_py

pytestmark = pytest.mark.gpu


def _bf16_bits(x):
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return u.astype(np.uint16)


def _bf16_value(bits):
    return (bits.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.parametrize("n,k", [(16, 16), (32, 32), (16, 32), (32, 64), (64, 128), (128, 128)])
def test_tile_product_matches_matmul(n, k):
    from internship_b200 import _lib
    rng = np.random.default_rng(n * 1000 + k)
    a = _bf16_bits(rng.uniform(-1, 1, (128, k)))
    b = _bf16_bits(rng.uniform(-1, 1, (n, k)))
    d = np.zeros((128, n), np.float32)
    _lib.check(_lib.load().mr_tc_selftest(n, k, a.ctypes.data, b.ctypes.data, d.ctypes.data))
    ref = _bf16_value(a).astype(np.float64) @ _bf16_value(b).astype(np.float64).T
    np.testing.assert_allclose(d, ref, rtol=1e-5, atol=1e-5 * k)


def test_bounded_wait_times_out_and_frees_tensor_memory():
    """The failure path of the kernels' bounded mbarrier waits: a wait on an
    mbarrier that nothing arrives on gives up after its limit (5 ms here),
    the call reports MR_ERR_TIMEOUT, and the tensor memory it held is free
    again: a tile product right after it allocates and computes normally."""
    from internship_b200 import _lib
    L = _lib.load()
    waited = C.c_int64()
    rc = L.mr_tc_wait_selftest(5000, C.byref(waited))
    assert rc == _lib.MR_ERR_TIMEOUT, rc
    assert b"gave up" in L.mr_last_error()
    assert 5_000_000 <= waited.value < 500_000_000, waited.value
    for _ in range(2):
        rng = np.random.default_rng(7)
        a = _bf16_bits(rng.uniform(-1, 1, (128, 16)))
        b = _bf16_bits(rng.uniform(-1, 1, (16, 16)))
        d = np.zeros((128, 16), np.float32)
        _lib.check(L.mr_tc_selftest(16, 16, a.ctypes.data, b.ctypes.data, d.ctypes.data))
        ref = _bf16_value(a).astype(np.float64) @ _bf16_value(b).astype(np.float64).T
        np.testing.assert_allclose(d, ref, rtol=1e-5, atol=1e-4)


def _predict(mr, w, desc, aux, precision):
    import torch
    from internship_b200 import _lib
    net = mr.Network(w)
    n = len(desc)
    dd = torch.from_numpy(np.ascontiguousarray(desc)).cuda()
    da = torch.from_numpy(np.ascontiguousarray(aux)).cuda()
    out = torch.empty(n, 3, device="cuda")
    _lib.check(_lib.load().mr_radiance_predict(net.handle, precision, C.c_void_p(dd.data_ptr()),
                                               C.c_void_p(da.data_ptr()), n, C.c_void_p(out.data_ptr()), None))
    torch.cuda.synchronize()
    _lib.check(_lib.load().mr_network_check(net.handle, 1))
    net.close()
    return out.cpu().numpy()


def _descriptors(n, seed):
    rng = np.random.default_rng(seed)
    desc = np.zeros((n, 576), np.float32)
    desc[:, :192] = np.log1p(rng.uniform(0, 2, (n, 192)) * (rng.uniform(size=(n, 192)) > 0.3))
    desc[:, 192:384] = rng.uniform(0, 1, (n, 192))
    desc[:, 384:] = np.log1p(rng.uniform(0, 3, (n, 192)))
    aux = np.zeros((n, 5), np.float32)
    aux[:, 0] = 0.857
    aux[:, 1] = rng.uniform(0, np.pi, n)
    aux[:, 2:5] = np.float32((0.99 / 1.001) ** 4)
    return desc, aux


def _compare(bf, ref):
    # compare the network's pre-exponential output X = log(1 + out/srp)
    srp = np.float32((0.99 / 1.001) ** 4)
    xb, xr = np.log1p(bf / srp), np.log1p(ref / srp)
    return np.abs(xb - xr)


def test_bf16_network_matches_fp32_oracle():
    import internship_b200 as mr
    from internship_b200 import _lib
    from internship_b200.weights import active_random_weights
    w = active_random_weights(1)
    desc, aux = _descriptors(1000, 4)  # 7 full tiles + a partial one
    ref = orc.predict(w, desc, aux)
    bf = _predict(mr, w, desc, aux, _lib.PREC_BF16)
    fp = _predict(mr, w, desc, aux, _lib.PREC_FP32)
    np.testing.assert_allclose(fp, ref, rtol=1e-4, atol=1e-6)
    # BF16 operands (8-bit mantissa) through ~30 dependent layers with FP32
    # accumulation: the pre-exponential output X (~7 here) moves by a few 1e-2.
    err = _compare(bf, ref)
    assert np.median(err) < 0.05, np.median(err)
    assert np.quantile(err, 0.99) < 0.2, np.quantile(err, 0.99)


def test_bf16_network_three_albedo_channels():
    import internship_b200 as mr
    from internship_b200 import _lib
    from internship_b200.weights import active_random_weights
    w = active_random_weights(1)
    desc, aux = _descriptors(300, 5)
    sr = np.array([0.9, 0.95, 0.99], np.float32) / np.float32(1.001)
    aux[:, 2:5] = (sr * sr) * (sr * sr)
    ref = orc.predict(w, desc, aux)
    bf = _predict(mr, w, desc, aux, _lib.PREC_BF16)
    x_b = np.log1p(bf / aux[:, 2:5])
    x_r = np.log1p(ref / aux[:, 2:5])
    assert np.median(np.abs(x_b - x_r)) < 0.05
    # the three channels are distinct heads
    assert not np.allclose(ref[:, 0], ref[:, 2])


def test_fp32_network_albedo_channel_patterns():
    """fp32 network rows whose three albedo channels are equal, pairwise
    equal in each position, or all distinct, mixed within 128-row tiles: the
    head computes a further channel for a tile when one of its rows needs it,
    and the tail evaluates per row only the channels that row needs."""
    import internship_b200 as mr
    from internship_b200 import _lib
    from internship_b200.weights import active_random_weights
    w = active_random_weights(1)
    n = 700
    desc, aux = _descriptors(n, 8)
    a, b, c = 0.9, 0.95, 0.99
    patterns = np.array([[c, c, c], [a, b, c], [a, a, c], [a, c, c], [c, a, c], [b, b, b]], np.float32)
    rng = np.random.default_rng(9)
    pick = rng.integers(0, len(patterns), n)
    pick[:128] = 0  # one tile with a single channel only
    sr = patterns[pick] / np.float32(1.001)
    aux[:, 2:5] = (sr * sr) * (sr * sr)
    ref = orc.predict(w, desc, aux)
    got = _predict(mr, w, desc, aux, _lib.PREC_FP32)
    assert (ref > 0).mean() > 0.9
    np.testing.assert_allclose(got, ref, rtol=1e-4, atol=1e-6)
    for k in range(len(patterns)):  # rows with equal channels give equal outputs
        rows = pick == k
        sp = aux[rows, 2:5]
        for i, j in ((0, 1), (1, 2), (0, 2)):
            same = sp[:, i] == sp[:, j]
            assert np.array_equal(got[rows][same, i] / sp[same, i], got[rows][same, j] / sp[same, j])


@pytest.mark.skipif(not ref_py.available(), reason="oracle/_ref not built")
def test_bf16_network_with_reference_weights():
    import internship_b200 as mr
    from internship_b200 import _lib
    w = ref_py.RefNet().read_weights()
    desc, aux = _descriptors(512, 6)
    ref = orc.predict(w, desc, aux)
    bf = _predict(mr, w, desc, aux, _lib.PREC_BF16)
    rel = np.abs(bf - ref) / (np.abs(ref) + 1e-2)
    assert np.median(rel) < 0.03, np.median(rel)
    assert np.quantile(rel, 0.99) < 0.2


def test_bf16_neural_render_close_to_fp32():
    import internship_b200 as mr
    from internship_b200 import _lib, scenes
    from internship_b200.weights import active_random_weights
    dens = scenes.sphere_density(128)
    v = mr.VolumeRender(128)
    v.SetDatas(dens)
    v.Update()
    v.SetWeights(active_random_weights(1), mr.builtin_stencil())
    out = {}
    for prec in (_lib.PREC_FP32, _lib.PREC_BF16):
        p = scenes.make_params(64, 64, 1, rt=_lib.RT_MRPNN, precision=prec)
        img = np.zeros(64 * 64 * 3, np.float32)
        _lib.check(_lib.load().mr_render_host(v.handle, v.network.handle, C.byref(p), img.ctypes.data))
        out[prec] = img
    a, b = out[_lib.PREC_FP32], out[_lib.PREC_BF16]
    active = a > 0
    assert active.mean() > 0.05
    rel = np.abs(np.log1p(b[active]) - np.log1p(a[active]))
    assert np.median(rel) < 0.05
    assert ((a == 0) == (b == 0)).all()
    v.close()


# ---- E4M3 (MR_PREC_FP8) -------------------------------------------------------------

def _e4m3_encode(x):
    """OCP E4M3 bytes of x (round to nearest even, saturating at 448)."""
    x = np.asarray(x, np.float64)
    out = np.zeros(x.shape, np.uint8)
    for idx, v in np.ndenumerate(x):
        s = 0x80 if v < 0 else 0
        a = min(abs(v), 448.0)
        if a < 2.0 ** -6:
            out[idx] = s | int(np.rint(a * 512))
            continue
        e = int(np.floor(np.log2(a)))
        q = int(np.rint((a / 2.0 ** e - 1) * 8))
        if q == 8:
            q, e = 0, e + 1
        out[idx] = s | ((e + 7) << 3) | q
    return out


def _e4m3_value(b):
    b = np.asarray(b, np.int32)
    sgn = np.where(b & 0x80, -1.0, 1.0)
    E, q = (b >> 3) & 15, b & 7
    return sgn * np.where(E == 0, q * 2.0 ** -9, (1 + q / 8.0) * 2.0 ** (E - 7.0))


@pytest.mark.parametrize("n,k", [(16, 32), (32, 32), (64, 128), (128, 128)])
def test_fp8_tile_product_matches_matmul(n, k):
    from internship_b200 import _lib
    rng = np.random.default_rng(n * 7 + k)
    a = _e4m3_encode(rng.uniform(-8, 8, (128, k)))
    b = _e4m3_encode(rng.uniform(-2, 2, (n, k)))
    d = np.zeros((128, n), np.float32)
    _lib.check(_lib.load().mr_tc_selftest_fp8(n, k, a.ctypes.data, b.ctypes.data, d.ctypes.data))
    ref = _e4m3_value(a) @ _e4m3_value(b).T  # E4M3 products are exact in FP32
    np.testing.assert_allclose(d, ref, rtol=1e-5, atol=1e-5 * k)


def test_fp8_network_close_to_fp32():
    """E4M3 operands carry 3 mantissa bits (up to 6 % rounding error per
    operand): through ~30 dependent layers the per-layer / per-row scaled
    network stays within a few percent of the fp32 oracle on X (a wrong scale
    would be off by a power of two)."""
    import internship_b200 as mr
    from internship_b200.weights import active_random_weights
    w = active_random_weights(1)
    desc, aux = _descriptors(512, 6)
    ref = orc.predict(w, desc, aux)
    f8 = _predict(mr, w, desc, aux, 2)
    bf = _predict(mr, w, desc, aux, 1)
    d8, db = _compare(f8, ref), _compare(bf, ref)
    xr = np.log1p(ref / np.float32((0.99 / 1.001) ** 4))
    rel8 = d8 / np.maximum(xr, 1e-3)
    print("median |dX| fp8 %.4f bf16 %.4f, median rel fp8 %.4f" % (np.median(d8), np.median(db), np.median(rel8)))
    assert np.all(np.isfinite(f8)) and (f8 > 0).mean() > 0.5
    assert np.median(rel8) < 0.08
    assert np.quantile(rel8, 0.99) < 0.3
    assert np.median(d8) > np.median(db)  # coarser than BF16, as it must be


@pytest.mark.parametrize("n,k", [(16, 16), (32, 32), (32, 64), (64, 128)])
def test_tf32_split_tile_product_is_fp32_accurate(n, k):
    """kind::tf32 tile product through the K-major 4-byte operand layout:
    one TF32 product carries ~11 bits per operand; the three-term split
    (A_hi B_hi + A_hi B_lo + A_lo B_hi) carries ~22, i.e. the error of an
    fp32 dot product."""
    from internship_b200 import _lib
    rng = np.random.default_rng(n * 13 + k)
    a = rng.standard_normal((128, k)).astype(np.float32)
    b = rng.standard_normal((n, k)).astype(np.float32)
    ref = a.astype(np.float64) @ b.astype(np.float64).T
    scale = np.abs(a).astype(np.float64) @ np.abs(b).astype(np.float64).T  # sum of |terms|
    L = _lib.load()
    d1 = np.zeros((128, n), np.float32)
    _lib.check(L.mr_tc_selftest_tf32(n, k, a.ctypes.data, b.ctypes.data, d1.ctypes.data, 0))
    d3 = np.zeros((128, n), np.float32)
    _lib.check(L.mr_tc_selftest_tf32(n, k, a.ctypes.data, b.ctypes.data, d3.ctypes.data, 1))
    e1 = np.abs(d1 - ref) / scale
    e3 = np.abs(d3 - ref) / scale
    print("max error / sum|terms|: tf32 %.3g, split %.3g" % (e1.max(), e3.max()))
    assert e1.max() < 2e-3  # one TF32 product per element
    assert e3.max() < 1e-6  # fp32-level
    assert e3.max() < e1.max() / 100


@pytest.mark.parametrize("n,k", [(64, 32), (128, 64), (128, 128), (64, 128)])
@pytest.mark.parametrize("a_mn,b_mn", [(0, 1), (1, 0), (1, 1)])
def test_mn_major_tile_product_matches_matmul(n, k, a_mn, b_mn):
    """The BF16 training's backward products read forward tiles transposed
    (MN-major operands): D = A B^T through those descriptors equals the fp32
    product of the BF16 inputs."""
    from internship_b200 import _lib
    rng = np.random.default_rng(n * 7 + k + 3 * a_mn + b_mn)
    a = _bf16_bits(rng.standard_normal((128, k)).astype(np.float32))
    b = _bf16_bits(rng.standard_normal((n, k)).astype(np.float32))
    d = np.zeros((128, n), np.float32)
    _lib.check(_lib.load().mr_tc_selftest_mn(n, k, a_mn, b_mn, a.ctypes.data, b.ctypes.data, d.ctypes.data))
    ref = _bf16_value(a).astype(np.float64) @ _bf16_value(b).astype(np.float64).T
    np.testing.assert_allclose(d, ref, rtol=1e-5, atol=1e-4)
