"""The reference's own device code and this library on the same GPU, on the
same scenes: the reference's per-pixel kernels (core/render.cuh
CalculateRadiance and NNPredict<MRPNN>, run through the harness in
oracle/ref/ref_harness.cu with the reference's 8 x 4 thread blocks, one
launch per pass) against mr_render. Square frames only: the reference's
RenderCamera indexing (pixel (i, j) at i * width + j) assumes width ==
height, so 1440 x 1440 stands in for 1920 x 1080 (the same 2,073,600
pixels). The times go to stdout (pytest -s)."""
import ctypes as C
import time

import numpy as np
import pytest

from oracle import ref_py

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mr():
    import torch
    assert torch.cuda.is_available()
    if not ref_py.available():
        pytest.skip("oracle/_ref not built")
    import internship_b200 as m
    return m


def _camera(p):
    return (np.array([p.ori.x, p.ori.y, p.ori.z], np.float32), np.array([p.up.x, p.up.y, p.up.z], np.float32),
            np.array([p.right.x, p.right.y, p.right.z], np.float32))


def _tables(v):
    from internship_b200 import _lib
    mips = np.concatenate([v.read(_lib.READ_MIP, k) for k in range(9)])
    tr = np.concatenate([v.read(_lib.READ_TR, k) for k in range(8)])
    return mips, tr, v.read(_lib.READ_HGLUT)


def _ref_pass_ms(ref, mode, p, L, bounces, passes, repeats=3):
    """Device time of one reference pass: wall time of passes + 1 passes
    minus that of one pass (the harness's allocations, the host copies of
    its FP64 sums and its final synchronisation cancel). Each wall time is
    the least of `repeats` runs, so that host noise in a single run (which
    once made the difference negative) does not enter."""
    ori, up, right = _camera(p)
    args = (p.width, p.height, ori, up, right, L, (1.0, 1.0, 1.0), p.alpha, bounces, p.g)
    ref.render(mode, *args, 1)  # warm-up
    one, many = [], []
    for _ in range(repeats):
        t0 = time.perf_counter()
        ref.render(mode, *args, 1)
        one.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        ref.render(mode, *args, passes + 1)
        many.append(time.perf_counter() - t0)
    ms = (min(many) - min(one)) * 1e3 / passes
    assert ms > 0, "reference pass time not resolved: %r, %r" % (one, many)
    return ms


def _ours_ms(v, p, frames):
    import torch
    from internship_b200 import _lib
    L_ = _lib.load()
    out = torch.empty(p.width * p.height * 3, device="cuda")
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    net = v.network.handle if v.network is not None else None
    for k in range(3):
        p.sample_offset = k
        _lib.check(L_.mr_render(v.handle, net, C.byref(p), C.c_void_p(out.data_ptr()), sp))
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for k in range(frames):
        p.sample_offset = 10 + k
        _lib.check(L_.mr_render(v.handle, net, C.byref(p), C.c_void_p(out.data_ptr()), sp))
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / frames


def test_neural_render_against_reference_kernel_same_gpu(mr):
    """The neural frame of the bench (512^3 fBm cloud, Xavier(seed 1)
    weights, 1 spp) at 1440 x 1440: the reference's NNPredict<MRPNN> per
    thread (fp32 network in registers, texture-filtered gather) against the
    fp32 / exact and BF16 / texture forms here."""
    import torch
    from internship_b200 import _lib, scenes
    W = 1440
    res = 512
    dens = torch.empty(res ** 3, device="cuda")
    scenes.generate_cloud_device(res, 7, dens.data_ptr())
    v = mr.VolumeRender(res)
    _lib.check(_lib.load().mr_volume_set_data_device(v.handle, C.c_void_p(dens.data_ptr()), dens.numel(), None))
    _lib.check(_lib.load().mr_volume_update(v.handle, None))
    md = C.c_float()
    _lib.check(_lib.load().mr_volume_max_density(v.handle, C.byref(md)))
    w = mr.xavier_weights(1)
    v.SetWeights(w, mr.builtin_stencil())
    p = scenes.cloud_scene_params(W, W, seed=0)
    ours = {}
    for name, prec, samp in (("fp32_exact", _lib.PREC_FP32, _lib.SAMPLER_EXACT),
                             ("bf16_texture", _lib.PREC_BF16, _lib.SAMPLER_TEXTURE)):
        p.precision, p.sampler = prec, samp
        ours[name] = _ours_ms(v, p, 10)
    mips, tr, lut = _tables(v)  # the tables the renders above used (light, alpha and g of p)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    ref = ref_py.Ref()
    ref.load_weights(w)
    ref.setup(dens.cpu().numpy(), md.value, mips, tr, lut, scatter=(0.99, 0.99, 0.99))
    ref_ms = _ref_pass_ms(ref, 1, p, L, 512, 16)
    print("\nneural %dx%d, 512^3 cloud: reference NNPredict<MRPNN> %.2f ms per frame (%.1f frames/s); "
          "here fp32/exact %.3f ms (%.1f frames/s, %.1fx), BF16/texture %.3f ms (%.1f frames/s, %.1fx)"
          % (W, W, ref_ms, 1e3 / ref_ms, ours["fp32_exact"], 1e3 / ours["fp32_exact"], ref_ms / ours["fp32_exact"],
             ours["bf16_texture"], 1e3 / ours["bf16_texture"], ref_ms / ours["bf16_texture"]))
    assert ours["fp32_exact"] < ref_ms
    v.close()


def test_delta_tracking_against_reference_kernel_same_gpu(mr):
    """Configuration 1 (128^3 sphere, 256 x 256, 64 spp, 512 bounces): the
    reference's CalculateRadiance, one thread per pixel and one launch per
    sample, against k_delta_track."""
    from internship_b200 import _lib, scenes
    dens = scenes.sphere_density(128)
    v = mr.VolumeRender(128)
    v.SetDatas(dens)
    v.Update()
    p = scenes.make_params(256, 256, 64)
    ours_ms = _ours_ms(v, p, 5)
    mips, tr, lut = _tables(v)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    ref = ref_py.Ref()
    ref.setup(dens, v.max_density, mips, tr, lut, scatter=(0.99, 0.99, 0.99))
    ref_ms = _ref_pass_ms(ref, 0, p, L, 512, 64)  # per sample pass
    samples = 256 * 256
    print("\ndelta tracking 256x256 x 64 spp, 128^3 sphere: reference %.3f ms per 1-spp pass (%.0f M samples/s); "
          "here %.3f ms per 64-spp frame (%.0f M samples/s, %.1fx)"
          % (ref_ms, samples / ref_ms / 1e3, ours_ms, 64 * samples / ours_ms / 1e3, 64 * ref_ms / ours_ms))
    assert ours_ms < 64 * ref_ms
    v.close()


def test_denoise_against_reference_kernel_same_gpu(mr):
    """The histogram denoiser at 1920 x 1080 with the filter active on every
    pixel (random counts 0..3 per bin, luminance variance 0.35, ACES): the
    reference's Denoise<true> kernel (one thread per pixel, 121 neighbour
    histograms read from memory per pixel; its device time from CUDA events
    in the harness) against mr_denoise (k_denoise). The packed outputs agree
    to one 8-bit step."""
    import torch
    from internship_b200 import _lib
    W, H = 1920, 1080
    n = W * H
    rng = np.random.default_rng(5)
    acc = (rng.random((n, 3), dtype=np.float32) * 2.0).astype(np.float32)
    hist = np.zeros((n, 33), np.float32)
    hist[:, :30] = rng.integers(0, 4, (n, 30)).astype(np.float32)
    hist[:, 30], hist[:, 31], hist[:, 32] = 16.0, 0.6, 0.5
    ref = ref_py.RefVolume()
    ref.denoise(acc, hist, W, H, 16, 0, 2, 1, timed=True)  # warm-up
    runs = [ref.denoise(acc, hist, W, H, 16, 0, 2, 1, timed=True) for _ in range(3)]
    ref_out, ref_ms = runs[0][0], min(r[1] for r in runs)
    da, dh = torch.from_numpy(acc).cuda(), torch.from_numpy(hist).cuda()
    out = torch.empty(n, dtype=torch.int32, device="cuda")
    it = _lib.Interactive()
    it.frame_index, it.tone, it.denoise, it.checkerboard, it.exposure = 16, 2, 1, 0, 1.0
    L_ = _lib.load()

    def run():
        _lib.check(L_.mr_denoise(C.c_void_p(da.data_ptr()), C.c_void_p(dh.data_ptr()), C.c_void_p(out.data_ptr()),
                                 W, H, C.byref(it), None))
    for _ in range(3):
        run()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(10):
        run()
    b.record()
    torch.cuda.synchronize()
    ours_ms = a.elapsed_time(b) / 10
    got = out.cpu().numpy().view(np.uint32)
    unpack = lambda x: np.stack([(x >> 16) & 255, (x >> 8) & 255, x & 255], -1).astype(np.int32)
    d = np.abs(unpack(got) - unpack(ref_out))
    print("\ndenoise 1920x1080, filter on every pixel: reference Denoise<true> %.2f ms; here k_denoise %.3f ms (%.1fx)"
          % (ref_ms, ours_ms, ref_ms / ours_ms))
    assert d.max() <= 1 and (d > 0).mean() < 0.01
    assert ours_ms < ref_ms
