"""Batched neural rendering: a batch of (volume, view) jobs must render what
the single-render path renders for each job, eagerly and through the captured
CUDA graph, with the autotuner's choices."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _jobs(mr, precision, sampler):
    from internship_b200 import _lib, scenes
    from internship_b200.weights import active_random_weights
    from oracle import cloud_np
    va = mr.VolumeRender(64)
    va.SetDatas(scenes.sphere_density(64))
    va.Update()
    vb = mr.VolumeRender(48)
    vb.SetDatas(cloud_np.cloud(48, 3))
    vb.Update()
    net = mr.Network(active_random_weights(1), mr.builtin_stencil())
    pa1 = scenes.make_params(40, 24, 1, rt=_lib.RT_MRPNN, precision=precision, sampler=sampler, alpha=32.0)
    pa2 = scenes.make_params(33, 50, 1, rt=_lib.RT_MRPNN, precision=precision, sampler=sampler, alpha=32.0,
                             distance=2.0, fov=50.0, seed=0, sample_offset=5)
    pb = scenes.make_params(56, 31, 1, rt=_lib.RT_MRPNN, precision=precision, sampler=sampler, alpha=80.0,
                            light_seed=3, albedo=0.95, sample_offset=2)
    return [(va, pa1), (va, pa2), (vb, pb)], net


def _single(torch, net, jobs, advance):
    from internship_b200 import _lib
    out = []
    for v, p in jobs:
        q = _lib.RenderParams.from_buffer_copy(p)
        q.sample_offset = p.sample_offset + advance
        img = torch.empty(q.width * q.height * 3, device="cuda")
        _lib.check(_lib.load().mr_render(v.handle, net.handle, C.byref(q), _ptr(img), None))
        torch.cuda.synchronize()
        out.append(img.cpu().numpy())
    return out


@pytest.mark.parametrize("precision,sampler,wave",
                         [(1, 0, 1000), (0, 0, 1000), (1, 1, 1000), (0, 0, 0), (0, 1, 0), (1, 1, 0), (1, 0, 0)])
def test_batch_matches_single_renders(torch, precision, sampler, wave):
    import internship_b200 as mr
    from internship_b200 import _lib
    L = _lib.load()
    jobs, net = _jobs(mr, precision, sampler)
    outs = [torch.full((p.width * p.height * 3,), -1.0, device="cuda") for _, p in jobs]
    b = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b)))
    for (v, p), o in zip(jobs, outs):
        _lib.check(L.mr_batch_add(b, v.handle, C.byref(p), _ptr(o)))
    # waves of 1000 pixels: every wave mixes jobs, records span wave
    # boundaries; wave 0: the whole batch in one wave, where the records of
    # both volumes share warps
    _lib.check(L.mr_batch_prepare(b, net.handle, wave, None))
    _lib.check(L.mr_batch_render(b, net.handle, None))
    torch.cuda.synchronize()
    got = [o.cpu().numpy() for o in outs]
    ref = _single(torch, net, jobs, 0)
    for g, r in zip(got, ref):
        assert (r > 0).mean() > 0.05
        # the batched and the single-render gathers are separately compiled
        # kernels of the same source; the compiler may contract a few fp32
        # expressions differently (measured: <= 3e-6 relative in <= 0.5 % of
        # the values, fp32 exact)
        np.testing.assert_allclose(g, r, rtol=5e-6, atol=1e-7)
    cnt = (C.c_uint64 * 4)()
    _lib.check(L.mr_batch_counters(b, cnt))
    assert cnt[3] == sum(int((r.reshape(-1, 3).max(1) > 0).sum()) for r in ref)
    L.mr_batch_destroy(b)
    net.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_with_distinct_albedo_channels(torch, precision):
    """A job whose three albedo channels differ (one head per channel; the
    tensor-core network spills its head input for the further channels) in
    one wave with a gray job on another volume."""
    import internship_b200 as mr
    from internship_b200 import _lib
    L = _lib.load()
    jobs, net = _jobs(mr, precision, 0)
    jobs[2][1].scatter_rate = _lib.f3((0.9, 0.95, 0.99))
    jobs = [jobs[0], jobs[2]]
    outs = [torch.full((p.width * p.height * 3,), -1.0, device="cuda") for _, p in jobs]
    b = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b)))
    for (v, p), o in zip(jobs, outs):
        _lib.check(L.mr_batch_add(b, v.handle, C.byref(p), _ptr(o)))
    _lib.check(L.mr_batch_prepare(b, net.handle, 0, None))
    _lib.check(L.mr_batch_render(b, net.handle, None))
    torch.cuda.synchronize()
    got = [o.cpu().numpy() for o in outs]
    ref = _single(torch, net, jobs, 0)
    for g, r in zip(got, ref):
        np.testing.assert_allclose(g, r, rtol=5e-6, atol=1e-7)  # as in test_batch_matches_single_renders
    rgb = ref[1].reshape(-1, 3)
    lit = rgb.max(1) > 0
    assert not np.allclose(rgb[lit, 0], rgb[lit, 2])  # the channels differ
    L.mr_batch_destroy(b)
    net.close()


def test_batch_graph_replays_advance_frames(torch):
    import internship_b200 as mr
    from internship_b200 import _lib
    L = _lib.load()
    jobs, net = _jobs(mr, 1, 0)
    outs = [torch.zeros(p.width * p.height * 3, device="cuda") for _, p in jobs]
    b = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b)))
    for (v, p), o in zip(jobs, outs):
        _lib.check(L.mr_batch_add(b, v.handle, C.byref(p), _ptr(o)))
    _lib.check(L.mr_batch_prepare(b, net.handle, 0, None))
    s = torch.cuda.Stream()
    sp = C.c_void_p(s.cuda_stream)
    _lib.check(L.mr_batch_capture(b, net.handle, sp))  # renders frame +0 eagerly
    _lib.check(L.mr_batch_launch(b, sp))               # frame +1
    _lib.check(L.mr_batch_launch(b, sp))               # frame +2
    s.synchronize()
    got = [o.cpu().numpy() for o in outs]
    for g, r in zip(got, _single(torch, net, jobs, 2)):
        np.testing.assert_allclose(g, r, rtol=5e-6, atol=1e-7)  # as in test_batch_matches_single_renders
    # the default stream cannot be captured
    assert L.mr_batch_capture(b, net.handle, None) == _lib.MR_ERR_ARG
    L.mr_batch_destroy(b)
    net.close()


def test_batch_autotune_and_errors(torch):
    import internship_b200 as mr
    from internship_b200 import _lib, scenes
    L = _lib.load()
    jobs, net = _jobs(mr, 1, 0)
    outs = [torch.zeros(p.width * p.height * 3, device="cuda") for _, p in jobs]
    b = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b)))
    assert L.mr_batch_render(b, net.handle, None) == _lib.MR_ERR_STATE  # not prepared
    for (v, p), o in zip(jobs, outs):
        _lib.check(L.mr_batch_add(b, v.handle, C.byref(p), _ptr(o)))
    # a PT job and a mixed precision are rejected
    bad = scenes.make_params(8, 8, 1)
    assert L.mr_batch_add(b, jobs[0][0].handle, C.byref(bad), _ptr(outs[0])) == _lib.MR_ERR_ARG
    bad = scenes.make_params(8, 8, 1, rt=_lib.RT_MRPNN, precision=_lib.PREC_FP32)
    assert L.mr_batch_add(b, jobs[0][0].handle, C.byref(bad), _ptr(outs[0])) == _lib.MR_ERR_ARG
    _lib.check(L.mr_batch_prepare(b, net.handle, 0, None))
    wave, tb, gb = C.c_int64(), C.c_int32(), C.c_int32()
    _lib.check(L.mr_batch_autotune(b, net.handle, C.byref(wave), C.byref(tb), C.byref(gb), None))
    total = sum(p.width * p.height for _, p in jobs)
    assert 0 < wave.value <= total and tb.value in (64, 128, 256) and gb.value in (64, 128, 256)
    s = torch.cuda.Stream()
    _lib.check(L.mr_batch_capture(b, net.handle, C.c_void_p(s.cuda_stream)))
    _lib.check(L.mr_batch_launch(b, C.c_void_p(s.cuda_stream)))
    s.synchronize()
    assert all(float(o.max()) > 0 for o in outs)
    L.mr_batch_destroy(b)
    # a second job on a volume whose tables serve another light is rejected
    b2 = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b2)))
    v, p = jobs[0]
    _lib.check(L.mr_batch_add(b2, v.handle, C.byref(p), _ptr(outs[0])))
    q = _lib.RenderParams.from_buffer_copy(p)
    q.alpha = p.alpha * 2
    _lib.check(L.mr_batch_add(b2, v.handle, C.byref(q), _ptr(outs[1])))
    assert L.mr_batch_prepare(b2, net.handle, 0, None) == _lib.MR_ERR_ARG
    L.mr_batch_destroy(b2)
    net.close()


def test_large_single_render_matches_waved_batch(torch):
    """A 1280 x 1280 single render against the same view through the batched
    path in waves of 64 Ki pixels (both gathers read a per-point table)."""
    import internship_b200 as mr
    from internship_b200 import _lib, scenes
    from internship_b200.weights import active_random_weights
    from oracle import cloud_np
    L = _lib.load()
    v = mr.VolumeRender(128)
    v.SetDatas(cloud_np.cloud(128, 5))
    v.Update()
    net = mr.Network(active_random_weights(1), mr.builtin_stencil())
    p = scenes.make_params(1280, 1280, 1, rt=_lib.RT_MRPNN, precision=0, sampler=0, alpha=48.0)
    out = torch.full((1280 * 1280 * 3,), -1.0, device="cuda")
    b = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b)))
    _lib.check(L.mr_batch_add(b, v.handle, C.byref(p), _ptr(out)))
    _lib.check(L.mr_batch_prepare(b, net.handle, 65536, None))
    _lib.check(L.mr_batch_render(b, net.handle, None))
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    ref = _single(torch, net, [(v, p)], 0)[0]
    cnt = (C.c_uint64 * 4)()
    _lib.check(L.mr_volume_counters(v.handle, cnt))
    # more active records than the single render's resident gather grid has
    # threads (148 SMs x 6 blocks x 128): its threads stride over records
    assert cnt[3] > 148 * 6 * 128, cnt[3]
    assert (ref > 0).mean() > 0.05
    np.testing.assert_allclose(got, ref, rtol=5e-6, atol=1e-7)
    L.mr_batch_destroy(b)
    net.close()
    v.close()


def test_batch_frame_times_follow_the_waves(torch):
    """mr_batch_set_timing: completion times per frame from events inside the
    captured graph; frames complete in add order (waves run in order) and
    the last one with the batch."""
    import internship_b200 as mr
    from internship_b200 import _lib
    L = _lib.load()
    jobs, net = _jobs(mr, 1, 0)
    b = C.c_void_p()
    _lib.check(L.mr_batch_create(C.byref(b)))
    outs = []
    for v, p in jobs:
        o = torch.empty(p.width * p.height * 3, device="cuda")
        outs.append(o)
        _lib.check(L.mr_batch_add(b, v.handle, C.byref(p), _ptr(o)))
    stream = torch.cuda.Stream()
    sp = C.c_void_p(stream.cuda_stream)
    _lib.check(L.mr_batch_prepare(b, net.handle, 1000, sp))  # several waves
    ft = np.zeros(len(jobs), np.float32)
    assert L.mr_batch_frame_times(b, ft.ctypes.data, len(jobs)) == _lib.MR_ERR_STATE
    _lib.check(L.mr_batch_set_timing(b, 1))
    _lib.check(L.mr_batch_capture(b, net.handle, sp))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    _lib.check(L.mr_batch_launch(b, sp))
    e1.record(stream)
    torch.cuda.synchronize()
    _lib.check(L.mr_batch_frame_times(b, ft.ctypes.data, len(jobs)))
    total = e0.elapsed_time(e1)
    assert np.all(ft > 0) and np.all(np.diff(ft) >= 0), ft
    assert ft[-1] <= total * 1.05 + 0.05
    assert ft[0] < ft[-1]  # the first job's frame finished in an earlier wave
    _lib.check(L.mr_batch_destroy(b))
    for v, _ in jobs[::2]:
        v.close()
    net.close()
