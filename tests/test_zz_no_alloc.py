"""mr_render_neural_noalloc: the neural render over the module-resident
scratch must give the same image as mr_render (which uses the volume's own
growable scratch), call after call, without allocating device memory.

Kept in its own file, collected after the other tests, so that it runs both
alone and after everything else in the same process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup():
    import torch
    import internship_b200 as mr
    from internship_b200 import scenes
    from internship_b200.weights import active_random_weights
    assert torch.cuda.is_available()
    v = mr.VolumeRender(128)
    v.SetDatas(scenes.sphere_density(128))
    v.Update()
    v.SetWeights(active_random_weights(1), mr.builtin_stencil())
    return torch, v


@pytest.mark.parametrize("width,height,albedo", [(128, 128, None), (100, 37, None), (96, 64, (0.9, 0.95, 0.99))])
@pytest.mark.parametrize("precision", [0, 1])  # MR_PREC_FP32, MR_PREC_BF16
def test_noalloc_matches_render_twice(width, height, albedo, precision):
    """albedo: three distinct channels, one network head each; the tensor-core
    network then spills the head inputs into the scratch's spill columns."""
    from internship_b200 import _lib, scenes
    torch, v = _setup()
    L = _lib.load()
    p = scenes.make_params(width, height, 1, rt=_lib.RT_MRPNN, precision=precision)
    if albedo is not None:
        p.scatter_rate.x, p.scatter_rate.y, p.scatter_rate.z = albedo
    n = width * height * 3
    ref = torch.empty(n, device="cuda")
    out = torch.full((n,), -1.0, device="cuda")
    for call in range(2):
        p.sample_offset = 11 + call
        # the existing entry point first: it also builds the HG table and the
        # transmittance pyramid the no-alloc call requires
        _lib.check(L.mr_render(v.handle, v.network.handle, C.byref(p), C.c_void_p(ref.data_ptr()), None))
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        _lib.check(L.mr_render_neural_noalloc(v.handle, v.network.handle, C.byref(p), C.c_void_p(out.data_ptr()),
                                              None))
        torch.cuda.synchronize()
        if call == 1:
            assert torch.cuda.mem_get_info()[0] == free0  # nothing allocated
        a, b = ref.cpu().numpy(), out.cpu().numpy()
        assert (a > 0).mean() > 0.05
        # mr_render's exact sampler reads texture gathers, the no-alloc call
        # texel loads: the same texels except subnormal ones, which the
        # texture unit reads as 0 (tests/test_gpu_sampler.py)
        np.testing.assert_allclose(b, a, rtol=1e-5, atol=1e-6)
    v.close()


def test_noalloc_rejects_what_it_cannot_do():
    from internship_b200 import _lib, scenes
    torch, v = _setup()
    L = _lib.load()
    out = torch.empty(_lib.NOALLOC_MAX_PIXELS * 3 + 3, device="cuda")
    dp = C.c_void_p(out.data_ptr())
    # tables not yet built for these parameters
    p = scenes.make_params(64, 64, 1, rt=_lib.RT_MRPNN)
    assert L.mr_render_neural_noalloc(v.handle, v.network.handle, C.byref(p), dp, None) == _lib.MR_ERR_STATE
    assert b"mr_volume_update" in L.mr_last_error()
    _lib.check(L.mr_render(v.handle, v.network.handle, C.byref(p), dp, None))
    # one pixel beyond the fixed scratch
    p = scenes.make_params(_lib.NOALLOC_MAX_PIXELS + 1, 1, 1, rt=_lib.RT_MRPNN)
    assert L.mr_render_neural_noalloc(v.handle, v.network.handle, C.byref(p), dp, None) == _lib.MR_ERR_ARG
    assert b"MR_NOALLOC_MAX_PIXELS" in L.mr_last_error()
    p = scenes.make_params(64, 64, 1, rt=_lib.RT_MRPNN, sampler=_lib.SAMPLER_TEXTURE)
    assert L.mr_render_neural_noalloc(v.handle, v.network.handle, C.byref(p), dp, None) == _lib.MR_ERR_ARG
    p = scenes.make_params(64, 64, 1, rt=_lib.RT_PT)
    assert L.mr_render_neural_noalloc(v.handle, v.network.handle, C.byref(p), dp, None) == _lib.MR_ERR_ARG
    torch.cuda.synchronize()
    v.close()
