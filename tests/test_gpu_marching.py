"""The marching form of the neural render (NNPredict<Type::marching_MRPNN>,
core/render.cuh:371-461, 524-633; render type MR_RT_MARCHING_MRPNN), with and
without a dielectric surface (SetSurfaceIOR): the CUDA path against the
oracle on the same Philox streams, and against the reference's own marching
code (tests/golden/ref_march.npz)."""
import ctypes as C

import numpy as np
import pytest

from conftest import golden
from oracle import orc, ref_py

pytestmark = pytest.mark.gpu


def _setup(res=96):
    import internship_b200 as mr
    from internship_b200 import scenes
    dens = scenes.sdf_sphere_density(res)
    v = mr.VolumeRender(res)
    v.SetDatas(dens)
    v.Update()
    return mr, v, dens


@pytest.mark.parametrize("ior", [-1.0, 1.33])
@pytest.mark.parametrize("precision", [0, 1])
def test_marching_matches_oracle(ior, precision):
    from internship_b200 import _lib, scenes
    from internship_b200.weights import active_random_weights
    mr, v, dens = _setup()
    w, st = active_random_weights(1), mr.builtin_stencil()
    v.SetWeights(w, st)
    _lib.check(_lib.load().mr_volume_set_surface_ior(v.handle, ior))
    md, mips, _ = orc.build_mips(dens)
    for k in range(3):
        p = scenes.make_params(24, 20, 1, rt=_lib.RT_MARCHING_MRPNN, alpha=32.0, sample_offset=k,
                               precision=precision)
        out = np.zeros(24 * 20 * 3, np.float32)
        _lib.check(_lib.load().mr_render_host(v.handle, v.network.handle, C.byref(p), out.ctypes.data))
        if k == 0:
            tr = np.concatenate([v.read(_lib.READ_TR, i) for i in range(8)])
            lut = v.read(_lib.READ_HGLUT)
        ref = orc.render_marching(dens, md, mips, tr, lut, w, st, orc.RenderParams.from_buffer_copy(p), ior)
        assert ref.max() > 0
        tol = 1e-3 if precision == 0 else 0.1
        close = np.abs(out - ref) <= tol * (np.abs(ref) + 1e-3) + 1e-6
        # the same streams; a rounding difference can move one reservoir pick or a surface bounce
        assert close.mean() > 0.85, (k, close.mean())
    v.close()


@pytest.mark.parametrize("name,ior", [("plain", -1.0), ("ior", 1.33)])
def test_marching_matches_reference(name, ior):
    """The reference's weights (read from its build) with the default
    stencil, against the reference's marching render: per-pixel z-scores with
    a pooled variance term (the pick of the network's point is heavy-tailed)
    and the image mean."""
    if not ref_py.available():
        pytest.skip("oracle/_ref not built")
    from internship_b200 import _lib, scenes
    import torch
    d = golden("ref_march.npz")
    n_ref = int(d["spp"])
    ref_mean = d[name + "_sum"] / n_ref
    ref_var = np.maximum(d[name + "_sumsq"] / n_ref - ref_mean ** 2, 0)
    mr, v, dens = _setup(128)
    v.SetWeights(ref_py.RefNet().read_weights(), None)
    _lib.check(_lib.load().mr_volume_set_surface_ior(v.handle, ior))
    p = scenes.make_params(32, 32, 1, rt=_lib.RT_MARCHING_MRPNN, alpha=float(d["alpha"]))
    K = 384
    acc = np.zeros(32 * 32 * 3)
    acc2 = np.zeros(32 * 32 * 3)
    out = torch.empty(32 * 32 * 3, device="cuda")
    for k in range(K):
        p.sample_offset = k
        _lib.check(_lib.load().mr_render(v.handle, v.network.handle, C.byref(p), C.c_void_p(out.data_ptr()), None))
        o = out.cpu().numpy().astype(np.float64)
        acc += o
        acc2 += o * o
    mean = acc / K
    var = np.maximum(acc2 / K - mean ** 2, 0)
    se = np.sqrt(ref_var / n_ref + var / K + (ref_var.mean() / n_ref + var.mean() / K))
    z = (mean - ref_mean) / (se + 1e-6)
    assert np.mean(np.abs(z) > 3) < 0.03, np.mean(np.abs(z) > 3)
    tot = np.sqrt((ref_var / n_ref + var / K).sum()) / ref_mean.size
    assert abs(mean.mean() - ref_mean.mean()) < 4 * tot + 5e-3 * abs(ref_mean.mean()), (mean.mean(), ref_mean.mean())
    v.close()
