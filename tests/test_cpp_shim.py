"""The C++ host interface (include/mrpnn.hpp): it compiles and links against
the library on CPU, and on the GPU it renders exactly what the C ABI renders
for the same request."""
import os
import struct
import subprocess

import numpy as np
import pytest

from conftest import ROOT

PKG = os.path.join(ROOT, "internship_b200")


def build_demo(tmp):
    exe = os.path.join(tmp, "shim_demo")
    cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"),
           os.path.join(ROOT, "tests", "cpp", "shim_demo.cpp"), "-L", PKG, "-lmrpnn_b200", "-Wl,-rpath," + PKG,
           "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_shim_compiles_and_links(tmp_path):
    build_demo(str(tmp_path))


@pytest.mark.gpu
def test_shim_renders_like_the_c_abi(tmp_path):
    import ctypes as C
    import internship_b200 as mr
    from internship_b200 import _lib
    exe = build_demo(str(tmp_path))
    pt_f, nn_f, bmp = (str(tmp_path / n) for n in ("pt.f32", "nn.f32", "demo"))
    r = subprocess.run([exe, pt_f, nn_f, bmp], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    pt = np.fromfile(pt_f, np.float32)
    nn = np.fromfile(nn_f, np.float32)
    # the same requests through the Python binding of the C ABI
    res = 64
    g = (np.arange(res) + 0.5) / res
    u, v, w = np.meshgrid(g, g, g, indexing="ij")
    dens = (((u - 0.5) ** 2 + (v - 0.5) ** 2 + (w - 0.5) ** 2) < 0.25 ** 2).astype(np.float32)
    vol = mr.VolumeRender(res)
    vol.SetDatas(dens)
    vol.Update()
    p = _lib.RenderParams()
    p.width, p.height = 48, 32
    p.ori, p.up, p.right = _lib.f3((0, 0, 2)), _lib.f3((0, 0.4, 0)), _lib.f3((0.4, 0, 0))
    p.light_dir, p.light_color = _lib.f3((0.3, 0.8, 0.52)), _lib.f3((1, 1, 1))
    p.alpha, p.g, p.scatter_rate, p.tr_scale = 16.0, 0.857, _lib.f3((0.99, 0.99, 0.99)), 1.0
    p.max_bounces, p.spp, p.seed = 64, 16, 0
    ref = np.zeros(48 * 32 * 3, np.float32)
    _lib.check(_lib.load().mr_render_host(vol.handle, None, C.byref(p), ref.ctypes.data))
    # samples are summed with float atomics, in no fixed order
    np.testing.assert_allclose(pt, ref, rtol=1e-6, atol=1e-7)
    vol.SetWeights(mr.xavier_weights(1))
    p.render_type, p.spp = _lib.RT_MRPNN, 1
    acc = np.zeros_like(ref)
    for k in range(2):
        p.sample_offset = k
        img = np.zeros_like(ref)
        _lib.check(_lib.load().mr_render_host(vol.handle, vol.network.handle, C.byref(p), img.ctypes.data))
        acc += (img - acc) / (k + 1)
    np.testing.assert_allclose(nn, acc, rtol=1e-6, atol=1e-7)
    vol.close()
    data = open(bmp + ".bmp", "rb").read()
    assert data[:2] == b"BM" and len(data) == 54 + 40 * 40 * 4
    w, h = struct.unpack("<ii", data[18:26])
    assert (w, h) == (40, -40)
    px = np.frombuffer(data[54:], np.uint8).reshape(40, 40, 4)
    assert np.all(px[..., 3] == 255) and px[..., :3].max() > 0
