"""Python mirror of the reference's host API for the cloud-rendering path.

`VolumeRender` and `Camera` keep the names, argument order and meaning of
core/volume.hpp:45-146 and core/camera.hpp:10-41; every call goes through the
C ABI of libmrpnn_b200.so. Images are numpy arrays (H, W, 3) float32,
row-major, top row first.
"""
import ctypes as C
import os

import numpy as np

from . import _lib
from ._lib import MRError, RenderParams, check, f3

PT, RPNN, MRPNN = _lib.RT_PT, _lib.RT_RPNN, _lib.RT_MRPNN


def read_volume_file(path):
    """The density grid of a volume file (.bin / .txt / .vox, resolved as
    VolumeRender(string) resolves it), parsed on the host: (r, r, r) float32."""
    L = _lib.load()
    r = C.c_int32()
    p = os.fsencode(path)
    check(L.mr_volume_file_read(p, None, 0, C.byref(r)))
    out = np.zeros(r.value ** 3, np.float32)
    check(L.mr_volume_file_read(p, out.ctypes.data, out.size, C.byref(r)))
    return out.reshape((r.value,) * 3)


def read_hdr(path):
    """load_hdr_float4 (core/hdr_loader.h:249): (h, w, 4) float32, alpha 0."""
    L = _lib.load()
    w, h = C.c_int32(), C.c_int32()
    p = os.fsencode(path)
    check(L.mr_hdr_read(p, None, 0, C.byref(w), C.byref(h)))
    out = np.zeros(w.value * h.value * 4, np.float32)
    check(L.mr_hdr_read(p, out.ctypes.data, out.size, C.byref(w), C.byref(h)))
    return out.reshape(h.value, w.value, 4)


def builtin_stencil():
    """The default stencil: the reference's 160 directions (core/vector.cu:77-172)."""
    out = np.zeros(480, np.float32)
    check(_lib.load().mr_builtin_stencil(out.ctypes.data, out.size))
    return out


def spiral_stencil():
    """The library's golden-angle stencil in the same shell layout (opt-in)."""
    out = np.zeros(480, np.float32)
    check(_lib.load().mr_spiral_stencil(out.ctypes.data, out.size))
    return out


def xavier_weights(seed=1, bias_range=None):
    """Xavier-uniform initial weights in the NNWeight.cuh blob layout (zero
    biases). With bias_range=(lo, hi) the biases are drawn uniformly from it
    (numpy generator seeded with `seed`), which keeps every ReLU of a random
    network active."""
    out = np.zeros(_lib.WEIGHT_TOTAL, np.float32)
    check(_lib.load().mr_weights_xavier(seed, out.ctypes.data, out.size))
    if bias_range is not None:
        from .weights import layout
        rng = np.random.default_rng(seed)
        off = 0
        for name, n in layout():
            if name.endswith("B"):
                out[off:off + n] = rng.uniform(bias_range[0], bias_range[1], n)
            off += n
    return out


class Network:
    """Radiance-predictor weights on the device (the NNWeight.cuh arrays)."""

    def __init__(self, weights, stencil=None):
        w = np.ascontiguousarray(weights, np.float32).ravel()
        st = None if stencil is None else np.ascontiguousarray(stencil, np.float32).ravel()
        if st is not None and st.size != 480:
            raise ValueError("stencil must have 160 x 3 values")
        h = C.c_void_p()
        check(_lib.load().mr_network_create(w.ctypes.data, w.size, None if st is None else st.ctypes.data,
                                            C.byref(h)))
        self.handle = h
        self.weights = w

    def close(self):
        if self.handle:
            _lib.load().mr_network_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class VolumeRender:
    """core/volume.hpp:45-146 on the B200 library."""

    PT, RPNN, MRPNN = PT, RPNN, MRPNN

    def __init__(self, resolution, write_cache=True):
        """VolumeRender(int resolution), or VolumeRender(string path)
        (core/volume.cu:835-911): a path loads <path>.bin, a .txt or a .vox
        file through mr_volume_load, which also runs Update()."""
        L = _lib.load()
        h = C.c_void_p()
        self.max_density = 0.00001
        if isinstance(resolution, (str, bytes, os.PathLike)):
            path = os.fsencode(resolution)
            check(L.mr_volume_load(path, 1 if write_cache else 0, C.byref(h), None))
            r = C.c_int32()
            check(L.mr_volume_resolution(h, C.byref(r)))
            self.resolution = r.value
            self.handle = h
            self.datas = self.read(_lib.READ_DENSITY).reshape((self.resolution,) * 3)
            md = C.c_float()
            check(L.mr_volume_max_density(h, C.byref(md)))
            self.max_density = md.value
        else:
            self.resolution = int(resolution)
            check(L.mr_volume_create(self.resolution, C.byref(h)))
            self.handle = h
            self.datas = np.zeros((self.resolution,) * 3, np.float32)
        self.scatter_rate = (1.001, 1.001, 1.001)  # core/render.cuh:16 default
        self.tr_scale = 1.0
        self.exposure = 1.0
        self.env_color = (0.0, 0.0, 0.0)
        self.network = None
        self.seed = 0
        self.checkerboard = False

    # -- data -------------------------------------------------------------
    def SetData(self, x, y, z, value):
        self.datas[x, y, z] = value

    def SetDatas(self, func_or_array):
        """Fill from an array (res^3, x-major) or func(x, y, z, u, v, w)
        evaluated on the grid with u = (x+0.5)/res (core/omp.cpp:4-18)."""
        r = self.resolution
        if callable(func_or_array):
            i = np.arange(r)
            x, y, z = np.meshgrid(i, i, i, indexing="ij")
            u, v, w = (x + 0.5) / r, (y + 0.5) / r, (z + 0.5) / r
            self.datas = np.asarray(func_or_array(x, y, z, u, v, w), np.float32).reshape(r, r, r)
        else:
            a = np.asarray(func_or_array, np.float32)
            if a.size != r ** 3:
                raise ValueError("expected %d values" % r ** 3)
            self.datas = a.reshape(r, r, r).copy()

    def Update(self):
        self.__dict__.pop("_levels", None)
        L = _lib.load()
        d = np.ascontiguousarray(self.datas, np.float32)
        check(L.mr_volume_set_data(self.handle, d.ctypes.data, d.size))
        check(L.mr_volume_update(self.handle, None))
        md = C.c_float()
        check(L.mr_volume_max_density(self.handle, C.byref(md)))
        self.max_density = md.value

    def Update_TR(self, lightDir, alpha=64.0):
        self.__dict__.pop("_levels", None)
        check(_lib.load().mr_volume_update_tr(self.handle, f3(lightDir), float(alpha), None))

    def UpdateHGLut(self, g):
        check(_lib.load().mr_volume_update_hglut(self.handle, float(g), self.seed, None))

    # -- settings (device globals of the reference become render params) ----
    def SetScatterRate(self, rate):
        self.scatter_rate = (rate,) * 3 if np.isscalar(rate) else tuple(float(r) for r in rate)

    def SetTrScale(self, scale):
        self.tr_scale = float(scale)

    def SetExposure(self, exp):
        self.exposure = float(exp)

    def SetEnvColor(self, color):
        self.env_color = tuple(float(c) for c in color)

    def SetHDRI(self, path_or_rgba):
        """SetHDRI (core/volume.cu:1426-1458): a Radiance .hdr path or an
        (h, w, 3|4) float array, row 0 straight up. The environment scale
        (SetEnvExp) becomes 1 unless one was set."""
        L = _lib.load()
        if isinstance(path_or_rgba, (str, bytes, os.PathLike)):
            check(L.mr_volume_load_hdri(self.handle, os.fsencode(path_or_rgba)))
        else:
            a = np.asarray(path_or_rgba, np.float32)
            if a.ndim != 3 or a.shape[2] not in (3, 4):
                raise ValueError("HDRI must be (h, w, 3) or (h, w, 4)")
            rgba = np.zeros(a.shape[:2] + (4,), np.float32)
            rgba[..., :a.shape[2]] = a
            check(L.mr_volume_set_hdri(self.handle, rgba.ctypes.data, rgba.shape[1], rgba.shape[0]))
        if not any(self.env_color):
            self.env_color = (1.0, 1.0, 1.0)

    def SetEnvExp(self, exp):
        """SetEnvExp: the scale of the environment map."""
        self.env_color = (float(exp),) * 3

    def SetWeights(self, weights, stencil=None):
        if self.network is not None:
            self.network.close()
        self.network = Network(weights, stencil)

    def SetSeed(self, seed):
        self.seed = int(seed)

    def SetSurfaceIOR(self, ior):
        """SetSurfaceIOR (core/volume.cu:1490-1493): the dielectric surface of
        MR_RT_MARCHING_MRPNN renders; <= 0 removes it."""
        check(_lib.load().mr_volume_set_surface_ior(self.handle, float(ior)))

    def SetCheckboard(self, on):
        """SetCheckboard: interactive delta tracking renders half the pixels
        per frame (RenderInteractive)."""
        self.checkerboard = bool(on)

    # -- host-side samplers of the tables (core/volume.cu:675-722,1495-1576) --
    def _level(self, what, level):
        key = (what, level)
        cache = self.__dict__.setdefault("_levels", {})
        if key not in cache:
            r = (256 if what != _lib.READ_TR else 128) >> level
            cache[key] = self.read(what, level).reshape(r, r, r)
        return cache[key]

    @staticmethod
    def _trilinear(data, uv, clamp):
        """Sample / SampleClamp (core/volume.cu:675-722): trilinear at
        uv * res - 1/2 over texels max(0, v), zero outside (or clamped)."""
        res = data.shape[0]
        uv = np.asarray(uv, np.float32)
        pos = uv * np.float32(res) - np.float32(0.5)
        i0 = np.floor(pos).astype(np.int64)
        w = (pos - i0).astype(np.float32)

        def at(dx, dy, dz):
            ix, iy, iz = i0[..., 0] + dx, i0[..., 1] + dy, i0[..., 2] + dz
            if clamp:
                ix, iy, iz = (np.clip(a, 0, res - 1) for a in (ix, iy, iz))
                ok = np.ones(ix.shape, bool)
            else:
                ok = (ix >= 0) & (iy >= 0) & (iz >= 0) & (ix < res) & (iy < res) & (iz < res)
            v = data[np.clip(ix, 0, res - 1), np.clip(iy, 0, res - 1), np.clip(iz, 0, res - 1)]
            return np.where(ok, np.maximum(v, 0.0), 0.0).astype(np.float32)

        def lerp(a, b, t):
            return a + (b - a) * t
        wx, wy, wz = w[..., 0], w[..., 1], w[..., 2]
        return lerp(lerp(lerp(at(0, 0, 0), at(0, 0, 1), wz), lerp(at(0, 1, 0), at(0, 1, 1), wz), wy),
                    lerp(lerp(at(1, 0, 0), at(1, 0, 1), wz), lerp(at(1, 1, 0), at(1, 1, 1), wz), wy), wx)

    def DensityAtUV(self, mip, uv):
        """DensityAtUV(int | float mip, uv): the density pyramid at uv in
        [0, 1]^3 (a fractional mip blends two levels)."""
        if isinstance(mip, (float, np.floating)) and float(mip) != int(mip):
            a = int(mip)
            t = np.float32(mip - a)
            return (self.DensityAtUV(a, uv) * (1 - t) + self.DensityAtUV(a + 1, uv) * t).astype(np.float32)
        return self._trilinear(self._level(_lib.READ_MIP, int(mip)), uv, False)

    def DensityAtPosition(self, mip, pos):
        """DensityAtPosition: DensityAtUV at pos + 1/2 (pos in [-1/2, 1/2]^3)."""
        return self.DensityAtUV(mip, np.asarray(pos, np.float32) + np.float32(0.5))

    def TrAtPosition(self, mip, pos, lightDir):
        """TrAtPosition: the transmittance pyramid at pos; outside the volume,
        at the volume entry towards the light, or 1 where that ray misses."""
        from .scenes import ray_box_offset_np
        pos = np.atleast_2d(np.asarray(pos, np.float32))
        data = self._level(_lib.READ_TR, int(mip))
        out = np.ones(len(pos), np.float32)
        inside = np.all((pos >= -0.5) & (pos <= 0.5), axis=1)
        if inside.any():
            out[inside] = self._trilinear(data, pos[inside] + np.float32(0.5), True)
        L = np.asarray(lightDir, np.float32)
        for k in np.nonzero(~inside)[0]:
            o = ray_box_offset_np(pos[k], L)
            if o >= 0:
                out[k] = self._trilinear(data, (pos[k] + np.float32(0.5) + L * np.float32(o))[None], True)[0]
        return out

    def VarianceAtUV(self, mip, uv):
        """VarianceAtUV (core/volume.cu:1533-1576), as the reference reads it:
        texel (x, y, z) at uv * res (truncated), the level indexed
        (z * res + y) * res + x, upper neighbours clamped, zero outside."""
        if mip < 0 or mip >= 9:
            return np.zeros(np.shape(uv)[:-1], np.float32)
        flat = self._level(_lib.READ_VARIANCE, int(mip)).ravel()
        res = 256 >> int(mip)
        pos = np.asarray(uv, np.float32) * np.float32(res)
        x0, y0, z0 = (pos[..., i].astype(np.int64) for i in range(3))
        x1, y1, z1 = (np.minimum(a + 1, res - 1) for a in (x0, y0, z0))
        fx, fy, fz = (pos[..., i] - p for i, p in enumerate((x0, y0, z0)))

        def gv(x, y, z):
            ok = (x >= 0) & (x < res) & (y >= 0) & (y < res) & (z >= 0) & (z < res)
            i = (np.clip(z, 0, res - 1) * res + np.clip(y, 0, res - 1)) * res + np.clip(x, 0, res - 1)
            return np.where(ok, flat[i], 0.0).astype(np.float32)
        c00 = gv(x0, y0, z0) * (1 - fx) + gv(x1, y0, z0) * fx
        c01 = gv(x0, y0, z1) * (1 - fx) + gv(x1, y0, z1) * fx
        c10 = gv(x0, y1, z0) * (1 - fx) + gv(x1, y1, z0) * fx
        c11 = gv(x0, y1, z1) * (1 - fx) + gv(x1, y1, z1) * fx
        return ((c00 * (1 - fy) + c10 * fy) * (1 - fz) + (c01 * (1 - fy) + c11 * fy) * fz).astype(np.float32)

    # -- queries ------------------------------------------------------------
    def read(self, what, level=0):
        L = _lib.load()
        if what == _lib.READ_DENSITY:
            n = self.resolution ** 3
        elif what in (_lib.READ_MIP, _lib.READ_VARIANCE):
            n = (256 >> level) ** 3
        elif what == _lib.READ_TR:
            n = (128 >> level) ** 3
        else:
            n = 512 * 512
        out = np.zeros(n, np.float32)
        check(L.mr_volume_read(self.handle, what, level, out.ctypes.data, n))
        return out

    def params(self, size, ori, up, right, lightDir, rt=PT, g=0.857, alpha=1.0, lightColor=(1, 1, 1),
               multiScatter=512, sampleNum=1024, sample_offset=0, precision=_lib.PREC_FP32):
        p = RenderParams()
        p.width, p.height = int(size[0]), int(size[1])
        p.ori, p.up, p.right = f3(ori), f3(up), f3(right)
        p.light_dir, p.light_color = f3(lightDir), f3(lightColor)
        p.alpha, p.g = float(alpha), float(g)
        p.scatter_rate = f3(self.scatter_rate)
        p.tr_scale = self.tr_scale
        p.env_color = f3(self.env_color)
        p.max_bounces, p.spp = int(multiScatter), int(sampleNum)
        p.seed, p.sample_offset = self.seed, int(sample_offset)
        p.render_type, p.precision = int(rt), int(precision)
        return p

    def Render(self, size, ori, up, right, lightDir, rt=PT, g=0.857, alpha=1.0, lightColor=(1, 1, 1),
               multiScatter=512, sampleNum=1024, precision=_lib.PREC_FP32):
        """core/volume.cu:410-467: returns the mean radiance image (H, W, 3).
        Neural renders average `sampleNum` primary samples."""
        L = _lib.load()
        w, h = int(size[0]), int(size[1])
        out = np.zeros((h, w, 3), np.float32)
        net = self.network.handle if self.network is not None else None
        if rt == PT:
            p = self.params(size, ori, up, right, lightDir, rt, g, alpha, lightColor, multiScatter, sampleNum,
                            precision=precision)
            check(L.mr_render_host(self.handle, net, C.byref(p), out.ctypes.data))
            return out
        acc = np.zeros_like(out, np.float64)
        for s in range(sampleNum):
            p = self.params(size, ori, up, right, lightDir, rt, g, alpha, lightColor, multiScatter, 1,
                            sample_offset=s, precision=precision)
            check(L.mr_render_host(self.handle, net, C.byref(p), out.ctypes.data))
            acc += out
        return (acc / sampleNum).astype(np.float32)

    def RenderInteractive(self, accum, hist, bgra, size, ori, up, right, lightDir, lightColor=(1, 1, 1), alpha=1.0,
                          multiScatter=512, g=0.857, randseed=0, rt=PT, toneType=2, denoise=False, prev=None,
                          stream=None):
        """The interactive Render(float3* accum, Histogram* hist, unsigned*
        bgra, ...) overload (core/volume.cu:469-547) into caller-owned device
        buffers (torch CUDA tensors: accum W*H*3 float32, hist W*H*33 float32,
        bgra W*H int32). randseed is the frame index (0 restarts the
        accumulation); prev = (ori, up, right) of the previous frame for the
        neural mode's reprojection. toneType 0 none, 1 gamma, 2 ACES."""
        L = _lib.load()
        p = self.params(size, ori, up, right, lightDir, rt, g, alpha, lightColor, multiScatter, 1,
                        sample_offset=randseed)
        it = _lib.Interactive()
        po, pu, pr = prev if prev is not None else (ori, up, right)
        it.prev_ori, it.prev_up, it.prev_right = f3(po), f3(pu), f3(pr)
        it.frame_index, it.checkerboard = int(randseed), 1 if self.checkerboard else 0
        it.tone, it.denoise, it.exposure = int(toneType), 1 if denoise else 0, float(self.exposure)
        net = self.network.handle if self.network is not None else None
        check(L.mr_render_interactive(self.handle, net, C.byref(p), C.byref(it), C.c_void_p(accum.data_ptr()),
                                      C.c_void_p(hist.data_ptr()), C.c_void_p(bgra.data_ptr()),
                                      None if stream is None else C.c_void_p(stream)))

    def GetSamples(self, points, dirs, lightDir, alpha, g, scatter, multiScatter=512, spp=1024, seed=0):
        """GetSamples (core/volume.cu:550-626, core/render.cuh:276-315): the
        multiple-scattering radiance at each point along its view direction
        (unit light, albedo `scatter`), the mean of `spp` paths accumulated in
        FP64 on the GPU. points, dirs: (n, 3); returns (n,) float64."""
        import torch
        pos = torch.as_tensor(np.ascontiguousarray(points, np.float32), device="cuda")
        dr = torch.as_tensor(np.ascontiguousarray(dirs, np.float32), device="cuda")
        n = pos.shape[0]
        acc = torch.zeros(n, dtype=torch.float64, device="cuda")
        check(_lib.load().mr_train_labels(self.handle, C.c_void_p(pos.data_ptr()), C.c_void_p(dr.data_ptr()), n,
                                          f3(lightDir), float(alpha), float(g), float(scatter), int(multiScatter),
                                          int(spp), int(seed), C.c_void_p(acc.data_ptr()), None))
        return (acc / spp).cpu().numpy()

    def close(self):
        if self.handle:
            _lib.load().mr_volume_destroy(self.handle)
            self.handle = None
        if self.network is not None:
            self.network.close()
            self.network = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- tone mapping and image output (core/camera.cu:10-160) --------------------
_SRGB_2_AP0 = np.array([[0.4397010, 0.3829780, 0.1773350], [0.0897923, 0.8134230, 0.0967616],
                        [0.0175440, 0.1115440, 0.8707040]], np.float64)
_AP0_2_AP1 = np.array([[1.4514393161, -0.2365107469, -0.2149285693], [-0.0765537734, 1.1762296998, -0.0996759264],
                       [0.0083161484, -0.0060324498, 0.9977163014]], np.float64)
_AP1_2_XYZ = np.array([[0.6624541811, 0.1340042065, 0.1561876870], [0.2722287168, 0.6740817658, 0.0536895174],
                       [-0.0055746495, 0.0040607335, 1.0103391003]], np.float64)
_XYZ_2_AP1 = np.array([[1.6410233797, -0.3248032942, -0.2364246952], [-0.6636628587, 1.6153315917, 0.0167563477],
                       [0.0117218943, -0.0082844420, 0.9883948585]], np.float64)
_D60_2_D65 = np.array([[0.98722400, -0.00611327, 0.0159533], [-0.00759836, 1.00186000, 0.0053302],
                       [0.00307257, -0.00509595, 1.0816800]], np.float64)
_XYZ_2_709 = np.array([[3.2409699419, -1.5373831776, -0.4986107603], [-0.9692436363, 1.8759675015, 0.0415550574],
                       [0.0556300797, -0.2039769589, 1.0569715142]], np.float64)
_AP1_Y = np.array([0.272229, 0.674082, 0.0536895])


def tone_gamma(c):
    return np.power(np.maximum(c, 0), 1.0 / 2.2)


def tone_none(c):
    return c


def tone_aces(c):
    """ACES RRT+ODT fit with dim-surround and desaturation steps
    (core/camera.cu:74-160 / core/render.cuh:640-732), on (..., 3) arrays."""
    c = np.asarray(c, np.float64)
    acescg = c @ (_AP0_2_AP1 @ _SRGB_2_AP0).T
    y = acescg @ _AP1_Y
    acescg = y[..., None] * (1 - 0.96) + acescg * 0.96
    x = acescg
    post = (x * (x * 278.5085 + 10.7772)) / (x * (x * 293.6045 + 88.7122) + 80.6889)
    xyz = post @ _AP1_2_XYZ.T
    div = np.maximum(xyz.sum(-1), 1e-4)
    xx, yy = xyz[..., 0] / div, xyz[..., 1] / div
    Y = np.minimum(np.maximum(xyz[..., 1], 0.0), 65504.0) ** 0.9811
    m = Y / np.maximum(yy, 1e-4)
    xyz = np.stack([xx * m, Y, (1.0 - xx - yy) * m], -1)
    lin = xyz @ _XYZ_2_AP1.T
    y = lin @ _AP1_Y
    lin = y[..., None] * (1 - 0.93) + lin * 0.93
    out = lin @ (_XYZ_2_709 @ _D60_2_D65 @ _AP1_2_XYZ).T
    return np.power(np.maximum(out, 0), 1.0 / 2.2).astype(np.float32)


def save_bmp(path, rgb8):
    """32-bit top-down BMP (core/camera.cu:10-64); `path` gets ".bmp" appended."""
    h, w, _ = rgb8.shape
    bgra = np.empty((h, w, 4), np.uint8)
    bgra[..., 0], bgra[..., 1], bgra[..., 2], bgra[..., 3] = rgb8[..., 2], rgb8[..., 1], rgb8[..., 0], 255
    header = bytearray(54)
    header[0:2] = b"BM"
    header[2:6] = int(w * h * 4 + 54).to_bytes(4, "little")
    header[10] = 0x36
    header[14] = 0x28
    header[18:22] = int(w).to_bytes(4, "little", signed=True)
    header[22:26] = int(-h).to_bytes(4, "little", signed=True)
    header[26] = 1
    header[28] = 32
    header[34:38] = int(w * h * 4).to_bytes(4, "little")
    with open(path + ".bmp", "wb") as f:
        f.write(bytes(header))
        f.write(bgra.tobytes())


class Camera:
    """core/camera.hpp:10-41: position on a sphere around the volume, 90 degree
    field of view (unit right/up) unless `fov_deg` is given."""

    def __init__(self, volume, name="test camera", position=(0.75, 0.75, 0.75), resolution=512, fov_deg=90.0):
        self.volume = volume
        self.name = name
        self.resolution = int(resolution)
        self.fov_deg = float(fov_deg)
        self.SetPosition(position)

    def SetPosition(self, position):
        ori = np.asarray(position, np.float64)
        fwd = -ori / np.linalg.norm(ori)
        right = np.cross([0.0, 1.0, 0.0], fwd)
        right /= np.linalg.norm(right)
        up = np.cross(fwd, right)
        if ori[0] == 0 and ori[2] == 0:  # core/camera.cu:178-188
            right = np.array([1.0, 0, 0])
            up = np.array([0, 0, 1.0]) if ori[1] > 0 else np.array([0, 0, -1.0])
        self.ori, self.forward, self.right, self.up = ori, fwd, right, up

    def GetPosition(self):
        return self.ori

    def _scaled(self):
        s = np.tan(np.radians(self.fov_deg) / 2)
        return self.up * s, self.right * s

    def Render(self, lightDir, lightColor=(1, 1, 1), alpha=1.0, multiScatter=1, g=0.0, sampleNum=1, rt=PT):
        up, right = self._scaled()
        return self.volume.Render((self.resolution, self.resolution), self.ori, up, right, lightDir, rt, g, alpha,
                                  lightColor, multiScatter, sampleNum)

    def RenderToFile(self, path, lightDir, lightColor=(1, 1, 1), alpha=1.0, multiScatter=1, g=0.0, sampleNum=1,
                     tone=tone_aces, rt=PT, exp=1.0):
        img = self.Render(lightDir, lightColor, alpha, multiScatter, g, sampleNum, rt)
        t = np.clip(tone(img * exp), 0.0, 1.0)
        save_bmp(path, (t * 255).astype(np.uint8))
        return img
