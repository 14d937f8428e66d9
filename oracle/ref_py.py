"""ctypes bindings of the reference harness libraries in oracle/_ref/ --
test infrastructure only. Both libraries run the reference's own device code
on the GPU; they exist only where oracle.build.build_reference() ran."""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libref_mrpnn.so")
INJ_SO = os.path.join(HERE, "_ref", "libref_net_inj.so")
VOL_SO = os.path.join(HERE, "_ref", "libref_volume.so")

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def available():
    return os.path.exists(REF_SO) and os.path.exists(INJ_SO)


class Ref:
    """The reference renderer (core/render.cuh, core/radiancePredict.cu)."""

    def __init__(self):
        L = C.CDLL(REF_SO)
        L.ref_setup.argtypes = [f32p, C.c_int, C.c_float, f32p, f32p, f32p, f32p, f32p, C.c_float]
        L.ref_render.argtypes = [C.c_int, C.c_int, C.c_int, f32p, f32p, f32p, f32p, f32p, C.c_float, C.c_int,
                                 C.c_float, C.c_int, f64p, f64p]
        L.ref_predict_frames.argtypes = [C.c_int, f32p, f32p, f32p, C.c_float, C.c_float, f32p, f32p]
        L.ref_load_weights.argtypes = [f32p, C.c_long]
        L.ref_read_weights.argtypes = [f32p, C.c_long]
        L.ref_read_stencil.argtypes = [f32p]
        L.ref_set_ior.argtypes = [C.c_float]
        self.L = L

    def setup(self, density, max_density, mips, tr, lut, env=(0, 0, 0), scatter=(0.99,) * 3, tr_scale=1.0):
        d = np.ascontiguousarray(density, np.float32).ravel()
        res = round(d.size ** (1 / 3))
        rc = self.L.ref_setup(d, res, float(max_density), np.ascontiguousarray(mips, np.float32),
                              np.ascontiguousarray(tr, np.float32), np.ascontiguousarray(lut, np.float32),
                              np.asarray(env, np.float32), np.asarray(scatter, np.float32), float(tr_scale))
        assert rc == 0, "ref_setup failed"

    def render(self, mode, w, h, ori, up, right, light, light_color, alpha, bounces, g, spp):
        s = np.zeros(w * h * 3, np.float64)
        s2 = np.zeros(w * h * 3, np.float64)
        a = lambda v: np.asarray(v, np.float32)
        rc = self.L.ref_render(mode, w, h, a(ori), a(up), a(right), a(light), a(light_color), float(alpha),
                               int(bounces), float(g), int(spp), s, s2)
        assert rc == 0, "ref_render failed"
        return s, s2

    def set_ior(self, ior):
        assert self.L.ref_set_ior(float(ior)) == 0

    def predict_frames(self, pos, frame, light, alpha, g, scatterrate):
        n = len(pos)
        out = np.zeros(3 * n, np.float32)
        rc = self.L.ref_predict_frames(n, np.ascontiguousarray(pos, np.float32).ravel(),
                                       np.ascontiguousarray(frame, np.float32).ravel(), np.asarray(light, np.float32),
                                       float(alpha), float(g), np.asarray(scatterrate, np.float32), out)
        assert rc == 0
        return out.reshape(n, 3)

    def load_weights(self, blob):
        assert self.L.ref_load_weights(np.ascontiguousarray(blob, np.float32), blob.size) == 0

    def read_weights(self):
        out = np.zeros(49673, np.float32)
        assert self.L.ref_read_weights(out, out.size) == 0
        return out

    def read_stencil(self):
        out = np.zeros(480, np.float32)
        assert self.L.ref_read_stencil(out) == 0
        return out


class RefNet:
    """The reference network on injected descriptor values (ref_inject.cu)."""

    def __init__(self):
        L = C.CDLL(INJ_SO)
        L.ref_inject_predict.argtypes = [C.c_int, f32p, f32p, f32p, C.c_float, f32p, f32p]
        L.ref_load_weights.argtypes = [f32p, C.c_long]
        L.ref_read_weights.argtypes = [f32p, C.c_long]
        self.L = L

    def load_weights(self, blob):
        assert self.L.ref_load_weights(np.ascontiguousarray(blob, np.float32), blob.size) == 0

    def read_weights(self):
        out = np.zeros(49673, np.float32)
        assert self.L.ref_read_weights(out, out.size) == 0
        return out

    def predict(self, raw, frame, light, g, scatterrate):
        n = len(raw)
        out = np.zeros(3 * n, np.float32)
        rc = self.L.ref_inject_predict(n, np.ascontiguousarray(raw, np.float32).ravel(),
                                       np.ascontiguousarray(frame, np.float32).ravel(), np.asarray(light, np.float32),
                                       float(g), np.asarray(scatterrate, np.float32), out)
        assert rc == 0
        return out.reshape(n, 3)


def raw_to_desc(raw, frame, light, g):
    """The descriptor the reference network sees for injected raw values
    (ref_inject.cu): density log(1+rho), transmittance as is, phase
    log(HG0+1) for i >= 1 and log(HG(X.L, g)+1) for i = 0."""
    raw = np.asarray(raw, np.float32)
    desc = np.empty_like(raw)
    desc[:, :192] = np.log(np.float32(1) + raw[:, :192])
    desc[:, 192:384] = raw[:, 192:384]
    desc[:, 385:576] = np.log(raw[:, 385:576] + np.float32(1))
    X = np.asarray(frame, np.float32)[:, 0:3]
    L = np.asarray(light, np.float32)
    c = (X * L).sum(1, dtype=np.float32)
    g2 = np.float32(g) * np.float32(g)
    d = np.float32(1) + g2 - np.float32(2) * np.float32(g) * c
    hg = ((np.float32(1) - g2) / (d * np.sqrt(d))) * np.float32(0.25)
    desc[:, 384] = np.log(hg + np.float32(1))
    return desc


def _f(v):
    return np.ascontiguousarray(v, np.float32).ravel()


class RefVolume:
    """The reference's VolumeRender and its table kernels (ref_volume.cu):
    Update, Fill_TR, Fill_Hg, Denoise, GetSamples, the interactive Render and
    SaveBMP, all the reference's own code."""

    def __init__(self, res=None):
        L = C.CDLL(VOL_SO)
        L.refv_create.argtypes = [C.c_int]
        L.refv_create.restype = C.c_void_p
        L.refv_destroy.argtypes = [C.c_void_p]
        L.refv_set_density_update.argtypes = [C.c_void_p, f32p, C.POINTER(C.c_float)]
        L.refv_set_scalars.argtypes = [C.c_void_p, C.c_float, f32p, C.c_float, f32p]
        L.refv_fill_tr.argtypes = [f32p, C.c_float, f32p, f32p]
        L.refv_fill_hg.argtypes = [C.c_float, C.c_int, f32p, f32p]
        L.refv_denoise.argtypes = [f32p, f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, u32p,
                                   C.POINTER(C.c_float)]
        L.refv_get_samples.argtypes = [C.c_void_p, C.c_int, f32p, f32p, f32p, C.c_float, C.c_float, C.c_float,
                                       C.c_int, C.c_int, C.c_int, f32p]
        L.refv_interactive.argtypes = [C.c_void_p, C.c_int, C.c_int, f32p, f32p, f32p, f32p, f32p, C.c_float, C.c_int,
                                       C.c_float, C.c_int, C.c_int, C.c_int, f32p, f32p, u32p]
        L.refv_save_bmp.argtypes = [u8p, C.c_int, C.c_int, C.c_char_p]
        L.refv_tone_host.argtypes = [C.c_int, f32p, C.c_int, f32p]
        L.refv_load_hdr.argtypes = [C.c_char_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.refv_set_hdri.argtypes = [C.c_void_p, C.c_char_p, C.c_float]
        L.refv_render_pt.argtypes = [C.c_void_p, C.c_int, C.c_int, f32p, f32p, f32p, f32p, f32p, C.c_float, C.c_int,
                                     C.c_float, C.c_int, f32p]
        L.refv_datagen_samples.argtypes = [C.c_void_p, f32p, C.c_float, C.c_float, C.c_int, f32p, f32p]
        self.L = L
        self.h = None
        self.res = res
        if res is not None:
            self.h = L.refv_create(int(res))

    def close(self):
        if self.h:
            self.L.refv_destroy(self.h)
            self.h = None

    def set_density(self, density):
        md = C.c_float()
        assert self.L.refv_set_density_update(self.h, _f(density), C.byref(md)) == 0
        return md.value

    def set_scalars(self, tr_scale=1.0, scatter=(0.99,) * 3, env_exp=1.0, env=(0, 0, 0)):
        assert self.L.refv_set_scalars(self.h, float(tr_scale), _f(scatter), float(env_exp), _f(env)) == 0

    def fill_tr(self, mips, alpha, light):
        out = np.zeros(sum((128 >> k) ** 3 for k in range(8)), np.float32)
        assert self.L.refv_fill_tr(_f(mips), float(alpha), _f(light), out) == 0
        return out

    def fill_hg(self, g, randnum=0):
        lut = np.zeros(512 * 512, np.float32)
        bn = np.zeros(512 * 512, np.float32)
        assert self.L.refv_fill_hg(float(g), int(randnum), lut, bn) == 0
        return lut, bn

    def denoise(self, accum, hist, w, h, frame, flip, tone, denoise, exposure=1.0, timed=False):
        """Packed output; with timed=True also the kernel's device time in ms."""
        out = np.zeros(w * h, np.uint32)
        ms = C.c_float(0.0)
        assert self.L.refv_denoise(_f(accum), _f(hist), w, h, int(frame), int(flip), int(tone), int(denoise),
                                   float(exposure), out, C.byref(ms)) == 0
        return (out, ms.value) if timed else out

    def get_samples(self, pos, dirs, light, alpha, g, scatter, bounces, spp, randnum=0):
        n = len(pos)
        out = np.zeros(3 * n, np.float32)
        assert self.L.refv_get_samples(self.h, n, _f(pos), _f(dirs), _f(light), float(alpha), float(g), float(scatter),
                                       int(bounces), int(spp), int(randnum), out) == 0
        return out.reshape(n, 3)

    def interactive(self, w, h, ori, up, right, light, light_color, alpha, bounces, g, frames, tone=2, denoise=1):
        acc = np.zeros(w * h * 3, np.float32)
        hist = np.zeros(w * h * 33, np.float32)
        bgra = np.zeros(w * h, np.uint32)
        assert self.L.refv_interactive(self.h, w, h, _f(ori), _f(up), _f(right), _f(light), _f(light_color),
                                       float(alpha), int(bounces), float(g), int(frames), int(tone), int(denoise),
                                       acc, hist, bgra) == 0
        return acc, hist, bgra

    def save_bmp(self, rgba, w, h, path):
        assert self.L.refv_save_bmp(np.ascontiguousarray(rgba, np.uint8).ravel(), w, h, path.encode()) == 0
        return path + ".bmp"

    def tone_host(self, rgb, tone):
        rgb = _f(rgb)
        out = np.zeros_like(rgb)
        assert self.L.refv_tone_host(rgb.size // 3, rgb, int(tone), out) == 0
        return out.reshape(-1, 3)

    def datagen_samples(self, mip0, max_density, alpha, n):
        """dataGen's GetDesiredCountSample(v, S, n, alpha, alpha) over the
        given 256^3 mip level 0: (pos n x 3, view n x 3)."""
        pos = np.zeros(3 * n, np.float32)
        view = np.zeros(3 * n, np.float32)
        m = self.L.refv_datagen_samples(self.h, _f(mip0), float(max_density), float(alpha), int(n), pos, view)
        return pos.reshape(n, 3)[:m], view.reshape(n, 3)[:m]

    def load_hdr(self, path):
        w, h = C.c_int(), C.c_int()
        assert self.L.refv_load_hdr(path.encode(), None, 0, C.byref(w), C.byref(h)) == 0, "load_hdr_float4 failed"
        out = np.zeros(w.value * h.value * 4, np.float32)
        assert self.L.refv_load_hdr(path.encode(), out.ctypes.data, out.size, C.byref(w), C.byref(h)) == 0
        return out.reshape(h.value, w.value, 4)

    def set_hdri(self, path, env_exp=1.0):
        assert self.L.refv_set_hdri(self.h, path.encode(), float(env_exp)) == 0

    def render_pt(self, w, h, ori, up, right, light, light_color, alpha, bounces, g, spp):
        out = np.zeros(w * h * 3, np.float32)
        assert self.L.refv_render_pt(self.h, w, h, _f(ori), _f(up), _f(right), _f(light), _f(light_color),
                                     float(alpha), int(bounces), float(g), int(spp), out) == 0
        return out
