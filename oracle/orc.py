"""ctypes bindings of the CPU oracle (oracle/liborc.so) -- test infrastructure only."""
import ctypes as C
import os

import numpy as np

from .build import build_oracle

_lib = None

f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")


class Float3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class RenderParams(C.Structure):
    """Mirror of mr_render_params (include/mrpnn_b200.h)."""
    _fields_ = [("width", C.c_int32), ("height", C.c_int32),
                ("ori", Float3), ("up", Float3), ("right", Float3),
                ("light_dir", Float3), ("light_color", Float3),
                ("alpha", C.c_float), ("g", C.c_float), ("scatter_rate", Float3),
                ("tr_scale", C.c_float), ("env_color", Float3),
                ("max_bounces", C.c_int32), ("spp", C.c_int32),
                ("seed", C.c_uint32), ("sample_offset", C.c_uint32),
                ("render_type", C.c_int32), ("precision", C.c_int32), ("sampler", C.c_int32)]


def lib():
    global _lib
    if _lib is None:
        path = build_oracle()
        L = C.CDLL(path)
        L.orc_philox.argtypes = [u32p, u32p, u32p]
        L.orc_weights_xavier.argtypes = [C.c_uint32, f32p]
        L.orc_render_neural_dist.argtypes = [f32p, C.c_int, C.c_float, f32p, f32p, f32p, f32p, f32p,
                                             C.c_void_p, C.c_int, C.c_int, f32p, f32p, C.c_int]
        L.orc_render_marching.argtypes = [f32p, C.c_int, C.c_float, f32p, f32p, f32p, f32p, f32p,
                                          C.c_void_p, C.c_float, C.c_int, C.c_int, f32p, C.c_int]
        L.orc_reproject.argtypes = [C.c_void_p, f32p, f32p, f32p, C.c_int, C.c_int, f32p, f32p, f32p, f32p]
        L.orc_set_env.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_select_env_light.argtypes = [C.c_void_p, f32p, f32p]
        L.orc_uniforms.argtypes = [C.c_uint32] * 4 + [C.c_int, f32p]
        L.orc_hg.argtypes = [C.c_float, C.c_float]
        L.orc_hg.restype = C.c_float
        L.orc_hg_sample_cos.argtypes = [C.c_float, C.c_float]
        L.orc_hg_sample_cos.restype = C.c_float
        L.orc_hg_sample_dir.argtypes = [C.c_float, C.c_float, f32p, C.c_float, f32p]
        L.orc_ray_box_offset.argtypes = [f32p, f32p]
        L.orc_ray_box_offset.restype = C.c_float
        L.orc_ray_box_distance.argtypes = [f32p, f32p]
        L.orc_ray_box_distance.restype = C.c_float
        L.orc_stencil_info.argtypes = [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_sample_border.argtypes = [f32p, C.c_int, f32p]
        L.orc_sample_border.restype = C.c_float
        L.orc_sample_clamp.argtypes = [f32p, C.c_int, f32p]
        L.orc_sample_clamp.restype = C.c_float
        L.orc_sample_lut.argtypes = [f32p, C.c_float, C.c_float]
        L.orc_sample_lut.restype = C.c_float
        L.orc_build_mips.argtypes = [f32p, C.c_int, f32p, f32p, C.c_int]
        L.orc_build_mips.restype = C.c_float
        L.orc_build_tr.argtypes = [f32p, C.c_float, f32p, f32p, C.c_int]
        L.orc_build_hglut.argtypes = [C.c_float, C.c_uint32, f32p, C.c_int]
        L.orc_hglut_texels.argtypes = [C.c_float, i32p, f32p, C.c_int, f32p, C.c_int]
        L.orc_render_pt.argtypes = [f32p, C.c_int, C.c_float, C.c_void_p, C.c_int,
                                    C.c_int, f64p, f64p, u64p, C.c_int]
        L.orc_render_neural.argtypes = [f32p, C.c_int, C.c_float, f32p, f32p, f32p, f32p, f32p,
                                        C.c_void_p, C.c_int, C.c_int, f32p, C.c_int]
        L.orc_gather.argtypes = [f32p, f32p, f32p, f32p, f32p, f32p, C.c_int, C.c_float,
                                 C.c_float, f32p, f32p, f32p, f32p]
        L.orc_predict.argtypes = [f32p, f32p, f32p, C.c_int, f32p]
        L.orc_get_samples.argtypes = [f32p, C.c_int, C.c_float, f32p, f32p, f32p, f32p, f32p,
                                      f32p, C.c_int, C.c_int, C.c_int, C.c_uint32, f64p, C.c_int]
        L.orc_train_points.argtypes = [f32p, C.c_int, C.c_float, C.c_float, C.c_float, C.c_uint32, C.c_int,
                                       C.c_int, f32p, f32p]
        L.orc_train_points.restype = C.c_int
        L.orc_train_frames.argtypes = [f32p, C.c_int, f32p, C.c_uint32, f32p]
        L.orc_train_loss.argtypes = [f32p, f32p, f32p, f32p, C.c_int]
        L.orc_train_loss.restype = C.c_double
        L.orc_histogram_frame.argtypes = [f32p, C.c_int, C.c_int, f32p, f32p]
        L.orc_denoise.argtypes = [f32p, f32p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float, u32p]
        _lib = L
    return _lib


def nthreads():
    return int(os.environ.get("MRPNN_ORACLE_THREADS", os.cpu_count() or 1))


def f3(v):
    return Float3(float(v[0]), float(v[1]), float(v[2]))


def _a(x, dt=np.float32):
    return np.ascontiguousarray(np.asarray(x, dtype=dt))


MIP_SIZES = [(256 >> k) ** 3 for k in range(9)]
TR_SIZES = [(128 >> k) ** 3 for k in range(8)]
MIP_TOTAL = sum(MIP_SIZES)
TR_TOTAL = sum(TR_SIZES)


def philox(ctr, key):
    out = np.zeros(4, np.uint32)
    lib().orc_philox(_a(ctr, np.uint32), _a(key, np.uint32), out)
    return out


def uniforms(seed, a, b, tag, n):
    out = np.zeros(n, np.float32)
    lib().orc_uniforms(seed, a, b, tag, n, out)
    return out


def set_env(rgba=None):
    """Environment map (h, w, 4) for the trackers; None clears it."""
    global _env_keep
    if rgba is None:
        lib().orc_set_env(None, 0, 0)
        _env_keep = None
        return
    a = np.ascontiguousarray(rgba, np.float32)
    _env_keep = a
    lib().orc_set_env(a.ctypes.data, a.shape[1], a.shape[0])


_env_keep = None


def select_env_light(params):
    """(light_dir, light_color) of neural pass params.sample_offset with the
    environment map set."""
    ld = np.zeros(3, np.float32)
    lc = np.zeros(3, np.float32)
    lib().orc_select_env_light(C.addressof(params), ld, lc)
    return ld, lc


def xavier_weights(seed):
    """The benchmark network's Xavier(seed) weights in the blob layout."""
    out = np.zeros(49673, np.float32)
    lib().orc_weights_xavier(int(seed), out)
    return out


def reference_stencil():
    """The reference's 160 stencil directions (core/vector.cu:77-172), read
    from the table the library is compiled with."""
    import re
    txt = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "internship_b200", "csrc",
                            "mr_ref_stencil.inc")).read()
    body = txt[txt.index("{") + 1:txt.index("}")]
    vals = np.array([float(t.rstrip("f")) for t in re.findall(r"-?[0-9.]+(?:e[-+]?[0-9]+)?f", body)], np.float32)
    assert vals.size == 480
    return vals


def build_mips(density):
    density = _a(density)
    res = round(density.size ** (1 / 3))
    mips = np.zeros(MIP_TOTAL, np.float32)
    var = np.zeros(MIP_TOTAL, np.float32)
    md = lib().orc_build_mips(density.ravel(), res, mips, var, nthreads())
    return float(md), mips, var


def build_tr(mips, alpha, light):
    tr = np.zeros(TR_TOTAL, np.float32)
    lib().orc_build_tr(_a(mips), float(alpha), _a(light), tr, nthreads())
    return tr


def build_hglut(g, seed):
    lut = np.zeros(512 * 512, np.float32)
    lib().orc_build_hglut(float(g), int(seed), lut, nthreads())
    return lut


def hglut_texels(g, texel, bn):
    """Fill_Hg's estimator at texels `texel` (i + 512 j) with offsets `bn`."""
    texel = np.ascontiguousarray(texel, np.int32)
    bn = np.ascontiguousarray(bn, np.float32)
    out = np.zeros(texel.size, np.float32)
    lib().orc_hglut_texels(float(g), texel, bn, texel.size, out, nthreads())
    return out


def render_pt(density, max_density, params, row0=0, row1=None):
    density = _a(density)
    res = round(density.size ** (1 / 3))
    n = params.width * params.height * 3
    s = np.zeros(n, np.float64)
    s2 = np.zeros(n, np.float64)
    cnt = np.zeros(2, np.uint64)
    lib().orc_render_pt(density.ravel(), res, float(max_density), C.addressof(params), row0,
                        params.height if row1 is None else row1, s, s2, cnt, nthreads())
    return s, s2, cnt


def render_neural(density, max_density, mips, tr, lut, weights, stencil, params, row0=0, row1=None):
    density = _a(density)
    res = round(density.size ** (1 / 3))
    out = np.zeros(params.width * params.height * 3, np.float32)
    lib().orc_render_neural(density.ravel(), res, float(max_density), _a(mips), _a(tr), _a(lut),
                            _a(weights), _a(stencil), C.addressof(params), row0,
                            params.height if row1 is None else row1, out, nthreads())
    return out


def render_neural_dist(density, max_density, mips, tr, lut, weights, stencil, params):
    """Neural render plus each pixel's first-hit distance (< 0: no medium)."""
    density = _a(density)
    res = round(density.size ** (1 / 3))
    n = params.width * params.height
    out = np.zeros(n * 3, np.float32)
    dist = np.zeros(n, np.float32)
    lib().orc_render_neural_dist(density.ravel(), res, float(max_density), _a(mips), _a(tr), _a(lut), _a(weights),
                                 _a(stencil), C.addressof(params), 0, params.height, out, dist, nthreads())
    return out, dist


def render_marching(density, max_density, mips, tr, lut, weights, stencil, params, ior=-1.0):
    """NNPredict<Type::marching_MRPNN> render (surface index of refraction ior)."""
    density = _a(density)
    res = round(density.size ** (1 / 3))
    out = np.zeros(params.width * params.height * 3, np.float32)
    lib().orc_render_marching(density.ravel(), res, float(max_density), _a(mips), _a(tr), _a(lut), _a(weights),
                              _a(stencil), C.addressof(params), float(ior), 0, params.height, out, nthreads())
    return out


def reproject(params, prev_ori, prev_up, prev_right, fnum, checker, rad, dist, hist):
    """One interactive neural frame's reprojection + ReprojectionDenoise:
    returns the blended colour (n x 3); `hist` (n x 33 float32, contiguous) is
    updated in place."""
    accum = np.zeros(params.width * params.height * 3, np.float32)
    lib().orc_reproject(C.addressof(params), _a(prev_ori), _a(prev_up), _a(prev_right), int(fnum), int(checker),
                        _a(rad).ravel(), _a(dist).ravel(), hist.ravel(), accum)
    return accum


def gather(mips, tr, lut, stencil, pos, frame, alpha, g, scatter, light):
    n = len(pos)
    desc = np.zeros((n, 576), np.float32)
    aux = np.zeros((n, 5), np.float32)
    lib().orc_gather(_a(mips), _a(tr), _a(lut), _a(stencil), _a(pos).ravel(), _a(frame).ravel(), n,
                     float(alpha), float(g), _a(scatter), _a(light), desc.ravel(), aux.ravel())
    return desc, aux


def predict(weights, desc, aux):
    n = len(desc)
    out = np.zeros((n, 3), np.float32)
    lib().orc_predict(_a(weights), _a(desc).ravel(), _a(aux).ravel(), n, out.ravel())
    return out


def get_samples(density, max_density, pos, dirs, light, alpha, g, scatter, max_bounces, spp, seed):
    density = _a(density)
    res = round(density.size ** (1 / 3))
    n = len(pos)
    out = np.zeros(n, np.float64)
    lib().orc_get_samples(density.ravel(), res, float(max_density), _a(pos).ravel(), _a(dirs).ravel(),
                          _a(light).ravel(), _a(alpha), _a(g), _a(scatter), n, max_bounces, spp,
                          int(seed), out, nthreads())
    return out


def cloud(res, seed, octaves=6, base_freq=4.0, lacunarity=2.0, gain=0.5, threshold=0.45):
    from .cloud_np import permutation
    L = lib()
    L.orc_cloud.argtypes = [C.c_int, np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS"), C.c_int,
                            C.c_float, C.c_float, C.c_float, C.c_float, f32p, C.c_int]
    out = np.zeros(res ** 3, np.float32)
    L.orc_cloud(res, permutation(seed).astype(np.int32), octaves, base_freq, lacunarity, gain, threshold, out,
                nthreads())
    return out


def train_points(density, max_density, alpha, g, seed, n_rays, cap):
    """MeanFreePathSample over the 256^3 mip level 0 of `density` (what
    DensityAtPosition(0, p) samples), under the density's majorant."""
    _, mips, _ = build_mips(density)
    mip0 = np.ascontiguousarray(mips[:256 ** 3])
    pos = np.zeros((cap, 3), np.float32)
    dirs = np.zeros((cap, 3), np.float32)
    n = lib().orc_train_points(mip0, 256, float(max_density), float(alpha), float(g), int(seed),
                               int(n_rays), int(cap), pos.ravel(), dirs.ravel())
    n = min(n, cap)
    return pos[:n], dirs[:n]


def train_frames(dirs, light, seed):
    dirs = _a(dirs)
    out = np.zeros((len(dirs), 12), np.float32)
    lib().orc_train_frames(dirs.ravel(), len(dirs), _a(light), int(seed), out.ravel())
    return out


def train_loss(weights, desc, aux, label):
    return float(lib().orc_train_loss(_a(weights), _a(desc).ravel(), _a(aux).ravel(), _a(label), len(label)))


def histogram_frame(rad, fnum, accum, hist):
    """In-place per-frame update of accum (n x 3) and hist (n x 33) from rad (n x 3)."""
    lib().orc_histogram_frame(_a(rad).ravel(), len(accum), int(fnum), accum.ravel(), hist.ravel())


def denoise(accum, hist, W, H, frame, flip, tone, denoise, exposure):
    out = np.zeros(W * H, np.uint32)
    lib().orc_denoise(_a(accum).ravel(), _a(hist).ravel(), W, H, int(frame), int(flip), int(tone), int(denoise),
                      float(exposure), out)
    return out
