"""Benchmark and test scenes (synthetic, seeded).

sphere_scene  : 128^3 solid sphere (centre 0.5, radius 0.25, density 1),
                extinction scale 64, albedo 0.99, HG g = 0.857, one unit
                directional light with a seeded direction, camera at distance
                2.5 looking at the centre with a 40 degree field of view,
                256 x 256, 64 spp, up to 512 bounces, Philox seed 0.
cloud_scene   : 512^3 seeded Perlin-fBm cloud (6 octaves, base frequency 4,
                lacunarity 2, gain 0.5, threshold 0.45, radial falloff) with
                the sphere scene's light, medium and camera at 1920 x 1080.

The module is plain Python and loads no library at import (the device
helpers import the package's loader when called), so a CPU-only process can
load it by path to build the same render requests.
"""
import ctypes as C
import math

import numpy as np

RT_PT, RT_MRPNN = 0, 2  # mr_render_type

M0, M1, W0, W1 = 0xD2511F53, 0xCD9E8D57, 0x9E3779B9, 0xBB67AE85


def philox4x32_10(ctr, key):
    """Philox4x32-10 (Salmon et al., SC'11) on python ints."""
    c = [int(x) & 0xFFFFFFFF for x in ctr]
    k0, k1 = int(key[0]) & 0xFFFFFFFF, int(key[1]) & 0xFFFFFFFF
    for r in range(10):
        if r:
            k0, k1 = (k0 + W0) & 0xFFFFFFFF, (k1 + W1) & 0xFFFFFFFF
        p0, p1 = M0 * c[0], M1 * c[2]
        c = [((p1 >> 32) ^ c[1] ^ k0) & 0xFFFFFFFF, p1 & 0xFFFFFFFF, ((p0 >> 32) ^ c[3] ^ k1) & 0xFFFFFFFF,
             p0 & 0xFFFFFFFF]
    return c


def u01(x):
    return ((x >> 9) + 0.5) * 1.1920928955078125e-7


def seeded_light(seed=0):
    """Uniform direction on the sphere from Philox(seed; 0, 0, 0, 8)."""
    w = philox4x32_10([0, 0, 0, 8], [seed, 0])
    ex, ey = u01(w[0]), u01(w[1])
    phi = 2 * math.pi * ex
    ct = 1 - 2 * ey
    st = math.sqrt(max(0.0, 1 - ct * ct))
    return (st * math.cos(phi), st * math.sin(phi), ct)


def camera_vectors(position, fov_deg):
    """Camera::SetPosition (core/camera.cu:173-189), right/up scaled by
    tan(fov/2) as VolumeRender::Render expects."""
    ori = np.asarray(position, np.float64)
    fwd = -ori / np.linalg.norm(ori)
    right = np.cross([0.0, 1.0, 0.0], fwd)
    right /= np.linalg.norm(right)
    up = np.cross(fwd, right)
    s = math.tan(math.radians(fov_deg) / 2)
    return tuple(ori), tuple(up * s), tuple(right * s)


def sphere_density(res=128):
    i = (np.arange(res) + 0.5) / res
    x, y, z = np.meshgrid(i, i, i, indexing="ij")
    d = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
    return (d < 0.25).astype(np.float32)


def sdf_sphere_density(res=128, radius=0.2):
    """A medium sphere (density 1) inside a signed-distance field: outside the
    sphere the density is minus the distance to its surface, the encoding the
    marching form reads as empty space to skip and as the side of a surface."""
    i = (np.arange(res) + 0.5) / res
    x, y, z = np.meshgrid(i, i, i, indexing="ij")
    d = np.sqrt((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
    return np.where(d < radius, 1.0, radius - d).astype(np.float32)


CAMERA_DIR = np.array([1.0, 0.55, 0.8]) / np.linalg.norm([1.0, 0.55, 0.8])


def _set3(field, v):
    field.x, field.y, field.z = (float(c) for c in v)


def make_params(width, height, spp=1, rt=RT_PT, bounces=512, seed=0, alpha=64.0, g=0.857, albedo=0.99,
                distance=2.5, fov=40.0, sample_offset=0, precision=0, light_seed=0, sampler=0, params_cls=None):
    """An mr_render_params request (params_cls: the ctypes mirror to fill,
    default the package's RenderParams)."""
    if params_cls is None:
        from ._lib import RenderParams as params_cls
    ori, up, right = camera_vectors(CAMERA_DIR * distance, fov)
    p = params_cls()
    p.width, p.height = width, height
    _set3(p.ori, ori)
    _set3(p.up, up)
    _set3(p.right, right)
    _set3(p.light_dir, seeded_light(light_seed))
    _set3(p.light_color, (1.0, 1.0, 1.0))
    p.alpha, p.g = alpha, g
    _set3(p.scatter_rate, (albedo, albedo, albedo))
    p.tr_scale = 1.0
    _set3(p.env_color, (0.0, 0.0, 0.0))
    p.max_bounces, p.spp = bounces, spp
    p.seed, p.sample_offset = seed, sample_offset
    p.render_type, p.precision, p.sampler = rt, precision, sampler
    return p


def sphere_scene(width=256, height=256, spp=64, **kw):
    return sphere_density(128), make_params(width, height, spp, **kw)


CLOUD_ARGS = dict(octaves=6, base_freq=4.0, lacunarity=2.0, gain=0.5, threshold=0.45)


def generate_cloud_device(res, seed, dev_ptr, stream=None, **over):
    from . import _lib
    a = dict(CLOUD_ARGS, **over)
    _lib.check(_lib.load().mr_generate_cloud(res, seed, a["octaves"], a["base_freq"], a["lacunarity"], a["gain"],
                                        a["threshold"], C.c_void_p(dev_ptr), stream))


def cloud_permutation(seed):
    from . import _lib
    out = np.zeros(256, np.int32)
    _lib.check(_lib.load().mr_cloud_permutation(seed, out.ctypes.data))
    return out


def cloud_scene_params(width=1920, height=1080, **kw):
    kw.setdefault("rt", RT_MRPNN)
    return make_params(width, height, 1, **kw)


def ray_box_offset_np(p, d):
    """RayBoxOffset (core/vector.cu:41-58) on the host: entry distance of the
    ray p + t d into the box +-0.4999, -1 on a miss (float32 arithmetic)."""
    p = np.asarray(p, np.float32)
    d = np.asarray(d, np.float32)
    with np.errstate(divide="ignore"):
        inv = np.where(d == 0, np.float32(999999999.0), np.float32(1.0) / np.where(d == 0, 1, d)).astype(np.float32)
    to_axis = (-p) * inv
    to_face = np.float32(0.4999) * inv
    d0, d1 = to_axis + to_face, to_axis - to_face
    tmi = float(np.max(np.minimum(d0, d1)))
    tma = float(np.min(np.maximum(d0, d1)))
    return max(tmi, 0.0) if tma >= tmi else -1.0
