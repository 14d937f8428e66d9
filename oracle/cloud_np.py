"""numpy restatement of the procedural cloud (test infrastructure only):
Perlin improved noise (Perlin 2002) summed as fBm, normalised, thresholded,
radial falloff -- the definition the GPU generator implements."""
import numpy as np

from . import orc


def permutation(seed):
    perm = list(range(256))
    for i in range(255, 0, -1):
        w = orc.philox([i, 0, 0, 7], [seed, 0])
        j = int(w[0]) % (i + 1)
        perm[i], perm[j] = perm[j], perm[i]
    return np.array(perm, np.int64)


def _fade(t):
    return t * t * t * (t * (t * 6.0 - 15.0) + 10.0)


def _grad(h, x, y, z):
    h = h & 15
    u = np.where(h < 8, x, y)
    v = np.where(h < 4, y, np.where((h == 12) | (h == 14), x, z))
    return np.where(h & 1, -u, u) + np.where(h & 2, -v, v)


def perlin(P, x, y, z):
    fx, fy, fz = np.floor(x), np.floor(y), np.floor(z)
    X, Y, Z = fx.astype(np.int64) & 255, fy.astype(np.int64) & 255, fz.astype(np.int64) & 255
    x, y, z = x - fx, y - fy, z - fz
    u, v, w = _fade(x), _fade(y), _fade(z)
    A = P[X] + Y
    AA, AB = P[A] + Z, P[A + 1] + Z
    B = P[X + 1] + Y
    BA, BB = P[B] + Z, P[B + 1] + Z
    lerp = lambda a, b, t: a * (1 - t) + b * t
    return lerp(lerp(lerp(_grad(P[AA], x, y, z), _grad(P[BA], x - 1, y, z), u),
                     lerp(_grad(P[AB], x, y - 1, z), _grad(P[BB], x - 1, y - 1, z), u), v),
                lerp(lerp(_grad(P[AA + 1], x, y, z - 1), _grad(P[BA + 1], x - 1, y, z - 1), u),
                     lerp(_grad(P[AB + 1], x, y - 1, z - 1), _grad(P[BB + 1], x - 1, y - 1, z - 1), u), v), w)


def cloud(res, seed, octaves=6, base_freq=4.0, lacunarity=2.0, gain=0.5, threshold=0.45):
    perm = permutation(seed)
    P = np.concatenate([perm, perm])
    i = (np.arange(res) + 0.5) / res
    x, y, z = np.meshgrid(i, i, i, indexing="ij")
    s, norm, amp, f = 0.0, 0.0, 1.0, base_freq
    for _ in range(octaves):
        s = s + amp * perlin(P, x * f, y * f, z * f)
        norm += amp
        amp *= gain
        f *= lacunarity
    n = 0.5 + 0.5 * s / norm
    r2 = 4.0 * ((x - 0.5) ** 2 + (y - 0.5) ** 2 + (z - 0.5) ** 2)
    return (np.maximum(0.0, n - threshold) / (1.0 - threshold) * np.maximum(0.0, 1.0 - r2)).astype(np.float32)
