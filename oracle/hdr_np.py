"""Radiance RGBE (.hdr) images in numpy (test infrastructure only): a writer
(flat or new-style run-length scanlines) for generated test images, and a
decoder restating the format as the reference's loader reads it
(core/hdr_loader.h:43-249)."""
import numpy as np


def encode_rgbe(rgb):
    """(h, w, 3) float -> (h, w, 4) uint8 RGBE: mantissas scaled by
    2^-(e - 128) so the largest channel lands in [128, 256)."""
    rgb = np.asarray(rgb, np.float64)
    m = rgb.max(-1)
    out = np.zeros(rgb.shape[:-1] + (4,), np.uint8)
    nz = m > 1e-32
    mant, ex = np.frexp(m[nz])  # m = mant * 2^ex, mant in [0.5, 1)
    scale = mant * 256.0 / m[nz]
    out[nz, :3] = np.clip(np.floor(rgb[nz] * scale[:, None]), 0, 255).astype(np.uint8)
    out[nz, 3] = (ex + 128).astype(np.uint8)
    return out


def _rle_component(vals):
    out = bytearray()
    i, n = 0, len(vals)
    while i < n:
        run = 1
        while i + run < n and run < 127 and vals[i + run] == vals[i]:
            run += 1
        if run >= 4:
            out += bytes([128 + run, vals[i]])
            i += run
            continue
        j = i
        while j < n and j - i < 128:
            if j + 3 < n and vals[j] == vals[j + 1] == vals[j + 2] == vals[j + 3]:
                break
            j += 1
        out += bytes([j - i]) + bytes(vals[i:j])
        i = j
    return bytes(out)


def write(path, rgb, rle=True):
    rgbe = encode_rgbe(rgb)
    h, w = rgbe.shape[:2]
    with open(path, "wb") as f:
        f.write(b"#?RADIANCE\n# generated test image\nFORMAT=32-bit_rle_rgbe\nEXPOSURE=1.0\n\n")
        f.write(("-Y %d +X %d\n" % (h, w)).encode())
        for j in range(h):
            if rle and 8 <= w <= 0x7fff:
                f.write(bytes([2, 2, w >> 8, w & 255]))
                for c in range(4):
                    f.write(_rle_component(rgbe[j, :, c].tolist()))
            else:
                f.write(rgbe[j].tobytes())
    return rgbe


def decode(rgbe):
    """(h, w, 4) uint8 -> (h, w, 4) float32 as load_hdr_float4 fills it:
    (c + 0.5) * 2^(e - 136) per channel, 0 when e = 0, alpha 0."""
    rgbe = np.asarray(rgbe)
    out = np.zeros(rgbe.shape[:-1] + (4,), np.float32)
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(np.float32(1.0), e - 136), 0).astype(np.float32)
    out[..., :3] = (rgbe[..., :3].astype(np.float32) + np.float32(0.5)) * scale[..., None]
    out[..., :3][e == 0] = 0
    return out
