"""numpy restatement of the reference's volume file readers (test
infrastructure only): VolumeRender(string path), core/volume.cu:835-911."""
import os

import numpy as np


def read(path):
    """(resolution, r^3 float32 array, from_bin) as the reference reads it:
    <path>.bin first (core/volume.cu:837-844), else .txt (:847-866) or .vox
    (:867-895)."""
    if os.path.exists(path + ".bin"):
        raw = open(path + ".bin", "rb").read()
        r = int(np.frombuffer(raw[:4], np.int32)[0])
        return r, np.frombuffer(raw[4:4 + 4 * r ** 3], np.float32).copy(), True
    if path.endswith("txt"):
        vals = open(path).read().split()
        r = int(vals[0])
        return r, np.array([float(v) for v in vals[1:1 + r ** 3]], np.float32), False
    if path.endswith("vox"):
        r = 256
        out = np.zeros(r ** 3, np.float32)
        inv = np.float32(64.0) / np.float32(255.0)
        i = 0
        for line in open(path):
            if i >= r ** 3:
                break
            if line[:1] in ("w", "h", "d") or not line.split():
                continue
            d = np.array(line.split()[:64], np.int64)
            out[i:i + 64] = d.astype(np.float32) * inv
            i += 64
        return r, out, False
    raise FileNotFoundError(path)
