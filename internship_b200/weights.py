"""Weight and stencil files of the reference, read on the host.

`load_nnweight_header(path)` parses a weight header in the format of the
reference's core/NNWeight.cuh (named fp32 arrays with initialisers) and
returns the flat blob in the order of include/mrpnn_weights.h, checking every
array's name and size. `load_stencil_source(path)` reads the 160 stencil
points from a source file in the format of core/vector.cu:77-172 (arrays
Spn0..Spn4 and SpVn5..SpVn7). `save_blob` / `load_blob` store a blob as a
small binary with a header (magic, version, count).
"""
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LAYOUT_H = os.path.join(os.path.dirname(HERE), "include", "mrpnn_weights.h")
MAGIC = b"MRPNNW01"


def layout():
    """[(name, size), ...] in blob order, read from include/mrpnn_weights.h."""
    txt = open(LAYOUT_H).read()
    return [(m.group(1), int(m.group(2))) for m in re.finditer(r"X\((\w+),\s*(\d+)\)", txt)]


_ARRAY = re.compile(r"(?:__device__\s+)?(?:__constant__\s+)?(?:const\s+)?float\s+(\w+)\s*\[\s*(\d+)\s*\]\s*=\s*\{([^}]*)\}",
                    re.S)


def load_nnweight_header(path):
    txt = open(path).read()
    arrays = {}
    for m in _ARRAY.finditer(txt):
        vals = [v for v in re.split(r"[\s,]+", m.group(3).strip()) if v]
        a = np.array([float(v.rstrip("fF")) for v in vals], np.float32)
        if a.size != int(m.group(2)):
            raise ValueError("%s: %d values for size %s" % (m.group(1), a.size, m.group(2)))
        arrays[m.group(1)] = a
    out = []
    for name, n in layout():
        if name not in arrays:
            raise ValueError("weight array %s missing from %s" % (name, path))
        if arrays[name].size != n:
            raise ValueError("weight array %s has %d values, expected %d" % (name, arrays[name].size, n))
        out.append(arrays[name])
    return np.concatenate(out)


_F3 = re.compile(r"float3\s*\{\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*,\s*([-+0-9.eE]+)\s*\}")


def load_stencil_source(path):
    txt = open(path).read()
    pts = []
    for name, n in (("Spn0", 8), ("Spn1", 8), ("Spn2", 16), ("Spn3", 16), ("Spn4", 16), ("SpVn5", 32),
                    ("SpVn6", 32), ("SpVn7", 32)):
        m = re.search(r"float3\s+%s\s*\[\s*%d\s*\]\s*=\s*\{(.*?)\};" % (name, n), txt, re.S)
        if not m:
            raise ValueError("stencil table %s[%d] not found in %s" % (name, n, path))
        vals = [tuple(float(v) for v in t) for t in _F3.findall(m.group(1))]
        if len(vals) != n:
            raise ValueError("stencil table %s has %d points, expected %d" % (name, len(vals), n))
        pts += vals
    return np.array(pts, np.float32).ravel()


def active_random_weights(seed=1):
    """Random network whose every ReLU, the last one included, is active on
    non-negative descriptors: Xavier(seed) weights, biases uniform in
    [0, 0.1], and the final 16->1 layer's weights made non-negative. Useful
    for parity tests, where all-zero outputs would prove nothing."""
    from .volume import xavier_weights
    w = xavier_weights(seed, bias_range=(0.0, 0.1))
    off = 0
    for name, n in layout():
        if name == "LX12W":
            w[off:off + n] = np.abs(w[off:off + n])
        off += n
    return w


def save_blob(path, weights, stencil=None):
    w = np.ascontiguousarray(weights, np.float32).ravel()
    st = np.zeros(480, np.float32) if stencil is None else np.ascontiguousarray(stencil, np.float32).ravel()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.array([w.size, 0 if stencil is None else 480], np.int32).tobytes())
        f.write(w.tobytes())
        f.write(st.tobytes())


def load_blob(path):
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError("%s is not a weight blob" % path)
        n, ns = np.frombuffer(f.read(8), np.int32)
        w = np.frombuffer(f.read(4 * n), np.float32).copy()
        st = np.frombuffer(f.read(4 * 480), np.float32).copy()
    return w, (st if ns else None)
