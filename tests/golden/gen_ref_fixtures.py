"""Generate golden fixtures by running the reference's own device code.

Needs a GPU and oracle/_ref/ (built by oracle.build.build_reference() where
the reference checkout exists). Usage:
    python tests/golden/gen_ref_fixtures.py OUT_DIR
The .npz files written to OUT_DIR are committed under tests/golden/. They hold
inputs generated here from fixed seeds and the reference's outputs; no
reference data (weights, tables) is stored.

ref_network.npz  -- the reference network (core/radiancePredict.cu:370-485)
                    on 256 injected descriptors, with random weights (weights.active_random_weights(1),
                    out_xavier) and with its compiled-in
                    weights (out_refw).
ref_pt_sphere.npz -- the reference delta tracker (CalculateRadiance) on the
                    sphere scene at 32x32, 2048 spp: per-pixel sums and sums
                    of squares.
ref_gather.npz   -- RadiancePredict with the reference's texture gather, on
                    200 points of the sphere scene with explicit frames, with
                    the reference's compiled-in weights and stencil.
ref_nn_sphere.npz -- NNPredict<MRPNN> on the sphere scene at 32x32, 1024
                    passes, the reference's weights: per-pixel sums / squares.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from internship_b200 import scenes, xavier_weights  # noqa: E402
from oracle import orc, ref_py  # noqa: E402


def rand_frames(rng, n, light):
    fr = np.zeros((n, 12), np.float32)
    for k in range(n):
        x = rng.normal(size=3)
        x /= np.linalg.norm(x)
        r = rng.normal(size=3)
        y = np.cross(x, r)
        y /= np.linalg.norm(y)
        z = np.cross(y, x)
        fr[k, 0:3], fr[k, 3:6], fr[k, 6:9], fr[k, 9:12] = x, y, z, light
    return fr


def main(out):
    os.makedirs(out, exist_ok=True)
    rng = np.random.default_rng(20261203)
    from internship_b200.weights import active_random_weights
    wx = active_random_weights(1)

    # -- network on injected descriptors --------------------------------------------
    net = ref_py.RefNet()
    ref_w = net.read_weights()
    n = 256
    raw = np.zeros((n, 576), np.float32)
    for sl in (slice(0, 192), slice(384, 576)):
        v = rng.uniform(0.05, 3.0, (n, 192)).astype(np.float32)
        v[rng.uniform(size=(n, 192)) < 0.2] = 0.0
        raw[:, sl] = v
    raw[:, 192:384] = rng.uniform(0, 1, (n, 192))
    light = np.asarray(scenes.seeded_light(0), np.float32)
    frames = rand_frames(rng, n, light)
    g = 0.857
    scatterrate = np.array([0.99, 0.99, 0.99], np.float32) / np.float32(1.001)
    net.load_weights(wx)
    out_x = net.predict(raw, frames, light, g, scatterrate)
    scatter3 = np.array([0.9, 0.95, 0.99], np.float32) / np.float32(1.001)
    out_x3 = net.predict(raw, frames, light, g, scatter3)
    net.load_weights(ref_w)
    out_r = net.predict(raw, frames, light, g, scatterrate)
    np.savez_compressed(os.path.join(out, "ref_network.npz"), raw=raw, frames=frames, light=light, g=np.float32(g),
                        scatterrate=scatterrate, scatterrate3=scatter3, out_xavier=out_x, out_xavier3=out_x3,
                        out_refw=out_r)
    print("network fixture done")

    # -- sphere scene tables (oracle) ------------------------------------------------
    dens = scenes.sphere_density(128)
    md, mips, var = orc.build_mips(dens)
    p = scenes.make_params(32, 32, 1)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    tr = orc.build_tr(mips, p.alpha, L)
    lut = orc.build_hglut(p.g, 0)
    ref = ref_py.Ref()
    ref.setup(dens, md, mips, tr, lut, scatter=(0.99, 0.99, 0.99))
    ori = np.array([p.ori.x, p.ori.y, p.ori.z], np.float32)
    up = np.array([p.up.x, p.up.y, p.up.z], np.float32)
    right = np.array([p.right.x, p.right.y, p.right.z], np.float32)

    s, s2 = ref.render(0, 32, 32, ori, up, right, L, (1, 1, 1), p.alpha, 512, p.g, 2048)
    np.savez_compressed(os.path.join(out, "ref_pt_sphere.npz"), sum=s, sumsq=s2, spp=2048, width=32, height=32)
    print("pt fixture done")

    # -- gather + network with explicit frames --------------------------------------
    m = 200
    pos = rng.uniform(-0.3, 0.3, (m, 3)).astype(np.float32)
    fr = rand_frames(rng, m, L)
    ref.load_weights(ref_w)
    outg = ref.predict_frames(pos, fr, L, p.alpha, p.g, scatterrate)
    np.savez_compressed(os.path.join(out, "ref_gather.npz"), pos=pos, frames=fr, light=L, alpha=np.float32(p.alpha),
                        g=np.float32(p.g), scatterrate=scatterrate, out=outg)
    print("gather fixture done")

    # -- full neural pixel ------------------------------------------------------------
    s, s2 = ref.render(1, 32, 32, ori, up, right, L, (1, 1, 1), p.alpha, 512, p.g, 1024)
    np.savez_compressed(os.path.join(out, "ref_nn_sphere.npz"), sum=s, sumsq=s2, spp=1024, width=32, height=32)
    print("neural fixture done")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "gpurun_out", "golden"))
