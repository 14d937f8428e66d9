"""Generate golden fixtures by running the reference's own device code.

Needs a GPU and oracle/_ref/ (built by oracle.build.build_reference() where
the reference checkout exists). Usage:
    python tests/golden/gen_ref_fixtures.py OUT_DIR [section ...]
with sections from SECTIONS (default: all). The .npz files written to
OUT_DIR are committed under tests/golden/. They hold inputs generated here
from fixed seeds and the reference's outputs; no reference data (weights,
tables) is stored.

ref_network.npz  -- the reference network (core/radiancePredict.cu:370-485)
                    on 256 injected descriptors, with random weights
                    (weights.active_random_weights(1), out_xavier) and with
                    its compiled-in weights (out_refw).
ref_pt_sphere.npz -- the reference delta tracker (CalculateRadiance) on the
                    sphere scene at 32x32, 2048 spp: per-pixel sums and sums
                    of squares.
ref_gather.npz   -- RadiancePredict with the reference's texture gather, on
                    200 points of the sphere scene with explicit frames, with
                    the reference's compiled-in weights and stencil, reading
                    the oracle's transmittance pyramid and HG table.
ref_nn_sphere.npz -- NNPredict<MRPNN> on the sphere scene at 32x32, 1024
                    passes, the reference's weights, reading the
                    transmittance pyramid its own Fill_TR built and the HG
                    table its own Fill_Hg built: per-pixel sums / squares.
ref_tables.npz   -- VolumeRender::Update's majorant, Fill_TR over the
                    oracle's mip pyramid (sphere 128^3 and a 64^3 fBm cloud;
                    levels 2..7 whole, 8192 voxels of levels 0 and 1) and
                    Fill_Hg for g = 0.857 / 0.65 / 0.3 (8192 texels with the
                    curand offsets they drew, and 8x8 block means).
ref_denoise.npz  -- 64 frames of the interactive Render (delta tracking,
                    sphere scene 32x32): accumulation, histograms, packed
                    pixels; then Denoise<bool> on those buffers and on random
                    histograms, over frame / flip / tone / exposure cases.
ref_labels.npz   -- GetSamples (training labels) for 48 points of the sphere
                    and 48 of a 64^3 cloud, 8 replicates of 1024 paths.
ref_bmp.npz      -- SaveBMP bytes of a 6x6 image and the host tone maps
                    Camera::ACES / Camera::Gamma of 256 colours.
ref_datagen.npz  -- dataGen's GetDesiredCountSample (MeanFreePathSample over
                    the 256^3 mip level 0, host code, mt19937 draws) on the
                    64^3 sphere (alpha 16) and the 64^3 cloud (alpha 24):
                    20000 training points each (position, view direction;
                    float16). Runs without a GPU.
ref_march.npz    -- NNPredict<Type::marching_MRPNN> (instantiated by the
                    harness; the reference's host code never does) on a
                    medium sphere inside a signed-distance field
                    (scenes.sdf_sphere_density(128)), 32x32, 512 passes,
                    the reference's weights and its own Fill_TR / Fill_Hg
                    tables, without a surface (IOR -1) and with IOR 1.33:
                    per-pixel sums / squares.
ref_hdri.npz     -- the offline VolumeRender::Render (delta tracking) of the
                    sphere scene (alpha 16) under an environment map loaded
                    with SetHDRI from a generated .hdr file (its RGBE pixels
                    are stored), SetEnvExp 1.5, 32x32, 1024 spp: mean image.
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from internship_b200 import scenes  # noqa: E402
from oracle import cloud_np, orc, ref_py  # noqa: E402

SECTIONS = ("network", "pt", "gather", "nn", "tables", "denoise", "labels", "bmp", "hdri", "datagen", "march")


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


def sphere_tables():
    dens = scenes.sphere_density(128)
    md, mips, var = orc.build_mips(dens)
    p = scenes.make_params(32, 32, 1)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    tr = orc.build_tr(mips, p.alpha, L)
    lut = orc.build_hglut(p.g, 0)
    return dens, md, mips, tr, lut, p, L


def camera(p):
    return (np.array([p.ori.x, p.ori.y, p.ori.z], np.float32), np.array([p.up.x, p.up.y, p.up.z], np.float32),
            np.array([p.right.x, p.right.y, p.right.z], np.float32))


# scenes of the table, label and interactive fixtures (the tests rebuild them)
CLOUD_RES, CLOUD_SEED = 64, 5
CLOUD_LIGHT = np.array([0.3, 0.8, -0.5], np.float32) / np.float32(np.linalg.norm([0.3, 0.8, -0.5]))


def gen_network(out, rng):
    from internship_b200.weights import active_random_weights
    wx = active_random_weights(1)
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


def gen_pt(out, rng):
    dens, md, mips, tr, lut, p, L = sphere_tables()
    ref = ref_py.Ref()
    ref.setup(dens, md, mips, tr, lut, scatter=(0.99, 0.99, 0.99))
    ori, up, right = camera(p)
    s, s2 = ref.render(0, 32, 32, ori, up, right, L, (1, 1, 1), p.alpha, 512, p.g, 2048)
    np.savez_compressed(os.path.join(out, "ref_pt_sphere.npz"), sum=s, sumsq=s2, spp=2048, width=32, height=32)


def gen_gather(out, rng):
    dens, md, mips, tr, lut, p, L = sphere_tables()
    ref = ref_py.Ref()
    ref.setup(dens, md, mips, tr, lut, scatter=(0.99, 0.99, 0.99))
    m = 200
    pos = rng.uniform(-0.3, 0.3, (m, 3)).astype(np.float32)
    fr = rand_frames(rng, m, L)
    scatterrate = np.array([0.99, 0.99, 0.99], np.float32) / np.float32(1.001)
    ref.load_weights(ref.read_weights())
    outg = ref.predict_frames(pos, fr, L, p.alpha, p.g, scatterrate)
    np.savez_compressed(os.path.join(out, "ref_gather.npz"), pos=pos, frames=fr, light=L, alpha=np.float32(p.alpha),
                        g=np.float32(p.g), scatterrate=scatterrate, out=outg)


def gen_nn(out, rng):
    dens, md, mips, _, _, p, L = sphere_tables()
    rv = ref_py.RefVolume()
    tr = rv.fill_tr(mips, p.alpha, L)
    lut, _ = rv.fill_hg(p.g, 0)
    ref = ref_py.Ref()
    ref.setup(dens, md, mips, tr, lut, scatter=(0.99, 0.99, 0.99))
    ori, up, right = camera(p)
    s, s2 = ref.render(1, 32, 32, ori, up, right, L, (1, 1, 1), p.alpha, 512, p.g, 1024)
    np.savez_compressed(os.path.join(out, "ref_nn_sphere.npz"), sum=s, sumsq=s2, spp=1024, width=32, height=32)


def _tr_sample(tr, rng, n=8192):
    levels, off, keep = {}, 0, {}
    for k in range(8):
        r = 128 >> k
        lv = tr[off:off + r ** 3]
        if k >= 2:
            keep["tr%d" % k] = lv
        else:
            idx = np.sort(rng.choice(r ** 3, n, replace=False)).astype(np.int32)
            keep["tr%d_idx" % k] = idx
            keep["tr%d" % k] = lv[idx]
        off += r ** 3
    return keep


def gen_tables(out, rng):
    res = {}
    p = scenes.make_params(32, 32, 1)
    Ls = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    for name, dens, alpha, L in (("sphere", scenes.sphere_density(128), 64.0, Ls),
                                 ("cloud", cloud_np.cloud(CLOUD_RES, CLOUD_SEED), 32.0, CLOUD_LIGHT)):
        r = round(dens.size ** (1 / 3))
        rv = ref_py.RefVolume(r)
        res[name + "_max_density"] = np.float32(rv.set_density(dens))
        rv.close()
        md, mips, _ = orc.build_mips(dens)
        tr = ref_py.RefVolume().fill_tr(mips, alpha, L)
        res[name + "_alpha"] = np.float32(alpha)
        res[name + "_light"] = L
        for k, v in _tr_sample(tr, rng).items():
            res[name + "_" + k] = v
    rv = ref_py.RefVolume()
    for gi, g in enumerate((0.857, 0.65, 0.3)):
        lut, bn = rv.fill_hg(g, gi)
        idx = np.sort(rng.choice(512 * 512, 8192, replace=False)).astype(np.int32)
        res["lut%d_g" % gi] = np.float32(g)
        res["lut%d_idx" % gi] = idx
        res["lut%d" % gi] = lut[idx]
        res["lut%d_bn" % gi] = bn[idx]
        res["lut%d_blocks" % gi] = lut.reshape(64, 8, 64, 8).mean(axis=(1, 3)).astype(np.float32)
    np.savez_compressed(os.path.join(out, "ref_tables.npz"), **res)


def gen_denoise(out, rng):
    W = H = 32
    frames = 64
    dens = scenes.sphere_density(128)
    p = scenes.make_params(W, H, 1)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    ori, up, right = camera(p)
    rv = ref_py.RefVolume(128)
    md = rv.set_density(dens)
    rv.set_scalars(1.0, (0.99, 0.99, 0.99), 1.0, (0, 0, 0))
    acc, hist, bgra = rv.interactive(W, H, ori, up, right, L, (1, 1, 1), p.alpha, 512, p.g, frames, tone=2, denoise=1)
    res = dict(width=W, height=H, frames=frames, max_density=np.float32(md), accum=acc, hist=hist, bgra=bgra)
    # Denoise<bool> cases on the interactive buffers and on random histograms
    cases = [(frames, 0, 2, 1, 1.0), (frames, 1, 1, 1, 1.5), (frames, 0, 0, 0, 1.0), (0, 0, 2, 0, 1.0),
             (0, 1, 2, 1, 0.7), (frames, 0, 2, 0, 2.0)]
    res["cases"] = np.array(cases, np.float32)
    for c, (fr, fl, tone, dn, ex) in enumerate(cases):
        res["case%d" % c] = rv.denoise(acc, hist, W, H, fr, fl, tone, dn, ex)
    W2, H2 = 45, 29
    racc = rng.uniform(0, 3, (W2 * H2, 3)).astype(np.float32)
    rh = np.zeros((W2 * H2, 33), np.float32)
    n = rng.integers(1, 40, W2 * H2)
    for k in range(W2 * H2):
        for ch in range(3):
            rh[k, ch * 10:(ch + 1) * 10] = np.bincount(rng.integers(0, 10, n[k]) if rng.uniform() < 0.7 else
                                                       rng.integers(0, 3, n[k]), minlength=10)[:10]
    rh[:, 30] = n
    lm = rng.uniform(0, 2, W2 * H2).astype(np.float32)
    rh[:, 32] = lm
    rh[:, 31] = lm * lm + rng.uniform(0, 0.3, W2 * H2).astype(np.float32)
    res["rand_accum"], res["rand_hist"] = racc.ravel(), rh.ravel()
    res["rand_width"], res["rand_height"] = W2, H2
    for c, (fr, fl, tone, dn, ex) in enumerate(cases):
        res["rand_case%d" % c] = rv.denoise(racc, rh, W2, H2, max(fr, 0), fl, tone, dn, ex)
    np.savez_compressed(os.path.join(out, "ref_denoise.npz"), **res)


def gen_labels(out, rng):
    res = {}
    for name, dens, alpha, L in (("sphere", scenes.sphere_density(128), 16.0, None),
                                 ("cloud", cloud_np.cloud(CLOUD_RES, CLOUD_SEED), 24.0, CLOUD_LIGHT)):
        if L is None:
            p = scenes.make_params(32, 32, 1)
            L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
        r = round(dens.size ** (1 / 3))
        rv = ref_py.RefVolume(r)
        rv.set_density(dens)
        rv.set_scalars(1.0, (1.0, 1.0, 1.0), 1.0, (0, 0, 0))
        n = 48
        # points where the medium is: rejection-sample voxels with density > 0
        idx = np.flatnonzero(dens.ravel() > 0.05)
        pick = rng.choice(idx, n, replace=False)
        x, y, z = pick // (r * r), (pick // r) % r, pick % r
        pos = ((np.stack([x, y, z], 1) + 0.5) / r - 0.5).astype(np.float32)
        d = rng.normal(size=(n, 3))
        d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
        g, scatter, bounces, spp, reps = 0.857, 0.95, 64, 1024, 8
        lab = np.stack([rv.get_samples(pos, d, L, alpha, g, scatter, bounces, spp, randnum=k)[:, 0]
                        for k in range(reps)])
        rv.close()
        res.update({name + "_pos": pos, name + "_dir": d, name + "_light": L, name + "_alpha": np.float32(alpha),
                    name + "_reps": lab})
    res.update(g=np.float32(0.857), scatter=np.float32(0.95), bounces=64, spp=1024)
    np.savez_compressed(os.path.join(out, "ref_labels.npz"), **res)


def gen_bmp(out, rng):
    rv = ref_py.RefVolume()
    img = rng.integers(0, 256, (6, 6, 4)).astype(np.uint8)
    img[..., 3] = 255  # RenderToFile writes alpha 255 (core/camera.cu:240-246)
    with tempfile.TemporaryDirectory() as td:
        path = rv.save_bmp(img, 6, 6, os.path.join(td, "img"))
        data = np.frombuffer(open(path, "rb").read(), np.uint8)
    rgb = np.concatenate([rng.uniform(0, 1, (128, 3)), rng.uniform(0, 20, (128, 3))]).astype(np.float32)
    np.savez_compressed(os.path.join(out, "ref_bmp.npz"), image=img, bmp=data, rgb=rgb, aces=rv.tone_host(rgb, 2),
                        gamma=rv.tone_host(rgb, 1))


def gen_march(out, rng):
    dens = scenes.sdf_sphere_density(128)
    md, mips, _ = orc.build_mips(dens)
    p = scenes.make_params(32, 32, 1, alpha=32.0)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    rv = ref_py.RefVolume()
    tr = rv.fill_tr(mips, p.alpha, L)
    lut, _ = rv.fill_hg(p.g, 0)
    ref = ref_py.Ref()
    ref.setup(dens, md, mips, tr, lut, scatter=(0.99, 0.99, 0.99))
    ori, up, right = camera(p)
    res = dict(spp=512, width=32, height=32, alpha=np.float32(p.alpha))
    for name, ior in (("plain", -1.0), ("ior", 1.33)):
        ref.set_ior(ior)
        s, s2 = ref.render(2, 32, 32, ori, up, right, L, (1, 1, 1), p.alpha, 512, p.g, 512)
        res[name + "_sum"], res[name + "_sumsq"] = s, s2
    ref.set_ior(-1.0)
    np.savez_compressed(os.path.join(out, "ref_march.npz"), **res)


def gen_datagen(out, rng):
    res = {}
    for name, dens, alpha in (("sphere", scenes.sphere_density(64), 16.0),
                              ("cloud", cloud_np.cloud(CLOUD_RES, CLOUD_SEED), 24.0)):
        md, mips, _ = orc.build_mips(dens)
        rv = ref_py.RefVolume(round(dens.size ** (1 / 3)))
        pos, view = rv.datagen_samples(mips[:256 ** 3], md, alpha, 20000)
        rv.close()
        res.update({name + "_pos": pos.astype(np.float16), name + "_view": view.astype(np.float16),
                    name + "_alpha": np.float32(alpha)})
    np.savez_compressed(os.path.join(out, "ref_datagen.npz"), **res)


def gen_hdri(out, rng):
    from oracle import hdr_np
    W = H = 32
    spp, alpha, env_exp = 1024, 16.0, 1.5
    v_ = (np.arange(24) + 0.5) / 24
    u_ = (np.arange(48) + 0.5) / 48
    U, Vv = np.meshgrid(u_, v_)
    img = np.stack([0.3 + 0.5 * (1 - Vv), 0.4 + 0.4 * (1 - Vv), 0.8 + 0.2 * np.cos(2 * np.pi * U)], -1)
    img = img + (40.0 * np.exp(-(((U - 0.3) / 0.05) ** 2 + ((Vv - 0.3) / 0.08) ** 2)))[..., None] * [1.0, 0.9, 0.7]
    p = scenes.make_params(W, H, 1, alpha=alpha)
    L = np.array([p.light_dir.x, p.light_dir.y, p.light_dir.z], np.float32)
    ori, up, right = camera(p)
    rv = ref_py.RefVolume(128)
    rv.set_density(scenes.sphere_density(128))
    rv.set_scalars(1.0, (0.99, 0.99, 0.99), 1.0, (0, 0, 0))
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "sky.hdr")
        rgbe = hdr_np.write(path, img.astype(np.float32))
        rv.set_hdri(path, env_exp)
        image = rv.render_pt(W, H, ori, up, right, L, (1, 1, 1), alpha, 512, p.g, spp)
    rv.close()
    np.savez_compressed(os.path.join(out, "ref_hdri.npz"), rgbe=rgbe, image=image, width=W, height=H, spp=spp,
                        alpha=np.float32(alpha), env_exp=np.float32(env_exp))


def main(out, sections):
    os.makedirs(out, exist_ok=True)
    for s in sections:
        rng = np.random.default_rng(20261203 + SECTIONS.index(s))
        globals()["gen_" + s](out, rng)
        print(s, "fixture done", flush=True)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: gen_ref_fixtures.py OUT_DIR [%s ...]" % " | ".join(SECTIONS))
    main(sys.argv[1], sys.argv[2:] or list(SECTIONS))
