"""CPU tests that pin the oracle's table builders, denoiser, label estimator,
tone maps and BMP writer to outputs of the reference's own code
(tests/golden/ref_tables.npz, ref_denoise.npz, ref_labels.npz, ref_bmp.npz,
written by tests/golden/gen_ref_fixtures.py from VolumeRender::Update,
Fill_TR, Fill_Hg, Denoise, GetSamples, the interactive Render, SaveBMP and
Camera::ACES / Gamma)."""
import os

import numpy as np
import pytest

from conftest import golden
from oracle import cloud_np, orc
from internship_b200 import scenes

CLOUD_RES, CLOUD_SEED = 64, 5  # the cloud of the table and label fixtures


def _scene(name):
    return scenes.sphere_density(128) if name == "sphere" else cloud_np.cloud(CLOUD_RES, CLOUD_SEED)


def _tr_levels(tr):
    out, off = [], 0
    for k in range(8):
        r = 128 >> k
        out.append(tr[off:off + r ** 3])
        off += r ** 3
    return out


@pytest.mark.parametrize("name", ["sphere", "cloud"])
def test_majorant_matches_reference_update(name):
    """VolumeRender::Update's max_density (core/volume.cu:1219-1224)."""
    d = golden("ref_tables.npz")
    md, _, _ = orc.build_mips(_scene(name))
    assert np.float32(md) == d[name + "_max_density"]


@pytest.mark.parametrize("name", ["sphere", "cloud"])
def test_transmittance_pyramid_matches_reference_fill_tr(name):
    """The oracle's TR pyramid against the reference's Fill_TR
    (core/volume.cu:1320-1345) run over the same mip levels. The reference
    samples through the texture unit (8-bit interpolation weights), the oracle
    in fp32, so the 128-step optical depths differ by a fraction of a percent."""
    d = golden("ref_tables.npz")
    _, mips, _ = orc.build_mips(_scene(name))
    tr = _tr_levels(orc.build_tr(mips, float(d[name + "_alpha"]), d[name + "_light"]))
    for k in range(8):
        ref = d["%s_tr%d" % (name, k)]
        ours = tr[k][d["%s_tr%d_idx" % (name, k)]] if k < 2 else tr[k]
        # compare optical depths -log(TR): the quantity the march sums
        tau_r, tau_o = -np.log(np.maximum(ref, 1e-30)), -np.log(np.maximum(ours, 1e-30))
        ok = tau_r < 30
        err = np.abs(tau_o - tau_r)[ok] / (tau_r[ok] + 0.05)
        assert np.median(err) < 2e-3, (k, np.median(err))
        assert np.quantile(err, 0.99) < 2e-2, (k, np.quantile(err, 0.99))


@pytest.mark.parametrize("gi", [0, 1, 2])
def test_hg_table_matches_reference_fill_hg_texel_by_texel(gi):
    """Fill_Hg (core/volume.cu:1082-1160) restated: with the curand offset
    each reference texel drew, the oracle's estimator reproduces the
    reference's texels (fast-math transcendentals on the reference side)."""
    d = golden("ref_tables.npz")
    g = float(d["lut%d_g" % gi])
    ours = orc.hglut_texels(g, d["lut%d_idx" % gi], d["lut%d_bn" % gi])
    ref = d["lut%d" % gi]
    err = np.abs(ours - ref) / (np.abs(ref) + 1e-6)
    assert np.median(err) < 1e-5, np.median(err)
    assert np.quantile(err, 0.999) < 2e-3, np.quantile(err, 0.999)


@pytest.mark.parametrize("gi", [0, 1, 2])
def test_hg_table_matches_reference_with_own_offsets(gi):
    """The whole table with this project's offsets (Philox instead of curand)
    against the reference's: 8 x 8 block means agree to the Monte Carlo noise
    of two independent offsets."""
    d = golden("ref_tables.npz")
    g = float(d["lut%d_g" % gi])
    lut = orc.build_hglut(g, 0)
    blocks = lut.reshape(64, 8, 64, 8).mean(axis=(1, 3))
    ref = d["lut%d_blocks" % gi]
    err = np.abs(blocks - ref) / (np.abs(ref) + 1e-6)
    assert np.median(err) < 2e-3, np.median(err)
    assert err.max() < 5e-2, err.max()


def _unpack(px):
    px = np.asarray(px, np.uint32)
    return np.stack([(px >> 16) & 255, (px >> 8) & 255, px & 255], -1).astype(np.int32)


def test_denoise_matches_reference_on_its_own_buffers():
    """Denoise<bool> (core/volume.cu:187-264): filter, checkerboard fill,
    exposure, Gamma / ACES and the pack, on the accumulation and histograms
    the reference's interactive Render produced and on random histograms."""
    d = golden("ref_denoise.npz")
    for pre, W, H in (("", int(d["width"]), int(d["height"])), ("rand_", int(d["rand_width"]), int(d["rand_height"]))):
        acc, hist = d[pre + "accum" if pre else "accum"], d[pre + "hist" if pre else "hist"]
        for c, (fr, fl, tone, dn, ex) in enumerate(d["cases"]):
            ours = _unpack(orc.denoise(acc, hist, W, H, int(fr), int(fl), int(tone), int(dn), float(ex)))
            ref = _unpack(d["%scase%d" % (pre, c)])
            diff = np.abs(ours - ref)
            assert diff.max() <= 1, (pre, c, diff.max())
            assert (diff > 0).mean() < 0.01, (pre, c, (diff > 0).mean())


def test_interactive_histograms_match_reference_accounting():
    """The reference's interactive Render after K frames: every pixel's
    histogram holds K samples per channel, and its scalar means are the
    means of the same samples the accumulation averages."""
    d = golden("ref_denoise.npz")
    K = int(d["frames"])
    h = d["hist"].reshape(-1, 33)
    assert np.all(h[:, 30] == K)
    for c in range(3):
        assert np.all(h[:, 10 * c:10 * c + 10].sum(1) == K)
    acc = d["accum"].reshape(-1, 3)
    # l = sum over channels of x / (1 + x) <= sum of x; E[l] >= 0
    assert np.all(h[:, 32] >= 0) and np.all(h[:, 32] <= acc.sum(1) + 1e-5)


@pytest.mark.parametrize("name", ["sphere", "cloud"])
def test_labels_match_reference_get_samples(name):
    """GetSample (core/render.cuh:276-315) through VolumeRender::GetSamples:
    the oracle's label estimate against the mean of 8 reference replicates
    (curand streams), per point within a z-bound from both estimates' errors."""
    d = golden("ref_labels.npz")
    dens = _scene(name)
    md, _, _ = orc.build_mips(dens)
    reps = d[name + "_reps"]
    n_rep, spp = reps.shape[0], int(d["spp"])
    ref_mean = reps.mean(0)
    ref_se = reps.std(0, ddof=1) / np.sqrt(n_rep)
    pos, dirs = d[name + "_pos"], d[name + "_dir"]
    alpha, g, sc, b = float(d[name + "_alpha"]), float(d["g"]), float(d["scatter"]), int(d["bounces"])
    K = 4
    light = np.tile(d[name + "_light"].reshape(1, 3), (len(pos), 1))  # one light for every point
    n = len(pos)
    ests = np.stack([orc.get_samples(dens, md, pos, dirs, light, np.full(n, alpha, np.float32),
                                     np.full(n, g, np.float32), np.full(n, sc, np.float32), b, spp,
                                     seed=11 + k) for k in range(K)])
    ours = ests.mean(0)
    our_se = ests.std(0, ddof=1) / np.sqrt(K)
    z = (ours - ref_mean) / np.sqrt(ref_se ** 2 + our_se ** 2 + 1e-12)
    assert np.abs(z).max() < 5.0, np.abs(z).max()
    assert np.mean(np.abs(z) > 3) < 0.05
    assert abs(ours.mean() - ref_mean.mean()) < 4 * np.sqrt((ref_se ** 2 + our_se ** 2).sum()) / len(pos) + 1e-6


def test_bmp_writer_matches_reference_save_bmp(tmp_path):
    """SaveBMP (core/camera.cu:10-61): the same bytes, except the image-size
    field, which the reference fixes at 0x100000 (the size of its 512 x 512
    frames) and this writer sets to the image's size."""
    from internship_b200 import volume as V
    d = golden("ref_bmp.npz")
    img = d["image"]
    V.save_bmp(str(tmp_path / "a"), img[..., :3])
    ours = open(str(tmp_path / "a.bmp"), "rb").read()
    ref = bytes(d["bmp"])
    assert len(ours) == len(ref)
    diff = [i for i in range(len(ref)) if ours[i] != ref[i]]
    assert set(diff) <= {34, 35, 36, 37}, diff
    h, w = img.shape[:2]
    assert int.from_bytes(ours[34:38], "little") == w * h * 4


def test_host_tone_maps_match_reference_camera():
    """Camera::ACES and Camera::Gamma (core/camera.cu:66-160). The
    reference's gamma leaves NaN where a channel is negative; its pack
    (saturate_) turns NaN into 0, which is what the clamped form here gives."""
    from internship_b200 import volume as V
    d = golden("ref_bmp.npz")
    for ours, ref in ((V.tone_aces(d["rgb"]), d["aces"]), (V.tone_gamma(d["rgb"]), d["gamma"])):
        ref = np.nan_to_num(ref, nan=0.0)
        np.testing.assert_allclose(ours, ref, rtol=2e-5, atol=2e-6)


def test_oracle_xavier_and_stencil_match_the_library():
    """The reference arm of the benchmark takes its weights and stencil from
    the oracle; they are the library's, value for value."""
    import internship_b200 as mr
    assert np.array_equal(orc.xavier_weights(1), mr.xavier_weights(1))
    assert np.array_equal(orc.reference_stencil(), mr.builtin_stencil())


def _two_sample_chi2(a, b, bins):
    """Two-sample chi-square statistic of histograms a, b (same bins) and its
    degrees of freedom."""
    ha, _ = np.histogram(a, bins)
    hb, _ = np.histogram(b, bins)
    na, nb = ha.sum(), hb.sum()
    k1, k2 = np.sqrt(nb / na), np.sqrt(na / nb)
    m = (ha + hb) > 0
    stat = float((((k1 * ha - k2 * hb) ** 2)[m] / (ha + hb)[m]).sum())
    return stat, int(m.sum()) - 1


@pytest.mark.parametrize("name", ["sphere", "cloud"])
def test_training_points_match_reference_datagen(name):
    """MeanFreePathSample / GetDesiredCountSample (dataGen.cu:148-216) run by
    the reference (mt19937 draws) against the oracle's restatement (Philox):
    the distributions of the training points' radius, of each coordinate and
    of the view directions agree (two-sample chi-square, p > 1e-4)."""
    from scipy.stats import chi2
    d = golden("ref_datagen.npz")
    dens = scenes.sphere_density(64) if name == "sphere" else cloud_np.cloud(CLOUD_RES, CLOUD_SEED)
    md, _, _ = orc.build_mips(dens)
    rp, rv = d[name + "_pos"].astype(np.float32), d[name + "_view"].astype(np.float32)
    op, ov = orc.train_points(dens, md, float(d[name + "_alpha"]), 0.857, 3, 60000, 40000)
    assert len(op) > 10000
    checks = [(np.linalg.norm(rp, axis=1), np.linalg.norm(op, axis=1), np.linspace(0, 0.5 * np.sqrt(3), 41))]
    for c in range(3):
        checks.append((rp[:, c], op[:, c], np.linspace(-0.51, 0.51, 41)))
        checks.append((rv[:, c], ov[:, c], np.linspace(-1.0, 1.0, 21)))
    for a, b, bins in checks:
        stat, dof = _two_sample_chi2(a, b, bins)
        assert chi2.sf(stat, dof) > 1e-4, (stat, dof)
