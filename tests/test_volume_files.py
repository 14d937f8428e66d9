"""Volume files (VolumeRender(string path), core/volume.cu:835-911): the
library's host parser against the oracle's restatement, on generated files,
and the load + render path on the GPU."""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import volfile_np
from internship_b200 import _lib, volume as V


def _write_txt(path, r, a, per_line=8):
    with open(path, "w") as f:
        f.write("%d\n" % r)
        for i in range(0, a.size, per_line):
            f.write(" ".join("%.7g" % x for x in a[i:i + per_line]) + "\n")


def _write_vox(path, vals):
    with open(path, "w") as f:
        f.write("w 256\nh 256\nd 256\n")
        for i in range(0, vals.size, 64):
            f.write(" ".join(str(int(x)) for x in vals[i:i + 64]) + "\n")


def test_txt_matches_oracle(tmp_path):
    r = 12
    a = np.random.default_rng(0).uniform(0, 3, r ** 3).astype(np.float32)
    p = str(tmp_path / "cloud_0.txt")
    _write_txt(p, r, a)
    ours = V.read_volume_file(p)
    rr, ref, from_bin = volfile_np.read(p)
    assert rr == r and not from_bin
    assert np.array_equal(ours.ravel(), ref)
    np.testing.assert_allclose(ours.ravel(), a, rtol=1e-6)


def test_vox_matches_oracle(tmp_path):
    vals = np.random.default_rng(1).integers(0, 256, 256 ** 3)
    p = str(tmp_path / "model.vox")
    _write_vox(p, vals)
    ours = V.read_volume_file(p)
    rr, ref, _ = volfile_np.read(p)
    assert ours.shape == (256, 256, 256) and rr == 256
    assert np.array_equal(ours.ravel(), ref)


def test_bin_cache_is_read_first(tmp_path):
    r = 6
    a = np.arange(r ** 3, dtype=np.float32)
    p = str(tmp_path / "x.txt")
    _write_txt(p, r, a)
    # a .bin beside it wins, as in the reference (convert.py writes this layout)
    b = a[::-1].copy()
    with open(p + ".bin", "wb") as f:
        f.write(np.int32(r).tobytes())
        f.write(b.tobytes())
    assert np.array_equal(V.read_volume_file(p).ravel(), b)
    assert np.array_equal(volfile_np.read(p)[1], b)


@pytest.mark.parametrize("case", ["missing", "truncated_bin", "short_txt", "bad_vox_line", "unknown_format"])
def test_bad_files_are_rejected(tmp_path, case):
    p = str(tmp_path / ("v.vox" if "vox" in case else "v.txt" if case != "unknown_format" else "v.raw"))
    if case == "truncated_bin":
        with open(p + ".bin", "wb") as f:
            f.write(np.int32(8).tobytes() + np.zeros(10, np.float32).tobytes())
    elif case == "short_txt":
        open(p, "w").write("4\n1 2 3\n")
    elif case == "bad_vox_line":
        open(p, "w").write("w 256\n1 2 3\n")
    elif case == "unknown_format":
        open(p, "w").write("4\n")
    with pytest.raises(_lib.MRError) as e:
        V.read_volume_file(p)
    assert e.value.code == _lib.MR_ERR_ARG


@pytest.mark.gpu
def test_load_renders_like_set_data(tmp_path):
    """mr_volume_load of a .txt file: same majorant and the same render as a
    volume filled with the same array; the .bin cache is written and read
    back identically."""
    import internship_b200 as mr
    from internship_b200 import scenes
    r = 32
    a = (scenes.sphere_density(r) * np.random.default_rng(2).uniform(0.5, 1.5, (r, r, r))).astype(np.float32)
    p = str(tmp_path / "sphere.txt")
    _write_txt(p, r, a.ravel())
    v1 = mr.VolumeRender(p)
    assert os.path.exists(p + ".bin")
    a_read = volfile_np.read(p)[1]  # now from the cache
    v2 = mr.VolumeRender(r)
    v2.SetDatas(a_read)
    v2.Update()
    assert v1.resolution == r and v1.max_density == v2.max_density
    q = scenes.make_params(16, 16, 8)
    o1, o2 = np.zeros(16 * 16 * 3, np.float32), np.zeros(16 * 16 * 3, np.float32)
    _lib.check(_lib.load().mr_render_host(v1.handle, None, C.byref(q), o1.ctypes.data))
    _lib.check(_lib.load().mr_render_host(v2.handle, None, C.byref(q), o2.ctypes.data))
    assert np.array_equal(o1, o2)
    v1.close()
    v2.close()
