"""CPU tests of the C ABI surface and host logic (no kernel launches)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, reference_file
import internship_b200 as mr
from internship_b200 import _lib, weights as W, scenes


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        txt = open(os.path.join(ROOT, "include", f)).read()
        names |= set(re.findall(r"^(?:int|const char\*)\s+(mr_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    declared = _declared()
    assert declared == set(_lib.EXPORTS)
    for name in declared:
        assert hasattr(L, name), name


def test_version_and_error_string():
    L = _lib.load()
    assert b"sm_100a" in L.mr_version()
    h = C.c_void_p()
    assert L.mr_volume_create(-3, C.byref(h)) == _lib.MR_ERR_ARG
    assert b"resolution" in L.mr_last_error()


def test_network_rejects_bad_blob():
    L = _lib.load()
    h = C.c_void_p()
    w = np.zeros(100, np.float32)
    assert L.mr_network_create(w.ctypes.data, w.size, None, C.byref(h)) == _lib.MR_ERR_ARG
    w = np.zeros(_lib.WEIGHT_TOTAL, np.float32)
    w[5] = np.nan
    assert L.mr_network_create(w.ctypes.data, w.size, None, C.byref(h)) == _lib.MR_ERR_ARG
    assert b"finite" in L.mr_last_error()


def test_xavier_weights_deterministic_and_scaled():
    a, b = mr.xavier_weights(1), mr.xavier_weights(1)
    assert (a == b).all() and not (a == mr.xavier_weights(2)).all()
    lay = W.layout()
    off = 0
    for name, n in lay:
        seg = a[off:off + n]
        if name.endswith("B"):
            assert (seg == 0).all()
        elif name == "LC0W":
            lim = np.sqrt(6 / 256)
            assert np.abs(seg).max() <= lim and seg.std() > 0.5 * lim / np.sqrt(3)
        off += n
    assert off == _lib.WEIGHT_TOTAL


@pytest.mark.parametrize("which", ["builtin", "spiral"])
def test_stencil_shape(which):
    s = (mr.builtin_stencil() if which == "builtin" else mr.spiral_stencil()).reshape(160, 3)
    r = np.linalg.norm(s, axis=1)
    assert r[0] == 0
    np.testing.assert_allclose(r[1:64], 1.0, atol=1e-6)
    assert (r[64:] <= 1.0 + 1e-6).all() and (r[64:] > 0.3).all()


def test_default_stencil_is_the_reference_table():
    """mr_network_create(stencil=NULL) gathers at the reference's own 160
    directions (core/vector.cu:77-172), bit for bit as the compiler reads them."""
    st = W.load_stencil_source(reference_file("core/vector.cu"))
    assert np.array_equal(mr.builtin_stencil(), st)
    assert not np.array_equal(mr.spiral_stencil(), st)


def test_layout_matches_header_total():
    lay = W.layout()
    assert len(lay) == 146 and sum(n for _, n in lay) == 49673


def test_parse_reference_weight_header_and_stencil():
    blob = W.load_nnweight_header(reference_file("core/NNWeight.cuh"))
    assert blob.size == 49673
    assert blob[0] == np.float32(0.6143062)
    st = W.load_stencil_source(reference_file("core/vector.cu"))
    assert st.size == 480 and tuple(st[3:6]) == (1.0, 0.0, 0.0)


def test_blob_roundtrip(tmp_path):
    w = mr.xavier_weights(3)
    st = mr.builtin_stencil()
    W.save_blob(str(tmp_path / "w.bin"), w, st)
    w2, st2 = W.load_blob(str(tmp_path / "w.bin"))
    assert (w == w2).all() and (st == st2).all()


def test_cloud_permutation_is_permutation():
    p = scenes.cloud_permutation(11)
    assert sorted(p.tolist()) == list(range(256))


def test_camera_vectors_match_reference_convention():
    ori, up, right = scenes.camera_vectors((0.0, 0.0, 2.5), 90.0)
    np.testing.assert_allclose(right, (-1, 0, 0), atol=1e-12)
    np.testing.assert_allclose(up, (0, 1, 0), atol=1e-12)


def test_aces_tonemap_range():
    x = np.array([[0.0, 0.0, 0.0], [0.18, 0.18, 0.18], [10.0, 5.0, 1.0]], np.float32)
    t = mr.tone_aces(x)
    assert t.shape == x.shape and (t >= 0).all() and t[0].max() < 1e-3 and t[2].max() <= 1.05


def test_bmp_writer(tmp_path):
    img = np.zeros((3, 4, 3), np.uint8)
    img[0, 0] = (255, 0, 0)
    mr.save_bmp(str(tmp_path / "x"), img)
    b = open(tmp_path / "x.bmp", "rb").read()
    assert b[:2] == b"BM" and len(b) == 54 + 3 * 4 * 4 and b[54:58] == bytes([0, 0, 255, 255])
