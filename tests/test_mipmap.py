"""Disparity mip-maps (CreateDispMipMaps + the packed mip-map surface): the
oracle's restatement against hand-computed values and the reference's layout
formulas, the C ABI's layout queries and argument checks (no GPU), and the
GPU kernels against the oracle bit-exactly."""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import to_dev


def test_layout_matches_reference_formulas(oracle):
    # DeviceSurfMipMap.cpp:130-132: x1 = W rounded up to 4, width x1 + (W - 1) / 2
    # _EvalMaxMipMapLevelCount: 1920x1080 -> 959x539, 479x269, 239x134, 119x66,
    # 59x32, 29x15, 14x7, 6x3, 2x1 -> 9 levels below level 0
    img, rects = oracle.disp_mipmaps(np.ones((1080, 1920), np.uint16), level_count=1)
    assert img.shape == (1080, 1920 + 959)
    assert len(rects) == 10
    assert rects[1] == (1920, 0, 959, 539)
    assert rects[2] == (1920, 539, 479, 269)
    assert rects[9] == (1920, 539 + 269 + 134 + 66 + 32 + 15 + 7 + 3, 2, 1)
    img, rects = oracle.disp_mipmaps(np.ones((6, 7), np.uint16), level_count=1)
    assert img.shape == (6, 8 + 3)
    assert rects == [(0, 0, 7, 6), (8, 0, 3, 2)]


def test_known_answers(oracle):
    # constant code 10 on 7x7: level 1 (3x3) = 0.5 * 10, level 2 (1x1) = 2.5;
    # with the default count (max = 2) level 2 is not written
    c = np.full((7, 7), 10, np.uint16)
    img, rects = oracle.disp_mipmaps(c, level_count=0)
    x, y, w, h = rects[1]
    np.testing.assert_array_equal(img[y:y + h, x:x + w], np.full((3, 3), 5.0, np.float32))
    x2, y2, _, _ = rects[2]
    assert img[y2, x2] == 0.0
    # unknown (0) and ID codes are skipped with their weights: row [0, 6, 0]
    # -> 6, row [4, 0xFFFF, 8] -> (4 + 8) / 2 = 6, row [3, 0, 0] -> 3;
    # vertically (6 + 2 * 6 + 3) / 4 = 5.25, times 0.5 (7x7 so that level 1 is
    # inside the default count: the reference writes levels 0 .. max - 1)
    c = np.array([[0, 6, 0], [4, 0xFFFF, 8], [3, 0, 0]], np.uint16)
    img, rects = oracle.disp_mipmaps(np.pad(c, ((0, 4), (0, 4))), level_count=2)
    x, y, _, _ = rects[1]
    assert img[y, x] == np.float32(2.625)
    np.testing.assert_array_equal(img[:3, :3], np.where((c >= 1) & (c <= 0xFFEF), c, 0).astype(np.float32))
    # all unknown -> 0; a 1/3 weight rounds in float32
    c = np.array([[0, 0, 0], [1, 0, 0], [0, 0, 0]], np.uint16)
    img, rects = oracle.disp_mipmaps(np.pad(c, ((0, 4), (0, 4))), level_count=2)
    assert img[rects[1][1], rects[1][0]] == np.float32(0.5)  # only h1 = 1 -> (2 * 1) / 2 * 0.5
    c = np.array([[1, 0, 0], [0, 0, 0], [2, 0, 0]], np.uint16)
    img, rects = oracle.disp_mipmaps(np.pad(c, ((0, 4), (0, 4))), level_count=2)
    assert img[rects[1][1], rects[1][0]] == np.float32(0.5) * (np.float32(3) / np.float32(2))


def test_level_count_rules(oracle):
    c = np.full((16, 16), 5, np.uint16)  # levels 7x7, 3x3, 1x1: max 3
    sentinel = np.full((16, 16 + 7), -7.0, np.float32)
    with pytest.raises(ValueError):
        oracle.disp_mipmaps(c, 4, sentinel)
    img, _ = oracle.disp_mipmaps(c, 1, sentinel)  # writes nothing
    np.testing.assert_array_equal(img, sentinel)
    img, rects = oracle.disp_mipmaps(c, 0, sentinel)  # max = 3: levels 0, 1, 2
    x, y, w, h = rects[2]
    assert (img[y:y + h, x:x + w] == np.float32(1.25)).all()
    x, y, w, h = rects[3]
    assert img[y, x] == np.float32(-7.0)


def test_division_by_three_through_double_is_correctly_rounded():
    # the kernels divide by the weight count 3 as float(double(s) * (1 / 3));
    # check it against IEEE float division over random floats of every
    # exponent the levels can hold and over the integers up to 2^24
    r = np.random.default_rng(3)
    bits = r.integers(0x3F000000 - (30 << 23), 0x47800000 + (10 << 23), 4_000_000, dtype=np.uint32)
    x = np.concatenate([bits.view(np.float32), np.arange(1, 1 << 24, 7, dtype=np.float32)])
    want = x / np.float32(3)
    got = (x.astype(np.float64) * (1.0 / 3.0)).astype(np.float32)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_capi_layout_queries(ct, oracle):
    for (W, H) in ((1920, 1080), (7, 6), (3, 3), (2, 9), (1, 1), (641, 479), (1000, 3)):
        opw, rects = oracle.mipmap_layout(W, H)
        pw, n = ct.disp_mipmap_format(W, H)
        assert pw == opw
        assert n == len(rects) - 1
        for k, r in enumerate(rects):
            assert ct.disp_mipmap_level(W, H, k) == r
        with pytest.raises(ct.CtError):
            ct.disp_mipmap_level(W, H, n + 1)


def test_capi_layout_sweep(ct, oracle):
    # the library's packed layout equals the reference's formulas for random sizes
    r = np.random.default_rng(12)
    for W, H in zip(r.integers(1, 9000, 300), r.integers(1, 9000, 300)):
        W, H = int(W), int(H)
        opw, rects = oracle.mipmap_layout(W, H)
        pw, n = ct.disp_mipmap_format(W, H)
        assert (pw, n) == (opw, len(rects) - 1)
        for k in (0, n // 2, n):
            x, y, w, h = ct.disp_mipmap_level(W, H, k)
            assert (x, y, w, h) == rects[k]
            assert x % 4 == 0 and y + h <= H and x + w <= pw  # 16-byte aligned, inside the image


def test_capi_argument_checks(ct):
    L = ct.lib()
    fake = 1 << 20  # never dereferenced: every check fails before a device call
    disp = ct.ct_image(C.c_void_p(fake), 64, 16, 16, ct.CT_PIX_U16, 0)
    mip = ct.ct_image(C.c_void_p(fake), 128, 23, 16, ct.CT_PIX_F32, 0)
    assert L.ct_disp_mipmaps(C.byref(mip), C.byref(disp), 4, None) == ct.CT_EINVAL  # max is 3
    bad = ct.ct_image(C.c_void_p(fake), 128, 22, 16, ct.CT_PIX_F32, 0)
    assert L.ct_disp_mipmaps(C.byref(bad), C.byref(disp), 0, None) == ct.CT_EFORMAT
    wrong = ct.ct_image(C.c_void_p(fake), 128, 23, 16, ct.CT_PIX_U16, 0)
    assert L.ct_disp_mipmaps(C.byref(wrong), C.byref(disp), 0, None) == ct.CT_ETYPE
    assert L.ct_disp_mipmaps(None, C.byref(disp), 0, None) == ct.CT_EINVAL
    assert L.ct_disp_mipmap_format(0, 5, None, None) == ct.CT_EINVAL


def _codes(H, W, seed):
    r = np.random.default_rng(seed)
    # a smooth disparity surface plus noise, 20% of the pixels IDs / unknown
    yy, xx = np.mgrid[0:H, 0:W]
    c = (40 + 30 * np.sin(xx / 37.0) + 20 * np.cos(yy / 23.0) + r.integers(0, 5, (H, W))).astype(np.uint16)
    ids = np.array([0, 0xFFFF, 0xFFFE, 0xFFFD, 0xFFFA, 0xFFF0, 0xFFEF, 1], np.uint16)
    m = r.random((H, W)) < 0.2
    c[m] = ids[r.integers(0, ids.size, m.sum())]
    return c


def _run(ct, cuda, dev_disp, W, H, level_count):
    pw, _ = ct.disp_mipmap_format(W, H)
    out = ct.alloc_image(H, pw, torch.float32, cuda)
    out.fill_(-7.0)
    ct.disp_mipmaps(out, dev_disp, level_count)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(1920, 1080), (641, 479), (200, 100), (2001, 29), (29, 2001), (37, 23), (16, 16),
                                 (8, 3), (5, 5), (2, 2)])
@pytest.mark.parametrize("level_count", [0, 1, 2, 3])
def test_mipmaps_match_oracle(ct, oracle, cuda, W, H, level_count):
    _, n = ct.disp_mipmap_format(W, H)
    codes = _codes(H, W, W * 7 + H)
    pw, _ = ct.disp_mipmap_format(W, H)
    sentinel = np.full((H, pw), -7.0, np.float32)
    if level_count > n:
        with pytest.raises(ct.CtError):
            _run(ct, cuda, to_dev(codes.view(np.int16), cuda), W, H, level_count)
        return
    got = _run(ct, cuda, to_dev(codes.view(np.int16), cuda), W, H, level_count)
    want, _ = oracle.disp_mipmaps(codes, level_count, sentinel)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
@pytest.mark.parametrize("W,H", [(1920, 1080), (641, 479), (200, 100)])
def test_mipmaps_default_count(ct, oracle, cuda, W, H):
    # every level the reference writes by default: two-level tiles, then the
    # shared-memory tail (1920x1080: levels 0-2, 3-4, 5-8; 200x100: 0-2, 3-4)
    codes = _codes(H, W, 11)
    pw, _ = ct.disp_mipmap_format(W, H)
    got = _run(ct, cuda, to_dev(codes.view(np.int16), cuda), W, H, 0)
    want, _ = oracle.disp_mipmaps(codes, 0, np.full((H, pw), -7.0, np.float32))
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_mipmaps_u8_input_and_full_depth(ct, oracle, cuda):
    H, W = 1080, 1920
    r = np.random.default_rng(5)
    u8 = r.integers(0, 128, (H, W)).astype(np.uint8)
    u8[r.random((H, W)) < 0.1] = 255
    codes = np.where(u8 == 255, 0xFFFF, u8.astype(np.int64) + 1).astype(np.uint16)
    _, n = ct.disp_mipmap_format(W, H)
    got = _run(ct, cuda, to_dev(u8, cuda), W, H, n)
    pw, _ = ct.disp_mipmap_format(W, H)
    want, _ = oracle.disp_mipmaps(codes, n, np.full((H, pw), -7.0, np.float32))
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))
