"""Disparity to 3D (MapDisparityTo3D with explicit pinhole cameras): the FP64
oracle against the analytic depth of a rectified pair, the C ABI's argument
checks (no GPU), and the GPU kernel against the oracle (FP32 against FP64,
relative tolerance 2e-4 of the point's distance, for rays at least 0.01 rad
apart) for U16, U8 and F32 maps, both output coordinate systems and a verged
camera pair. Parity of the camera model itself is unpinned: the reference's
camera class is not in the reference tree."""
import ctypes as C
import math

import numpy as np
import pytest
import torch

from conftest import to_dev

F, CX, CY, B = 800.0, 320.0, 240.0, 0.12
RECT = [(F, F, CX, CY, np.eye(3), (0.0, 0.0, 0.0)), (F, F, CX, CY, np.eye(3), (B, 0.0, 0.0))]


def _roty(deg):
    a = math.radians(deg)
    return np.array([[math.cos(a), 0, math.sin(a)], [0, 1, 0], [-math.sin(a), 0, math.cos(a)]])


VERGED = [(810.0, 805.0, 330.0, 236.0, _roty(1.5), (0.0, 0.0, 0.0)),
          (790.0, 795.0, 312.0, 244.0, _roty(-1.5), (0.1, 0.002, -0.003))]


def _codes(H, W, seed, lo=8, hi=100):
    r = np.random.default_rng(seed)
    c = r.integers(lo + 1, hi + 2, (H, W)).astype(np.uint16)
    c[r.random((H, W)) < 0.1] = 0xFFFF
    c[r.random((H, W)) < 0.02] = 0xFFFA
    return c


def test_oracle_rectified_known_answer(oracle):
    # Z = f B / d, X = (x - cx) Z / f, Y = (y - cy) Z / f
    codes = np.array([[11, 21, 0xFFFF], [41, 1, 81]], np.uint16)
    out, rng, hit = oracle.map3d(codes, RECT, 1, 0xFFEF)
    for (y, x) in [(0, 0), (0, 1), (1, 0), (1, 2)]:
        d = float(codes[y, x]) - 1
        Z = F * B / d
        np.testing.assert_allclose(out[y, x, :3], [(x - CX) * Z / F, (y - CY) * Z / F, Z], rtol=1e-12)
        assert out[y, x, 3] == 1.0
    assert not hit[1, 1] and (out[1, 1] == 0).all()          # d = 0: parallel rays
    assert out[0, 2, 3] == 0.0 and hit[0, 2]                   # invalid: disparity disp_min (= 1), alpha 0
    np.testing.assert_allclose(out[0, 2, 2], F * B / 1.0)
    rut, _, _ = oracle.map3d(codes, RECT, 1, 0xFFEF, cs_rut=True)
    np.testing.assert_allclose(rut[..., :3], out[..., :3] * np.array([1, -1, -1]))
    good = out[..., 3] == 1
    np.testing.assert_allclose(rng[0], out[good][:, :3].min(0))
    np.testing.assert_allclose(rng[1], out[good][:, :3].max(0))


def test_capi_argument_checks(ct):
    L = ct.lib()
    h = C.c_void_p()
    assert L.ct_map3d_create(C.byref(h)) == ct.CT_OK
    cams = (ct.ct_pinhole * 2)(ct.pinhole(F, F, CX, CY), ct.pinhole(F, F, CX, CY, center=(B, 0, 0)))
    fmt = ct.ct_format(64, 32, ct.CT_PIX_U16)
    bad_type = ct.ct_format(64, 32, ct.CT_PIX_RGBA8)
    assert L.ct_map3d_configure(h, 0, C.byref(bad_type), C.byref(ct.ct_map3d_params(1, 100, 0, 0, cams))) == ct.CT_ETYPE
    assert L.ct_map3d_configure(h, 0, C.byref(fmt), C.byref(ct.ct_map3d_params(1, 100, 0, 7, cams))) == ct.CT_EINVAL
    assert L.ct_map3d_configure(h, 0, C.byref(fmt), C.byref(ct.ct_map3d_params(9, 3, 0, 0, cams))) == ct.CT_EINVAL
    zero = (ct.ct_pinhole * 2)(ct.pinhole(0, F, CX, CY), ct.pinhole(F, F, CX, CY))
    assert L.ct_map3d_configure(h, 0, C.byref(fmt), C.byref(ct.ct_map3d_params(1, 100, 0, 0, zero))) == ct.CT_EINVAL
    assert L.ct_map3d_configure(h, 0, C.byref(fmt), None) == ct.CT_EINVAL
    assert L.ct_map3d_process(h, None, None, None) == ct.CT_ESTATE  # not configured
    lo, hi = (C.c_float * 3)(), (C.c_float * 3)()
    assert L.ct_map3d_range(h, lo, hi) == ct.CT_ESTATE
    c = C.c_void_p()
    assert L.ct_crosscheck_create(C.byref(c)) == ct.CT_OK
    assert L.ct_map3d_process(c, None, None, None) == ct.CT_ESTATE  # wrong handle kind
    L.ct_destroy(c)
    L.ct_destroy(h)


def _cams(ct, cams):
    return [ct.pinhole(fx, fy, cx, cy, R, c) for (fx, fy, cx, cy, R, c) in cams]


def _check(got, want, hit, rtol=2e-4):
    dist = np.linalg.norm(want[..., :3], axis=-1, keepdims=True)
    err = np.abs(got[..., :3] - want[..., :3])
    assert (err <= rtol * dist + 1e-6).all(), float((err / (dist + 1e-12)).max())
    np.testing.assert_array_equal(got[..., 3], want[..., 3])
    assert (got[~hit] == 0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("cams_name,cs_rut", [("rect", False), ("rect", True), ("verged", False)])
def test_map3d_u16_matches_oracle(ct, oracle, cuda, cams_name, cs_rut):
    cams = RECT if cams_name == "rect" else VERGED
    H, W = 480, 640
    codes = _codes(H, W, 5)
    m = ct.MapDisparityTo3D()
    m.configure(0, W, H, *_cams(ct, cams), disp_min=1, disp_max=0xFFEF, cs_rut=cs_rut)
    out = ct.alloc_map3d(H, W, cuda)
    m.process(out, to_dev(codes.view(np.int16), cuda))
    lo, hi = m.range()
    got = out.cpu().numpy().astype(np.float64)
    want, rng, hit = oracle.map3d(codes, cams, 1, 0xFFEF, cs_rut)
    _check(got, want, hit)
    scale = np.abs(np.concatenate([rng[0], rng[1]])).max()
    np.testing.assert_allclose(lo, rng[0], atol=2e-4 * scale)
    np.testing.assert_allclose(hi, rng[1], atol=2e-4 * scale)


@pytest.mark.gpu
def test_map3d_u8_f32_inputs_and_range_limits(ct, oracle, cuda):
    H, W = 200, 333
    r = np.random.default_rng(9)
    u8 = r.integers(8, 120, (H, W)).astype(np.uint8)
    u8[r.random((H, W)) < 0.1] = 255
    codes = np.where(u8 == 255, 0xFFFF, u8.astype(np.int64) + 1)
    # only codes 20 .. 90 are valid; the others use disparity disp_min = 20
    m = ct.MapDisparityTo3D()
    m.configure(0, W, H, *_cams(ct, RECT), disp_min=20, disp_max=90, type_=ct.CT_PIX_U8)
    out = ct.alloc_map3d(H, W, cuda)
    m.process(out, to_dev(u8, cuda))
    want, _, hit = oracle.map3d(codes, RECT, 20, 90)
    _check(out.cpu().numpy().astype(np.float64), want, hit)
    # F32 sub-pixel map (negative = invalid)
    f = (u8.astype(np.float32) + r.random((H, W)).astype(np.float32)).astype(np.float32)
    f[u8 == 255] = -1.0
    m2 = ct.MapDisparityTo3D()
    m2.configure(0, W, H, *_cams(ct, RECT), type_=ct.CT_PIX_F32)
    out2 = ct.alloc_map3d(H, W, cuda)
    m2.process(out2, to_dev(f, cuda))
    fcodes = np.where(f >= 0, f.astype(np.float64) + 1, 0xFFFF)
    want2, _, hit2 = oracle.map3d(fcodes, RECT, 1, 0xFFEF)
    _check(out2.cpu().numpy().astype(np.float64), want2, hit2)
    # no valid pixel: the range keeps its reset values
    m3 = ct.MapDisparityTo3D()
    m3.configure(0, W, H, *_cams(ct, RECT), disp_min=200, disp_max=210, type_=ct.CT_PIX_U8)
    m3.process(out, to_dev(u8, cuda))
    lo, hi = m3.range()
    assert lo == (pytest.approx(3.4028234663852886e38),) * 3 and hi == (pytest.approx(-3.4028234663852886e38),) * 3
