"""Minimum disparity (the reference's xDispConfig.Min() / SAD1 iOffset): every
matcher searches dmin .. dmin + D - 1, matching base column x against
x -/+ d, and its maps hold the absolute disparity. Bit-exact against the
oracle for the census matcher (both directions, odd and even dmin, D over
several disparity blocks, and the cross-checked pipeline), SAD, NCC (plain
and guided) and the adaptive-window matcher (integer and sub-pixel, plain
and guided)."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu


def pair(ct, kind, seed, W, H, dmax):
    return ct.synth_pair(kind, seed, W, H, dmax)[:2]


CENSUS = [(131, 47, 64, 5, True), (131, 47, 64, 6, False), (333, 111, 100, 16, True),
          (257, 90, 128, 33, False), (640, 480, 64, 7, True), (200, 64, 7, 150, True)]


@pytest.mark.parametrize("W,H,D,dmin,lr", CENSUS)
def test_census_min_disparity(ct, oracle, cuda, W, H, D, dmin, lr):
    L, R = pair(ct, 2, W + D + dmin, W, H, dmin + D - 1)
    want, _ = oracle.match_census(L, R, D, 2, lr, dmin=dmin)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D, left_to_right=lr, disp_min=dmin)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    for dtype, enc in ((torch.uint8, oracle.to_u8), (torch.int16, oracle.to_u16)):
        if dtype == torch.uint8 and dmin + D > 255:
            continue
        out = ct.alloc_image(H, W, dtype, cuda)
        out.fill_(0x5A)
        m.process(out, dl, dr)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_array_equal(got.view(np.uint16) if dtype == torch.int16 else got, enc(want))
    assert m.device_status() == 0


@pytest.mark.parametrize("dmin", [3, 12])
def test_census_lr_crosscheck_min_disparity(ct, oracle, cuda, dmin):
    W, H, D = 400, 150, 96
    L, R = pair(ct, 2, 77 + dmin, W, H, dmin + D - 1)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D, disp_min=dmin)
    lr, rl, ck = (ct.alloc_image(H, W, torch.int16, cuda) for _ in range(3))
    m.process_lr(to_dev(L, cuda), to_dev(R, cuda), disp_lr=lr, disp_rl=rl, disp_checked=ck, tol=1)
    torch.cuda.synchronize()
    wl, _ = oracle.match_census(L, R, D, 2, True, dmin=dmin)
    wr, _ = oracle.match_census(L, R, D, 2, False, dmin=dmin)
    wc, _ = oracle.crosscheck(wl, wr, 1, True)
    for got, want in ((lr, wl), (rl, wr), (ck, wc)):
        np.testing.assert_array_equal(got.cpu().numpy().view(np.uint16), oracle.to_u16(want))


def test_census_u8_range_check(ct, cuda):
    m = ct.BlockMatcherCensus()
    m.configure(0, 64, 32, 64, disp_min=200)
    a = ct.alloc_image(32, 64, torch.uint8, cuda)
    with pytest.raises(ct.CtError) as e:
        m.process(a, a, a)
    assert e.value.code == ct.CT_ETYPE


@pytest.mark.parametrize("r,lr,dmin", [(4, True, 5), (4, False, 8), (1, True, 31), (2, False, 1)])
def test_sad_min_disparity(ct, oracle, cuda, r, lr, dmin):
    W, H, D = 203, 77, 70
    L, R = pair(ct, 1, 11 * r + dmin, W, H, dmin + D - 1)
    m = ct.BlockMatcherSAD1()
    m.configure(0, W, H, D, radius=r, left_to_right=lr, disp_min=dmin)
    out = ct.alloc_image(H, W, torch.int16, cuda)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    want, _ = oracle.match_sad(L, R, D, r, lr, dmin=dmin)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint16), oracle.to_u16(want))


@pytest.mark.parametrize("dmin", [9, 64])
def test_ncc_min_disparity(ct, oracle, cuda, dmin):
    W, H, D = 260, 90, 80
    L, R = pair(ct, 2, 5 + dmin, W, H, dmin + D - 1)
    m = ct.BlockMatcherNCC()
    m.configure(0, W, H, D, radius=5, disp_min=dmin)
    out = ct.alloc_image(H, W, torch.int16, cuda)
    score = ct.alloc_image(H, W, torch.float32, cuda)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    m.process(out, dl, dr, score=score)
    torch.cuda.synchronize()
    want, s32, _ = oracle.match_ncc(L, R, D, 5, dmin=dmin)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint16), oracle.to_u16(want))
    np.testing.assert_array_equal(score.cpu().numpy()[want >= 0], s32[want >= 0])
    # guided: a coarse map at 1/2 scale of the true disparities
    coarse = np.where(want[::2, ::2] >= 0, want[::2, ::2] // 2, -1).astype(np.int16)
    m.process(out, dl, dr, disp_init=to_dev(oracle.to_u16(coarse).view(np.int16), cuda))
    torch.cuda.synchronize()
    wg, _, _ = oracle.match_ncc_guided(L, R, D, coarse, 5, dmin=dmin)
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint16), oracle.to_u16(wg))


@pytest.mark.parametrize("dmin", [4, 17])
def test_aw_min_disparity(ct, oracle, cuda, dmin):
    W, H, D = 300, 80, 90
    L, R = pair(ct, 3, 3 + dmin, W, H, dmin + D - 1)
    m = ct.BlockMatcherAW()
    m.configure(0, W, H, D, disp_min=dmin)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    d16 = ct.alloc_image(H, W, torch.int16, cuda)
    f32 = ct.alloc_image(H, W, torch.float32, cuda)
    m.process(d16, dl, dr)
    m.process(f32, dl, dr)
    torch.cuda.synchronize()
    want, _, s32, s64 = oracle.match_aw(L, R, D, dmin=dmin)
    np.testing.assert_array_equal(d16.cpu().numpy().view(np.uint16), oracle.to_u16(want))
    np.testing.assert_array_equal(f32.cpu().numpy(), s32)
    ok = want >= 0
    assert np.abs(f32.cpu().numpy()[ok].astype(np.float64) - s64[ok]).max() < 1e-4
    coarse = np.where(want[::4, ::4] >= 0, want[::4, ::4] // 4, -1).astype(np.int16)
    m.process(f32, dl, dr, disp_init=to_dev(oracle.to_u16(coarse).view(np.int16), cuda))
    torch.cuda.synchronize()
    wg, _, g32, _ = oracle.match_aw_guided(L, R, D, coarse, dmin=dmin)
    np.testing.assert_array_equal(f32.cpu().numpy(), g32)
