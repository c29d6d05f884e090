"""Census path on the GPU against the CPU oracle: bit-exact descriptors,
disparity maps (both directions, U8 and U16 encodings) and cross-check."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu


def pair(ct, kind, seed, W, H, dmax):
    L, R, G, O = ct.synth_pair(kind, seed, W, H, dmax)
    return L, R


@pytest.mark.parametrize("W,H", [(67, 43), (640, 480), (1920, 1080)])
def test_census9x7_bit_exact(ct, oracle, cuda, W, H):
    L, _ = pair(ct, 2, 3, W, H, 64)
    ctr = ct.CensusTransform()
    ctr.configure(0, W, H, ct.CENSUS_9X7)
    src = to_dev(L, cuda)
    dst = ct.alloc_image(H, W, torch.int64, cuda)
    ctr.process(dst, src)
    torch.cuda.synchronize()
    got = dst.cpu().numpy().view(np.uint64)
    np.testing.assert_array_equal(got, oracle.census9x7(L))
    assert ctr.device_status() == 0


@pytest.mark.parametrize("W,H", [(131, 45), (640, 480)])
def test_census9x7_pair_launch_equals_two_calls(ct, oracle, cuda, W, H):
    L, R = pair(ct, 1, 9, W, H, 64)
    ctr = ct.CensusTransform()
    ctr.configure(0, W, H, ct.CENSUS_9X7)
    dl, dr = ct.alloc_image(H, W, torch.int64, cuda), ct.alloc_image(H, W, torch.int64, cuda)
    ctr.process_pair(dl, dr, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dl.cpu().numpy().view(np.uint64), oracle.census9x7(L))
    np.testing.assert_array_equal(dr.cpu().numpy().view(np.uint64), oracle.census9x7(R))
    assert ctr.device_status() == 0


def test_census3x3_reference_semantics(ct, oracle, cuda):
    W, H = 95, 61
    L, _ = pair(ct, 1, 4, W, H, 30)
    ctr = ct.CensusTransform()
    ctr.configure(0, W, H, ct.CENSUS_3X3)
    src = to_dev(L, cuda)
    dst = ct.alloc_image(H, W, torch.uint8, cuda)
    dst.fill_(0xAB)
    ctr.process(dst, src)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(dst.cpu().numpy(), oracle.census3x3(L, fill=0xAB))


CASES = [
    # W, H, D, generator kind
    (67, 43, 13, 1),
    (130, 37, 64, 1),     # exactly one CTA of disparities
    (333, 111, 128, 2),   # two disparity CTAs merged through global keys
    (257, 90, 200, 2),    # partial last warp group
    (96, 64, 1, 1),       # D = 1
    (640, 480, 64, 1),
]


@pytest.mark.parametrize("W,H,D,kind", CASES)
@pytest.mark.parametrize("lr", [True, False])
def test_census_match_bit_exact(ct, oracle, cuda, W, H, D, kind, lr):
    L, R = pair(ct, kind, W * 7 + D, W, H, max(1, D - 1))
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D, left_to_right=lr)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    want, _ = oracle.match_census(L, R, D, 2, lr)
    for dtype, enc in ((torch.uint8, oracle.to_u8), (torch.int16, oracle.to_u16)):
        if dtype == torch.uint8 and D > 255:
            continue
        out = ct.alloc_image(H, W, dtype, cuda)
        out.fill_(0x5A)
        m.process(out, dl, dr)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        if dtype == torch.int16:
            got = got.view(np.uint16)
        np.testing.assert_array_equal(got, enc(want))
    assert m.device_status() == 0


def test_census_match_full_size_1080p_d128(ct, oracle, cuda):
    W, H, D = 1920, 1080, 128
    L, R = pair(ct, 2, 2024, W, H, D - 1)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    out = ct.alloc_image(H, W, torch.uint8, cuda)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    want, _ = oracle.match_census(L, R, D)
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.to_u8(want))


def test_process_lr_and_crosscheck(ct, oracle, cuda):
    W, H, D = 400, 150, 96
    L, R = pair(ct, 2, 77, W, H, D - 1)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    lr = ct.alloc_image(H, W, torch.int16, cuda)
    rl = ct.alloc_image(H, W, torch.int16, cuda)
    ck = ct.alloc_image(H, W, torch.int16, cuda)
    m.process_lr(dl, dr, disp_lr=lr, disp_rl=rl, disp_checked=ck, tol=1)
    torch.cuda.synchronize()
    wl, _ = oracle.match_census(L, R, D, 2, True)
    wr, _ = oracle.match_census(L, R, D, 2, False)
    wc, _ = oracle.crosscheck(wl, wr, 1, True)
    np.testing.assert_array_equal(lr.cpu().numpy().view(np.uint16), oracle.to_u16(wl))
    np.testing.assert_array_equal(rl.cpu().numpy().view(np.uint16), oracle.to_u16(wr))
    np.testing.assert_array_equal(ck.cpu().numpy().view(np.uint16), oracle.to_u16(wc))
    # checked map only (internal scratch maps), U8
    ck8 = ct.alloc_image(H, W, torch.uint8, cuda)
    m.process_lr(dl, dr, disp_checked=ck8, tol=1)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ck8.cpu().numpy(), oracle.to_u8(np.where(wc == -2, -1, wc)))


@pytest.mark.parametrize("dtype", [torch.uint8, torch.int16])
def test_crosscheck_driver_and_range(ct, oracle, cuda, dtype):
    W, H, D = 300, 120, 48
    L, R = pair(ct, 1, 5, W, H, D - 1)
    wl, _ = oracle.match_census(L, R, D, 2, True)
    wr, _ = oracle.match_census(L, R, D, 2, False)
    enc = oracle.to_u8 if dtype == torch.uint8 else oracle.to_u16
    base, other = to_dev(enc(wl).view(np.int16) if dtype == torch.int16 else enc(wl), cuda), \
        to_dev(enc(wr).view(np.int16) if dtype == torch.int16 else enc(wr), cuda)
    cc = ct.CrossCheckDisparityMaps()
    cc.configure(0, W, H, ct.CT_PIX_U8 if dtype == torch.uint8 else ct.CT_PIX_U16, disp_delta_thresh=1)
    res = ct.alloc_image(H, W, dtype, cuda)
    res.fill_(0x5A)
    cc.process(res, base, other)
    lo, hi = cc.disp_range()
    want, (wlo, whi) = oracle.crosscheck(wl, wr, 1, True)
    got = res.cpu().numpy()
    if dtype == torch.int16:
        got, want = got.view(np.uint16), oracle.to_u16(want)
    else:
        want = oracle.to_u8(np.where(want == -2, -1, want))
    # the driver leaves the 1-pixel frame unwritten, as the reference kernel
    np.testing.assert_array_equal(got[1:-1, 1:-1], want[1:-1, 1:-1])
    frame = np.ones((H, W), bool)
    frame[1:-1, 1:-1] = False
    assert (got[frame] == 0x5A).all()
    assert (lo, hi) == (wlo, whi)


@pytest.mark.parametrize("W,H,D,tol,lr", [(37, 23, 8, 1, True), (300, 77, 40, 0, False), (129, 64, 5, 12, True),
                                          (1920, 1080, 128, 1, True)])
def test_crosscheck_driver_reference_rule_on_codes(ct, oracle, cuda, W, H, D, tol, lr):
    """U16 code maps with Unknown and IDs mixed in: the driver follows the
    reference rule exactly (raw code compare, frame unwritten, range over the
    kept codes), as the oracle that tests/test_ref_pin.py pins to the
    reference's own kernel."""
    rng = np.random.default_rng(W + H + D)

    def codes():
        c = rng.integers(1, D + 1, (H, W)).astype(np.uint16)
        m = rng.random((H, W))
        c[m < 0.05] = 0xFFFF
        c[(m >= 0.05) & (m < 0.09)] = 0
        c[(m >= 0.09) & (m < 0.11)] = 0xFFFA
        c[(m >= 0.12) & (m < 0.13)] = 0xFFEF
        return c

    a, b = codes(), codes()
    init = rng.integers(0, 65536, (H, W)).astype(np.uint16)
    cc = ct.CrossCheckDisparityMaps()
    cc.configure(0, W, H, ct.CT_PIX_U16, disp_delta_thresh=tol, left_to_right=lr)
    res = to_dev(init.view(np.int16), cuda)
    cc.process(res, to_dev(a.view(np.int16), cuda), to_dev(b.view(np.int16), cuda))
    lo, hi = cc.disp_range()
    want, (wlo, whi) = oracle.crosscheck_codes(a, b, tol, lr, frame=True, out=init)
    np.testing.assert_array_equal(res.cpu().numpy().view(np.uint16), want)
    if wlo <= whi:
        assert (lo, hi) == (wlo - 1, whi - 1)
    else:
        assert lo > hi


def test_format_mismatch_is_an_error(ct, cuda):
    m = ct.BlockMatcherCensus()
    m.configure(0, 64, 32, 16)
    a = ct.alloc_image(32, 64, torch.uint8, cuda)
    b = ct.alloc_image(31, 64, torch.uint8, cuda)
    with pytest.raises(ct.CtError) as e:
        m.process(a, a, b)
    assert e.value.code == ct.CT_EFORMAT
    f = ct.alloc_image(32, 64, torch.float32, cuda)
    with pytest.raises(ct.CtError) as e:
        m.process(f, a, a)
    assert e.value.code == ct.CT_ETYPE


@pytest.mark.parametrize("dpw", [4, 8])
@pytest.mark.parametrize("th", [11, 36, 121, 511])
def test_every_launch_shape_is_bit_exact(ct, oracle, cuda, dpw, th):
    """Results do not depend on the kernel variant or strip height."""
    W, H, D = 301, 157, 100
    L, R = pair(ct, 2, 9, W, H, D - 1)
    want, _ = oracle.match_census(L, R, D, 2, True)
    wrl, _ = oracle.match_census(L, R, D, 2, False)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    m.set_tuning(th, dpw)
    assert m.tuning() == {"strip_height": th, "disp_per_warp": dpw}
    lr = ct.alloc_image(H, W, torch.uint8, cuda)
    rl = ct.alloc_image(H, W, torch.uint8, cuda)
    m.process_lr(to_dev(L, cuda), to_dev(R, cuda), disp_lr=lr, disp_rl=rl)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(lr.cpu().numpy(), oracle.to_u8(want))
    np.testing.assert_array_equal(rl.cpu().numpy(), oracle.to_u8(wrl))


def test_autotune_keeps_results(ct, oracle, cuda):
    W, H, D = 640, 480, 64
    L, R = pair(ct, 1, 21, W, H, D - 1)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    t = m.autotune(dl, dr)
    assert t["disp_per_warp"] in (4, 8) and (t["strip_height"] + 4) % 5 == 0
    out = ct.alloc_image(H, W, torch.uint8, cuda)
    m.process(out, dl, dr)
    torch.cuda.synchronize()
    want, _ = oracle.match_census(L, R, D)
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.to_u8(want))
    with pytest.raises(ct.CtError):
        m.set_tuning(12, 4)


@pytest.mark.parametrize("W,H,D,dmin,kind,dtype", [
    (67, 43, 40, 0, 1, torch.int16),     # one column tile, D below one disparity block
    (400, 150, 96, 0, 2, torch.int16),   # D split over two blocks (last-arriver merge)
    (333, 111, 128, 5, 1, torch.int16),  # odd minimum disparity (relative d = 0 excluded)
    (515, 97, 200, 2, 2, torch.uint8),   # ragged D and width, U8 maps
    (1280, 720, 256, 0, 2, torch.int16),
])
def test_process_lr_fused_equals_two_passes(ct, oracle, cuda, W, H, D, dmin, kind, dtype):
    """ct_bm_census_process_lr decides both directions in one pass (the right
    view's winners from the left-to-right costs); its three maps equal the
    two-pass result and, where the oracle is quick, the oracle's."""
    L, R = pair(ct, kind, 1000 + W, W, H, dmin + D - 1)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D, disp_min=dmin)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    maps = {}
    for fused in (True, False):
        m.set_fused_lr(fused)
        out = [ct.alloc_image(H, W, dtype, cuda) for _ in range(3)]
        for o in out:
            o.fill_(0x5A5A if dtype == torch.int16 else 0x5A)
        m.process_lr(dl, dr, disp_lr=out[0], disp_rl=out[1], disp_checked=out[2], tol=1)
        torch.cuda.synchronize()
        assert m.device_status() == 0
        maps[fused] = [o.cpu().numpy() for o in out]
    for a, b, name in zip(maps[True], maps[False], ("lr", "rl", "checked")):
        np.testing.assert_array_equal(a, b, err_msg=name)
    if W * H * D <= 400 * 150 * 128:
        wl, _ = oracle.match_census(L, R, D, 2, True, dmin=dmin)
        wr, _ = oracle.match_census(L, R, D, 2, False, dmin=dmin)
        wc, _ = oracle.crosscheck(wl, wr, 1, True)
        enc = (lambda v: oracle.to_u16(v)) if dtype == torch.int16 else (
            lambda v: oracle.to_u8(np.where(v == -2, -1, v)))
        for got, want, name in zip(maps[True], (wl, wr, wc), ("lr", "rl", "checked")):
            view = got.view(np.uint16) if dtype == torch.int16 else got
            np.testing.assert_array_equal(view, enc(want), err_msg=name)


@pytest.mark.parametrize("W,H,D,dmin", [
    (8, 8, 1, 0),        # smallest image, one disparity
    (16, 9, 3, 1),       # odd minimum disparity, D tiny
    (96, 64, 1, 0),      # D = 1
    (130, 37, 64, 0),    # exactly one block of disparities, two column tiles
    (124, 40, 65, 0),    # one column tile, D one past a block
    (60, 30, 20, 50),    # minimum disparity close to the width: most pixels search nothing
    (50, 20, 10, 60),    # minimum disparity beyond the width: no disparity anywhere
])
def test_process_lr_fused_edge_shapes(ct, oracle, cuda, W, H, D, dmin):
    """The fused pass on degenerate shapes: all three maps equal the two-pass
    result and the oracle's."""
    L, R = pair(ct, 1, 500 + W + D, W, H, max(1, dmin + D - 1))
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D, disp_min=dmin)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    maps = {}
    for fused in (True, False):
        m.set_fused_lr(fused)
        out = [ct.alloc_image(H, W, torch.int16, cuda) for _ in range(3)]
        for o in out:
            o.fill_(0x2B2B)
        m.process_lr(dl, dr, disp_lr=out[0], disp_rl=out[1], disp_checked=out[2], tol=1)
        torch.cuda.synchronize()
        assert m.device_status() == 0
        maps[fused] = [o.cpu().numpy().view(np.uint16) for o in out]
    wl, _ = oracle.match_census(L, R, D, 2, True, dmin=dmin)
    wr, _ = oracle.match_census(L, R, D, 2, False, dmin=dmin)
    wc, _ = oracle.crosscheck(wl, wr, 1, True)
    for k, (want, name) in enumerate(zip((wl, wr, wc), ("lr", "rl", "checked"))):
        np.testing.assert_array_equal(maps[True][k], maps[False][k], err_msg=name)
        np.testing.assert_array_equal(maps[True][k], oracle.to_u16(want), err_msg=name)


@pytest.mark.parametrize("dtype", [torch.uint8, torch.int16])
def test_process_lr_fused_many_calls(ct, cuda, dtype):
    """The fused pass keeps the right view's keys between calls and tells this
    call's apart by a tag that wraps every 32 calls. Over 70 calls that
    alternate two pairs (with different disparity ranges, so a stale key
    would change a map) and the subsets of outputs, every map equals the
    two-pass one."""
    W, H, D = 300, 70, 64
    pairs = [pair(ct, 1, 31, W, H, D - 1), pair(ct, 2, 32, W, H, 20)]
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    dev = [(to_dev(L, cuda), to_dev(R, cuda)) for L, R in pairs]
    want = []
    m.set_fused_lr(False)
    for dl, dr in dev:
        out = [ct.alloc_image(H, W, dtype, cuda) for _ in range(3)]
        m.process_lr(dl, dr, disp_lr=out[0], disp_rl=out[1], disp_checked=out[2], tol=1)
        want.append([o.cpu().numpy() for o in out])
    m.set_fused_lr(True)
    out = [ct.alloc_image(H, W, dtype, cuda) for _ in range(3)]
    for call in range(70):
        k = call % 2
        dl, dr = dev[k]
        for o in out:
            o.fill_(0x1234 if dtype == torch.int16 else 0x5A)
        mode = (call // 2) % 3
        if mode == 0:
            m.process_lr(dl, dr, disp_lr=out[0], disp_rl=out[1], disp_checked=out[2], tol=1)
            check = (0, 1, 2)
        elif mode == 1:
            m.process_lr(dl, dr, disp_rl=out[1], disp_checked=out[2], tol=1)
            check = (1, 2)
        else:
            m.process_lr(dl, dr, disp_lr=out[0], disp_rl=out[1])
            check = (0, 1)
        torch.cuda.synchronize()
        for i in check:
            np.testing.assert_array_equal(out[i].cpu().numpy(), want[k][i], err_msg=f"call {call} map {i}")
    assert m.device_status() == 0
