"""SAD, adaptive-window (+ sub-pixel) and NCC matchers on the GPU against the
CPU oracle. Integer disparities are bit-exact; FP32 scores and sub-pixel
disparities are compared with the FP64 oracle at an absolute tolerance of
1e-4 (the maximum error seen is printed), and with the FP32 restatement
bit-exactly (same IEEE operations)."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu

TOL = 1e-4


def run_sad(ct, cuda, L, R, D, r, lr, dtype):
    H, W = L.shape
    m = ct.BlockMatcherSAD1()
    m.configure(0, W, H, D, radius=r, left_to_right=lr)
    out = ct.alloc_image(H, W, dtype, cuda)
    out.fill_(0x5A)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    assert m.device_status() == 0
    got = out.cpu().numpy()
    return got.view(np.uint16) if dtype == torch.int16 else got


@pytest.mark.parametrize("W,H,D,r", [(67, 43, 13, 4), (640, 480, 64, 4), (300, 100, 100, 4), (129, 70, 64, 1),
                                     (129, 70, 65, 2), (200, 50, 30, 3)])
@pytest.mark.parametrize("lr", [True, False])
def test_sad_bit_exact(ct, oracle, cuda, W, H, D, r, lr):
    L, R, _, _ = ct.synth_pair(1, W + D, W, H, D - 1)
    want, _ = oracle.match_sad(L, R, D, r, lr)
    np.testing.assert_array_equal(run_sad(ct, cuda, L, R, D, r, lr, torch.uint8), oracle.to_u8(want))
    np.testing.assert_array_equal(run_sad(ct, cuda, L, R, D, r, lr, torch.int16), oracle.to_u16(want))


def test_sad_config1_accuracy(ct, oracle, cuda):
    """640x480, D = 64, 9x9: bit-exact and mostly right against ground truth."""
    L, R, G, O = ct.synth_pair(1, 1, 640, 480, 63)
    got = run_sad(ct, cuda, L, R, 64, 4, True, torch.uint8)
    want, _ = oracle.match_sad(L, R, 64, 4, True)
    np.testing.assert_array_equal(got, oracle.to_u8(want))
    v = (got != 255) & (O == 0)
    assert (np.abs(got[v].astype(int) - G[v]) <= 1).mean() > 0.8


def run_aw(ct, cuda, L, R, D, dtype):
    H, W = L.shape
    m = ct.BlockMatcherAW()
    m.configure(0, W, H, D)
    out = ct.alloc_image(H, W, dtype, cuda)
    out.fill_(0)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    assert m.device_status() == 0
    got = out.cpu().numpy()
    return got.view(np.uint16) if dtype == torch.int16 else got


@pytest.mark.parametrize("W,H,D", [(67, 43, 13), (300, 120, 100), (640, 200, 256)])
def test_aw_integer_and_subpixel(ct, oracle, cuda, W, H, D):
    L, R, _, _ = ct.synth_pair(3, W * 3 + D, W, H, D - 1)
    d, c, s32, s64 = oracle.match_aw(L, R, D)
    if D <= 255:
        np.testing.assert_array_equal(run_aw(ct, cuda, L, R, D, torch.uint8), oracle.to_u8(d))
    np.testing.assert_array_equal(run_aw(ct, cuda, L, R, D, torch.int16), oracle.to_u16(d))
    sub = run_aw(ct, cuda, L, R, D, torch.float32)
    np.testing.assert_array_equal(sub, s32)  # same IEEE operations
    v = d >= 0
    err = np.abs(sub[v].astype(np.float64) - s64[v]).max()
    print(f"AW {W}x{H} D={D}: max |sub32 - sub64| = {err:.3g}")
    assert err <= TOL


@pytest.mark.slow
def test_aw_config3_full_size(ct, oracle, cuda):
    W, H, D = 2560, 1440, 256
    L, R, G, O = ct.synth_pair(3, 33, W, H, D - 1)
    d, c, s32, s64 = oracle.match_aw(L, R, D)
    sub = run_aw(ct, cuda, L, R, D, torch.float32)
    v = d >= 0
    np.testing.assert_array_equal(sub, s32)
    err = np.abs(sub[v].astype(np.float64) - s64[v]).max()
    print(f"AW 2560x1440 D=256: max |sub32 - sub64| = {err:.3g}")
    assert err <= TOL


def run_ncc(ct, cuda, L, R, D, r, dtype=torch.uint8):
    H, W = L.shape
    m = ct.BlockMatcherNCC()
    m.configure(0, W, H, D, radius=r)
    out = ct.alloc_image(H, W, dtype, cuda)
    score = ct.alloc_image(H, W, torch.float32, cuda)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda), score=score)
    torch.cuda.synchronize()
    assert m.device_status() == 0
    got = out.cpu().numpy()
    return (got.view(np.uint16) if dtype == torch.int16 else got), score.cpu().numpy()


@pytest.mark.parametrize("W,H,D,r", [(67, 43, 13, 5), (400, 150, 96, 5), (150, 60, 40, 4), (150, 60, 70, 2)])
def test_ncc(ct, oracle, cuda, W, H, D, r):
    L, R, _, _ = ct.synth_pair(2, W + 5 * D, W, H, D - 1)
    L[5:25, 5:30] = 128  # flat patch: the sigma < 1 rule
    d, s32, s64 = oracle.match_ncc(L, R, D, r)
    got, score = run_ncc(ct, cuda, L, R, D, r)
    np.testing.assert_array_equal(got, oracle.to_u8(d))
    v = d >= 0
    np.testing.assert_array_equal(score[v], s32[v])
    err = np.abs(score[v].astype(np.float64) - s64[v]).max()
    print(f"NCC {W}x{H} D={D} r={r}: max |score32 - score64| = {err:.3g}")
    assert err <= TOL
    got16, _ = run_ncc(ct, cuda, L, R, D, r, torch.int16)
    np.testing.assert_array_equal(got16, oracle.to_u16(d))


@pytest.mark.slow
def test_ncc_config2_full_size(ct, oracle, cuda):
    W, H, D = 1920, 1080, 128
    L, R, _, _ = ct.synth_pair(2, 2024, W, H, D - 1)
    d, s32, s64 = oracle.match_ncc(L, R, D, 5)
    got, score = run_ncc(ct, cuda, L, R, D, 5)
    np.testing.assert_array_equal(got, oracle.to_u8(d))
    v = d >= 0
    err = np.abs(score[v].astype(np.float64) - s64[v]).max()
    print(f"NCC 1920x1080 D=128: max |score32 - score64| = {err:.3g}")
    assert err <= TOL


def _coarse_map(ct, oracle, L, R, D, s, holes, seed):
    """Coarse disparities at 1/s: NCC (oracle) on s x s box-averaged images,
    with a fraction `holes` of them removed (-1)."""
    H, W = L.shape
    Hc, Wc = -(-H // s), W // s

    def down(img):
        pad = np.zeros((Hc * s, Wc * s), np.float64)
        pad[:H] = img[:, :Wc * s]
        pad[H:] = img[-1, :Wc * s]
        return np.round(pad.reshape(Hc, s, Wc, s).mean(axis=(1, 3))).astype(np.uint8)

    c, _, _ = oracle.match_ncc(down(L), down(R), max(2, D // s), 2)
    rng = np.random.default_rng(seed)
    c = np.where(rng.random(c.shape) < holes, -1, c).astype(np.int16)
    return c


@pytest.mark.parametrize("W,H,D,r,s,holes,ctype", [
    (200, 90, 64, 5, 2, 0.0, torch.uint8),
    (332, 111, 128, 5, 4, 0.3, torch.int16),    # two disparity blocks per tile
    (160, 64, 48, 2, 8, 0.5, torch.uint8),      # empty guide blocks
    (128, 48, 64, 4, 1, 0.8, torch.int16),      # scale 1: per-pixel coarse hints
])
def test_ncc_guided_matches_oracle(ct, oracle, cuda, W, H, D, r, s, holes, ctype):
    L, R, _, _ = ct.synth_pair(2, 40 + W + s, W, H, D - 1)
    coarse = _coarse_map(ct, oracle, L, R, D, s, holes, seed=W)
    d, s32, _ = oracle.match_ncc_guided(L, R, D, coarse, r)
    enc = oracle.to_u8(coarse) if ctype == torch.uint8 else oracle.to_u16(coarse)
    init = to_dev(np.ascontiguousarray(enc), cuda)
    m = ct.BlockMatcherNCC()
    m.configure(0, W, H, D, radius=r)
    out = ct.alloc_image(H, W, torch.uint8, cuda)
    score = ct.alloc_image(H, W, torch.float32, cuda)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda), score=score, disp_init=init)
    torch.cuda.synchronize()
    assert m.device_status() == 0
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.to_u8(d))
    v = d >= 0
    np.testing.assert_array_equal(score.cpu().numpy()[v], s32[v])
    # the guide restricts the search: most pixels keep the unguided answer
    du, _, _ = oracle.match_ncc(L, R, D, r)
    if holes == 0.0:
        assert (d == du).mean() > 0.8


def test_ncc_guided_rejects_a_scale_that_does_not_divide(ct, cuda):
    m = ct.BlockMatcherNCC()
    m.configure(0, 64, 32, 16)
    a = ct.alloc_image(32, 64, torch.uint8, cuda)
    for w, h in ((48, 32), (32, 15)):
        init = ct.alloc_image(h, w, torch.uint8, cuda)
        with pytest.raises(ct.CtError) as e:
            m.process(a, a, a, disp_init=init)
        assert e.value.code == ct.CT_EFORMAT


@pytest.mark.parametrize("W,H,D,s,holes,ctype", [
    (200, 90, 64, 2, 0.0, torch.uint8),
    (332, 111, 128, 4, 0.3, torch.int16),     # two disparity blocks per tile
    (160, 64, 48, 8, 0.5, torch.uint8),       # empty guide blocks
])
def test_aw_guided_matches_oracle(ct, oracle, cuda, W, H, D, s, holes, ctype):
    L, R, _, _ = ct.synth_pair(3, 70 + W + s, W, H, D - 1)
    coarse = _coarse_map(ct, oracle, L, R, D, s, holes, seed=W + 1)
    d, _, s32, _ = oracle.match_aw_guided(L, R, D, coarse)
    enc = oracle.to_u8(coarse) if ctype == torch.uint8 else oracle.to_u16(coarse)
    init = to_dev(np.ascontiguousarray(enc), cuda)
    m = ct.BlockMatcherAW()
    m.configure(0, W, H, D)
    dL, dR = to_dev(L, cuda), to_dev(R, cuda)
    out = ct.alloc_image(H, W, torch.uint8, cuda)
    sub = ct.alloc_image(H, W, torch.float32, cuda)
    m.process(out, dL, dR, disp_init=init)
    m.process(sub, dL, dR, disp_init=init)
    torch.cuda.synchronize()
    assert m.device_status() == 0
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.to_u8(d))
    np.testing.assert_array_equal(sub.cpu().numpy(), s32)


@pytest.mark.parametrize("W,H,D,r,dmin", [
    (67, 43, 13, 5, 0), (400, 150, 96, 5, 0), (150, 60, 40, 4, 0), (150, 60, 70, 2, 0),
    (300, 100, 200, 5, 0),   # two blocks of 128 disparities, merged through global keys
    (257, 90, 128, 5, 7),    # minimum disparity, ragged width
    (129, 200, 128, 5, 0),   # one pixel past a 128-pixel tile, several strips
    (140, 33, 64, 5, 0),     # strips of 16, 16 and 1 rows
    (300, 50, 96, 4, 0),     # strips of 16, 16, 16 and 2 rows
    (200, 70, 256, 2, 3),    # 5x5, two disparity blocks, odd minimum disparity
])
def test_ncc_tensor_cores_equal_cuda_cores(ct, oracle, cuda, W, H, D, r, dmin):
    """Unguided NCC on the tensor cores gives the CUDA-core kernel's maps and
    scores bit for bit (flat patches, noise-only rows and textured scenes)."""
    L, R, _, _ = ct.synth_pair(2, 3 * W + D + dmin, W, H, dmin + D - 1)
    L[5:25, 5:30] = 128                    # flat: the sigma < 1 rule
    R[H // 2:H // 2 + 8] = np.random.default_rng(1).integers(0, 256, (8, W), dtype=np.uint8)  # no match
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    res = {}
    for tcores in (True, False):
        m = ct.BlockMatcherNCC()
        m.configure(0, W, H, D, radius=r, disp_min=dmin)
        m.set_tensor_cores(tcores)
        out = ct.alloc_image(H, W, torch.int16, cuda)
        score = ct.alloc_image(H, W, torch.float32, cuda)
        out.fill_(0x1111)
        score.fill_(-7.0)
        m.process(out, dl, dr, score=score)
        torch.cuda.synchronize()
        assert m.device_status() == 0
        res[tcores] = (out.cpu().numpy().view(np.uint16), score.cpu().numpy())
    np.testing.assert_array_equal(res[True][0], res[False][0])
    np.testing.assert_array_equal(res[True][1].view(np.uint32), res[False][1].view(np.uint32))
    if W * H * D <= 400 * 150 * 96:
        d, s32, _ = oracle.match_ncc(L, R, D, r, dmin=dmin)
        np.testing.assert_array_equal(res[True][0], oracle.to_u16(d))
