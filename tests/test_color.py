"""Disparity visualisation (ColorDisparityImage): the oracle's restatement
against hand-computed values, and the GPU kernel against the oracle
bit-exactly for every style, on U16 code maps holding every EDisparityId and
on U8 maps."""
import numpy as np
import pytest
import torch

from conftest import to_dev


def test_color_ramp_known_answers(oracle):
    # t = 0: b = 1, g = 1 - 0.5 / 0.59, r = 0 -> (0, 39, 255)
    # t = 0.5: b = 1 - 0.5 / 0.7, g = 1, r = 1 - 0.3 / 0.7 -> (146, 255, 73)
    codes = np.array([[1, 51]], np.uint16)  # range 1 .. 101: t = 0 and 0.5
    c = oracle.color_disparity(codes, 2, 1, 101)
    rgb = [(int(v) & 0xFF, (int(v) >> 8) & 0xFF, (int(v) >> 16) & 0xFF, int(v) >> 24) for v in c.ravel()]
    assert rgb == [(0, 39, 255, 255), (146, 255, 73, 255)]
    g = oracle.color_disparity(np.array([[26]], np.uint16), 1, 1, 101)  # t = 0.25 -> rint(16383.75)
    assert int(g[0, 0]) == 16384
    rel = oracle.color_disparity(np.array([[1, 11, 0]], np.uint16), 4, inf_offset=5)
    assert rel.tolist() == [[0x7FFF + 5, 0x7FFF + 5 - 10, 0]]


def _codes(H, W, seed):
    r = np.random.default_rng(seed)
    c = r.integers(1, 140, (H, W)).astype(np.uint16)
    ids = np.array([0, 0xFFFF, 0xFFFE, 0xFFFD, 0xFFFC, 0xFFFB, 0xFFFA, 0xFFF5, 0xFFEF, 0xFFF0], np.uint16)
    m = r.random((H, W)) < 0.2
    c[m] = ids[r.integers(0, ids.size, m.sum())]
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("style", [0, 1, 2, 3, 4])
def test_color_styles_match_oracle(ct, oracle, cuda, style):
    H, W = 37, 203
    codes = _codes(H, W, style)
    p = ct.color_params(style)
    p.disp_min, p.disp_max, p.inf_offset = 3, 131, 7
    rgba = style in (0, 2)
    out = ct.alloc_image(H, W, torch.int32 if rgba else torch.int16, cuda)
    ct.color_disparity(out, to_dev(codes.view(np.int16), cuda), p)
    # U8 input: d -> code d + 1, 255 -> CannotEvaluate
    u8 = np.where(codes == 0xFFFF, 255, np.clip(codes.astype(np.int64) - 1, 0, 254)).astype(np.uint8)
    u8codes = np.where(u8 == 255, 0xFFFF, u8.astype(np.int64) + 1).astype(np.uint16)
    out8 = ct.alloc_image(H, W, torch.int32 if rgba else torch.int16, cuda)
    ct.color_disparity(out8, to_dev(u8, cuda), p)
    torch.cuda.synchronize()
    dt = np.uint32 if rgba else np.uint16
    for o, c in ((out, codes), (out8, u8codes)):
        want = oracle.color_disparity(c, style, p.disp_min, p.disp_max, p.inf_offset, list(p.colors))
        np.testing.assert_array_equal(o.cpu().numpy().view(dt), want)
