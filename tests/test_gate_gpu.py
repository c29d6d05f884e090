"""Gradient gate of the plain matchers (ct_bm_set_gradient_gate, the
reference's EvalGrad): gated pixels get no disparity, the others keep the
winner-take-all result, bit-exact against the oracle's map with the oracle's
gate mask applied."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu


def lib_gate(ct, m, t):
    m.set_gradient_gate(t)


@pytest.mark.parametrize("r,lr,thresh", [(4, True, 6.0), (2, False, 9.0), (3, True, 0.0)])
def test_sad_gate(ct, oracle, cuda, r, lr, thresh):
    W, H, D = 211, 83, 48
    L, R, _, _ = ct.synth_pair(1, 40 + r, W, H, D - 1)
    m = ct.BlockMatcherSAD1()
    m.configure(0, W, H, D, radius=r, left_to_right=lr)
    lib_gate(ct, m, thresh)
    out = ct.alloc_image(H, W, torch.int16, cuda)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    want, _ = oracle.match_sad(L, R, D, r, lr)
    g = oracle.gate_mask(L if lr else R, 0, 2 * r + 1, thresh)
    assert thresh == 0.0 or 0.05 < g.mean() < 0.9  # the gate fires on part of the image
    exp = oracle.to_u16(want)
    exp[g] = 0xFFFF
    np.testing.assert_array_equal(out.cpu().numpy().view(np.uint16), exp)


def test_ncc_gate_with_score(ct, oracle, cuda):
    W, H, D = 260, 90, 64
    L, R, _, _ = ct.synth_pair(2, 8, W, H, D - 1)
    m = ct.BlockMatcherNCC()
    m.configure(0, W, H, D, radius=5)
    lib_gate(ct, m, 7.0)
    out = ct.alloc_image(H, W, torch.uint8, cuda)
    score = ct.alloc_image(H, W, torch.float32, cuda)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda), score=score)
    torch.cuda.synchronize()
    want, s32, _ = oracle.match_ncc(L, R, D, 5)
    g = oracle.gate_mask(L, 0, 11, 7.0)
    assert 0.05 < g.mean() < 0.9
    exp = oracle.to_u8(want)
    exp[g] = 0xFF
    np.testing.assert_array_equal(out.cpu().numpy(), exp)
    ok = (want >= 0) & ~g
    np.testing.assert_array_equal(score.cpu().numpy()[ok], s32[ok])
    assert (score.cpu().numpy()[g] == 0).all()


def test_aw_gate_subpixel(ct, oracle, cuda):
    W, H, D = 300, 80, 64
    L, R, _, _ = ct.synth_pair(3, 12, W, H, D - 1)
    m = ct.BlockMatcherAW()
    m.configure(0, W, H, D)
    lib_gate(ct, m, 12.0)
    out = ct.alloc_image(H, W, torch.float32, cuda)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    _, _, s32, _ = oracle.match_aw(L, R, D)
    g = oracle.gate_mask(L, 1, 13, 12.0)
    assert 0.05 < g.mean() < 0.95
    exp = s32.copy()
    exp[g] = -1.0
    np.testing.assert_array_equal(out.cpu().numpy(), exp)


def test_gate_argument_checks(ct, cuda):
    m = ct.BlockMatcherCensus()
    with pytest.raises(ct.CtError) as e:
        lib_gate(ct, m, 1.0)
    assert e.value.code == ct.CT_ESTATE
    s = ct.BlockMatcherSAD1()
    with pytest.raises(ct.CtError) as e:
        lib_gate(ct, s, -1.0)
    assert e.value.code == ct.CT_EINVAL
