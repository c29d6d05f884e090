"""Reference-compat output (ct_bm_compat_*): the 4 x uint16 pixel of
BlockMatcherSAD1 / NCC / AW1 / AW2 / BlockMatcher1 (disparity or
EDisparityId, score, specificity channels) with their gradient gates, score
and minimum-delta thresholds, bit-exact against the CPU restatement
(oracle/compat.cpp) for every method, window, similarity type, direction and
a minimum disparity, with thresholds that make every ID rule fire."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu

IDS = {"cannot": 0xFFFF, "saturated": 0xFFFE, "not_found": 0xFFFD, "not_specific": 0xFFFC}

# method, patch, sim_type, left_to_right, dmin, grad, score, delta
CASES = [
    ("sad1", 9, 0, True, 0, 3.0, 30.0, 40),
    ("sad1", 16, 0, True, 4, 3.0, 40.0, 60),
    ("sad1", 5, 0, False, 0, 0.0, 25.0, 10),
    ("ncc", 11, 0, True, 0, 2.0, 0.6, 3),
    ("ncc", 5, 0, False, 3, 4.0, 0.5, 2),
    ("ncc", 9, 0, True, 0, 0.0, 0.0, 0),
    ("aw1", 3, 0, True, 0, 5.0, 88.0, 0.5),
    ("aw1", 5, 0, True, 2, 5.0, 90.0, 0.3),
    ("aw1", 3, 1, True, 0, 8.0, 10.0, 1.0),
    ("aw1", 5, 1, False, 0, 0.0, 5.0, 0.5),
    ("aw2", 3, 0, True, 0, 3.0, 20.0, 30),
    ("aw2", 5, 0, True, 6, 3.0, 25.0, 60),
    ("bm1", 9, 0, True, 0, 5.0, 44.0, 0.2),
    ("bm1", 15, 0, False, 1, 5.0, 45.0, 0.1),
    ("bm1", 11, 1, True, 0, 8.0, 5.0, 0.5),
    ("bm1", 5, 1, True, 0, 0.0, 0.0, 0.0),
]


def run_gpu(ct, cuda, L, R, method, patch, sim, lr, dmin, D, grad, score, delta, u16x4=True):
    H, W = L.shape
    m = ct.BlockMatcherCompat()
    m.configure(0, W, H, getattr(ct, f"CT_COMPAT_{method.upper()}"), D, patch, disp_min=dmin, sim_type=sim,
                left_to_right=lr, grad_thresh=grad, score_thresh=score, min_delta_thresh=delta)
    out = ct.alloc_u16x4(H, W, cuda) if u16x4 else ct.alloc_image(H, W, torch.int16, cuda)
    out.fill_(0x2222)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    assert m.device_status() == 0
    return out.cpu().numpy().view(np.uint16)


@pytest.mark.parametrize("method,patch,sim,lr,dmin,grad,score,delta", CASES)
def test_compat_bit_exact(ct, oracle, cuda, method, patch, sim, lr, dmin, grad, score, delta):
    W, H, D = 157, 71, 40
    L, R, _, _ = ct.synth_pair(1 + (patch % 3 == 0), 3 * patch + dmin + sim, W, H, dmin + D - 1)
    want = oracle.compat_match(L, R, method, D, patch, dmin=dmin, sim_type=sim, left_to_right=lr,
                               grad_thresh=grad, score_thresh=score, min_delta_thresh=delta)
    got = run_gpu(ct, cuda, L, R, method, patch, sim, lr, dmin, D, grad, score, delta)
    for ch in range(4):
        np.testing.assert_array_equal(got[..., ch], want[..., ch], err_msg=f"channel {'xyzw'[ch]}")
    # the x channel alone into a U16 map
    x_only = run_gpu(ct, cuda, L, R, method, patch, sim, lr, dmin, D, grad, score, delta, u16x4=False)
    np.testing.assert_array_equal(x_only, want[..., 0])


@pytest.mark.parametrize("method,patch,sim", [("ncc", 11, 0), ("sad1", 16, 0), ("aw1", 5, 0), ("bm1", 9, 1),
                                              ("aw2", 3, 0)])
def test_compat_640x480(ct, oracle, cuda, method, patch, sim):
    W, H, D = 640, 480, 64
    L, R, _, _ = ct.synth_pair(1, 7, W, H, D - 1)
    thr = {"ncc": (2.0, 0.6, 3), "sad1": (3.0, 40.0, 60), "aw1": (5.0, 90.0, 0.3), "bm1": (8.0, 5.0, 0.5),
           "aw2": (3.0, 20.0, 30)}[method]
    want = oracle.compat_match(L, R, method, D, patch, sim_type=sim, grad_thresh=thr[0], score_thresh=thr[1],
                               min_delta_thresh=thr[2])
    got = run_gpu(ct, cuda, L, R, method, patch, sim, True, 0, D, *thr)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("method,patch,sim,thr", [("ncc", 11, 0, (2.0, 0.6, 3)), ("sad1", 9, 0, (3.0, 40.0, 60)),
                                                  ("aw1", 5, 0, (5.0, 90.0, 0.3)), ("aw2", 3, 0, (3.0, 20.0, 30)),
                                                  ("bm1", 9, 1, (8.0, 5.0, 0.5))])
def test_compat_1080p_d128(ct, oracle, cuda, method, patch, sim, thr):
    """The 1920x1080 D=128 slanted-plane pair (generator kind 2, seed 2024),
    every channel bit-exact with the gates and ID thresholds active."""
    W, H, D = 1920, 1080, 128
    L, R, _, _ = ct.synth_pair(2, 2024, W, H, D - 1)
    want = oracle.compat_match(L, R, method, D, patch, sim_type=sim, grad_thresh=thr[0], score_thresh=thr[1],
                               min_delta_thresh=thr[2])
    got = run_gpu(ct, cuda, L, R, method, patch, sim, True, 0, D, *thr)
    np.testing.assert_array_equal(got, want)
