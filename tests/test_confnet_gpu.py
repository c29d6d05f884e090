"""Learned-confidence path on the GPU: the census matcher's cost-curve export
(bit-exact against the oracle's curves), sample gathering, the training
forward and gradients against the FP64 oracle of the network, and the
tensor-core inference kernel against the training forward."""
import numpy as np
import pytest
import torch

import confnet as cn
from conftest import to_dev

pytestmark = pytest.mark.gpu


def curves_of(ct, cuda, L, R, D, lr=True, tuning=None):
    H, W = L.shape
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D, left_to_right=lr)
    if tuning:
        m.set_tuning(*tuning)
    cv = ct.CurveVolume(W, H, D, cuda)
    disp = ct.alloc_image(H, W, torch.int16, cuda)
    m.process_curves(disp, cv, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    assert m.device_status() == 0
    return cv, disp.cpu().numpy()


@pytest.mark.parametrize("W,H,D,kind,lr,tuning", [
    (333, 111, 128, 2, True, None),
    (257, 90, 200, 2, True, (36, 8)),     # partial warp group, 8 disparities per warp
    (130, 37, 64, 1, False, (46, 4)),     # right-to-left
    (640, 480, 128, 1, True, None),
])
def test_curves_bit_exact(ct, oracle, cuda, W, H, D, kind, lr, tuning):
    L, R, _, _ = ct.synth_pair(kind, 11 + W, W, H, D - 1)
    cv, disp = curves_of(ct, cuda, L, R, D, lr, tuning)
    want_d, _, want_c = oracle.match_census(L, R, D, 2, lr, curve_shift=3)
    # border pixels (within 2 of the edge) have no disparity and unspecified codes
    np.testing.assert_array_equal(cv.to_hwd()[2:-2, 2:-2], want_c[2:-2, 2:-2])
    np.testing.assert_array_equal(disp.view(np.uint16), oracle.to_u16(want_d))


def _winners(d):
    return np.where(d >= 0, d, 0)


@pytest.mark.parametrize("dtype", [torch.int16, torch.uint8])
def test_gather_recentres(ct, oracle, cuda, dtype):
    W, H, D = 200, 64, 128
    L, R, _, _ = ct.synth_pair(1, 5, W, H, D - 1)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    cv = ct.CurveVolume(W, H, D, cuda)
    disp = ct.alloc_image(H, W, dtype, cuda)
    m.process_curves(disp, cv, to_dev(L, cuda), to_dev(R, cuda))
    want_d, _, want_c = oracle.match_census(L, R, D, 2, True, curve_shift=3)
    r = np.random.default_rng(1)
    xs, ys = r.integers(2, W - 2, 777), r.integers(2, H - 2, 777)  # pixels with a disparity
    xy = np.stack([xs, ys], 1).astype(np.int32)
    net = ct.ConfNet()
    net.configure(0, 1024)
    samples = torch.empty((777, 128), dtype=torch.uint8, device=cuda)
    net.gather(samples, cv, disp, torch.from_numpy(xy).to(cuda))
    torch.cuda.synchronize()
    assert net.device_status() == 0
    want = cn.recenter(want_c[ys, xs], _winners(want_d[ys, xs]))
    np.testing.assert_array_equal(samples.cpu().numpy(), want)


def _real_samples(ct, oracle, n, seed):
    W, H, D = 333, 111, 128
    L, R, _, _ = ct.synth_pair(1, seed, W, H, D - 1)
    d, _, curve = oracle.match_census(L, R, D, 2, True, curve_shift=3)
    r = np.random.default_rng(seed)
    ys, xs = r.integers(0, H, n), r.integers(0, W, n)
    return cn.recenter(curve[ys, xs], _winners(d[ys, xs]))


def _params(seed):
    r = np.random.default_rng(seed)
    p = cn.init_params(seed).astype(np.float64)
    # non-zero biases so every term of the gradient is exercised
    for off, k in ((160, 32), (5312, 32), (10464, 32), (12544, 64), (12672, 1)):
        p[off:off + k] = r.normal(0, 0.3, k)
    return p.astype(np.float32)


@pytest.mark.parametrize("n", [600, 37, 1023])
def test_training_forward_and_gradient_vs_oracle(ct, oracle, cuda, n):
    """Scores, loss and gradient of a batch against the FP64 oracle. The
    batch sizes cover partial 128-row GEMM tiles, a batch below one tile and
    batches that are not a multiple of 8 (the zero-padded sample columns of
    the weight-gradient GEMMs) and of the 256-sample chunks."""
    x = _real_samples(ct, oracle, n, 7)
    y = (np.random.default_rng(2).random(n) < 0.7).astype(np.uint8)
    p = _params(3)
    net = ct.ConfNet()
    net.configure(0, 1024)
    net.set_params(p)
    np.testing.assert_array_equal(net.get_params(), p)
    xs = torch.from_numpy(x).to(cuda)
    ys = torch.from_numpy(y).to(cuda)
    sc = torch.empty(n, dtype=torch.float32, device=cuda)
    grad = torch.empty(ct.CT_CONFNET_PARAMS, dtype=torch.float32, device=cuda)
    loss = torch.empty(1, dtype=torch.float32, device=cuda)
    net.scores(sc, xs)
    net.loss_grad(xs, ys, grad, loss)
    torch.cuda.synchronize()
    assert net.device_status() == 0
    want_s = cn.scores(x, p)
    want_l, want_g = cn.loss_and_grad(x, y, p)
    err_s = np.abs(sc.cpu().numpy() - want_s).max()
    assert err_s < 2e-3, err_s
    assert abs(loss.item() - want_l) < 1e-4 * max(1.0, abs(want_l))
    g = grad.cpu().numpy().astype(np.float64)
    rel = np.linalg.norm(g - want_g) / np.linalg.norm(want_g)
    assert rel < 1e-2, rel
    # per layer, so a wrong layer cannot hide behind a large one
    o = 0
    for name, shape in cn.SHAPES:
        k = int(np.prod(shape))
        ref = want_g[o:o + k]
        if np.linalg.norm(ref) > 0:
            assert np.linalg.norm(g[o:o + k] - ref) / np.linalg.norm(ref) < 3e-2, name
        o += k


def test_adam_step_moves_towards_lower_loss(ct, oracle, cuda):
    n = 1000
    x = _real_samples(ct, oracle, n, 9)
    y = (x.min(axis=1) < 60).astype(np.uint8)  # a learnable rule
    net = ct.ConfNet()
    net.configure(0, n)
    net.init(5)
    xs, ys = torch.from_numpy(x).to(cuda), torch.from_numpy(y).to(cuda)
    loss = torch.empty(1, dtype=torch.float32, device=cuda)
    losses = []
    for _ in range(150):
        net.train_step(xs, ys, 5e-3, loss)
        losses.append(loss.item())
    assert net.device_status() == 0
    assert losses[-1] < 0.6 * losses[0], losses[::15]


@pytest.mark.parametrize("W,H", [(333, 70), (128, 9)])
def test_tensor_core_inference_matches_training_forward(ct, oracle, cuda, W, H):
    D = 128
    L, R, _, _ = ct.synth_pair(2, 21 + W, W, max(H, 16), D - 1)
    L, R = np.ascontiguousarray(L[:H]), np.ascontiguousarray(R[:H])
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    cv = ct.CurveVolume(W, H, D, cuda)
    disp = ct.alloc_image(H, W, torch.int16, cuda)
    m.process_curves(disp, cv, to_dev(L, cuda), to_dev(R, cuda))
    net = ct.ConfNet()
    net.configure(0, W * H)
    p = _params(4)
    net.set_params(p)
    score = ct.alloc_image(H, W, torch.float32, cuda)
    score.fill_(-1.0)
    net.infer(score, cv, disp)
    xy = np.stack(np.meshgrid(np.arange(W), np.arange(H)), -1).reshape(-1, 2).astype(np.int32)
    samples = torch.empty((W * H, 128), dtype=torch.uint8, device=cuda)
    net.gather(samples, cv, disp, torch.from_numpy(xy).to(cuda))
    ref = torch.empty(W * H, dtype=torch.float32, device=cuda)
    net.scores(ref, samples)
    torch.cuda.synchronize()
    assert net.device_status() == 0
    got = score.cpu().numpy().ravel()
    want = ref.cpu().numpy()
    # Both paths accumulate in fp32 but in different orders; a conv
    # activation that lands on a bf16 rounding boundary can then round one
    # ulp apart, which moves the score by at most a few 1e-3.
    err = np.abs(got - want)
    assert err.max() < 6e-3 and err.mean() < 2e-4, (err.max(), err.mean())
    # and against the FP64 oracle on a subset
    sub = np.random.default_rng(0).choice(W * H, min(500, W * H), replace=False)
    err_o = np.abs(got[sub] - cn.scores(samples.cpu().numpy()[sub], p)).max()
    assert err_o < 3e-3, err_o


@pytest.mark.parametrize("dtype", [torch.int16, torch.uint8])
def test_infer_checked_map_marks_low_scores(ct, cuda, dtype):
    """The checked output is the winner map with every disparity scoring below
    the threshold marked the way the cross-check marks it."""
    import confnet_train as T
    W, H, D = 257, 40, 128
    L, R, _, _ = ct.synth_pair(1, 77, W, H, D - 1)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    cv = ct.CurveVolume(W, H, D, cuda)
    disp = ct.alloc_image(H, W, dtype, cuda)
    m.process_curves(disp, cv, to_dev(L, cuda), to_dev(R, cuda))
    net = ct.ConfNet()
    net.configure(0, 16)
    net.set_params(T.load_weights())
    score = ct.alloc_image(H, W, torch.float32, cuda)
    checked = ct.alloc_image(H, W, dtype, cuda)
    net.infer(score, cv, disp, checked=checked, threshold=0.6)
    torch.cuda.synchronize()
    assert net.device_status() == 0
    s, d, c = score.cpu().numpy(), disp.cpu().numpy(), checked.cpu().numpy()
    if dtype == torch.uint8:
        want = np.where(s >= 0.6, d, 255).astype(np.uint8)
    else:
        du = d.view(np.uint16)
        want = np.where((du >= 1) & (du <= 0xFFEF) & (s < 0.6), 0xFFFA, du).astype(np.uint16).view(np.int16)
    np.testing.assert_array_equal(c, want)
    assert 0.02 < (s < 0.6).mean() < 0.9
