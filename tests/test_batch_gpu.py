"""Batched census stereo: every pair of a mixed batch equals the pair
processed alone (ct_bm_census_process_lr), bit for bit, through process()
and through the captured CUDA graph, before and after autotuning."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu


def make_batch(ct, cuda, shapes, dtype=torch.int16, seed0=100):
    pairs, host = [], []
    for i, (W, H, D) in enumerate(shapes):
        L, R, _, _ = ct.synth_pair(1, seed0 + i, W, H, D - 1)
        out = ct.alloc_image(H, W, dtype, cuda)
        out.fill_(0x33)
        pairs.append((to_dev(L, cuda), to_dev(R, cuda), out))
        host.append((L, R))
    return pairs, host


def alone(ct, cuda, L, R, D, dtype):
    H, W = L.shape
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    out = ct.alloc_image(H, W, dtype, cuda)
    m.process_lr(to_dev(L, cuda), to_dev(R, cuda), disp_checked=out, tol=1)
    torch.cuda.synchronize()
    return out.cpu().numpy()


SHAPES = [(320, 240, 32), (640, 480, 64), (333, 111, 128), (200, 90, 256), (131, 77, 64), (640, 480, 256),
          (96, 40, 1)]


@pytest.mark.parametrize("dtype", [torch.int16, torch.uint8])
def test_batch_equals_alone(ct, cuda, dtype):
    shapes = [s for s in SHAPES if dtype == torch.int16 or s[2] <= 255]
    b = ct.BatchStereo()
    b.configure(0, shapes, tol=1)
    pairs, host = make_batch(ct, cuda, shapes, dtype)
    b.process(pairs)
    torch.cuda.synchronize()
    assert b.device_status() == 0
    for (W, H, D), (l, r, out), (L, R) in zip(shapes, pairs, host):
        np.testing.assert_array_equal(out.cpu().numpy(), alone(ct, cuda, L, R, D, dtype), err_msg=f"{W}x{H} D={D}")


def test_batch_graph_and_autotune(ct, cuda):
    shapes = SHAPES[:5]
    b = ct.BatchStereo()
    b.configure(0, shapes, tol=1)
    pairs, host = make_batch(ct, cuda, shapes)
    want = [alone(ct, cuda, L, R, D, torch.int16) for (W, H, D), (L, R) in zip(shapes, host)]
    ths = b.autotune(pairs)
    assert all((t + 4) % 5 == 0 for t in ths)
    for (_, _, out) in pairs:
        out.fill_(0x44)
    b.graph_create(pairs)
    for _ in range(2):  # replays give the same maps
        b.graph_launch()
        torch.cuda.synchronize()
        for (l, r, out), w in zip(pairs, want):
            np.testing.assert_array_equal(out.cpu().numpy(), w)
    assert b.device_status() == 0


def test_batch_rejects_mismatched_items(ct, cuda):
    b = ct.BatchStereo()
    b.configure(0, [(64, 32, 16)])
    pairs, _ = make_batch(ct, cuda, [(64, 31, 16)])
    with pytest.raises(ct.CtError) as e:
        b.process(pairs)
    assert e.value.code == ct.CT_EFORMAT


def test_batch_back_to_back_default_stream(ct, cuda):
    """Calls queued back to back on the legacy default stream (handle 0) with
    no host synchronisation: each call's staged pair table and tensor maps
    must reach the device intact while the host fills the next call."""
    shapes = [(96 + 32 * (i % 5), 48 + 16 * (i % 3), 16 * (1 + i % 4)) for i in range(48)]
    b = ct.BatchStereo()
    b.configure(0, shapes, tol=1)
    pairs, host = make_batch(ct, cuda, shapes)
    want = [alone(ct, cuda, L, R, D, torch.int16) for (W, H, D), (L, R) in zip(shapes, host)]
    default = torch.cuda.default_stream(cuda)
    assert default.cuda_stream == 0
    for _ in range(6):
        b.process(pairs, stream=default)
    torch.cuda.synchronize()
    assert b.device_status() == 0
    for (W, H, D), (l, r, out), w in zip(shapes, pairs, want):
        np.testing.assert_array_equal(out.cpu().numpy(), w, err_msg=f"{W}x{H} D={D}")
