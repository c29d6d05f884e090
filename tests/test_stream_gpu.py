"""Streamed census stereo (ct_census_stream_*): frames submitted from host
memory come back as the same cross-checked maps ct_bm_census_process_lr
gives for each pair, whatever the mix of page-locked and pageable buffers,
row pitches and output types, with up to three frames in flight."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu


def _host(a, pinned, pad=0):
    t = torch.zeros((a.shape[0], a.shape[1] + pad), dtype=torch.from_numpy(a).dtype)
    if pinned:
        t = t.pin_memory()
    t = t[:, :a.shape[1]]
    t.copy_(torch.from_numpy(a))
    return t


@pytest.mark.parametrize("out_dtype", [torch.uint8, torch.int16])
def test_stream_frames_equal_process_lr(ct, cuda, out_dtype):
    W, H, D = 333, 120, 64
    s = ct.CensusStream()
    s.configure(0, W, H, D, tol=1, out_type=out_dtype)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    frames = []
    for i in range(8):
        L, R, _, _ = ct.synth_pair(1 + i % 3, 500 + i, W, H, D - 1)
        pinned = i % 2 == 0
        out = _host(np.zeros((H, W), dtype=np.uint8 if out_dtype == torch.uint8 else np.int16), pinned, pad=3 * (i % 2))
        k = s.submit(_host(L, pinned, pad=16 * (i % 3)), _host(R, pinned), out)
        assert k == i
        frames.append((k, L, R, out))
    for k, L, R, out in frames:
        s.wait(k)
        ck = ct.alloc_image(H, W, out_dtype, cuda)
        m.process_lr(to_dev(L, cuda), to_dev(R, cuda), disp_checked=ck, tol=1)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.numpy(), ck.cpu().numpy(), err_msg=f"frame {k}")
    assert s.device_status() == 0


def test_stream_timer_covers_the_frames(ct, cuda):
    W, H, D = 640, 480, 64
    s = ct.CensusStream()
    s.configure(0, W, H, D)
    L, R, _, _ = ct.synth_pair(1, 9, W, H, D - 1)
    hL, hR = _host(L, True), _host(R, True)
    outs = [_host(np.zeros((H, W), np.uint8), True) for _ in range(4)]
    k = s.submit(hL, hR, outs[0])
    s.wait(k)
    s.timer_start()
    for i in range(12):
        k = s.submit(hL, hR, outs[i % 4])
    ms = s.timer_stop()
    s.wait(k)
    assert 0.0 < ms < 1000.0
    assert all(np.array_equal(o.numpy(), outs[0].numpy()) for o in outs)
