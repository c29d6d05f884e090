"""ct_bm_census_process_static: census matching for callers that cannot call
cudaMalloc (stream capture, frozen real-time allocators, memory owned by
another framework). It must give exactly what the allocating entry point
ct_bm_census_process gives, call after call, while allocating nothing.
This file is collected last so that a stop-at-first-failure run has already
run every other test."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu


def reference_map(ct, L, R, D, lr, dev, dtype):
    H, W = L.shape
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D, left_to_right=lr)
    out = ct.alloc_image(H, W, dtype, dev)
    m.process(out, to_dev(L, dev), to_dev(R, dev))
    torch.cuda.synchronize()
    return out.cpu().numpy()


def test_static_matches_allocating_entry_point_two_calls(ct, cuda):
    W, H = 1920, 1080  # the largest frame the static scratch takes
    cases = [(2, 11, 128, True, torch.uint8), (1, 12, 96, True, torch.int16), (2, 13, 128, False, torch.uint8)]
    inputs, want = [], []
    for kind, seed, D, lr, dtype in cases:
        L, R, _, _ = ct.synth_pair(kind, seed, W, H, D - 1)
        inputs.append((to_dev(L, cuda), to_dev(R, cuda)))
        want.append(reference_map(ct, L, R, D, lr, cuda, dtype))
    outs = [ct.alloc_image(H, W, dtype, cuda) for *_, dtype in cases]
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    torch.cuda.synchronize()
    free_before = None
    for i, ((kind, seed, D, lr, dtype), (dl, dr)) in enumerate(zip(cases, inputs)):
        outs[i].fill_(0x33)
        torch.cuda.synchronize()
        if i >= 1:
            free_before = torch.cuda.mem_get_info()[0]
        ct.census_match_static(outs[i], dl, dr, D, lr, device_status=status)
        torch.cuda.synchronize()
        if i >= 1:  # calls after the first allocate no device memory at all
            assert torch.cuda.mem_get_info()[0] == free_before
    for o, w in zip(outs, want):
        np.testing.assert_array_equal(o.cpu().numpy(), w)
    assert int(status.item()) == 0


def test_static_without_status_word_reports_through_the_getter(ct, cuda):
    """Callers that cannot allocate may pass no status word; the static word
    then takes the device-side reports, and the getter reads and clears it."""
    W, H, D = 640, 480, 64
    L, R, _, _ = ct.synth_pair(1, 21, W, H, D - 1)
    want = reference_map(ct, L, R, D, True, cuda, torch.uint8)
    out = ct.alloc_image(H, W, torch.uint8, cuda)
    ct.census_match_static(out, to_dev(L, cuda), to_dev(R, cuda), D)
    assert ct.census_static_status() == 0
    np.testing.assert_array_equal(out.cpu().numpy(), want)


def test_static_rejects_images_beyond_its_scratch(ct, cuda):
    a = ct.alloc_image(1100, 1920, torch.uint8, cuda)
    with pytest.raises(ct.CtError) as e:
        ct.census_match_static(a, a, a, 64)
    assert e.value.code == ct.CT_EINVAL
    assert "static scratch" in str(e.value)
