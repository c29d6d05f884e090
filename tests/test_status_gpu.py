"""Failure reporting of bounded device waits, without a GPU fault: a wait on
an mbarrier that nothing completes gives up after its poll limit, the kernel
records CT_ETIMEOUT in the handle's status word and returns, and the handle
and context keep working."""
import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu


def test_wait_that_runs_out_reports_timeout(ct, oracle, cuda):
    W, H, D = 160, 96, 32
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    m.test_wait_timeout(1024)
    assert m.device_status() == ct.CT_ETIMEOUT
    assert m.device_status() == 0  # read and cleared
    L, R, _, _ = ct.synth_pair(1, 3, W, H, D - 1)
    out = ct.alloc_image(H, W, torch.uint8, cuda)
    m.process(out, to_dev(L, cuda), to_dev(R, cuda))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy(), oracle.to_u8(oracle.match_census(L, R, D)[0]))
    assert m.device_status() == 0


def test_timeout_hook_checks_its_arguments(ct, cuda):
    m = ct.BlockMatcherCensus()
    with pytest.raises(ct.CtError) as e:
        m.test_wait_timeout(16)  # not configured: no status word yet
    assert e.value.code == ct.CT_ESTATE
    m.configure(0, 64, 32, 16)
    with pytest.raises(ct.CtError) as e:
        m.test_wait_timeout(0)
    assert e.value.code == ct.CT_EINVAL
