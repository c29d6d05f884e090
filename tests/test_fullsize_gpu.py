"""The exact workloads the throughput numbers are measured on, at full size,
against the CPU oracle:

* the census stereo step at 1920x1080, D = 128 (generator kind 2, seed 2024):
  9x7 census of both views, 5x5 Hamming aggregation, winner-take-all
  left-to-right and right-to-left, cross-check with tolerance 1
  (CrossCheckDisparityMaps.cu:63-110 semantics). All three maps are compared,
  with the default launch shape and after the autotuner has picked one;
* the 64-pair mixed batch (sizes from {320x240 .. 1920x1080}, D from
  {32 .. 256}, the bench's seeded draw), through process() and through two
  replays of the captured CUDA graph, every pair against the oracle's
  cross-checked map."""
import sys
from pathlib import Path

import numpy as np
import pytest
import torch

from conftest import to_dev

pytestmark = pytest.mark.gpu

sys.path.insert(0, str(Path(__file__).resolve().parents[1]))


def headline_pair(ct):
    return ct.synth_pair(2, 2024, 1920, 1080, 127)[:2]


def test_headline_step_all_three_maps(ct, oracle, cuda):
    W, H, D = 1920, 1080, 128
    L, R = headline_pair(ct)
    wl, _ = oracle.match_census(L, R, D, 2, True)
    wr, _ = oracle.match_census(L, R, D, 2, False)
    wc, _ = oracle.crosscheck(wl, wr, 1, True)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    dl, dr = to_dev(L, cuda), to_dev(R, cuda)
    maps = [ct.alloc_image(H, W, torch.uint8, cuda) for _ in range(3)]

    def run_and_compare(tag):
        for t in maps:
            t.fill_(0x77)
        m.process_lr(dl, dr, disp_lr=maps[0], disp_rl=maps[1], disp_checked=maps[2], tol=1)
        torch.cuda.synchronize()
        for got, want, name in zip(maps, (wl, wr, np.where(wc == -2, -1, wc)), ("L->R", "R->L", "checked")):
            np.testing.assert_array_equal(got.cpu().numpy(), oracle.to_u8(want), err_msg=f"{tag}: {name}")

    run_and_compare("default launch shape")
    m.autotune(dl, dr)
    run_and_compare(f"autotuned {m.tuning()}")
    assert m.device_status() == 0


def test_headline_step_u16_ids(ct, oracle, cuda):
    """The same step with EDisparityId-coded U16 maps (Inconsistent kept apart
    from CannotEvaluate)."""
    W, H, D = 1920, 1080, 128
    L, R = headline_pair(ct)
    wl, _ = oracle.match_census(L, R, D, 2, True)
    wr, _ = oracle.match_census(L, R, D, 2, False)
    wc, _ = oracle.crosscheck(wl, wr, 1, True)
    m = ct.BlockMatcherCensus()
    m.configure(0, W, H, D)
    ck = ct.alloc_image(H, W, torch.int16, cuda)
    m.process_lr(to_dev(L, cuda), to_dev(R, cuda), disp_checked=ck, tol=1)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(ck.cpu().numpy().view(np.uint16), oracle.to_u16(wc))


def test_batch64_exact_config_against_oracle(ct, oracle, cuda):
    import bench
    shapes = bench.batch_shapes()
    assert len(shapes) == 64
    pairs, want = [], []
    for i, (W, H, D) in enumerate(shapes):
        L, R, _, _ = ct.synth_pair(1, 1000 + i, W, H, D - 1)
        out = ct.alloc_image(H, W, torch.int16, cuda)
        out.fill_(0x33)
        pairs.append((to_dev(L, cuda), to_dev(R, cuda), out))
        wc, _ = oracle.crosscheck(oracle.match_census(L, R, D, 2, True)[0],
                                  oracle.match_census(L, R, D, 2, False)[0], 1, True)
        want.append(oracle.to_u16(wc))
    b = ct.BatchStereo()
    b.configure(0, shapes, tol=1)

    def compare(tag):
        for i, ((W, H, D), (_, _, out), w) in enumerate(zip(shapes, pairs, want)):
            np.testing.assert_array_equal(out.cpu().numpy().view(np.uint16), w,
                                          err_msg=f"{tag}: pair {i} {W}x{H} D={D}")

    b.process(pairs)
    torch.cuda.synchronize()
    compare("process")
    b.autotune(pairs)
    for (_, _, out) in pairs:
        out.fill_(0x44)
    b.graph_create(pairs)
    for k in range(2):
        b.graph_launch()
        torch.cuda.synchronize()
        compare(f"graph replay {k}")
    assert b.device_status() == 0
