"""Synthetic stereo generator: determinism and ground-truth consistency."""
import numpy as np
import pytest


@pytest.mark.parametrize("kind,dmax", [(1, 63), (2, 127), (3, 255)])
def test_deterministic_and_in_range(ct, kind, dmax):
    a = ct.synth_pair(kind, 1234, 160, 96, dmax)
    b = ct.synth_pair(kind, 1234, 160, 96, dmax)
    c = ct.synth_pair(kind, 1235, 160, 96, dmax)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    assert not np.array_equal(a[0], c[0])
    L, R, G, O = a
    assert G.min() >= 0 and G.max() <= dmax
    assert L.std() > 20 and R.std() > 20   # textured
    assert set(np.unique(O)) <= {0, 1}


def test_warp_matches_ground_truth(ct):
    L, R, G, O = ct.synth_pair(1, 7, 200, 120, 40)
    H, W = L.shape
    ys, xs = np.nonzero(O == 0)
    xr = xs - G[ys, xs]
    diff = np.abs(L[ys, xs].astype(int) - R[ys, xr].astype(int))
    # noise sigma 2: visible pixels agree to a few grey levels
    assert np.median(diff) <= 3 and (diff > 12).mean() < 0.01


def test_config1_background_and_rectangles(ct):
    L, R, G, O = ct.synth_pair(1, 3, 640, 480, 63)
    vals, counts = np.unique(G, return_counts=True)
    assert 4 in vals and len(vals) <= 9
    assert O.mean() < 0.3


def test_thread_count_does_not_change_output(ct, monkeypatch):
    import subprocess, sys, os
    code = ("import sys; sys.path.insert(0, 'module.clutec.cuda_b200'); import ctstereo, hashlib;"
            "L,R,G,O = ctstereo.synth_pair(2, 99, 321, 123, 100);"
            "print(hashlib.sha1(L.tobytes()+R.tobytes()+G.tobytes()+O.tobytes()).hexdigest())")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    outs = []
    for n in ("1", "5"):
        env = dict(os.environ, OMP_NUM_THREADS=n)
        outs.append(subprocess.run([sys.executable, "-c", code], cwd=root, env=env, capture_output=True,
                                   text=True, check=True).stdout.strip())
    assert outs[0] == outs[1]
