"""Training the confidence net end to end on the GPU (its own data, its own
kernels) and what that buys: on held-out pairs the trained net ranks invalid
disparities far better than the same net untrained, and the invalid-pixel
AUC is compared with the plain left-right check's."""
import pytest

pytestmark = pytest.mark.gpu


def test_training_gain_on_held_out_pairs(ct, cuda):
    import confnet_train as T
    net = ct.ConfNet()
    net.configure(0, 4096)
    net.init(1)
    samples, labels = T.make_training_set(net, 0, n_pairs=60, W=320, H=240, per_pair=1024)
    assert samples.shape == (60 * 1024, 128)
    frac = float(labels.float().mean().item())
    assert 0.5 < frac < 0.99, frac
    hist = T.train(net, samples, labels, steps=400, batch=4096, lr=3e-3)
    assert hist[-1][1] < hist[0][1]
    untrained = ct.ConfNet()
    untrained.configure(0, 16)
    untrained.init(1)
    res = T.evaluate({"net": net, "untrained": untrained}, 0, n_pairs=3, W=640, H=480)
    print(res)
    assert net.device_status() == 0
    assert res["net"] > res["untrained"] + 0.05, res
    assert res["net"] > 0.75, res
