"""FP64 restatement of the learned confidence network (forward + backward).

TEST INFRASTRUCTURE ONLY: the checker for the GPU training and inference
kernels of the confidence net (csrc/confnet_*.cu). Only tests/ and the
cpu_baseline leg of bench.py import it; the product never does.

The network reads a pixel's uint8 census cost curve c[0..127] (aggregated
5x5 Hamming cost >> 3, 0..196; 255 for unsearchable disparities), re-centred
on the pixel's winner-take-all disparity d: the sample is the 128-long
r[k] = c[d - 64 + k] (255 outside 0..127), so r[64] is the winning cost. The
convolution stack reads its 35 central codes x[k] = r[52 + k], i.e. the
disparities d - 12 .. d + 22, and returns a validity logit. Its numerics are
defined exactly as the GPU runs them:

  conv1  1 -> 32, k=5, stride 5        : z1[p,o] = b1[o] + sum_j w1[o,j] x[5p+j]     p = 0..6
         ReLU, rounded to bf16 -> a1[7,32]
  conv2 32 -> 32, k=5, stride 3, pad 1 : z2[r,o] = b2[o] + sum_{j,i} w2[o,i,j] a1[3r+j-1,i]  r = 0, 1
         ReLU, rounded to bf16 -> a2[2,32]
  conv3 32 -> 32, k=5, pad 2 (one output): z3[o] = b3[o] + sum_{j,i} w3[o,i,j] a2[j-2,i]
         (taps 0, 1, 4 meet the padding) ReLU, rounded to bf16 -> a3[32]
  fc1   32 -> 64 : z4 = b4 + W4 a3, a4 = ReLU(z4) (fp32)
  fc2   64 -> 1  : logit = b5 + w5 . a4, score = sigmoid(logit) = P(disparity correct)

Weights w1..w5 are bf16 values (fp32 master copies rounded to nearest-even);
biases are fp32. Out-of-range inputs of a convolution are zero. The loss is
the mean binary cross-entropy with logits. The backward pass treats the bf16
roundings of activations as identity (straight-through).
"""
import numpy as np

# Parameter order and shapes of the flat fp32 parameter vector.
SHAPES = [("w1", (32, 5)), ("b1", (32,)), ("w2", (32, 32, 5)), ("b2", (32,)),
          ("w3", (32, 32, 5)), ("b3", (32,)), ("w4", (64, 32)), ("b4", (64,)),
          ("w5", (64,)), ("b5", (1,))]
WEIGHTS = {"w1", "w2", "w3", "w4", "w5"}
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)  # 12673
CURVE_LEN = 128
CROP_LO = 52   # first code of r the convolutions read (disparity d - 12)
CROP_LEN = 35


def recenter(curve, d):
    """(n, 128) curves and (n,) winning disparities -> (n, 128) samples
    r[k] = curve[d - 64 + k], 255 outside the curve."""
    curve = np.asarray(curve)
    idx = np.asarray(d, np.int64)[:, None] - 64 + np.arange(128)[None, :]
    ok = (idx >= 0) & (idx < 128)
    return np.where(ok, np.take_along_axis(curve, np.clip(idx, 0, 127), 1), 255).astype(np.uint8)


def unflatten(flat):
    flat = np.asarray(flat)
    out, o = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = flat[o:o + n].reshape(shape)
        o += n
    assert o == flat.size == N_PARAMS
    return out


def flatten(p):
    return np.concatenate([np.asarray(p[name], np.float64).ravel() for name, _ in SHAPES])


def bf16(a):
    """Round to the nearest bf16 value (ties to even), returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def init_params(seed):
    """He-style initialisation (conv1 scaled for inputs in 0..255)."""
    r = np.random.default_rng(seed)
    p = {"w1": r.normal(0, 1.0 / (np.sqrt(5) * 128.0), (32, 5)), "b1": np.zeros(32),
         "w2": r.normal(0, np.sqrt(2.0 / 160), (32, 32, 5)), "b2": np.zeros(32),
         "w3": r.normal(0, np.sqrt(2.0 / 128), (32, 32, 5)), "b3": np.zeros(32),
         "w4": r.normal(0, np.sqrt(2.0 / 32), (64, 32)), "b4": np.zeros(64),
         "w5": r.normal(0, np.sqrt(1.0 / 64), (64,)), "b5": np.zeros(1)}
    return flatten(p).astype(np.float32)


def _conv_idx(n_out, stride, pad, n_in, k=5):
    idx = stride * np.arange(n_out)[:, None] + np.arange(k)[None, :] - pad
    ok = (idx >= 0) & (idx < n_in)
    return np.where(ok, idx, 0), ok


def forward(curves, flat, emulate=True):
    """curves: (n, 128) uint8 re-centred samples (see recenter). Returns
    (logits, cache). emulate=False skips the bf16 roundings (plain float64
    network, for finite differences)."""
    p = unflatten(np.asarray(flat, np.float64))
    rw = bf16 if emulate else (lambda a: np.asarray(a, np.float64))
    w = {k: (rw(v) if k in WEIGHTS else np.asarray(v, np.float64)) for k, v in p.items()}
    x = np.asarray(curves, np.float64)
    n = x.shape[0]
    i1 = CROP_LO + 5 * np.arange(7)[:, None] + np.arange(5)[None, :]
    X1 = x[:, i1]                                             # (n, 7, 5)
    m1 = np.einsum("npj,oj->npo", X1, w["w1"]) + w["b1"]      # (n, 7, 32)
    a1 = rw(np.maximum(m1, 0.0))
    i2, ok2 = _conv_idx(2, 3, 1, 7)
    A1 = a1[:, i2, :] * ok2[None, :, :, None]                 # (n, 2, 5, 32)
    z2 = np.einsum("nrji,oij->nro", A1, w["w2"]) + w["b2"]    # (n, 2, 32)
    a2 = rw(np.maximum(z2, 0.0))
    i3, ok3 = _conv_idx(1, 1, 2, 2)
    A2 = a2[:, i3[0], :] * ok3[0][None, :, None]              # (n, 5, 32)
    z3 = np.einsum("nji,oij->no", A2, w["w3"]) + w["b3"]      # (n, 32)
    a3 = rw(np.maximum(z3, 0.0))
    z4 = a3 @ w["w4"].T + w["b4"]                             # (n, 64)
    a4 = np.maximum(z4, 0.0)
    logit = a4 @ w["w5"] + w["b5"][0]
    cache = dict(w=w, X1=X1, m1=m1, A1=A1, z2=z2, A2=A2, z3=z3, a3=a3, z4=z4, a4=a4,
                 i2=i2, ok2=ok2, i3=i3, ok3=ok3, n=n)
    return logit, cache


def loss_and_grad(curves, labels, flat, emulate=True):
    """Mean BCE-with-logits loss and its gradient w.r.t. the flat parameters."""
    logit, c = forward(curves, flat, emulate)
    y = np.asarray(labels, np.float64)
    n = c["n"]
    loss = float(np.mean(np.logaddexp(0.0, logit) - y * logit))
    w = c["w"]
    g = {}
    dl = (1.0 / (1.0 + np.exp(-logit)) - y) / n               # (n,)
    g["b5"] = np.array([dl.sum()])
    g["w5"] = dl @ c["a4"]
    dz4 = dl[:, None] * w["w5"][None, :] * (c["z4"] > 0)
    g["b4"] = dz4.sum(0)
    g["w4"] = dz4.T @ c["a3"]
    dz3 = (dz4 @ w["w4"]) * (c["z3"] > 0)                     # (n, 32)
    g["b3"] = dz3.sum(0)
    g["w3"] = np.einsum("no,nji->oij", dz3, c["A2"])
    dA2 = np.einsum("no,oij->nji", dz3, w["w3"]) * c["ok3"][0][None, :, None]
    da2 = np.zeros((n, 2, 32))
    for j in range(5):
        if c["ok3"][0][j]:
            da2[:, c["i3"][0][j], :] += dA2[:, j, :]
    dz2 = da2 * (c["z2"] > 0)
    g["b2"] = dz2.sum((0, 1))
    g["w2"] = np.einsum("nro,nrji->oij", dz2, c["A1"])
    dA1 = np.einsum("nro,oij->nrji", dz2, w["w2"]) * c["ok2"][None, :, :, None]
    da1 = np.zeros((n, 7, 32))
    for r in range(2):
        for j in range(5):
            if c["ok2"][r, j]:
                da1[:, c["i2"][r, j], :] += dA1[:, r, j, :]
    dm1 = da1 * (c["m1"] > 0)
    g["b1"] = dm1.sum((0, 1))
    g["w1"] = np.einsum("npo,npj->oj", dm1, c["X1"])
    return loss, flatten(g)


def scores(curves, flat, emulate=True):
    logit, _ = forward(curves, flat, emulate)
    return 1.0 / (1.0 + np.exp(-logit))


def auc(score_invalid, labels_valid):
    """Area under the ROC curve for ranking INVALID pixels first by
    score_invalid (higher = more likely invalid); ties count one half."""
    s = np.asarray(score_invalid, np.float64).ravel()
    inv = ~np.asarray(labels_valid, bool).ravel()
    n_pos, n_neg = int(inv.sum()), int((~inv).sum())
    if n_pos == 0 or n_neg == 0:
        return float("nan")
    order = np.argsort(s, kind="mergesort")
    ss = s[order]
    ranks = np.empty(s.size)
    # average ranks over ties
    pos = np.arange(1, s.size + 1, dtype=np.float64)
    starts = np.r_[0, np.flatnonzero(np.diff(ss)) + 1]
    ends = np.r_[starts[1:], s.size]
    avg = (pos[starts] + pos[ends - 1]) / 2.0
    ranks[order] = np.repeat(avg, ends - starts)
    return float((ranks[inv].sum() - n_pos * (n_pos + 1) / 2.0) / (n_pos * n_neg))
