"""Training and evaluation of the learned confidence net (ct_confnet_*).

The net replaces the right-to-left pass of the left-right check: it reads each
pixel's census cost curve (D = 128) from the left-to-right pass, re-centred
on the pixel's winning disparity, and scores how likely that winner-take-all
disparity is correct. Everything it
learns from is produced by the library itself on seeded synthetic pairs:

  * pairs: ct_synth_pair kind 1 (fractal-noise texture, 8 fronto-parallel
    rectangles over a background, occlusions filled with fresh noise);
    --kinds 1,2 alternates it with kind 2 (24 slanted planes);
  * cost curves and winner-take-all disparities: ct_bm_census_process_curves;
  * labels: a pixel with a disparity is "correct" iff it is not occluded in
    the right view and |d_wta - d_gt| <= 1 (generator ground truth);
  * baseline: the plain left-right check (ct_bm_census_process_lr, tolerance
    1), which flags a pixel as invalid when the two directions disagree.

Quality is the area under the ROC curve for ranking INVALID pixels first
(net: by 1 - score; left-right check: by its binary flag, ties counted half),
accumulated exactly over all pixels with a disparity of the evaluation pairs.

Usage (training runs on the GPU with the library's own kernels):
    python module.clutec.cuda_b200/confnet_train.py --train-pairs 2000 \\
        --eval-pairs 200 --out module.clutec.cuda_b200/confnet_census128.f32
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

_PKG = Path(__file__).resolve().parent
if str(_PKG) not in sys.path:
    sys.path.insert(0, str(_PKG))
import ctstereo as ct  # noqa: E402

D = 128
KIND = 1
WEIGHTS = _PKG / "confnet_census128.f32"
TRAIN_SEED0 = 1_000_000   # training pairs use seeds TRAIN_SEED0 + i
EVAL_SEED0 = 9_000_000    # held-out pairs use seeds EVAL_SEED0 + i
N_BINS = 1 << 16


def load_weights(path=WEIGHTS) -> np.ndarray:
    p = np.fromfile(path, dtype="<f4")
    if p.size != ct.CT_CONFNET_PARAMS:
        raise ValueError(f"{path}: {p.size} floats, expected {ct.CT_CONFNET_PARAMS}")
    return p


def save_weights(params: np.ndarray, path=WEIGHTS) -> None:
    np.asarray(params, dtype="<f4").tofile(path)


def _pairs(seeds, W, H, kind=KIND):
    """Seeded pairs, generated one ahead on a worker thread."""
    with ThreadPoolExecutor(1) as ex:
        fut = ex.submit(ct.synth_pair, kind, int(seeds[0]), W, H, D - 1)
        for k in range(len(seeds)):
            cur = fut.result()
            if k + 1 < len(seeds):
                fut = ex.submit(ct.synth_pair, kind, int(seeds[k + 1]), W, H, D - 1)
            yield cur


def _labels(disp_u16, gt, occ):
    """(has_disparity, correct) masks from a U16 winner-take-all map."""
    d = disp_u16.astype(np.int32)
    has = (d >= 1) & (d <= D)
    correct = has & (occ == 0) & (np.abs(d - 1 - gt.astype(np.int32)) <= 1)
    return has, correct


class _Device:
    def __init__(self, device, W, H):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        self.W, self.H = W, H
        self.m = ct.BlockMatcherCensus()
        self.m.configure(device, W, H, D)
        self.cv = ct.CurveVolume(W, H, D, self.dev)
        self.disp = ct.alloc_image(H, W, torch.int16, self.dev)
        self.chk = ct.alloc_image(H, W, torch.int16, self.dev)
        self.L = ct.alloc_image(H, W, torch.uint8, self.dev)
        self.R = ct.alloc_image(H, W, torch.uint8, self.dev)
        self.score = ct.alloc_image(H, W, torch.float32, self.dev)

    def upload(self, L, R):
        self.L.copy_(self.torch.from_numpy(L))
        self.R.copy_(self.torch.from_numpy(R))

    def curves(self):
        self.m.process_curves(self.disp, self.cv, self.L, self.R)
        return self.disp.cpu().numpy().view(np.uint16)


def _mixed_pairs(seeds, W, H, kinds):
    """Seeded pairs, pair i of generator kind kinds[i % len(kinds)]."""
    with ThreadPoolExecutor(1) as ex:
        nxt = lambda k: ex.submit(ct.synth_pair, kinds[k % len(kinds)], int(seeds[k]), W, H, D - 1)  # noqa: E731
        fut = nxt(0)
        for k in range(len(seeds)):
            cur = fut.result()
            if k + 1 < len(seeds):
                fut = nxt(k + 1)
            yield cur


def make_training_set(net, device=0, n_pairs=2000, W=640, H=480, per_pair=2048, seed=0, log=None, kinds=(KIND,)):
    """Samples (n, 128) uint8 and labels (n,) uint8 on the GPU; pair i comes
    from generator kind kinds[i % len(kinds)]."""
    import torch
    g = _Device(device, W, H)
    rng = np.random.default_rng(seed)
    n = n_pairs * per_pair
    samples = torch.empty((n, D), dtype=torch.uint8, device=g.dev)
    labels = np.empty(n, np.uint8)
    seeds = TRAIN_SEED0 + np.arange(n_pairs)
    t0 = time.perf_counter()
    for i, (L, R, G, O) in enumerate(_mixed_pairs(seeds, W, H, kinds)):
        g.upload(L, R)
        has, correct = _labels(g.curves(), G, O)
        idx = np.flatnonzero(has.ravel())
        pick = rng.choice(idx, per_pair, replace=idx.size < per_pair)
        xy = np.stack([pick % W, pick // W], 1).astype(np.int32)
        net.gather(samples[i * per_pair:(i + 1) * per_pair], g.cv, g.disp, torch.from_numpy(xy).to(g.dev))
        labels[i * per_pair:(i + 1) * per_pair] = correct.ravel()[pick]
        if log and (i + 1) % 250 == 0:
            log(f"  training pairs {i + 1}/{n_pairs} ({time.perf_counter() - t0:.1f} s)")
    torch.cuda.synchronize()
    return samples, torch.from_numpy(labels).to(g.dev)


def train(net, samples, labels, steps=6000, batch=8192, lr=3e-3, seed=0, log=None):
    """Adam with a cosine learning-rate decay on random minibatches."""
    import torch
    n = samples.shape[0]
    gen = torch.Generator(device=samples.device)
    gen.manual_seed(seed)
    loss = torch.empty(1, dtype=torch.float32, device=samples.device)
    hist = []
    for s in range(steps):
        idx = torch.randint(0, n, (batch,), device=samples.device, generator=gen)
        cur = lr * 0.5 * (1.0 + math.cos(math.pi * s / steps)) + 1e-5
        report = s % 500 == 0 or s == steps - 1
        net.train_step(samples.index_select(0, idx), labels.index_select(0, idx), cur, loss if report else None)
        if report:
            hist.append((s, float(loss.item())))
            if log:
                log(f"  step {s:5d}  loss {hist[-1][1]:.4f}  lr {cur:.2e}")
    return hist


def _auc_from_hist(h_inv, h_val):
    """AUC of ranking invalid pixels first by a score whose histograms are
    h_inv / h_val over increasing bins of 'invalidity' (ties count half)."""
    n_inv, n_val = h_inv.sum(), h_val.sum()
    below = np.cumsum(h_val) - h_val  # valid pixels with a strictly lower bin
    return float((h_inv * (below + 0.5 * h_val)).sum() / (float(n_inv) * float(n_val)))


def _matched_operating_point(h_inv, h_val, fpr_target):
    """Flagging the pixels whose invalidity bin is >= k: the smallest k whose
    false-positive rate (valid pixels flagged) is <= fpr_target; returns
    (tpr, fpr, score threshold 1 - k / N_BINS)."""
    val_tail = np.cumsum(h_val[::-1])[::-1] / max(1, h_val.sum())   # FPR when flagging bins >= k
    inv_tail = np.cumsum(h_inv[::-1])[::-1] / max(1, h_inv.sum())
    ok = np.flatnonzero(val_tail <= fpr_target)
    k = int(ok[0]) if ok.size else N_BINS
    if k >= N_BINS:
        return 0.0, 0.0, 0.0
    return float(inv_tail[k]), float(val_tail[k]), 1.0 - k / N_BINS


def evaluate(nets, device=0, n_pairs=200, W=1920, H=1080, log=None, kind=KIND, threshold=0.5):
    """AUCs over held-out pairs of generator `kind`: {name: auc} for each net
    in `nets` (a dict name -> ConfNet) plus 'lr_check', the invalid-pixel
    statistics, and each net's operating points: its true/false-positive
    rates for flagging invalid pixels at score < threshold (the threshold the
    checked map uses) and at the score threshold whose false-positive rate
    matches the left-right check's."""
    g = _Device(device, W, H)
    hists = {k: (np.zeros(N_BINS, np.int64), np.zeros(N_BINS, np.int64)) for k in nets}
    at_thr = {k: np.zeros((2, 2), np.int64) for k in nets}  # [invalid?][score < threshold?]
    lr_counts = np.zeros((2, 2), np.int64)  # [invalid?][flagged?]
    seeds = EVAL_SEED0 + (0 if kind == KIND else 100_000 * kind) + np.arange(n_pairs)
    t0 = time.perf_counter()
    for i, (L, R, G, O) in enumerate(_pairs(seeds, W, H, kind)):
        g.upload(L, R)
        g.m.process_lr(g.L, g.R, disp_checked=g.chk, tol=1)
        has, correct = _labels(g.curves(), G, O)
        flagged = g.chk.cpu().numpy().view(np.uint16) == 0xFFFA
        inv = has & ~correct
        val = has & correct
        lr_counts[1, 1] += int((inv & flagged).sum())
        lr_counts[1, 0] += int((inv & ~flagged).sum())
        lr_counts[0, 1] += int((val & flagged).sum())
        lr_counts[0, 0] += int((val & ~flagged).sum())
        for name, net in nets.items():
            net.infer(g.score, g.cv, g.disp)
            s = g.score.cpu().numpy()
            b = np.minimum((((1.0 - s) * N_BINS)).astype(np.int64), N_BINS - 1)  # invalidity bin
            hists[name][0][:] += np.bincount(b[inv], minlength=N_BINS)
            hists[name][1][:] += np.bincount(b[val], minlength=N_BINS)
            low = s < threshold
            at_thr[name] += np.array([[int((val & ~low).sum()), int((val & low).sum())],
                                      [int((inv & ~low).sum()), int((inv & low).sum())]], np.int64)
        if log and (i + 1) % 25 == 0:
            log(f"  eval pairs {i + 1}/{n_pairs} ({time.perf_counter() - t0:.1f} s)")
    out = {name: _auc_from_hist(*hists[name]) for name in nets}
    tpr = lr_counts[1, 1] / max(1, lr_counts[1].sum())
    fpr = lr_counts[0, 1] / max(1, lr_counts[0].sum())
    out["lr_check"] = 0.5 * (1.0 + tpr - fpr)
    out["lr_check_tpr"] = float(tpr)
    out["lr_check_fpr"] = float(fpr)
    out["invalid_fraction"] = float(lr_counts[1].sum() / max(1, lr_counts.sum()))
    out["pixels"] = int(lr_counts.sum())
    out["pairs"] = int(n_pairs)
    out["kind"] = int(kind)
    for name in nets:
        c = at_thr[name]
        out[f"{name}_tpr"] = float(c[1, 1] / max(1, c[1].sum()))
        out[f"{name}_fpr"] = float(c[0, 1] / max(1, c[0].sum()))
        out[f"{name}_threshold"] = float(threshold)
        m_tpr, m_fpr, m_thr = _matched_operating_point(*hists[name], out["lr_check_fpr"])
        out[f"{name}_tpr_at_lr_fpr"], out[f"{name}_fpr_at_lr_fpr"] = m_tpr, m_fpr
        out[f"{name}_threshold_at_lr_fpr"] = m_thr
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--train-pairs", type=int, default=2000)
    ap.add_argument("--train-size", default="640x480")
    ap.add_argument("--per-pair", type=int, default=2048)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--eval-pairs", type=int, default=200)
    ap.add_argument("--eval-size", default="1920x1080")
    ap.add_argument("--kinds", default="1",
                    help="generator kinds of the training pairs, alternating (1: fronto-parallel rectangles, "
                         "2: slanted planes)")
    ap.add_argument("--out", default=str(WEIGHTS))
    ap.add_argument("--report", default=None, help="write the JSON summary here too")
    a = ap.parse_args(argv)
    log = lambda msg: print(msg, file=sys.stderr, flush=True)  # noqa: E731
    tw, th = map(int, a.train_size.split("x"))
    ew, eh = map(int, a.eval_size.split("x"))
    net = ct.ConfNet()
    net.configure(a.device, a.batch)
    net.init(1)
    t0 = time.perf_counter()
    kinds = tuple(int(k) for k in a.kinds.split(","))
    samples, labels = make_training_set(net, a.device, a.train_pairs, tw, th, a.per_pair, log=log, kinds=kinds)
    t_data = time.perf_counter() - t0
    t0 = time.perf_counter()
    hist = train(net, samples, labels, a.steps, a.batch, a.lr, log=log)
    t_train = time.perf_counter() - t0
    params = net.get_params()
    save_weights(params, a.out)
    untrained = ct.ConfNet()
    untrained.configure(a.device, 16)
    untrained.init(1)
    res = {f"kind{k}": evaluate({"net": net, "untrained": untrained}, a.device, a.eval_pairs, ew, eh, log=log,
                                 kind=k) for k in (1, 2)}
    summary = {"train_pairs": a.train_pairs, "train_kinds": list(kinds), "train_size": a.train_size,
               "samples": int(samples.shape[0]),
               "positive_fraction": float(labels.float().mean().item()), "steps": a.steps, "batch": a.batch,
               "lr": a.lr, "loss_history": hist, "data_s": round(t_data, 1), "train_s": round(t_train, 1),
               "eval_size": a.eval_size, "auc": res, "weights": str(a.out)}
    print(json.dumps(summary))
    if a.report:
        Path(a.report).write_text(json.dumps(summary, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())
