#!/usr/bin/env python
"""bench.py — census stereo matching throughput on B200.

Default workload (one "step"): the census stereo pipeline on one seeded
synthetic 1920x1080 pair with D = 128: 9x7 census of both images, census
Hamming cost + 5x5 box aggregation + winner-take-all left-to-right AND
right-to-left, then the left-right cross-check with tolerance 1 px. The metric
counts pixel x disparity evaluations: 2 directions x W x H x D per step.

  value       device time of the whole pipeline, inputs resident in HBM, L2
              flushed (256 MiB memset) before every timed step.
  e2e         the same pipeline through the public C ABI with host buffers,
              as a stream of frames (ct_census_stream_*): every frame's two
              images copied in from pinned host memory and its checked map
              copied out, the copies of neighbouring frames overlapping the
              matching; device time from before the first upload to the end
              of the last download. e2e.serial is the one-frame-at-a-time
              variant (copies in line with the matching on one stream).
  roofline    the dominant kernel (the fused matching pass: each 5x5 Hamming
              cost evaluated once, both directions' winners) timed with CUDA
              events on its stream, against the POPC-pipe bound (2 POPC per
              cost) measured live on this GPU by ct_probe_pipe_rates; also the
              one-direction kernel of process() alone.
  cpu_baseline  the CPU restatement (OpenMP, all host threads) on the same
              pair, rank 0 only.

--impl reference times that CPU implementation of the pipeline (the
reference's own code cannot be built, so the oracle port stands in for it).
Multi-GPU: independent replicas, one pair per rank ("scaling": "weak"), no
collective on the data path; timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "module.clutec.cuda_b200"))

W_, H_, D_ = 1920, 1080, 128
SEED = 2024
METRIC = "Mpix*disp/s census 9x7 + 5x5 Hamming + L-R check, 1920x1080 D=128"
UNIT = "Mpix*disp/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="census1080",
                    choices=["census1080", "sad640", "ncc1080", "ncc1080g", "aw1440", "batch64", "confnet1080",
                             "compat1080", "mip1080", "map3d1080"],
                    help="census1080 (default, the headline) or another configuration, one JSON line each")
    ap.add_argument("--eval-pairs", type=int, default=None,
                    help="held-out 1080p pairs for the confidence-net AUC (default 4 in the census line, 24 in confnet1080)")
    ap.add_argument("--profile", default=None,
                    choices=["census_match", "census_fused", "confnet_infer", "pipelines", "sad640", "ncc1080",
                             "ncc1080_cuda_cores", "aw1440", "batch64", "compat_ncc1080"],
                    help="for ncu captures, then exit: census_match or confnet_infer = that kernel twice on the "
                         "1080p D=128 pair; pipelines = the plain L-R pipeline 3x (one fused pass), 3x in two "
                         "passes, then the learned one 3x; a "
                         "configuration name = its step twice (no autotuning, no CPU work); ncc1080_cuda_cores = "
                         "the ncc1080 step with the window sums on the CUDA cores")
    ap.add_argument("--no-configs", action="store_true",
                    help="default run: measure the headline only, without the other configurations")
    return ap.parse_args()


def dist_info():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(
        os.environ.get("LOCAL_RANK", 0))


# Ranks are independent replicas (one pair per GPU, no collective on the data
# path); the only collectives are barriers around the timed regions and the
# max over ranks of the timings. NCCL on GPUs, gloo for CPU processes.
def init_ranks(world, dev):
    if world > 1:
        import datetime
        import torch.distributed as dist
        kw = {"device_id": dev} if dev.type == "cuda" else {}
        dist.init_process_group("nccl" if dev.type == "cuda" else "gloo",
                                timeout=datetime.timedelta(seconds=120), **kw)


def rank_barrier(world, dev):
    import torch
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(v, world, dev):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def close_ranks(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def replica_seed(rank):
    """Each replica matches its own seeded pair."""
    return SEED + rank


def units_per_step():
    return 2 * W_ * H_ * D_


def census_config():
    """The headline workload, identical in both arms."""
    return {"workload": "census9x7_5x5_lrcheck_1920x1080_d128", "width": W_, "height": H_, "D": D_,
            "census": "9x7", "agg": "5x5", "crosscheck_tol": 1, "seed": SEED, "generator": "kind 2 (slanted planes)",
            "l2": "GPU L2 flushed before every timed step (256 MiB memset); the CPU arm has no GPU L2"}


_ORACLE = None


def cpu_oracle():
    """The CPU restatement (oracle/), built on this host with -march=native
    for the timed CPU legs; -> (module, march actually used)."""
    global _ORACLE
    if _ORACLE is None:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle  # the CPU restatement: CPU baseline, reference arm and parity checks only
        march = oracle.use_native()
        oracle.lib()
        _ORACLE = (oracle, march)
    return _ORACLE


# ---------------------------------------------------------------------------
# CPU implementation (oracle port) — the cpu_baseline leg and --impl reference
# ---------------------------------------------------------------------------

def cpu_pipeline_time(L, R, reps: int) -> tuple[float, int]:
    oracle, _ = cpu_oracle()
    t0 = time.perf_counter()
    for _ in range(reps):
        dl, _ = oracle.match_census(L, R, D_, 2, True)
        dr, _ = oracle.match_census(L, R, D_, 2, False)
        oracle.crosscheck(dl, dr, 1, True)
    return (time.perf_counter() - t0) / reps, oracle.num_threads()


def run_reference(args):
    rank, world, _ = dist_info()
    if rank != 0:
        return 0
    import ctstereo as ct
    L, R, _, _ = ct.synth_pair(2, SEED, W_, H_, D_ - 1)
    for _ in range(args.warmup):
        cpu_pipeline_time(L, R, 1)
    times = []
    for _ in range(args.steps):
        t, cores = cpu_pipeline_time(L, R, 1)
        times.append(t)
    ms = 1e3 * sum(times) / len(times)
    value = units_per_step() / (ms * 1e-3) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8 pixels / u64 census / int costs",
        "data": "synthetic (seeded generator)", "config": census_config(),
        "cpu_baseline": {"value": round(value, 1), "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": "one full 1920x1080 D=128 pipeline per step (LR + RL + check)",
                         "build": f"-O3 -march={cpu_oracle()[1]} -fopenmp"},
        "e2e": {"value": round(value, 1), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during timing."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        for ln in Path(self.f.name).read_text().splitlines():
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def traffic_from_profile():
    """DRAM bytes per launch of the fused census_match_kernel (the headline's
    dominant kernel) from the committed ncu summary."""
    p = ROOT / "profiles" / "census_match_1080p_d128.json"
    if p.exists():
        try:
            return json.loads(p.read_text()).get("dram_bytes_per_launch")
        except Exception:
            return None
    return None


def confnet_compare(ct, dev, stream, m, dL, dR, hL, hR, flush, steps, eval_pairs, device_index):
    """The learned-confidence pipeline against the plain left-right pipeline
    on the resident pair, both producing the same checked U8 map:
      plain   ct_bm_census_process_lr (census x2, L->R, R->L, cross-check)
      learned ct_bm_census_process_curves (census x2, L->R + cost curves) +
              ct_confnet_infer (checked map = L->R with low scores marked)
    Device time and end-to-end time (pinned H2D of both images + D2H of the
    checked map in every step), and the invalid-pixel AUC of both methods
    over held-out 1080p pairs with the committed weights."""
    import torch
    import confnet_train as T
    net = ct.ConfNet()
    net.configure(device_index, 16)
    net.set_params(T.load_weights())
    cv = ct.CurveVolume(W_, H_, D_, dev)
    disp = ct.alloc_image(H_, W_, torch.uint8, dev)
    ck_plain = ct.alloc_image(H_, W_, torch.uint8, dev)
    ck_learned = ct.alloc_image(H_, W_, torch.uint8, dev)
    hOut = torch.empty((H_, W_), dtype=torch.uint8).pin_memory()

    def plain():
        m.process_lr(dL, dR, disp_checked=ck_plain, tol=1, stream=stream)

    def learned():
        m.process_curves(disp, cv, dL, dR, stream=stream)
        net.infer(None, cv, disp, checked=ck_learned, threshold=0.5, stream=stream)

    def timed(fn, out=None):
        for _ in range(3):
            flush()
            fn()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize(dev)
        for k in range(steps):
            flush()
            ev[k][0].record(stream)
            if out is not None:
                dL.copy_(hL, non_blocking=True)
                dR.copy_(hR, non_blocking=True)
            fn()
            if out is not None:
                hOut.copy_(out, non_blocking=True)
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
        return sum(a.elapsed_time(b) for a, b in ev) / steps

    res = {"plain_ms": timed(plain), "learned_ms": timed(learned),
           "plain_e2e_ms": timed(plain, ck_plain), "learned_e2e_ms": timed(learned, ck_learned),
           "infer_ms": timed(lambda: net.infer(None, cv, disp, checked=ck_learned, threshold=0.5, stream=stream))}
    # the plain pipeline as the reference runs it: one matching pass per
    # direction (the default process_lr decides both from one pass)
    m.set_fused_lr(False)
    res["plain_two_pass_ms"] = timed(plain)
    res["plain_two_pass_e2e_ms"] = timed(plain, ck_plain)
    m.set_fused_lr(True)
    if m.device_status() != 0 or net.device_status() != 0:
        raise RuntimeError("device status set in the confidence-net comparison")
    res = {k: round(v, 4) for k, v in res.items()}
    # quality on held-out pairs of the training generator (kind 1) and of the
    # headline's slanted-plane generator (kind 2)
    evals = {}
    for kind in (1, 2):
        a = T.evaluate({"net": net}, device_index, eval_pairs, W_, H_, kind=kind)
        evals[f"kind{kind}"] = {
            "auc_net": round(a["net"], 4), "auc_lr_check": round(a["lr_check"], 4),
            "lr_check_tpr": round(a["lr_check_tpr"], 4), "lr_check_fpr": round(a["lr_check_fpr"], 5),
            "net_tpr_at_0.5": round(a["net_tpr"], 4), "net_fpr_at_0.5": round(a["net_fpr"], 5),
            "net_tpr_at_lr_fpr": round(a["net_tpr_at_lr_fpr"], 4),
            "net_fpr_at_lr_fpr": round(a["net_fpr_at_lr_fpr"], 5),
            "net_threshold_at_lr_fpr": round(a["net_threshold_at_lr_fpr"], 4),
            "invalid_fraction": round(a["invalid_fraction"], 4), "eval_pairs": a["pairs"],
            "eval_pixels": a["pixels"]}
    auc = evals["kind1"]
    macs = 1120 + 9216 + 2048 + 2048 + 64  # per pixel: conv1, conv2, conv3, fc1, fc2
    flops = 2.0 * macs * W_ * H_
    try:
        peak, src = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["bf16_tflops"], "of measured (burst)"
    except (OSError, KeyError, ValueError):
        peak, src = 1590.0, "of fallback"
    ach = flops / (res["infer_ms"] * 1e-3) / 1e12
    res.update({"speedup": round(res["plain_ms"] / res["learned_ms"], 3),
                "speedup_e2e": round(res["plain_e2e_ms"] / res["learned_e2e_ms"], 3),
                "speedup_vs_two_pass": round(res["plain_two_pass_ms"] / res["learned_ms"], 3),
                "speedup_e2e_vs_two_pass": round(res["plain_two_pass_e2e_ms"] / res["learned_e2e_ms"], 3),
                "auc_net": auc["auc_net"], "auc_lr_check": auc["auc_lr_check"],
                "lr_check_tpr": auc["lr_check_tpr"], "lr_check_fpr": auc["lr_check_fpr"],
                "invalid_fraction": auc["invalid_fraction"], "eval_pairs": auc["eval_pairs"],
                "eval_pixels": auc["eval_pixels"], "threshold": 0.5, "eval": evals,
                "eval_200_pairs": "module.clutec.cuda_b200/confnet_census128.json (200 held-out kind-1 pairs)",
                "infer_roofline": {"bound": "tensor", "achieved": round(ach, 2), "peak": peak, "unit": "TFLOP/s",
                                   "frac": round(ach / peak, 4), "traffic": None, "peak_source": src,
                                   "algorithmic_per_unit": f"{macs} MAC per pixel (bf16 x bf16, fp32 accumulate)"},
                "weights": "module.clutec.cuda_b200/confnet_census128.f32 (2000 seeded training pairs)",
                "launches_learned": 3, "launches_plain": 3, "launches_plain_two_pass": 4,
                "plain_note": "plain = process_lr in one matching pass (both directions' winners from the "
                              "left-to-right costs); plain_two_pass = one pass per direction"})
    return res


def confnet_entry(c):
    """The learned-confidence pipeline as an entry of the default run's configs."""
    return {"metric": "frames/s census 1080p D=128 + learned confidence (replaces the R->L pass and the L-R check)",
            "value": round(1e3 / c["learned_ms"], 1), "unit": "frames/s", "ms_per_step": c["learned_ms"],
            "plain_lr_pipeline_ms": c["plain_ms"], "speedup": c["speedup"], "speedup_e2e": c["speedup_e2e"],
            "plain_two_pass_ms": c["plain_two_pass_ms"], "speedup_vs_two_pass": c["speedup_vs_two_pass"],
            "speedup_e2e_vs_two_pass": c["speedup_e2e_vs_two_pass"],
            "roofline": c["infer_roofline"], "eval": c["eval"],
            "config": {"workload": "confnet_1920x1080_d128", "width": W_, "height": H_, "D": D_},
            "gpu_launches": None}


def run_ours(args):
    import torch
    import ctstereo as ct

    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    init_ranks(world, dev)
    stream = torch.cuda.current_stream(dev)

    L, R, G, O = ct.synth_pair(2, replica_seed(rank), W_, H_, D_ - 1)
    dL = ct.alloc_image(H_, W_, torch.uint8, dev)
    dR = ct.alloc_image(H_, W_, torch.uint8, dev)
    dL.copy_(torch.from_numpy(L))
    dR.copy_(torch.from_numpy(R))
    lr = ct.alloc_image(H_, W_, torch.uint8, dev)
    rl = ct.alloc_image(H_, W_, torch.uint8, dev)
    ck = ct.alloc_image(H_, W_, torch.uint8, dev)
    m = ct.BlockMatcherCensus()
    m.configure(local, W_, H_, D_)
    tuning = m.autotune(dL, dR, stream=stream)  # one-time launch-shape search (configure cost)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def flush():
        flush_buf.zero_()

    def step():
        m.process_lr(dL, dR, disp_lr=lr, disp_rl=rl, disp_checked=ck, tol=1, stream=stream)

    # pipe-rate peaks for the integer roofline
    rates = ct.probe_pipe_rates(local)

    def barrier():
        rank_barrier(world, dev)

    for _ in range(max(3, args.warmup)):
        flush()
        step()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    with ClockSampler(torch.cuda.current_device()) as clk:
        for k in range(args.steps):
            flush()
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        barrier()
        step_ms = [a.elapsed_time(b) for a, b in ev]
        total_ms = max_over_ranks(sum(step_ms), world, dev)

        # dominant kernel: one left-to-right pass (census of both images in
        # one launch + census_match_kernel) minus that census launch, both
        # timed here with events on the launching stream
        desc_l = ct.alloc_image(H_, W_, torch.int64, dev)
        desc_r = ct.alloc_image(H_, W_, torch.int64, dev)
        cen = ct.CensusTransform()
        cen.configure(local, W_, H_)
        for _ in range(3):
            m.process(lr, dL, dR, stream=stream)
        kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        cev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        barrier()
        for k in range(args.steps):
            flush()
            kev[k][0].record(stream)
            m.process(lr, dL, dR, stream=stream)
            kev[k][1].record(stream)
            flush()
            cev[k][0].record(stream)
            cen.process_pair(desc_l, desc_r, dL, dR, stream=stream)  # the launch process() makes
            cev[k][1].record(stream)
        barrier()
        census_ms = sum(a.elapsed_time(b) for a, b in cev) / args.steps
        match_ms = sum(a.elapsed_time(b) for a, b in kev) / args.steps - census_ms
        # the headline step's dominant kernel: the fused pass (left-to-right
        # winners, and the right-to-left ones from the same costs), timed as
        # process_lr(lr, rl) minus the census launch (the right-view finalize,
        # a few microseconds, stays in)
        fev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        barrier()
        for k in range(args.steps):
            flush()
            fev[k][0].record(stream)
            m.process_lr(dL, dR, disp_lr=lr, disp_rl=rl, stream=stream)
            fev[k][1].record(stream)
        barrier()
        fused_ms = sum(a.elapsed_time(b) for a, b in fev) / args.steps - census_ms

        # end-to-end through the public API with host buffers
        hL = torch.from_numpy(L).pin_memory()
        hR = torch.from_numpy(R).pin_memory()
        hOut = torch.empty((H_, W_), dtype=torch.uint8).pin_memory()
        for _ in range(2):
            dL.copy_(hL, non_blocking=True)
            dR.copy_(hR, non_blocking=True)
            step()
            hOut.copy_(ck, non_blocking=True)
        eev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(args.steps)]
        barrier()
        for k in range(args.steps):
            flush()
            eev[k][0].record(stream)
            dL.copy_(hL, non_blocking=True)
            dR.copy_(hR, non_blocking=True)
            step()
            hOut.copy_(ck, non_blocking=True)
            eev[k][1].record(stream)
        barrier()
        e2e_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in eev) / args.steps, world, dev)

        # end-to-end as a stream of frames through ct_census_stream_*: the
        # same host buffers, every frame uploaded and its checked map
        # downloaded, neighbouring frames' copies overlapping the matching
        cs = ct.CensusStream()
        cs.configure(local, W_, H_, D_, tol=1)
        souts = [torch.empty((H_, W_), dtype=torch.uint8).pin_memory() for _ in range(3)]
        for i in range(3):
            k = cs.submit(hL, hR, souts[i])
        cs.wait(k)
        barrier()
        cs.timer_start()
        for i in range(args.steps):
            k = cs.submit(hL, hR, souts[i % 3])
        stream_ms = max_over_ranks(cs.timer_stop() / args.steps, world, dev)
        cs.wait(k)
        if cs.device_status() != 0:
            raise RuntimeError("device status set in the streamed run")
        stream_ok = bool(torch.equal(souts[(args.steps - 1) % 3], hOut))
        conf = confnet_compare(ct, dev, stream, m, dL, dR, hL, hR, flush, args.steps,
                               args.eval_pairs or 12, local) if rank == 0 else None
    clocks = clk.summary()

    status = m.device_status()
    if status != 0:
        raise RuntimeError(f"device status {status} after the timed runs")

    # correctness of the timed step's three maps against the oracle (rank 0)
    parity = None
    if rank == 0:
        import numpy as np
        oracle, _ = cpu_oracle()
        want_l, _ = oracle.match_census(L, R, D_, 2, True)
        want_r, _ = oracle.match_census(L, R, D_, 2, False)
        want_c, _ = oracle.crosscheck(want_l, want_r, 1, True)
        parity = {name: bool(np.array_equal(got.cpu().numpy(), oracle.to_u8(np.where(want == -2, -1, want))))
                  for name, got, want in (("lr", lr, want_l), ("rl", rl, want_r), ("checked", ck, want_c))}
        parity["all"] = all(parity.values())

    ms = total_ms / args.steps
    value = world * units_per_step() / (ms * 1e-3) / 1e6
    e2e = world * units_per_step() / (e2e_ms * 1e-3) / 1e6
    e2e_stream = world * units_per_step() / (stream_ms * 1e-3) / 1e6

    sms = rates["sm_count"]
    clock_hz = (clocks["sm_mhz"] or rates["sm_clock_mhz"]) * 1e6
    popc_peak = rates["popc_per_clk_sm"] * sms * clock_hz          # POPC ops / s
    units_launch = W_ * H_ * D_
    # the fused pass evaluates each 5x5 Hamming cost C(x, d) once (2 POPC)
    # and decides both directions' winners from it
    achieved_popc = 2.0 * units_launch / (fused_ms * 1e-3)
    single_popc = 2.0 * units_launch / (match_ms * 1e-3)           # one direction alone, 2 POPC per unit
    int_peak = rates["iadd3_per_clk_sm"] * sms * clock_hz
    launches = 3  # census of both views, the fused matching pass, the right-view map + cross-check

    out = {
        "metric": METRIC, "value": round(value, 1), "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8 pixels / u64 census / int costs", "data": "synthetic (seeded generator)",
        "config": census_config(), "parallelism": f"replicas x{world}", "launch_shape": tuning,
        "e2e": {"value": round(e2e_stream, 1), "unit": UNIT, "ms_per_step": round(stream_ms, 4),
                "h2d_bytes_per_step": 2 * W_ * H_, "d2h_bytes_per_step": W_ * H_,
                "api": "ct_census_stream_submit per frame (pinned host images in, checked map out), "
                       "device time from before the first upload to the end of the last download; "
                       "no L2 flush between frames (every frame's inputs are fresh host copies)",
                "same_map_as_serial": stream_ok,
                "serial": {"value": round(e2e, 1), "ms_per_step": round(e2e_ms, 4),
                           "api": "ct_bm_census_process_lr with the copies in line on one stream, "
                                  "L2 flushed before every step"}},
        "roofline": {"bound": "popc", "achieved": round(achieved_popc / 1e12, 4),
                     "peak": round(popc_peak / 1e12, 4), "unit": "Tpopc/s",
                     "frac": round(achieved_popc / popc_peak, 4),
                     "traffic": traffic_from_profile(),
                     "kernel": "census_match_kernel<0,4,false,true> (the fused pass: 5x5 Hamming costs of "
                               "1920x1080x128 evaluated once, left-to-right and right-to-left winners; timed as "
                               "process_lr(lr, rl) minus the census transform of both views)",
                     "kernel_ms": round(fused_ms, 4), "census_transform_ms": round(census_ms, 4),
                     "algorithmic_per_unit": "2 POPC per cost C(x, d), one cost per pixel x disparity for both "
                                             "directions (+ ~9 INT per direction's winner-take-all)",
                     "frac_per_direction_units": round(2 * achieved_popc / popc_peak, 4),
                     "frac_per_direction_units_note": "2 W H D direction units per step (the metric's units) "
                                                      "x 2 POPC each against the same peak",
                     "single_direction": {"kernel": "census_match_kernel<0,4> (left-to-right alone, process())",
                                          "kernel_ms": round(match_ms, 4),
                                          "frac": round(single_popc / popc_peak, 4),
                                          "int_frac_at_9_ops": round(9.0 * units_launch / (match_ms * 1e-3)
                                                                     / int_peak, 4)},
                     "peak_source": "ct_probe_pipe_rates measured in this run (POPC/clk/SM x SMs x median SM clock)",
                     "pipe_rates_per_clk_sm": {k: round(v, 2) for k, v in rates.items()
                                               if k.endswith("per_clk_sm")}},
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
        "parity_rank0": parity,
        "confnet": conf,
    }
    if rank == 0:
        cpu_ms, cores = cpu_pipeline_time(L, R, 3)
        out["cpu_baseline"] = {"value": round(units_per_step() / cpu_ms / 1e6, 1), "unit": UNIT, "cores": cores,
                               "kind": "port", "sample": "3 full pipelines (1920x1080, D=128, LR+RL+check)",
                               "build": f"-O3 -march={cpu_oracle()[1]} -fopenmp"}
    if world == 1 and not args.no_configs:
        # the other configurations, one entry each (1 GPU only: at N > 1 the
        # headline alone is measured)
        out["configs"] = {}
        keys = ("metric", "value", "unit", "ms_per_step", "config", "roofline", "cpu_baseline", "parity_rank0",
                "clocks", "gpu_launches", "cuda_core_kernel")
        for wl in CONFIG_WORKLOADS:
            line = workload_line(wl, args, ct, dev, stream, flush_buf, world, rank, local, rates)
            out["configs"][wl] = {k: line.get(k) for k in keys if k in line or k != "cuda_core_kernel"}
        if conf is not None:
            out["configs"]["confnet1080"] = confnet_entry(conf)
        # the other rows of the path, beyond the five configurations: one
        # entry each; a failure is reported in its entry, not raised
        out["extras"] = {}
        for wl in EXTRA_WORKLOADS:
            try:
                line = workload_line(wl, args, ct, dev, stream, flush_buf, world, rank, local, rates)
                out["extras"][wl] = {k: line.get(k) for k in keys if k in line or k != "cuda_core_kernel"}
            except Exception as e:  # noqa: BLE001 - reported in the line
                out["extras"][wl] = {"error": f"{type(e).__name__}: {e}"}
        out["gpu_launches_configs"] = sum(v.get("gpu_launches") or 0 for d in (out["configs"], out["extras"])
                                          for v in d.values())
    if rank == 0:
        print(json.dumps(out), flush=True)
    close_ranks(world)
    return 0


def profile_config(args):
    """--profile <configuration>: that configuration's step twice on its own
    inputs (the sizes the bench measures), nothing else."""
    import torch
    import ctstereo as ct
    dev = torch.device("cuda", 0)

    def up(a):
        t = ct.alloc_image(a.shape[0], a.shape[1], torch.from_numpy(a).dtype, dev)
        t.copy_(torch.from_numpy(a))
        return t

    wl = args.profile
    if wl == "batch64":
        shapes = batch_shapes()
        pairs = []
        for i, (W, H, D) in enumerate(shapes):
            L, R, _, _ = ct.synth_pair(1, 1000 + i, W, H, D - 1)
            pairs.append((up(L), up(R), ct.alloc_image(H, W, torch.int16, dev)))
        m = ct.BatchStereo()
        m.configure(0, shapes, tol=1)
        step = lambda: m.process(pairs)
    else:
        W, H, D, kind = {"sad640": (640, 480, 64, 1), "ncc1080": (1920, 1080, 128, 2), "aw1440": (2560, 1440, 256, 3),
                         "compat_ncc1080": (1920, 1080, 128, 2), "ncc1080_cuda_cores": (1920, 1080, 128, 2)}[wl]
        L, R, _, _ = ct.synth_pair(kind, SEED, W, H, D - 1)
        dL, dR = up(L), up(R)
        if wl == "sad640":
            m = ct.BlockMatcherSAD1()
            m.configure(0, W, H, D, radius=4)
            out = ct.alloc_image(H, W, torch.uint8, dev)
            step = lambda: m.process(out, dL, dR)
        elif wl in ("ncc1080", "ncc1080_cuda_cores"):
            m = ct.BlockMatcherNCC()
            m.configure(0, W, H, D, radius=5)
            m.set_tensor_cores(wl == "ncc1080")
            out = ct.alloc_image(H, W, torch.uint8, dev)
            score = ct.alloc_image(H, W, torch.float32, dev)
            step = lambda: m.process(out, dL, dR, score=score)
        elif wl == "aw1440":
            m = ct.BlockMatcherAW()
            m.configure(0, W, H, D)
            out = ct.alloc_image(H, W, torch.float32, dev)
            step = lambda: m.process(out, dL, dR)
        else:
            m = ct.BlockMatcherCompat()
            m.configure(0, W, H, ct.CT_COMPAT_NCC, D, 11, score_thresh=0.5, min_delta_thresh=2)
            out = ct.alloc_u16x4(H, W, dev)
            step = lambda: m.process(out, dL, dR)
    for _ in range(2):
        step()
    torch.cuda.synchronize()
    if m.device_status() != 0:
        raise RuntimeError("device status set")
    return 0


def run_profile(args):
    """Two launches of one kernel on the default workload, nothing else (or
    the two pipelines, three times each, or a configuration's step twice)."""
    import torch
    import ctstereo as ct
    if args.profile not in ("census_match", "census_fused", "confnet_infer", "pipelines"):
        return profile_config(args)
    dev = torch.device("cuda", 0)
    if args.profile in ("confnet_infer", "pipelines"):
        import confnet_train as T
        L, R, _, _ = ct.synth_pair(1, SEED, W_, H_, D_ - 1)
        dL = ct.alloc_image(H_, W_, torch.uint8, dev)
        dR = ct.alloc_image(H_, W_, torch.uint8, dev)
        dL.copy_(torch.from_numpy(L))
        dR.copy_(torch.from_numpy(R))
        m = ct.BlockMatcherCensus()
        m.configure(0, W_, H_, D_)
        m.set_tuning(126, 4)
        net = ct.ConfNet()
        net.configure(0, 16)
        net.set_params(T.load_weights())
        cv = ct.CurveVolume(W_, H_, D_, dev)
        disp = ct.alloc_image(H_, W_, torch.uint8, dev)
        ck = ct.alloc_image(H_, W_, torch.uint8, dev)
        m.process_curves(disp, cv, dL, dR)
        net.infer(None, cv, disp, checked=ck)  # packs the weights
        torch.cuda.synchronize()
        if args.profile == "confnet_infer":
            for _ in range(2):
                net.infer(None, cv, disp, checked=ck)
        else:  # plain (one fused pass), plain in two passes, learned: three times each
            for fused in (True, False):
                m.set_fused_lr(fused)
                for _ in range(3):
                    m.process_lr(dL, dR, disp_checked=ck, tol=1)
            m.set_fused_lr(True)
            for _ in range(3):
                m.process_curves(disp, cv, dL, dR)
                net.infer(None, cv, disp, checked=ck)
        torch.cuda.synchronize()
        if m.device_status() != 0 or net.device_status() != 0:
            raise RuntimeError("device status set")
        return 0
    L, R, _, _ = ct.synth_pair(2, SEED, W_, H_, D_ - 1)
    dL = ct.alloc_image(H_, W_, torch.uint8, dev)
    dR = ct.alloc_image(H_, W_, torch.uint8, dev)
    dL.copy_(torch.from_numpy(L))
    dR.copy_(torch.from_numpy(R))
    desc_l = ct.alloc_image(H_, W_, torch.int64, dev)
    desc_r = ct.alloc_image(H_, W_, torch.int64, dev)
    cen = ct.CensusTransform()
    cen.configure(0, W_, H_)
    cen.process(desc_l, dL)
    cen.process(desc_r, dR)
    m = ct.BlockMatcherCensus()
    m.configure(0, W_, H_, D_)
    out = ct.alloc_image(H_, W_, torch.uint8, dev)
    if args.profile == "census_fused":  # process_lr with both maps: census x2, the fused pass, finalize
        rl = ct.alloc_image(H_, W_, torch.uint8, dev)
        for _ in range(2):
            m.process_lr(dL, dR, disp_lr=out, disp_rl=rl)
    else:
        for _ in range(2):
            m.match_desc(out, desc_l, desc_r, True)
    torch.cuda.synchronize()
    if m.device_status() != 0:
        raise RuntimeError("device status set")
    return 0


# ---------------------------------------------------------------------------
# Other configurations (--workload): one JSON line each, same timing rules
# ---------------------------------------------------------------------------

# the other configurations measured by the default run (configs entry of its line)
CONFIG_WORKLOADS = ["sad640", "ncc1080", "aw1440", "batch64"]
EXTRA_WORKLOADS = ["ncc1080g", "compat1080", "mip1080", "map3d1080"]
BATCH_SIZES = [(320, 240), (640, 480), (1280, 720), (1920, 1080)]
BATCH_DISPS = [32, 64, 128, 256]


def batch_shapes(n=64, seed=4):
    """64 pairs: sizes and D drawn uniformly (seeded) from the two lists."""
    import numpy as np
    r = np.random.default_rng(seed)
    return [(*BATCH_SIZES[int(r.integers(4))], BATCH_DISPS[int(r.integers(4))]) for _ in range(n)]


# Algorithmic cost per pixel x disparity of each matcher (the roofline's
# numerator) and the pipe that bounds it.
#   sad640 : |a - b| (2 INT) + 4 box add/sub + compare/select (2) = 8 INT
#   aw1440 : |a - b| (2) + 7x7 running box (4) + 5-window min and add (5)
#            + compare/select (2) = 13 INT
#   ncc1080: product + 4 box add/sub (5 INT) + normalisation and argmax
#            (~10 FP32/INT) = 15 lane operations at the issue rate
#            (128 per SM per clock: 4 schedulers x 32 lanes)
#   batch64: as the census headline, 2 POPC (64-bit Hamming) per direction
#            unit; the fused pass evaluates each cost once for both
#            directions, so frac counts direction units and frac_costs_once
#            the costs it evaluates
#   compat1080: the reference's per-disparity NCC (BlockMatcherNCC.cu:218-271:
#            the cross mean, the test mean and mean square, the test
#            standard deviation, the normalised and quantised score: 3
#            divisions, a square root and ~10 other FP32 operations) + the
#            window sum (5) + the scan update (~8) = 30 lane operations
ROOF = {"sad640": ("int", 8, "iadd3_per_clk_sm"), "aw1440": ("int", 13, "iadd3_per_clk_sm"),
        "ncc1080": ("issue", 15, None), "batch64": ("popc", 2, "popc_per_clk_sm"),
        "compat1080": ("issue", 30, None)}


def pipe_roofline(kind, ops_per_unit, rate_key, units_per_s, rates, sm_mhz):
    """Integer / issue roofline of a matcher: achieved operations per second
    (units/s x algorithmic ops per unit) against the pipe peak measured on
    this GPU by ct_probe_pipe_rates (per SM per clock x SMs x SM clock)."""
    clock_hz = (sm_mhz or rates["sm_clock_mhz"]) * 1e6
    per_clk = 128.0 if rate_key is None else rates[rate_key]
    peak = per_clk * rates["sm_count"] * clock_hz
    ach = units_per_s * ops_per_unit
    return {"bound": kind, "achieved": round(ach / 1e12, 4), "peak": round(peak / 1e12, 4),
            "unit": {"int": "Tintop/s", "popc": "Tpopc/s", "issue": "Tlaneop/s"}[kind],
            "frac": round(ach / peak, 4), "traffic": None, "algorithmic_per_unit": f"{ops_per_unit} {kind} ops",
            "peak_source": ("ct_probe_pipe_rates measured in this run" if rate_key else
                            "issue limit 128 lane-ops/clk/SM") + " x SMs x median SM clock"}


def workload_line(wl, args, ct, dev, stream, flush_buf, world, rank, local, rates=None):
    """Measures one configuration (--workload, or an entry of the default
    run's `configs`) with the bench's timing rules; returns the JSON line on
    rank 0 (None elsewhere)."""
    import numpy as np
    import torch
    oracle, march = cpu_oracle()  # CPU baseline leg and post-timing parity check only
    alt_kernel = None
    unit = UNIT

    def up(a):
        t = ct.alloc_image(a.shape[0], a.shape[1], torch.from_numpy(a).dtype, dev)
        t.copy_(torch.from_numpy(a))
        return t

    if wl == "batch64":
        shapes = batch_shapes()
        pairs, host = [], []
        for i, (W, H, D) in enumerate(shapes):
            L, R, _, _ = ct.synth_pair(1, 1000 + 97 * rank + i, W, H, D - 1)
            pairs.append((up(L), up(R), ct.alloc_image(H, W, torch.int16, dev)))
            host.append((L, R, D))
        b = ct.BatchStereo()
        b.configure(local, shapes, tol=1)
        ths = b.autotune(pairs, stream=stream)
        b.graph_create(pairs)
        step = lambda: b.graph_launch(stream=stream)
        units = sum(2 * W * H * D for W, H, D in shapes)
        metric = "Mpix*disp/s batched census + L-R check, 64 mixed pairs, one graph"
        cfg = {"workload": "batch64_census_lrcheck_mixed", "pairs": 64, "sizes": BATCH_SIZES, "disps": BATCH_DISPS,
               "strip_heights": sorted(set(ths))}
        check_fn = lambda: all(np.array_equal(  # every pair vs the oracle
            pairs[i][2].cpu().numpy().view(np.uint16),
            oracle.to_u16(oracle.crosscheck(oracle.match_census(host[i][0], host[i][1], host[i][2])[0],
                                            oracle.match_census(host[i][0], host[i][1], host[i][2], 2, False)[0],
                                            1, True)[0])) for i in range(len(host)))

        def cpu_sample():
            L, R, D = host[0]
            t0 = time.perf_counter()
            dl, _ = oracle.match_census(L, R, D, 2, True)
            dr, _ = oracle.match_census(L, R, D, 2, False)
            oracle.crosscheck(dl, dr, 1, True)
            return 2 * L.shape[0] * L.shape[1] * D / (time.perf_counter() - t0) / 1e6, f"pair 0 alone ({L.shape[1]}x{L.shape[0]}, D={D})"
        launches = 2
    elif wl == "mip1080":
        # disparity mip-maps of a 1920x1080 U16 code map: the ground truth of
        # the seeded census pair (codes d + 1, occluded pixels CannotEvaluate),
        # every level the reference writes by default (levels 0 .. max - 1)
        W, H, D = 1920, 1080, 128
        _, _, G, O = ct.synth_pair(2, SEED + rank, W, H, D - 1)
        codes = np.where(np.asarray(O) != 0, 0xFFFF, np.asarray(G).astype(np.int64) + 1).astype(np.uint16)
        disp = up(codes.view(np.int16))
        pw, nmax = ct.disp_mipmap_format(W, H)
        mipmap = ct.alloc_image(H, pw, torch.float32, dev)
        step = lambda: ct.disp_mipmaps(mipmap, disp, 0, stream=stream)
        _, rects = oracle.mipmap_layout(W, H)
        written = sum(w * h for (_, _, w, h) in rects[:nmax])
        alg_bytes = 2 * W * H + 4 * written

        def check_fn():
            want, _ = oracle.disp_mipmaps(codes, 0, np.zeros((H, pw), np.float32))
            got = mipmap.cpu().numpy()
            return all(np.array_equal(got[y:y + h, x:x + w].view(np.uint32), want[y:y + h, x:x + w].view(np.uint32))
                       for (x, y, w, h) in rects[:nmax])

        def cpu_sample():
            t0 = time.perf_counter()
            for _ in range(5):
                oracle.disp_mipmaps(codes, 0)
            return 5 * W * H / (time.perf_counter() - t0) / 1e6, "5 full pyramids (numpy restatement, 1 thread)"
        units, unit = W * H, "Mpix/s"
        metric = "Mpix/s disparity mip-maps (CreateDispMipMaps, all default levels), 1920x1080 U16"
        big = sum(1 for (_, _, w, h) in rects[2:nmax] if w * h > 16384)
        launches = 1 + big + (1 if nmax - 1 > 1 + big else 0)
        cfg = {"workload": "mip1080_disp_mipmaps", "width": W, "height": H, "levels_written": nmax,
               "packed_width": pw}
    elif wl == "map3d1080":
        # 3D points of a 1920x1080 U16 code map (the seeded pair's ground
        # truth, occluded pixels CannotEvaluate) for a rectified pinhole pair
        # (f = 1400 px, baseline 0.12)
        W, H, D = 1920, 1080, 128
        _, _, G, O = ct.synth_pair(2, SEED + rank, W, H, D - 1)
        codes = np.where(np.asarray(O) != 0, 0xFFFF, np.asarray(G).astype(np.int64) + 1).astype(np.uint16)
        disp = up(codes.view(np.int16))
        cams = [(1400.0, 1400.0, W / 2, H / 2, np.eye(3), (0.0, 0.0, 0.0)),
                (1400.0, 1400.0, W / 2, H / 2, np.eye(3), (0.12, 0.0, 0.0))]
        m3 = ct.MapDisparityTo3D()
        m3.configure(local, W, H, *[ct.pinhole(fx, fy, cx, cy, R, c) for (fx, fy, cx, cy, R, c) in cams])
        pts = ct.alloc_map3d(H, W, dev)
        step = lambda: m3.process(pts, disp, stream=stream)
        alg_bytes = 2 * W * H + 16 * W * H

        def check_fn():
            want, _, hit = oracle.map3d(codes, cams)
            got = pts.cpu().numpy().astype(np.float64)
            dist = np.linalg.norm(want[..., :3], axis=-1, keepdims=True)
            return bool((np.abs(got[..., :3] - want[..., :3]) <= 2e-4 * dist + 1e-6).all()
                        and np.array_equal(got[..., 3], want[..., 3]))

        def cpu_sample():
            t0 = time.perf_counter()
            oracle.map3d(codes, cams)
            return W * H / (time.perf_counter() - t0) / 1e6, "one 1920x1080 map (numpy FP64 restatement, 1 thread)"
        units, unit = W * H, "Mpix/s"
        metric = "Mpix/s disparity to 3D points (MapDisparityTo3D, pinhole pair), 1920x1080 U16"
        launches = 1
        cfg = {"workload": "map3d1080_disparity_to_3d", "width": W, "height": H, "focal_px": 1400.0, "baseline": 0.12}
    elif wl == "compat1080":
        # the reference-compat output of the NCC 11x11 driver (the 4 x uint16
        # TPixelEx pixel: disparity or EDisparityId, uint8-quantised score,
        # specificity channels) with its gradient gate and thresholds active
        W, H, D = 1920, 1080, 128
        L, R, _, _ = ct.synth_pair(2, SEED + rank, W, H, D - 1)
        dL, dR = up(L), up(R)
        thr = dict(grad_thresh=2.0, score_thresh=0.6, min_delta_thresh=3)
        m = ct.BlockMatcherCompat()
        m.configure(local, W, H, ct.CT_COMPAT_NCC, D, 11, **thr)
        out = ct.alloc_u16x4(H, W, dev)
        step = lambda: m.process(out, dL, dR, stream=stream)
        check_fn = lambda: np.array_equal(out.cpu().numpy().view(np.uint16),
                                          oracle.compat_match(L, R, "ncc", D, 11, **thr))

        def cpu_sample():
            t0 = time.perf_counter()
            oracle.compat_match(L, R, "ncc", D, 11, **thr)
            return W * H * D / (time.perf_counter() - t0) / 1e6, f"one full frame {W}x{H} D={D}"
        units = W * H * D
        metric = ("Mpix*disp/s NCC 11x11 reference-compat output (4 x u16: ID, quantised score, specificity), "
                  "1920x1080 D=128")
        launches = 2
        cfg = {"workload": "compat1080_ncc11_u16x4", "width": W, "height": H, "D": D, **thr}
    else:
        W, H, D, kind = {"sad640": (640, 480, 64, 1), "ncc1080": (1920, 1080, 128, 2),
                         "ncc1080g": (1920, 1080, 128, 2), "aw1440": (2560, 1440, 256, 3)}[wl]
        L, R, G, O = ct.synth_pair(kind, SEED + rank, W, H, D - 1)
        dL, dR = up(L), up(R)
        if wl == "sad640":
            m = ct.BlockMatcherSAD1()
            m.configure(local, W, H, D, radius=4)
            out = ct.alloc_image(H, W, torch.uint8, dev)
            step = lambda: m.process(out, dL, dR, stream=stream)
            check_fn = lambda: np.array_equal(out.cpu().numpy(), oracle.to_u8(oracle.match_sad(L, R, D, 4)[0]))
            cpu_fn = lambda: oracle.match_sad(L, R, D, 4)
            metric, launches = "Mpix*disp/s SAD 9x9 WTA, 640x480 D=64", 1
        elif wl == "ncc1080":
            m = ct.BlockMatcherNCC()
            m.configure(local, W, H, D, radius=5)
            out = ct.alloc_image(H, W, torch.uint8, dev)
            score = ct.alloc_image(H, W, torch.float32, dev)
            step = lambda: m.process(out, dL, dR, score=score, stream=stream)
            check_fn = lambda: np.array_equal(out.cpu().numpy(), oracle.to_u8(oracle.match_ncc(L, R, D, 5)[0]))
            cpu_fn = lambda: oracle.match_ncc(L, R, D, 5)
            metric, launches = "Mpix*disp/s NCC 11x11 FP32, 1920x1080 D=128", 2  # statistics of both views, matcher
            # the same step with the window sums on the CUDA cores, timed
            # after the headline timing for comparison
            alt_kernel = (m.set_tensor_cores,
                          lambda: (out.cpu().numpy().copy(), score.cpu().numpy().view(np.uint32).copy()))
        elif wl == "ncc1080g":
            # coarse-to-fine: census + L-R check on the 4x box-averaged pair
            # (480x270, D=32; the pyramid level is prepared on the host, as a
            # camera pipeline would deliver it), then the guided 11x11 NCC at
            # full resolution searching [min - 4, max + 4] of the scaled
            # coarse disparities per 16x16 block
            def down4(img):
                return np.round(img.reshape(H // 4, 4, W // 4, 4).mean(axis=(1, 3))).astype(np.uint8)
            Lc, Rc = down4(L), down4(R)
            dLc, dRc = up(Lc), up(Rc)
            mc = ct.BlockMatcherCensus()
            mc.configure(local, W // 4, H // 4, D // 4)
            coarse = ct.alloc_image(H // 4, W // 4, torch.uint8, dev)
            m = ct.BlockMatcherNCC()
            m.configure(local, W, H, D, radius=5)
            out = ct.alloc_image(H, W, torch.uint8, dev)
            score = ct.alloc_image(H, W, torch.float32, dev)

            def step():
                mc.process_lr(dLc, dRc, disp_checked=coarse, tol=1, stream=stream)
                m.process(out, dL, dR, score=score, disp_init=coarse, stream=stream)

            def coarse_cpu():
                c, _ = oracle.crosscheck(oracle.match_census(Lc, Rc, D // 4, 2, True)[0],
                                         oracle.match_census(Lc, Rc, D // 4, 2, False)[0], 1, True)
                return np.where(c >= 0, c, -1).astype(np.int16)

            def check_fn():
                c = coarse_cpu()
                if not np.array_equal(coarse.cpu().numpy(), oracle.to_u8(c)):
                    return False
                return np.array_equal(out.cpu().numpy(), oracle.to_u8(oracle.match_ncc_guided(L, R, D, c, 5)[0]))

            def cpu_fn():
                oracle.match_ncc_guided(L, R, D, coarse_cpu(), 5)
            # census pair, fused pass, right-view map + check; guide ranges,
            # statistics of both views, guided matcher
            metric, launches = "frames/s coarse-to-fine NCC (census L-R at 1/4, guided 11x11), 1920x1080 D=128", 6
        else:
            m = ct.BlockMatcherAW()
            m.configure(local, W, H, D)
            out = ct.alloc_image(H, W, torch.float32, dev)
            step = lambda: m.process(out, dL, dR, stream=stream)
            check_fn = lambda: np.array_equal(out.cpu().numpy(), oracle.match_aw(L, R, D)[2])
            cpu_fn = lambda: oracle.match_aw(L, R, D)
            metric, launches = "Mpix*disp/s adaptive window (5 x 7x7) + sub-pixel, 2560x1440 D=256", 2
        units = W * H * D
        cfg = {"workload": f"{wl}", "width": W, "height": H, "D": D}
        if wl == "ncc1080":
            cfg.update(window_sums="tensor cores (ncc_tc_kernel: tcgen05 kind::f16 MMAs, fp32 sums in TMEM)")
        if wl == "ncc1080g":
            units, unit = 1e6, "frames/s"  # value = frames per second
            cfg.update(coarse="480x270 D=32 census 9x7 + 5x5 + L-R check (tol 1) of the 4x box-averaged pair",
                       guide_block=16, guide_margin=4)

        def cpu_sample():
            t0 = time.perf_counter()
            cpu_fn()
            return units / (time.perf_counter() - t0) / 1e6, f"one full frame {W}x{H} D={D}"

    for _ in range(max(3, args.warmup)):
        flush_buf.zero_()
        step()
    rank_barrier(world, dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(torch.cuda.current_device()) as clk:
        for k in range(args.steps):
            flush_buf.zero_()
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
    clocks = clk.summary()
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / args.steps, world, dev)
    value = world * units / (ms * 1e-3) / 1e6
    alt_line = None
    if alt_kernel is not None:  # the CUDA-core kernel on the same step, same timing rules
        set_tc, snap = alt_kernel
        maps_tc = snap()
        set_tc(False)
        for _ in range(max(3, args.warmup)):
            flush_buf.zero_()
            step()
        ev2 = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush_buf.zero_()
            ev2[k][0].record(stream)
            step()
            ev2[k][1].record(stream)
        torch.cuda.synchronize(dev)
        ms2 = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev2) / args.steps, world, dev)
        maps_cc = snap()
        set_tc(True)
        alt_line = {"kernel": "ncc_match_kernel (window sums on the CUDA cores)", "ms_per_step": round(ms2, 4),
                    "value": round(world * units / (ms2 * 1e-3) / 1e6, 1),
                    "same_maps_and_scores": bool(all(np.array_equal(a, b) for a, b in zip(maps_tc, maps_cc)))}
    out_line = {
        "metric": metric, "value": round(value, 1), "unit": unit, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u8 pixels / integer costs" + (" / fp32 score" if wl in ("ncc1080", "ncc1080g", "compat1080") else ""),
        "data": "synthetic (seeded generator)", "config": dict(cfg, l2="flushed before every timed step"),
        "gpu_launches": launches * args.steps, "clocks": clocks,
    }
    if alt_line is not None:
        out_line["cuda_core_kernel"] = alt_line
    if wl in ("mip1080", "map3d1080"):
        out_line["dtype"] = "u16 codes / fp32 levels" if wl == "mip1080" else "u16 codes / fp32 points"
        try:
            peak, src = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"], "of measured"
        except (OSError, KeyError, ValueError):
            peak, src = 6650.0, "of fallback"
        ach = alg_bytes / (ms * 1e-3) / 1e9
        out_line["roofline"] = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                                "frac": round(ach / peak, 4), "traffic": None, "peak_source": src,
                                "algorithmic_bytes": alg_bytes,
                                "note": ("whole call (all launches) timed; 2 B read + 4 B per written level pixel"
                                         if wl == "mip1080" else "2 B read + 16 B written per pixel")}
    elif wl in ROOF:
        if rates is None:
            rates = ct.probe_pipe_rates(local)
        kind, ops, key = ROOF[wl]
        out_line["roofline"] = pipe_roofline(kind, ops, key, units / (ms * 1e-3), rates, clocks.get("sm_mhz"))
        out_line["roofline"]["note"] = "whole call timed (all its launches)"
        if wl == "batch64":  # one fused pass per pair decides both directions
            rf = out_line["roofline"]
            rf["frac_costs_once"] = round(rf["frac"] / 2, 4)
            rf["note"] += ("; one fused matching pass per pair evaluates each cost once for both directions: "
                           "frac counts the metric's direction units (2 per cost), frac_costs_once the costs")
    if rank != 0:
        return None
    out_line["parity_rank0"] = bool(check_fn())
    v, sample = cpu_sample()
    out_line["cpu_baseline"] = {"value": round(v, 1), "unit": unit, "cores": oracle.num_threads(),
                                "kind": "port", "sample": sample, "build": f"-O3 -march={march} -fopenmp"}
    return out_line


def run_workload(args):
    import torch
    import ctstereo as ct
    rank, world, local = dist_info()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    init_ranks(world, dev)
    stream = torch.cuda.current_stream(dev)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    line = workload_line(args.workload, args, ct, dev, stream, flush_buf, world, rank, local)
    if line is not None:
        print(json.dumps(line), flush=True)
    close_ranks(world)
    return 0


def run_confnet(args):
    """--workload confnet1080: the learned-confidence pipeline as its own line."""
    import torch
    import ctstereo as ct
    rank, world, local = dist_info()
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    L, R, _, _ = ct.synth_pair(1, SEED, W_, H_, D_ - 1)
    hL, hR = torch.from_numpy(L).pin_memory(), torch.from_numpy(R).pin_memory()
    dL = ct.alloc_image(H_, W_, torch.uint8, dev)
    dR = ct.alloc_image(H_, W_, torch.uint8, dev)
    dL.copy_(hL)
    dR.copy_(hR)
    m = ct.BlockMatcherCensus()
    m.configure(local, W_, H_, D_)
    tuning = m.autotune(dL, dR, stream=stream)
    flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    with ClockSampler(torch.cuda.current_device()) as clk:
        c = confnet_compare(ct, dev, stream, m, dL, dR, hL, hR, flush_buf.zero_, args.steps,
                            args.eval_pairs or 24, local)
    fps = 1e3 / c["learned_ms"]
    print(json.dumps({
        "metric": "frames/s census 1080p D=128 + learned confidence (replaces the R->L pass and the L-R check)",
        "value": round(fps, 1), "unit": "frames/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": c["learned_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8 codes / bf16 weights / fp32 accumulate", "data": "synthetic (seeded generator kind 1)",
        "config": {"workload": "confnet_1920x1080_d128", "width": W_, "height": H_, "D": D_, "seed": SEED,
                   "l2": "flushed before every timed step (256 MiB memset)", "launch_shape": tuning},
        "e2e": {"value": round(1e3 / c["learned_e2e_ms"], 1), "unit": "frames/s", "ms_per_step": c["learned_e2e_ms"],
                "h2d_bytes_per_step": 2 * W_ * H_, "d2h_bytes_per_step": W_ * H_},
        "plain_lr_pipeline": {"value": round(1e3 / c["plain_ms"], 1), "e2e": round(1e3 / c["plain_e2e_ms"], 1),
                              "unit": "frames/s"},
        "confnet": c, "gpu_launches": c["launches_learned"] * args.steps, "clocks": clk.summary()}), flush=True)
    return 0


def main():
    args = parse()
    if args.profile:
        return run_profile(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "confnet1080":
        return run_confnet(args)
    if args.workload != "census1080":
        return run_workload(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
