"""bench.py's multi-GPU plumbing on CPU: two gloo ranks on 127.0.0.1 run the
same init / barrier / max-over-ranks / teardown steps that the GPU arm runs
over NCCL (ranks are independent replicas, each on its own seeded pair, so
these are the only collectives), and the reference arm under two ranks
prints exactly one line, from rank 0."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import torch
    import bench
    dev = torch.device("cpu")
    r, w, _ = bench.dist_info()
    bench.init_ranks(w, dev)
    bench.rank_barrier(w, dev)
    got = bench.max_over_ranks(float(10 * (r + 1)), w, dev)
    seed = bench.replica_seed(r)
    bench.close_ranks(w)
    q.put((r, got, seed))


def test_two_gloo_ranks_reduce_timings_to_their_max():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [g for _, g, _ in res] == [20.0, 20.0]
    assert res[0][2] != res[1][2]  # replicas match different pairs


def test_reference_arm_prints_once_under_two_ranks(ct, oracle):
    env = dict(os.environ, PYTHONPATH=str(ROOT))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    assert lines[0]["impl"] == "reference" and lines[0]["n_gpus"] == 2 and lines[0]["value"] > 0
