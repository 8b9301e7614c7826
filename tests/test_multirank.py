"""The multi-rank path of bench.py on CPU (gloo, world size 2).

The path shards with no exchange: every rank steps its own replica of the
workload (its own action seeds), and the only collectives are the barrier and
the max-over-ranks reduction of the timed region.  These tests run those
collectives over gloo in two processes, and the reference arm under torchrun
with two ranks (rank 0 alone measures and prints one JSON line)."""
import json
import os
import socket
import subprocess
import sys

import numpy as np
import torch.multiprocessing as mp

from fa_pkg import ROOT, carts

sys.path.insert(0, str(ROOT))
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group(bench.dist_backend(), rank=rank, world_size=world)
    try:
        ms = [12.5, 30.25][rank]
        got = bench.max_over_ranks(ms, world)
        acts = carts.actions(seed=bench.replica_seed(rank, 0), n=64, frames=4)
        dist.barrier()
        out.put((rank, got, acts.tobytes()))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_independent_replicas():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [30.25, 30.25]          # every rank sees the slowest time
    assert res[0][2] != res[1][2]                          # each rank its own replica's actions
    assert bench.max_over_ranks(7.0, 1) == 7.0


def test_reference_arm_under_torchrun_two_ranks():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(ROOT / "bench.py"),
           "--impl", "reference", "--workload", "plain", "--gpus", "2", "--steps", "1", "--warmup", "3",
           "--ref-step-seconds", "0.3"]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=300, cwd=str(ROOT))
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
    assert np.isfinite(d["value"])
