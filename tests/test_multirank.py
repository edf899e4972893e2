"""The replicas-only multi-GPU path on CPU: two gloo ranks, each with its own
batch, report the whole job as every rank's bead-steps over the slowest
rank's time (bench.reduce_over_ranks), and every rank generates a different
batch."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(REPO, "sop-gpu_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    specs = bench.batch_specs(count=6, lo=40, hi=80, rank=rank)
    beads = sum(s.n for s in specs)
    total, seconds = bench.reduce_over_ranks(dist, beads * 10, 1.0 + rank, "cpu")
    out.put((rank, beads, total, seconds, [int(s.n) for s in specs]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_sum_work_and_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, b0, t0, s0, n0), (r1, b1, t1, s1, n1) = res
    assert t0 == t1 == 10.0 * (b0 + b1)        # every rank's work counted once
    assert s0 == s1 == 2.0                      # the slowest rank's time
    assert n0 != n1                             # each rank owns a different batch


def test_one_process_needs_no_collective():
    sys.path.insert(0, REPO)
    import bench
    assert bench.reduce_over_ranks(None, 123, 4.5, "cpu") == (123.0, 4.5)


def test_reference_arm_under_two_ranks_prints_one_line():
    # the driver launches the reference arm like its own (torchrun, one
    # process per GPU): rank 0 times the CPU restatement and prints the one
    # JSON line, the other rank exits 0 without work
    import json
    import subprocess
    port = 30500 + os.getpid() % 1000
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.join(REPO, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "0", "--ref-seconds", "0.3"]
    r = subprocess.run(cmd, cwd=REPO, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0
