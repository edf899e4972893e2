#!/usr/bin/env python
"""Benchmark of the SOP Langevin step on B200.

Workload (default, one GPU): the ragged batch of 512 independent replicas,
sizes log-normal in [60, 600] beads (seeded), each a synthetic globular chain
with its own native map and RNG seed, force-clamp at U(100, 300) pN, pairlist
every 10 steps at 20 A, FP32, no HI.  One bench "step" is `--chunk` Langevin
steps of the whole batch (one pass of the resident kernel).  The plain path
(one 200-bead force-ramp job at a time, same kernels) is measured beside it.

Metric: bead-steps/s (sum over jobs of N_job x steps / s).  value: device
time (CUDA events on the launching stream) with state resident in HBM and L2
flushed between timed iterations; e2e: the same through the C ABI with the
coordinates uploaded from pinned host memory and downloaded back every step.

Multi-GPU: replicas only -- every rank advances its own batch, no collective
on the data path; the time is the max over ranks and value is the total.

--impl reference: the reference's step math on the host cores (the CPU
restatement in oracle/, OpenMP over jobs), same workload, bounded sample.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
for sub in ("sop-gpu_b200", "oracle"):
    sys.path.insert(0, os.path.join(REPO, sub))

import numpy as np  # noqa: E402

from sopb_workloads import batch_config, batch_specs, capsid_spec, hi_spec, plain_params, plain_spec  # noqa: E402,F401

METRIC = "bead-steps/s (batched ragged 512-replica stream)"
UNIT = "bead-steps/s"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
def list_stats(jobs, specs):
    """Mean per-bead list lengths (for the algorithmic-bytes model)."""
    tot = nb = nn = npl = npp = 0
    for j, sp in zip(jobs, specs):
        c_pl, _ = j.pairlist(False, cap=1)
        c_pp, _ = j.pairlist(True, cap=1)
        tot += sp.n
        nb += 2 * sp.bonds.shape[0]
        nn += 2 * sp.natives.shape[0]
        npl += int(c_pl.sum())
        npp += int(c_pp.sum())
    return dict(beads=tot, n_bond=nb / tot, n_native=nn / tot, n_pair=npl / tot, n_possible=npp / tot)


def alg_bytes_per_bead_step(st, pairs_freq):
    # compulsory traffic of the reference data model per bead-step:
    # coords r+w, RNG state r+w, ext-force/flag read, bond (int+float),
    # native (int + 2 floats), pair index, and the amortised rebuild
    # (possible-pair index read + pair index write per pairs_freq steps)
    return (32 + 32 + 16 + 8 * st["n_bond"] + 12 * st["n_native"] + 4 * st["n_pair"]
            + (4 * st["n_possible"] + 4 * st["n_pair"]) / pairs_freq)


# Figures of ncu captures of the shipped kernels (profiles/ncu_figures.json):
# DRAM bytes per bead-step and SM-side counters per workload, each recorded
# with a hash of the CUDA sources it was captured from.  A figure whose hash
# no longer matches the sources is stale and not reported.
FIGURES = os.path.join(REPO, "profiles", "ncu_figures.json")


def strip_comments(src):
    """C/C++/CUDA source without its comments and blank lines (string and
    character literals kept), so that a comment edit leaves the hash of the
    code unchanged."""
    out, i, n = [], 0, len(src)
    while i < n:
        c = src[i]
        if c in "\"'":
            j = i + 1
            while j < n and src[j] != c:
                j += 2 if src[j] == "\\" else 1
            out.append(src[i:j + 1])
            i = j + 1
        elif src.startswith("//", i):
            j = src.find("\n", i)
            i = n if j < 0 else j
        elif src.startswith("/*", i):
            j = src.find("*/", i + 2)
            i = n if j < 0 else j + 2
        else:
            out.append(c)
            i += 1
    return "\n".join(l.rstrip() for l in "".join(out).splitlines() if l.strip())


def source_hash():
    """Hash of the CUDA sources' code (comments excluded)."""
    import hashlib
    h = hashlib.sha256()
    d = os.path.join(REPO, "sop-gpu_b200", "csrc")
    for f in sorted(os.listdir(d)):
        if f.endswith((".cu", ".cuh", ".cpp", ".h")):
            h.update(f.encode())
            with open(os.path.join(d, f), encoding="utf-8") as fh:
                h.update(strip_comments(fh.read()).encode())
    return h.hexdigest()[:16]


def ncu_figures(workload):
    try:
        with open(FIGURES) as f:
            e = json.load(f).get(workload)
    except (OSError, ValueError):
        return None
    return e if e and e.get("source_sha") == source_hash() else None


def traffic_per_step(workload, bead_steps):
    e = ncu_figures(workload)
    return None if e is None else e["dram_bytes_per_bead_step"] * bead_steps


def peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        for l in self.lines:
            t = [x.strip() for x in l.split(",")]
            if len(t) < 9:
                continue
            try:
                sm.append(float(t[1]))
                mx = float(t[2])
            except ValueError:
                continue
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), t[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference arm: the CPU restatement on the host cores
# ---------------------------------------------------------------------------
def cpu_rate(specs, target_s=10.0, nthreads=0):
    """bead-steps/s of the oracle on the host cores over a bounded sample."""
    import oracle_py as O
    jobs = [O.OracleJob(sp) for sp in specs]
    beads = sum(sp.n for sp in specs)
    threads = nthreads or os.cpu_count()
    t0 = time.perf_counter()
    O.jobs_advance(jobs, 10, threads)      # includes the step-0 list builds
    probe = time.perf_counter() - t0
    steps = max(10, int(target_s / max(probe / 10, 1e-9)))
    steps = min(steps, 5000)
    t0 = time.perf_counter()
    O.jobs_advance(jobs, steps, threads)
    dt = time.perf_counter() - t0
    for j in jobs:
        j.close()
    return beads * steps / dt, threads, "%d jobs (%d beads) x %d steps" % (len(specs), beads, steps)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle_py
    import sopb
    specs = batch_specs(rank=0, defaults=oracle_py.default_params)
    threads = os.cpu_count()
    vals = []
    sample = ""
    for k in range(args.warmup + args.steps):
        v, threads, sample = cpu_rate(specs, target_s=args.ref_seconds, nthreads=threads)
        if k >= args.warmup:
            vals.append(v)
    value = statistics.median(vals)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded globular chains; no public dataset)",
        "config": batch_config(specs, args.chunk, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if sopb._lib is not None:
        raise RuntimeError("the CPU reference arm loaded the product library")
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def reduce_over_ranks(dist, bead_steps, seconds, device):
    """Whole-job totals of a replicas-only run: every rank's bead-steps summed
    and the slowest rank's time (each rank owns its own batch, so the job
    ends when the last rank does).  `dist` is None on one process."""
    if dist is None:
        return float(bead_steps), float(seconds)
    import torch
    t = torch.tensor([float(bead_steps), float(seconds)], dtype=torch.float64, device=device)
    s = t.clone()
    dist.all_reduce(s[:1], op=dist.ReduceOp.SUM)
    dist.all_reduce(t[1:], op=dist.ReduceOp.MAX)
    return float(s[0].item()), float(t[1].item())


def roofline_batch(achieved, peak, peak_kind, bps, stats, bead_steps):
    """The batch512 roofline entry: the reference data model's bytes against
    the HBM peak (frac), the DRAM traffic an ncu capture of the shipped
    kernel measured, and what limits the kernel per that capture: the SM
    (issue slots and shared-memory wavefronts), not HBM."""
    fig = ncu_figures("batch512")
    r = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
         "traffic": traffic_per_step("batch512", bead_steps),
         "traffic_scope": "DRAM bytes of one bench step (all launch classes), ncu capture of the shipped kernel",
         "peak_kind": peak_kind, "alg_bytes_per_bead_step": bps, "lists": stats}
    if fig:
        r["limiter"] = "sm"
        r["sm_side"] = {k: fig[k] for k in ("issue_active_pct", "shared_wavefronts_per_bead_step",
                                            "shared_bank_conflict_frac", "warps_active_pct") if k in fig}
        r["ncu_capture"] = {"date": fig.get("date"), "source_sha": fig.get("source_sha")}
    else:
        r["limiter"] = None
        r["traffic_note"] = "no ncu capture of the current kernel sources in profiles/ncu_figures.json"
    return r


def run_gpu(args):
    import torch
    import sopb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = local
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = sopb.Context(dev, stream=stream.cuda_stream)

    t0 = time.perf_counter()
    specs = batch_specs(rank=rank)
    log("rank %d: generated %d systems in %.1fs" % (rank, len(specs), time.perf_counter() - t0))
    tuned = None
    if args.policy and not args.autotune:
        lpb, bpg, maxb = args.policy.split(",")
        ctx.set_shape_policy(int(lpb), float(bpg), int(maxb))
        tuned = {"policy": (int(lpb), float(bpg), int(maxb))}
    elif args.autotune:
        import sopb_autotune
        t0 = time.perf_counter()
        tuned = sopb_autotune.autotune(ctx, specs, steps=1000, log=log if rank == 0 else None)
        log("rank %d: autotuned shape policy %s in %.1fs" % (rank, tuned["policy"], time.perf_counter() - t0))
    jobs = [ctx.job(sp) for sp in specs]
    beads = sum(sp.n for sp in specs)
    chunk = args.chunk
    classes = sorted({j.shape()[1] for j in jobs})

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)   # 256 MB > L2

    def one(n=chunk):
        ctx.run(jobs, n)

    # warm-up (also builds the lists at step 0)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            one()
    ctx.sync()
    stats = list_stats(jobs, specs)
    for j in jobs:
        if j.status() != 0:
            raise RuntimeError("job failed during warm-up: status %d" % j.status())

    # timed: device events around each chunk, L2 flushed in between
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        with torch.cuda.stream(stream):
            for k in range(args.steps):
                flush.fill_(float(k))
                starts[k].record(stream)
                one()
                ends[k].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    bead_steps = beads * chunk * args.steps
    all_bead_steps, total_s = reduce_over_ranks(dist, bead_steps, sum(ms) / 1e3, dev)
    total_ms = total_s * 1e3
    value = all_bead_steps / total_s
    launches = len(classes) * args.steps

    # e2e through the C ABI with host buffers
    host = torch.empty((beads, 4), dtype=torch.float32, pin_memory=True)
    host_np = host.numpy()
    ctx.download_coords(jobs, host_np)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(args.steps):
        ctx.upload_coords(jobs, host_np)
        one()
        ctx.download_coords(jobs, host_np)
    torch.cuda.synchronize()
    _, e2e_s = reduce_over_ranks(dist, bead_steps, time.perf_counter() - t0, dev)
    e2e = all_bead_steps / e2e_s
    for j in jobs:
        if j.status() != 0:
            raise RuntimeError("job failed: status %d" % j.status())

    # plain path: one 200-bead job alone, same kernels
    plain = None
    if rank == 0:
        pj = ctx.job(plain_spec())
        with torch.cuda.stream(stream):
            ctx.run([pj], 1000)
        ctx.sync()
        pe0, pe1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        psteps = 20000
        with torch.cuda.stream(stream):
            pe0.record(stream)
            ctx.run([pj], psteps)
            pe1.record(stream)
        torch.cuda.synchronize()
        pms = pe0.elapsed_time(pe1)
        plain = {"workload": "plain_200bead_ramp", "value": 200 * psteps / (pms / 1e3), "unit": UNIT,
                 "steps": psteps, "ms": pms}
        pj.destroy()

    out = None
    if rank == 0:
        peak, peak_kind = peaks()
        bps = alg_bytes_per_bead_step(stats, 10)
        avg_launch_s = (total_ms / 1e3) / args.steps
        achieved = bps * beads * chunk / avg_launch_s / 1e9
        cpu = None
        if world == 1 and not args.no_cpu:
            sample = specs[:: max(1, len(specs) // 64)]
            v, cores, desc = cpu_rate(sample, target_s=args.ref_seconds)
            v1, _, desc1 = cpu_rate(sample[:8], target_s=args.ref_seconds / 2, nthreads=1)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                   "sample": "CPU restatement, OpenMP over jobs: " + desc,
                   "single_thread": {"value": v1, "unit": UNIT, "cores": 1, "sample": desc1}}
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded globular chains; no public dataset)",
            "config": batch_config(specs, chunk, world),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": beads * 16, "d2h_bytes_per_step": beads * 16},
            "gpu_launches": launches,
            "shape_policy": None if tuned is None else {"lanes_per_bead": tuned["policy"][0],
                                                        "beads_per_group": tuned["policy"][1],
                                                        "max_block": tuned["policy"][2]},
            "roofline": roofline_batch(achieved, peak, peak_kind, bps, stats, beads * chunk),
            "plain": plain,
            "batched_over_plain": value / plain["value"] if plain else None,
            "cpu_baseline": cpu,
            "clocks": clk.summary(),
        }
    if rank == 0 and world == 1 and not args.batch_only:
        # compact lines of the other single-GPU workloads: the 198k-bead
        # capsid indentation and exact HI / TEA at 4000 beads
        ctx.sync()
        out["capsid"] = measure_capsid(dev, 3, 1, chunk, None if args.no_cpu else args.ref_seconds)
        out["hi"] = measure_hi(dev, 4000, 2, 1, 10)
    if rank == 0:
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def capsid_cpu_rate(target_s=10.0):
    """The oracle on a bounded sample of the capsid workload: the 18 000-bead
    shell of 180 copies of a 100-bead chain (same lattice, indentation and
    cell-list parameters), one job, one thread."""
    import oracle_py as O
    sp, _ = capsid_spec(copies_per_unit=3, chain_n=100, cell_list=1)
    o = O.OracleJob(sp)
    t0 = time.perf_counter()
    o.advance(10)                                  # includes the step-0 list builds
    probe = time.perf_counter() - t0
    steps = max(10, min(2000, int(target_s / max(probe / 10, 1e-9))))
    t0 = time.perf_counter()
    o.advance(steps)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": sp.n * steps / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "CPU restatement, one job: the 18000-bead shell (180 copies of a 100-bead chain) x %d steps" % steps}


def measure_capsid(dev, steps, warmup, chunk, cpu_seconds=None, copies_per_unit=3, chain_n=1100):
    """The 198k-bead capsid indentation job on the grid path: device-timed
    bead-steps/s (L2 flushed between timed steps), end to end through the C
    ABI with host buffers, the roofline against HBM, clocks."""
    import torch
    import sopb
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    ctx = sopb.Context(dev, stream=stream.cuda_stream)
    t0 = time.perf_counter()
    spec, info = capsid_spec(copies_per_unit=copies_per_unit, chain_n=chain_n,
                             cell_list=1 if copies_per_unit * 60 * chain_n <= 16384 else 0)
    log("capsid: generated %d beads in %.1fs (shell radius %.1f A)" % (spec.n, time.perf_counter() - t0,
                                                                       info["radius_A"]))
    job = ctx.job(spec)
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            ctx.run([job], chunk)
    ctx.sync()
    if job.status() != 0:
        raise RuntimeError("capsid job failed in warm-up: status %d" % job.status())
    stats = list_stats([job], [spec])
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        with torch.cuda.stream(stream):
            for k in range(steps):
                flush.fill_(float(k))
                starts[k].record(stream)
                ctx.run([job], chunk)
                ends[k].record(stream)
        torch.cuda.synchronize()
    total_ms = sum(s_.elapsed_time(e) for s_, e in zip(starts, ends))
    if job.status() != 0:
        raise RuntimeError("capsid job failed: status %d" % job.status())
    value = spec.n * chunk * steps / (total_ms / 1e3)
    host = torch.empty((spec.n, 4), dtype=torch.float32, pin_memory=True).numpy()
    ctx.download_coords([job], host)
    t0 = time.perf_counter()
    for k in range(steps):
        ctx.upload_coords([job], host)
        ctx.run([job], chunk)
        ctx.download_coords([job], host)
    torch.cuda.synchronize()
    e2e = spec.n * chunk * steps / (time.perf_counter() - t0)
    peak, peak_kind = peaks()
    bps = alg_bytes_per_bead_step(stats, 10)
    achieved = bps * spec.n * chunk / ((total_ms / 1e3) / steps) / 1e9
    traffic = traffic_per_step("capsid198k", spec.n * chunk)
    out = {"workload": "capsid198k_indentation", "value": value, "unit": UNIT, "steps": steps, "warmup": warmup,
           "ms_per_step": total_ms / steps,
           "config": {"beads": spec.n, "langevin_steps_per_step": chunk, "pairs_threshold_A": 40.0,
                      "pairlist": "cell list, every 10 steps", "shell_radius_A": info["radius_A"],
                      "copies": info["copies"], "chain_n": info["chain_n"], "inter_natives": info["inter_natives"],
                      "l2": "flushed between timed steps"},
           "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": spec.n * 16, "d2h_bytes_per_step": spec.n * 16},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": traffic,
                        "traffic_scope": "DRAM bytes of one bench step (every launch of the step), scaled from an "
                                         "ncu capture of the 18000-bead shell by bead-steps",
                        "peak_kind": peak_kind, "alg_bytes_per_bead_step": bps, "lists": stats},
           "tip": job.read(sopb.TIPSTATE)[:11].tolist(), "clocks": clk.summary()}
    ctx.close()
    if cpu_seconds:
        out["cpu_baseline"] = capsid_cpu_rate(cpu_seconds)
    return out


def run_capsid(args):
    """Large-assembly workload: one 198k-bead job on the grid path."""
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    r = measure_capsid(dev, args.steps, args.warmup, args.chunk, None if args.no_cpu else args.ref_seconds,
                       args.capsid_copies, args.capsid_chain)
    out = {"metric": "bead-steps/s (198k-bead capsid indentation)", "value": r["value"], "unit": UNIT,
           "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
           "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded shell of chain copies)",
           "config": dict(r["config"], workload="capsid198k_indentation"), "e2e": r["e2e"],
           "roofline": r["roofline"], "tip": r["tip"], "clocks": r["clocks"], "cpu_baseline": r.get("cpu_baseline")}
    print(json.dumps(out), flush=True)
    return 0


def factor_error(job, ctx, spec):
    """||L L^T - D|| / ||D|| (Frobenius) of the factor the job holds, with D
    assembled in FP64 from the coordinates it was factorised at; FP64 on the
    device with torch (measurement only)."""
    import torch
    import sopb
    x0 = job.read(sopb.COORDS)[:, :3].astype(np.float64)
    ctx.run([job], 1)                       # the next step refreshes at x0
    ctx.sync()
    L = torch.from_numpy(job.read(sopb.HIFACTOR)).cuda().double().tril_()
    x = torch.from_numpy(x0).cuda()
    n, a = x.shape[0], float(spec.params.hi_a)
    d = x[None, :, :] - x[:, None, :]                       # d[i, q] = x_q - x_i
    r = d.norm(dim=2)
    r.fill_diagonal_(1.0)
    e = d / r[:, :, None]
    ra = r / a
    far = ra > 2.0
    crr = torch.where(far, 0.75 / ra * (1.0 - 2.0 / ra ** 2), 3.0 * ra / 32.0)
    cii = torch.where(far, 0.75 / ra * (1.0 + 2.0 / 3.0 / ra ** 2), 1.0 - 9.0 * ra / 32.0)
    blk = e[:, :, :, None] * e[:, :, None, :] * crr[:, :, None, None] + \
        torch.eye(3, dtype=torch.float64, device=x.device) * cii[:, :, None, None]
    idx = torch.arange(n, device=x.device)
    blk[idx, idx] = torch.eye(3, dtype=torch.float64, device=x.device)
    D = blk.permute(0, 2, 1, 3).reshape(3 * n, 3 * n)
    del blk, d, e
    err = float(torch.linalg.matrix_norm(L @ L.T - D) / torch.linalg.matrix_norm(D))
    del L, D
    torch.cuda.empty_cache()
    return err


def tf32_peak():
    """TF32 dense tensor peak: half the measured BF16 GEMM burst (TF32 runs at
    half the BF16 rate on B200), else half the fallback."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["bf16_tflops"]) / 2.0, "measured bf16 burst / 2"
    return 1590.0 / 2.0, "fallback bf16 / 2"


def measure_hi(dev, n, steps, warmup, chunk, check_factor=True):
    """One n-bead globule with exact HI (blocked Cholesky of the 3n x 3n
    tensor, refreshed every 10 steps) and with TEA, on the grid path.  The
    exact path's roofline counts the (3n)^3/3 useful flops of a refresh
    against the TF32 tensor peak (the TF32 x3 split issues three times as
    many)."""
    import torch
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(dev)
    import sopb
    ctx = sopb.Context(dev, stream=stream.cuda_stream)
    res = {}
    clocks = None
    e2e = None
    for kind in ("exact", "tea"):
        spec = hi_spec(n, kind == "exact")
        job = ctx.job(spec)
        with torch.cuda.stream(stream):
            for _ in range(warmup):
                ctx.run([job], chunk)
        ctx.sync()
        if job.status() != 0:
            raise RuntimeError("hi %s job failed in warm-up: status %d" % (kind, job.status()))
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
        torch.cuda.synchronize()
        with ClockSampler(dev) as clk:
            with torch.cuda.stream(stream):
                for k in range(steps):
                    starts[k].record(stream)
                    ctx.run([job], chunk)
                    ends[k].record(stream)
            torch.cuda.synchronize()
        total_ms = sum(s_.elapsed_time(e) for s_, e in zip(starts, ends))
        if job.status() != 0:
            raise RuntimeError("hi %s job failed: status %d" % (kind, job.status()))
        res[kind] = {"value": n * chunk * steps / (total_ms / 1e3), "ms_per_langevin_step": total_ms / (chunk * steps)}
        if kind == "exact":
            clocks = clk.summary()
            host = torch.empty((n, 4), dtype=torch.float32, pin_memory=True).numpy()
            ctx.download_coords([job], host)
            t0 = time.perf_counter()
            for k in range(steps):
                ctx.upload_coords([job], host)
                ctx.run([job], chunk)
                ctx.download_coords([job], host)
            torch.cuda.synchronize()
            e2e = n * chunk * steps / (time.perf_counter() - t0)
            if check_factor:
                left = (-job.step()) % 10      # land on a refresh boundary, measure the factor made there
                if left:
                    ctx.run([job], left)
                res["exact"]["factor_rel_error_fp64"] = factor_error(job, ctx, spec)
        job.destroy()
    ctx.close()
    m = 3 * n
    refresh_flop = m ** 3 / 3.0
    peak, peak_kind = tf32_peak()
    # refreshes every 10 steps: the useful factorisation flops per Langevin step
    achieved = refresh_flop / 10.0 / (res["exact"]["ms_per_langevin_step"] / 1e3) / 1e12
    return {"workload": "hi%d_exact_refresh10" % n, "value": res["exact"]["value"], "unit": UNIT,
            "steps": steps, "warmup": warmup,
            "config": {"beads": n, "langevin_steps_per_step": chunk, "hi_a_A": 3.8, "hi_refresh": 10,
                       "tensor": "%d x %d FP32" % (m, m), "chol_panel_tiles": 4},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": n * 16, "d2h_bytes_per_step": n * 16},
            "exact": res["exact"], "tea": res["tea"], "flop_per_refresh": refresh_flop,
            "roofline": {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "note": "useful (3n)^3/3 flops per refresh, one refresh per 10 steps, over the whole step "
                                 "time (apply and D F included); TF32 x3 issues 3x these"},
            "clocks": clocks}


def run_hi(args):
    """HI workload: one 4000-bead job with exact hydrodynamics (blocked
    Cholesky of the 12 000 x 12 000 tensor, refreshed every 10 steps) and the
    same job with TEA, on the grid path."""
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    r = measure_hi(dev, args.hi_beads, args.steps, args.warmup, args.chunk)
    out = {"metric": "bead-steps/s (exact HI, %d beads)" % args.hi_beads, "value": r["value"], "unit": UNIT,
           "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "dtype": "f32",
           "data": "synthetic (seeded globule)", "config": dict(r["config"], workload=r["workload"]),
           "e2e": r["e2e"], "exact": r["exact"], "tea": r["tea"], "flop_per_refresh": r["flop_per_refresh"],
           "roofline": r["roofline"], "clocks": r["clocks"]}
    print(json.dumps(out), flush=True)
    return 0


def run_serve(args):
    """Serving workload: a seeded Poisson stream of pulling, clamp and
    indentation jobs (sizes log-normal in [50, 5000], 30% with HI: exact for
    n <= 1500, TEA above, steps log-uniform in [1e4, 1e5] times
    --serve-step-scale), served by continuous batching.  Reports the served
    throughput and p50/p99 completion latency, and the plain path on the same
    request set: every job alone, one at a time, its rate timed over
    min(steps, 2000) of its steps and its alone time scaled to its steps."""
    import torch
    import sopb
    import sopb_serve
    sys.path.insert(0, os.path.join(REPO, "tests"))
    from serve_mix import poisson_stream
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    ctx = sopb.Context(dev)
    lo_steps, hi_steps = int(1e4 * args.serve_step_scale), int(1e5 * args.serve_step_scale)
    t0 = time.perf_counter()
    reqs = poisson_stream(args.serve_jobs, args.serve_rate, 2024, steps_lo=lo_steps, steps_hi=hi_steps)
    log("serve: generated %d requests in %.1fs" % (len(reqs), time.perf_counter() - t0))
    for r in reqs[:4]:                     # warm-up: one small job of each path
        j = ctx.job(r.spec)
        ctx.run([j], 20)
        j.destroy()
    ctx.sync()
    srv = sopb_serve.Server(ctx, quantum=args.serve_quantum, grid_lanes=args.serve_lanes,
                            slice_us=args.serve_slice_us, long_lanes=args.serve_long_lanes)
    with ClockSampler(dev) as clk:
        t0 = time.perf_counter()
        res = srv.serve(reqs)
        wall = time.perf_counter() - t0
    summ = sopb_serve.summarize(res, wall)
    served = {x.rid: x for x in res}
    # the plain path: each job alone
    alone_s, slow, bead_steps = [], [], 0.0
    for r in ([] if args.serve_no_plain else reqs):
        j = ctx.job(r.spec)
        ctx.run([j], 10)                   # step-0 updaters outside the timed part
        ctx.sync()
        k = min(r.steps, 2000)
        ta = time.perf_counter()
        ctx.run([j], k)
        ctx.sync()
        t_alone = (time.perf_counter() - ta) * r.steps / k
        j.destroy()
        alone_s.append(t_alone)
        bead_steps += r.spec.n * r.steps
        if served[r.rid].status == 0:
            slow.append(served[r.rid].latency / t_alone)
    if args.serve_no_plain:
        alone_s, slow, bead_steps = [float("nan")], [float("nan")], float("nan")
    plain = bead_steps / sum(alone_s)
    by_kind = {}
    for x in res:
        by_kind.setdefault(x.kind, []).append(x.latency)
    out = {"metric": "bead-steps/s (served Poisson stream)", "value": summ["throughput"], "unit": UNIT,
           "n_gpus": 1, "higher_is_better": True, "dtype": "f32", "data": "synthetic (seeded)",
           "config": {"workload": "serve_poisson", "jobs": len(reqs), "rate_per_s": args.serve_rate,
                      "sizes": "lognormal [50, 5000]", "hi_fraction": 0.3,
                      "steps": "log-uniform [%d, %d]" % (lo_steps, hi_steps), "quantum": args.serve_quantum,
                      "grid_lanes": args.serve_lanes, "slice_us": args.serve_slice_us,
                      "long_lanes": args.serve_long_lanes},
           "serve": summ, "peak_inflight": srv.peak_inflight, "peak_hbm_bytes": srv.peak_used,
           "plain": {"value": plain, "unit": UNIT, "method": "each job alone, one at a time; rate over "
                                                              "min(steps, 2000) steps scaled to the job's steps",
                     "total_s": float(sum(alone_s)), "p50_s": float(np.percentile(alone_s, 50)),
                     "p99_s": float(np.percentile(alone_s, 99))},
           "served_over_plain": summ["throughput"] / plain,
           "slowdown_vs_alone": {"p50": float(np.percentile(slow, 50)), "p99": float(np.percentile(slow, 99))},
           "latency_by_kind_p50_s": {k: float(np.percentile(v, 50)) for k, v in sorted(by_kind.items())},
           "slowest": [{"rid": x.rid, "n": x.n, "kind": x.kind, "steps": x.steps, "latency_s": x.latency,
                        "queued_s": x.admitted - x.arrival}
                       for x in sorted(res, key=lambda x: -x.latency)[:5]],
           "clocks": clk.summary()}
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def run_autotune(args):
    """The tuner's tables: the resident shape on the 512-replica batch
    (1000-step trials, best of two) and the HI policy on the 4000-bead exact
    and TEA jobs (20-step trials, best of two)."""
    import torch
    import sopb
    import sopb_autotune
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    ctx = sopb.Context(dev)
    specs = batch_specs()
    beads = sum(sp.n for sp in specs)
    r = sopb_autotune.autotune(ctx, specs, steps=args.autotune_steps, log=log)
    h = sopb_autotune.autotune(ctx, [hi_spec(4000, True), hi_spec(4000, False)], log=log)
    fmt = lambda t: [{"policy": list(p), "seconds": dt, "bead_steps_per_s": v} for p, dt, v in t]
    out = {"workload": "autotune", "resident": {"jobs": len(specs), "beads": beads, "steps": args.autotune_steps,
                                                "best": list(r["policy"]), "table": fmt(r["table"])},
           "hi": {"jobs": "exact + TEA at 4000 beads", "steps": 20, "best": list(h["hi_policy"]),
                  "table": fmt(h["hi_table"])}}
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--chunk", type=int, default=200, help="Langevin steps per bench step")
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--batch-only", action="store_true",
                    help="the batch512 line without the capsid and HI sub-objects")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the shape policy by short timed runs instead of --policy")
    ap.add_argument("--workload", default="batch512", choices=["batch512", "serve", "capsid", "hi", "autotune"])
    ap.add_argument("--autotune-steps", type=int, default=1000)
    ap.add_argument("--hi-beads", type=int, default=4000)
    ap.add_argument("--capsid-copies", type=int, default=3, help="copies per icosahedral unit (60 units)")
    ap.add_argument("--capsid-chain", type=int, default=1100, help="beads per chain copy")
    ap.add_argument("--serve-jobs", type=int, default=200)
    ap.add_argument("--serve-rate", type=float, default=200.0)
    ap.add_argument("--serve-quantum", type=int, default=1000)
    ap.add_argument("--serve-step-scale", type=float, default=1.0)
    ap.add_argument("--serve-lanes", type=int, default=16, help="grid-path streams of the serving loop")
    ap.add_argument("--serve-no-plain", action="store_true", help="skip the one-at-a-time comparison")
    ap.add_argument("--serve-slice-us", type=float, default=1.0e4, help="device time of a grid quantum")
    ap.add_argument("--serve-long-lanes", type=int, default=4, help="lanes for the jobs with the most work left")
    # 4 lanes per bead, one bead per lane group, CTAs of up to 1024 threads:
    # the fastest policy on this workload in full-length runs (the autotuner's
    # 100-step trials cannot separate it from its neighbours reliably)
    ap.add_argument("--policy", default="4,1,1024", help="lanes_per_bead,beads_per_group,max_block")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serve":
        return run_serve(args)
    if args.workload == "capsid":
        return run_capsid(args)
    if args.workload == "hi":
        return run_hi(args)
    if args.workload == "autotune":
        return run_autotune(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
