#!/usr/bin/env python
"""Epsilon self-join throughput on B200: pairs/s of one full self-join step.

Workload (default c2): 2-D, n = 2,000,000 points with i.i.d. exponential(40)
coordinates clipped to [0, 1] (seeded synthetic), eps = 0.0015, B-Unicomp
traversal with workload-sorted tasks on a persistent work queue, FP64, result
batches of at most 5e7 pairs.  One step = grid-index build + estimate + batched
join (per batch: count pass recording hit masks, scan of the per-key counts,
key expansion, pair emission from the masks) + an on-device fold of every batch
into the pair count and set hash, with the points already resident in HBM.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c1..c5] [--n N]

N > 1 (launched by torch.distributed.run): every rank runs its own replica of
the workload on its own seed (weak scaling, no data-path collective); the
per-step time is the maximum over ranks.

--impl reference times the CPU restatement of the reference's path (the
oracle port) on the host cores, on a bounded sample of the same workload,
because the reference's own CUDA build does not produce pairs with this
toolchain (its device cell lookups call a host-only comparison operator).
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

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "self-join-hpbdc2019_b200"))

# dram__bytes_read.sum + dram__bytes_write.sum per output pair of the emission
# kernel (k_emit): 31.4 MB read + 115.2 MB written for a batch of ~28.8 M pairs
# in one ncu capture of the c2 shape at n = 600,000 (profiles/k_emit_c2_n600k.md);
# the traffic grows with the pairs, so a full-size launch is scaled by its pairs
EMIT_TRAFFIC_BYTES_PER_PAIR = (31.4e6 + 115.2e6) / 28.8e6

# CUDA-core lanes per SM (B200): FP64 FMA and FP32 FMA per clock
FP64_LANES, FP32_LANES, NUM_SM = 64, 128, 148

L2_BYTES = 126 * 1024 * 1024


def _peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        busy = [s for s in sm if mx and s > 0.3 * max(mx)] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def combine_ranks(ms, pairs, pair_hash, device):
    """(max step ms, summed pairs, summed set hash mod 2^64) over all ranks.

    The set hash is a wrapping 64-bit sum over pairs, so the hashes of disjoint
    shards add up (mod 2^64) to the hash of their union; it travels as int64,
    whose two's-complement sum wraps the same way."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    h = pair_hash - (1 << 64) if pair_hash >= (1 << 63) else pair_hash
    v = torch.tensor([pairs, h], dtype=torch.int64, device=device)
    dist.all_reduce(v)
    return float(t.item()), int(v[0].item()), int(v[1].item()) % (1 << 64)


def host_threads() -> int:
    """Host CPUs this process may run on.  Passed to the oracle explicitly:
    torchrun sets OMP_NUM_THREADS=1 in every rank, which would otherwise leave
    the CPU legs on one thread."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_oracle_rate(pts, eps, k, target_s=12.0, threads=0):
    """Oracle grid join on a bounded sample of query points: (pairs/s, cores, sample text)."""
    import oracle
    threads = threads or host_threads()
    ix = oracle.OracleIndex(pts, eps, k)
    n = len(pts)
    stride = max(1, n // 2000)
    t0 = time.perf_counter()
    P, _, E = ix.stats(qstride=stride, threads=threads)
    dt = time.perf_counter() - t0
    if dt < target_s / 4:
        stride = max(1, int(stride * dt / target_s))
        t0 = time.perf_counter()
        P, _, E = ix.stats(qstride=stride, threads=threads)
        dt = time.perf_counter() - t0
    cores = threads
    nq = (n + stride - 1) // stride
    sample = f"every {stride}th query point ({nq} of {n}), full stencil, {E} candidate evaluations, {dt:.1f} s"
    return P / dt, cores, sample, dt


def run_reference(args):
    import sjoin
    ws, rank, _ = _dist()
    if rank != 0:
        return
    pts, eps, k, spec = sjoin.datasets.make(args.workload, n=args.n)
    times, rates = [], []
    for i in range(args.warmup + args.steps):
        rate, cores, sample, dt = cpu_oracle_rate(pts, eps, k, target_s=args.ref_seconds)
        if i >= args.warmup:
            rates.append(rate)
            times.append(dt)
    v = statistics.mean(rates)
    line = {
        "impl": "reference", "metric": "self-join pairs/s", "value": v, "unit": "pairs/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "config": _config(args, spec),
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _config(args, spec):
    mode_name = {3: "full stencil", 4: "Unicomp", 5: "B-Unicomp", 6: "linear-ID Unicomp", 7: "full stencil",
                 8: "full stencil", 9: "work queue", 10: "linear-ID Unicomp"}[spec["mode"]]
    return {
        "workload": (f"{args.workload}: {spec['D']}-D {spec['kind']}, n={spec['n']}, eps={spec['eps']}, "
                     f"{mode_name} + workload-sorted work queue, "
                     f"{'FP64' if spec['precision'] == 0 else 'FP32 filter + FP64 refine'}, "
                     f"batches <= {spec['capacity'] or 'auto'} pairs"),
        "n": spec["n"], "dims": spec["D"], "indexed_dims": spec["k"], "eps": spec["eps"],
        "search_mode": spec["mode"], "batch_capacity_pairs": spec["capacity"],
        "l2": "flushed between steps (256 MiB write); outputs far exceed L2",
        "parallelism": (f"task shards x{_dist()[0]}" if getattr(args, "shard", False) else f"replicas x{_dist()[0]}"),
    }


def rank_host_threads() -> int:
    """Host threads for one rank's engine (task preparation, host key
    expansion): every usable CPU in a single process, an equal share of them
    per rank under torchrun (which sets OMP_NUM_THREADS=1 in its ranks)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return host_threads()
    local_ws = int(os.environ.get("LOCAL_WORLD_SIZE", str(ws)))
    return max(1, host_threads() // max(1, local_ws))


def run_ours(args):
    import torch

    import sjoin
    ws, rank, local = _dist()
    # the engine's OpenMP regions start on this thread and share torch's OpenMP runtime
    torch.set_num_threads(rank_host_threads())
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    # replicas (default): every rank joins its own seeded set (weak scaling);
    # --shard: all ranks share one set and each runs one shard of its
    # cost-ordered task list (strong scaling, no data-path exchange)
    seed = sjoin.datasets.SEEDS[args.workload] + (0 if args.shard else 1000 * rank)
    pts, eps, k, spec = sjoin.datasets.make(args.workload, n=args.n, seed=seed)
    if args.capacity is not None:
        spec["capacity"] = args.capacity
    prec = spec["precision"] if args.precision is None else args.precision
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
    sj = sjoin.SelfJoin(spec["D"], eps, indexed_dims=k, mode=spec["mode"], precision=prec,
                        scheduler=sjoin.SCHED_LEARNED if args.learned else sjoin.SCHED_SAMPLING,
                        capacity=spec["capacity"], device=local,
                        shard_index=rank if args.shard else 0, shard_count=ws if args.shard else 1)
    if args.learned:
        sj.load_estimator(args.learned)
    host = torch.from_numpy(pts).pin_memory()
    sj.set_points(host.numpy())
    stream = torch.cuda.ExternalStream(sj.stream())

    def step():
        sj.build_index()
        return sj.join(sjoin.DELIVER_NONE)

    for _ in range(args.warmup):
        step()
    sampler = ClockSampler(torch.cuda.current_device())
    sampler.start()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = sjoin.kernel_launch_count()
    step_ms, stats = [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = step()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        stats.append(st.as_dict())
    torch.cuda.synchronize()
    launches = sjoin.kernel_launch_count() - launches0
    if ws > 1:
        torch.distributed.barrier()
    clocks = sampler.stop()
    ms = statistics.mean(step_ms)
    pairs = stats[-1]["total_pairs"]
    job_ms, job_pairs, job_hash = ms, pairs, stats[-1]["pair_hash"]
    if ws > 1:
        job_ms, job_pairs, job_hash = combine_ranks(ms, pairs, job_hash, "cuda")

    # end to end through the C ABI with host buffers: pinned H2D of the points,
    # index, join, and every batch copied device-to-host into pinned buffers
    e2e = None
    if not args.no_e2e:
        def e2e_step():
            sj.set_points(host.numpy())
            sj.build_index()
            return sj.join(sjoin.DELIVER_HOST, lambda i, kk, vv: None)

        e2e_step()
        torch.cuda.synchronize()
        ems = []
        for _ in range(max(1, min(args.steps, args.e2e_steps))):
            flush.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st_e = e2e_step()
            e1.record(stream)
            e1.synchronize()
            ems.append(e0.elapsed_time(e1))
        e_ms = statistics.mean(ems)
        if ws > 1:
            t = torch.tensor([e_ms], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e_ms = float(t.item())
        # host delivery copies each batch's values and its per-key run offsets
        # (the host expands the keys from them)
        e2e = {"value": job_pairs / (e_ms / 1e3), "unit": "pairs/s", "ms_per_step": e_ms,
               "h2d_bytes_per_step": int(pts.nbytes),
               "d2h_bytes_per_step": int(st_e.total_pairs) * 4 + int(st_e.num_batches) * 4 * spec["n"]}

    if rank != 0:
        if ws > 1:
            torch.distributed.destroy_process_group()
        return
    peak, peak_kind = _peaks()
    s = stats[-1]
    nb = max(1, s["num_batches"])
    # per-stage device time (CUDA events around every launch) and algorithmic bytes
    stages = {
        "emit": (s["ms_fill_kernel"], 4 * pairs, "k_emit: pair values from the hit masks into their row slots"),
        "expand": (s["ms_expand"], 4 * pairs + 4 * spec["n"] * nb, "k_expand_keys: key array from row offsets"),
        "hash": (s["ms_deliver"], 8 * pairs, "k_hash_pairs_dev: consumer fold of every batch"),
        "count": (s["ms_count"], None, "k_join count pass (distance loop)"),
    }
    top = max(("emit", "expand", "hash"), key=lambda k2: stages[k2][0])
    t_ms, algo_bytes, kdesc = stages[top]
    achieved = algo_bytes / (t_ms / 1e3) / 1e9 if t_ms > 0 else None
    traffic = (EMIT_TRAFFIC_BYTES_PER_PAIR * pairs / nb) if (EMIT_TRAFFIC_BYTES_PER_PAIR and top == "emit") else None
    # distance loop against the CUDA-core pipe it runs on: 3*D flops (subtract,
    # multiply, add per dimension) per evaluated candidate, nominal lanes x the
    # SM clock sampled during the timed steps
    mhz = clocks.get("sm_mhz") or 1965.0
    lanes = FP64_LANES if prec == 0 else FP32_LANES
    pipe_tflops = NUM_SM * lanes * 2 * mhz * 1e6 / 1e12
    dist_tflops = (3 * spec["D"] * s["distance_calcs"]) / (s["ms_count"] / 1e3) / 1e12 if s["ms_count"] > 0 else None
    cpu = None
    if not args.no_cpu and ws == 1:   # the CPU baseline is rank 0's at N = 1 only
        rate, cores, sample, _ = cpu_oracle_rate(pts, eps, k, target_s=args.cpu_seconds)
        cpu = {"value": rate, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": sample}
    line = {
        "metric": "self-join pairs/s", "value": job_pairs / (job_ms / 1e3), "unit": "pairs/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": job_ms, "higher_is_better": True,
        "scaling": "strong" if args.shard else "weak", "vs_baseline": None,
        "dtype": "f64" if prec == 0 else "f32+f64",
        "data": "synthetic (seeded generator, same shapes and distributions)", "config": _config(args, spec),
        "time_s": job_ms / 1e3, "pairs_per_step": job_pairs, "pair_hash": job_hash,
        "roofline": {"bound": "hbm", "kernel": kdesc, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": algo_bytes / nb, "launches": nb, "traffic": traffic,
                     "stage_ms": {k2: round(v[0], 3) for k2, v in stages.items()}},
        "roofline_distance_loop": {"bound": "fp64 pipe" if prec == 0 else "fp32 pipe",
                                   "kernel": stages["count"][2], "achieved": dist_tflops, "peak": pipe_tflops,
                                   "unit": "TFLOP/s", "frac": (dist_tflops / pipe_tflops) if dist_tflops else None,
                                   "peak_kind": "nominal lanes x sampled SM clock",
                                   "flops_per_candidate": 3 * spec["D"]},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
        "host_threads_per_rank": rank_host_threads(),
        "phases_ms": {k2: round(s[k2], 3) for k2 in ("ms_index", "ms_tasks", "ms_estimate", "ms_count", "ms_scan",
                                                     "ms_fill", "ms_expand", "ms_deliver", "ms_total")},
        "batches": s["num_batches"], "overflow_retries": s["overflow_retries"],
        "distance_calcs": s["distance_calcs"], "full_stencil_calcs": s["full_stencil_calcs"],
        "refined_pairs": s["refined_pairs"], "step_ms": step_ms,
        "scheduler": "learned" if args.learned else "sampling", "estimated_pairs": s["estimated_pairs"],
        "estimator_batch_rel_err": s["estimator_mean_abs_rel_err"], "estimator_task_rel_err": s["estimator_task_rel_err"],
    }
    print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: split one join over the ranks (strong scaling) instead of N replicas")
    ap.add_argument("--capacity", type=int, default=None, help="batch capacity in pairs (default: the workload's)")
    ap.add_argument("--precision", type=int, default=None)
    ap.add_argument("--learned", default=None,
                    help="estimator weights file: learned scheduler instead of the sampling estimate")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
