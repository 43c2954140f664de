#!/usr/bin/env python
"""Epsilon self-join on B200: pairs/s of one full self-join step, mixed
precision + learned scheduling against plain FP64 on the same points.

Workload (default c4): 6-D, n = 10,000,000 points with i.i.d. exponential(40)
coordinates clipped to [0, 1] (seeded synthetic), eps = 0.03, linear-ID
Unicomp traversal with workload-sorted tasks on a persistent work queue,
result batches of at most 2e9 pairs.

  * `value`: the FP32 filter + FP64 borderline refine with the learned
    estimator ordering the queue and sizing the batches.
  * `fp64`: the plain FP64 method (FP64 predicate, sampling estimator) on the
    same points in the same invocation; `speedup_vs_fp64` is the ratio of the
    step times and `identical_pair_set` checks the two pair counts and set
    hashes (the run exits non-zero if they differ).

One step = grid-index build + estimate + batched join (per batch: count pass
recording hit masks, scan of the per-key counts, key expansion, pair emission
from the masks) + an on-device fold of every batch into the pair count and set
hash, with the points already resident in HBM.  `e2e` is the same join through
the C ABI with host buffers: the points copied from pinned host memory and
every batch's pairs delivered to host memory.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c1..c5] [--n N] [--precision 0|1]
                  [--scheduler learned|sampling] [--fp64-steps S]

N > 1 (launched by torch.distributed.run): every rank runs its own replica of
the workload on its own seed (weak scaling, no data-path collective); the
per-step time is the maximum over ranks.

--impl reference times the CPU restatement of the reference's path (the
oracle port) on the host cores, on a bounded sample of the same workload (the
reference has no CPU implementation of the join), and beside it the
reference's own CUDA pipeline, built from its sources for sm_100a, on the two
small workloads it can complete (2-D uniform, n = 1e5; the c2 shape at
n = 5e5); the engine's arm times itself on the same two workloads.
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

ESTIMATOR_WEIGHTS = os.path.join(REPO, "self-join-hpbdc2019_b200", "sjoin", "estimator_c4.bin")

# dram__bytes_read.sum + dram__bytes_write.sum per output pair of the emission
# kernel (k_emit) in one ncu capture (profiles/k_emit_c4_n2M.md: the c4
# generator at n = 2e6, one batch); the traffic grows with the pairs, so a
# full-size launch is scaled by its pairs
EMIT_TRAFFIC_BYTES_PER_PAIR = None

# CUDA-core lanes per SM (B200): FP64 FMA and FP32 FMA per clock
FP64_LANES, FP32_LANES, NUM_SM = 64, 128, 148

L2_BYTES = 126 * 1024 * 1024

# the two workloads the reference's own CUDA pipeline completes (its per-batch
# host arrays hold every pair): (name, workload, n, mode, reference binary tag)
SMALL_CASES = [("c1", "c1", 100_000, 3), ("c2_n500k", "c2", 500_000, 5)]


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
    """The oracle's grid self-join on the host cores, on a bounded sample of query points:
    (pairs/s, cores, sample text).  Linear-ID Unicomp: each sampled point evaluates the
    candidates it owns (its own cell's points with a larger id, the stencil cells with a
    larger linear id) and counts both directions of every hit, so every pair is evaluated once
    and a sample of points carries its share of the pairs."""
    import oracle
    threads = threads or host_threads()
    ix = oracle.OracleIndex(pts, eps, k)
    n = len(pts)
    stride = max(1, n // 2000)
    t0 = time.perf_counter()
    P, _, E = ix.stats(qstride=stride, threads=threads, unicomp=True)
    dt = time.perf_counter() - t0
    if dt < target_s / 4:
        stride = max(1, int(stride * dt / target_s))
        t0 = time.perf_counter()
        P, _, E = ix.stats(qstride=stride, threads=threads, unicomp=True)
        dt = time.perf_counter() - t0
    cores = threads
    nq = (n + stride - 1) // stride
    sample = (f"every {stride}th query point ({nq} of {n}), linear-ID Unicomp grid join ({E} candidate "
              f"evaluations, each pair once, both directions counted), {dt:.1f} s")
    return P / dt, cores, sample, dt


def reference_cuda_runs(timeout_s=300):
    """The reference's own batched CUDA pipeline (distanceTableNDGridBatches,
    built from its sources for sm_100a with its cell comparison made
    device-callable) on the SMALL_CASES, timed by its own harness the way its
    main() times it (import and host grid build excluded)."""
    import sjoin
    from oracle import build_ref
    out = {}
    with tempfile.TemporaryDirectory() as td:
        for name, wl, n, mode in SMALL_CASES:
            pts, eps, k, spec = sjoin.datasets.make(wl, n=n)
            path = os.path.join(td, name + ".csv")
            sjoin.datasets.write_csv(path, pts)
            rec = {"workload": f"{spec['D']}-D {spec['kind']}, n={n}, eps={eps}", "mode": mode}
            for sort in (0, 1):
                exe = build_ref.binary("pipeline", spec["D"], k, sort)
                key = f"sort_by_workload_{sort}"
                if not os.path.exists(exe):
                    rec[key] = {"unavailable": "reference binary not built"}
                    continue
                try:
                    r = subprocess.run([exe, path, repr(eps), str(mode)], capture_output=True, text=True,
                                       timeout=timeout_s)
                    js = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
                    rec[key] = ({"time_s": js[-1]["time_s"], "total_pairs": js[-1]["total_neighbors"]}
                                if r.returncode == 0 and js else {"unavailable": f"exit {r.returncode}"})
                except subprocess.TimeoutExpired:
                    rec[key] = {"unavailable": f"did not finish in {timeout_s} s"}
            out[name] = rec
    return out


def engine_small_runs(device):
    """The engine on the SMALL_CASES end to end through the C ABI with host
    buffers (points from pinned host memory, every pair delivered to host
    memory), best of 3 after one warm-up call."""
    import torch

    import sjoin
    out = {}
    for name, wl, n, mode in SMALL_CASES:
        pts, eps, k, spec = sjoin.datasets.make(wl, n=n)
        host = torch.from_numpy(pts).pin_memory()
        with sjoin.SelfJoin(spec["D"], eps, indexed_dims=k, mode=mode, precision=0, device=device) as sj:
            stream = torch.cuda.ExternalStream(sj.stream())
            best, st = None, None
            for i in range(4):
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                sj.set_points(host.numpy())
                sj.build_index()
                st = sj.join(sjoin.DELIVER_HOST, lambda i, kk, vv: None)
                e1.record(stream)
                e1.synchronize()
                if i > 0:
                    t = e0.elapsed_time(e1) / 1e3
                    best = t if best is None else min(best, t)
        out[name] = {"workload": f"{spec['D']}-D {spec['kind']}, n={n}, eps={eps}", "mode": mode,
                     "e2e_time_s": best, "total_pairs": int(st.total_pairs)}
    return out


def _config(args, spec, prec, learned):
    mode_name = {3: "full stencil", 4: "Unicomp", 5: "B-Unicomp", 6: "linear-ID Unicomp", 7: "full stencil",
                 8: "full stencil", 9: "work queue", 10: "linear-ID Unicomp"}[spec["mode"]]
    return {
        "workload": (f"{args.workload}: {spec['D']}-D {spec['kind']}, n={spec['n']}, eps={spec['eps']}, "
                     f"{mode_name} + workload-sorted work queue, "
                     f"{'FP64' if prec == 0 else 'FP32 filter + FP64 refine'}, "
                     f"{'learned' if learned else 'sampling'} scheduler, "
                     f"batches <= {spec['capacity'] or 'auto'} pairs"),
        "n": spec["n"], "dims": spec["D"], "indexed_dims": spec["k"], "eps": spec["eps"],
        "search_mode": spec["mode"], "batch_capacity_pairs": spec["capacity"],
        "precision": "fp64" if prec == 0 else "fp32 filter + fp64 refine",
        "scheduler": "learned" if learned else "sampling",
        "l2": "flushed between steps (256 MiB write); outputs far exceed L2",
        "parallelism": (f"task shards x{_dist()[0]}" if getattr(args, "shard", False) else f"replicas x{_dist()[0]}"),
        **({"task_sample": f"task shard 0 of {args.task_sample} (every {args.task_sample}th task of the cost "
                           f"order; a reduced case for profiler captures)"}
           if getattr(args, "task_sample", 1) > 1 else {}),
    }


def _spec_and_prec(args):
    import sjoin
    spec = dict(sjoin.datasets.WORKLOADS[args.workload])
    if getattr(args, "mode", None) is not None:
        spec["mode"] = args.mode
    prec = spec["precision"] if args.precision is None else args.precision
    learned = args.scheduler == "learned" if args.scheduler else (args.workload == "c4" and prec == 1)
    return spec, prec, learned


def run_reference(args):
    import sjoin
    ws, rank, _ = _dist()
    if rank != 0:
        return
    pts, eps, k, spec = sjoin.datasets.make(args.workload, n=args.n)
    if args.mode is not None:
        spec["mode"] = args.mode
    _, prec, learned = _spec_and_prec(args)
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
        "data": "synthetic (seeded)", "config": _config(args, spec, prec, learned),
        "cpu_baseline": {"value": v, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_ref_cuda:
        import torch
        line["reference_cuda"] = (reference_cuda_runs() if torch.cuda.is_available()
                                  else {"unavailable": "no CUDA device"})
    print(json.dumps(line), flush=True)


def rank_host_threads() -> int:
    """Host threads for one rank's engine (task preparation, host key
    expansion): every usable CPU in a single process, an equal share of them
    per rank under torchrun (which sets OMP_NUM_THREADS=1 in its ranks)."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return host_threads()
    local_ws = int(os.environ.get("LOCAL_WORLD_SIZE", str(ws)))
    return max(1, host_threads() // max(1, local_ws))


def timed_steps(sj, step, steps, warmup, flush, stream):
    """`warmup` untimed steps, then `steps` steps each bracketed by CUDA events
    on the engine's stream (L2 flushed and the device idle before each)."""
    import torch
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    step_ms, stats = [], []
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st = step()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        stats.append(st.as_dict())
    return step_ms, stats


def run_ours(args):
    import torch

    import sjoin
    ws, rank, local = _dist()
    # the engine's OpenMP regions start on this thread and share torch's OpenMP runtime
    torch.set_num_threads(rank_host_threads())
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    # replicas (default): every rank joins its own seeded set (weak scaling);
    # --shard: all ranks share one set and each runs one shard of its
    # cost-ordered task list (strong scaling, no data-path exchange)
    seed = sjoin.datasets.SEEDS[args.workload] + (0 if args.shard else 1000 * rank)
    pts, eps, k, spec = sjoin.datasets.make(args.workload, n=args.n, seed=seed)
    if args.capacity is not None:
        spec["capacity"] = args.capacity
    if args.mode is not None:
        spec["mode"] = args.mode
    _, prec, learned = _spec_and_prec(args)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
    host = torch.from_numpy(pts).pin_memory()

    def make_ctx(precision, use_learned):
        sj = sjoin.SelfJoin(spec["D"], eps, indexed_dims=k, mode=spec["mode"], precision=precision,
                            scheduler=sjoin.SCHED_LEARNED if use_learned else sjoin.SCHED_SAMPLING,
                            capacity=spec["capacity"], device=local,
                            shard_index=rank if args.shard else 0,
                            shard_count=ws if args.shard else max(1, args.task_sample))
        if use_learned:
            sj.load_estimator(args.weights)
        sj.set_points(host.numpy())
        return sj

    sj = make_ctx(prec, learned)
    stream = torch.cuda.ExternalStream(sj.stream())

    delivery = {"none": sjoin.DELIVER_NONE, "device": sjoin.DELIVER_DEVICE}[args.delivery]

    def step():
        sj.build_index()
        if delivery == sjoin.DELIVER_DEVICE:   # every batch handed to a consumer that reads nothing
            return sj.join(delivery, lambda i, kp, vp, cnt: None)
        return sj.join(delivery)

    sampler = ClockSampler(torch.cuda.current_device())
    # warm-up, then the timed steps (clocks sampled throughout the timed region)
    for _ in range(args.warmup):
        step()
    sampler.start()
    if ws > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    launches0 = sjoin.kernel_launch_count()
    step_ms, stats = timed_steps(sj, step, args.steps, 0, flush, stream)
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

    # stage probe: one more step with every stage on one stream (the engine's
    # SJ_SERIAL knob), so each kernel's CUDA-event time is its own, not shared
    # with the other stream's kernels; the rooflines use these times
    probe = None
    if not args.no_stage_probe:
        prior = os.environ.get("SJ_SERIAL")
        os.environ["SJ_SERIAL"] = "1"
        try:
            probe = step().as_dict()
        finally:
            if prior is None:
                del os.environ["SJ_SERIAL"]
            else:
                os.environ["SJ_SERIAL"] = prior

    # end to end through the C ABI with host buffers: pinned H2D of the points,
    # index, join, and every batch's pairs delivered into pinned host memory
    e2e = None
    if args.e2e_steps > 0:
        def e2e_step():
            sj.set_points(host.numpy())
            sj.build_index()
            return sj.join(sjoin.DELIVER_HOST, lambda i, kk, vv: None)

        ems, est = timed_steps(sj, e2e_step, args.e2e_steps, 0, flush, stream)
        e_ms = statistics.mean(ems)
        if ws > 1:
            t = torch.tensor([e_ms], device="cuda", dtype=torch.float64)
            torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
            e_ms = float(t.item())
        st_e = est[-1]
        if st_e["total_pairs"] != pairs or st_e["pair_hash"] != stats[-1]["pair_hash"]:
            raise RuntimeError("host delivery produced a different pair set than the device fold")
        # host delivery copies each batch's values and its per-key run offsets
        # (the host expands the keys from them)
        e2e = {"value": job_pairs / (e_ms / 1e3), "unit": "pairs/s", "ms_per_step": e_ms, "steps": args.e2e_steps,
               "h2d_bytes_per_step": int(pts.nbytes),
               "d2h_bytes_per_step": int(st_e["total_pairs"]) * 4 + int(st_e["num_batches"]) * 4 * spec["n"],
               "delivery": "every pair to pinned host memory (values copied, keys expanded on the host)"}
    sj.close()

    # the plain FP64 method on the same points: FP64 predicate, sampling estimator
    fp64 = None
    if args.fp64_steps > 0 and not (prec == 0 and not learned):
        sj64 = make_ctx(0, False)
        stream64 = torch.cuda.ExternalStream(sj64.stream())

        def step64():
            sj64.build_index()
            return sj64.join(sjoin.DELIVER_NONE)

        f_ms, f_stats = timed_steps(sj64, step64, args.fp64_steps, 1, flush, stream64)
        sj64.close()
        fm = statistics.mean(f_ms)
        fp, fh = f_stats[-1]["total_pairs"], f_stats[-1]["pair_hash"]
        if ws > 1:
            fm, fp, fh = combine_ranks(fm, fp, fh, "cuda")
        fs = f_stats[-1]
        fp64 = {"ms_per_step": fm, "step_ms": f_ms, "steps": args.fp64_steps, "warmup": 1,
                "pairs_per_step": fp, "pair_hash": fh, "scheduler": "sampling", "precision": "fp64",
                "batches": fs["num_batches"], "exact_plan_batches": fs["exact_plan_batches"], "overflow_retries": fs["overflow_retries"],
                "phases_ms": {k2: round(fs[k2], 3) for k2 in ("ms_index", "ms_tasks", "ms_estimate", "ms_count",
                                                              "ms_scan", "ms_fill", "ms_expand", "ms_deliver",
                                                              "ms_total")},
                "distance_loop": _pipe_roofline(fs, 0, spec["D"], clocks)}

    if rank != 0:
        if ws > 1:
            torch.distributed.destroy_process_group()
        return
    peak, peak_kind = _peaks()
    s = stats[-1]
    ps = probe or s   # per-kernel times: the stage probe's when it ran
    nb = max(1, ps["num_batches"])
    emit_ms = ps["ms_fill_kernel"]
    achieved = (4 * pairs) / (emit_ms / 1e3) / 1e9 if emit_ms > 0 else None
    traffic = EMIT_TRAFFIC_BYTES_PER_PAIR * pairs / nb if EMIT_TRAFFIC_BYTES_PER_PAIR else None
    fold_ms = ps["ms_deliver"]
    fold_gbs = (8 * pairs) / (fold_ms / 1e3) / 1e9 if fold_ms > 0 else None
    cpu = None
    if not args.no_cpu and ws == 1:   # the CPU baseline is rank 0's at N = 1 only
        rate, cores, sample, _ = cpu_oracle_rate(pts, eps, k, target_s=args.cpu_seconds)
        cpu = {"value": rate, "unit": "pairs/s", "cores": cores, "kind": "port", "sample": sample}
    small = None
    if not args.no_ref_cuda and ws == 1:
        small = engine_small_runs(local)
    line = {
        "metric": "self-join pairs/s", "value": job_pairs / (job_ms / 1e3), "unit": "pairs/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": job_ms, "higher_is_better": True,
        "scaling": "strong" if args.shard else "weak", "vs_baseline": None,
        "dtype": "f64" if prec == 0 else "f32+f64",
        "data": "synthetic (seeded generator, same shapes and distributions)",
        "config": _config(args, spec, prec, learned),
        "time_s": job_ms / 1e3, "pairs_per_step": job_pairs, "pair_hash": job_hash,
        "roofline": {"bound": "hbm", "kernel": "k_emit: pair values from the hit masks into their key runs",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": 4 * pairs / nb, "launches": nb, "traffic": traffic,
                     "note": ("4 B of values written per pair; launch times from CUDA events around each launch "
                              "in the stage probe (every stage on one stream)" if probe else
                              "4 B of values written per pair; launch times from CUDA events on the emission's "
                              "stream, shared with the next batch's count pass")},
        "roofline_fold": {"bound": "hbm", "kernel": "k_fold: values read back, keys written, set hash",
                          "achieved": fold_gbs, "peak": peak, "unit": "GB/s",
                          "frac": (fold_gbs / peak) if fold_gbs else None, "peak_kind": peak_kind,
                          "algorithmic_bytes_per_launch": 8 * pairs / nb},
        "roofline_distance_loop": _pipe_roofline(ps, prec, spec["D"], clocks),
        "stage_probe_ms": ({k2: round(probe[k2], 3) for k2 in ("ms_count", "ms_scan", "ms_fill", "ms_deliver",
                                                               "ms_total")} if probe else None),
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clocks,
        "host_threads_per_rank": rank_host_threads(),
        "phases_ms": {k2: round(s[k2], 3) for k2 in ("ms_index", "ms_tasks", "ms_estimate", "ms_count", "ms_scan",
                                                     "ms_fill", "ms_expand", "ms_deliver", "ms_total")},
        "batches": s["num_batches"], "exact_plan_batches": s["exact_plan_batches"], "overflow_retries": s["overflow_retries"], "tasks": s["num_tasks"],
        "distance_calcs": s["distance_calcs"], "full_stencil_calcs": s["full_stencil_calcs"],
        "refined_pairs": s["refined_pairs"], "step_ms": step_ms,
        "scheduler": "learned" if learned else "sampling", "estimated_pairs": s["estimated_pairs"],
        "estimator_batch_rel_err": s["estimator_mean_abs_rel_err"], "estimator_task_rel_err": s["estimator_task_rel_err"],
    }
    ok = True
    if fp64 is not None:
        line["fp64"] = fp64
        line["speedup_vs_fp64"] = fp64["ms_per_step"] / job_ms
        ok = fp64["pairs_per_step"] == job_pairs and fp64["pair_hash"] == job_hash
        line["identical_pair_set"] = ok
    if small is not None:
        line["engine_small_e2e"] = small
    print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()
    if not ok:
        sys.exit("the mixed-precision pair set differs from the FP64 pair set")


def _pipe_roofline(s, prec, D, clocks):
    """Distance loop (count pass) against the CUDA-core pipe it runs on.

    Operations per candidate evaluation on that pipe: FP64 predicate 2*D (D
    subtractions, D-1 FMAs and one multiply); FP32 filter D + 1 (the norm add
    and D FMAs; a packed f32x2 instruction counts as two; the borderline-band
    test is an integer minimum on the ALU pipe).  Peak = lanes x SM clock
    sampled during the timed steps (nominal lanes: 64 FP64 and 128 FP32 FMA
    per SM per clock)."""
    mhz = clocks.get("sm_mhz") or 1965.0
    lanes = FP64_LANES if prec == 0 else FP32_LANES
    ops = 2 * D if prec == 0 else D + 1
    peak = NUM_SM * lanes * mhz * 1e6 / 1e12
    t = s["ms_count"] / 1e3
    ach = ops * s["distance_calcs"] / t / 1e12 if t > 0 else None
    return {"bound": "fp64 pipe" if prec == 0 else "fp32 pipe", "kernel": "k_join count pass (distance loop)",
            "achieved": ach, "peak": peak, "unit": "Tops/s", "frac": (ach / peak) if ach else None,
            "peak_kind": "nominal lanes x sampled SM clock", "ops_per_evaluation": ops,
            "evaluations": s["distance_calcs"], "count_pass_ms": s["ms_count"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="c4")
    ap.add_argument("--n", type=int, default=None)
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: split one join over the ranks (strong scaling) instead of N replicas")
    ap.add_argument("--capacity", type=int, default=None, help="batch capacity in pairs (default: the workload's)")
    ap.add_argument("--task-sample", type=int, default=1,
                    help="K > 1: join only task shard 0 of K (every Kth task of the cost order), a reduced case "
                         "with the full workload's cell density for profiler captures")
    ap.add_argument("--precision", type=int, default=None, help="0 FP64, 1 FP32 filter + FP64 refine")
    ap.add_argument("--mode", type=int, default=None, help="search mode (default: the workload's)")
    ap.add_argument("--scheduler", choices=["learned", "sampling"], default=None,
                    help="batch/queue estimator (default: learned for the mixed-precision c4 workload)")
    ap.add_argument("--weights", default=ESTIMATOR_WEIGHTS, help="learned-estimator weights file")
    ap.add_argument("--fp64-steps", type=int, default=2,
                    help="timed steps of the plain FP64 method on the same points (0: skip)")
    ap.add_argument("--e2e-steps", type=int, default=1, help="timed end-to-end steps with host delivery (0: skip)")
    ap.add_argument("--delivery", choices=["none", "device"], default="none",
                    help="timed steps: on-device fold of every batch (none) or every batch handed to a "
                         "device-memory consumer one at a time (device)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-stage-probe", action="store_true",
                    help="skip the extra step whose stages run one after another (per-kernel times)")
    ap.add_argument("--no-ref-cuda", action="store_true",
                    help="skip the small workloads timed beside the reference's own CUDA pipeline")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
