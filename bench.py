#!/usr/bin/env python
"""AMEn solves/s and p50/p99 latency at relative residual 1e-8 on B200.

One step = solving one batch of synthetic requests (a seeded mix of 2-D QTT
Poisson problems with 6-20 cores and parametric diffusion problems with
d in {4, 5}, n in {16, 32}), each to relative residual 1e-8.  The requests
are identical in every step.  ``--engine plain`` solves them one at a time
through the drop-in ``amen``; ``--engine served`` (the default once
available) admits all of them into the batched serving engine.

Prints one JSON line (rank 0).  ``--impl reference`` times the CPU oracle
(the NumPy/SciPy restatement of the reference path) on the host cores
instead, on a bounded sample of the same requests.

Launch: ``python bench.py`` (1 GPU) or, for N GPUs,
``python -m torch.distributed.run --nproc-per-node N ... bench.py --gpus N``:
every rank serves its own copy of the request batch (replicas; independent
solves need no collective), ``value`` = all ranks' solves / max time.
"""

from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "AMEn solves/s at relative residual 1e-8"
UNIT = "solves/s"
TOL = 1e-8
MAX_SWEEPS = 30


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--engine", default="persistent", choices=["plain", "served", "persistent"])
    ap.add_argument("--requests", type=int, default=1184,
                    help="requests per step (1184 = 8 per SM of a B200)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="requests in the CPU baseline sample (0: automatic)")
    ap.add_argument("--serve-requests", type=int, default=0,
                    help="requests in the served stream (0: three times --requests, the "
                         "batch's requests cycled)")
    ap.add_argument("--serve-mem-gb", type=float, default=48.0,
                    help="device memory the server may hold in slabs of requests in flight")
    ap.add_argument("--serve-rate", type=float, default=0.0,
                    help="arrival rate of the served run (0: twice the measured batch rate)")
    ap.add_argument("--plain-sample", type=int, default=8,
                    help="requests timed through the plain one-at-a-time drop-in (0: skip)")
    ap.add_argument("--diffusion-dims", default="4,5",
                    help="dimensions d the diffusion requests draw from")
    ap.add_argument("--diffusion-modes", default="16,32",
                    help="mode sizes n the diffusion requests draw from")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------


def make_requests(count: int, seed: int, dims=(4, 5), modes=(16, 32)):
    """Seeded request mix: half 2-D QTT Poisson (N ~ U{3..10}, sin*sin
    right-hand side), half parametric diffusion (d ~ U(dims), n ~ U(modes),
    theta ~ U(-1, 1))."""
    from ttnumpy_b200 import problems as P

    rng = np.random.default_rng(seed)
    dims, modes = tuple(dims), tuple(modes)
    reqs = []
    for i in range(count):
        if i % 2 == 0:
            N = int(rng.integers(3, 11))
            p = P.qtt_poisson_2d(N)
            p.meta["kind"] = "qtt"
        else:
            d = int(dims[int(rng.integers(0, len(dims)))])
            n = int(rng.choice(modes))
            p = P.parametric_diffusion(d, n, rng.uniform(-1.0, 1.0, size=d))
            p.meta["kind"] = "diffusion"
        reqs.append(p)
    return reqs


# DRAM bytes (read + write) of one k_amen launch of the standard mix at
# 1184 and 592 requests per step, from ncu captures of `python bench.py`
# (profiles/k_amen_bench_*req.md); other workloads report null
MEASURED_TRAFFIC = {1184: 1658012785152 + 1601813339392, 592: 655255445760 + 720370022144}


def _traffic(args):
    standard = (args.seed == 0 and _ints(args.diffusion_dims) == [4, 5]
                and _ints(args.diffusion_modes) == [16, 32])
    return MEASURED_TRAFFIC.get(args.requests) if standard else None


def aggregate_rate(solved: int, ms: float, world: int, device: str = "cuda"):
    """Whole-job rate over the ranks: all ranks' solves over the slowest
    rank's time.  Returns (solves per second, max milliseconds); a single
    process needs no process group."""
    if world > 1:
        import torch
        import torch.distributed as dist

        t = torch.tensor([float(solved), float(ms)], dtype=torch.float64, device=device)
        mx = t.clone()
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        solved, ms = float(t[0].item()), float(mx[1].item())
    return solved / (ms * 1e-3), ms


def _ints(text):
    return [int(v) for v in str(text).split(",") if v.strip()]


def solve_kwargs(p):
    return dict(residual_tol=TOL, symmetric=True, max_sweeps=MAX_SWEEPS, seed=0,
                stagnation_factor=None)


def x0_cores(p):
    """Initial guess: rank-3 all-ones for QTT Poisson (the reference
    benchmark's choice), the default (all-ones with b's ranks) otherwise."""
    if p.meta.get("kind") == "qtt":
        return 3
    return None


# ---------------------------------------------------------------------------
# CPU oracle (reference arm and cpu_baseline)
# ---------------------------------------------------------------------------


def _cpu_solve(p):
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    from threadpoolctl import threadpool_limits

    from oracle import tt_oracle as O

    with threadpool_limits(1):
        A, b = O.Train(p.A), O.Train(p.b)
        x0 = None
        r = x0_cores(p)
        if r is not None:
            x0 = O.orthonormalize(O.ones(b.row_modes, ranks=r), "right")
        t0 = time.perf_counter()
        x, info = O.amen(A, b, x0=x0, **solve_kwargs(p))
        dt = time.perf_counter() - t0
    return dt, info.stop_reason, (info.residuals[-1] if info.residuals else float("nan"))


def cpu_run(reqs, workers: int):
    """Solve ``reqs`` on a spawn pool of single-threaded workers; returns
    (seconds, per-request results)."""
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(workers) as pool:
        res = pool.map(_cpu_solve, reqs, chunksize=1)
    return time.perf_counter() - t0, res


def cpu_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(reqs, n):
    # every other request is QTT, so a prefix keeps the mix
    return reqs[: max(2, n)]


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [v.strip() for v in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = max(mx, float(parts[1]))
            except ValueError:
                continue
            for name, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh)
    except OSError:
        return {}


def fp64_peak_tflops(K, torch):
    """Measured FP64 FMA throughput of this GPU (own probe kernel)."""
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = K.lib()
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    blocks, iters = sms * 8, 4096
    lib.ttb_fma_peak(out.data_ptr(), blocks, iters, K.stream())
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        lib.ttb_fma_peak(out.data_ptr(), blocks, iters, K.stream())
        b.record()
        torch.cuda.synchronize()
        flops = 2.0 * 8 * iters * 256 * blocks
        best = max(best, flops / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best


class Engine:
    """Solves a list of requests; returns results and per-request latencies (ms).

    ``plain``: one drop-in ``amen`` call after another; ``served``: the
    lockstep batch engine; ``persistent``: one persistent launch in which
    every request is a thread block running its whole solve.
    """

    RMAX = 64

    def __init__(self, kind: str):
        import torch

        import ttnumpy_b200 as tt

        self.kind = kind
        self.tt = tt
        self.torch = torch

    def upload(self, reqs):
        """Inputs made resident on the device (not timed)."""
        tt = self.tt
        if self.kind == "persistent":
            from ttnumpy_b200.persistent import PersistentBatch, prepare

            return PersistentBatch(prepare([(p.A, p.b, self.x0_host(p), solve_kwargs(p))
                                            for p in reqs]), self.RMAX)
        out = []
        for p in reqs:
            A, b = tt.TensorTrain(p.A), tt.TensorTrain(p.b)
            r = x0_cores(p)
            x0 = tt.ones(b.physical_dims(), ranks=r).orthonormalize("right") if r else None
            out.append((A, b, x0, p))
        return out

    @staticmethod
    def x0_host(p):
        r = x0_cores(p)
        if r is None:
            return None
        modes = [c.shape[1] for c in p.b]
        ranks = [1] + [r] * (len(modes) - 1) + [1]
        return [np.ones((ranks[i], modes[i], 1, ranks[i + 1])) for i in range(len(modes))]

    def solve_all(self, handle, download: bool = False):
        torch = self.torch
        if self.kind == "persistent":
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            handle.launch()
            e.record()
            res = handle.collect()
            ms = s.elapsed_time(e)
            for r in res:
                if r.status != 0:
                    raise RuntimeError(f"persistent solve failed with status {r.status}")
            results = [(r.x, r.info) for r in res]
            if download:
                for x, _ in results:
                    x.to_numpy()
            return results, handle.latencies_ms()
        lat = []
        results = []
        if self.kind == "plain":
            for A, b, x0, p in handle:
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record()
                x, info = self.tt.amen(A, b, x0=x0, return_info=True, **solve_kwargs(p))
                if download:
                    x.to_numpy()
                e.record()
                results.append((x, info))
                lat.append((s, e))
            torch.cuda.synchronize()
            return results, [s.elapsed_time(e) for s, e in lat]
        from ttnumpy_b200.serving import serve_batch

        return serve_batch(handle, solve_kwargs, download=download)


def flush_l2(torch, buf):
    from ttnumpy_b200 import kernels as K

    K.fill_(buf, 0.0)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference" and rank != 0:
        return  # the reference arm runs on rank 0's host cores alone
    reqs = make_requests(args.requests, args.seed, _ints(args.diffusion_dims),
                         _ints(args.diffusion_modes))
    cores = cpu_cores()
    n_sample = args.cpu_sample or min(len(reqs), max(2 * cores, 8))

    if args.impl == "reference":
        sample = cpu_sample(reqs, n_sample)
        for _ in range(args.warmup):
            cpu_run(sample[: min(len(sample), cores)], cores)
        total, n = 0.0, 0
        for _ in range(args.steps):
            dt, res = cpu_run(sample, cores)
            total += dt
            n += sum(1 for r in res if str(r[1]) == "converged")
        value = n / total
        line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config(args, reqs),
                "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                                 "sample": f"{len(sample)} of the {len(reqs)} requests per step "
                                           f"(the first ones, same mix), {cores} single-threaded "
                                           "oracle workers"},
                "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch

    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    from ttnumpy_b200 import kernels as K

    K.lib()
    engine_kind = args.engine
    eng = Engine(engine_kind)
    dev_reqs = eng.upload(reqs)
    flush = torch.empty(64 << 20, dtype=torch.float64, device="cuda")  # 512 MB > L2

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        eng.solve_all(dev_reqs)
    barrier()

    lib = K.lib()
    if engine_kind == "persistent":
        return persistent_main(args, eng, dev_reqs, reqs, flush, barrier, world, rank, local)
    # which kernel class dominates: one profiled pass, all classes
    lib.ttb_profile_reset()
    lib.ttb_profile_enable((1 << 12) - 1)
    eng.solve_all(dev_reqs)
    torch.cuda.synchronize()
    lib.ttb_profile_enable(0)
    shares = profile_read(lib)
    dominant = max(shares, key=lambda c: shares[c]["ms"])
    lib.ttb_profile_reset()

    # timed region: device time per step, L2 flushed between steps
    step_ms, lats, ok, launches = [], [], 0, 0
    barrier()
    with ClockSampler(local) as clocks:
        lib.ttb_profile_enable(1 << dominant)
        for _ in range(args.steps):
            flush_l2(torch, flush)
            torch.cuda.synchronize()
            l0 = K.launch_count()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            results, lat = eng.solve_all(dev_reqs)
            e.record()
            torch.cuda.synchronize()
            launches += K.launch_count() - l0
            step_ms.append(s.elapsed_time(e))
            lats.extend(lat)
            ok += sum(1 for _, info in results if info.converged)
        lib.ttb_profile_enable(0)
    barrier()
    dom = profile_read(lib)[dominant]
    value, total_ms = aggregate_rate(ok, sum(step_ms), world)

    # end to end through the public API from pinned host buffers
    e2e = e2e_run(eng, reqs, args, torch, flush)

    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    pk = peaks()
    fp64 = fp64_peak_tflops(K, torch)
    roof = roofline(dominant, dom, pk, fp64)
    cpu = None
    if world == 1:
        sample = cpu_sample(reqs, n_sample)
        dt, res = cpu_run(sample, cores)
        conv = sum(1 for r in res if str(r[1]) == "converged")
        cpu = {"value": conv / dt, "unit": UNIT, "cores": cores, "kind": "port",
               "sample": f"{len(sample)} of the {len(reqs)} requests (same mix), one pass, "
                         f"{cores} single-threaded oracle workers"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config(args, reqs, engine_kind),
            "latency_ms": {"p50": percentile(lats, 50), "p99": percentile(lats, 99)},
            "converged": f"{ok}/{len(reqs) * args.steps}",
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clocks.summary(),
            "kernel_shares": {CLASS_NAMES[c]: round(v["ms"], 3) for c, v in shares.items()
                              if v["ms"] > 0}}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def persistent_main(args, eng, batch, reqs, flush, barrier, world, rank, local):
    """Timed region for the persistent engine: one launch per step.  Steps
    alternate between two device-resident copies of the batch on two
    streams, so a step's last (longest-running) solves overlap the next
    step's first ones, as back-to-back batches do in service; a copy is
    launched again only after its previous step has been collected."""
    import torch

    from ttnumpy_b200 import kernels as K

    batches = [batch, eng.upload(reqs)]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    ok, lats, flops = 0, [], 0.0

    def collect(j):
        nonlocal ok, flops
        with torch.cuda.stream(streams[j]):  # host reads on the batch's own stream
            res = batches[j].collect()
            lats.extend(batches[j].latencies_ms())
            flops += batches[j].gemm_flops()
        ok += sum(1 for r in res if r.status == 0 and r.info.converged)

    barrier()
    with ClockSampler(local) as clocks:
        K.fill_(flush, 0.0)
        torch.cuda.synchronize()
        l0 = K.launch_count()
        start = torch.cuda.Event(enable_timing=True)
        start.record()
        done = [None, None]
        for k in range(args.steps):
            j = k % 2
            if done[j] is not None:
                done[j].synchronize()
                collect(j)
            streams[j].wait_event(start)
            batches[j].launch(streams[j])
            done[j] = torch.cuda.Event()
            done[j].record(streams[j])
        for k in range(max(0, args.steps - 2), args.steps):
            done[k % 2].synchronize()
            collect(k % 2)
        cur = torch.cuda.current_stream()
        for st in streams:
            cur.wait_stream(st)
        end = torch.cuda.Event(enable_timing=True)
        end.record()
        torch.cuda.synchronize()
        launches = K.launch_count() - l0
    step_ms = [start.elapsed_time(end)]
    barrier()
    value, total_ms = aggregate_rate(ok, sum(step_ms), world)
    for b in batches:  # the served run admits its own requests by device memory
        b.release()
    torch.cuda.empty_cache()
    e2e = served_run(reqs, args, torch, rate=args.serve_rate or 2.0 * value / world)
    e2e["value"], _ = aggregate_rate(e2e.pop("_solved"), 1e3 * e2e.pop("_seconds"), world)
    plain = plain_run(reqs, args) if (world == 1 and args.plain_sample > 0) else None
    if rank != 0:
        if world > 1:
            torch.distributed.destroy_process_group()
        return
    fp64 = fp64_peak_tflops(K, torch)
    ach = flops / (sum(step_ms) * 1e-3) / 1e12
    roof = {"kernel": "k_amen (ttb_amen_persistent)", "bound": "tensor", "unit": "TFLOP/s",
            "achieved": ach, "peak": fp64, "peak_source": "measured FP64 FMA probe "
            "(ttb_fma_peak); MEASURED_PEAKS.json has no FP64 figure",
            "frac": ach / fp64, "traffic": _traffic(args),
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of "
                              f"this workload (profiles/k_amen_bench_{args.requests}req.md)",
            "flops_counted": "2mnk of every dense product the blocks ran; QR/SVD/LU not counted",
            "per_launch_us": 1e3 * sum(step_ms) / args.steps, "launches": args.steps,
            "timing": "aggregate over the timed steps (consecutive launches overlap on two "
                      "streams)"}
    cpu = None
    if world == 1:
        n_sample = args.cpu_sample or min(len(reqs), max(2 * cpu_cores(), 8))
        sample = cpu_sample(reqs, n_sample)
        dt, res = cpu_run(sample, cpu_cores())
        conv = sum(1 for r in res if str(r[1]) == "converged")
        cpu = {"value": conv / dt, "unit": UNIT, "cores": cpu_cores(), "kind": "port",
               "sample": f"{len(sample)} of the {len(reqs)} requests (same mix), one pass, "
                         f"{cpu_cores()} single-threaded oracle workers"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config(args, reqs, "persistent"),
            "latency_ms": {"p50": percentile(lats, 50), "p99": percentile(lats, 99)},
            "converged": f"{ok}/{len(reqs) * args.steps}", "roofline": roof,
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "plain_gpu": plain,
            "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


CLASS_NAMES = ["gemm", "copy", "kron", "norm", "local_matrix", "qr", "svd", "lu", "rank",
               "minres", "gmres", "round"]


def profile_read(lib):
    import ctypes as C

    out = {}
    for c in range(len(CLASS_NAMES)):
        ms, n, fl, by = C.c_double(), C.c_longlong(), C.c_double(), C.c_double()
        lib.ttb_profile_read(c, C.byref(ms), C.byref(n), C.byref(fl), C.byref(by))
        out[c] = {"ms": ms.value, "n": n.value, "flops": fl.value, "bytes": by.value}
    return out


def roofline(cls, rec, pk, fp64_tflops):
    """Achieved algorithmic rate of the dominant kernel class over the
    timed region against its measured peak."""
    name = CLASS_NAMES[cls]
    if rec["n"] == 0 or rec["ms"] <= 0:
        return {"kernel": name, "bound": None, "achieved": None, "peak": None, "frac": None,
                "traffic": None}
    if rec["flops"] > 0:
        ach = rec["flops"] / (rec["ms"] * 1e-3) / 1e12
        return {"kernel": name, "bound": "tensor", "unit": "TFLOP/s", "achieved": ach,
                "peak": fp64_tflops, "peak_source": "measured FP64 FMA probe (ttb_fma_peak)",
                "frac": ach / fp64_tflops, "traffic": None,
                "per_launch_us": 1e3 * rec["ms"] / rec["n"], "launches": rec["n"]}
    gbs = rec["bytes"] / (rec["ms"] * 1e-3) / 1e9
    peak = pk.get("hbm_gbs", 6650.0)
    return {"kernel": name, "bound": "hbm", "unit": "GB/s", "achieved": gbs, "peak": peak,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in pk else "fallback",
            "frac": gbs / peak, "traffic": None, "per_launch_us": 1e3 * rec["ms"] / rec["n"],
            "launches": rec["n"]}


def served_run(reqs, args, torch, rate):
    """End to end through the serving API: the requests (host cores) arrive
    as a seeded Poisson stream at ``rate`` per second and are served by
    continuous batching on concurrent persistent launches (inputs copied to
    the device per launch, solutions read back).  ``args.steps`` passes,
    each timed with CUDA events around the whole stream."""
    from ttnumpy_b200.persistent_serving import PersistentServer

    n_serve = args.serve_requests or 3 * len(reqs)
    batch_host = [(p.A, p.b, Engine.x0_host(p), solve_kwargs(p)) for p in reqs]
    host = [batch_host[i % len(batch_host)] for i in range(n_serve)]
    rng = np.random.default_rng(args.seed + 1)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(host)))
    arrivals -= arrivals[0]
    budget = int(args.serve_mem_gb * 2**30)
    # untimed warm-up of the serving path (streams, pinned staging, allocator)
    warm = min(len(host), 64)
    PersistentServer(mem_budget=budget).serve(host[:warm], list(arrivals[:warm] * 0.0))
    torch.cuda.synchronize()
    seconds, solved, lats, launches, h2d, d2h, peak = 0.0, 0, [], 0, 0, 0, 0
    steps = max(1, args.steps)
    for _ in range(steps):
        server = PersistentServer(mem_budget=budget)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        jobs = server.serve(host, list(arrivals))
        torch.cuda.synchronize()
        e.record()
        e.synchronize()
        seconds += s.elapsed_time(e) * 1e-3
        solved += sum(1 for j in jobs if j.result.status == 0 and j.result.info.converged)
        lats.extend(1e3 * j.latency for j in jobs)
        launches += server.launches
        h2d, d2h = server.h2d_bytes, server.d2h_bytes
        peak = max(peak, server.peak_bytes)
        # outside the timed region: drop this pass's results and return the
        # cached blocks, so every pass starts from the same allocator state
        jobs = server = None
        torch.cuda.empty_cache()
    return {"value": solved / seconds, "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h,
            "mode": f"served: {len(host)} requests per step (the batch's {len(reqs)} cycled) "
                    f"arriving as a Poisson stream at {rate:.1f}/s, continuous batching over 16 "
                    f"streams of persistent launches admitted by a {args.serve_mem_gb:g} GB "
                    "slab budget, inputs copied from host per launch, solutions read back",
            "requests_per_step": len(host),
            "peak_slab_gb": peak / 2**30,
            "launches_per_step": launches / steps,
            "latency_ms": {"p50": percentile(lats, 50), "p99": percentile(lats, 99)},
            "_seconds": seconds, "_solved": solved}


def plain_run(reqs, args):
    """The plain one-solve-at-a-time GPU AMEn (the drop-in ``amen``) on the
    first requests of the mix, for the served-versus-plain ratio."""
    import torch

    eng = Engine("plain")
    sample = reqs[: args.plain_sample]
    handle = eng.upload(sample)
    eng.solve_all(handle[:1])
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    results, _ = eng.solve_all(handle)
    e.record()
    torch.cuda.synchronize()
    ok = sum(1 for _, info in results if info.converged)
    return {"value": ok / (s.elapsed_time(e) * 1e-3), "unit": UNIT,
            "sample": f"the first {len(sample)} requests of the mix, solved one after another by "
                      "the drop-in amen (every contraction and factorisation a library call)"}


def e2e_run(eng, reqs, args, torch, flush):
    """Same metric through the public API: each step uploads the requests
    from host memory and downloads the solutions."""
    from ttnumpy_b200 import kernels as K

    total, ok, d2h, h2d = 0.0, 0, 0, 0
    steps = max(1, args.steps)
    for _ in range(steps):
        K.fill_(flush, 0.0)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        handle = eng.upload(reqs)
        results, _ = eng.solve_all(handle, download=False)
        host = [x.to_numpy() for x, _ in results]
        e.record()
        torch.cuda.synchronize()
        total += s.elapsed_time(e)
        ok += sum(1 for _, info in results if info.converged)
        d2h = sum(sum(c.nbytes for c in h) for h in host)
        h2d = sum(sum(np.asarray(c).nbytes for c in p.A) + sum(np.asarray(c).nbytes for c in p.b)
                  for p in reqs)
    return {"value": ok / (total * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h}


def percentile(v, q):
    if not v:
        return None
    return float(np.percentile(np.asarray(v, dtype=np.float64), q))


def config(args, reqs, engine="reference"):
    kinds = {}
    for p in reqs:
        kinds[p.meta["kind"]] = kinds.get(p.meta["kind"], 0) + 1
    return {"workload": "AMEn request mix: 2-D QTT Poisson (6-20 cores, mode 2) and parametric "
                        f"diffusion (d in {args.diffusion_dims}, mode in {args.diffusion_modes}), "
                        "residual 1e-8",
            "requests_per_step": len(reqs), "mix": kinds, "engine": engine,
            "max_sweeps": MAX_SWEEPS, "stagnation_factor": None,
            "parallelism": f"replicas x{args.gpus}", **_timing_notes(engine)}


def _timing_notes(engine):
    if engine == "persistent":
        return {"l2": "inputs larger than L2 (two batches of slabs, tens of GB); 512 MB flush "
                      "before the timed region",
                "steps": "alternate between two device-resident copies of the batch on two "
                         "streams, so one step's last solves overlap the next step's first"}
    if engine == "reference":
        return {"host": "the CPU oracle on the host cores; no device memory involved"}
    return {"l2": "flushed (512 MB write) before every timed step"}


if __name__ == "__main__":
    main()
