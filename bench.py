#!/usr/bin/env python3
"""Benchmark of the KsPIR online answer on B200.

Workload (one "step"): one client's online answer over the 256 MB database of
tests/test-pir.cpp -- 32768 records x 8 KB = r = 16 sub-databases of
4096 x 2048 16-bit entries, preprocessed to 1 GiB of packed CRT words --
with N = 4096, N1 = 128, N2 = 16 (reference tests/test-pir.cpp:14-29).
Synthetic, seeded inputs of that shape (kspir_b200.synth).

Reported (one JSON line on rank 0):
  value      whole-job queries/s of single-query answers, inputs resident in
             HBM, issued round-robin on --streams streams so one answer's key
             switches overlap another's database scan; device-timed with CUDA
             events on the launching stream (max over ranks).  latency_ms is
             one answer at a time on one stream, with its phases
  e2e        queries/s through the public C ABI (kspir_answer, blocking) from
             --streams host threads, each query in pinned host memory and its
             response read back, per step; one_caller_queries_per_s from one
             thread
  roofline   the dominant kernel (the database scan): algorithmic bytes per
             launch (r * N * N/2 * 8 = 1 GiB) / its mean CUDA-event duration
  batched    the batched answer (kspir_answer_batch) at B = 1, 8, 32, 64, 128
             queries of distinct clients: device-timed and end-to-end
             queries/s, the scan variant the autotuner picked, per-phase
             times, and the tensor roofline of the batched scan (int8 limb
             products: 2 comp x 2 primes x 16 limb pairs per database word
             and query)
  cpu_baseline  the reference's CPU answer (oracle/_ref, or the C port)
             on the host cores, on a bounded sample

--impl reference times the reference's own CPU implementation instead
(rank 0 only), on the same metric.
Multi-GPU (torchrun): each rank is an independent replica answering its own
queries (no data-path collective); scaling "weak".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "answer ms/query & batched queries/s at 256 MB DB (bit-exact); GB/s vs HBM peak"
N = 4096
CRTMOD = 268369921 * 249561089


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="kspir", choices=["kspir", "reference"])
    ap.add_argument("--r", type=int, default=16)
    ap.add_argument("--N1", type=int, default=128)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--streams", type=int, default=8,
                    help="streams (and host threads, end to end) the single answers are issued on")
    ap.add_argument("--batches", default="1,8,32,64,128", help="batch sizes of the batched sweep ('' = none)")
    ap.add_argument("--clients", type=int, default=128, help="distinct client key sets of the batched sweep")
    ap.add_argument("--no-extras", dest="extras", action="store_false",
                    help="skip the 1 GB database and the serving run")
    ap.add_argument("--serving-rates", default="1000,4000", help="offered queries/s of the serving run")
    return ap.parse_args()


def workload_config(args):
    records = args.r * N // 2                 # 8 KB records: N / 2 per sub-database
    pre = args.r * N * N // 2 * 8             # preprocessed bytes (u64 per NTT slot)
    l2 = (f"inputs larger than L2: the {pre / 2**30:g} GiB preprocessed database is streamed every step"
          if pre > 126 * 10**6 else f"the {pre / 2**20:g} MiB preprocessed database fits in L2 (no flush)")
    return {"workload": f"single-query online answer, {records * 8 // 1024} MB DB ({records} x 8 KB records), "
                        f"r={args.r} N1={args.N1} N2={N // 2 // args.N1} N={N}",
            "r": args.r, "N1": args.N1, "N2": N // 2 // args.N1,
            "db_bytes_preprocessed": pre,
            "l2": l2,
            "parallelism": "replicas"}


# ---------------------------------------------------------------------------
# clocks during the timed region (NVML reads only)

class ClockSampler:
    def __init__(self, index: int, period: float = 0.001):
        self.samples = []
        self.max_mhz = None
        self.reasons = set()
        self._stop = threading.Event()
        self._ok = False
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self._ok = True
        except Exception:
            self.nv = None
        self.period = period
        self._t = None

    def _run(self):
        nv = self.nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwSlowdown", 0x8),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksThrottleReasonSwThermalSlowdown", 0x20),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksThrottleReasonHwThermalSlowdown", 0x40),
            "sw_power_cap": getattr(nv, "nvmlClocksThrottleReasonSwPowerCap", 0x4),
        }
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                mask = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                for n, bit in names.items():
                    if mask & bit:
                        self.reasons.add(n)
            except Exception:
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        if self._ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# CPU baseline: the reference's answer on the host cores

def cpu_answer_rate(db, client, perms, r, N1, seconds, threads):
    """Independent answers on `threads` host threads for about `seconds`;
    returns (queries/s, kind, answers, threads)."""
    import ctypes

    from oracle import pyoracle as po
    c = dict(client, perms=perms)
    if po.ref_available():
        L, kind = po.ref(), "reference"

        def one():
            resp = np.zeros(2 * N, np.uint64)
            t = ctypes.c_double()
            L.ref_answer(po._p(db), r, N1, po._p(c["query"]), po._p(c["baby"]), po._p(c["giant"]),
                         po._p(c["packing"]), po._p(c["rgsw"]), po._p(c["perms"]), po._p(resp), None, None,
                         ctypes.byref(t))
    else:
        kind = "port"

        def one():
            po.answer(db, r, N1, c)
    counts = [0] * threads
    t_end = [0.0]
    start = time.perf_counter()
    deadline = start + seconds

    def worker(i):
        while True:
            one()
            counts[i] += 1
            if time.perf_counter() >= deadline:
                break
    ths = [threading.Thread(target=worker, args=(i,)) for i in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    t_end[0] = time.perf_counter() - start
    n = sum(counts)
    return n / t_end[0], kind, n, threads


def host_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------

def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s, earlier measurement on this pool)"


def read_int8_peak():
    """Dense int8 tensor peak, TOP/s: twice the measured bf16 burst (B200 issues
    twice as many int8 as bf16 MMA operations per cycle: ncu peak_sustained
    16384 vs 8192 per SM)."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return 2 * float(json.load(open(p))["bf16_tflops"]), "2 x measured bf16 burst (MEASURED_PEAKS.json)"
    return 2 * 1590.0, "2 x fallback bf16 1.59 PFLOP/s"


def read_traffic(r):
    """DRAM bytes per scan launch from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "k_scan_single_query_8192_records.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.strip().startswith("dram_bytes_per_launch_r16:"):
            try:
                return int(float(line.split(":", 1)[1].split()[0]) * r / 16)
            except ValueError:
                return None
    return None


def bench_preprocess(args, ctx, raw, rank):
    """Server preprocessing (database_tobsgsntt + database_tocrt of all r
    sub-databases) through kspir_db_preprocess: host raw database in (pageable
    memory, host->device copy inside), resident datacrt out.  Reports the
    device time (CUDA events on the context stream), the end-to-end time, and
    on rank 0 the reference's own preprocessing timed on one sub-database of
    the same raw database (oracle/_ref, when built) scaled to r."""
    r = args.r
    dev, wall = [], []
    for _ in range(3):
        t0 = time.perf_counter()
        dev.append(ctx.preprocess_db(raw))
        wall.append((time.perf_counter() - t0) * 1e3)
    out = {"workload": f"r={r} sub-databases of N x N/2 raw words < 65537 ({r * 16} MB of records)",
           "device_ms": float(np.median(dev)), "e2e_ms": float(np.median(wall)),
           "h2d_bytes": int(raw.nbytes), "reference_published_ms": 4144.0 if r == 16 else None}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import pyoracle as po
        if po.ref_available():
            num = N * N // 2
            t0 = time.perf_counter()
            po.ref_db_preprocess(raw[:num], 1, args.N1)
            one = time.perf_counter() - t0
            out["cpu_reference_ms"] = one * 1e3 * r
            out["cpu_reference_sample"] = f"1 of {r} sub-databases, 1 thread, scaled by {r}"
    return out


def bench_client(ctx, n=128, reps=5):
    """Device test clients: query_bsgs_rns for n clients in one call, and
    decrypt_bsgs_total of n responses (host buffers in and out, timed end to
    end on the host; synthetic ternary secrets)."""
    rng = np.random.default_rng(99)
    sec = rng.integers(-1, 2, size=(n, N)).astype(np.int64)
    sec = np.where(sec < 0, sec + CRTMOD, sec).astype(np.uint64)
    rows = rng.integers(0, N // 2, size=n).astype(np.uint32)
    q = ctx.client_queries(sec, rows, seed=1)          # warm-up (tables, allocation)
    tq = []
    for i in range(reps):
        t0 = time.perf_counter()
        q = ctx.client_queries(sec, rows, seed=2 + i)
        tq.append(time.perf_counter() - t0)
    resp = np.ascontiguousarray(q[:, :2 * N])          # any canonical crtMod words
    ctx.client_decrypt(sec, resp, 16)
    td = []
    for _ in range(reps):
        t0 = time.perf_counter()
        ctx.client_decrypt(sec, resp, 16)
        td.append(time.perf_counter() - t0)
    return {"batch": n, "queries_per_s": n / float(np.median(tq)), "decrypts_per_s": n / float(np.median(td)),
            "calls_ms": {"queries": [round(t * 1e3, 3) for t in tq], "decrypts": [round(t * 1e3, 3) for t in td]},
            "note": "end to end through kspir_client_queries / kspir_client_decrypt with host buffers; "
                    f"median of {reps} calls"}


def run_gpu(args, rank, world, local_rank):
    import torch

    import kspir_b200 as kb
    from kspir_b200 import synth

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    r, N1 = args.r, args.N1
    batches = [int(x) for x in args.batches.split(",") if x.strip()]
    bmax = max(batches) if batches else 1
    nclients = max(1, min(args.clients, bmax))
    cl = synth.gen_client(args.seed + rank, r, N1)
    perms = kb.permutation_matrix(N1)
    ctx = kb.Context(r, N1, device=local_rank, max_clients=nclients, max_inflight=bmax)
    # the resident database comes from the device preprocessing of a raw one
    prep = bench_preprocess(args, ctx, synth.gen_raw_db(args.seed, r), rank)
    db = ctx.download_db()
    ctx.upload_perms(perms)
    ctx.upload_client(0, cl["baby"], cl["giant"], cl["packing"], cl["rgsw"])

    # device-resident query and response
    dq = torch.from_numpy(cl["query"].view(np.int64).copy()).cuda()
    dr = torch.empty(2 * N, dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    host_ref = ctx.answer(0, cl["query"])   # host path, for a consistency check of the device path

    S = max(1, args.streams)
    streams = [stream] + [torch.cuda.Stream() for _ in range(S - 1)]
    drs = [dr] + [torch.empty(2 * N, dtype=torch.int64, device="cuda") for _ in range(S - 1)]

    def step(i=0):
        k = i % S
        ctx.answer_device(0, dq.data_ptr(), drs[k].data_ptr(), streams[k].cuda_stream)

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            step()
    torch.cuda.synchronize()
    if not np.array_equal(dr.cpu().numpy().view(np.uint64), host_ref):
        raise RuntimeError("device-path response differs from the host-path response")

    def timed(nstreams):
        """Device time of args.steps answers issued round-robin on `nstreams`
        streams, bracketed by events on the main stream."""
        main = torch.cuda.current_stream()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev0.record(main)
        for st in streams[:nstreams]:
            st.wait_event(ev0)
        for i in range(args.steps):
            step(i % nstreams)
        for st in streams[:nstreams]:
            main.wait_stream(st)
        ev1.record(main)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        return ev0.elapsed_time(ev1)

    # one answer at a time: the latency and its phases
    ctx.timing_reset()
    ms_serial = timed(1)
    answers, _, tot_ms, phases = ctx.timing_summary()
    # answers on S streams at once: one's key switches overlap another's scan
    for i in range(3 * S):
        step(i)
    torch.cuda.synchronize()
    ctx.timing_reset()
    with ClockSampler(local_rank) as clocks:
        ms = timed(S)
    _, launches, _, _ = ctx.timing_summary()
    ctx.sync()
    for k in range(S):
        if not np.array_equal(drs[k].cpu().numpy().view(np.uint64), host_ref):
            raise RuntimeError(f"stream {k}: overlapped response differs from the host-path response")

    # end to end through the C ABI: pinned host query in, response out, every
    # step; S host threads each call kspir_answer (blocking) on its own buffers
    qhs = [torch.from_numpy(cl["query"].view(np.int64).copy()).pin_memory() for _ in range(S)]
    rhs = [torch.empty(2 * N, dtype=torch.int64).pin_memory() for _ in range(S)]
    qh_np = [q.numpy().view(np.uint64) for q in qhs]
    rh_np = [r_.numpy().view(np.uint64) for r_ in rhs]

    def e2e_run(nthreads, steps):
        def worker(t):
            for _ in range(t, steps, nthreads):
                ctx.answer(0, qh_np[t], out=rh_np[t])
        ths = [threading.Thread(target=worker, args=(t,)) for t in range(nthreads)]
        t0 = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        return time.perf_counter() - t0

    e2e_run(S, 3 * S)
    if dist:
        dist.barrier()
    e2e_s = e2e_run(S, args.steps)
    e2e_serial_s = e2e_run(1, max(args.steps // 4, 10))
    for t in range(S):
        if not np.array_equal(rh_np[t], host_ref):
            raise RuntimeError("e2e response differs")

    if dist:
        t = torch.tensor([ms, e2e_s, ms_serial], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_s, ms_serial = float(t[0]), float(t[1]), float(t[2])

    clients16 = [cl]
    batched = run_batched(args, ctx, batches, nclients, rank, dist, torch, clients16) if batches else None
    rotating = bench_rotating(args, ctx, nclients, torch) if nclients >= 16 else None
    extra = {}
    if args.extras and world == 1 and len(clients16) >= 32:
        ctx64, clients64 = None, None
        try:
            ctx64, clients64, extra["db_1gb"] = bench_1gb(args, torch)
            extra["serving"] = bench_serving(args, ctx, clients16, ctx64, clients64)
        finally:
            if ctx64 is not None:
                ctx64.close()

    if rank == 0:
        db_bytes = r * N * N // 2 * 8
        scan_ms = phases[1] / max(answers, 1)
        peak, peak_src = read_peaks()
        achieved = db_bytes / (scan_ms * 1e-3) / 1e9
        out = {
            "metric": METRIC,
            "value": world * args.steps / (ms * 1e-3),
            "unit": "queries/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "u64",
            "data": "synthetic (seeded uniform canonical words; reference shapes)",
            "config": workload_config(args),
            "streams": S,
            "latency_ms": ms_serial / args.steps,
            "phases_ms_per_step": {"baby_steps": phases[0] / answers, "db_scan": scan_ms,
                                   "giant_steps": phases[2] / answers, "external_products": phases[3] / answers,
                                   "packing": phases[4] / answers},
            "roofline": {"bound": "hbm", "kernel": "k_scan", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_src,
                         "algorithmic_bytes_per_launch": db_bytes, "traffic": read_traffic(r),
                         "timed_in": "the latency run (one answer at a time): mean CUDA-event duration "
                                     "of the scan launch on the answer's stream"},
            "e2e": {"value": world * args.steps / e2e_s, "unit": "queries/s",
                    "h2d_bytes_per_step": 4 * N * 8, "d2h_bytes_per_step": 2 * N * 8,
                    "host_threads": S, "one_caller_queries_per_s": world * max(args.steps // 4, 10) / e2e_serial_s},
            # the whole answer against the bytes it must touch: the database,
            # one client's keys and the 8 MiB rotated-query buffer
            "answer_gbs": (db_bytes + ctx.lib.kspir_client_key_bytes(ctx.handle) + N * N1 * 2 * 8)
                          / (ms_serial / args.steps * 1e-3) / 1e9,
            "gpu_launches": int(launches) * world,
            "clocks": clocks.summary(),
        }
        if batched:
            out["batched"] = batched
        if rotating:
            out["single_rotating_clients"] = rotating
        out.update(extra)
        out["db_preprocess"] = prep
        out["client"] = bench_client(ctx)
        if world == 1 and not args.no_cpu_baseline:
            threads = host_threads()
            rate, kind, n, th = cpu_answer_rate(db, cl, perms, r, N1, args.cpu_seconds, threads)
            out["cpu_baseline"] = {"value": rate, "unit": "queries/s", "cores": th, "kind": kind, "host": host_model(),
                                   "sample": f"{n} full answers (r={r}, N1={N1}) in ~{args.cpu_seconds:.0f} s, "
                                             f"one independent query per thread"}
            # the reference's path is single-threaded: its latency on one core
            rate1, kind1, n1, _ = cpu_answer_rate(db, cl, perms, r, N1, min(3.0, args.cpu_seconds), 1)
            out["cpu_baseline_1core"] = {"ms_per_query": 1e3 / rate1, "kind": kind1,
                                         "sample": f"{n1} answers on one thread"}
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def run_batched(args, ctx, batches, nclients, rank, dist, torch, keep):
    """Batched answers of distinct clients at each batch size (the answer of
    every query equals its single-query answer; tests/test_gpu_batch.py).
    Client key sets 1..31 are appended to `keep` (for the serving run)."""
    import kspir_b200 as kb
    from kspir_b200 import synth
    r, N1 = args.r, args.N1
    for i in range(1, nclients):
        c = synth.gen_client(args.seed + 1000 * (rank + 1) + i, r, N1)
        ctx.upload_client(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
        if i < 32:
            keep.append(c)
    rng = np.random.default_rng(args.seed + 77 + rank)
    bmax = max(batches)
    qall = np.empty((bmax, 4 * N), np.uint64)
    qall[:, :2 * N] = rng.integers(0, kb.CRTMOD, size=(bmax, 2 * N), dtype=np.uint64)
    qall[:, 2 * N:] = rng.integers(0, kb.BSMOD, size=(bmax, 2 * N), dtype=np.uint64)
    dq = torch.from_numpy(qall.view(np.int64).copy()).cuda()
    dr = torch.empty((bmax, 2 * N), dtype=torch.int64, device="cuda")
    qh = torch.from_numpy(qall.view(np.int64).copy()).pin_memory()
    rh = torch.empty((bmax, 2 * N), dtype=torch.int64).pin_memory()
    stream = torch.cuda.Stream()
    db_words = r * N * N // 2
    int8_ops_per_query = db_words * 2 * 2 * 16 * 2
    peak8, peak8_src = read_int8_peak()
    res = {}
    for B in batches:
        cl = (np.arange(B, dtype=np.int32) % nclients)
        kind, tried = ctx.tune_batch(B)
        reps = max(5, min(args.steps, 2048 // B))

        def step():
            ctx.answer_batch_device(cl, dq.data_ptr(), dr.data_ptr(), stream.cuda_stream)
        for _ in range(max(args.warmup, 3)):
            step()
        torch.cuda.synchronize()
        ctx.timing_reset()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        nq, launches, tot, ph = ctx.timing_summary()
        ctx.sync()
        # end to end: pinned host queries in, responses out, through kspir_answer_batch
        qv = qh.numpy().view(np.uint64)[:B]
        rv = rh.numpy().view(np.uint64)[:B]
        ctx.answer_batch(cl, qv, out=rv)
        t0 = time.perf_counter()
        for _ in range(reps):
            ctx.answer_batch(cl, qv, out=rv)
        e2e_s = time.perf_counter() - t0
        if not np.array_equal(rv, dr.cpu().numpy().view(np.uint64)[:B]):
            raise RuntimeError(f"batch {B}: host-path and device-path responses differ")
        if dist:
            t = torch.tensor([ms, e2e_s], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms, e2e_s = float(t[0]), float(t[1])
        world = dist.get_world_size() if dist else 1
        scan_ms = ph[1] / reps
        entry = {
            "queries_per_s": world * B * reps / (ms * 1e-3),
            "ms_per_batch": ms / reps,
            "e2e_queries_per_s": world * B * reps / e2e_s,
            "scan_kind": kb.SCAN_NAMES[kind],
            "tuned_scan_ms": {kb.SCAN_NAMES[k]: v for k, v in tried.items()},
            "phases_ms_per_batch": {"baby_steps": ph[0] / reps, "db_scan": scan_ms, "giant_steps": ph[2] / reps,
                                    "external_products": ph[3] / reps, "packing": ph[4] / reps},
            "launches_per_batch": launches / reps,
        }
        if kind != kb.SCAN_CUDA:
            ach = int8_ops_per_query * B / (scan_ms * 1e-3) / 1e12
            entry["roofline_scan"] = {"bound": "tensor", "achieved": ach, "peak": peak8, "unit": "TOP/s (int8)",
                                      "frac": ach / peak8, "peak_source": peak8_src,
                                      "algorithmic_ops_per_launch": int8_ops_per_query * B,
                                      "note": "scan phase = query limb split + tcgen05 scan"}
        res[str(B)] = entry
    if "1" in res:
        base = res["1"]["queries_per_s"]
        for k, v in res.items():
            v["speedup_vs_batch1"] = v["queries_per_s"] / base
    return res


def bench_rotating(args, ctx, nclients, torch):
    """Single-query answers cycling through 16+ clients' keys (22 MiB each, so
    a client's keys are not left in the 126 MB L2 by its previous answer, as
    they are when one client asks repeatedly): device-timed."""
    rng = np.random.default_rng(args.seed + 5)
    q = np.empty(4 * N, np.uint64)
    q[:2 * N] = rng.integers(0, CRTMOD, 2 * N, dtype=np.uint64)
    q[2 * N:] = rng.integers(0, 16760833, 2 * N, dtype=np.uint64)
    dq = torch.from_numpy(q.view(np.int64).copy()).cuda()
    dr = torch.empty(2 * N, dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    n = max(args.steps, 2 * nclients)
    for i in range(nclients):
        ctx.answer_device(i, dq.data_ptr(), dr.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(n):
        ctx.answer_device(i % nclients, dq.data_ptr(), dr.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ctx.sync()
    ms = e0.elapsed_time(e1)
    return {"queries_per_s": n / (ms * 1e-3), "ms_per_answer": ms / n, "answers": n, "clients": nclients,
            "note": "one query at a time, client i % clients, keys of 22 MiB per client (not L2-resident)"}


def bench_1gb(args, torch):
    """The 1 GB database (131072 records x 8 KB: r = 64, N1 = 128, 4 GiB
    preprocessed): the raw database is drawn on the device and preprocessed
    there; single answers (device-timed) and a batch of 32 distinct clients."""
    import kspir_b200 as kb
    from kspir_b200 import synth
    r, N1, B = 64, args.N1, 32
    ctx = kb.Context(r, N1, max_clients=B, max_inflight=B)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(args.seed + 64)
    raw = torch.randint(0, 65537, (r * N * N // 2,), dtype=torch.int64, device="cuda", generator=gen)
    prep_ms = ctx.preprocess_db_device(raw.data_ptr(), raw.numel())
    del raw
    ctx.upload_perms(kb.permutation_matrix(N1))
    clients = []
    for i in range(B):
        c = synth.gen_client(args.seed + 6400 + i, r, N1)
        ctx.upload_client(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
        clients.append(c)
    qs = np.stack([c["query"] for c in clients])
    dq = torch.from_numpy(qs.view(np.int64).copy()).cuda()
    dr = torch.empty((B, 2 * N), dtype=torch.int64, device="cuda")
    stream = torch.cuda.Stream()
    for i in range(B):   # every client once (each key slot's first use) before timing
        ctx.answer_device(i, dq[i].data_ptr(), dr[0].data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    ctx.timing_reset()
    reps = 100   # enough answers that a host-side enqueue stall does not dominate the events
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(reps):
        ctx.answer_device(i % B, dq[i % B].data_ptr(), dr[0].data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms1 = e0.elapsed_time(e1) / reps
    n1, _, _, ph1 = ctx.timing_summary()
    ctx.sync()
    cl = np.arange(B, dtype=np.int32)
    kind, _ = ctx.tune_batch(B)
    for _ in range(3):
        ctx.answer_batch_device(cl, dq.data_ptr(), dr.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    ctx.timing_reset()
    reps_b = 5
    e0.record(stream)
    for _ in range(reps_b):
        ctx.answer_batch_device(cl, dq.data_ptr(), dr.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize()
    msb = e0.elapsed_time(e1) / reps_b
    nb, _, _, phb = ctx.timing_summary()
    ctx.sync()
    db_bytes = r * N * N // 2 * 8
    names = ("baby_steps", "db_scan", "giant_steps", "external_products", "packing")
    out = {"workload": f"1 GB database: 131072 x 8 KB records, r={r} N1={N1}, {db_bytes >> 30} GiB preprocessed",
           "preprocess_device_ms": prep_ms,
           "single": {"ms_per_answer": ms1, "queries_per_s": 1e3 / ms1,
                      "scan_gbs": db_bytes / (ph1[1] / n1 * 1e-3) / 1e9,
                      "phases_ms": {k: v / n1 for k, v in zip(names, ph1)},
                      "note": "device-timed, clients rotating over 32 key sets"},
           "batch32": {"ms_per_batch": msb, "queries_per_s": B / (msb * 1e-3), "scan_kind": kb.SCAN_NAMES[kind],
                       "phases_ms": {k: v / reps_b for k, v in zip(names, phb)}}}
    return ctx, clients, out


def bench_serving(args, ctx16, clients16, ctx64, clients64):
    """Serving with the 256 MB and the 1 GB databases resident together
    (kspir_server_*: continuous batching over lanes, client keys in device
    slots): seeded compound-Poisson arrivals (bursts of 1..64 queries, 3:1
    between the databases) at each offered rate; served queries/s and
    submit-to-response p50/p95/p99, beside the plain per-query path through
    the same servers (one request at a time)."""
    import types

    import kspir_b200 as kb
    from kspir_b200 import serving
    lanes = {16: (2, 64), 64: (1, 32)}
    deps = []
    for r, ctx, keys in ((16, ctx16, clients16), (64, ctx64, clients64)):
        nl, ls = lanes[r]
        srv = kb.Server(ctx, lanes=nl, lane_size=ls)
        n_cl = len(keys)
        for i, c in enumerate(keys):
            srv.register(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
        deps.append(types.SimpleNamespace(r=r, server=srv, clients=list(range(n_cl))))
    try:
        plain = {}
        q1 = serving.random_queries(np.random.default_rng(1), 1)[0]
        for d in deps:
            d.server.wait(d.server.submit(0, q1))
            d.server.reset_stats()
            for _ in range(20):
                d.server.wait(d.server.submit(0, q1))
            lat = d.server.latencies_us()
            plain[f"r{d.r}"] = {"p50_us": float(np.percentile(lat, 50)), "queries_per_s": 1e6 / float(np.mean(lat))}
        serving.drive(deps, [3, 1], serving.poisson_schedule(1000, 0.5, args.seed + 99, 64), args.seed + 98)
        rows = []
        for rate in [float(x) for x in args.serving_rates.split(",") if x.strip()]:
            for d in deps:
                d.server.reset_stats()
            wall, nq = serving.drive(deps, [3, 1], serving.poisson_schedule(rate, 1.5, args.seed + int(rate), 64),
                                     args.seed + 7 * int(rate))
            lat = np.concatenate([d.server.latencies_us() for d in deps])
            row = {"offered_qps": rate, "queries": nq, "served_qps": nq / wall,
                   "p50_ms": float(np.percentile(lat, 50)) / 1e3, "p95_ms": float(np.percentile(lat, 95)) / 1e3,
                   "p99_ms": float(np.percentile(lat, 99)) / 1e3, "per_db": {}}
            for d in deps:
                st = d.server.stats()
                row["per_db"][f"r{d.r}"] = {"served": st["served"], "mean_batch": st["mean_batch"],
                                            "p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3,
                                            "max_running_lanes": st["max_running_lanes"]}
            rows.append(row)
    finally:
        for d in deps:
            d.server.close()
    return {"workload": "256 MB (r=16) and 1 GB (r=64) databases resident together; 32 clients each; "
                        "lanes 2 x 64 (256 MB) and 1 x 32 (1 GB); bursts of 1..64, 3:1 between the databases",
            "plain_per_query": plain, "rates": rows}


def run_reference(args, rank, world):
    if rank != 0:
        return
    from kspir_b200 import synth
    from oracle import pyoracle as po
    r, N1 = args.r, args.N1
    db = synth.gen_db(args.seed, r, N1)
    cl = synth.gen_client(args.seed, r, N1)
    perms = po.permutation_matrix(N1)
    threads = host_threads()
    # each step: one answer per host thread, all at once
    per_step = 1
    for _ in range(args.warmup):
        cpu_answer_rate(db, cl, perms, r, N1, 0.0, threads)
    t0 = time.perf_counter()
    total = 0
    kind = "port"
    for _ in range(args.steps):
        _, kind, n, _ = cpu_answer_rate(db, cl, perms, r, N1, 0.0, threads)
        total += n
    dt = time.perf_counter() - t0
    value = total / dt
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
        "data": "synthetic (seeded uniform canonical words; reference shapes)", "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": kind,
                         "sample": f"{per_step} answer per thread per step on {threads} threads"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus if args.gpus == 1 else 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
