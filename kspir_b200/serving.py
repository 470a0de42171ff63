"""Serving-loop load driver: seeded Poisson arrivals against one or more
resident databases, each behind a :class:`kspir_b200.Server` (continuous
batching, client keys admitted by HBM budget).

Arrivals are a compound Poisson process: groups of 1..max_group queries
(uniform) arrive at exponential gaps, scaled so the offered rate is `rate`
queries/s.  Each query picks a database at random (weights), a client of that
database at random, and a fresh seeded query.  Latency is the server's
submit-to-response time; percentiles are over every request of the run.

Run ``python -m kspir_b200.serving`` on a GPU for the table of both databases
(256 MB: r = 16 and 1 GB: r = 64, N1 = 128) resident together at offered rates
of 100..5000 queries/s.
"""
from __future__ import annotations

import argparse
import json
import threading
import time

import numpy as np

from . import native, synth
from .native import N, Context, Server


def poisson_schedule(rate: float, duration: float, seed: int, max_group: int = 128):
    """[(arrival time s, group size)] with mean rate `rate` queries/s."""
    rng = np.random.default_rng(seed)
    mean_group = (1 + max_group) / 2
    gap = mean_group / rate
    t, out = 0.0, []
    while True:
        t += rng.exponential(gap)
        if t >= duration:
            return out
        out.append((t, int(rng.integers(1, max_group + 1))))


def random_queries(rng, n):
    q = np.empty((n, 4 * N), np.uint64)
    q[:, :2 * N] = rng.integers(0, native.CRTMOD, size=(n, 2 * N), dtype=np.uint64)
    q[:, 2 * N:] = rng.integers(0, native.BSMOD, size=(n, 2 * N), dtype=np.uint64)
    return q


class Deployment:
    """One resident database with its server and registered clients."""

    def __init__(self, r, N1, n_clients, lanes, lane_size, key_budget_slots, seed, device=0):
        self.r, self.N1 = r, N1
        stride = (lane_size + 31) // 32 * 32
        self.ctx = Context(r, N1, device=device, max_clients=key_budget_slots,
                           max_inflight=stride * (lanes - 1) + lane_size)
        self.ctx.upload_db(synth.gen_db(seed, r, N1))
        self.ctx.upload_perms(native.permutation_matrix(N1))
        self.server = Server(self.ctx, lanes=lanes, lane_size=lane_size,
                             key_budget_bytes=key_budget_slots * self.ctx.lib.kspir_client_key_bytes(self.ctx.handle))
        self.clients = []
        for i in range(n_clients):
            c = synth.gen_client(seed * 1000 + i, r, N1)
            self.server.register(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
            self.clients.append(i)

    def close(self):
        self.server.close()
        self.ctx.close()


def drive(deps, weights, schedule, seed):
    """Submits the schedule (real time) and waits for every response; returns
    (wall seconds, number of queries)."""
    rng = np.random.default_rng(seed)
    w = np.asarray(weights, float) / np.sum(weights)
    tickets = []
    lock = threading.Lock()
    done = threading.Event()
    pool = random_queries(rng, 256)

    def waiter():
        i = 0
        while True:
            with lock:
                pending = tickets[i:]
            if not pending and done.is_set():
                return
            for dep, t in pending:
                dep.server.wait(t)
                i += 1
            if not pending:
                time.sleep(0.0005)

    th = threading.Thread(target=waiter)
    th.start()
    t0 = time.perf_counter()
    nq = 0
    for at, g in schedule:
        now = time.perf_counter() - t0
        if at > now:
            time.sleep(at - now)
        for _ in range(g):
            dep = deps[int(rng.choice(len(deps), p=w))]
            client = int(rng.integers(0, len(dep.clients)))
            q = pool[int(rng.integers(0, len(pool)))]
            t = dep.server.submit(client, q)
            with lock:
                tickets.append((dep, t))
            nq += 1
    done.set()
    th.join()
    return time.perf_counter() - t0, nq


def run(rates, duration, seed, dbs, lanes, lane_size, clients, key_slots, weights, max_group):
    deps = [Deployment(r, 128, clients, lanes, lane_size, key_slots, seed + i) for i, r in enumerate(dbs)]
    try:
        # plain per-query GPU path of each database (for the comparison)
        plain = {}
        for d in deps:
            sched = [(0.0, 1)] * 20
            for dep in deps:
                dep.server.reset_stats()
            for at, g in sched:     # one at a time: each waits for the previous
                t = d.server.submit(0, random_queries(np.random.default_rng(1), 1)[0])
                d.server.wait(t)
            lat = d.server.latencies_us()
            plain[d.r] = {"p50_us": float(np.percentile(lat[5:], 50)), "queries_per_s": 1e6 / float(np.mean(lat[5:]))}
        # warm-up: every batch size's launch graphs
        drive(deps, weights, poisson_schedule(2000, 1.0, seed + 99, max_group), seed + 98)
        rows = []
        for rate in rates:
            for dep in deps:
                dep.server.reset_stats()
            wall, nq = drive(deps, weights, poisson_schedule(rate, duration, seed + int(rate), max_group),
                             seed + 7 * int(rate))
            lat = np.concatenate([d.server.latencies_us() for d in deps])
            row = {"offered_qps": rate, "queries": nq, "achieved_qps": nq / wall,
                   "p50_us": float(np.percentile(lat, 50)), "p95_us": float(np.percentile(lat, 95)),
                   "p99_us": float(np.percentile(lat, 99)), "per_db": {}}
            for d in deps:
                st = d.server.stats()
                row["per_db"][f"r{d.r}"] = {k: st[k] for k in ("served", "batches", "mean_batch", "p50_us", "p95_us",
                                                                "p99_us", "key_uploads", "evictions",
                                                                "max_running_lanes")}
            rows.append(row)
            print(json.dumps(row), flush=True)
        return {"plain_per_query": plain, "rows": rows}
    finally:
        for d in deps:
            d.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--rates", default="100,500,1000,2000,5000")
    ap.add_argument("--duration", type=float, default=3.0)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--dbs", default="16,64", help="packing numbers r of the resident databases (16: 256 MB, 64: 1 GB)")
    ap.add_argument("--weights", default="3,1", help="share of queries per database")
    ap.add_argument("--lanes", type=int, default=2)
    ap.add_argument("--lane-size", type=int, default=64)
    ap.add_argument("--clients", type=int, default=48, help="registered clients per database")
    ap.add_argument("--key-slots", type=int, default=48,
                    help="device key slots per database (HBM budget); below --clients, keys are evicted and re-admitted")
    ap.add_argument("--max-group", type=int, default=128)
    a = ap.parse_args()
    res = run([float(x) for x in a.rates.split(",")], a.duration, a.seed, [int(x) for x in a.dbs.split(",")],
              a.lanes, a.lane_size, a.clients, a.key_slots, [float(x) for x in a.weights.split(",")], a.max_group)
    print(json.dumps({"serving": res}), flush=True)


if __name__ == "__main__":
    main()
