"""Small, seeded answer workloads to run under a profiler.

Each case builds a context with a synthetic database and client keys of the
reference's shapes (kspir_b200.synth), answers a few times and prints the
last answer's device time and phases.  They are sized for kernel captures:
the database and keys are larger than L2 where the case is meant to show DRAM
traffic, but the whole case holds a few GB at most.

    python -m kspir_b200.profile_cases batch --r 2 --batch 64 --clients 8
    python -m kspir_b200.profile_cases single --r 16 --answers 4
"""
from __future__ import annotations

import argparse

import numpy as np

import kspir_b200 as kb
from kspir_b200 import synth

N = kb.N


def random_queries(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    q = np.empty((n, 4 * N), np.uint64)
    q[:, :2 * N] = rng.integers(0, kb.CRTMOD, size=(n, 2 * N), dtype=np.uint64)
    q[:, 2 * N:] = rng.integers(0, kb.BSMOD, size=(n, 2 * N), dtype=np.uint64)
    return q


def make_context(r: int, N1: int, clients: int, inflight: int) -> kb.Context:
    ctx = kb.Context(r, N1, max_clients=clients, max_inflight=inflight)
    ctx.upload_db(synth.gen_db(1, r, N1))
    ctx.upload_perms(kb.permutation_matrix(N1))
    for i in range(clients):
        c = synth.gen_client(10 + i, r, N1)
        ctx.upload_client(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
    return ctx


def batch(args) -> None:
    """A batch of `batch` queries of `clients` clients (query i of client
    i % clients), answered `answers` times with the given scan kind."""
    ctx = make_context(args.r, args.N1, args.clients, args.batch)
    q = random_queries(3, args.batch)
    cl = np.arange(args.batch, dtype=np.int32) % args.clients
    ctx.set_scan_kind(args.batch, args.kind)
    for _ in range(args.answers):
        ctx.answer_batch(cl, q)
    tot, ph = ctx.last_timing()
    print("batch", args.batch, "ms", round(tot, 3), [round(x, 3) for x in ph])
    ctx.close()


def single(args) -> None:
    """`answers` single answers of client 0's query, one at a time."""
    ctx = make_context(args.r, args.N1, 1, 1)
    q = random_queries(3, 1)[0]
    for _ in range(args.answers):
        ctx.answer(0, q)
    tot, ph = ctx.last_timing()
    print("single ms", round(tot, 3), [round(x, 3) for x in ph])
    ctx.close()


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("case", choices=["batch", "single"])
    ap.add_argument("--r", type=int, default=2)
    ap.add_argument("--N1", type=int, default=128)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--clients", type=int, default=8)
    ap.add_argument("--answers", type=int, default=2)
    ap.add_argument("--kind", type=int, default=kb.SCAN_MMA32, help="scan kind of the batch (kspir_b200.SCAN_*)")
    args = ap.parse_args()
    {"batch": batch, "single": single}[args.case](args)


if __name__ == "__main__":
    main()
