"""Single answers that overlap on the device: word-for-word parity.

kspir_answer may be called from several host threads at once (each call owns
one of eight workspace slots and its stream while it runs) and
kspir_answer_device rotates over the same slots on the caller's streams.
Every response must equal the one the same query gets alone, and the oracle's
(oracle/kspir_oracle.c); other entry points issued between them must be
ordered after the answers still running.  Integer work: the bar is bit-exact.
"""
import threading

import numpy as np
import pytest
import torch

import kspir_b200 as kb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
N = po.N
R, N1 = 2, 128


def random_queries(seed, n):
    rng = np.random.default_rng(seed)
    q = np.empty((n, 4 * N), dtype=np.uint64)
    q[:, :2 * N] = rng.integers(0, po.CRTMOD, size=(n, 2 * N), dtype=np.uint64)
    q[:, 2 * N:] = rng.integers(0, po.BSMOD, size=(n, 2 * N), dtype=np.uint64)
    return q


@pytest.fixture(scope="module")
def setup():
    db = po.gen_db(301, R, N1)
    clients = [po.gen_client(310 + i, R, N1) for i in range(3)]
    queries = random_queries(11, 6)
    ctx = kb.Context(R, N1, max_clients=3, max_inflight=8)
    ctx.upload_db(db)
    ctx.upload_perms(clients[0]["perms"])
    for i, c in enumerate(clients):
        ctx.upload_client(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
    # each (client, query) pair answered alone, one call at a time
    alone = {(i % 3, i): ctx.answer(i % 3, queries[i]) for i in range(len(queries))}
    yield ctx, db, clients, queries, alone
    ctx.close()


def test_alone_matches_oracle(setup):
    ctx, db, clients, queries, alone = setup
    for i in (0, 4):
        want = po.answer(db, R, N1, dict(clients[i % 3], query=queries[i]))
        assert (alone[(i % 3, i)] == want).all(), f"query {i}"


def test_host_threads_overlap(setup):
    ctx, db, clients, queries, alone = setup
    errors = []

    def worker(t):
        try:
            for k in range(12):
                i = (t + k) % len(queries)
                got = ctx.answer(i % 3, queries[i])
                if not (got == alone[(i % 3, i)]).all():
                    errors.append(f"thread {t}, answer {k}, query {i}")
        except Exception as e:   # noqa: BLE001 -- reported below
            errors.append(f"thread {t}: {e!r}")

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(6)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors


def test_bad_query_in_one_thread_leaves_the_others_exact(setup):
    ctx, db, clients, queries, alone = setup
    bad = queries[0].copy()
    bad[5] = po.CRTMOD   # not canonical
    results, errors = {}, []

    def good(t):
        try:
            for k in range(6):
                i = (t + k) % len(queries)
                results[(t, k)] = (i, ctx.answer(i % 3, queries[i]))
        except Exception as e:   # noqa: BLE001
            errors.append(repr(e))

    def wrong():
        for _ in range(3):
            with pytest.raises(kb.KspirError):
                ctx.answer(0, bad)

    threads = [threading.Thread(target=good, args=(t,)) for t in range(3)] + [threading.Thread(target=wrong)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    for (t, k), (i, got) in results.items():
        assert (got == alone[(i % 3, i)]).all(), f"thread {t}, answer {k}"


def test_device_streams_overlap_and_batches_between(setup):
    ctx, db, clients, queries, alone = setup
    n = len(queries)
    dq = torch.from_numpy(queries.view(np.int64).copy()).cuda()
    streams = [torch.cuda.Stream() for _ in range(3)]
    dr = torch.zeros((3 * n, 2 * N), dtype=torch.int64, device="cuda")
    db_resp = torch.zeros((n, 2 * N), dtype=torch.int64, device="cuda")
    cl = np.array([i % 3 for i in range(n)], dtype=np.int32)
    for k in range(3 * n):
        i = k % n
        if k == n:   # a batch on a fourth stream, while singles are in flight
            side = torch.cuda.Stream()
            ctx.answer_batch_device(cl, dq.data_ptr(), db_resp.data_ptr(), side.cuda_stream)
        ctx.answer_device(i % 3, dq[i].data_ptr(), dr[k].data_ptr(), streams[k % 3].cuda_stream)
    ctx.sync()
    got = dr.cpu().numpy().view(np.uint64)
    for k in range(3 * n):
        i = k % n
        assert (got[k] == alone[(i % 3, i)]).all(), f"device answer {k} (query {i})"
    gb = db_resp.cpu().numpy().view(np.uint64)
    for i in range(n):
        assert (gb[i] == alone[(i % 3, i)]).all(), f"batched query {i}"
    # a host batch right after: ordered behind the device singles
    for k in range(n):
        ctx.answer_device(k % 3, dq[k].data_ptr(), dr[k].data_ptr(), streams[k % 3].cuda_stream)
    hb = ctx.answer_batch(cl, queries)
    ctx.sync()
    for i in range(n):
        assert (hb[i] == alone[(i % 3, i)]).all(), f"host batch query {i}"
        assert (dr[i].cpu().numpy().view(np.uint64) == alone[(i % 3, i)]).all(), f"device answer {i}"
