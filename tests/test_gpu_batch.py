"""Batched answers (kspir_answer_batch): word-for-word parity per query.

Every query of a batch must get exactly the response it gets alone, and that
response must equal the oracle's (oracle/kspir_oracle.c, pinned to the
reference in test_oracle.py).  The database scan of a batch runs either on
the CUDA cores (one database pass per query) or on the tensor cores
(tcgen05 kind::i8, 8-bit limbs, one database pass per batch) with query tiles
of 4..32; every variant is checked.  Integer work: the bar is bit-exact.
"""
import numpy as np
import pytest

import kspir_b200 as kb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
N = po.N
KINDS = [kb.SCAN_CUDA, kb.SCAN_MMA4, kb.SCAN_MMA8, kb.SCAN_MMA16, kb.SCAN_MMA32]


def random_queries(seed, n):
    rng = np.random.default_rng(seed)
    q = np.empty((n, 4 * N), dtype=np.uint64)
    q[:, :2 * N] = rng.integers(0, po.CRTMOD, size=(n, 2 * N), dtype=np.uint64)
    q[:, 2 * N:] = rng.integers(0, po.BSMOD, size=(n, 2 * N), dtype=np.uint64)
    return q


def make_ctx(r, N1, db, clients, max_inflight):
    ctx = kb.Context(r, N1, max_clients=len(clients), max_inflight=max_inflight)
    ctx.upload_db(db)
    ctx.upload_perms(clients[0]["perms"])
    for i, c in enumerate(clients):
        ctx.upload_client(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
    return ctx


@pytest.mark.parametrize("kind", KINDS, ids=lambda k: kb.SCAN_NAMES[k])
def test_batch_every_scan_variant_matches_oracle(kind):
    r, N1, n = 4, 128, 6
    db = po.gen_db(101, r, N1)
    clients = [po.gen_client(110 + i, r, N1) for i in range(3)]
    cl = np.array([i % 3 for i in range(n)], dtype=np.int32)
    queries = random_queries(7, n)
    with make_ctx(r, N1, db, clients, max_inflight=8) as ctx:
        ctx.set_scan_kind(n, kind)
        assert ctx.scan_kind(n) == kind
        got = ctx.answer_batch(cl, queries)
        for i in range(n):
            c = dict(clients[cl[i]], query=queries[i])
            want, bsgs, _ = po.answer(db, r, N1, c, with_stages=True)
            assert (ctx.fetch_stage(kb.STAGE_RESULT, slot=i) == bsgs).all(), f"query {i}: first dimension"
            assert (got[i] == want).all(), f"query {i}: response"


def test_batch_scan_stage_matches_oracle_scan():
    # the tensor-core scan output of every query equals the oracle's scan of its cipherbuf
    r, N1, n = 2, 128, 5
    db = po.gen_db(121, r, N1)
    clients = [po.gen_client(122, r, N1)]
    queries = random_queries(8, n)
    with make_ctx(r, N1, db, clients, max_inflight=n) as ctx:
        ctx.set_scan_kind(n, kb.SCAN_MMA4)
        ctx.answer_batch(np.zeros(n, np.int32), queries)
        num = N * N // 2
        for i in range(n):
            cb = ctx.fetch_stage(kb.STAGE_CIPHERBUF, slot=i)
            want = np.concatenate([po.scan(db[k * num:(k + 1) * num], cb, N1) for k in range(r)])
            assert (ctx.fetch_stage(kb.STAGE_SCAN, slot=i) == want).all(), f"query {i}"


def test_batch_database_extremes():
    # database halves at 2^32 - 1: the 64-bit sums wrap exactly like the reference's
    r, N1, n = 2, 128, 3
    clients = [po.gen_client(131, r, N1)]
    queries = random_queries(9, n)
    db = np.full(r * N * N // 2, np.uint64(0xFFFFFFFFFFFFFFFF))
    with make_ctx(r, N1, db, clients, max_inflight=4) as ctx:
        for kind in (kb.SCAN_MMA4, kb.SCAN_MMA32):
            ctx.set_scan_kind(n, kind)
            got = ctx.answer_batch(np.zeros(n, np.int32), queries)
            for i in range(n):
                assert (got[i] == po.answer(db, r, N1, dict(clients[0], query=queries[i]))).all()


def test_batch_full_size_alone_equals_in_batch():
    # 256 MB-record database (r = 16): 64 queries of 8 clients answered in one
    # batch equal the same queries answered one at a time; two of them are
    # also checked against the oracle
    r, N1, n = 16, 128, 64
    db = po.gen_db(141, r, N1)
    clients = [po.gen_client(150 + i, r, N1) for i in range(8)]
    cl = np.array([(5 * i) % 8 for i in range(n)], dtype=np.int32)
    queries = random_queries(10, n)
    with make_ctx(r, N1, db, clients, max_inflight=n) as ctx:
        kind, times = ctx.tune_batch(n)
        assert kind in times
        got = ctx.answer_batch(cl, queries)
        for i in range(n):
            alone = ctx.answer(int(cl[i]), queries[i])
            assert (got[i] == alone).all(), f"query {i}"
        for i in (0, 37):
            assert (got[i] == po.answer(db, r, N1, dict(clients[cl[i]], query=queries[i]))).all()
        # a partial batch after a full one (uneven counts reuse the workspaces)
        got5 = ctx.answer_batch(cl[:5], queries[-5:])
        for i in range(5):
            assert (got5[i] == ctx.answer(int(cl[i]), queries[-5 + i])).all()


def test_batch_128_full_size():
    # the largest batch of the benchmark: 128 queries of 8 distinct clients at
    # r = 16 (256 MB of records), slots 0..127 of one launch, with the scan
    # variant the autotuner picks and with tcgen05 query tiles of 32 forced;
    # every query equals its single answer, four of them the oracle
    r, N1, n = 16, 128, 128
    db = po.gen_db(181, r, N1)
    clients = [po.gen_client(190 + i, r, N1) for i in range(8)]
    cl = np.array([(3 * i + i // 16) % 8 for i in range(n)], dtype=np.int32)
    queries = random_queries(18, n)
    with make_ctx(r, N1, db, clients, max_inflight=n) as ctx:
        alone = np.stack([ctx.answer(int(cl[i]), queries[i]) for i in range(n)])
        tuned, _ = ctx.tune_batch(n)
        for kind in dict.fromkeys((tuned, kb.SCAN_MMA32)):
            ctx.set_scan_kind(n, kind)
            got = ctx.answer_batch(cl, queries)
            bad = [i for i in range(n) if not np.array_equal(got[i], alone[i])]
            assert not bad, f"{kb.SCAN_NAMES[kind]}: queries {bad[:8]} differ from their single answers"
        for i in (0, 63, 64, 127):
            want = po.answer(db, r, N1, dict(clients[cl[i]], query=queries[i]))
            assert np.array_equal(alone[i], want), f"query {i} against the oracle"


def test_batch_rejects_bad_input():
    r, N1 = 2, 128
    clients = [po.gen_client(161, r, N1)]
    db = po.gen_db(161, r, N1)
    with make_ctx(r, N1, db, clients, max_inflight=4) as ctx:
        q = random_queries(11, 2)
        with pytest.raises(kb.KspirError) as ei:
            ctx.answer_batch(np.array([0, 1], np.int32), q)    # client slot 1 does not exist
        assert ei.value.code == -1
        with pytest.raises(kb.KspirError):
            ctx.answer_batch(np.zeros(5, np.int32), random_queries(12, 5))   # more than max_inflight
        bad = q.copy()
        bad[1, 3] = po.CRTMOD
        with pytest.raises(kb.KspirError) as ei:
            ctx.answer_batch(np.zeros(2, np.int32), bad)
        assert ei.value.code == -1
        # the context still answers afterwards
        got = ctx.answer_batch(np.zeros(2, np.int32), q)
        assert (got[1] == po.answer(db, r, N1, dict(clients[0], query=q[1]))).all()


@pytest.mark.parametrize("r,N1", [(1, 64), (4, 256), (2, 64)])
def test_batch_other_shapes_match_oracle(r, N1):
    # N1 != 128 batches run the CUDA-core scan (the tensor-core scan needs
    # N1 = 128) with the batched baby-step shape; r = 1 has no packing level
    n = 3
    db = po.gen_db(170 + r + N1, r, N1)
    clients = [po.gen_client(171 + i + N1, r, N1) for i in range(2)]
    cl = np.array([0, 1, 0], dtype=np.int32)
    queries = random_queries(13 + N1, n)
    with make_ctx(r, N1, db, clients, max_inflight=4) as ctx:
        got = ctx.answer_batch(cl, queries)
        for i in range(n):
            want = po.answer(db, r, N1, dict(clients[cl[i]], query=queries[i]))
            assert (got[i] == want).all(), f"query {i}"
            assert (ctx.answer(int(cl[i]), queries[i]) == want).all()
