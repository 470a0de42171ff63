"""The serving loop (kspir_server_*): continuous batching with overlapping
lanes and client keys admitted within an HBM budget.  Every response must be
identical to the same query answered alone (which the parity tests pin to the
reference); integer work, so identical means word for word."""
import threading
import time

import numpy as np
import pytest

import kspir_b200 as kb
from kspir_b200 import serving
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
N = po.N


def test_serving_in_mix_equals_alone_with_key_eviction():
    r, N1, n_clients = 4, 128, 6
    db = po.gen_db(201, r, N1)
    keys = [po.gen_client(210 + i, r, N1) for i in range(n_clients)]
    rng = np.random.default_rng(3)
    queries = serving.random_queries(rng, 90)
    owner = rng.integers(0, n_clients, size=len(queries))
    # two lanes of 32 queries; key slots for 3 of the 6 clients (evictions)
    ctx = kb.Context(r, N1, max_clients=3, max_inflight=64)
    ctx.upload_db(db)
    ctx.upload_perms(keys[0]["perms"])
    srv = kb.Server(ctx, lanes=2, lane_size=32, key_budget_bytes=3 * ctx.lib.kspir_client_key_bytes(ctx.handle))
    for i, c in enumerate(keys):
        srv.register(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
    outs = [np.zeros(2 * N, np.uint64) for _ in queries]
    tickets = [None] * len(queries)

    def submitter():   # bursts of uneven size with gaps, so batches overlap and vary
        i = 0
        while i < len(queries):
            g = int(rng.integers(1, 24))
            for j in range(i, min(i + g, len(queries))):
                tickets[j] = srv.submit(int(owner[j]), queries[j], out=outs[j])
            i += g
            time.sleep(0.002)

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    for t in tickets:
        srv.wait(t)
    st = srv.stats()
    srv.close()
    assert st["served"] == len(queries)
    assert st["key_slots"] == 3
    assert st["key_uploads"] > n_clients - 1 and st["evictions"] > 0
    assert st["batches"] < len(queries)          # requests were batched
    # the same queries answered one at a time
    ctx2 = kb.Context(r, N1)
    ctx2.upload_db(db)
    ctx2.upload_perms(keys[0]["perms"])
    for cl in range(n_clients):
        c = keys[cl]
        ctx2.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        for j in np.flatnonzero(owner == cl):
            assert np.array_equal(outs[j], ctx2.answer(0, queries[j])), f"request {j}"
    # and one of them against the oracle
    assert np.array_equal(outs[0], po.answer(db, r, N1, dict(keys[owner[0]], query=queries[0])))
    ctx2.close()
    ctx.close()


def test_serving_lanes_overlap_under_load():
    r, N1 = 4, 128
    db = po.gen_db(221, r, N1)
    keys = [po.gen_client(222, r, N1)]
    ctx = kb.Context(r, N1, max_clients=1, max_inflight=64)
    ctx.upload_db(db)
    ctx.upload_perms(keys[0]["perms"])
    with kb.Server(ctx, lanes=2, lane_size=32) as srv:
        srv.register(0, keys[0]["baby"], keys[0]["giant"], keys[0]["packing"], keys[0]["rgsw"])
        q = serving.random_queries(np.random.default_rng(4), 1)[0]
        ts = [srv.submit(0, q) for _ in range(200)]
        res = [srv.wait(t) for t in ts]
        st = srv.stats()
    assert st["max_running_lanes"] == 2, st
    assert st["served"] == 200 and st["p99_us"] >= st["p50_us"] > 0
    ref = res[0]
    assert all(np.array_equal(x, ref) for x in res)
    ctx.upload_client(0, keys[0]["baby"], keys[0]["giant"], keys[0]["packing"], keys[0]["rgsw"])
    assert np.array_equal(ref, ctx.answer(0, q))
    ctx.close()


def test_serving_rejects_unknown_client_and_bad_query():
    r, N1 = 2, 128
    keys = po.gen_client(231, r, N1)
    ctx = kb.Context(r, N1, max_clients=1, max_inflight=32)
    ctx.upload_db(po.gen_db(231, r, N1))
    ctx.upload_perms(keys["perms"])
    with kb.Server(ctx, lanes=1, lane_size=8) as srv:
        with pytest.raises(kb.KspirError) as ei:
            srv.submit(5, keys["query"])
        assert ei.value.code == kb.native.ERR_NOT_READY
        srv.register(0, keys["baby"], keys["giant"], keys["packing"], keys["rgsw"])
        bad = keys["query"].copy()
        bad[0] = po.CRTMOD
        with pytest.raises(kb.KspirError) as ei:
            srv.submit(0, bad)
        assert ei.value.code == kb.native.ERR_INVALID_ARG
        out = srv.wait(srv.submit(0, keys["query"]))
    assert np.array_equal(out, po.answer(po.gen_db(231, r, N1), r, N1, keys))
    ctx.close()


def _rolled_db(seed, r, N1):
    """r sub-databases: one seeded sub-database, rotated by a different word
    count in each (cheap to build at r = 64, every word canonical)."""
    base = po.gen_db(seed, 1, N1)
    num = base.size
    out = np.empty(r * num, np.uint64)
    for k in range(r):
        out[k * num:(k + 1) * num] = np.roll(base, 4099 * k + 17)
    return out


def test_serving_256mb_and_1gb_resident_together():
    # the serving configuration of the benchmark: the 256 MB (r = 16) and the
    # 1 GB (r = 64) databases resident at once, each behind its own server,
    # lanes of 128 queries, bursts of 1..128 arriving while other batches run,
    # fewer key slots than clients (evictions); every response must equal the
    # same query answered alone
    N1 = 128
    spec = {16: dict(lanes=2, lane_size=128, slots=3, clients=5),
            64: dict(lanes=1, lane_size=128, slots=2, clients=3)}
    deps = {}
    for r, sp in spec.items():
        db = _rolled_db(400 + r, r, N1)
        keys = [po.gen_client(410 + 10 * r + i, r, N1) for i in range(sp["clients"])]
        ctx = kb.Context(r, N1, max_clients=sp["slots"], max_inflight=128 * (sp["lanes"] - 1) + sp["lane_size"])
        ctx.upload_db(db)
        ctx.upload_perms(keys[0]["perms"])
        srv = kb.Server(ctx, lanes=sp["lanes"], lane_size=sp["lane_size"],
                        key_budget_bytes=sp["slots"] * ctx.lib.kspir_client_key_bytes(ctx.handle))
        for i, c in enumerate(keys):
            srv.register(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
        deps[r] = dict(db=db, keys=keys, ctx=ctx, srv=srv, reqs=[])
    rng = np.random.default_rng(6)
    pool = serving.random_queries(rng, 64)
    total = 0
    while total < 420:
        r = 16 if rng.random() < 0.7 else 64
        d = deps[r]
        for _ in range(int(rng.integers(1, 129))):
            cl, qi = int(rng.integers(0, spec[r]["clients"])), int(rng.integers(0, len(pool)))
            out = np.zeros(2 * N, np.uint64)
            d["reqs"].append((cl, qi, out, d["srv"].submit(cl, pool[qi], out=out)))
            total += 1
        time.sleep(0.001 * int(rng.integers(0, 6)))
    stats = {}
    for r, d in deps.items():
        for _, _, _, t in d["reqs"]:
            d["srv"].wait(t)
        stats[r] = d["srv"].stats()
        d["srv"].close()
    for r, d in deps.items():
        st = stats[r]
        assert st["served"] == len(d["reqs"]), (r, st)
        assert st["batches"] < st["served"], (r, st)               # arrivals were batched
        assert st["evictions"] > 0 and st["key_uploads"] > spec[r]["clients"] - 1, (r, st)
        # the same queries answered alone, client by client, in the same context
        ctx = d["ctx"]
        for cl in range(spec[r]["clients"]):
            c = d["keys"][cl]
            ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
            alone = {}
            for j, (rc, qi, out, _) in enumerate(d["reqs"]):
                if rc != cl:
                    continue
                if qi not in alone:
                    alone[qi] = ctx.answer(0, pool[qi])
                assert np.array_equal(out, alone[qi]), f"r={r} request {j}"
        cl, qi, out, _ = d["reqs"][0]
        want = po.answer(d["db"], r, N1, dict(d["keys"][cl], query=pool[qi]))
        assert np.array_equal(out, want), f"r={r}: first request against the oracle"
        ctx.close()
