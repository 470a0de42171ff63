"""The 1 GB database (131072 records x 8 KB: r = 64 sub-databases, N1 = 128,
N2 = 16, 4 GiB preprocessed; reference tests/test-pir.cpp:15 with r = 64),
single query and a batch of 32.  Integer work: bit-exact."""
import ctypes

import numpy as np
import pytest

import kspir_b200 as kb
from kspir_b200 import serving
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
N = po.N
R, N1 = 64, 128


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref not present")
def test_1gb_reference_known_answer():
    # the reference's own test-pir flow at r = 64 (keys, query and database
    # from its key generation after srand(7)); our response must equal the
    # reference's answer word for word, and then decrypts the same way
    L = po.ref()
    L.ref_pir_setup(7, R, N1)
    sz = po.sizes(R, N1)
    db = np.zeros(sz["db"], np.uint64)
    c = {k: np.zeros(sz[k], np.uint64) for k in ("query", "baby", "giant", "packing", "rgsw")}
    c["perms"] = np.zeros(sz["perms"], np.int32)
    L.ref_pir_get_inputs(*[po._p(x) for x in (db, c["query"], c["baby"], c["giant"], c["packing"], c["rgsw"],
                                                c["perms"])])
    with kb.Context(R, N1) as ctx:
        ctx.upload_db(db)
        ctx.upload_perms(c["perms"])
        ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        got = ctx.answer(0, c["query"])
    want = np.zeros(2 * N, np.uint64)
    secs = ctypes.c_double()
    L.ref_answer(po._p(db), R, N1, po._p(c["query"]), po._p(c["baby"]), po._p(c["giant"]), po._p(c["packing"]),
                 po._p(c["rgsw"]), po._p(c["perms"]), po._p(want), None, None, ctypes.byref(secs))
    assert np.array_equal(got, want)
    msg = np.zeros(N, np.uint64)
    L.ref_pir_decrypt(po._p(got), po._p(msg))
    assert (msg == np.arange(1, N + 1)).all(), "the 1 GB answer decrypts to the planted record"


def test_1gb_batch32_equals_single_and_oracle():
    db = po.gen_db(301, R, N1)
    keys = [po.gen_client(310 + i, R, N1) for i in range(4)]
    queries = serving.random_queries(np.random.default_rng(5), 32)
    cl = np.arange(32, dtype=np.int32) % 4
    with kb.Context(R, N1, max_clients=4, max_inflight=32) as ctx:
        ctx.upload_db(db)
        ctx.upload_perms(keys[0]["perms"])
        for i, c in enumerate(keys):
            ctx.upload_client(i, c["baby"], c["giant"], c["packing"], c["rgsw"])
        kind, _ = ctx.tune_batch(32)
        batch = ctx.answer_batch(cl, queries)
        for i in range(32):
            assert np.array_equal(batch[i], ctx.answer(int(cl[i]), queries[i])), f"query {i}"
    assert np.array_equal(batch[3], po.answer(db, R, N1, dict(keys[3], query=queries[3])))
    del kind
