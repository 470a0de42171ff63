"""Word-for-word parity of the CUDA path with the reference, through the C ABI.

The checker is the CPU oracle (oracle/kspir_oracle.c, itself pinned to the
reference in test_oracle.py) on the same seeded inputs, plus the committed
golden digests that the reference produced (tests/golden/golden.json).
Integer work: the bar is bit-exact equality of every word.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import kspir_b200 as kb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
N = po.N
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make_ctx(r, N1, db, c, max_clients=1):
    ctx = kb.Context(r, N1, max_clients=max_clients)
    ctx.upload_db(db)
    ctx.upload_perms(c["perms"])
    ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
    return ctx


def oracle_stages(db, r, N1, c):
    res, q, cb = po.matrix_vector_mul(db, r, N1, c, want_cipherbuf=True)
    num = N * N // 2
    scan = np.concatenate([po.scan(db[k * num:(k + 1) * num], cb, N1) for k in range(r)])
    return dict(result=res, query=q, cipherbuf=cb, scan=scan)


@pytest.mark.parametrize("case", GOLDEN["answer"], ids=lambda c: f"r{c['r']}_N1{c['N1']}_s{c['seed']}")
def test_answer_matches_reference_golden_and_oracle(case):
    r, N1, seed = case["r"], case["N1"], case["seed"]
    db = po.gen_db(seed, r, N1)
    c = po.gen_client(seed, r, N1)
    with make_ctx(r, N1, db, c) as ctx:
        resp = ctx.answer(0, c["query"])
        st = oracle_stages(db, r, N1, c)
        assert (ctx.fetch_stage(kb.STAGE_CIPHERBUF) == st["cipherbuf"]).all(), "baby steps / reorient"
        assert (ctx.fetch_stage(kb.STAGE_SCAN) == st["scan"]).all(), "database scan"
        assert (ctx.fetch_stage(kb.STAGE_RESULT) == st["result"]).all(), "giant steps"
        assert sha(ctx.fetch_stage(kb.STAGE_RESULT)) == case["bsgs_sha"]
        assert sha(resp) == case["response_sha"], "response"
        assert (resp == po.answer(db, r, N1, c)).all()


def test_full_size_256mb_random():
    r, N1, seed = 16, 128, 31
    db = po.gen_db(seed, r, N1)
    c = po.gen_client(seed, r, N1)
    with make_ctx(r, N1, db, c) as ctx:
        resp = ctx.answer(0, c["query"])
        want, bsgs, _ = po.answer(db, r, N1, c, with_stages=True)
        assert (ctx.fetch_stage(kb.STAGE_RESULT) == bsgs).all()
        assert (resp == want).all()
        # deterministic and reusable: a second call on the same workspace
        assert (ctx.answer(0, c["query"]) == want).all()


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref not present")
def test_testpir_known_answer():
    import ctypes
    g = GOLDEN["testpir"]
    seed, r, N1 = g["seed"], g["r"], g["N1"]
    L = po.ref()
    L.ref_pir_setup(seed, r, N1)
    sz = po.sizes(r, N1)
    db = np.zeros(sz["db"], np.uint64)
    c = {k: np.zeros(sz[k], np.uint64) for k in ("query", "baby", "giant", "packing", "rgsw")}
    c["perms"] = np.zeros(sz["perms"], np.int32)
    L.ref_pir_get_inputs(*[po._p(x) for x in (db, c["query"], c["baby"], c["giant"], c["packing"], c["rgsw"],
                                                c["perms"])])
    with make_ctx(r, N1, db, c) as ctx:
        resp = ctx.answer(0, c["query"])
    assert sha(resp) == g["response_sha"]
    msg = np.zeros(N, np.uint64)
    L.ref_pir_decrypt(po._p(resp), po._p(msg))
    assert (msg == np.arange(1, N + 1)).all()
    del ctypes


def test_staged_entry_points():
    r, N1, seed = 4, 128, 41
    db = po.gen_db(seed, r, N1)
    c = po.gen_client(seed, r, N1)
    with make_ctx(r, N1, db, c) as ctx:
        res, q = ctx.matrix_vector_mul(0, c["query"])
        want_res, want_q = po.matrix_vector_mul(db, r, N1, c)
        assert (res == want_res).all()
        assert (q == want_q).all()
        # externalProduct accumulating onto a non-zero NTT-domain result
        rng = np.random.default_rng(5)
        acc = rng.integers(0, po.CRTMOD, 2 * 2 * N, dtype=np.uint64)
        fd = want_res[:2 * 2 * N].copy()
        got_acc, got_fd = ctx.external_product(0, acc, fd)
        for j in range(2):
            e, f = po.external_product(fd[j * 2 * N:(j + 1) * 2 * N], c["rgsw"], ext=acc[j * 2 * N:(j + 1) * 2 * N])
            assert (got_acc[j * 2 * N:(j + 1) * 2 * N] == e).all()
            assert (got_fd[j * 2 * N:(j + 1) * 2 * N] == f).all()
        rl = rng.integers(0, po.CRTMOD, r * 2 * N, dtype=np.uint64)
        got_rl, want_rl = np.empty_like(rl), np.empty_like(rl)
        assert (ctx.packing(0, rl, rlwes_out=got_rl) == po.packing(rl, r, c["packing"], rlwes_out=want_rl)).all()
        assert (got_rl == want_rl).all()   # rlwes left as the reference leaves them


def test_edge_inputs():
    r, N1 = 2, 128
    c = po.gen_client(51, r, N1)
    db = np.zeros(r * N * N // 2, dtype=np.uint64)
    with make_ctx(r, N1, db, c) as ctx:
        q = c["query"].copy()
        q[:2 * N] = po.CRTMOD - 1
        q[2 * N:] = po.BSMOD - 1
        q[::7] = 0
        assert (ctx.answer(0, q) == po.answer(db, r, N1, dict(c, query=q))).all()
        # database words with every half at 2^32-1: the 64-bit sums wrap the same way as the reference's
        db2 = np.full(r * N * N // 2, np.uint64(0xFFFFFFFFFFFFFFFF))
        ctx.upload_db(db2)
        assert (ctx.answer(0, c["query"]) == po.answer(db2, r, N1, c)).all()
        # non-canonical words are rejected
        bad = c["query"].copy()
        bad[3] = po.CRTMOD
        with pytest.raises(kb.KspirError) as ei:
            ctx.answer(0, bad)
        assert ei.value.code == -1


def test_two_clients_are_independent():
    r, N1 = 2, 128
    db = po.gen_db(61, r, N1)
    c0 = po.gen_client(61, r, N1)
    c1 = po.gen_client(62, r, N1)
    with make_ctx(r, N1, db, c0, max_clients=2) as ctx:
        ctx.upload_client(1, c1["baby"], c1["giant"], c1["packing"], c1["rgsw"])
        a1 = ctx.answer(1, c1["query"])
        a0 = ctx.answer(0, c0["query"])
        assert (a0 == po.answer(db, r, N1, c0)).all()
        assert (a1 == po.answer(db, r, N1, c1)).all()


def test_reference_named_mirror():
    r, N1 = 2, 128
    db = po.gen_db(71, r, N1)
    c = po.gen_client(71, r, N1)
    result = np.zeros((r, 2, N), dtype=np.uint64)
    query1 = c["query"].reshape(2, 2, N).copy()
    kb.matrix_vector_mul_bsgs_rns_crt_large(result, query1, db, kb.AutoKeyBSGSRNS(c["baby"], c["giant"]), N1,
                                            c["perms"].reshape(N1, N), r)
    want_res, want_q = po.matrix_vector_mul(db, r, N1, c)
    assert (result.reshape(-1) == want_res).all()
    assert (query1.reshape(-1) == want_q).all()
    ext = np.zeros((r, 2, N), dtype=np.uint64)
    for j in range(r):
        kb.externalProduct(ext[j], result[j], kb.RGSWCiphertext(c["rgsw"]), r=r, N1=N1)
    want_resp, _, want_ext = po.answer(db, r, N1, c, with_stages=True)
    assert (ext.reshape(-1) == want_ext).all()
    out = np.zeros((2, N), dtype=np.uint64)
    kb.packingRLWEs(out, ext, kb.AutoKey(c["packing"]), N1=N1)
    assert (out.reshape(-1) == want_resp).all()


def test_back_to_back_device_answers():
    # many answers queued without host synchronisation exercise the scan's
    # producer/consumer ring across every stage phase; all must be identical
    torch = pytest.importorskip("torch")
    r, N1, seed, n = 16, 128, 81, 48
    db = po.gen_db(seed, r, N1)
    c = po.gen_client(seed, r, N1)
    want = po.answer(db, r, N1, c)
    with make_ctx(r, N1, db, c) as ctx:
        dq = torch.from_numpy(c["query"].view(np.int64).copy()).cuda()
        out = torch.zeros((n, 2 * N), dtype=torch.int64, device="cuda")
        stream = torch.cuda.Stream()
        torch.cuda.synchronize()
        for i in range(n):
            ctx.answer_device(0, dq.data_ptr(), out[i].data_ptr(), stream.cuda_stream)
        ctx.sync()
        got = out.cpu().numpy().view(np.uint64)
    for i in range(n):
        assert np.array_equal(got[i], want), f"answer {i} differs"
