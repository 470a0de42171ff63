"""Database preprocessing on the device (kspir_db_preprocess, and the one-for-one
kspir_database_tobsgsntt / kspir_database_tocrt): the reference's
database_tobsgsntt + database_tocrt (twosteps.cpp:42-179, crt.cpp:859-885).

Integer work, so the bar is word-for-word equality with the oracle's
restatement (pinned to the reference in test_oracle.py) and with the golden
digests the reference produced (tests/golden/golden.json).  The preprocessed
database must also answer exactly like the same database uploaded
preprocessed (kspir_db_upload).
"""
import hashlib
import json
import os

import numpy as np
import pytest

import kspir_b200 as kb
from kspir_b200 import synth
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
N = po.N
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", [c for c in GOLDEN["preprocess"] if c["kind"] != "testpir"],
                         ids=lambda c: f"{c['kind']}_r{c['r']}_N1{c['N1']}")
def test_preprocess_matches_reference_golden(case):
    r, N1 = case["r"], case["N1"]
    raw = synth.edge_raw_db() if case["kind"] == "edges" else synth.gen_raw_db(case["seed"], r)
    assert sha(raw) == case["raw_sha"]
    with kb.Context(r, N1) as ctx:
        ms = ctx.preprocess_db(raw)
        got = ctx.download_db()
    assert ms > 0
    if sha(got) != case["datacrt_sha"]:
        want = po.db_preprocess(raw, r, N1)
        bad = np.flatnonzero(got != want)
        pytest.fail(f"{bad.size} words differ, first at {bad[:4]}: got {got[bad[:4]]} want {want[bad[:4]]}")


def test_preprocess_full_size_equals_oracle_and_answers_alike():
    # 256 MB-record database (r = 16, N1 = 128): every word against the oracle,
    # then answers from the device-preprocessed database equal answers from the
    # uploaded oracle datacrt, and the oracle's answer
    r, N1 = 16, 128
    raw = synth.gen_raw_db(41, r)
    want = po.db_preprocess(raw, r, N1)
    c = po.gen_client(42, r, N1)
    with kb.Context(r, N1) as a, kb.Context(r, N1) as b:
        a.preprocess_db(raw)
        assert (a.download_db() == want).all()
        b.upload_db(want)
        for ctx in (a, b):
            ctx.upload_perms(c["perms"])
            ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        ra = a.answer(0, c["query"])
        assert (ra == b.answer(0, c["query"])).all()
    assert (ra == po.answer(want, r, N1, c)).all()


def test_preprocess_from_device_buffer():
    torch = pytest.importorskip("torch")
    r, N1 = 2, 64
    raw = synth.gen_raw_db(51, r)
    d = torch.from_numpy(raw.view(np.int64).copy()).cuda()
    torch.cuda.synchronize()
    with kb.Context(r, N1) as ctx:
        ctx.preprocess_db_device(d.data_ptr(), d.numel())
        got = ctx.download_db()
    assert (got == po.db_preprocess(raw, r, N1)).all()


def test_preprocess_rejects_out_of_range_and_keeps_database():
    r, N1 = 1, 128
    raw = synth.gen_raw_db(61, r)
    with kb.Context(r, N1) as ctx:
        ctx.preprocess_db(raw)
        before = ctx.download_db()
        bad = raw.copy()
        bad[777777] = po.P
        with pytest.raises(kb.KspirError) as ei:
            ctx.preprocess_db(bad)
        assert ei.value.code == kb.native.ERR_INVALID_ARG
        assert (ctx.download_db() == before).all()
        with pytest.raises(kb.KspirError):
            ctx.preprocess_db(raw[:-1])           # wrong size
    with kb.Context(r, N1) as ctx:                # nothing resident yet
        with pytest.raises(kb.KspirError) as ei:
            ctx.download_db()
        assert ei.value.code == kb.native.ERR_NOT_READY


@pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref not present")
def test_preprocess_testpir_database_recovers_the_record():
    # the database test-pir.cpp samples (planted record included), preprocessed
    # on the device, equals the reference's datacrt and answers the reference's
    # query so that the reference's decryption recovers the record
    g = [c for c in GOLDEN["preprocess"] if c["kind"] == "testpir"][0]
    seed, r, N1 = g["seed"], g["r"], g["N1"]
    L = po.ref()
    L.ref_pir_keep_raw(1)
    L.ref_pir_setup(seed, r, N1)
    L.ref_pir_keep_raw(0)
    sz = po.sizes(r, N1)
    raw = np.zeros(sz["db"], np.uint64)
    L.ref_pir_get_raw(po._p(raw))
    c = {k: np.zeros(sz[k], np.uint64) for k in ("query", "baby", "giant", "packing", "rgsw")}
    c["perms"] = np.zeros(sz["perms"], np.int32)
    L.ref_pir_get_inputs(None, *[po._p(c[k]) for k in ("query", "baby", "giant", "packing", "rgsw", "perms")])
    with kb.Context(r, N1) as ctx:
        ctx.preprocess_db(raw)
        assert sha(ctx.download_db()) == g["datacrt_sha"]
        ctx.upload_perms(c["perms"])
        ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        resp = ctx.answer(0, c["query"])
    msg = np.zeros(N, np.uint64)
    L.ref_pir_decrypt(po._p(resp), po._p(msg))
    assert (msg == np.arange(1, N + 1)).all(), msg[:8]


@pytest.mark.parametrize("N1", [64, 128, 256])
def test_database_tobsgsntt_and_tocrt_one_for_one(N1):
    # the reference's two functions separately, one sub-database: the rows mod
    # crtMod of database_tobsgsntt, and database_tocrt on arbitrary 64-bit words
    raw = synth.gen_raw_db(70 + N1, 1)
    raw[:9] = synth.edge_raw_db()[:9]
    rng = np.random.default_rng(N1)
    words = rng.integers(0, 2 ** 64 - 1, size=N * N // 2, dtype=np.uint64, endpoint=True)
    words[:6] = [0, 2 ** 64 - 1, po.Q1, po.Q2, po.CRTMOD, po.CRTMOD - 1]
    with kb.Context(1, N1) as ctx:
        rows = ctx.database_tobsgsntt(raw)
        assert (rows == po.database_tobsgsntt(raw, N1)).all()
        assert (ctx.database_tocrt(rows) == po.db_preprocess(raw, 1, N1)).all()
        assert (ctx.database_tocrt(words) == po.database_tocrt(words)).all()
        bad = raw.copy()
        bad[5] = 1 << 40
        with pytest.raises(kb.KspirError) as ei:
            ctx.database_tobsgsntt(bad)
        assert ei.value.code == kb.native.ERR_INVALID_ARG
    if po.ref_available():
        assert (rows == po.ref_database_tobsgsntt(raw, N1)).all()
