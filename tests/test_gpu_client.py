"""The client side on the device (kspir_client_queries / kspir_client_decrypt):
query_bsgs_rns (twosteps.cpp:279-318) and decrypt_bsgs_total
(twosteps.cpp:388-418).

Decryption is deterministic: word for word the reference's, on the test-pir
response and on random responses.  The query uses Philox draws instead of the
reference's rand(), so it is checked by its algebra -- b - a * s minus the
scaled message is the same ternary error in both moduli, the scaled message
computed by the oracle with the reference's own long double expression --
and end to end: the server's answer to a device-made query decrypts, under
the reference's decryption, to the planted record."""
import numpy as np
import pytest

import kspir_b200 as kb
from oracle import pyoracle as po

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref not present")]
N = po.N


def replay(seed=3, r=2, N1=128):
    L = po.ref()
    L.ref_pir_setup(seed, r, N1)
    sz = po.sizes(r, N1)
    db = np.zeros(sz["db"], np.uint64)
    c = {k: np.zeros(sz[k], np.uint64) for k in ("query", "baby", "giant", "packing", "rgsw")}
    c["perms"] = np.zeros(sz["perms"], np.int32)
    L.ref_pir_get_inputs(po._p(db), *[po._p(c[k]) for k in ("query", "baby", "giant", "packing", "rgsw", "perms")])
    sec = np.zeros(N, np.uint64)
    L.ref_pir_get_secret(po._p(sec))
    col, slot = np.zeros(1, np.uint32), np.zeros(1, np.uint32)
    L.ref_pir_target(po._p(col), po._p(slot))
    return L, db, c, sec, int(col[0])


def ref_decrypt(L, resp, r):
    m = np.zeros(N, np.uint64)
    L.ref_pir_decrypt_r(po._p(resp), r, po._p(m))
    return m


def polymul(a, b, q):
    """a * b mod (X^N + 1, q) through the oracle's transforms."""
    return po.ntt(mulmod(po.ntt(a, q), po.ntt(b, q), q), q, inverse=True)


def mulmod(x, y, q):
    return np.array([(int(u) * int(v)) % q for u, v in zip(x, y)], dtype=np.uint64)


def centred(x, q):
    x = np.asarray(x, dtype=object)
    return np.array([int(v) if v <= q // 2 else int(v) - q for v in x], dtype=object)


def test_decrypt_matches_reference():
    r = 2
    L, db, c, sec, col = replay(r=r)
    with kb.Context(r, 128) as ctx:
        ctx.upload_db(db)
        ctx.upload_perms(c["perms"])
        ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        resp = ctx.answer(0, c["query"])
        rng = np.random.default_rng(11)
        rand = rng.integers(0, po.CRTMOD, size=(3, 2 * N), dtype=np.uint64)
        for rr in (r, 16):
            allr = np.vstack([resp[None, :], rand])
            got = ctx.client_decrypt(np.tile(sec, (4, 1)), allr, rr)
            for i in range(4):
                assert np.array_equal(got[i], ref_decrypt(L, allr[i], rr)), (rr, i)
    with kb.Context(r, 128) as ctx:
        assert np.array_equal(ctx.client_decrypt(sec[None, :], resp[None, :], r)[0], np.arange(1, N + 1))


def test_query_algebra():
    L, db, c, sec, col = replay()
    rows = np.array([col, 0, N // 2 - 1], np.uint32)
    with kb.Context(2, 128) as ctx:
        qs = ctx.client_queries(np.tile(sec, (3, 1)), rows, seed=12345)
        again = ctx.client_queries(np.tile(sec, (3, 1)), rows, seed=12345)
        other = ctx.client_queries(np.tile(sec, (3, 1)), rows, seed=54321)
    assert np.array_equal(qs, again)
    assert not np.array_equal(qs[0, :N], other[0, :N])
    s_bs = np.array([int(v) if v <= po.CRTMOD // 2 else int(v) - po.CRTMOD + po.BSMOD for v in sec], np.uint64)
    for i, t in enumerate(rows):
        a1, b1, a2, b2 = (qs[i, k * N:(k + 1) * N] for k in range(4))
        assert (a1 < po.CRTMOD).all() and (a2 < po.BSMOD).all()
        dm = po.query_message(int(t))
        e1 = centred((b1.astype(object) - polymul(a1, sec, po.CRTMOD).astype(object)
                      - dm.astype(object) * po.BSMOD) % po.CRTMOD, po.CRTMOD)
        e2 = centred((b2.astype(object) - polymul(a2, s_bs, po.BSMOD).astype(object)) % po.BSMOD, po.BSMOD)
        assert set(e1) <= {-1, 0, 1}, f"row {t}: crt error out of range"
        assert all(u == v for u, v in zip(e1, e2)), f"row {t}: the two moduli must share the error"


def test_device_query_answers_decrypt_to_the_record():
    r = 2
    L, db, c, sec, col = replay(r=r)
    with kb.Context(r, 128) as ctx:
        q = ctx.client_queries(sec[None, :], np.array([col], np.uint32), seed=7)[0]
        ctx.upload_db(db)
        ctx.upload_perms(c["perms"])
        ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        resp = ctx.answer(0, q)
        mine = ctx.client_decrypt(sec[None, :], resp[None, :], r)[0]
    assert np.array_equal(ref_decrypt(L, resp, r), np.arange(1, N + 1))
    assert np.array_equal(mine, np.arange(1, N + 1))


def test_client_rejects_bad_input():
    L, db, c, sec, col = replay()
    with kb.Context(2, 128) as ctx:
        with pytest.raises(kb.KspirError):
            ctx.client_queries(sec[None, :], np.array([N // 2], np.uint32), seed=1)
        big = sec.copy()
        big[3] = po.CRTMOD // 2
        with pytest.raises(kb.KspirError):
            ctx.client_queries(big[None, :], np.array([1], np.uint32), seed=1)
        with pytest.raises(kb.KspirError):
            ctx.client_decrypt(sec[None, :], np.full((1, 2 * N), po.CRTMOD, np.uint64), 2)
