"""Wire and file formats (include/kspir_b200.h): the client key bundle, the
query and response messages (host-only, run on CPU), and the database file
(on the GPU, marked).  Integer words: every round trip must be exact, and
every malformed container must be refused."""
import os

import numpy as np
import pytest

import kspir_b200 as kb
from oracle import pyoracle as po

N = po.N


def test_key_bundle_round_trip_and_size():
    for r, N1 in ((16, 128), (2, 64), (1, 256)):
        c = po.gen_client(300 + r, r, N1)
        b = kb.key_bundle_write(r, N1, c["baby"], c["giant"], c["packing"], c["rgsw"])
        assert b.size == kb.key_bundle_bytes(r, N1)
        back = kb.key_bundle_read(b, r, N1)
        for k in ("baby", "giant", "packing", "rgsw"):
            assert np.array_equal(back[k], np.asarray(c[k]).reshape(-1)), k
    # 256 MB database shape: 17.7 MiB against 27.1 MiB of u64 words
    assert kb.key_bundle_bytes(16, 128) == 64 + 64 * 2 * N * 30 + (15 * 4 + 4 * 8 + 8) * N * 7
    assert kb.key_bundle_bytes(3, 128) == 0


def test_key_bundle_refuses_bad_input():
    r, N1 = 2, 128
    c = po.gen_client(310, r, N1)
    b = kb.key_bundle_write(r, N1, c["baby"], c["giant"], c["packing"], c["rgsw"])
    bad = b.copy()
    bad[64 + 1000] ^= 1                                      # payload bit flip
    with pytest.raises(kb.KspirError) as ei:
        kb.key_bundle_read(bad, r, N1)
    assert ei.value.code == kb.native.ERR_IO
    with pytest.raises(kb.KspirError) as ei:
        kb.key_bundle_read(b[:-1], r, N1)                    # truncated
    assert ei.value.code == kb.native.ERR_IO
    with pytest.raises(kb.KspirError) as ei:
        kb.key_bundle_read(b, 4, N1)                         # another shape
    assert ei.value.code == kb.native.ERR_INVALID_ARG
    bad = b.copy()
    bad[0] = ord("X")                                        # magic
    with pytest.raises(kb.KspirError) as ei:
        kb.key_bundle_read(bad, r, N1)
    assert ei.value.code == kb.native.ERR_IO
    baby = np.asarray(c["baby"]).copy().reshape(-1)
    baby[3 * 2 * N + 5] = po.BSMOD                           # a bsMod row word out of range
    with pytest.raises(kb.KspirError) as ei:
        kb.key_bundle_write(r, N1, baby, c["giant"], c["packing"], c["rgsw"])
    assert ei.value.code == kb.native.ERR_INVALID_ARG


def test_query_and_response_messages():
    rng = np.random.default_rng(5)
    q = np.concatenate([rng.integers(0, po.CRTMOD, 2 * N, dtype=np.uint64),
                        rng.integers(0, po.BSMOD, 2 * N, dtype=np.uint64)])
    q[0], q[1], q[2 * N], q[2 * N + 1] = 0, po.CRTMOD - 1, 0, po.BSMOD - 1
    m = kb.query_pack(q)
    assert m.size == kb.QUERY_WIRE_BYTES == 81936
    assert np.array_equal(kb.query_unpack(m), q)
    resp = rng.integers(0, po.CRTMOD, 2 * N, dtype=np.uint64)
    mr = kb.response_pack(resp)
    assert mr.size == kb.RESPONSE_WIRE_BYTES == 57360
    assert np.array_equal(kb.response_unpack(mr), resp)
    with pytest.raises(kb.KspirError) as ei:
        kb.response_unpack(m)                                # a query is not a response
    assert ei.value.code == kb.native.ERR_IO
    bad = mr.copy()
    bad[100] ^= 0x40
    with pytest.raises(kb.KspirError) as ei:
        kb.response_unpack(bad)
    assert ei.value.code == kb.native.ERR_IO
    q2 = q.copy()
    q2[2 * N + 7] = po.BSMOD
    with pytest.raises(kb.KspirError) as ei:
        kb.query_pack(q2)
    assert ei.value.code == kb.native.ERR_INVALID_ARG


@pytest.mark.gpu
def test_database_file_and_bundle_upload(tmp_path):
    # save -> load into a fresh context answers exactly like the original (and
    # the oracle); a corrupted or mismatched file is refused and leaves the
    # resident database as it was; keys uploaded from a bundle answer alike
    r, N1 = 2, 128
    db = po.gen_db(321, r, N1)
    c = po.gen_client(322, r, N1)
    path = str(tmp_path / "db.kspir")
    with kb.Context(r, N1) as a:
        a.upload_db(db)
        a.save_db(path)
    assert os.path.getsize(path) == 64 + db.nbytes
    bundle = kb.key_bundle_write(r, N1, c["baby"], c["giant"], c["packing"], c["rgsw"])
    with kb.Context(r, N1, max_clients=1, max_inflight=2) as b:
        b.load_db(path)
        assert np.array_equal(b.download_db(), db)
        b.upload_perms(c["perms"])
        b.upload_client_bundle(0, bundle)
        got = b.answer(0, c["query"])
        assert np.array_equal(got, po.answer(db, r, N1, c))
        raw = bytearray(open(path, "rb").read())
        raw[64 + 12345] ^= 1
        bad = str(tmp_path / "bad.kspir")
        open(bad, "wb").write(bytes(raw))
        with pytest.raises(kb.KspirError) as ei:
            b.load_db(bad)
        assert ei.value.code == kb.native.ERR_IO
        assert np.array_equal(b.answer(0, c["query"]), got)
    with kb.Context(4, N1) as d:
        with pytest.raises(kb.KspirError) as ei:
            d.load_db(path)
        assert ei.value.code == kb.native.ERR_INVALID_ARG
