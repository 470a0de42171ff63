"""Pins the CPU oracle (oracle/kspir_oracle.c) to the KsPIR reference.

* against the committed golden fixtures (tests/golden/golden.json, produced by
  the reference's own sources through tests/golden/make_golden.py);
* against the reference build itself (oracle/_ref) when it is present;
* against known answers the reference relies on: the CRT root of unity
  (crt.h:81 vs test-utils.cpp:345-348), HEXL's slot order
  [1, 4097, 2049, 6145, ...] (utils.cpp:1476-1478), the automorphism /
  permutation identity (test-utils.cpp:361-396), and decryption of the
  test-pir replay to [1, 2, ..., 4096] (README.md:65).
"""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as po

N = po.N
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
needs_ref = pytest.mark.skipif(not po.ref_available(), reason="reference build oracle/_ref not present")


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def brv12(x):
    return int(f"{x:012b}"[::-1], 2)


# ---------------------------------------------------------------------------
# known answers

def test_crt_root_is_crt_of_minimal_roots():
    # reference crt.h:81 root_of_unity_crt == crt_compose(minroot(q1), minroot(q2)) (test-utils.cpp:345-348)
    lib = po.lib()
    psi = lib.ko_ntt_root(po.CRTMOD)
    assert psi == 3375402822066082
    assert psi % po.Q1 == lib.ko_ntt_root(po.Q1) == 62736
    assert psi % po.Q2 == lib.ko_ntt_root(po.Q2) == 32309
    assert pow(psi, N, po.CRTMOD) == po.CRTMOD - 1
    assert po.crt_compose(62736, 32309) == psi
    # HEXL MinimalPrimitiveRoot(2N, q) for the other transform moduli
    assert lib.ko_ntt_root(po.BSMOD) == 3689
    assert lib.ko_ntt_root(po.P) == 13


@pytest.mark.parametrize("modulus", [po.CRTMOD, po.BSMOD, po.P, po.Q1, po.Q2])
def test_ntt_definition_and_order(modulus):
    rng = np.random.default_rng(modulus % 1000)
    x = rng.integers(0, modulus, N, dtype=np.uint64)
    y = po.ntt(x, modulus)
    psi = po.lib().ko_ntt_root(modulus)
    xs = [int(v) for v in x]
    for j in (0, 1, 2, 3, 777, N - 1):
        e = 2 * brv12(j) + 1
        w = pow(psi, e, modulus)
        acc, p = 0, 1
        for v in xs:
            acc += v * p
            p = p * w % modulus
        assert int(y[j]) == acc % modulus
    # slot exponents [1, 4097, 2049, 6145, 1025, ...] (utils.cpp:1476-1478)
    assert [2 * brv12(j) + 1 for j in range(5)] == [1, 4097, 2049, 6145, 1025]
    assert (po.ntt(y, modulus, inverse=True) == x).all()


def _auto(x, g, q):
    out = np.zeros_like(x)
    for i in range(N):
        d = (i * g) % (2 * N)
        if d >= N:
            out[d - N] = (q - int(x[i])) % q
        else:
            out[d] = x[i]
    return out


@pytest.mark.parametrize("rot", [1, 2, 63, 64])
def test_automorphism_is_slot_permutation(rot):
    # NTT(X -> X^(5^rot)) == NTT(x)[perms[rot]] (test-utils.cpp:361-396)
    perms = po.permutation_matrix(128).reshape(128, N)
    rng = np.random.default_rng(rot)
    x = rng.integers(0, po.CRTMOD, N, dtype=np.uint64)
    g = pow(5, rot, 2 * N)
    lhs = po.ntt(_auto(x, g, po.CRTMOD), po.CRTMOD)
    rhs = po.ntt(x, po.CRTMOD)[perms[rot]]
    assert (lhs == rhs).all()


def test_crt_compose_is_residue_crt():
    # crt_compose (crt.cpp:368-377) == the canonical crtMod value with residues (x mod q1, y mod q2)
    for x, y, want in GOLDEN["units"]["crt_compose"]:
        got = po.crt_compose(x, y)
        assert got == want
        v = ((x % po.Q1) * po.Q2 * pow(po.Q2, -1, po.Q1) + (y % po.Q2) * po.Q1 * pow(po.Q1, -1, po.Q2)) % po.CRTMOD
        assert got == v
    rng = np.random.default_rng(9)
    for x, y in rng.integers(0, 2 ** 63, (2000, 2), dtype=np.uint64):
        x, y = int(x), int(y)
        v = ((x % po.Q1) * po.Q2 * pow(po.Q2, -1, po.Q1) + (y % po.Q2) * po.Q1 * pow(po.Q1, -1, po.Q2)) % po.CRTMOD
        assert po.crt_compose(x, y) == v


def test_barrett_coeff_is_exact_mod():
    rng = np.random.default_rng(4)
    vals = [0, 1, po.Q1 - 1, po.Q1, po.Q2, 2 ** 56 - 1, 2 ** 63, 2 ** 64 - 1]
    vals += [int(v) for v in rng.integers(0, 2 ** 63, 2000, dtype=np.uint64)]
    for v in vals:
        assert po.barrett_coeff(v, 0) == v % po.Q1
        assert po.barrett_coeff(v, 1) == v % po.Q2


def test_decompositions_match_golden():
    u = GOLDEN["units"]["decompose"]
    rng = np.random.default_rng(u["seed"])
    a = rng.integers(0, po.CRTMOD, N, dtype=np.uint64)
    a[:6] = [0, 1, po.CRTMOD - 1, po.CRTMOD // 2, po.CRTMOD // 2 + 1, 2 ** 55]
    b = rng.integers(0, po.BSMOD, N, dtype=np.uint64)
    b[:4] = [0, 1, po.BSMOD - 1, po.BSMOD // 2]
    L = po.lib()
    d1 = np.zeros(3 * N, np.uint64)
    d2 = np.zeros(3 * N, np.uint64)
    L.ko_decompose_bsgs(po._p(a), po._p(b), 3, 1 << 20, 1 << 20, po._p(d1), po._p(d2))
    assert sha(d1) == u["bsgs_crt_sha"] and sha(d2) == u["bsgs_bs_sha"]
    dv = np.zeros(2 * N, np.uint64)
    L.ko_decompose(po._p(a), 2, 1 << 20, 1 << 18, po.CRTMOD, po._p(dv))
    assert sha(dv) == u["varB_giant_sha"]
    dp = np.zeros(4 * N, np.uint64)
    L.ko_decompose(po._p(a), 4, 0, 1 << 14, po.CRTMOD, po._p(dp))
    assert sha(dp) == u["varB_pack_sha"]
    dr = np.zeros(4 * N, np.uint64)
    L.ko_decompose_rlwe(po._p(a), po._p(b), 2, 1 << 20, 1 << 18, po.CRTMOD, po._p(dr))
    assert sha(dr) == u["rlwe_sha"]


def test_decompose_treats_q_like_zero():
    # the reference feeds decompose a word equal to q from `modulus - 0`
    # (twosteps.cpp:629, answer.cpp:606); it must give the digits of 0
    L = po.lib()
    for ell, base, bg in ((2, 1 << 20, 1 << 18), (4, 0, 1 << 14)):
        x = np.zeros(N, np.uint64)
        x[1] = po.CRTMOD
        out = np.zeros(ell * N, np.uint64)
        L.ko_decompose(po._p(x), ell, base, bg, po.CRTMOD, po._p(out))
        o = out.reshape(ell, N)
        assert (o[:, 0] == o[:, 1]).all()


def test_ntt_golden():
    rng = np.random.default_rng(123)
    # replay the generator's draws to reach the NTT inputs
    rng.integers(0, po.CRTMOD, N, dtype=np.uint64)
    rng.integers(0, po.BSMOD, N, dtype=np.uint64)
    for m in (po.CRTMOD, po.BSMOD, po.P):
        x = rng.integers(0, m, N, dtype=np.uint64)
        g = GOLDEN["units"]["ntt"][str(m)]
        assert sha(x) == g["in_sha"]
        assert sha(po.ntt(x, m)) == g["out_sha"]


# ---------------------------------------------------------------------------
# whole answer against the golden digests

@pytest.mark.parametrize("case", GOLDEN["answer"], ids=lambda c: f"r{c['r']}_N1{c['N1']}_s{c['seed']}")
def test_answer_matches_reference_golden(case):
    r, N1, seed = case["r"], case["N1"], case["seed"]
    db = po.gen_db(seed, r, N1)
    c = po.gen_client(seed, r, N1)
    assert sha(db) == case["inputs"]["db_sha"] and sha(c["query"]) == case["inputs"]["query_sha"]
    resp, bsgs, ext = po.answer(db, r, N1, c, with_stages=True)
    assert sha(bsgs) == case["bsgs_sha"]
    assert sha(ext) == case["ext_sha"]
    assert sha(resp) == case["response_sha"]
    _, q = po.matrix_vector_mul(db, r, N1, c)
    assert sha(q) == case["query_modswitched_sha"]


# ---------------------------------------------------------------------------
# live comparison with the reference build

@needs_ref
def test_oracle_equals_reference_live():
    r, N1 = 2, 128
    db = po.gen_db(21, r, N1)
    c = po.gen_client(21, r, N1)
    resp, bsgs, ext = po.answer(db, r, N1, c, with_stages=True)
    L = po.ref()
    R = np.zeros(2 * N, np.uint64)
    RB = np.zeros(r * 2 * N, np.uint64)
    RE = np.zeros(r * 2 * N, np.uint64)
    t = ctypes.c_double()
    L.ref_answer(po._p(db), r, N1, po._p(c["query"]), po._p(c["baby"]), po._p(c["giant"]), po._p(c["packing"]),
                 po._p(c["rgsw"]), po._p(c["perms"]), po._p(R), po._p(RB), po._p(RE), ctypes.byref(t))
    assert (bsgs == RB).all() and (ext == RE).all() and (resp == R).all()
    perms_ref = np.zeros(128 * N, np.int32)
    L.ref_permutation_matrix(po._p(perms_ref), 128)
    assert (perms_ref == c["perms"]).all()


@needs_ref
@pytest.mark.parametrize("r", [1, 2, 8])
def test_packing_leaves_rlwes_like_the_reference(r):
    # packingRLWEs overwrites its input vector (answer.cpp:821-828): rlwes[0]
    # ends as the response, rlwes[I + j] as X^I c + r of each merge
    rng = np.random.default_rng(30 + r)
    keys = rng.integers(0, po.CRTMOD, max(r.bit_length() - 1, 0) * 4 * 2 * N, dtype=np.uint64)
    rl = rng.integers(0, po.CRTMOD, r * 2 * N, dtype=np.uint64)
    rl[5 * 2 * N % rl.size: 5 * 2 * N % rl.size + 64] = 0   # zeros: the multConst negation quirk
    got_rl = np.empty_like(rl)
    got = po.packing(rl, r, keys, rlwes_out=got_rl)
    ref_rl = rl.copy()
    ref_resp = np.zeros(2 * N, np.uint64)
    po.ref().ref_packing(po._p(ref_rl), r, po._p(keys), po._p(ref_resp))
    assert (got == ref_resp).all()
    assert (got_rl == ref_rl).all()
    assert (got_rl[:2 * N] == got).all()


@needs_ref
@pytest.mark.parametrize("case", GOLDEN["offline"], ids=lambda c: f"N1_{c['N1']}")
def test_offline_derivation_reference_matches_golden(case):
    # the reference build's genAutoKeyFromOffline on the seeded input keys
    keys = po.gen_offline_keys(case["seed"])
    assert {k: sha(v) for k, v in keys.items()} == case["inputs_sha"]
    res = po.ref_gen_autokey_from_offline(case["N1"], keys)
    for k in ("chain1", "chain2", "baby", "giant"):
        assert sha(res[k]) == case[k + "_sha"], k


@needs_ref
def test_testpir_replay_known_answer():
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
    assert sha(db) == g["db_sha"]
    resp = po.answer(db, r, N1, c)
    assert sha(resp) == g["response_sha"]
    msg = np.zeros(N, np.uint64)
    L.ref_pir_decrypt(po._p(resp), po._p(msg))
    assert (msg == np.arange(1, N + 1)).all()


# ---------------------------------------------------------------------------
# database preprocessing (database_tobsgsntt + database_tocrt)

@pytest.mark.parametrize("case", GOLDEN["preprocess"], ids=lambda c: f"{c['kind']}_r{c['r']}_N1{c['N1']}")
def test_db_preprocess_matches_reference_golden(case):
    from kspir_b200 import synth
    if case["kind"] == "testpir":
        pytest.skip("the raw database of the test-pir.cpp replay comes from the reference build")
    if case["kind"] == "edges":
        raw = synth.edge_raw_db()
    else:
        raw = synth.gen_raw_db(case["seed"], case["r"])
    assert sha(raw) == case["raw_sha"]
    out = po.db_preprocess(raw, case["r"], case["N1"])
    assert [int(x) for x in out[:8]] == case["datacrt_head"]
    assert sha(out) == case["datacrt_sha"]


def test_db_preprocess_rejects_words_at_or_above_p():
    raw = np.zeros(N * N // 2, np.uint64)
    raw[12345] = po.P
    with pytest.raises(ValueError):
        po.db_preprocess(raw, 1, 128)


@needs_ref
def test_db_preprocess_equals_reference_on_testpir_database():
    g = [c for c in GOLDEN["preprocess"] if c["kind"] == "testpir"][0]
    seed, r, N1 = g["seed"], g["r"], g["N1"]
    L = po.ref()
    L.ref_pir_keep_raw(1)
    L.ref_pir_setup(seed, r, N1)
    L.ref_pir_keep_raw(0)
    raw = np.zeros(r * N * N // 2, np.uint64)
    L.ref_pir_get_raw(po._p(raw))
    assert sha(raw) == g["raw_sha"]
    out = po.db_preprocess(raw, r, N1)
    assert sha(out) == g["datacrt_sha"]
    live = np.zeros_like(out)
    L.ref_pir_get_inputs(po._p(live), None, None, None, None, None, None)
    assert (live == out).all()


@needs_ref
def test_db_preprocess_steps_equal_reference():
    from kspir_b200 import synth
    raw = synth.gen_raw_db(35, 1)
    rows = po.database_tobsgsntt(raw, 64)
    assert (rows == po.ref_database_tobsgsntt(raw, 64)).all()
    rng = np.random.default_rng(36)
    words = rng.integers(0, 2 ** 64 - 1, size=N * N // 2, dtype=np.uint64, endpoint=True)
    words[:4] = [0, 2 ** 64 - 1, po.Q1, po.CRTMOD]
    assert (po.database_tocrt(words) == po.ref_database_tocrt(words)).all()
    assert (po.database_tocrt(rows) == po.db_preprocess(raw, 1, 64)).all()
