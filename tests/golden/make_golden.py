"""Generates the committed golden fixtures from the KsPIR reference itself.

Runs the reference's own sources (compiled by ``make -C oracle ref`` into
``oracle/_ref/libkspir_ref.so``, against the HEXL restatement) on:

* seeded synthetic inputs (``oracle.pyoracle.gen_db`` / ``gen_client``) --
  digests of every stage of the online answer;
* a replay of ``tests/test-pir.cpp`` (glibc ``rand()`` stream after
  ``srand(seed)``, reference keygen, preprocessing and query) -- the response
  digest and the decrypted record (the known answer [1, 2, ..., 4096]);
* database preprocessing (database_tobsgsntt + database_tocrt) of seeded
  raw databases (``kspir_b200.synth.gen_raw_db``), of an edge-value pattern
  and of the database test-pir.cpp samples -- input and output digests;
* small unit vectors of the reference helpers (crt_compose, barrett_coeff,
  the decompositions) on edge values;
* the offline key derivation (genAutoKeyFromOffline) of seeded input keys
  (``oracle.pyoracle.gen_offline_keys``) at N1 = 64 (tests/test-two-steps-key.cpp)
  and 128 -- digests of every output key map.

Usage:  python tests/golden/make_golden.py   (needs /root/reference to build oracle/_ref)
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402

N = po.N
CASES = [(2, 128, 5), (1, 128, 3), (4, 64, 7), (2, 256, 11)]
TESTPIR = (1, 16, 128)   # seed, r, N1
PREPROCESS = [(31, 1, 128), (32, 1, 64), (33, 1, 256), (34, 2, 128)]
PREPROCESS_TESTPIR = (3, 2, 128)
OFFLINE = [(41, 64), (42, 128)]   # seed, N1


def sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def head(a: np.ndarray, n: int = 8) -> list[int]:
    return [int(x) for x in np.asarray(a).reshape(-1)[:n]]


def ref_answer(L, db, r, N1, c):
    resp = np.zeros(2 * N, np.uint64)
    bsgs = np.zeros(r * 2 * N, np.uint64)
    ext = np.zeros(r * 2 * N, np.uint64)
    t = ctypes.c_double()
    L.ref_answer(po._p(db), r, N1, po._p(c["query"]), po._p(c["baby"]), po._p(c["giant"]),
                 po._p(c["packing"]), po._p(c["rgsw"]), po._p(c["perms"]), po._p(resp),
                 po._p(bsgs), po._p(ext), ctypes.byref(t))
    return resp, bsgs, ext


def main():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "oracle"], check=True)
    L = po.ref()
    out = {"generator": "tests/golden/make_golden.py", "answer": [], "units": {}}
    for r, N1, seed in CASES:
        db = po.gen_db(seed, r, N1)
        c = po.gen_client(seed, r, N1)
        resp, bsgs, ext = ref_answer(L, db, r, N1, c)
        q = c["query"].copy()
        res = np.zeros(r * 2 * N, np.uint64)
        L.ref_matrix_vector_mul(po._p(db), r, N1, po._p(q), po._p(c["baby"]), po._p(c["giant"]),
                                po._p(c["perms"]), po._p(res))
        out["answer"].append(dict(r=r, N1=N1, seed=seed, response_sha=sha(resp), response_head=head(resp),
                                  bsgs_sha=sha(bsgs), ext_sha=sha(ext), query_modswitched_sha=sha(q),
                                  inputs=dict(db_sha=sha(db), query_sha=sha(c["query"]),
                                              perms_sha=sha(c["perms"]))))
        print("case", r, N1, seed, "done", file=sys.stderr)

    seed, r, N1 = TESTPIR
    L.ref_pir_setup(seed, r, N1)
    sz = po.sizes(r, N1)
    db = np.zeros(sz["db"], np.uint64)
    c = {k: np.zeros(sz[k], np.uint64) for k in ("query", "baby", "giant", "packing", "rgsw")}
    c["perms"] = np.zeros(sz["perms"], np.int32)
    L.ref_pir_get_inputs(*[po._p(x) for x in (db, c["query"], c["baby"], c["giant"], c["packing"],
                                                c["rgsw"], c["perms"])])
    col, slot = ctypes.c_uint32(), ctypes.c_uint32()
    L.ref_pir_target(ctypes.byref(col), ctypes.byref(slot))
    resp, bsgs, ext = ref_answer(L, db, r, N1, c)
    msg = np.zeros(N, np.uint64)
    L.ref_pir_decrypt(po._p(resp), po._p(msg))
    out["testpir"] = dict(seed=seed, r=r, N1=N1, target_col=col.value, target_packing=slot.value,
                          db_sha=sha(db), query_sha=sha(c["query"]), response_sha=sha(resp),
                          response_head=head(resp), bsgs_sha=sha(bsgs), ext_sha=sha(ext),
                          decrypted_head=head(msg, 16), decrypted_is_1_to_N=bool((msg == np.arange(1, N + 1)).all()))

    # database preprocessing
    from kspir_b200 import synth
    pre = []
    for seed, r, N1 in PREPROCESS:
        raw = synth.gen_raw_db(seed, r)
        dc = po.ref_db_preprocess(raw, r, N1)
        pre.append(dict(kind="synthetic", seed=seed, r=r, N1=N1, raw_sha=sha(raw), datacrt_sha=sha(dc),
                        datacrt_head=head(dc)))
    raw = synth.edge_raw_db()
    dc = po.ref_db_preprocess(raw, 1, 128)
    pre.append(dict(kind="edges", r=1, N1=128, raw_sha=sha(raw), datacrt_sha=sha(dc), datacrt_head=head(dc)))
    seed, r, N1 = PREPROCESS_TESTPIR
    L.ref_pir_keep_raw(1)
    L.ref_pir_setup(seed, r, N1)
    L.ref_pir_keep_raw(0)
    raw = np.zeros(r * N * N // 2, np.uint64)
    L.ref_pir_get_raw(po._p(raw))
    dc = np.zeros(r * N * N // 2, np.uint64)
    L.ref_pir_get_inputs(po._p(dc), None, None, None, None, None, None)
    pre.append(dict(kind="testpir", seed=seed, r=r, N1=N1, raw_sha=sha(raw), datacrt_sha=sha(dc),
                    datacrt_head=head(dc)))
    out["preprocess"] = pre

    # unit vectors on edge values
    edge64 = [0, 1, 2 ** 28 - 1, po.Q1 - 1, po.Q1, po.Q2, 2 ** 32 - 1, 2 ** 56 - 1, 2 ** 62, 2 ** 63 - 1,
              2 ** 64 - 1]
    out["units"]["crt_compose"] = [[x, y, int(L.ref_crt_compose(x, y))] for x in edge64 for y in edge64]
    rng = np.random.default_rng(123)
    a = rng.integers(0, po.CRTMOD, N, dtype=np.uint64)
    a[:6] = [0, 1, po.CRTMOD - 1, po.CRTMOD // 2, po.CRTMOD // 2 + 1, 2 ** 55]
    b = rng.integers(0, po.BSMOD, N, dtype=np.uint64)
    b[:4] = [0, 1, po.BSMOD - 1, po.BSMOD // 2]
    d1 = np.zeros(3 * N, np.uint64)
    d2 = np.zeros(3 * N, np.uint64)
    L.ref_decompose_bsgs(po._p(a), po._p(b), po._p(d1), po._p(d2))
    dv = np.zeros(2 * N, np.uint64)
    L.ref_decompose(po._p(a), 2, 1 << 20, 1 << 18, po._p(dv))
    dp = np.zeros(4 * N, np.uint64)
    L.ref_decompose(po._p(a), 4, 0, 1 << 14, po._p(dp))
    dr = np.zeros(4 * N, np.uint64)
    L.ref_decompose_rlwe(po._p(a), po._p(b), 2, 1 << 20, 1 << 18, po._p(dr))
    out["units"]["decompose"] = dict(seed=123, bsgs_crt_sha=sha(d1), bsgs_bs_sha=sha(d2), varB_giant_sha=sha(dv),
                                     varB_pack_sha=sha(dp), rlwe_sha=sha(dr))
    ntt = {}
    for m in (po.CRTMOD, po.BSMOD, po.P):
        x = rng.integers(0, m, N, dtype=np.uint64)
        y = x.copy()
        L.ref_ntt(po._p(y), m, 0)
        ntt[str(m)] = dict(in_sha=sha(x), out_sha=sha(y), out_head=head(y))
    out["units"]["ntt"] = ntt
    off = []
    for seed, N1 in OFFLINE:
        keys = po.gen_offline_keys(seed)
        res = po.ref_gen_autokey_from_offline(N1, keys)
        off.append(dict(seed=seed, N1=N1, inputs_sha={k: sha(v) for k, v in keys.items()},
                        **{k + "_sha": sha(res[k]) for k in ("chain1", "chain2", "baby", "giant")},
                        giant_head=head(res["giant"])))
    out["offline"] = off
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", os.path.join(HERE, "golden.json"), file=sys.stderr)


if __name__ == "__main__":
    main()
