"""TEST INFRASTRUCTURE ONLY -- Python bindings of the CPU oracle.

Loads ``oracle/libkspir_oracle.so`` (the plain-C restatement of the KsPIR
online answer, reference tests/test-pir.cpp:110-116) and, when it was built,
``oracle/_ref/libkspir_ref.so`` (the reference's own sources compiled against
the HEXL restatement).  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` import this module; the product path never
does.

The seeded synthetic inputs come from ``kspir_b200.synth`` (shared with the
benchmark); the permutation matrix from the oracle's own restatement.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

from kspir_b200 import synth as _synth

N = 4096
Q1 = 268369921
Q2 = 249561089
CRTMOD = Q1 * Q2
BSMOD = 16760833
P = 65537

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORACLE_SO = os.path.join(_HERE, "libkspir_oracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libkspir_ref.so")
_lock = threading.Lock()
_lib = None
_ref = None

_u64p = ctypes.POINTER(ctypes.c_uint64)
_i32p = ctypes.POINTER(ctypes.c_int32)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def build_oracle() -> str:
    """Compiles the C restatement with the committed Makefile if needed."""
    src = os.path.join(_HERE, "kspir_oracle.c")
    if not os.path.exists(_ORACLE_SO) or os.path.getmtime(_ORACLE_SO) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE, "oracle"], check=True)
    return _ORACLE_SO


def lib():
    global _lib
    with _lock:
        if _lib is None:
            build_oracle()
            L = ctypes.CDLL(_ORACLE_SO)
            vp = ctypes.c_void_p
            L.ko_answer.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp]
            L.ko_matrix_vector_mul.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp]
            L.ko_external_product.argtypes = [vp, vp, vp]
            L.ko_packing.argtypes = [vp, ctypes.c_int, vp, vp]
            L.ko_scan.argtypes = [vp, vp, ctypes.c_int, vp]
            L.ko_ntt_forward.argtypes = [vp, ctypes.c_uint64]
            L.ko_ntt_inverse.argtypes = [vp, ctypes.c_uint64]
            L.ko_ntt_root.argtypes = [ctypes.c_uint64]
            L.ko_ntt_root.restype = ctypes.c_uint64
            L.ko_decompose_bsgs.argtypes = [vp, vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, vp, vp]
            L.ko_decompose.argtypes = [vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, vp]
            L.ko_decompose_rlwe.argtypes = [vp, vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64,
                                            ctypes.c_uint64, vp]
            L.ko_crt_compose.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
            L.ko_crt_compose.restype = ctypes.c_uint64
            L.ko_barrett_coeff.argtypes = [ctypes.c_uint64, ctypes.c_int]
            L.ko_barrett_coeff.restype = ctypes.c_uint64
            L.ko_permutation_matrix.argtypes = [vp, ctypes.c_int]
            L.ko_pow_mod_index.argtypes = [ctypes.c_int, ctypes.c_int]
            L.ko_giant_steps.argtypes = [vp, vp, ctypes.c_int, vp]
            L.ko_db_preprocess.argtypes = [vp, ctypes.c_int, vp]
            L.ko_database_tobsgsntt.argtypes = [vp, ctypes.c_int, vp]
            L.ko_database_tocrt.argtypes = [vp, vp]
            L.ko_query_message.argtypes = [ctypes.c_int, vp]
            _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF_SO)


def ref():
    """The reference compiled from its own sources (built here by ``make -C oracle ref``)."""
    global _ref
    with _lock:
        if _ref is None:
            if not os.path.exists(_REF_SO):
                raise FileNotFoundError(_REF_SO)
            L = ctypes.CDLL(_REF_SO)
            vp = ctypes.c_void_p
            L.ref_pir_setup.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_int]
            L.ref_pir_target.argtypes = [vp, vp]
            L.ref_pir_get_inputs.argtypes = [vp] * 7
            L.ref_pir_decrypt.argtypes = [vp, vp]
            L.ref_answer.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
            L.ref_matrix_vector_mul.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, vp, vp]
            L.ref_external_product.argtypes = [vp, vp, vp]
            L.ref_packing.argtypes = [vp, ctypes.c_int, vp, vp]
            L.ref_scan.argtypes = [vp, vp, ctypes.c_int, vp]
            L.ref_crt_compose.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
            L.ref_crt_compose.restype = ctypes.c_uint64
            L.ref_permutation_matrix.argtypes = [vp, ctypes.c_int]
            L.ref_ntt.argtypes = [vp, ctypes.c_uint64, ctypes.c_int]
            L.ref_decompose_bsgs.argtypes = [vp, vp, vp, vp]
            L.ref_decompose.argtypes = [vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, vp]
            L.ref_decompose_rlwe.argtypes = [vp, vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, vp]
            L.ref_pir_keep_raw.argtypes = [ctypes.c_int]
            L.ref_pir_get_raw.argtypes = [vp]
            L.ref_db_preprocess.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp]
            L.ref_gen_autokey_from_offline.argtypes = [ctypes.c_int] + [vp] * 9
            L.ref_database_tobsgsntt.argtypes = [vp, ctypes.c_int, vp]
            L.ref_database_tocrt.argtypes = [vp, ctypes.c_int, vp]
            L.ref_pir_get_secret.argtypes = [vp]
            L.ref_pir_decrypt_r.argtypes = [vp, ctypes.c_int, vp]
            _ref = L
    return _ref


# ---------------------------------------------------------------------------
# sizes and seeded synthetic inputs

def sizes(r: int, N1: int) -> dict:
    N2 = N // 2 // N1
    levels = int(r).bit_length() - 1
    return dict(N2=N2, db=r * N * N // 2, query=4 * N, baby=(N1 // 2) * 6 * 2 * N,
                giant=(N2 - 1) * 2 * 2 * N, packing=levels * 4 * 2 * N, rgsw=4 * 2 * N,
                perms=N1 * N, result=r * 2 * N, response=2 * N)


def gen_db(seed: int, r: int, N1: int) -> np.ndarray:
    """Seeded synthetic database (kspir_b200.synth.gen_db)."""
    return _synth.gen_db(seed, r, N1)


def gen_client(seed: int, r: int, N1: int) -> dict:
    """Seeded synthetic client material plus the permutation matrix of the
    oracle's restatement of compute_permutation_matrix (utils.cpp:1591-1619)."""
    c = _synth.gen_client(seed, r, N1)
    c["perms"] = permutation_matrix(N1)
    return c


# ---------------------------------------------------------------------------
# C restatement wrappers

def permutation_matrix(N1: int) -> np.ndarray:
    out = np.empty(N1 * N, dtype=np.int32)
    lib().ko_permutation_matrix(_p(out), N1)
    return out


def answer(db, r, N1, c, with_stages=False):
    resp = np.zeros(2 * N, dtype=np.uint64)
    bsgs = np.zeros(r * 2 * N, dtype=np.uint64) if with_stages else None
    ext = np.zeros(r * 2 * N, dtype=np.uint64) if with_stages else None
    rc = lib().ko_answer(_p(db), r, N1, _p(c["query"]), _p(c["baby"]), _p(c["giant"]),
                         _p(c["packing"]), _p(c["rgsw"]), _p(c["perms"]), _p(resp), _p(bsgs), _p(ext))
    if rc:
        raise RuntimeError(f"ko_answer rc={rc}")
    return (resp, bsgs, ext) if with_stages else resp


def matrix_vector_mul(db, r, N1, c, want_cipherbuf=False):
    q = c["query"].copy()
    res = np.zeros(r * 2 * N, dtype=np.uint64)
    cb = np.zeros(N * 2 * N1, dtype=np.uint64) if want_cipherbuf else None
    rc = lib().ko_matrix_vector_mul(_p(db), r, N1, _p(q), _p(c["baby"]), _p(c["giant"]),
                                    _p(c["perms"]), _p(res), _p(cb))
    if rc:
        raise RuntimeError(f"ko_matrix_vector_mul rc={rc}")
    return (res, q, cb) if want_cipherbuf else (res, q)


def external_product(first_dim, rgsw, ext=None):
    fd = first_dim.copy()
    e = np.zeros(2 * N, dtype=np.uint64) if ext is None else ext.copy()
    lib().ko_external_product(_p(e), _p(fd), _p(rgsw))
    return e, fd


def packing(rlwes, r, keys, rlwes_out=None):
    """Packed response; rlwes_out (or None) receives rlwes as the reference's
    packingRLWEs leaves them."""
    rl = rlwes.copy()
    resp = np.zeros(2 * N, dtype=np.uint64)
    rc = lib().ko_packing(_p(rl), r, _p(keys), _p(resp))
    if rc:
        raise RuntimeError(f"ko_packing rc={rc}")
    if rlwes_out is not None:
        rlwes_out.reshape(-1)[:] = rl
    return resp


def giant_steps(output, N1, giant):
    """evalAutoRNSCRT of one sub-database on its scan output ([N2][2][N] words)."""
    out = output.copy()
    res = np.zeros(2 * N, dtype=np.uint64)
    lib().ko_giant_steps(_p(res), _p(out), N1, _p(giant))
    return res


def scan(db_sub, cipherbuf, N1):
    out = np.zeros((N // 2 // N1) * 2 * N, dtype=np.uint64)
    lib().ko_scan(_p(db_sub), _p(cipherbuf), N1, _p(out))
    return out


def db_preprocess(raw, r, N1):
    """database_tobsgsntt + database_tocrt of every sub-database (restatement)."""
    num = N * N // 2
    raw = np.ascontiguousarray(raw, dtype=np.uint64)
    out = np.empty(r * num, dtype=np.uint64)
    for k in range(r):
        if lib().ko_db_preprocess(_p(raw[k * num:(k + 1) * num]), N1, _p(out[k * num:(k + 1) * num])):
            raise ValueError("database entries must be below p")
    return out


def database_tobsgsntt(raw_sub, N1):
    """database_tobsgsntt of one sub-database (restatement): rows [N/2][N]."""
    raw_sub = np.ascontiguousarray(raw_sub, dtype=np.uint64)
    out = np.empty(N * N // 2, dtype=np.uint64)
    if lib().ko_database_tobsgsntt(_p(raw_sub), N1, _p(out)):
        raise ValueError("database entries must be below p")
    return out


def database_tocrt(rows):
    """database_tocrt of one sub-database (restatement): datacrt [N][N/2]."""
    rows = np.ascontiguousarray(rows, dtype=np.uint64)
    out = np.empty(N * N // 2, dtype=np.uint64)
    lib().ko_database_tocrt(_p(rows), _p(out))
    return out


def ref_database_tobsgsntt(raw_sub, N1):
    raw_sub = np.ascontiguousarray(raw_sub, dtype=np.uint64)
    out = np.empty(N * N // 2, dtype=np.uint64)
    ref().ref_database_tobsgsntt(_p(raw_sub), N1, _p(out))
    return out


def ref_database_tocrt(rows, N1=128):
    rows = np.ascontiguousarray(rows, dtype=np.uint64)
    out = np.empty(N * N // 2, dtype=np.uint64)
    ref().ref_database_tocrt(_p(rows), N1, _p(out))
    return out


def query_message(t: int) -> np.ndarray:
    """The scaled message dm of query_bsgs_rns for row t (restatement)."""
    out = np.empty(N, dtype=np.uint64)
    lib().ko_query_message(t, _p(out))
    return out


def ref_db_preprocess(raw, r, N1):
    """The same through the reference's own database_tobsgsntt / database_tocrt."""
    raw = np.ascontiguousarray(raw, dtype=np.uint64)
    out = np.empty(r * N * N // 2, dtype=np.uint64)
    ref().ref_db_preprocess(_p(raw), r, N1, _p(out))
    return out


def ntt(a, modulus, inverse=False):
    x = np.ascontiguousarray(a, dtype=np.uint64).copy()
    fn = lib().ko_ntt_inverse if inverse else lib().ko_ntt_forward
    if fn(_p(x), modulus):
        raise ValueError("unsupported modulus")
    return x


def crt_compose(x: int, y: int) -> int:
    return lib().ko_crt_compose(x, y)


def barrett_coeff(v: int, n: int) -> int:
    return lib().ko_barrett_coeff(v, n)


# ---------------------------------------------------------------------------
# offline key derivation (reference genAutoKeyFromOffline, twosteps.cpp:1749-1864)

AUXMOD = 268361729          # crt.h:37
CRTBAMOD = BSMOD * AUXMOD   # crt.h:51


def gen_offline_keys(seed: int) -> dict:
    """Seeded input keys of the derivation (any words canonical for their
    moduli): offline1 [10][2][N] (rows 0-4 mod crtMod, 5-9 mod crtBaMod),
    offline2 [10][2][N] (5-9 mod auxMod), auto1 [6][2][N] (3-5 mod crtBaMod),
    auto2 [6][2][N] (3-5 mod auxMod)."""
    rng = np.random.default_rng(np.random.SeedSequence([seed, 0x0FF]))

    def key(rows, m2):
        k = np.empty((2 * rows, 2, N), np.uint64)
        k[:rows] = rng.integers(0, CRTMOD, (rows, 2, N), dtype=np.uint64)
        k[rows:] = rng.integers(0, m2, (rows, 2, N), dtype=np.uint64)
        return k.reshape(-1)
    return dict(offline1=key(5, CRTBAMOD), offline2=key(5, AUXMOD), auto1=key(3, CRTBAMOD), auto2=key(3, AUXMOD))


def ref_gen_autokey_from_offline(N1: int, keys: dict) -> dict:
    """The reference build's genAutoKeyFromOffline on these input keys."""
    N2 = N // 2 // N1
    out = dict(chain1=np.zeros(max(N1 - 2, 0) * 12 * N, np.uint64), chain2=np.zeros(max(N2 - 2, 0) * 12 * N, np.uint64),
               baby=np.zeros((N1 - 1) * 12 * N, np.uint64), giant=np.zeros((N2 - 1) * 6 * N, np.uint64))
    t = ctypes.c_double()
    ref().ref_gen_autokey_from_offline(N1, *[_p(keys[k]) for k in ("offline1", "offline2", "auto1", "auto2")],
                                       *[_p(out[k]) for k in ("chain1", "chain2", "baby", "giant")], ctypes.byref(t))
    out["seconds"] = t.value
    return out
