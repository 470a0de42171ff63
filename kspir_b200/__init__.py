"""kspir_b200: B200-native online answer of the KsPIR single-server PIR.

The product is the CUDA library ``libkspir_b200.so`` behind the C ABI of
``include/kspir_b200.h``.  This package is its Python host binding:

* :class:`Context` -- the device context (resident database, permutations,
  per-client keys, query workspaces) and the C-ABI calls, including the
  batched answer;
* :class:`Server` -- the serving loop (continuous batching, key admission by
  HBM budget, p50/p95/p99 latency);
* a mirror of the reference's own answer interface, with the reference's
  names, argument meaning and in-place effects, over numpy arrays laid out
  like the reference objects (an ``RlweCiphertext`` is a ``[2][N]`` u64 array
  ``(a, b)``):

  - :func:`matrix_vector_mul_bsgs_rns_crt_large` (reference src/twosteps.h:55-57)
  - :func:`externalProduct` (reference src/lwe.h:292)
  - :func:`packingRLWEs` (reference src/answer.h:79-80)
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .native import (BSMOD, CRTMOD, N, Q1, Q2, QUERY_WIRE_BYTES, RESPONSE_WIRE_BYTES, SCAN_CUDA, SCAN_MMA4,
                     SCAN_MMA8, SCAN_MMA16, SCAN_MMA32, SCAN_NAMES, Context, KspirError, LIB_PATH, STAGE_CIPHERBUF,
                     STAGE_EXT, STAGE_RESULT, STAGE_SCAN, Server, key_bundle_bytes, key_bundle_read,
                     key_bundle_write, load, permutation_matrix, query_pack, query_unpack, response_pack,
                     response_unpack)

__all__ = [
    "N", "Q1", "Q2", "CRTMOD", "BSMOD", "Context", "Server", "KspirError", "load", "LIB_PATH", "permutation_matrix",
    "STAGE_CIPHERBUF", "STAGE_SCAN", "STAGE_RESULT", "STAGE_EXT",
    "SCAN_CUDA", "SCAN_MMA4", "SCAN_MMA8", "SCAN_MMA16", "SCAN_MMA32", "SCAN_NAMES",
    "AutoKeyBSGSRNS", "AutoKey", "RGSWCiphertext",
    "matrix_vector_mul_bsgs_rns_crt_large", "externalProduct", "packingRLWEs", "invalidate",
    "key_bundle_bytes", "key_bundle_write", "key_bundle_read", "query_pack", "query_unpack", "response_pack",
    "response_unpack", "QUERY_WIRE_BYTES", "RESPONSE_WIRE_BYTES",
]


@dataclass
class AutoKeyBSGSRNS:
    """Key-switching keys of the BSGS first dimension (reference lwe.h:381-466).

    baby:  [N1/2][6][2][N] u64, keyMap[5^i] for i = 1..N1/2 (rows 0-2 mod crtMod, 3-5 mod bsMod)
    giant: [N2-1][2][2][N] u64, keyMap[5^(N1 c)] for c = 1..N2-1
    """
    baby: np.ndarray
    giant: np.ndarray


@dataclass
class AutoKey:
    """Packing keys (reference lwe.h:175-234): [log2 r][4][2][N] u64, keyMap[N/2^l + 1]."""
    keys: np.ndarray


@dataclass
class RGSWCiphertext:
    """RGSW query (reference lwe.h:113-170): [4][2][N] u64 rows (a[j], b[j]), NTT form."""
    rows: np.ndarray


class _Session:
    """Device context reused across mirror calls; uploads only what changed.

    Key parts and permutations are compared word for word with the copies
    last uploaded, so an object rewritten in place, or a new object at a
    freed one's address, is uploaded again.  The database (1 GiB at r = 16) is
    recognised by its address, size and a fingerprint of 4096 words spread
    over it: a caller that edits a few words of the same array in place calls
    :func:`invalidate` (or passes a new array) before the next answer."""

    PARTS = ("baby", "giant", "packing", "rgsw")

    def __init__(self):
        self.ctx = None
        self.key = None
        self.db_id = None
        self.perms = None
        self.parts = {}
        self.uploaded = False

    def get(self, r: int, N1: int) -> Context:
        if self.ctx is None or self.key != (r, N1):
            if self.ctx is not None:
                self.ctx.close()
            self.ctx = Context(r, N1)
            self.key = (r, N1)
            self.invalidate()
        return self.ctx

    def current(self, r: int | None = None, N1: int | None = None) -> Context:
        """The session's context, or a new one of (r, N1) (defaults r = 1, N1 = 128)."""
        if self.ctx is not None and (r is None or r == self.key[0]) and (N1 is None or N1 == self.key[1]):
            return self.ctx
        return self.get(r if r is not None else (self.key[0] if self.key else 1),
                        N1 if N1 is not None else (self.key[1] if self.key else 128))

    def ensure(self, ctx: Context, data=None, perms=None, **keys):
        if data is not None and self.db_id != _db_fingerprint(data):
            ctx.upload_db(data)
            self.db_id = _db_fingerprint(data)
        if perms is not None:
            p = np.asarray(perms, dtype=np.int32).reshape(-1)
            if self.perms is None or not np.array_equal(self.perms, p):
                ctx.upload_perms(p)
                self.perms = p.copy()
        changed = False
        for name in self.PARTS:
            a = keys.get(name)
            if a is None:
                continue
            a = np.asarray(a, dtype=np.uint64).reshape(-1)
            cur = self.parts.get(name)
            if cur is None or not np.array_equal(cur, a):
                self.parts[name] = a.copy()
                changed = True
        if changed or not self.uploaded:
            ctx.upload_client(0, *_fill_keys(ctx, *(self.parts.get(n) for n in self.PARTS)))
            self.uploaded = True

    def invalidate(self):
        self.db_id = None
        self.perms = None
        self.parts = {}
        self.uploaded = False


def _db_fingerprint(a):
    flat = np.asarray(a).reshape(-1)
    idx = np.linspace(0, flat.size - 1, num=min(4096, flat.size), dtype=np.int64)
    return (flat.ctypes.data, flat.nbytes, flat[idx].tobytes())


def _fill_keys(ctx: Context, baby, giant, packing, rgsw):
    """Zero-filled stand-ins for key parts no call has supplied yet."""
    if baby is None:
        baby = np.zeros((ctx.N1 // 2) * 6 * 2 * N, dtype=np.uint64)
    if giant is None:
        giant = np.zeros(max(ctx.N2 - 1, 0) * 2 * 2 * N, dtype=np.uint64)
    if packing is None:
        packing = np.zeros(ctx.levels * 4 * 2 * N, dtype=np.uint64)
    if rgsw is None:
        rgsw = np.zeros(4 * 2 * N, dtype=np.uint64)
    return baby, giant, packing, rgsw


def invalidate() -> None:
    """Forget what the reference-named mirror uploaded: the next call uploads
    its database, permutations and keys again."""
    _session.invalidate()


_session = _Session()


def matrix_vector_mul_bsgs_rns_crt_large(result: np.ndarray, input: np.ndarray, data: np.ndarray,
                                         autoKey: AutoKeyBSGSRNS, N1: int, permutations: np.ndarray,
                                         r: int = 1) -> None:
    """Reference twosteps.cpp:1527-1579.  result: [r][2][N] (written, NTT form);
    input: [2][2][N] query1 (input[0] is modswitched to NTT form in place, as
    the reference does); data: the preprocessed database (r*N*N/2 words)."""
    ctx = _session.get(r, N1)
    _session.ensure(ctx, data=data, perms=permutations, baby=autoKey.baby, giant=autoKey.giant)
    res, q = ctx.matrix_vector_mul(0, input)
    result.reshape(-1)[:] = res
    input.reshape(-1)[:] = q


def externalProduct(result: np.ndarray, firstDim: np.ndarray, query: RGSWCiphertext, r: int | None = None,
                    N1: int | None = None) -> None:
    """Reference lwe.cpp:761-808: result ([2][N]) += g^-1(firstDim) x query,
    returned in coefficient form; firstDim (NTT form) becomes coefficient form.
    Runs in the session's current context unless r / N1 name another one."""
    ctx = _session.current(r, N1)
    _session.ensure(ctx, rgsw=query.rows)
    res, fd = ctx.external_product(0, result, firstDim)
    result.reshape(-1)[:] = res
    firstDim.reshape(-1)[:] = fd


def packingRLWEs(result: np.ndarray, rlwes: np.ndarray, autokey: AutoKey, N1: int | None = None) -> None:
    """Reference answer.cpp:800-835: packs rlwes ([r][2][N], coefficient form)
    into result ([2][N]) and leaves rlwes as the reference does (rlwes[0] =
    the result, rlwes[I + j] = X^I rlwes[I + j] + rlwes[j] of each merge)."""
    r = rlwes.reshape(-1).size // (2 * N)
    ctx = _session.current(r, N1)
    _session.ensure(ctx, packing=autokey.keys)
    result.reshape(-1)[:] = ctx.packing(0, rlwes, rlwes_out=rlwes)
