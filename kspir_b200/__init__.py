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
    "matrix_vector_mul_bsgs_rns_crt_large", "externalProduct", "packingRLWEs",
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
    """Device context reused across mirror calls; re-uploads only what changed."""

    def __init__(self):
        self.ctx = None
        self.key = None
        self.db_id = None
        self.perm_id = None
        self.client_ids = None

    def get(self, r: int, N1: int) -> Context:
        if self.ctx is None or self.key != (r, N1):
            if self.ctx is not None:
                self.ctx.close()
            self.ctx = Context(r, N1)
            self.key = (r, N1)
            self.db_id = self.perm_id = self.client_ids = None
        return self.ctx

    def ensure(self, ctx: Context, data=None, perms=None, baby=None, giant=None, packing=None, rgsw=None):
        if data is not None and self.db_id != _ident(data):
            ctx.upload_db(data)
            self.db_id = _ident(data)
        if perms is not None and self.perm_id != _ident(perms):
            ctx.upload_perms(perms)
            self.perm_id = _ident(perms)
        ids = tuple(_ident(a) for a in (baby, giant, packing, rgsw))
        if self.client_ids != ids:
            ctx.upload_client(0, *_fill_keys(ctx, baby, giant, packing, rgsw))
            self.client_ids = ids


def _ident(a):
    return None if a is None else (a.ctypes.data, a.nbytes, a.__array_interface__["data"][0])


def _fill_keys(ctx: Context, baby, giant, packing, rgsw):
    """Zero-filled stand-ins for key parts a staged call does not use."""
    if baby is None:
        baby = np.zeros((ctx.N1 // 2) * 6 * 2 * N, dtype=np.uint64)
    if giant is None:
        giant = np.zeros(max(ctx.N2 - 1, 0) * 2 * 2 * N, dtype=np.uint64)
    if packing is None:
        packing = np.zeros(ctx.levels * 4 * 2 * N, dtype=np.uint64)
    if rgsw is None:
        rgsw = np.zeros(4 * 2 * N, dtype=np.uint64)
    return baby, giant, packing, rgsw


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


def externalProduct(result: np.ndarray, firstDim: np.ndarray, query: RGSWCiphertext, r: int = 1,
                    N1: int = 128) -> None:
    """Reference lwe.cpp:761-808: result ([2][N]) += g^-1(firstDim) x query,
    returned in coefficient form; firstDim (NTT form) becomes coefficient form."""
    ctx = _session.get(r, N1)
    _session.ensure(ctx, rgsw=query.rows, baby=None, giant=None, packing=None)
    res, fd = ctx.external_product(0, result, firstDim)
    result.reshape(-1)[:] = res
    firstDim.reshape(-1)[:] = fd


def packingRLWEs(result: np.ndarray, rlwes: np.ndarray, autokey: AutoKey, N1: int = 128) -> None:
    """Reference answer.cpp:800-835: packs rlwes ([r][2][N], coefficient form) into result ([2][N])."""
    r = rlwes.reshape(-1).size // (2 * N)
    ctx = _session.get(r, N1)
    _session.ensure(ctx, packing=autokey.keys)
    result.reshape(-1)[:] = ctx.packing(0, rlwes)
