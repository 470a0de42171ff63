"""ctypes binding of the C ABI in ``include/kspir_b200.h``.

The product path always runs through ``libkspir_b200.so``; there is no CPU
fallback.  Loading fails loudly when the library has not been built.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

N = 4096
Q1 = 268369921
Q2 = 249561089
CRTMOD = Q1 * Q2
BSMOD = 16760833

OK = 0
ERR_INVALID_ARG = -1
ERR_CUDA = -2
ERR_NOT_READY = -3
ERR_OOM = -4
ERR_TIMEOUT = -5
ERR_BUSY = -6

STAGE_CIPHERBUF = 0
STAGE_SCAN = 1
STAGE_RESULT = 2
STAGE_EXT = 3

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libkspir_b200.so")

# every entry point of include/kspir_b200.h with its ctypes signature
_vp = ctypes.c_void_p
_i = ctypes.c_int
_sz = ctypes.c_size_t
SIGNATURES = {
    "kspir_ctx_create": (_i, [_i, _vp, _vp]),
    "kspir_ctx_destroy": (_i, [_vp]),
    "kspir_last_error": (ctypes.c_char_p, [_vp]),
    "kspir_strerror": (ctypes.c_char_p, [_i]),
    "kspir_db_upload": (_i, [_vp, _vp, _sz]),
    "kspir_db_preprocess": (_i, [_vp, _vp, _sz, _vp]),
    "kspir_db_preprocess_device": (_i, [_vp, _vp, _sz, _vp]),
    "kspir_db_download": (_i, [_vp, _vp, _sz]),
    "kspir_key_bundle_bytes": (_sz, [_i, _i]),
    "kspir_key_bundle_write": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _sz]),
    "kspir_key_bundle_read": (_i, [_vp, _sz, _i, _i, _vp, _vp, _vp, _vp]),
    "kspir_client_keys_upload_bundle": (_i, [_vp, _i, _vp, _sz]),
    "kspir_query_pack": (_i, [_vp, _vp]),
    "kspir_query_unpack": (_i, [_vp, _sz, _vp]),
    "kspir_response_pack": (_i, [_vp, _vp]),
    "kspir_response_unpack": (_i, [_vp, _sz, _vp]),
    "kspir_db_save": (_i, [_vp, ctypes.c_char_p]),
    "kspir_db_load": (_i, [_vp, ctypes.c_char_p]),
    "kspir_client_queries": (_i, [_vp, _i, _vp, _vp, ctypes.c_uint64, _vp]),
    "kspir_client_decrypt": (_i, [_vp, _i, _vp, _vp, _i, _vp]),
    "kspir_database_tobsgsntt": (_i, [_vp, _vp, _vp]),
    "kspir_database_tocrt": (_i, [_vp, _vp, _vp]),
    "kspir_perms_upload": (_i, [_vp, _vp, _sz]),
    "kspir_client_keys_upload": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "kspir_answer": (_i, [_vp, _i, _vp, _vp]),
    "kspir_answer_device": (_i, [_vp, _i, _vp, _vp, _vp]),
    "kspir_sync": (_i, [_vp]),
    "kspir_matrix_vector_mul_bsgs_rns_crt_large": (_i, [_vp, _i, _vp, _vp]),
    "kspir_external_product": (_i, [_vp, _i, _vp, _vp, _i]),
    "kspir_packing_rlwes": (_i, [_vp, _i, _vp, _vp]),
    "kspir_last_timing": (_i, [_vp, _vp, _vp]),
    "kspir_fetch_stage": (_i, [_vp, _i, _vp, _sz]),
    "kspir_permutation_matrix": (_i, [_vp, _i]),
    "kspir_external_product_noalloc": (_i, [_i, _vp, _vp, _vp, _i, _vp]),
    "kspir_timing_reset": (_i, [_vp]),
    "kspir_timing_summary": (_i, [_vp, _vp, _vp, _vp, _vp]),
    "kspir_answer_batch": (_i, [_vp, _i, _vp, _vp, _vp]),
    "kspir_answer_batch_device": (_i, [_vp, _i, _vp, _vp, _vp, _vp]),
    "kspir_tune_batch": (_i, [_vp, _i, _vp, _vp]),
    "kspir_set_scan_kind": (_i, [_vp, _i, _i]),
    "kspir_get_scan_kind": (_i, [_vp, _i]),
    "kspir_fetch_stage_slot": (_i, [_vp, _i, _i, _vp, _sz]),
    "kspir_client_key_bytes": (_sz, [_vp]),
    "kspir_debug_scan_fault": (_i, [_vp, ctypes.c_int64, ctypes.c_long]),
    "kspir_set_fused": (_i, [_vp, _i]),
    "kspir_gen_autokey_from_offline": (_i, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "kspir_get_fused": (_i, [_vp]),
    "kspir_server_create": (_i, [_vp, _vp, _vp]),
    "kspir_server_destroy": (_i, [_vp]),
    "kspir_server_register_client": (_i, [_vp, ctypes.c_int64, _vp, _vp, _vp, _vp]),
    "kspir_server_submit": (_i, [_vp, ctypes.c_int64, _vp, _vp, _vp]),
    "kspir_server_poll": (_i, [_vp, ctypes.c_uint64]),
    "kspir_server_wait": (_i, [_vp, ctypes.c_uint64, _i]),
    "kspir_server_get_stats": (_i, [_vp, _vp]),
    "kspir_server_reset_stats": (_i, [_vp]),
    "kspir_server_latencies": (_i, [_vp, _vp, _sz, _vp]),
}

# database-scan variants of kspir_tune_batch / kspir_set_scan_kind
SCAN_CUDA = 0
SCAN_MMA4 = 1
SCAN_MMA8 = 2
SCAN_MMA16 = 3
SCAN_MMA32 = 4
SCAN_NAMES = {SCAN_CUDA: "cuda-core", SCAN_MMA4: "tcgen05-bt4", SCAN_MMA8: "tcgen05-bt8",
              SCAN_MMA16: "tcgen05-bt16", SCAN_MMA32: "tcgen05-bt32"}


class Params(ctypes.Structure):
    _fields_ = [("r", ctypes.c_int32), ("N1", ctypes.c_int32),
                ("max_clients", ctypes.c_int32), ("max_inflight", ctypes.c_int32)]


class ServerParams(ctypes.Structure):
    _fields_ = [("lanes", ctypes.c_int32), ("lane_size", ctypes.c_int32), ("key_budget_bytes", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    _fields_ = [("served", ctypes.c_long), ("batches", ctypes.c_long), ("mean_batch", ctypes.c_double),
                ("p50_us", ctypes.c_double), ("p95_us", ctypes.c_double), ("p99_us", ctypes.c_double),
                ("max_us", ctypes.c_double), ("queries_per_s", ctypes.c_double), ("key_uploads", ctypes.c_long),
                ("evictions", ctypes.c_long), ("key_slots", ctypes.c_int32), ("max_running_lanes", ctypes.c_int32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads the CUDA library (raises if it is missing or incomplete)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"kspir_b200 CUDA library not built: {path} (run kspir_b200/build.py)")
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a: np.ndarray | None):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def permutation_matrix(N1: int) -> np.ndarray:
    """[N1][N] int32, the reference's compute_permutation_matrix (utils.cpp:1591-1619)."""
    out = np.empty(N1 * N, dtype=np.int32)
    rc = load().kspir_permutation_matrix(ptr(out), N1)
    if rc:
        raise KspirError(rc, "permutation_matrix")
    return out


class KspirError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"kspir error {code}: {msg}")
        self.code = code


ERR_IO = -7
QUERY_WIRE_BYTES = 16 + 2 * N * 7 + 2 * N * 3
RESPONSE_WIRE_BYTES = 16 + 2 * N * 7


def _host_check(rc: int):
    if rc:
        lib = load()
        raise KspirError(rc, lib.kspir_last_error(None).decode() or lib.kspir_strerror(rc).decode())


def _key_shapes(r: int, N1: int) -> dict:
    N2, levels = N // 2 // N1, max(0, int(r).bit_length() - 1)
    return dict(baby=(N1 // 2) * 6 * 2 * N, giant=(N2 - 1) * 2 * 2 * N, packing=levels * 4 * 2 * N, rgsw=4 * 2 * N)


def key_bundle_bytes(r: int, N1: int) -> int:
    return int(load().kspir_key_bundle_bytes(r, N1))


def key_bundle_write(r: int, N1: int, baby, giant, packing, rgsw) -> np.ndarray:
    """One client's key material as a checksummed bundle (packed words)."""
    arrs = [None if a is None or np.size(a) == 0 else _u64(a).reshape(-1) for a in (baby, giant, packing, rgsw)]
    out = np.empty(key_bundle_bytes(r, N1), dtype=np.uint8)
    _host_check(load().kspir_key_bundle_write(r, N1, *[ptr(a) for a in arrs], ptr(out), out.size))
    return out


def key_bundle_read(bundle, r: int, N1: int) -> dict:
    b = np.ascontiguousarray(bundle, dtype=np.uint8).reshape(-1)
    shapes = _key_shapes(r, N1)
    keys = {k: np.empty(n, dtype=np.uint64) for k, n in shapes.items()}
    args = [ptr(keys[k]) if shapes[k] else None for k in ("baby", "giant", "packing", "rgsw")]
    _host_check(load().kspir_key_bundle_read(ptr(b), b.size, r, N1, *args))
    return keys


def query_pack(query) -> np.ndarray:
    q = _u64(query).reshape(-1)
    out = np.empty(QUERY_WIRE_BYTES, dtype=np.uint8)
    _host_check(load().kspir_query_pack(ptr(q), ptr(out)))
    return out


def query_unpack(msg) -> np.ndarray:
    m = np.ascontiguousarray(msg, dtype=np.uint8).reshape(-1)
    out = np.empty(4 * N, dtype=np.uint64)
    _host_check(load().kspir_query_unpack(ptr(m), m.size, ptr(out)))
    return out


def response_pack(response) -> np.ndarray:
    r = _u64(response).reshape(-1)
    out = np.empty(RESPONSE_WIRE_BYTES, dtype=np.uint8)
    _host_check(load().kspir_response_pack(ptr(r), ptr(out)))
    return out


def response_unpack(msg) -> np.ndarray:
    m = np.ascontiguousarray(msg, dtype=np.uint8).reshape(-1)
    out = np.empty(2 * N, dtype=np.uint64)
    _host_check(load().kspir_response_unpack(ptr(m), m.size, ptr(out)))
    return out


def _u64(a) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return a


class Context:
    """One device context: resident database, permutations, client keys and
    query workspaces (include/kspir_b200.h)."""

    def __init__(self, r: int, N1: int = 128, device: int = 0, max_clients: int = 1, max_inflight: int = 1):
        self.lib = load()
        self.r, self.N1, self.N2 = r, N1, N // 2 // N1
        self.levels = r.bit_length() - 1
        self._h = ctypes.c_void_p()
        p = Params(r, N1, max_clients, max_inflight)
        rc = self.lib.kspir_ctx_create(device, ctypes.byref(p), ctypes.byref(self._h))
        if rc:
            detail = self.lib.kspir_last_error(None).decode()
            raise KspirError(rc, detail or self.lib.kspir_strerror(rc).decode())

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc: int):
        if rc:
            msg = self.lib.kspir_last_error(self._h).decode() if self._h else ""
            raise KspirError(rc, msg or self.lib.kspir_strerror(rc).decode())

    def close(self):
        if self._h:
            self.lib.kspir_ctx_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def handle(self):
        return self._h

    # -- resident data ----------------------------------------------------
    def upload_db(self, datacrt):
        d = _u64(datacrt).reshape(-1)
        self._check(self.lib.kspir_db_upload(self._h, ptr(d), d.size))

    def upload_client_bundle(self, client: int, bundle):
        b = np.ascontiguousarray(bundle, dtype=np.uint8).reshape(-1)
        self._check(self.lib.kspir_client_keys_upload_bundle(self._h, client, ptr(b), b.size))

    def save_db(self, path: str):
        """The resident database as a checksummed file (kspir_db_save)."""
        self._check(self.lib.kspir_db_save(self._h, os.fsencode(path)))

    def load_db(self, path: str):
        """Replaces the resident database with a file of kspir_db_save."""
        self._check(self.lib.kspir_db_load(self._h, os.fsencode(path)))

    def preprocess_db(self, raw) -> float:
        """Reference database_tobsgsntt + database_tocrt of every sub-database
        (twosteps.cpp:42-179, crt.cpp:859-885) on the device; the result
        becomes the resident database.  Returns the device time in ms."""
        d = _u64(raw).reshape(-1)
        ms = ctypes.c_float(0.0)
        self._check(self.lib.kspir_db_preprocess(self._h, ptr(d), d.size, ctypes.byref(ms)))
        return ms.value

    def preprocess_db_device(self, d_raw: int, words: int) -> float:
        ms = ctypes.c_float(0.0)
        self._check(self.lib.kspir_db_preprocess_device(self._h, ctypes.c_void_p(d_raw), words, ctypes.byref(ms)))
        return ms.value

    def client_queries(self, secrets, rows, seed: int) -> np.ndarray:
        """query_bsgs_rns on the device for each (secret, row): [n][4N] words."""
        sec = _u64(secrets).reshape(-1, N)
        rw = np.ascontiguousarray(rows, dtype=np.uint32).reshape(-1)
        if sec.shape[0] != rw.size:
            raise ValueError("one secret per row")
        out = np.empty((rw.size, 4 * N), dtype=np.uint64)
        self._check(self.lib.kspir_client_queries(self._h, rw.size, ptr(sec), ptr(rw), seed, ptr(out)))
        return out

    def client_decrypt(self, secrets, responses, r: int) -> np.ndarray:
        """decrypt_bsgs_total on the device: [n][N] message words."""
        sec = _u64(secrets).reshape(-1, N)
        rsp = _u64(responses).reshape(-1, 2 * N)
        if sec.shape[0] != rsp.shape[0]:
            raise ValueError("one secret per response")
        out = np.empty((rsp.shape[0], N), dtype=np.uint64)
        self._check(self.lib.kspir_client_decrypt(self._h, rsp.shape[0], ptr(sec), ptr(rsp), r, ptr(out)))
        return out

    def database_tobsgsntt(self, data) -> np.ndarray:
        """Reference database_tobsgsntt of one sub-database on the device:
        data [N][N/2] words < 65537 -> rows [N/2][N] mod crtMod."""
        d = _u64(data).reshape(-1)
        if d.size != N * N // 2:
            raise ValueError("one sub-database: N * N / 2 words")
        out = np.empty(N * N // 2, dtype=np.uint64)
        self._check(self.lib.kspir_database_tobsgsntt(self._h, ptr(d), ptr(out)))
        return out

    def database_tocrt(self, data_ntt) -> np.ndarray:
        """Reference database_tocrt of one sub-database on the device:
        rows [N/2][N] -> datacrt [N][N/2]."""
        d = _u64(data_ntt).reshape(-1)
        if d.size != N * N // 2:
            raise ValueError("one sub-database: N * N / 2 words")
        out = np.empty(N * N // 2, dtype=np.uint64)
        self._check(self.lib.kspir_database_tocrt(self._h, ptr(d), ptr(out)))
        return out

    def download_db(self, out: np.ndarray | None = None) -> np.ndarray:
        words = self.r * N * N // 2
        if out is None:
            out = np.empty(words, dtype=np.uint64)
        self._check(self.lib.kspir_db_download(self._h, ptr(out), out.size))
        return out

    def upload_perms(self, perms):
        p = np.ascontiguousarray(perms, dtype=np.int32).reshape(-1)
        self._check(self.lib.kspir_perms_upload(self._h, ptr(p), p.size))

    def upload_client(self, client: int, baby, giant, packing, rgsw):
        arrs = [None if a is None else _u64(a).reshape(-1) for a in (baby, giant, packing, rgsw)]
        self._check(self.lib.kspir_client_keys_upload(self._h, client, *[ptr(a) for a in arrs]))

    # -- answer -----------------------------------------------------------
    def answer(self, client: int, query, out: np.ndarray | None = None) -> np.ndarray:
        q = _u64(query).reshape(-1)
        if out is None:
            out = np.empty(2 * N, dtype=np.uint64)
        self._check(self.lib.kspir_answer(self._h, client, ptr(q), ptr(out)))
        return out

    def answer_device(self, client: int, d_query: int, d_response: int, stream: int | None = None):
        self._check(self.lib.kspir_answer_device(self._h, client, ctypes.c_void_p(d_query),
                                                 ctypes.c_void_p(d_response),
                                                 ctypes.c_void_p(stream) if stream else None))

    def sync(self):
        self._check(self.lib.kspir_sync(self._h))

    def gen_autokey_from_offline(self, offline1, offline2, auto1, auto2):
        """Reference genAutoKeyFromOffline (twosteps.cpp:1749-1864) on the
        device: dict(chain1, chain2, baby, giant, device_ms) in the layouts of
        kspir_gen_autokey_from_offline."""
        ins = [_u64(a).reshape(-1) for a in (offline1, offline2, auto1, auto2)]
        N1, N2 = self.N1, self.N2
        out = {"chain1": np.empty(max(N1 - 2, 0) * 12 * N, np.uint64),
               "chain2": np.empty(max(N2 - 2, 0) * 12 * N, np.uint64),
               "baby": np.empty((N1 - 1) * 12 * N, np.uint64), "giant": np.empty((N2 - 1) * 6 * N, np.uint64)}
        ms = ctypes.c_float()
        self._check(self.lib.kspir_gen_autokey_from_offline(self._h, *[ptr(a) for a in ins], ptr(out["chain1"]),
                                                            ptr(out["chain2"]), ptr(out["baby"]), ptr(out["giant"]),
                                                            ctypes.byref(ms)))
        out["device_ms"] = ms.value
        return out

    def set_fused(self, enable: bool):
        """Single answers as the one fused kernel (kspir_set_fused)."""
        self._check(self.lib.kspir_set_fused(self._h, 1 if enable else 0))

    @property
    def fused(self) -> bool:
        return self.lib.kspir_get_fused(self._h) == 1

    def debug_scan_fault(self, wait_limit_ns: int = 0, skip_item: int = -1):
        """Test hook (kspir_debug_scan_fault): the limit of the database scan's
        bounded device waits, and a work item the next single-answer scan skips."""
        self._check(self.lib.kspir_debug_scan_fault(self._h, wait_limit_ns, skip_item))

    def answer_batch(self, clients, queries, out: np.ndarray | None = None) -> np.ndarray:
        """Responses [n][2][N] of n queries ([n][2][2][N]) of the given client slots."""
        cl = np.ascontiguousarray(clients, dtype=np.int32).reshape(-1)
        q = _u64(queries).reshape(-1)
        n = cl.size
        if q.size != n * 4 * N:
            raise ValueError("queries must be [n][2][2][N]")
        if out is None:
            out = np.empty((n, 2 * N), dtype=np.uint64)
        self._check(self.lib.kspir_answer_batch(self._h, n, ptr(cl), ptr(q), ptr(out)))
        return out

    def answer_batch_device(self, clients, d_queries: int, d_responses: int, stream: int | None = None):
        cl = np.ascontiguousarray(clients, dtype=np.int32).reshape(-1)
        self._check(self.lib.kspir_answer_batch_device(self._h, cl.size, ptr(cl), ctypes.c_void_p(d_queries),
                                                       ctypes.c_void_p(d_responses),
                                                       ctypes.c_void_p(stream) if stream else None))

    def tune_batch(self, n: int):
        """Times every scan variant for batches of n; returns (chosen kind, {kind: ms})."""
        kind = ctypes.c_int()
        ms = (ctypes.c_float * 5)()
        self._check(self.lib.kspir_tune_batch(self._h, n, ctypes.byref(kind), ms))
        return kind.value, {k: ms[k] for k in range(5) if ms[k] < 1e29}

    def set_scan_kind(self, n: int, kind: int):
        self._check(self.lib.kspir_set_scan_kind(self._h, n, kind))

    def scan_kind(self, n: int) -> int:
        return self.lib.kspir_get_scan_kind(self._h, n)

    def last_timing(self):
        tot = ctypes.c_float()
        ph = (ctypes.c_float * 5)()
        self._check(self.lib.kspir_last_timing(self._h, ctypes.byref(tot), ph))
        return tot.value, list(ph)

    def timing_reset(self):
        self._check(self.lib.kspir_timing_reset(self._h))

    def timing_summary(self):
        """(answers, kernel launches, summed ms, summed ms per phase) since timing_reset."""
        n = ctypes.c_int()
        la = ctypes.c_long()
        tot = ctypes.c_float()
        ph = (ctypes.c_float * 5)()
        self._check(self.lib.kspir_timing_summary(self._h, ctypes.byref(n), ctypes.byref(la), ctypes.byref(tot), ph))
        return n.value, la.value, tot.value, list(ph)

    # -- the reference's three functions ------------------------------------
    def matrix_vector_mul(self, client: int, query):
        q = _u64(query).reshape(-1).copy()
        res = np.empty(self.r * 2 * N, dtype=np.uint64)
        self._check(self.lib.kspir_matrix_vector_mul_bsgs_rns_crt_large(self._h, client, ptr(q), ptr(res)))
        return res, q

    def external_product(self, client: int, result, first_dim):
        res = _u64(result).reshape(-1).copy()
        fd = _u64(first_dim).reshape(-1).copy()
        count = res.size // (2 * N)
        self._check(self.lib.kspir_external_product(self._h, client, ptr(res), ptr(fd), count))
        return res, fd

    def packing(self, client: int, rlwes, rlwes_out: np.ndarray | None = None):
        """The packed response of rlwes ([r][2][N]); rlwes_out (or None)
        receives rlwes as the reference's packingRLWEs leaves them."""
        rl = _u64(rlwes).reshape(-1).copy()
        out = np.empty(2 * N, dtype=np.uint64)
        self._check(self.lib.kspir_packing_rlwes(self._h, client, ptr(rl), ptr(out)))
        if rlwes_out is not None:
            rlwes_out.reshape(-1)[:] = rl
        return out

    def fetch_stage(self, stage: int, slot: int = 0) -> np.ndarray:
        sizes = {STAGE_CIPHERBUF: N * self.N1 * 2, STAGE_SCAN: self.r * self.N2 * 2 * N,
                 STAGE_RESULT: self.r * 2 * N, STAGE_EXT: self.r * 2 * N}
        out = np.empty(sizes[stage], dtype=np.uint64)
        self._check(self.lib.kspir_fetch_stage_slot(self._h, slot, stage, ptr(out), out.size))
        return out


class Server:
    """Serving loop over a Context (kspir_server_* of include/kspir_b200.h):
    continuous batching on `lanes` lanes of up to `lane_size` queries, client
    keys cached in device key slots within `key_budget_bytes`."""

    def __init__(self, ctx: Context, lanes: int = 2, lane_size: int = 64, key_budget_bytes: int = 0):
        self.ctx = ctx
        self.lib = ctx.lib
        self._h = ctypes.c_void_p()
        self._keep = {}      # caller-owned key arrays must outlive the server
        self._inflight = {}  # ticket -> (query, response) buffers
        p = ServerParams(lanes, lane_size, key_budget_bytes)
        self._check(self.lib.kspir_server_create(ctx.handle, ctypes.byref(p), ctypes.byref(self._h)))

    def _check(self, rc):
        if rc < 0:
            raise KspirError(rc, self.lib.kspir_last_error(self.ctx.handle).decode() or
                             self.lib.kspir_strerror(rc).decode())
        return rc

    def register(self, client: int, baby, giant, packing, rgsw):
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.uint64).reshape(-1)
                for a in (baby, giant, packing, rgsw)]
        self._keep[client] = arrs
        self._check(self.lib.kspir_server_register_client(self._h, client, *[ptr(a) for a in arrs]))

    def submit(self, client: int, query, out: np.ndarray | None = None) -> int:
        q = np.ascontiguousarray(query, dtype=np.uint64).reshape(-1)
        if out is None:
            out = np.empty(2 * N, dtype=np.uint64)
        t = ctypes.c_uint64()
        self._check(self.lib.kspir_server_submit(self._h, client, ptr(q), ptr(out), ctypes.byref(t)))
        self._inflight[t.value] = (q, out)
        return t.value

    def poll(self, ticket: int):
        """The response when done, else None."""
        rc = self._check(self.lib.kspir_server_poll(self._h, ticket))
        return self._inflight.pop(ticket)[1] if rc == 1 else None

    def wait(self, ticket: int, timeout_ms: int = 60000) -> np.ndarray:
        rc = self._check(self.lib.kspir_server_wait(self._h, ticket, timeout_ms))
        if rc != 1:
            raise TimeoutError(f"request {ticket} not done after {timeout_ms} ms")
        return self._inflight.pop(ticket)[1]

    def stats(self) -> dict:
        st = ServerStats()
        self._check(self.lib.kspir_server_get_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def reset_stats(self):
        self._check(self.lib.kspir_server_reset_stats(self._h))

    def latencies_us(self) -> np.ndarray:
        n = ctypes.c_size_t()
        self._check(self.lib.kspir_server_latencies(self._h, None, 0, ctypes.byref(n)))
        out = np.empty(n.value, dtype=np.float64)
        self._check(self.lib.kspir_server_latencies(self._h, ptr(out), out.size, ctypes.byref(n)))
        return out[:min(out.size, n.value)]

    def close(self):
        if self._h:
            self.lib.kspir_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
