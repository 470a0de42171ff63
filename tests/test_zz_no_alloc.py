"""The allocation-free external product (kspir_external_product_noalloc).

This entry point exists for callers that cannot call cudaMalloc -- a plugin
whose host process owns all device memory through its own pool, or code that
must not cause the device synchronisation an allocation can.  Its scratch is a
fixed device array inside the library, shared by every call.

The test calls it through the C ABI on device buffers the test owns, twice in
a row, and checks every output word against the context-based
kspir_external_product (the integer path is bit-exact, so the tolerance is
zero).  It lives in its own file, collected last, and passes alone in a fresh
process as well as after the other tests.
"""
import ctypes

import numpy as np
import pytest

import kspir_b200 as kb
from kspir_b200 import native
from kspir_b200 import synth

pytestmark = pytest.mark.gpu
N = native.N


def _inputs(seed, count):
    rng = np.random.default_rng(seed)
    rgsw = rng.integers(0, native.CRTMOD, 4 * 2 * N, dtype=np.uint64)
    acc = rng.integers(0, native.CRTMOD, count * 2 * N, dtype=np.uint64)
    acc[: 2 * N] = 0      # a fresh product starts from zero accumulators
    fd = rng.integers(0, native.CRTMOD, count * 2 * N, dtype=np.uint64)
    return rgsw, acc, fd


def _existing(rgsw, acc, fd, count):
    with kb.Context(16, 128) as ctx:
        c = synth.gen_client(1, 16, 128)
        ctx.upload_client(0, c["baby"], c["giant"], c["packing"], rgsw)
        return ctx.external_product(0, acc, fd)


def _noalloc(lib, torch, rgsw, acc, fd, count, stream):
    d_rgsw = torch.from_numpy(rgsw.view(np.int64).copy()).cuda()
    d_res = torch.from_numpy(acc.view(np.int64).copy()).cuda()
    d_fd = torch.from_numpy(fd.view(np.int64).copy()).cuda()
    torch.cuda.synchronize()
    rc = lib.kspir_external_product_noalloc(0, ctypes.c_void_p(d_rgsw.data_ptr()), ctypes.c_void_p(d_res.data_ptr()),
                                            ctypes.c_void_p(d_fd.data_ptr()), count, ctypes.c_void_p(stream))
    return rc, d_res.cpu().numpy().view(np.uint64), d_fd.cpu().numpy().view(np.uint64)


def test_noalloc_matches_context_path_twice():
    torch = pytest.importorskip("torch")
    lib = native.load()
    stream = torch.cuda.Stream()
    for call, (seed, count) in enumerate(((11, 3), (12, 5))):
        rgsw, acc, fd = _inputs(seed, count)
        want_res, want_fd = _existing(rgsw, acc, fd, count)
        rc, got_res, got_fd = _noalloc(lib, torch, rgsw, acc, fd, count, stream.cuda_stream)
        assert rc == native.OK, f"call {call}: rc={rc}"
        assert np.array_equal(got_res, want_res), f"call {call}: results differ"
        assert np.array_equal(got_fd, want_fd), f"call {call}: first_dim differs"


def test_noalloc_full_scratch_and_oracle():
    # count = KSPIR_NOALLOC_MAX_COUNT fills the whole static scratch and job
    # list; every ciphertext equals the context path, and two of them the
    # oracle's externalProduct (lwe.cpp:761-808) directly
    torch = pytest.importorskip("torch")
    from oracle import pyoracle as po
    lib = native.load()
    count = 16
    rgsw, acc, fd = _inputs(14, count)
    rc, got_res, got_fd = _noalloc(lib, torch, rgsw, acc, fd, count, 0)
    assert rc == native.OK
    want_res, want_fd = _existing(rgsw, acc, fd, count)
    assert np.array_equal(got_res, want_res)
    assert np.array_equal(got_fd, want_fd)
    for j in (0, count - 1):
        s = slice(j * 2 * N, (j + 1) * 2 * N)
        e, f = po.external_product(fd[s], rgsw, ext=acc[s])
        assert np.array_equal(got_res[s], e), f"ciphertext {j}: result"
        assert np.array_equal(got_fd[s], f), f"ciphertext {j}: first_dim"


def test_noalloc_rejects_oversize_and_bad_words():
    torch = pytest.importorskip("torch")
    lib = native.load()
    rgsw, acc, fd = _inputs(13, 2)
    rc, _, _ = _noalloc(lib, torch, rgsw, np.zeros(17 * 2 * N, np.uint64), np.zeros(17 * 2 * N, np.uint64), 17, 0)
    assert rc == native.ERR_INVALID_ARG
    bad = fd.copy()
    bad[5] = native.CRTMOD
    rc, got_res, _ = _noalloc(lib, torch, rgsw, acc, bad, 2, 0)
    assert rc == native.ERR_INVALID_ARG
    assert np.array_equal(got_res, acc)   # outputs untouched
