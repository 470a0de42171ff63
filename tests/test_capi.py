"""The C-ABI boundary without a GPU: the library builds for sm_100a, loads,
exports every entry point include/kspir_b200.h declares, and rejects bad
arguments before touching the device."""
import ctypes
import os
import re
import subprocess

import pytest

from kspir_b200 import build as kbuild
from kspir_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "kspir_b200.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(kspir_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    kbuild.build()
    return native.load()


def test_header_declares_the_reference_boundary():
    names = declared_functions()
    for must in ("kspir_matrix_vector_mul_bsgs_rns_crt_large", "kspir_external_product", "kspir_packing_rlwes",
                 "kspir_answer", "kspir_db_upload", "kspir_client_keys_upload"):
        assert must in names


def test_library_exports_every_declared_symbol(lib):
    nm = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True, check=True)
    exported = set(re.findall(r"\bT (kspir_[a-z0-9_]+)", nm.stdout))
    for name in declared_functions():
        assert name in exported, name
        assert hasattr(lib, name)
    assert set(native.SIGNATURES) == set(declared_functions())


def test_invalid_params_rejected_before_device(lib):
    h = ctypes.c_void_p()
    for r, n1 in ((3, 128), (16, 100), (16, 16), (1024, 128), (0, 128)):
        p = native.Params(r, n1, 1, 1)
        assert lib.kspir_ctx_create(0, ctypes.byref(p), ctypes.byref(h)) == native.ERR_INVALID_ARG
    assert lib.kspir_ctx_create(0, None, ctypes.byref(h)) == native.ERR_INVALID_ARG


def test_strerror(lib):
    for code in (0, -1, -2, -3, -4, -5, -6, -7):
        assert lib.kspir_strerror(code)
    assert lib.kspir_answer(None, 0, None, None) == native.ERR_INVALID_ARG


@pytest.mark.parametrize("N1", [64, 128, 256])
def test_permutation_matrix_is_the_references(lib, N1):
    """kspir_permutation_matrix is host code: it must equal the oracle's
    compute_permutation_matrix (utils.cpp:1591-1619) and, where the reference
    is built here, the reference's own."""
    import numpy as np

    from oracle import pyoracle as po

    got = native.permutation_matrix(N1)
    assert (got == po.permutation_matrix(N1)).all()
    if po.ref_available():
        want = np.zeros(N1 * native.N, np.int32)
        po.ref().ref_permutation_matrix(po._p(want), N1)
        assert (got == want).all()


def test_permutation_matrix_rejects_bad_shapes(lib):
    import numpy as np

    out = np.zeros(128 * native.N, np.int32)   # rejected shapes write nothing
    for N1 in (0, -1, native.N // 2 + 1, 8192):
        assert lib.kspir_permutation_matrix(native.ptr(out), N1) == native.ERR_INVALID_ARG
    assert lib.kspir_permutation_matrix(None, 128) == native.ERR_INVALID_ARG
