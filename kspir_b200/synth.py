"""Seeded synthetic inputs with the shapes and value ranges of the reference's
online answer (the reference samples its database and keys with glibc rand();
these stand in for them, with every word canonical for its modulus).

* ``gen_db``: a preprocessed database in the packed CRT layout of
  database_tocrt (reference src/crt.cpp:859-885): word = (v mod q1) | (v mod q2) << 32,
  v uniform mod crtMod -- r sub-databases of N x N/2 words (r = 16: the
  256 MB-record database of tests/test-pir.cpp, 1 GiB preprocessed).
* ``gen_raw_db``: a database before preprocessing (input of
  database_tobsgsntt, reference src/twosteps.cpp:42): r sub-databases of
  N x N/2 plaintext words uniform in [0, bsgsp = 65537).
* ``gen_client``: query (mod crtMod, mod bsMod), baby/giant/packing keys and
  the RGSW query, uniformly random canonical words in the layouts of
  include/kspir_b200.h.
"""
from __future__ import annotations

import numpy as np

N = 4096
Q1 = 268369921
Q2 = 249561089
CRTMOD = Q1 * Q2
BSMOD = 16760833
P = 65537


def _uniform(rng, n, q):
    return rng.integers(0, q, size=n, dtype=np.uint64)


def gen_db(seed: int, r: int, N1: int) -> np.ndarray:
    rng = np.random.default_rng(np.random.SeedSequence([seed, 0xDB]))
    n = r * N * N // 2
    out = np.empty(n, dtype=np.uint64)
    step = 1 << 24
    for s in range(0, n, step):
        m = min(step, n - s)
        lo = rng.integers(0, Q1, size=m, dtype=np.uint64)
        hi = rng.integers(0, Q2, size=m, dtype=np.uint64)
        out[s:s + m] = lo | (hi << np.uint64(32))
    return out


def gen_raw_db(seed: int, r: int) -> np.ndarray:
    rng = np.random.default_rng(np.random.SeedSequence([seed, 0xDA]))
    return rng.integers(0, P, size=r * N * N // 2, dtype=np.uint64)


def edge_raw_db() -> np.ndarray:
    """One raw sub-database cycling through the edge values of the signed lift
    (v > bsgsp / 2, reference twosteps.cpp:165-166) and of the input range."""
    edges = np.array([0, 1, 2, 32767, 32768, 32769, 32770, 65535, 65536], np.uint64)
    return np.resize(edges, N * N // 2)


def gen_client(seed: int, r: int, N1: int) -> dict:
    N2 = N // 2 // N1
    levels = int(r).bit_length() - 1
    rng = np.random.default_rng(np.random.SeedSequence([seed, 0xC1]))
    q = np.concatenate([_uniform(rng, 2 * N, CRTMOD), _uniform(rng, 2 * N, BSMOD)])
    baby = np.empty((N1 // 2, 6, 2 * N), dtype=np.uint64)
    baby[:, :3] = _uniform(rng, (N1 // 2) * 3 * 2 * N, CRTMOD).reshape(N1 // 2, 3, 2 * N)
    baby[:, 3:] = _uniform(rng, (N1 // 2) * 3 * 2 * N, BSMOD).reshape(N1 // 2, 3, 2 * N)
    giant = _uniform(rng, (N2 - 1) * 2 * 2 * N, CRTMOD)
    packing = _uniform(rng, levels * 4 * 2 * N, CRTMOD)
    rgsw = _uniform(rng, 4 * 2 * N, CRTMOD)
    return dict(query=q, baby=baby.reshape(-1), giant=giant, packing=packing, rgsw=rgsw)
