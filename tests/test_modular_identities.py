"""The word-level identities the CUDA kernels rely on, restated on Python
integers with 32- and 64-bit wrap-around, checked on edge values and seeded
random words for the three moduli of the path (crt.h:16-17, 32).

- reduce64 (csrc/common.cuh): Barrett with floor(2^64 / q), the quotient
  estimate truncated to 32 bits, then one unsigned-minimum correction.
- add / sub / negate / signed-to-residue / Shoup multiply as unsigned minima
  (for x < 2m, x - m wraps above x exactly when x < m).
- canon4q: a lazy transform output in [0, 4q) back to canonical.
- the giant-step accumulator (csrc/k_second.cuh): at most 16 canonical terms
  per u32 word, and the split of N1 = 64's 31 giant steps over two words.
- the 64-bit multiply-accumulates fed by lazy [0, 4q) digits do not wrap.
"""
import numpy as np
import pytest

Q1, Q2, BS = 268369921, 249561089, 16760833
M32, M64 = (1 << 32) - 1, (1 << 64) - 1
N = 4096


def umin(a, b):
    return a if a < b else b


def reduce64(p, q):
    barrett = (1 << 64) // q
    qh = ((p * barrett) >> 64) & M32
    r = (p - qh * q) & M32
    return umin(r, (r - q) & M32)


def addmod(a, b, q):
    s = (a + b) & M32
    return umin(s, (s - q) & M32)


def submod(a, b, q):
    d = (a - b) & M32
    return umin(d, (d + q) & M32)


def negmod(x, q):
    return umin((q - x) & M32, (0 - x) & M32)


def signed_to_res(v, q):
    u = v & M32
    return umin(u, (u + q) & M32)


def shoup_mul(x, w, q):
    wp = (w << 32) // q
    t = (x * wp) >> 32
    r = (x * w - t * q) & M32
    return umin(r, (r - q) & M32)


def canon4q(x, q):
    x = umin(x, (x - 2 * q) & M32)
    return umin(x, (x - q) & M32)


def edge_words(q):
    out = [0, 1, q - 1, q, q + 1, 2 * q - 1, 2 * q, 3 * q + 5, (q - 1) ** 2, 4 * (q - 1) ** 2,
           (1 << 32) - 1, 1 << 32, (1 << 63) - 1, 1 << 63, M64, M64 - q, (M64 // q) * q, (M64 // q) * q - 1]
    return [w for w in out if 0 <= w <= M64]


@pytest.mark.parametrize("q", [Q1, Q2, BS])
def test_reduce64_exact(q):
    rng = np.random.default_rng(q)
    words = edge_words(q) + [int(x) for x in rng.integers(0, 1 << 63, 20000, dtype=np.uint64)] \
        + [int(x) << 1 | 1 for x in rng.integers(0, 1 << 63, 5000, dtype=np.uint64)]
    for p in words:
        assert reduce64(p, q) == p % q, p


@pytest.mark.parametrize("q", [Q1, Q2, BS])
def test_minimum_form_residue_ops(q):
    rng = np.random.default_rng(q + 1)
    vals = [0, 1, q - 1, q // 2] + [int(x) for x in rng.integers(0, q, 3000)]
    for a, b in zip(vals, vals[::-1]):
        assert addmod(a, b, q) == (a + b) % q
        assert submod(a, b, q) == (a - b) % q
        assert negmod(a, q) == (-a) % q
    for v in [0, 1, -1, q - 1, -(q - 1)] + [int(x) for x in rng.integers(-(q - 1), q, 3000)]:
        assert signed_to_res(v, q) == v % q
    for w in [0, 1, q - 1] + [int(x) for x in rng.integers(0, q, 50)]:
        for x in [0, 1, q - 1, 2 * q - 1, M32] + [int(y) for y in rng.integers(0, 1 << 32, 50, dtype=np.uint64)]:
            assert shoup_mul(x, w, q) == (x * w) % q


@pytest.mark.parametrize("q", [Q1, Q2, BS])
def test_lazy_transform_outputs_canonicalise(q):
    assert 4 * q <= M32                     # [0, 4q) words fit in 32 bits
    rng = np.random.default_rng(q + 2)
    for x in [0, q - 1, q, 2 * q - 1, 2 * q, 3 * q, 4 * q - 1] + [int(y) for y in rng.integers(0, 4 * q, 5000)]:
        assert canon4q(x, q) == x % q


def test_lazy_digits_feed_wide_accumulators_without_wrap():
    # ell lazy digits (< 4q) times canonical key words (< q), summed in 64 bits
    for q, ell in ((Q1, 4), (Q2, 4), (BS, 4)):
        assert ell * (4 * q - 1) * (q - 1) <= M64


def test_giant_accumulator_bound():
    per_word = 16
    assert per_word * (Q1 - 1) <= M32 < (per_word + 1) * (Q1 - 1)
    assert Q2 < Q1
    for N1 in (64, 128, 256):
        N2 = N // 2 // N1
        steps = list(range(1, N2))
        if len(steps) > per_word:           # two words: rows c odd and c even
            odd = [c for c in steps if c & 1]
            even = [c for c in steps if not c & 1]
            assert len(odd) <= per_word and len(even) <= per_word
            words = 2
        else:
            words = 1
        # k_giant_finish adds output[0] (< q) to the words in 64 bits
        assert words * per_word * (Q1 - 1) + (Q1 - 1) <= M64
        assert (N1, words) in ((64, 2), (128, 1), (256, 1))
