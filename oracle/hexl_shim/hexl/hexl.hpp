// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle, never part of the product.
//
// A restatement of the subset of Intel HEXL v1.2.5 (`intel::hexl`, Apache-2.0,
// https://github.com/intel/hexl, tag v1.2.5) that the KsPIR reference calls on
// its online-answer path.  HEXL itself is a third-party dependency that is not
// vendored with the reference (reference CMakeLists.txt:32-35 does
// `find_package(HEXL 1.2.5 REQUIRED)`), so the oracle re-derives its published
// behaviour from the mathematics:
//
//   * NTT(n, q[, root]): negacyclic number-theoretic transform of length n over
//     Z_q.  Forward output slot j holds  sum_k x_k * psi^((2*bitrev(j)+1)*k)
//     (bit-reversed evaluation order; reference utils.cpp:1473-1478 relies on
//     exactly this order).  Without an explicit root, psi is HEXL's
//     MinimalPrimitiveRoot(2n, q): the smallest primitive 2n-th root of unity.
//     The inverse includes the factor n^-1.  Outputs are canonical ([0, q)).
//   * EltwiseAddMod / EltwiseSubMod: HEXL's single conditional correction,
//     i.e. (a+b >= q ? a+b-q : a+b) and (a >= b ? a-b : a+q-b).  These keep
//     HEXL's behaviour on the one non-canonical operand the reference feeds
//     them (a word equal to q, from `modulus - 0`).
//   * EltwiseMultMod / EltwiseFMAMod: exact canonical modular results.
//   * EltwiseReduceMod(result, operand, n, q, input_mod_factor,
//     output_mod_factor): HEXL documents that the operand is assumed to lie in
//     [0, input_mod_factor * q) and reduces it to [0, output_mod_factor * q);
//     with equal factors there is nothing to reduce and HEXL copies the
//     operand unchanged.  The reference's offline key derivation calls it with
//     factors (1, 1) on words that are not below q (twosteps.cpp:1776-1777,
//     1793-1794), so this restatement copies there too; every other call
//     reduces exactly.
//
// The transforms use Harvey's lazy butterflies with Shoup precomputation on
// 64-bit words (valid for q < 2^62); every value they return is the exact
// canonical residue, which is all the reference depends on.
#pragma once

#include <stdint.h>
#include <stddef.h>
#include <memory>
#include <vector>
#include <stdexcept>
// HEXL's public header pulls these in transitively; the reference relies on that.
#include <cmath>
#include <cstring>
#include <algorithm>
#include <iostream>

__extension__ typedef __int128 int128_t;
__extension__ typedef unsigned __int128 uint128_t;

namespace intel {
namespace hexl {

namespace shim_detail {

inline uint64_t mulhi64(uint64_t a, uint64_t b) {
    return (uint64_t)(((uint128_t)a * b) >> 64);
}

inline uint64_t mulmod_exact(uint64_t a, uint64_t b, uint64_t q) {
    return (uint64_t)(((uint128_t)a * b) % q);
}

inline uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = mulmod_exact(r, a, q);
        a = mulmod_exact(a, a, q);
        e >>= 1;
    }
    return r;
}

// Modular inverse by the extended Euclidean algorithm (q need not be prime).
inline uint64_t invmod(uint64_t a, uint64_t q) {
    int128_t t = 0, newt = 1;
    int128_t r = q, newr = a % q;
    while (newr != 0) {
        int128_t quo = r / newr;
        int128_t tmp = t - quo * newt; t = newt; newt = tmp;
        tmp = r - quo * newr; r = newr; newr = tmp;
    }
    if (r != 1) throw std::invalid_argument("hexl shim: value not invertible");
    if (t < 0) t += q;
    return (uint64_t)t;
}

inline uint64_t bitrev(uint64_t x, int bits) {
    uint64_t r = 0;
    for (int i = 0; i < bits; i++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

// floor(w * 2^64 / q), the Shoup companion of a constant w < q.
inline uint64_t shoup(uint64_t w, uint64_t q) {
    return (uint64_t)(((uint128_t)w << 64) / q);
}

// x * w mod q, lazily in [0, 2q), for any 64-bit x.
inline uint64_t shoup_mul_lazy(uint64_t x, uint64_t w, uint64_t wp, uint64_t q) {
    uint64_t t = mulhi64(x, wp);
    return x * w - t * q;
}

// Barrett reduction of a 128-bit product for q < 2^62: mu = floor(2^128 / q).
struct Barrett128 {
    uint64_t q = 0, mu_hi = 0, mu_lo = 0;
    Barrett128() = default;
    explicit Barrett128(uint64_t modulus_value) : q(modulus_value) {
        // floor(2^128 / q) computed as ((2^128 - 1) / q) (q is never a power of two here)
        uint128_t all = ~(uint128_t)0;
        uint128_t mu = all / q;
        mu_hi = (uint64_t)(mu >> 64);
        mu_lo = (uint64_t)mu;
    }
    inline uint64_t reduce(uint128_t z) const {
        uint64_t zl = (uint64_t)z, zh = (uint64_t)(z >> 64);
        // quotient estimate floor(z * mu / 2^128), up to 2 below the true quotient
        uint128_t t = ((uint128_t)zl * mu_lo) >> 64;
        t += (uint128_t)zl * mu_hi;
        uint128_t u = (uint128_t)zh * mu_lo + (uint64_t)t;
        uint64_t qhat = (uint64_t)(t >> 64) + (uint64_t)(u >> 64) + zh * mu_hi;
        uint64_t r = zl - qhat * q;
        while (r >= q) r -= q;
        return r;
    }
    inline uint64_t mul(uint64_t a, uint64_t b) const { return reduce((uint128_t)a * b); }
};

struct NttTables {
    uint64_t n = 0, q = 0, root = 0;
    int logn = 0;
    std::vector<uint64_t> w, wp, iw, iwp;  // psi^{brv(k)} and psi^{-brv(k)}, with Shoup companions
    uint64_t ninv = 0, ninvp = 0;
};

}  // namespace shim_detail

// Smallest primitive `degree`-th root of unity modulo prime q (degree a power of two).
inline uint64_t MinimalPrimitiveRoot(uint64_t degree, uint64_t q) {
    using namespace shim_detail;
    if ((q - 1) % degree != 0) throw std::invalid_argument("hexl shim: q != 1 mod degree");
    uint64_t root = 0;
    for (uint64_t g = 2; g < q; g++) {
        uint64_t c = powmod(g, (q - 1) / degree, q);
        if (powmod(c, degree / 2, q) == q - 1) { root = c; break; }
    }
    if (!root) throw std::invalid_argument("hexl shim: no primitive root");
    // all primitive degree-th roots are the odd powers of one of them
    uint64_t sq = mulmod_exact(root, root, q), cur = root, best = root;
    for (uint64_t i = 0; i < degree / 2; i++) {
        if (cur < best) best = cur;
        cur = mulmod_exact(cur, sq, q);
    }
    return best;
}

class NTT {
public:
    NTT() = default;
    NTT(uint64_t degree, uint64_t q) : NTT(degree, q, MinimalPrimitiveRoot(2 * degree, q)) {}
    NTT(uint64_t degree, uint64_t q, uint64_t root_of_unity) {
        using namespace shim_detail;
        auto t = std::make_shared<NttTables>();
        t->n = degree; t->q = q; t->root = root_of_unity;
        while ((1ULL << t->logn) < degree) t->logn++;
        if ((1ULL << t->logn) != degree) throw std::invalid_argument("hexl shim: degree not a power of two");
        if (powmod(root_of_unity, degree, q) != q - 1) throw std::invalid_argument("hexl shim: not a primitive 2n-th root");
        uint64_t rinv = invmod(root_of_unity, q);
        t->w.resize(degree); t->wp.resize(degree); t->iw.resize(degree); t->iwp.resize(degree);
        for (uint64_t k = 0; k < degree; k++) {
            uint64_t e = bitrev(k, t->logn);
            t->w[k] = powmod(root_of_unity, e, q);
            t->iw[k] = powmod(rinv, e, q);
            t->wp[k] = shoup(t->w[k], q);
            t->iwp[k] = shoup(t->iw[k], q);
        }
        t->ninv = invmod(degree % q, q);
        t->ninvp = shoup(t->ninv, q);
        tables_ = t;
    }

    uint64_t GetModulus() const { return tables_->q; }
    uint64_t GetDegree() const { return tables_->n; }
    uint64_t GetMinimalRootOfUnity() const { return tables_->root; }
    uint64_t GetRootOfUnityPower(size_t i) const { return tables_->w[i]; }

    // Cooley-Tukey, natural order in, bit-reversed order out.
    void ComputeForward(uint64_t* result, const uint64_t* operand,
                        uint64_t /*input_mod_factor*/, uint64_t /*output_mod_factor*/) const {
        using namespace shim_detail;
        const NttTables& t = *tables_;
        const uint64_t n = t.n, q = t.q, q2 = 2 * q;
        for (uint64_t i = 0; i < n; i++) {
            uint64_t x = operand[i];
            result[i] = x < q ? x : x % q;
        }
        for (uint64_t m = 1, h = n >> 1; m < n; m <<= 1, h >>= 1) {
            for (uint64_t i = 0; i < m; i++) {
                const uint64_t W = t.w[m + i], Wp = t.wp[m + i];
                uint64_t* X = result + 2 * i * h;
                uint64_t* Y = X + h;
                for (uint64_t j = 0; j < h; j++) {
                    uint64_t x = X[j];
                    if (x >= q2) x -= q2;                       // [0, 2q)
                    uint64_t wy = shoup_mul_lazy(Y[j], W, Wp, q); // [0, 2q)
                    X[j] = x + wy;                              // [0, 4q)
                    Y[j] = x - wy + q2;                         // (0, 4q)
                }
            }
        }
        for (uint64_t i = 0; i < n; i++) {
            uint64_t x = result[i];
            if (x >= q2) x -= q2;
            if (x >= q) x -= q;
            result[i] = x;
        }
    }

    // Gentleman-Sande, bit-reversed order in, natural order out, times n^-1.
    void ComputeInverse(uint64_t* result, const uint64_t* operand,
                        uint64_t /*input_mod_factor*/, uint64_t /*output_mod_factor*/) const {
        using namespace shim_detail;
        const NttTables& t = *tables_;
        const uint64_t n = t.n, q = t.q, q2 = 2 * q;
        for (uint64_t i = 0; i < n; i++) {
            uint64_t x = operand[i];
            result[i] = x < q ? x : x % q;
        }
        for (uint64_t m = n >> 1, h = 1; m >= 1; m >>= 1, h <<= 1) {
            for (uint64_t i = 0; i < m; i++) {
                const uint64_t W = t.iw[m + i], Wp = t.iwp[m + i];
                uint64_t* X = result + 2 * i * h;
                uint64_t* Y = X + h;
                for (uint64_t j = 0; j < h; j++) {
                    uint64_t x = X[j], y = Y[j];                // [0, 2q)
                    uint64_t s = x + y;
                    if (s >= q2) s -= q2;
                    X[j] = s;
                    Y[j] = shoup_mul_lazy(x - y + q2, W, Wp, q); // [0, 2q)
                }
            }
        }
        for (uint64_t i = 0; i < n; i++) {
            uint64_t x = shoup_mul_lazy(result[i], t.ninv, t.ninvp, q);
            if (x >= q) x -= q;
            result[i] = x;
        }
    }

private:
    std::shared_ptr<const shim_detail::NttTables> tables_;
};

inline void EltwiseAddMod(uint64_t* result, const uint64_t* operand1,
                          const uint64_t* operand2, uint64_t n, uint64_t modulus) {
    for (uint64_t i = 0; i < n; i++) {
        uint64_t s = operand1[i] + operand2[i];
        result[i] = s >= modulus ? s - modulus : s;
    }
}

inline void EltwiseAddMod(uint64_t* result, const uint64_t* operand1,
                          uint64_t operand2, uint64_t n, uint64_t modulus) {
    for (uint64_t i = 0; i < n; i++) {
        uint64_t s = operand1[i] + operand2;
        result[i] = s >= modulus ? s - modulus : s;
    }
}

inline void EltwiseSubMod(uint64_t* result, const uint64_t* operand1,
                          const uint64_t* operand2, uint64_t n, uint64_t modulus) {
    for (uint64_t i = 0; i < n; i++) {
        uint64_t a = operand1[i], b = operand2[i];
        result[i] = a >= b ? a - b : a + modulus - b;
    }
}

inline void EltwiseSubMod(uint64_t* result, const uint64_t* operand1,
                          uint64_t operand2, uint64_t n, uint64_t modulus) {
    for (uint64_t i = 0; i < n; i++) {
        uint64_t a = operand1[i];
        result[i] = a >= operand2 ? a - operand2 : a + modulus - operand2;
    }
}

inline void EltwiseMultMod(uint64_t* result, const uint64_t* operand1,
                           const uint64_t* operand2, uint64_t n, uint64_t modulus,
                           uint64_t /*input_mod_factor*/) {
    shim_detail::Barrett128 br(modulus);
    for (uint64_t i = 0; i < n; i++) result[i] = br.mul(operand1[i], operand2[i]);
}

inline void EltwiseFMAMod(uint64_t* result, const uint64_t* arg1, uint64_t arg2,
                          const uint64_t* arg3, uint64_t n, uint64_t modulus,
                          uint64_t /*input_mod_factor*/) {
    shim_detail::Barrett128 br(modulus);
    uint64_t c = arg2 % modulus;
    for (uint64_t i = 0; i < n; i++) {
        uint128_t z = (uint128_t)arg1[i] * c;
        if (arg3) z += arg3[i];
        result[i] = br.reduce(z);
    }
}

inline void EltwiseReduceMod(uint64_t* result, const uint64_t* operand, uint64_t n,
                             uint64_t modulus, uint64_t input_mod_factor,
                             uint64_t output_mod_factor) {
    if (input_mod_factor == output_mod_factor) {
        if (result != operand) std::memcpy(result, operand, n * sizeof(uint64_t));
        return;
    }
    for (uint64_t i = 0; i < n; i++) result[i] = operand[i] % modulus;
}

}  // namespace hexl
}  // namespace intel
