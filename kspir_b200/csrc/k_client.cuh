// The client side of the protocol on the device, for test clients and load
// generation: the query of query_bsgs_rns (reference twosteps.cpp:279-318,
// encrypt_rns_bsgs encrypt.cpp:443-493 with encrypt encrypt.cpp:117-152) and
// the decryption decrypt_bsgs_total (twosteps.cpp:388-418).
//
// Query of row t for secret s (coefficients mod crtMod, small):
//   m  = 0 except m[query_encode[t]] = m[query_encode[N-1-t]] = 1
//   me = INTT_p(m);  dm_i = round((long double)me_i * crtMod / p)   (twosteps.cpp:296-307;
//        the reference's unqualified round is round(double): the long double
//        quotient is rounded to a double first)
//   crt part:  a1 uniform (NTT form), b1 = a1 * NTT(s) + NTT(dm * bsMod + e)   mod crtMod
//   bs part:   a2 uniform (NTT form), b2 = a2 * NTT(s~) + NTT(e~)             mod bsMod
//   then all four to coefficient form (encrypt_rns_bsgs, encrypt.cpp:486-491);
//   e ternary, the same e in both parts, s~ and e~ their centred lifts mod
//   bsMod (guass_to_modulus, samples.cpp:56-65).
// dm depends only on me_i < p: the host computes it once, with the
// reference's own expression (x87 long double there too), into a 65537-entry
// table.
//
// Randomness: the reference draws a, e and s from glibc rand(); a device
// client draws them from Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), a
// counter-based generator: word j of stream k of query q is a pure function
// of (seed, q, k, j), so every CTA regenerates the e it shares with the
// others.  Uniform residues come from 64 random bits mod q (the pair
// (a mod q1, a mod q2) is then uniform mod crtMod by CRT); e is uniform in
// {-1, 0, 1} from 32 bits mod 3.
#pragma once

#include "common.cuh"
#include "ntt.cuh"

namespace kspir {

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int i = 0; i < 10; i++) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// 64 random bits: word j of stream `stream` of query q
__device__ __forceinline__ uint64_t client_rand64(uint64_t seed, uint32_t q, uint32_t stream, uint32_t j) {
    const uint4 r = philox4x32_10(make_uint4(j, stream, q, 0x6b737072u),
                                  make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    return (uint64_t)r.x | (uint64_t)r.y << 32;
}

enum ClientStream : uint32_t { RS_A_Q1 = 0, RS_A_Q2 = 1, RS_A_BS = 2, RS_ERR = 3 };

// e_j in {-1, 0, 1} as (value mod q)
__device__ __forceinline__ uint32_t client_err(uint64_t seed, uint32_t q, uint32_t j, uint32_t mod) {
    const uint32_t t = (uint32_t)client_rand64(seed, q, RS_ERR, j) % 3u;
    return t == 0 ? mod - 1 : t - 1;
}

// centred lift of a small secret word mod crtMod into channel ch
// (guass_to_modulus for bsMod; for the crt primes the plain residue)
__device__ __forceinline__ uint32_t secret_res(uint64_t s, int ch) {
    if (ch == CH_BS) return s > kCrtMod / 2 ? (uint32_t)(s + kBsMod - kCrtMod) : (uint32_t)s;
    return (uint32_t)(s % (ch == CH_Q1 ? kQ1 : kQ2));
}

struct ClientQueryArgs {
    const uint64_t* secrets;   // [n][N] coefficient form mod crtMod
    const uint32_t* rows;      // [n] target rows < N/2
    const int32_t* qenc;       // [N] query_encode
    const uint64_t* dm;        // [p] the scaled message of each me < p (host table)
    uint64_t seed;
    uint32_t* out;             // [n][3 ch][2 (a, b)][N] residues, coefficient form
};

constexpr int kClientSmem = 2 * kN * 8 + 3 * kPadN * 4;   // forward + inverse twiddles, 3 polynomials

// grid (3 channels: q1, q2, bsMod; n queries), 512 threads
__global__ void __launch_bounds__(kNttThreads) k_client_query(ClientQueryArgs a, NttTables tabs) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* twf = reinterpret_cast<uint2*>(smem_raw);
    uint2* twi = twf + kN;
    uint32_t* S = reinterpret_cast<uint32_t*>(smem_raw + 2 * kN * 8);
    uint32_t* A = S + kPadN;
    uint32_t* T = A + kPadN;
    const int ch = blockIdx.x == 0 ? CH_Q1 : blockIdx.x == 1 ? CH_Q2 : CH_BS;
    const uint32_t qi = blockIdx.y, tid = threadIdx.x;
    const uint32_t q = c_dev.ch[ch].q;
    const uint64_t* s = a.secrets + (size_t)qi * kN;
    const uint32_t row = a.rows[qi];

    // me = INTT_p(m) first (its twiddles in twf), then the channel's tables
    stage_twiddles(twf, tabs, CH_P, NTT_INV);
    for (int i = tid; i < kN; i += kNttThreads) T[pidx(i)] = 0;
    __syncthreads();
    if (tid == 0) {
        T[pidx(a.qenc[row])] = 1;
        T[pidx(a.qenc[kN - 1 - row])] = 1;
    }
    cta_ntt_inverse(T, twf, CH_P);
    stage_twiddles(twf, tabs, ch, NTT_FWD);
    stage_twiddles(twi, tabs, ch, NTT_INV);
    const uint32_t bsq = ch == CH_BS ? 0u : (uint32_t)(kBsMod % q);
    for (int i = tid; i < kN; i += kNttThreads) {
        const uint32_t e = client_err(a.seed, qi, i, q);
        uint32_t t = e;
        if (ch != CH_BS) {
            // dm * bsMod + e mod q (encrypt.cpp:144)
            const uint32_t dm = (uint32_t)(a.dm[T[pidx(i)]] % q);
            t = addmod(mulmod(dm, bsq, ch), e, q);
        }
        T[pidx(i)] = t;
        S[pidx(i)] = secret_res(s[i], ch);
        const uint32_t stream = ch == CH_Q1 ? RS_A_Q1 : ch == CH_Q2 ? RS_A_Q2 : RS_A_BS;
        A[pidx(i)] = (uint32_t)(client_rand64(a.seed, qi, stream, i) % q);
    }
    cta_ntt_forward_m<2>(S, 2 * kPadN, twf, ch);   // S and T
    for (int i = tid; i < kN; i += kNttThreads) {
        const int p = pidx(i);
        S[p] = addmod(mulmod(A[p], S[p], ch), T[p], q);   // b = a * s + t, NTT form
    }
    cta_ntt_inverse_m<2>(S, kPadN, twi, ch);           // b (S) and a (A) to coefficient form
    uint32_t* o = a.out + ((size_t)qi * 3 + (ch == CH_Q1 ? 0 : ch == CH_Q2 ? 1 : 2)) * 2 * kN;
    for (int i = tid; i < kN; i += kNttThreads) {
        o[i] = A[pidx(i)];
        o[kN + i] = S[pidx(i)];
    }
}

// residues -> query words [n][2][2][N]: (a, b) mod crtMod, then (a, b) mod bsMod
__global__ void k_client_query_words(const uint32_t* __restrict__ res, uint64_t* __restrict__ query, int n) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * 2 * kN) return;
    const long qi = idx / (2 * kN);
    const int j = (int)(idx % (2 * kN));   // comp * N + k
    const uint32_t* r = res + qi * 3 * 2 * kN;
    uint64_t* o = query + qi * 4 * kN;
    o[j] = crt_compose_res(r[j], r[2 * kN + j]);
    o[2 * kN + j] = r[4 * kN + j];
}

// decrypt_bsgs_total up to the rounding, one CTA per (crt prime, response):
// out = INTT(NTT(b) - NTT(a) * NTT(s)) * qinv   (residues, coefficient form)
__global__ void __launch_bounds__(kNttThreads) k_client_decrypt(const uint64_t* __restrict__ secrets,
                                                                const uint64_t* __restrict__ resp, uint64_t qinv,
                                                                uint32_t* __restrict__ out, NttTables tabs) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* twf = reinterpret_cast<uint2*>(smem_raw);
    uint2* twi = twf + kN;
    uint32_t* P = reinterpret_cast<uint32_t*>(smem_raw + 2 * kN * 8);   // a, b, s
    const int ch = blockIdx.x;
    const uint32_t qi = blockIdx.y, tid = threadIdx.x;
    const uint32_t q = c_dev.ch[ch].q;
    const uint64_t* rp = resp + (size_t)qi * 2 * kN;
    const uint64_t* s = secrets + (size_t)qi * kN;
    stage_twiddles(twf, tabs, ch, NTT_FWD);
    stage_twiddles(twi, tabs, ch, NTT_INV);
    for (int i = tid; i < kN; i += kNttThreads) {
        P[pidx(i)] = (uint32_t)(rp[i] % q);
        P[kPadN + pidx(i)] = (uint32_t)(rp[kN + i] % q);
        P[2 * kPadN + pidx(i)] = (uint32_t)(s[i] % q);
    }
    cta_ntt_forward_m<3>(P, kPadN, twf, ch);
    const uint32_t qv = (uint32_t)(qinv % q);
    for (int i = tid; i < kN; i += kNttThreads) {
        const int p = pidx(i);
        const uint32_t as = mulmod(P[p], P[2 * kPadN + p], ch);
        P[kPadN + p] = mulmod(submod(P[kPadN + p], as, q), qv, ch);   // INTT is linear: scale first
    }
    cta_ntt_inverse(P + kPadN, twi, ch);
    uint32_t* o = out + ((size_t)qi * 2 + ch) * kN;
    for (int i = tid; i < kN; i += kNttThreads) o[i] = P[kPadN + pidx(i)];
}

// The rounding of decrypt_bsgs_total (twosteps.cpp:407-417) on the composed
// value me mod crtMod: me > crtMod/2 -> round((me - crtMod) / Delta) + p, else
// round(me / Delta), Delta = bsgsDelta, as the reference compiles it: the
// quotient is a long double (64-bit significand, rounded to nearest even),
// the unqualified round is the C library's round(double), so the quotient is
// rounded again to a double (53-bit significand, nearest even), then to an
// integer (halves away from zero).  round_ref_quotient reproduces the three
// roundings exactly in integer arithmetic (all of them are symmetric in sign,
// so the negative branch is minus the positive one).
constexpr uint64_t kBsgsDelta = 1021937069741ull;   // params.h:98

__device__ __forceinline__ int bitlen64(uint64_t x) { return x ? 64 - __clzll((long long)x) : 0; }

// round(double(long double(y) / Delta)) for 0 <= y < 2^56
__device__ __forceinline__ uint64_t round_ref_quotient(uint64_t y) {
    if (y == 0) return 0;
    using u128 = unsigned __int128;
    // exponent e of x = y / Delta (2^e <= x < 2^(e+1)), -40 <= e <= 16
    int e = bitlen64(y) - bitlen64(kBsgsDelta);
    u128 num = e <= 63 ? (u128)y << (63 - e) : (u128)y >> (e - 63);
    uint64_t q = (uint64_t)(num / kBsgsDelta);
    if (q < (1ull << 63)) {   // x < 2^e after all
        e -= 1;
        num = (u128)y << (63 - e);
        q = (uint64_t)(num / kBsgsDelta);
    }
    const uint64_t rem = (uint64_t)(num - (u128)q * kBsgsDelta);
    // long double significand: nearest (Delta is odd, so no exact tie)
    u128 m64 = (u128)q + (2 * (u128)rem > kBsgsDelta ? 1 : 0);
    if (m64 >> 64) { m64 >>= 1; e += 1; }
    // double significand: 11 bits fewer, nearest even
    uint64_t m53 = (uint64_t)(m64 >> 11);
    const uint32_t low = (uint32_t)m64 & 2047u;
    if (low > 1024u || (low == 1024u && (m53 & 1))) m53 += 1;
    if (m53 >> 53) { m53 >>= 1; e += 1; }
    // the double is m53 * 2^(e - 52); round half away from zero
    const int sh = 52 - e;   // >= 36 since e <= 16
    if (sh >= 64) return 0;  // below 2^-11
    const uint64_t ip = m53 >> sh;
    const uint64_t frac = m53 & ((1ull << sh) - 1);
    return ip + (frac >= (1ull << (sh - 1)) ? 1 : 0);
}

__global__ void k_client_round(const uint32_t* __restrict__ res, uint64_t* __restrict__ msg, int n) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)n * kN) return;
    const long qi = idx / kN;
    const int k = (int)(idx % kN);
    const uint64_t me = crt_compose_res(res[(qi * 2) * kN + k], res[(qi * 2 + 1) * kN + k]);
    if (me > kCrtMod / 2)
        msg[idx] = (uint64_t)kP - round_ref_quotient(kCrtMod - me);
    else
        msg[idx] = round_ref_quotient(me);
}

}  // namespace kspir
