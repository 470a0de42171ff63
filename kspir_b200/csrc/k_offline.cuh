// Offline key derivation on the device: the reference's genAutoKeyFromOffline
// (twosteps.cpp:1749-1864) and its key switch evalAutoRNSKey (twosteps.cpp:
// 1587-1743), with the key parameters of tests/test-two-steps-key.cpp:149-155.
//
// From one offline key per chain and one automorphism key per chain, the
// reference builds every baby-step key by a chain of N1 - 2 key switches by
// X -> X^5 (autoKey1, moduli crtMod and crtBaMod = bsMod * auxMod) and every
// giant-step key by a chain of N2 - 2 key switches by X -> X^(5^N1) (autoKey2,
// moduli crtMod and auxMod), then modulus-switches every key of both chains
// into the answer's key map.  Each link of a chain depends on the previous
// one, and within a link the three gadget rows are independent, so a link is
// three launches (decomposition, transforms and key products, word
// composition) over the three rows and the RNS channels.
//
// Everything is exact integer arithmetic on the reference's words, and the
// reference's quirks are kept because the words must be identical:
//   * the automorphism negates with `modulus - x`, which is the modulus itself
//     (not 0) for x = 0 (twosteps.cpp:1631-1636);
//   * the decomposition of the crtBaMod chain reconstructs its 108-bit value
//     with compute_mult_qinvqi_bsgs_ba (utils.cpp:434-459), whose products
//     wrap modulo 2^128; crt_ref below repeats that arithmetic step for step
//     (for the auxMod chain the same steps happen not to wrap);
//   * the modulus switch reads the crtBaMod rows through EltwiseReduceMod with
//     factors (1, 1), which leaves them unreduced (twosteps.cpp:1776-1777), so
//     the bsMod rows of the derived baby keys come out zero.
#pragma once

#include "k_util.cuh"
#include "ntt.cuh"

namespace kspir {

// ---------------------------------------------------------------------------
// 128-bit words with the wrap-around of unsigned __int128

__device__ __forceinline__ u128 u128_of(uint64_t lo, uint64_t hi = 0) { u128 r; r.lo = lo; r.hi = hi; return r; }
__device__ __forceinline__ bool ge128(u128 a, u128 b) { return a.hi > b.hi || (a.hi == b.hi && a.lo >= b.lo); }
// a * b mod 2^128
__device__ __forceinline__ u128 mullo128(u128 a, u128 b) {
    u128 r;
    r.lo = a.lo * b.lo;
    r.hi = __umul64hi(a.lo, b.lo) + a.lo * b.hi + a.hi * b.lo;
    return r;
}
__device__ __forceinline__ u128 shl128(u128 a, int s) {   // 0 <= s < 128
    if (s == 0) return a;
    if (s >= 64) return u128_of(0, a.lo << (s - 64));
    return u128_of(a.lo << s, (a.hi << s) | (a.lo >> (64 - s)));
}
__device__ __forceinline__ u128 shr128_any(u128 a, int s) {   // 0 <= s < 128
    if (s == 0) return a;
    if (s >= 64) return u128_of(a.hi >> (s - 64), 0);
    return u128_of((a.lo >> s) | (a.hi << (64 - s)), a.hi >> s);
}
__device__ __forceinline__ int clz128(u128 a) { return a.hi ? __clzll(a.hi) : 64 + __clzll(a.lo); }
// a mod m (m > 0) by binary long division
__device__ __forceinline__ u128 mod128(u128 a, u128 m) {
    if (!ge128(a, m)) return a;
    int s = clz128(m) - clz128(a);
    u128 d = shl128(m, s);
    for (; s >= 0; s--) {
        if (ge128(a, d)) a = sub128(a, d);
        d = shr128_any(d, 1);
    }
    return a;
}

// The reference's CRT of (x1 mod m1 = crtMod, x2 mod m2) into [0, m1 m2):
// crt_inv_bsgs_ba / crt_inv_bsgs_aux (utils.cpp:535-570) over
// compute_mult_qinvqi_bsgs_ba / _aux (utils.cpp:434-487), including the
// wrap-around of their unsigned __int128 products.
struct CrtRef {
    u128 M;          // m1 * m2
    u128 two128;     // 2^128 mod M
    uint64_t qi1, qinv1;   // term of x1: m2 and m2^-1 mod m1
    uint64_t qi2, qinv2;   // term of x2: m1 and m1^-1 mod m2
};

__device__ __forceinline__ u128 crt_ref_term(const CrtRef& c, uint64_t input, uint64_t qinv, uint64_t qi) {
    const u128 factor = mul_64x64(qi, qinv);                 // qi * qinv
    const u128 a = u128_of(factor.hi), b = u128_of(factor.lo);
    const u128 temp = mullo128(u128_of(input), a);           // input * a
    u128 r = mod128(mullo128(u128_of(temp.hi), c.two128), c.M);   // (temp >> 64) * two128 % M
    r = add128(r, mod128(u128_of(0, temp.lo), c.M));         // + (temp << 64) % M
    r = add128(r, mullo128(u128_of(input), b));             // + input * b
    return mod128(r, c.M);
}

__device__ __forceinline__ u128 crt_ref(const CrtRef& c, uint64_t x1, uint64_t x2) {
    u128 r = crt_ref_term(c, x1, c.qinv1, c.qi1);
    r = add128(r, crt_ref_term(c, x2, c.qinv2, c.qi2));
    return mod128(r, c.M);
}

// decompose_bsgs_ba / decompose_bsgs_aux (utils.cpp:1190-1330) after the CRT:
// unsigned digits of X + offset (once reduced by the strict d > M), each
// shifted down by Bg/2.
struct OffGadget {
    int32_t ell, base_bits, gbits;
    u128 offset;
};

__device__ __forceinline__ void off_decompose(u128 X, const CrtRef& c, const OffGadget& g, int32_t* dig) {
    u128 d = add128(X, g.offset);
    if (gt128(d, c.M)) d = sub128(d, c.M);
    d = shr128_any(d, g.base_bits);
    const uint64_t mask = (1ull << g.gbits) - 1;
    const int32_t half = 1 << (g.gbits - 1);
#pragma unroll
    for (int j = 0; j < 5; j++) {
        if (j < g.ell) {
            dig[j] = (int32_t)(d.lo & mask) - half;
            d = shr128_any(d, g.gbits);
        }
    }
}

// One chain of the derivation.  Channels of the second modulus: the crtBaMod
// chain has two (CH_BA_BS, CH_BA_AUX), the auxMod chain one (CH_AUX).
struct OffChain {
    int nch2;                 // channels of the second modulus: 2 (crtBaMod) or 1 (auxMod)
    int ch2[2];
    uint64_t m2;              // the second modulus
    uint32_t ginv;            // index^-1 mod 2N of the automorphism (5 or 5^N1)
    CrtRef crt;
    OffGadget g;
};

constexpr int kOffRows = 3;    // gadget rows of autoKey1 / autoKey2 (ellnum 3)
constexpr int kOffEll = 5;     // gadget rows of the offline keys (ellnum 5)

__device__ __forceinline__ int off_chan2(const OffChain& ch, int c) { return c == 0 ? ch.ch2[0] : ch.ch2[1]; }

// residue of a word of the second modulus on its channel c (0 or 1)
__device__ __forceinline__ uint32_t off_res2(const OffChain& ch, uint64_t w, int c) {
    return (uint32_t)(w % (uint64_t)c_dev.ch[off_chan2(ch, c)].q);
}

// (a) one link, step 1: per row j and coefficient k, the automorphism of the
// link's input (a and b of both moduli, coefficient-form words), the
// decomposition of a, and the residues the transforms need:
//   dig  [3 rows][5 digits][4 channel slots][N]   (slots: q1, q2, then the second modulus)
//   bres [3 rows][4 channel slots][N]             b after the automorphism
// in: key words [6][2][N] (rows 0-2 mod crtMod, 3-5 mod m2)
__global__ void k_off_decomp(const uint64_t* __restrict__ in, uint32_t* __restrict__ dig, uint32_t* __restrict__ bres,
                             OffChain ch) {
    const int j = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kN) return;
    bool neg;
    const int src = auto_src(k, ch.ginv, &neg);
    const uint64_t* k1 = in + (size_t)j * 2 * kN;
    const uint64_t* k2 = in + (size_t)(j + kOffRows) * 2 * kN;
    uint64_t a1 = k1[src], b1 = k1[kN + src], a2 = k2[src], b2 = k2[kN + src];
    if (neg) {   // modulus - x: the modulus itself for x = 0
        a1 = kCrtMod - a1; b1 = kCrtMod - b1;
        a2 = ch.m2 - a2; b2 = ch.m2 - b2;
    }
    int32_t d[5];
    off_decompose(crt_ref(ch.crt, a1, a2), ch.crt, ch.g, d);
    uint32_t* dj = dig + (size_t)j * kOffEll * 4 * kN;
    for (int i = 0; i < ch.g.ell; i++) {
        dj[(i * 4 + 0) * kN + k] = signed_to_res(d[i], kQ1);
        dj[(i * 4 + 1) * kN + k] = signed_to_res(d[i], kQ2);
        for (int c = 0; c < ch.nch2; c++) dj[(i * 4 + 2 + c) * kN + k] = signed_to_res(d[i], c_dev.ch[off_chan2(ch, c)].q);
    }
    uint32_t* bj = bres + (size_t)j * 4 * kN;
    bj[0 * kN + k] = (uint32_t)(b1 % kQ1);
    bj[1 * kN + k] = (uint32_t)(b1 % kQ2);
    for (int c = 0; c < ch.nch2; c++) bj[(2 + c) * kN + k] = off_res2(ch, b2, c);
}

constexpr int kOffPolys = kOffEll + 1;                       // b and the five digits
constexpr int kOffSmem = kN * 8 + kOffPolys * kPadN * 4;     // twiddles + six padded polynomials

// (b) per row j and channel slot s (0, 1: q1, q2; 2.. : the second modulus):
// transforms of b and of the digits, the key products with the offline key
//   a' = -sum_i d_i key[i].a,  b' = NTT(b) - sum_i d_i key[i].b
// (rows i of crtMod for slots 0-1, rows 5 + i for the second modulus), and the
// inverse transforms: res [3 rows][4 slots][2 comp][N] residues, coefficient form.
// okey: offline key residues [10 rows][2 comp][4 slots][N].
__global__ void __launch_bounds__(kNttThreads) k_off_keyswitch(const uint32_t* __restrict__ dig,
                                                               const uint32_t* __restrict__ bres,
                                                               const uint32_t* __restrict__ okey,
                                                               uint32_t* __restrict__ res, NttTables tabs,
                                                               OffChain ch) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* P = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);   // [b, d0..d4][N]
    const int j = blockIdx.y, s = blockIdx.x;
    const int chan = s == 0 ? CH_Q1 : s == 1 ? CH_Q2 : off_chan2(ch, s - 2);
    const int ell = ch.g.ell;
    const int tid = threadIdx.x;
    const uint32_t q = c_dev.ch[chan].q;
    const uint64_t bar = c_dev.ch[chan].barrett;
    stage_twiddles(tws, tabs, chan, NTT_FWD);
    poly_to_smem(P, bres + ((size_t)j * 4 + s) * kN);
    for (int i = 0; i < ell; i++) poly_to_smem(P + (1 + i) * kPadN, dig + (((size_t)j * kOffEll + i) * 4 + s) * kN);
    cta_ntt_forward_m<kOffPolys>(P, kPadN, tws, chan);
    const int krow0 = s < 2 ? 0 : kOffEll;   // offline key rows of this modulus
    uint32_t outa[kN / kNttThreads], outb[kN / kNttThreads];
#pragma unroll
    for (int it = 0; it < kN / kNttThreads; it++) {
        const int k = tid + it * kNttThreads;
        const int pk = pidx(tid) + it * kPadStep;
        uint64_t sa = 0, sb = 0;
        for (int i = 0; i < ell; i++) {
            const uint32_t dv = P[(1 + i) * kPadN + pk];
            const uint32_t* kr = okey + ((size_t)(krow0 + i) * 2 * 4 + s) * kN;
            sa += (uint64_t)dv * __ldg(kr + k);             // comp a (slot s)
            sb += (uint64_t)dv * __ldg(kr + 4 * kN + k);    // comp b
        }
        outa[it] = negmod(reduce64(sa, q, bar), q);
        outb[it] = submod(P[pk], reduce64(sb, q, bar), q);
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kN / kNttThreads; it++) {
        const int pk = pidx(tid) + it * kPadStep;
        P[pk] = outa[it];
        P[kPadN + pk] = outb[it];
    }
    stage_twiddles(tws, tabs, chan, NTT_INV);   // the forward transforms ended with a barrier
    cta_ntt_inverse_m<2>(P, kPadN, tws, chan);
    uint32_t* o = res + ((size_t)j * 4 + s) * 2 * kN;
    poly_from_smem(o, P);
    poly_from_smem(o + kN, P + kPadN);
}

// Canonical word of two residues (r1 mod p1, r2 mod p2), p1 < p2, p1 p2 < 2^62:
// Garner with p1^-1 mod p2.
__device__ __forceinline__ uint64_t garner2(uint32_t r1, uint32_t r2, uint32_t p1, uint32_t p2, uint32_t p1inv) {
    const uint32_t r1m = r1 % p2;
    const uint32_t d = r2 >= r1m ? r2 - r1m : r2 + p2 - r1m;
    const uint32_t t = (uint32_t)(((uint64_t)d * p1inv) % p2);
    return (uint64_t)r1 + (uint64_t)p1 * t;
}

// (c) the link's output key words [6][2][N] from res: rows j (crtMod) and
// j + 3 (the second modulus), coefficient form.  p1inv: bsMod^-1 mod auxMod
// for the crtBaMod chain.
__global__ void k_off_compose(const uint32_t* __restrict__ res, uint64_t* __restrict__ out, OffChain ch,
                              uint32_t p1inv) {
    const int j = blockIdx.z, comp = blockIdx.y;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kN) return;
    const uint32_t* r = res + (size_t)j * 4 * 2 * kN + (size_t)comp * kN;   // slot s at r + s * 2N
    out[((size_t)j * 2 + comp) * kN + k] = crt_compose_res(r[k], r[2 * kN + k]);
    uint64_t w2;
    if (ch.nch2 == 2)
        w2 = garner2(r[2 * 2 * kN + k], r[3 * 2 * kN + k], c_dev.ch[CH_BA_BS].q, c_dev.ch[CH_BA_AUX].q, p1inv);
    else
        w2 = r[2 * 2 * kN + k];
    out[((size_t)(j + kOffRows) * 2 + comp) * kN + k] = w2;
}

// Words of a key [rows][2][N] as residues on the channel slots of its rows:
// dst [rows][2 comp][4 slots][N]; rows < rows1 are mod crtMod (slots 0, 1),
// the others mod the second modulus (slots 2..).
__global__ void k_off_key_residues(const uint64_t* __restrict__ w, uint32_t* __restrict__ dst, int rows, int rows1,
                                   OffChain ch) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)rows * 2 * kN) return;
    const int k = (int)(idx % kN);
    const long rc = idx / kN;   // row * 2 + comp
    const int row = (int)(rc / 2);
    const uint64_t v = w[idx];
    uint32_t* d = dst + (size_t)rc * 4 * kN;
    if (row < rows1) {
        d[k] = (uint32_t)(v % kQ1);
        d[kN + k] = (uint32_t)(v % kQ2);
    } else {
        for (int c = 0; c < ch.nch2; c++) d[(2 + c) * kN + k] = off_res2(ch, v, c);
    }
}

// The first link's input is the automorphism key as generated (NTT form):
// one CTA per (row of 6, comp, slot) brings it to coefficient form, into the
// layout of k_off_keyswitch's res ([row j][slot][comp][N]: rows 0-2 of crtMod
// in slots 0, 1, rows 3-5 of the second modulus in slots 2..).
__global__ void __launch_bounds__(kNttThreads) k_off_intt_key(const uint32_t* __restrict__ kres,
                                                              uint32_t* __restrict__ res, NttTables tabs,
                                                              OffChain ch) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* P = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);
    const int row = blockIdx.z, comp = blockIdx.y, s = blockIdx.x;
    const int j = row % kOffRows;
    const bool second = row >= kOffRows;
    if ((second && s >= ch.nch2) || (!second && s >= 2)) return;   // the whole CTA leaves together
    const int slot = second ? 2 + s : s;
    const int chan = slot == 0 ? CH_Q1 : slot == 1 ? CH_Q2 : off_chan2(ch, slot - 2);
    stage_twiddles(tws, tabs, chan, NTT_INV);
    poly_to_smem(P, kres + ((size_t)row * 2 + comp) * 4 * kN + (size_t)slot * kN);
    cta_ntt_inverse(P, tws, chan);
    poly_from_smem(res + (((size_t)j * 4 + slot) * 2 + comp) * kN, P);
}

// (d) the modulus switch of the derivation (twosteps.cpp:1764-1810, 1835-1862)
// for `nkeys` keys of a chain, key words in [nkeys][6][2][N]: rows j < 3 of
// each key become NTT_crtMod(((a - x) mod crtMod) * auxMod^-1 mod crtMod),
// x the unreduced word of row j + 3 (EltwiseReduceMod with factors (1, 1)
// copies it), as residues res [nkeys][3][2 comp][2 primes][N].  One CTA per
// (key, row, comp, prime).
__global__ void __launch_bounds__(kNttThreads) k_off_modswitch(const uint64_t* __restrict__ keys,
                                                               uint32_t* __restrict__ res, uint64_t aux_inv,
                                                               NttTables tabs) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* P = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);
    const int ch = blockIdx.x & 1, comp = (blockIdx.x >> 1) & 1, j = (blockIdx.x >> 2) % kOffRows;
    const int key = blockIdx.x / (4 * kOffRows);
    const uint32_t q = c_dev.ch[ch].q;
    const uint64_t bar = c_dev.ch[ch].barrett;
    const uint32_t ainv = (uint32_t)(aux_inv % q);
    stage_twiddles(tws, tabs, ch, NTT_FWD);
    const uint64_t* kw = keys + (size_t)key * 6 * 2 * kN;
    const uint64_t* a = kw + ((size_t)j * 2 + comp) * kN;
    const uint64_t* x = kw + ((size_t)(j + kOffRows) * 2 + comp) * kN;
    for (int k = threadIdx.x; k < kN; k += kNttThreads) {
        const uint64_t av = a[k], xv = x[k];
        const uint64_t v = av >= xv ? av - xv : av + kCrtMod - xv;   // EltwiseSubMod, both below crtMod
        P[pidx(k)] = reduce64((uint64_t)(uint32_t)(v % q) * ainv, q, bar);
    }
    cta_ntt_forward(P, tws, ch);
    poly_from_smem(res + (((size_t)key * kOffRows + j) * 2 + comp) * 2 * kN + (size_t)ch * kN, P);
}

}  // namespace kspir
