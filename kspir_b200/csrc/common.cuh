// Device-side arithmetic shared by every KsPIR kernel.
//
// Representation.  The reference computes modulo crtMod = q1*q2 (56 bits,
// reference src/crt.h:16-18) and bsMod (24 bits, crt.h:32) on 64-bit words
// through HEXL.  Every HEXL operation on the answer path is exact modular
// arithmetic with canonical outputs, so a value mod crtMod is held here as its
// two 28-bit residues (mod q1, mod q2) in 32-bit words, and bsMod is a third
// 32-bit channel.  The NTT with root_of_unity_crt (crt.h:81) is, residue by
// residue, the NTT with psi mod q1 and psi mod q2.  A canonical 56-bit (or
// crtMod*bsMod 80-bit) integer is formed by CRT only where the reference
// leaves modular arithmetic: the gadget decompositions and the response words.
#pragma once

#include <stdint.h>

namespace kspir {

constexpr int kN = 4096;          // ring dimension, reference params.h:16
constexpr int kLogN = 12;
constexpr uint32_t kQ1 = 268369921u;   // crt.h:16
constexpr uint32_t kQ2 = 249561089u;   // crt.h:17
constexpr uint64_t kCrtMod = (uint64_t)kQ1 * kQ2;
constexpr uint32_t kBsMod = 16760833u; // crt.h:32
constexpr uint64_t kBsModInvCrt = 51309461009346113ull;  // bsMod^-1 mod crtMod, crt.h:33
constexpr uint32_t kCrtModInvBs = 3920321u;              // crtMod^-1 mod bsMod, crt.h:34

constexpr uint32_t kP = 65537u;        // plaintext modulus bsgsp, params.h:94
constexpr uint32_t kAuxMod = 268361729u;   // auxiliary modulus of the offline key derivation, crt.h:37

// channels of the RNS representation (p: only for the database preprocessing;
// the last three only for the offline key derivation: crtBaMod = bsMod * auxMod
// transformed with root_of_unity_crt_bamod, crt.h:82, as its two residues, and
// auxMod with HEXL's minimal root)
enum Chan : int { CH_Q1 = 0, CH_Q2 = 1, CH_BS = 2, CH_P = 3, CH_BA_BS = 4, CH_BA_AUX = 5, CH_AUX = 6, CH_COUNT = 7 };

// Per-channel constants, filled on the host (context.cu) and kept in
// __constant__ memory.
struct ChanConst {
    uint32_t q;
    uint32_t two_q;
    uint64_t barrett;      // floor(2^64 / q)
    uint32_t ninv, ninv_p; // N^-1 mod q and its Shoup companion
    uint32_t ninv_w, ninv_w_p;   // N^-1 times the last inverse layer's twiddle (psi^-N/2), Shoup
    uint32_t bsinv, bsinv_p;  // bsMod^-1 mod crtMod, reduced mod q (crt channels only)
};

struct DevConst {
    ChanConst ch[CH_COUNT];
    uint32_t q1inv_mod_q2;     // q1^-1 mod q2 (Garner)
    uint32_t q1inv_mod_q2_p;
};

// Defined here: the library is one translation unit (kspir.cu includes every
// kernel header), so no relocatable device code is needed.
__constant__ DevConst c_dev;

// ---------------------------------------------------------------------------
// 32-bit residue arithmetic (q < 2^28)

__device__ __forceinline__ uint32_t shoup_lazy(uint32_t x, uint32_t w, uint32_t wp, uint32_t q) {
    // x*w mod q in [0, 2q) for any 32-bit x; wp = floor(w * 2^32 / q)
    uint32_t t = __umulhi(x, wp);
    return x * w - t * q;
}

// Conditional subtractions as an unsigned minimum: for x < 2m, x - m wraps
// above x exactly when x < m.
__device__ __forceinline__ uint32_t shoup_mul(uint32_t x, uint32_t w, uint32_t wp, uint32_t q) {
    const uint32_t r = shoup_lazy(x, w, wp, q);
    return umin(r, r - q);
}

// Exact reduction of any 64-bit p by Barrett with barrett = floor(2^64 / q):
// qh = floor(p * barrett / 2^64) is floor(p / q) or one less (p * barrett
// falls short of p * 2^64 / q by less than p < 2^64), so p - qh q is in
// [0, 2q) and is computed in 32 bits.
__device__ __forceinline__ uint32_t reduce64(uint64_t p, uint32_t q, uint64_t barrett) {
    const uint32_t qh = (uint32_t)__umul64hi(p, barrett);
    const uint32_t r = (uint32_t)p - qh * q;
    return umin(r, r - q);
}

__device__ __forceinline__ uint32_t mulmod(uint32_t a, uint32_t b, int ch) {
    return reduce64((uint64_t)a * b, c_dev.ch[ch].q, c_dev.ch[ch].barrett);
}

__device__ __forceinline__ uint32_t addmod(uint32_t a, uint32_t b, uint32_t q) {
    const uint32_t s = a + b;
    return umin(s, s - q);
}

__device__ __forceinline__ uint32_t submod(uint32_t a, uint32_t b, uint32_t q) {
    const uint32_t d = a - b;   // wraps when a < b, and d + q is then the residue
    return umin(d, d + q);
}

// A signed small integer (|v| < q) as a canonical residue.
__device__ __forceinline__ uint32_t signed_to_res(int64_t v, uint32_t q) {
    const uint32_t u = (uint32_t)v;   // above 2^32 - q exactly when v < 0, and u + q then wraps to v + q
    return umin(u, u + q);
}

// ---------------------------------------------------------------------------
// crtMod <-> residues

// canonical value mod crtMod from its residues (Garner)
__device__ __forceinline__ uint64_t crt_compose_res(uint32_t r1, uint32_t r2) {
    const uint32_t r1m = umin(r1, r1 - kQ2);             // r1 mod q2 (q1 < 2 q2)
    const uint32_t d = submod(r2, r1m, kQ2);             // (r2 - r1) mod q2
    uint32_t t = shoup_mul(d, c_dev.q1inv_mod_q2, c_dev.q1inv_mod_q2_p, kQ2);
    return (uint64_t)r1 + (uint64_t)kQ1 * t;
}

// unsigned minimum for code compiled for the host as well
__host__ __device__ __forceinline__ uint32_t min_u32(uint32_t a, uint32_t b) { return a < b ? a : b; }

// x mod q, exact for every 64-bit x, q a prime in (2^27, 2^28); mu1 = 2^59 / q,
// c32 = 2^32 mod q, mu2 = 2^57 / q.  Two Barrett steps with 32x32 products.
__host__ __device__ __forceinline__ uint32_t mod28(uint64_t x, uint32_t q, uint32_t mu1, uint32_t c32, uint32_t mu2) {
    const uint32_t xh = (uint32_t)(x >> 32), xl = (uint32_t)x;
    // conditional subtractions as minima (x - m wraps above x when x < m)
    uint32_t r = xh - (uint32_t)(((uint64_t)xh * mu1) >> 59) * q;   // in [0, 2q)
    r = min_u32(r, r - q);
    const uint64_t y = (uint64_t)r * c32 + xl;                       // < 2^57, same residue
    const uint32_t qh = (uint32_t)(((y >> 26) * mu2) >> 31);
    uint32_t t = (uint32_t)y - qh * q;                                // in [0, 3q)
    t = min_u32(t, t - 2 * q);                                        // in [0, 2q)
    return min_u32(t, t - q);
}

// x mod q_ch for the crt primes (ch 0: q1, 1: q2), any 64-bit x.  (mod28 measured
// no faster than this Barrett reduction inside the key-switch kernels.)
__device__ __forceinline__ uint32_t mod_crt(uint64_t x, int ch) {
    return reduce64(x, ch ? kQ2 : kQ1, c_dev.ch[ch].barrett);
}

__device__ __forceinline__ uint32_t mod_q1(uint64_t v) { return reduce64(v, kQ1, c_dev.ch[CH_Q1].barrett); }
__device__ __forceinline__ uint32_t mod_q2(uint64_t v) { return reduce64(v, kQ2, c_dev.ch[CH_Q2].barrett); }
__device__ __forceinline__ uint32_t mod_bs(uint64_t v) { return reduce64(v, kBsMod, c_dev.ch[CH_BS].barrett); }

// ---------------------------------------------------------------------------
// 128-bit helpers (hi:lo pairs)

struct u128 { uint64_t lo, hi; };

__device__ __forceinline__ u128 mul_64x64(uint64_t a, uint64_t b) {
    u128 r; r.lo = a * b; r.hi = __umul64hi(a, b); return r;
}

__device__ __forceinline__ u128 add128(u128 a, u128 b) {
    u128 r; r.lo = a.lo + b.lo; r.hi = a.hi + b.hi + (r.lo < a.lo ? 1 : 0); return r;
}

__device__ __forceinline__ u128 sub128(u128 a, u128 b) {
    u128 r; r.lo = a.lo - b.lo; r.hi = a.hi - b.hi - (a.lo < b.lo ? 1 : 0); return r;
}

__device__ __forceinline__ bool gt128(u128 a, u128 b) {
    return a.hi > b.hi || (a.hi == b.hi && a.lo > b.lo);
}

__device__ __forceinline__ u128 shr128(u128 a, int s) {  // 0 < s < 64
    u128 r; r.lo = (a.lo >> s) | (a.hi << (64 - s)); r.hi = a.hi >> s; return r;
}

// ---------------------------------------------------------------------------
// automorphism X -> X^g, coefficient domain, as a gather:
// out[k] = +-in[i] with i*g = k or k+N (mod 2N).  `neg_canonical` selects the
// negation: the reference's automorphic_rns writes 0 for -0 (twosteps.cpp:776-778);
// the inline loops of evalAutoRNSCRT / evalAuto write q (twosteps.cpp:629-630,
// answer.cpp:606-607).  Downstream every consumer treats q exactly like 0, so
// the kernels only need the canonical form.
__device__ __forceinline__ int auto_src(int k, uint32_t ginv, bool* neg) {
    uint32_t i0 = ((uint32_t)k * ginv) & (2 * kN - 1);
    *neg = i0 >= (uint32_t)kN;
    return (int)(i0 & (kN - 1));
}

// q - x, and 0 for x = 0 (0 - x wraps above q - x for every other x)
__device__ __forceinline__ uint32_t negmod(uint32_t x, uint32_t q) { return umin(q - x, 0u - x); }

// acc += a * b with a 32x32->64-bit product, as one fused wide multiply-add
__device__ __forceinline__ void mad_wide(uint64_t& acc, uint32_t a, uint32_t b) {
    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(acc) : "r"(a), "r"(b));
}

}  // namespace kspir
