// Gadget decompositions of the reference, as per-coefficient device functions.
// Each returns small signed digits; callers turn them into residues.
#pragma once

#include "common.cuh"

namespace kspir {

constexpr int kMaxEll = 4;

// decompose, VARIANT B (reference utils.cpp:754-811; DECOMPOSE_VARIANT_A is
// off at utils.cpp:690): unsigned digits of x + offset, each shifted down by
// Bg/2.  Note the strict `d > q` of the reference.
struct GadgetB {
    int32_t ell, base_bits, gbits;
    uint64_t offset;   // sum_i 2^(base_bits + i*gbits) * Bg/2 + base/2
};

__device__ __forceinline__ void decompose_b(uint64_t x, uint64_t q, const GadgetB& g, int32_t* dig) {
    uint64_t d = x + g.offset;
    if (d > q) d -= q;
    d >>= g.base_bits;
    const uint64_t mask = (1ull << g.gbits) - 1;
    const int32_t half = 1 << (g.gbits - 1);
#pragma unroll
    for (int j = 0; j < kMaxEll; j++) {
        if (j < g.ell) {
            dig[j] = (int32_t)(d & mask) - half;
            d >>= g.gbits;
        }
    }
}

// decompose_bsgs (reference utils.cpp:1120-1189) over crt_inv_bsgs
// (utils.cpp:516-532): the 80-bit CRT value of (x mod crtMod, y mod bsMod),
// then VARIANT-B digits of it modulo M = crtMod * bsMod.
struct GadgetBsgs {
    int32_t ell, base_bits, gbits;
    u128 offset;
    u128 M;
};

__device__ __forceinline__ void decompose_bsgs(uint64_t x_crt, uint32_t x_bs, const GadgetBsgs& g,
                                               int32_t* dig) {
    // Garner: X = x_crt + crtMod * ((x_bs - x_crt) * crtMod^-1 mod bsMod), X in [0, M)
    uint32_t xb = mod_bs(x_crt);
    uint32_t diff = submod(x_bs, xb, kBsMod);
    uint32_t t = mulmod(diff, kCrtModInvBs, CH_BS);
    u128 X = mul_64x64(kCrtMod, t);
    u128 xc; xc.lo = x_crt; xc.hi = 0;
    X = add128(X, xc);
    u128 d = add128(X, g.offset);
    if (gt128(d, g.M)) d = sub128(d, g.M);
    if (g.base_bits) d = shr128(d, g.base_bits);
    const uint64_t mask = (1ull << g.gbits) - 1;
    const int32_t half = 1 << (g.gbits - 1);
#pragma unroll
    for (int j = 0; j < kMaxEll; j++) {
        if (j < g.ell) {
            dig[j] = (int32_t)(d.lo & mask) - half;
            d = shr128(d, g.gbits);
        }
    }
}

// decompose_rlwe (reference utils.cpp:974-1044): centred lift, arithmetic
// shift by base (dropped bits truncated, not rounded), then signed digits by
// sign extension.
struct GadgetS {
    int32_t ell, base_bits, gbits;
};

__device__ __forceinline__ void decompose_signed(uint64_t x, uint64_t q, const GadgetS& g, int32_t* dig) {
    int64_t d = x > (q >> 1) ? (int64_t)(x - q) : (int64_t)x;
    d >>= g.base_bits;
    const int sh = 64 - g.gbits;
#pragma unroll
    for (int j = 0; j < kMaxEll; j++) {
        if (j < g.ell) {
            int64_t r = ((int64_t)((uint64_t)d << sh)) >> sh;
            d -= r;
            d >>= g.gbits;
            dig[j] = (int32_t)r;
        }
    }
}

}  // namespace kspir
