// Giant steps (reference evalAutoRNSCRT, twosteps.cpp:599-677), the external
// product (externalProduct, lwe.cpp:761-808) and the RLWE packing tree
// (packingRLWEs / convertTwoRLWEs / evalAuto, answer.cpp:576-835).
//
// All three are key switches of the same shape: bring `a` to coefficient form,
// apply an automorphism, gadget-decompose, transform the digits, multiply by
// the key and accumulate.  They run as element-wise kernels (decompose,
// accumulate) around batched transforms (k_ntt_jobs) and a fused
// multiply-accumulate + inverse-transform kernel.
#pragma once

#include "ntt.cuh"
#include "pipeline.cuh"

namespace kspir {

// ---------------------------------------------------------------------------
// giant steps

// For every (r, c >= 1) and coefficient k: the digits of
// decompose(auto_g(INTT(output[c].a))), g = 5^(N1 c)  (twosteps.cpp:612-641).
// The reference's inline automorphism leaves q for a negated zero
// (twosteps.cpp:629); decompose maps q and 0 to the same digits (d = q + offset
// > q is reduced back to offset), so the canonical negation is equivalent.
__global__ void k_giant_decomp(const uint32_t* __restrict__ gcoef, uint32_t* __restrict__ gdig, int R,
                               int N1, GadgetB g) {
    const int N2 = kN / 2 / N1;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)R * (N2 - 1) * kN) return;
    const int k = (int)(idx % kN);
    const long rc = idx / kN;               // r * (N2-1) + (c-1)
    const int c = (int)(rc % (N2 - 1)) + 1;
    const uint32_t e = (uint32_t)(N1 * c) & 2047u;
    uint32_t gi = 1, b = 5, x = (2048u - e) & 2047u;   // g^-1 = 5^(2048 - N1 c) mod 2N
    while (x) { if (x & 1) gi = (gi * b) & (2 * kN - 1); b = (b * b) & (2 * kN - 1); x >>= 1; }
    bool neg;
    const int src = auto_src(k, gi, &neg);
    const uint32_t* a = gcoef + rc * 2 * kN;
    uint64_t v = crt_compose_res(a[src], a[kN + src]);
    if (neg && v) v = kCrtMod - v;
    int32_t dig[kMaxEll];
    decompose_b(v, kCrtMod, g, dig);
    uint32_t* o = gdig + rc * g.ell * 2 * kN;
    for (int j = 0; j < g.ell; j++) {
        o[(j * 2 + 0) * kN + k] = signed_to_res(dig[j], kQ1);
        o[(j * 2 + 1) * kN + k] = signed_to_res(dig[j], kQ2);
    }
}

// result[r] = output[0] + sum_{c>=1} ( -sum_j d_j * key_c[j].a ,
//                                       NTT(auto_g b_c) - sum_j d_j * key_c[j].b )
// with NTT(auto_g b_c) = b_c[sigma_g] taken in the NTT domain (twosteps.cpp:642-672).
__global__ void k_giant_accum(const uint32_t* __restrict__ sout, const uint32_t* __restrict__ gdig,
                              const uint32_t* __restrict__ gkeys, const uint16_t* __restrict__ gsigma,
                              uint32_t* __restrict__ result, int R, int N1, int ell) {
    const int N2 = kN / 2 / N1;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)R * 2 * kN) return;
    const int k = (int)(idx % kN);
    const int ch = (int)((idx / kN) % 2);
    const long r = idx / (2 * kN);
    const ChanConst cc = c_dev.ch[ch];
    const uint32_t* so = sout + (size_t)r * N2 * 4 * kN;      // [N2][2 comp][2 ch][N]
    uint32_t ra = so[(0 * 2 + ch) * kN + k];
    uint32_t rb = so[(1 * 2 + ch) * kN + k];
#pragma unroll 5
    for (int c = 1; c < N2; c++) {
        const uint32_t* d = gdig + ((size_t)r * (N2 - 1) + (c - 1)) * ell * 2 * kN;
        const uint32_t* key = gkeys + (size_t)(c - 1) * ell * 2 * 2 * kN;
        uint64_t sa = 0, sb = 0;
        for (int j = 0; j < ell; j++) {
            const uint64_t dj = d[(j * 2 + ch) * kN + k];
            sa += dj * key[((j * 2 + 0) * 2 + ch) * kN + k];
            sb += dj * key[((j * 2 + 1) * 2 + ch) * kN + k];
        }
        const uint32_t bc = so[((size_t)c * 4 + 1 * 2 + ch) * kN + gsigma[(size_t)(c - 1) * kN + k]];
        ra = submod(ra, reduce64(sa, cc.q, cc.barrett), cc.q);
        rb = addmod(rb, bc, cc.q);
        rb = submod(rb, reduce64(sb, cc.q, cc.barrett), cc.q);
    }
    uint32_t* o = result + (size_t)r * 4 * kN;
    o[(0 * 2 + ch) * kN + k] = ra;
    o[(1 * 2 + ch) * kN + k] = rb;
}

// ---------------------------------------------------------------------------
// external product

// Signed digits of decompose_rlwe(a, b) (utils.cpp:974-1044) of the
// coefficient-form first-dimension result: edig[r][row][ch][k], rows 0..ell-1
// from a and ell..2ell-1 from b.
__global__ void k_ext_decomp(const uint32_t* __restrict__ ecoef, uint32_t* __restrict__ edig, int R, GadgetS g) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)R * kN) return;
    const int k = (int)(idx % kN);
    const long r = idx / kN;
    const uint32_t* e = ecoef + (size_t)r * 4 * kN;
    uint32_t* o = edig + (size_t)r * 2 * g.ell * 2 * kN;
    for (int comp = 0; comp < 2; comp++) {
        const uint64_t v = crt_compose_res(e[(comp * 2 + 0) * kN + k], e[(comp * 2 + 1) * kN + k]);
        int32_t dig[kMaxEll];
        decompose_signed(v, kCrtMod, g, dig);
        for (int j = 0; j < g.ell; j++) {
            const int row = comp * g.ell + j;
            o[(row * 2 + 0) * kN + k] = signed_to_res(dig[j], kQ1);
            o[(row * 2 + 1) * kN + k] = signed_to_res(dig[j], kQ2);
        }
    }
}

// dynamic shared memory of the fused multiply-accumulate + inverse-transform kernels
constexpr int kMacSmem = kN * 8 + kN * 4;

// One CTA per (r, comp, ch): ext = INTT( init + sum_row digit_row * rgsw[row].comp ),
// init being the caller's NTT-domain accumulator (zero on the answer path,
// test-pir.cpp:102-104) or null.
__global__ void __launch_bounds__(kNttThreads) k_ext_mac_intt(const uint32_t* __restrict__ edig,
                                                              const uint32_t* __restrict__ rgsw,
                                                              const uint32_t* __restrict__ init,
                                                              uint32_t* __restrict__ ext, int rows, NttTables tabs) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* s = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);
    constexpr int T = kNttThreads;
    const int ch = blockIdx.x % 2, comp = (blockIdx.x / 2) % 2, r = blockIdx.x / 4;
    const ChanConst cc = c_dev.ch[ch];
    stage_twiddles(tws, tabs, ch, NTT_INV);
    const uint32_t* d = edig + (size_t)r * rows * 2 * kN;
#pragma unroll
    for (int k = threadIdx.x; k < kN; k += T) {
        uint64_t acc = 0;
        for (int row = 0; row < rows; row++)
            acc += (uint64_t)d[(row * 2 + ch) * kN + k] * rgsw[((row * 2 + comp) * 2 + ch) * kN + k];
        const uint32_t m = reduce64(acc, cc.q, cc.barrett);
        s[k] = init ? addmod(init[((size_t)r * 4 + comp * 2 + ch) * kN + k], m, cc.q) : m;
    }
    cta_ntt_inverse(s, tws, ch);
    uint32_t* o = ext + ((size_t)r * 4 + comp * 2 + ch) * kN;
#pragma unroll
    for (int k = threadIdx.x; k < kN; k += T) o[k] = s[k];
}

// ---------------------------------------------------------------------------
// packing, one level of the tree (pairs j < I; rlwes[j] absorbs rlwes[I + j])

// convertTwoRLWEs (answer.cpp:720-739) up to the key switch of evalAuto:
//   c' = X^I * c  (multConst, lwe.cpp:102-119),  r1 = r0 - c',  c2 = c' + r0,
//   temp = auto_g(r1), g = N/I + 1, digits of decompose(temp.a) and temp.b.
// multConst and evalAuto leave q for negated zeros; the HEXL add/sub that
// consume c' and the decomposition treat q exactly like 0.
__global__ void k_pack_prep(const uint32_t* __restrict__ ext, uint32_t* __restrict__ pdig,
                            uint32_t* __restrict__ ptb, uint32_t* __restrict__ pc2, int I, uint32_t ginv,
                            GadgetB g) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)I * kN) return;
    const int k = (int)(idx % kN);
    const int j = (int)(idx / kN);
    const uint32_t* r0 = ext + (size_t)j * 4 * kN;
    const uint32_t* cc = ext + (size_t)(I + j) * 4 * kN;
    bool neg;   // ginv = (N/I + 1)^-1 mod 2N
    const int src = auto_src(k, ginv, &neg);
    // c' at position src: coefficient src - I of c, negated when it wraps
    const int cs = src - I;
    uint32_t r1v[2][2];
#pragma unroll
    for (int comp = 0; comp < 2; comp++) {
#pragma unroll
        for (int ch = 0; ch < 2; ch++) {
            const uint32_t q = ch ? kQ2 : kQ1;
            // c2 at position k
            const int ck = k - I;
            uint32_t cpk = ck >= 0 ? cc[(comp * 2 + ch) * kN + ck] : negmod(cc[(comp * 2 + ch) * kN + ck + kN], q);
            pc2[((size_t)j * 4 + comp * 2 + ch) * kN + k] = addmod(cpk, r0[(comp * 2 + ch) * kN + k], q);
            // r1 at position src
            uint32_t cps = cs >= 0 ? cc[(comp * 2 + ch) * kN + cs] : negmod(cc[(comp * 2 + ch) * kN + cs + kN], q);
            uint32_t v = submod(r0[(comp * 2 + ch) * kN + src], cps, q);
            r1v[comp][ch] = neg ? negmod(v, q) : v;
        }
    }
    // temp.b -> ptb, temp.a -> digits
    ptb[((size_t)j * 2 + 0) * kN + k] = r1v[1][0];
    ptb[((size_t)j * 2 + 1) * kN + k] = r1v[1][1];
    const uint64_t va = crt_compose_res(r1v[0][0], r1v[0][1]);
    int32_t dig[kMaxEll];
    decompose_b(va, kCrtMod, g, dig);
    uint32_t* o = pdig + (size_t)j * g.ell * 2 * kN;
    for (int d = 0; d < g.ell; d++) {
        o[(d * 2 + 0) * kN + k] = signed_to_res(dig[d], kQ1);
        o[(d * 2 + 1) * kN + k] = signed_to_res(dig[d], kQ2);
    }
}

// One CTA per (j, comp, ch): the key switch of evalAuto (answer.cpp:617-645)
// and the final addAndEqual of convertTwoRLWEs:
//   a' = -sum_d dig_d * key[d].a,  b' = NTT(temp.b) - sum_d dig_d * key[d].b,
//   rlwes[j] = INTT(a', b') + c2.
__global__ void __launch_bounds__(kNttThreads) k_pack_mac_intt(const uint32_t* __restrict__ pdig,
                                                               const uint32_t* __restrict__ ptb,
                                                               const uint32_t* __restrict__ pc2,
                                                               const uint32_t* __restrict__ key,
                                                               uint32_t* __restrict__ ext, int ell, NttTables tabs) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* s = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);
    constexpr int T = kNttThreads;
    const int ch = blockIdx.x % 2, comp = (blockIdx.x / 2) % 2, j = blockIdx.x / 4;
    const ChanConst cc = c_dev.ch[ch];
    stage_twiddles(tws, tabs, ch, NTT_INV);
    const uint32_t* d = pdig + (size_t)j * ell * 2 * kN;
#pragma unroll
    for (int k = threadIdx.x; k < kN; k += T) {
        uint64_t acc = 0;
        for (int dd = 0; dd < ell; dd++)
            acc += (uint64_t)d[(dd * 2 + ch) * kN + k] * key[((dd * 2 + comp) * 2 + ch) * kN + k];
        const uint32_t m = reduce64(acc, cc.q, cc.barrett);
        s[k] = comp == 0 ? negmod(m, cc.q) : submod(ptb[((size_t)j * 2 + ch) * kN + k], m, cc.q);
    }
    cta_ntt_inverse(s, tws, ch);
    const uint32_t* c2 = pc2 + ((size_t)j * 4 + comp * 2 + ch) * kN;
    uint32_t* o = ext + ((size_t)j * 4 + comp * 2 + ch) * kN;
#pragma unroll
    for (int k = threadIdx.x; k < kN; k += T) o[k] = addmod(s[k], c2[k], cc.q);
}

}  // namespace kspir
