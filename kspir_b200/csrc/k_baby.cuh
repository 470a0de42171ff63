// The hoisted baby steps (reference evalAutoSRNSFirst / evalAutoSRNSSecond,
// twosteps.cpp:937-1204) fused with the RNS modswitch and reorientCipher
// (twosteps.cpp:1386-1403): one CTA produces one rotation of the query and
// writes it, as residue pairs, straight into its cipherbuf column.
//
// Per rotation g = 5^(i+1) (key index i), with digits d_j of the source a in
// NTT form (hoisted: decomposed once, reference :960-979 / :1109-1127):
//   A_c = -sum_j d_j[perm[k]] * key_j.a     (crtMod channels c and bsMod)
//   B_c = -sum_j d_j[perm[k]] * key_j.b
// The reference then leaves the NTT domain for the modswitch:
//   out.a = NTT((INTT(A_crt) - x2a) * bsMod^-1),  x2a = INTT_bs(A_bs)
//   out.b = NTT((INTT(B_crt) + auto_g(b) - x2b) * bsMod^-1),
//           x2b = INTT_bs(B_bs) + auto_g(b mod bsMod)
// (twosteps.cpp:1034-1071).  All of it is exact arithmetic mod crtMod with
// canonical values, so by linearity of the transform the same words are
//   out.a = (A_crt - NTT(x2a)) * bsMod^-1
//   out.b = (B_crt + NTT(b)[sigma_g] - NTT(x2b)) * bsMod^-1
// where sigma_g is the slot permutation of X -> X^g in the NTT domain.  Only
// the bsMod channel is brought to coefficient form (x2 must be the canonical
// integer < bsMod); the crt channels stay in the NTT domain throughout.
#pragma once

#include "ntt.cuh"
#include "pipeline.cuh"

namespace kspir {

struct BabyArgs {
    const uint32_t* dig;     // [ell][3 ch][N] source digits, NTT form
    const uint32_t* srcB;    // [2 ch][N] NTT form of the source b (crt)
    const uint32_t* srcBbs;  // [N] source b mod bsMod, coefficient form
    const int32_t* perms;    // caller permutations [N1][N] (reference test-pir.cpp:92-93)
    const uint16_t* sigma;   // [N1/2][N] slot permutation of X -> X^(5^(i+1))
    uint64_t* cipherbuf;     // [N][N1][2]
    uint32_t* interA;        // outputs of the intermediate rotation (or null)
    uint32_t* interB;
    uint32_t* inter_bs;
    int32_t N1;
    int32_t col_base;        // cipherbuf column of key index 0
    int32_t inter_idx;       // key index whose pre-modswitch state is exported, or -1
    int32_t ell;
};

// 5^e mod 2N
__device__ __forceinline__ uint32_t pow5_mod2n(uint32_t e) {
    uint32_t r = 1, b = 5;
    while (e) {
        if (e & 1) r = (r * b) & (2 * kN - 1);
        b = (b * b) & (2 * kN - 1);
        e >>= 1;
    }
    return r;
}

template <int T>
__global__ void __launch_bounds__(T) k_baby_rot(BabyArgs a, ClientKeysDev keys, NttTables tabs) {
    extern __shared__ uint32_t sm[];
    uint32_t* Sa = sm;
    uint32_t* Sb = sm + kN;
    uint32_t* W = sm + 2 * kN;
    uint32_t* Ra = sm + 3 * kN;
    uint32_t* Rb = sm + 4 * kN;

    const int ki = blockIdx.x;                 // key index: rotation by 5^(ki+1)
    const int col = a.col_base + ki;
    const bool inter = (ki == a.inter_idx);
    const int ell = a.ell;
    const int32_t* __restrict__ perm = a.perms + (size_t)(ki + 1) * kN;
    const uint16_t* __restrict__ sig = a.sigma + (size_t)ki * kN;
    const uint32_t* __restrict__ kbs = keys.baby_bs + (size_t)ki * ell * 2 * kN;
    const uint32_t* __restrict__ kcrt = keys.baby_crt + (size_t)ki * ell * 2 * 2 * kN;
    const uint32_t* __restrict__ dig = a.dig;
    const ChanConst cb = c_dev.ch[CH_BS];

    // bsMod channel: A_bs, B_bs
    for (int k = threadIdx.x; k < kN; k += T) {
        const int p = perm[k];
        uint64_t sa = 0, sb = 0;
        for (int j = 0; j < ell; j++) {
            const uint64_t d = dig[(j * 3 + CH_BS) * kN + p];
            sa += d * kbs[(j * 2 + 0) * kN + k];
            sb += d * kbs[(j * 2 + 1) * kN + k];
        }
        Sa[k] = negmod(reduce64(sa, cb.q, cb.barrett), cb.q);
        Sb[k] = negmod(reduce64(sb, cb.q, cb.barrett), cb.q);
    }
    cta_ntt_inverse<T>(Sa, tabs.tw[CH_BS], CH_BS);
    cta_ntt_inverse<T>(Sb, tabs.tw[CH_BS], CH_BS);

    // x2b += auto_g(b mod bsMod)   (automorphic_rns, twosteps.cpp:1045-1048)
    const uint32_t ginv = pow5_mod2n(2048u - (uint32_t)(ki + 1));
    for (int k = threadIdx.x; k < kN; k += T) {
        bool neg;
        const int src = auto_src(k, ginv, &neg);
        uint32_t v = a.srcBbs[src];
        if (neg) v = negmod(v, cb.q);
        Sb[k] = addmod(Sb[k], v, cb.q);
        if (inter) {
            a.inter_bs[k] = Sa[k];
            a.inter_bs[kN + k] = Sb[k];
        }
    }
    __syncthreads();

    uint64_t* __restrict__ cbuf = a.cipherbuf;
#pragma unroll 1
    for (int ch = CH_Q1; ch <= CH_Q2; ch++) {
        const ChanConst cc = c_dev.ch[ch];
        // a component
        for (int k = threadIdx.x; k < kN; k += T) W[k] = Sa[k];
        cta_ntt_forward<T>(W, tabs.tw[ch], ch);
        for (int k = threadIdx.x; k < kN; k += T) {
            const int p = perm[k];
            uint64_t s = 0;
            for (int j = 0; j < ell; j++)
                s += (uint64_t)dig[(j * 3 + ch) * kN + p] * kcrt[((j * 2 + 0) * 2 + ch) * kN + k];
            const uint32_t A = negmod(reduce64(s, cc.q, cc.barrett), cc.q);
            if (inter) a.interA[ch * kN + k] = A;
            const uint32_t ra = shoup_mul(submod(A, W[k], cc.q), cc.bsinv, cc.bsinv_p, cc.q);
            if (ch == CH_Q1) Ra[k] = ra;
            else cbuf[((size_t)k * a.N1 + col) * 2 + 0] = (uint64_t)Ra[k] | ((uint64_t)ra << 32);
        }
        __syncthreads();
        // b component
        for (int k = threadIdx.x; k < kN; k += T) W[k] = Sb[k];
        cta_ntt_forward<T>(W, tabs.tw[ch], ch);
        for (int k = threadIdx.x; k < kN; k += T) {
            const int p = perm[k];
            uint64_t s = 0;
            for (int j = 0; j < ell; j++)
                s += (uint64_t)dig[(j * 3 + ch) * kN + p] * kcrt[((j * 2 + 1) * 2 + ch) * kN + k];
            const uint32_t Bn = negmod(reduce64(s, cc.q, cc.barrett), cc.q);
            const uint32_t Bt = addmod(Bn, a.srcB[ch * kN + sig[k]], cc.q);
            if (inter) a.interB[ch * kN + k] = Bt;
            const uint32_t rb = shoup_mul(submod(Bt, W[k], cc.q), cc.bsinv, cc.bsinv_p, cc.q);
            if (ch == CH_Q1) Rb[k] = rb;
            else cbuf[((size_t)k * a.N1 + col) * 2 + 1] = (uint64_t)Rb[k] | ((uint64_t)rb << 32);
        }
        __syncthreads();
    }
}

}  // namespace kspir
