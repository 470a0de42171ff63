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

#include <type_traits>

#include "ntt.cuh"
#include "pipeline.cuh"
#include "ptx.cuh"

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
    int32_t cb_rm;           // 1: write cipherbuf rotation-major (see cipherbuf_rm_idx)
};

// Rotation-major cipherbuf, the layout the tensor-core scan's operand split
// reads: u32 [N1 columns][2 comp][2 primes][N slots], so that a rotation's
// CTA writes whole contiguous polynomials.  The reference layout
// ([N][N1][2] words, primes packed in one word) scatters every 4-byte store
// across a 16 * N1-byte stride; the CUDA-core scan streams it per slot.
__host__ __device__ __forceinline__ size_t cipherbuf_rm_idx(int col, int comp, int ch, int z) {
    return ((size_t)(col * 2 + comp) * 2 + ch) * kN + z;
}

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

constexpr int kBabyPairSmem = kN * 8 + 2 * kPadN * 4;   // twiddles + two padded polynomials
constexpr int kPerThread = kN / kNttThreads; // 8 coefficients per thread

// Per-rotation state shared by the two kernel shapes below.
struct BabyRot {
    int ki, comp, col, tid;
    bool inter;
    size_t wo;              // workspace offset of the query
    const uint32_t* kbs;    // bsMod keys of rotation ki
    const uint32_t* kcrt;   // crt keys of rotation ki
    const int32_t* perm;    // caller permutation of rotation ki
};

// Loads of the query-side inputs (digits, b): written by earlier kernels, so a
// stand-alone launch (CtaSync) reads them through L1 (their gathers reuse
// lines across the rotations on an SM); inside the fused answer kernel other
// CTAs write them during the launch, so those loads bypass L1.
template <class Sync>
__device__ __forceinline__ uint32_t ld_query(const uint32_t* p) {
    if constexpr (std::is_same<Sync, CtaSync>::value) return __ldg(p);
    else return __ldcg(p);
}

// perm[k] of this thread's coefficients (reloaded by each multiply-accumulate
// rather than held in registers across the transforms)
__device__ __forceinline__ void baby_perm(const BabyRot& R, int* pk) {
#pragma unroll
    for (int it = 0; it < kPerThread; it++) pk[it] = __ldg(R.perm + R.tid + it * kNttThreads);
}

// The workspace pointers of BabyArgs are slot-0 pointers: each use adds the
// query's workspace offset R.wo (kept as one value rather than seven shifted
// pointers, which would pin fourteen registers for the whole kernel).
template <int ELL>
__device__ __forceinline__ void baby_setup(BabyRot& R, const BabyArgs& a, const ClientKeysDev& keys,
                                           const Batch& bt, int ki, int comp) {
    R.ki = ki;
    R.comp = comp;
    R.col = a.col_base + ki;
    R.tid = threadIdx.x;
    R.inter = (ki == a.inter_idx);
    R.wo = ws_off(bt);
    const size_t ko = key_off(bt);
    R.kbs = shifted(keys.baby_bs, ko) + (size_t)ki * ELL * 2 * kN;
    R.kcrt = shifted(keys.baby_crt, ko) + (size_t)ki * ELL * 2 * 2 * kN;
    R.perm = a.perms + (size_t)(ki + 1) * kN;
}

// x2 of this component into S (coefficient form, canonical mod bsMod):
//   INTT_bs(-sum_j d_j[perm] * key_j) (+ auto_g(b mod bsMod) for comp 1).
// The caller has staged the bsMod inverse twiddles into tws (unsynchronised).
// export_inter: this CTA writes the intermediate rotation's x2.
template <int ELL, class Sync = CtaSync>
__device__ __forceinline__ void baby_bs_part(const BabyRot& R, const BabyArgs& a, uint32_t* S, const uint2* tws,
                                             bool export_inter) {
    const int tid = R.tid;
    {
        const ChanConst cb = c_dev.ch[CH_BS];
        int pk[kPerThread];
        baby_perm(R, pk);
        uint64_t acc[kPerThread];
#pragma unroll
        for (int it = 0; it < kPerThread; it++) acc[it] = 0;
#pragma unroll
        for (int j = 0; j < ELL; j++) {
            const uint32_t* d = shifted(a.dig, R.wo) + (size_t)(j * 3 + CH_BS) * kN;
            const uint32_t* kk = R.kbs + (size_t)(j * 2 + R.comp) * kN;
#pragma unroll
            for (int it = 0; it < kPerThread; it++)
                acc[it] += (uint64_t)ld_query<Sync>(d + pk[it]) * __ldg(kk + tid + it * kNttThreads);
        }
#pragma unroll
        for (int it = 0; it < kPerThread; it++)
            S[pidx(tid) + it * kPadStep] = negmod(reduce64(acc[it], cb.q, cb.barrett), cb.q);
    }
    cta_ntt_inverse<Sync>(S, tws, CH_BS);

    if (R.comp == 1) {
        // x2b += auto_g(b mod bsMod)   (automorphic_rns, twosteps.cpp:1045-1048)
        const uint32_t ginv = pow5_mod2n(2048u - (uint32_t)(R.ki + 1));
        const uint32_t qb = c_dev.ch[CH_BS].q;
#pragma unroll
        for (int it = 0; it < kPerThread; it++) {
            const int k = tid + it * kNttThreads;
            const int pk2 = pidx(tid) + it * kPadStep;
            bool neg;
            const int src = auto_src(k, ginv, &neg);
            uint32_t v = ld_query<Sync>(shifted(a.srcBbs, R.wo) + src);
            if (neg) v = negmod(v, qb);
            S[pk2] = addmod(S[pk2], v, qb);
        }
    }
    if (R.inter && export_inter) {
#pragma unroll
        for (int it = 0; it < kPerThread; it++) {
            const int k = tid + it * kNttThreads;
            shifted(a.inter_bs, R.wo)[R.comp * kN + k] = S[pidx(tid) + it * kPadStep];
        }
    }
}

// Prime ch of the rotation: NTT_ch(x2) from S (in place), the crt
// multiply-accumulate, the modswitch, and the cipherbuf store.  Starts with
// a barrier (x2 complete, tws free) and stages the forward twiddles itself.
template <int ELL, class Sync = CtaSync>
__device__ __forceinline__ void baby_crt_part(const BabyRot& R, const BabyArgs& a, uint32_t* S, uint2* tws,
                                              const NttTables& tabs, int ch) {
    const int tid = R.tid, comp = R.comp;
    const uint16_t* __restrict__ sig = a.sigma + (size_t)R.ki * kN;
    uint32_t* cb32 = reinterpret_cast<uint32_t*>(shifted(a.cipherbuf, R.wo));
    uint32_t* inter_out = shifted(comp == 0 ? a.interA : a.interB, R.wo);
    Sync::sync();   // x2 complete and the previous twiddles no longer read
    stage_twiddles(tws, tabs, ch, NTT_FWD);
    cta_ntt_forward<Sync, true>(S, tws, ch);   // NTT_ch(x2), x2 < bsMod < q; outputs in [0, 4q)

    const ChanConst cc = c_dev.ch[ch];
    int pk[kPerThread];
    baby_perm(R, pk);
    uint64_t acc[kPerThread];
#pragma unroll
    for (int it = 0; it < kPerThread; it++) acc[it] = 0;
#pragma unroll
    for (int j = 0; j < ELL; j++) {
        const uint32_t* d = shifted(a.dig, R.wo) + (size_t)(j * 3 + ch) * kN;
        const uint32_t* kk = R.kcrt + (size_t)((j * 2 + comp) * 2 + ch) * kN;
#pragma unroll
        for (int it = 0; it < kPerThread; it++)
            acc[it] += (uint64_t)ld_query<Sync>(d + pk[it]) * __ldg(kk + tid + it * kNttThreads);
    }
#pragma unroll
    for (int it = 0; it < kPerThread; it++) {
        const int k = tid + it * kNttThreads;
        uint32_t A = negmod(mod_crt(acc[it], ch), cc.q);
        if (comp == 1) A = addmod(A, ld_query<Sync>(shifted(a.srcB, R.wo) + ch * kN + sig[k]), cc.q);
        if (R.inter) inter_out[ch * kN + k] = A;
        // (A - S) bsMod^-1 with S in [0, 4q): A + 4q - S is in (0, 5q), and the
        // Shoup product reduces any 32-bit input to a canonical residue
        const uint32_t r = shoup_mul(A + 2 * cc.two_q - S[pidx(tid) + it * kPadStep], cc.bsinv, cc.bsinv_p, cc.q);
        if (a.cb_rm)
            cb32[cipherbuf_rm_idx(R.col, comp, ch, k)] = r;
        else
            cb32[(((size_t)k * a.N1 + R.col) * 2 + comp) * 2 + ch] = r;
    }
}

// One CTA per (rotation, component): blockIdx.x = 2*ki + comp, blockIdx.y =
// query of the batch.  The bsMod part runs once for both primes (six
// transforms per rotation; a shape with one CTA per prime as well, which
// recomputes it, ran eight and measured slower for single queries too once
// the reductions were minimum-form).  MINB 2: at 3 CTAs per SM (40-42 registers) it spills, and
// measured slower (batch of 64: baby steps 1.55 ms at 3, 1.32 ms at 2).
template <int ELL, int MINB>
__global__ void __launch_bounds__(kNttThreads, MINB) k_baby_pair(BabyArgs a, ClientKeysDev keys, NttTables tabs, Batch bt) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* S = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);
    uint32_t* S2 = S + kPadN;
    BabyRot R;
    pdl_launch_dependents();
    stage_twiddles(tws, tabs, CH_BS, NTT_INV);
    baby_setup<ELL>(R, a, keys, bt, blockIdx.x >> 1, blockIdx.x & 1);
    pdl_wait();   // the digits come from the previous kernel
    baby_bs_part<ELL>(R, a, S, tws, true);
    // the second prime transforms its own copy of x2 (each thread copies the
    // coefficients it wrote: no barrier needed)
#pragma unroll
    for (int it = 0; it < kPerThread; it++) S2[pidx(R.tid) + it * kPadStep] = S[pidx(R.tid) + it * kPadStep];
    baby_crt_part<ELL>(R, a, S, tws, tabs, 0);
    baby_crt_part<ELL>(R, a, S2, tws, tabs, 1);
}

}  // namespace kspir
