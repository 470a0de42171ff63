// Giant steps (reference evalAutoRNSCRT, twosteps.cpp:599-677), the external
// product (externalProduct, lwe.cpp:761-808) and the RLWE packing tree
// (packingRLWEs / convertTwoRLWEs / evalAuto, answer.cpp:576-835).
//
// All three are key switches of the same shape: bring `a` to coefficient form,
// apply an automorphism, gadget-decompose, transform the digits, multiply by
// the key and accumulate.  Each runs as one fused kernel whose intermediates
// stay in shared memory (k_giant_fused, k_ext_fused, k_pack_fused).  The
// unfused element-wise decomposition and multiply-accumulate kernels of the
// external product remain for the allocation-free entry point.
#pragma once

#include "ntt.cuh"
#include "pipeline.cuh"
#include "ptx.cuh"

namespace kspir {

// ---------------------------------------------------------------------------
// giant steps

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
constexpr int kMacSmem = kN * 8 + kPadN * 4;

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
        s[pidx(k)] = init ? addmod(init[((size_t)r * 4 + comp * 2 + ch) * kN + k], m, cc.q) : m;
    }
    cta_ntt_inverse(s, tws, ch);
    uint32_t* o = ext + ((size_t)r * 4 + comp * 2 + ch) * kN;
#pragma unroll
    for (int k = threadIdx.x; k < kN; k += T) o[k] = s[pidx(k)];
}

}  // namespace kspir

namespace kspir {

// ---------------------------------------------------------------------------
// fused giant step: one CTA per (r, c >= 1) (blockIdx.y = query of the batch) runs the whole key switch of
// evalAutoRNSCRT for output[c] (twosteps.cpp:612-672) in shared memory:
//   INTT(a) per prime -> compose -> X -> X^g -> decompose (ell digits)
//   -> digit transforms -> -sum_j d_j * key[j]  and  b[sigma_g] - sum_j d_j * key[j]
// and adds both, canonical, into the sub-database's accumulator (u32 words
// in L2; the scan output is only read).  k_giant_finish then adds output[0]
// and reduces.  A u32 word holds at most kGiantTermsPerAcc terms below
// q1 (16 (q1 - 1) < 2^32); with more giant steps per sub-database (N1 = 64:
// 31) rows c odd go to acc0 and rows c even to acc1.
constexpr int kGiantTermsPerAcc = 16;
static_assert((uint64_t)kGiantTermsPerAcc * (kQ1 - 1) < (1ull << 32) && kQ2 < kQ1, "giant accumulator width");

constexpr int kGiantPolys = 4;   // two primes x two digits (ell = 2)
constexpr int kPerThreadG = kN / kNttThreads;
// The transforms read the device twiddle tables through L1 rather than a
// staged shared-memory copy: 72 KiB of shared memory and 40 registers give 3
// CTAs per SM (a staged copy made it 104 KiB and 2 CTAs per SM, 8 % slower).
constexpr int kGiantSmem = kGiantPolys * kPadN * 4;

template <int ELL>
__global__ void __launch_bounds__(kNttThreads, 3)
    k_giant_fused(const uint32_t* __restrict__ sout, uint32_t* acc0, uint32_t* acc1,
                  const uint32_t* __restrict__ gkeys, const uint16_t* __restrict__ gsigma, int N1, NttTables tabs,
                  GadgetB g, int R, Batch bt) {
    static_assert(2 * ELL <= kGiantPolys, "shared-memory polynomials");
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint32_t* P = reinterpret_cast<uint32_t*>(smem_raw);   // [kGiantPolys][N]
    const int N2 = kN / 2 / N1;
    const int rows = R * N2;
    const int rc = blockIdx.x;
    const int r = rc / (N2 - 1), c = rc % (N2 - 1) + 1;
    const int row = r * N2 + c;
    const int tid = threadIdx.x;
    sout = shifted(sout, ws_off(bt));
    gkeys = shifted(gkeys, key_off(bt));
    uint32_t* acc = shifted((acc1 && !(c & 1)) ? acc1 : acc0, ws_off(bt)) + (size_t)r * 4 * kN;
    pdl_launch_dependents();

    // a of output[c], both primes, to coefficient form
#pragma unroll
    for (int ch = 0; ch < 2; ch++) {
        pdl_wait();   // the scan output comes from the previous kernel
#pragma unroll
        for (int k = tid; k < kN / 4; k += kNttThreads)
            *reinterpret_cast<uint4*>(P + ch * kPadN + pidx(4 * k)) =
                __ldcg(reinterpret_cast<const uint4*>(sout + sout_idx(row, 0 * 2 + ch, 4 * k, rows)));
        cta_ntt_inverse(P + ch * kPadN, twiddle_table(tabs, ch, NTT_INV), ch);
    }
    // X -> X^g, g = 5^(N1 c), then the digits (registers first: P is overwritten)
    const uint32_t e = (uint32_t)(N1 * c) & 2047u;
    uint32_t ginv = 1, b5 = 5, x = (2048u - e) & 2047u;
    while (x) { if (x & 1) ginv = (ginv * b5) & (2 * kN - 1); b5 = (b5 * b5) & (2 * kN - 1); x >>= 1; }
    uint32_t dres[kPerThreadG][ELL][2];
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
        bool neg;
        const int src = auto_src(k, ginv, &neg);
        uint64_t v = crt_compose_res(P[pidx(src)], P[kPadN + pidx(src)]);
        if (neg && v) v = kCrtMod - v;
        int32_t dig[kMaxEll];
        decompose_b(v, kCrtMod, g, dig);
#pragma unroll
        for (int j = 0; j < ELL; j++) {
            dres[it][j][0] = signed_to_res(dig[j], kQ1);
            dres[it][j][1] = signed_to_res(dig[j], kQ2);
        }
    }
    __syncthreads();
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++)
#pragma unroll
        for (int j = 0; j < ELL; j++)
#pragma unroll
            for (int ch = 0; ch < 2; ch++) P[(j * 2 + ch) * kPadN + pidx(tid) + it * kPadStep] = dres[it][j][ch];
    // digit transforms and the key multiply-accumulate, prime by prime
    const uint32_t* key = gkeys + (size_t)(c - 1) * ELL * 2 * 2 * kN;   // [ELL][2 comp][2 ch][N]
    const uint16_t* sig = gsigma + (size_t)(c - 1) * kN;
#pragma unroll 1
    for (int ch = 0; ch < 2; ch++) {
        __syncthreads();
        // digits j of this prime: P[j*2+ch], left in [0, 4q) (they only feed the
        // exact multiply-accumulate below)
        cta_ntt_forward_m<ELL, CtaSync, true>(P + ch * kPadN, 2 * kPadN, twiddle_table(tabs, ch, NTT_FWD), ch);
        const ChanConst cc = c_dev.ch[ch];
#pragma unroll
        for (int it = 0; it < kPerThreadG; it++) {
            const int k = tid + it * kNttThreads;
            uint64_t sa = 0, sb = 0;
#pragma unroll
            for (int j = 0; j < ELL; j++) {
                const uint32_t d = P[(j * 2 + ch) * kPadN + pidx(tid) + it * kPadStep];
                mad_wide(sa, d, __ldg(key + ((j * 2 + 0) * 2 + ch) * kN + k));
                mad_wide(sb, d, __ldg(key + ((j * 2 + 1) * 2 + ch) * kN + k));
            }
            const uint32_t bv = __ldcg(sout + sout_idx(row, 1 * 2 + ch, sig[k], rows));
            atomicAdd(acc + (size_t)(0 * 2 + ch) * kN + k, negmod(mod_crt(sa, ch), cc.q));
            atomicAdd(acc + (size_t)(1 * 2 + ch) * kN + k, addmod(bv, negmod(mod_crt(sb, ch), cc.q), cc.q));
        }
    }
}

// result[r][comp][ch][k] = (output[0] + the giant-step accumulators) mod q,
// in place over acc0 (= result).  One thread per four consecutive slots.
__global__ void k_giant_finish(const uint32_t* __restrict__ sout, uint32_t* result, const uint32_t* acc1, int R,
                               int N2, Batch bt) {
    pdl_launch_dependents();
    pdl_wait();
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)R * 4 * (kN / 4)) return;
    sout = shifted(sout, ws_off(bt));
    result = shifted(result, ws_off(bt));
    const int z = (int)(idx % (kN / 4)) * 4;
    const int cc_ = (int)((idx / (kN / 4)) % 4);      // comp * 2 + ch
    const int r = (int)(idx / (4 * (kN / 4)));
    const ChanConst q = c_dev.ch[cc_ & 1];
    uint4* res = reinterpret_cast<uint4*>(result + ((size_t)r * 4 + cc_) * kN + z);
    const uint4 a = __ldcg(res);
    const uint4 w = __ldcg(reinterpret_cast<const uint4*>(sout + sout_idx(r * N2, cc_, z, R * N2)));
    uint64_t v0 = (uint64_t)a.x + w.x, v1 = (uint64_t)a.y + w.y, v2 = (uint64_t)a.z + w.z, v3 = (uint64_t)a.w + w.w;
    if (acc1) {
        const uint4 b = __ldcg(reinterpret_cast<const uint4*>(shifted(acc1, ws_off(bt)) + ((size_t)r * 4 + cc_) * kN + z));
        v0 += b.x; v1 += b.y; v2 += b.z; v3 += b.w;
    }
    *res = make_uint4(reduce64(v0, q.q, q.barrett), reduce64(v1, q.q, q.barrett), reduce64(v2, q.q, q.barrett),
                      reduce64(v3, q.q, q.barrett));
}

}  // namespace kspir

namespace kspir {

// ---------------------------------------------------------------------------
// fused packing level: one CTA per (pair j, prime ch) runs convertTwoRLWEs
// (answer.cpp:720-739) with its evalAuto key switch (answer.cpp:576-648) in
// shared memory.  It reads level input `in` and writes level output `out`
// (two buffers: both primes of in[j] are read while the other CTA of the pair
// writes its prime of out[j]).
//   c' = X^I c,  r1 = r0 - c',  c2 = c' + r0,  temp = auto_g(r1), g = N/I + 1
//   a' = -sum_d dig_d * key[d].a,  b' = NTT(temp.b) - sum_d dig_d * key[d].b
//   out[j] = INTT(a', b') + c2
constexpr int kPackPolys = 5;    // ell = 4 digits + temp.b
constexpr int kPackSmem = kN * 8 + kPackPolys * kPadN * 4;

template <int ELL>
__global__ void __launch_bounds__(kNttThreads) k_pack_fused(const uint32_t* __restrict__ in,
                                                            uint32_t* __restrict__ out,
                                                            const uint32_t* __restrict__ key, int I, uint32_t ginv,
                                                            NttTables tabs, GadgetB g, Batch bt) {
    static_assert(ELL + 1 <= kPackPolys, "shared-memory polynomials");
    extern __shared__ __align__(16) uint8_t smem_raw[];
    in = shifted(in, ws_off(bt));
    out = shifted(out, ws_off(bt));
    key = shifted(key, key_off(bt));
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* P = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);   // [kPackPolys][N]
    const int j = blockIdx.x >> 1, ch = blockIdx.x & 1;
    const int tid = threadIdx.x;
    const uint32_t* r0 = in + (size_t)j * 4 * kN;
    const uint32_t* cc = in + (size_t)(I + j) * 4 * kN;
    const uint32_t q = c_dev.ch[ch].q;
    pdl_launch_dependents();
    stage_twiddles(tws, tabs, ch, NTT_FWD);
    pdl_wait();   // the level input comes from the previous kernel
    // launched after that kernel completes (no early launch), and no CTA writes
    // the level input: its gathers below read through L1
    // X^I c at position p of polynomial (comp, prime)
    auto cshift = [&](int comp, int pch, int p) -> uint32_t {
        const int s = p - I;
        const uint32_t qq = pch ? kQ2 : kQ1;
        return s >= 0 ? __ldg(cc + (comp * 2 + pch) * kN + s) : negmod(__ldg(cc + (comp * 2 + pch) * kN + s + kN), qq);
    };
    uint32_t c2v[kPerThreadG][2];
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
#pragma unroll
        for (int comp = 0; comp < 2; comp++)
            c2v[it][comp] = addmod(cshift(comp, ch, k), __ldg(r0 + (comp * 2 + ch) * kN + k), q);
        bool neg;
        const int src = auto_src(k, ginv, &neg);
        uint32_t ra[2];
#pragma unroll
        for (int pch = 0; pch < 2; pch++) {
            const uint32_t qq = pch ? kQ2 : kQ1;
            const uint32_t v = submod(__ldg(r0 + (0 * 2 + pch) * kN + src), cshift(0, pch, src), qq);
            ra[pch] = neg ? negmod(v, qq) : v;
        }
        int32_t dig[kMaxEll];
        decompose_b(crt_compose_res(ra[0], ra[1]), kCrtMod, g, dig);
        const int pk = pidx(tid) + it * kPadStep;
#pragma unroll
        for (int d = 0; d < ELL; d++) P[d * kPadN + pk] = signed_to_res(dig[d], q);
        const uint32_t vb = submod(__ldg(r0 + (1 * 2 + ch) * kN + src), cshift(1, ch, src), q);
        P[ELL * kPadN + pk] = neg ? negmod(vb, q) : vb;
    }
    cta_ntt_forward_m<ELL + 1, CtaSync, true>(P, kPadN, tws, ch);   // outputs in [0, 4q)
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
        uint64_t sa = 0, sb = 0;
#pragma unroll
        for (int d = 0; d < ELL; d++) {
            const uint32_t dv = P[d * kPadN + pidx(tid) + it * kPadStep];
            mad_wide(sa, dv, __ldg(key + ((d * 2 + 0) * 2 + ch) * kN + k));
            mad_wide(sb, dv, __ldg(key + ((d * 2 + 1) * 2 + ch) * kN + k));
        }
        const uint32_t a2 = negmod(mod_crt(sa, ch), q);
        const int pk = pidx(tid) + it * kPadStep;
        const uint32_t b2 = submod(canon4q(P[ELL * kPadN + pk], q), mod_crt(sb, ch), q);
        P[pk] = a2;            // only this thread reads index k of these rows
        P[kPadN + pk] = b2;
    }
    stage_twiddles(tws, tabs, ch, NTT_INV);   // the forward transforms ended with a barrier
    cta_ntt_inverse_m<2>(P, kPadN, tws, ch);
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
#pragma unroll
        for (int comp = 0; comp < 2; comp++)
            out[((size_t)j * 4 + comp * 2 + ch) * kN + k] = addmod(P[comp * kPadN + pidx(tid) + it * kPadStep], c2v[it][comp], q);
    }
}

// ---------------------------------------------------------------------------
// packing level split over more CTAs, for single queries and small batches:
// the fused kernel's CTA runs ELL + 1 forward and 2 inverse transforms in a
// row, and the last levels have only 2 * I CTAs, so a level's latency is
// those seven transforms.  Split, each CTA runs one:
//   k_pack_split_fwd  (pair j, prime ch, d <= ELL): digit d (or temp.b for
//                     d = ELL) -> transform -> its terms dig_d * key[d].a/.b
//                     into part[j][ch][d][comp]
//   k_pack_split_inv  (pair j, prime ch, comp): the sum of the terms ->
//                     inverse transform -> + c2 into out[j]
// Same residues as k_pack_fused (sums mod q in another order).
constexpr int kPackPartPolys = 2 * 5 * 2;   // per pair: [prime][ELL + 1][comp]
constexpr int kPackSplitSmem = kN * 8 + kPadN * 4;

// One split forward task, pair j, prime ch, digit d (d = ELL: temp.b); in,
// part and key already point at the query's workspace and key slot.  Shared
// with the fused answer kernel (Sync = its named barrier).
template <int ELL, class Sync>
__device__ __forceinline__ void pack_split_fwd_body(const uint32_t* __restrict__ in, uint32_t* __restrict__ part,
                                                    const uint32_t* __restrict__ key, int I, uint32_t ginv,
                                                    const NttTables& tabs, const GadgetB& g, int j, int ch, int d,
                                                    uint8_t* smem_raw) {
    static_assert(2 * (ELL + 1) * 2 <= kPackPartPolys, "term buffer");
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* S = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);
    const int tid = threadIdx.x;
    const uint32_t* r0 = in + (size_t)j * 4 * kN;
    const uint32_t* cc = in + (size_t)(I + j) * 4 * kN;
    const uint32_t q = c_dev.ch[ch].q;
    pdl_launch_dependents();
    stage_twiddles(tws, tabs, ch, NTT_FWD);
    // the key words of this digit, loaded while the previous kernel finishes
    // (keys are never written by the answer), used after the transform
    uint32_t ka[kPerThreadG], kb[kPerThreadG];
    if (d < ELL) {
#pragma unroll
        for (int it = 0; it < kPerThreadG; it++) {
            ka[it] = __ldg(key + ((d * 2 + 0) * 2 + ch) * kN + tid + it * kNttThreads);
            kb[it] = __ldg(key + ((d * 2 + 1) * 2 + ch) * kN + tid + it * kNttThreads);
        }
    }
    pdl_wait();   // the level input comes from the previous kernel
    auto cshift = [&](int comp, int pch, int p) -> uint32_t {   // (X^I c)[p]
        const int s = p - I;
        const uint32_t qq = pch ? kQ2 : kQ1;
        return s >= 0 ? __ldcg(cc + (comp * 2 + pch) * kN + s) : negmod(__ldcg(cc + (comp * 2 + pch) * kN + s + kN), qq);
    };
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
        bool neg;
        const int src = auto_src(k, ginv, &neg);
        uint32_t v;
        if (d < ELL) {
            uint32_t ra[2];
#pragma unroll
            for (int pch = 0; pch < 2; pch++) {
                const uint32_t qq = pch ? kQ2 : kQ1;
                const uint32_t x = submod(__ldcg(r0 + (0 * 2 + pch) * kN + src), cshift(0, pch, src), qq);
                ra[pch] = neg ? negmod(x, qq) : x;
            }
            int32_t dig[kMaxEll];
            decompose_b(crt_compose_res(ra[0], ra[1]), kCrtMod, g, dig);
            v = signed_to_res(dig[d], q);
        } else {
            const uint32_t vb = submod(__ldcg(r0 + (1 * 2 + ch) * kN + src), cshift(1, ch, src), q);
            v = neg ? negmod(vb, q) : vb;
        }
        S[pidx(tid) + it * kPadStep] = v;
    }
    cta_ntt_forward<Sync, true>(S, tws, ch);   // outputs in [0, 4q)
    uint32_t* pa = part + (((size_t)j * 2 + ch) * (ELL + 1) + d) * 2 * kN;
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
        const uint32_t dv = S[pidx(tid) + it * kPadStep];
        if (d < ELL) {
            pa[k] = mod_crt((uint64_t)dv * ka[it], ch);
            pa[kN + k] = mod_crt((uint64_t)dv * kb[it], ch);
        } else {
            pa[k] = canon4q(dv, q);   // NTT(temp.b)
        }
    }
}

template <int ELL>
__global__ void __launch_bounds__(kNttThreads) k_pack_split_fwd(const uint32_t* __restrict__ in,
                                                                uint32_t* __restrict__ part,
                                                                const uint32_t* __restrict__ key, int I,
                                                                uint32_t ginv, NttTables tabs, GadgetB g, Batch bt) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int d = blockIdx.x % (ELL + 1), ch = (blockIdx.x / (ELL + 1)) & 1, j = blockIdx.x / (ELL + 1) / 2;
    pack_split_fwd_body<ELL, CtaSync>(shifted(in, ws_off(bt)), shifted(part, ws_off(bt)), shifted(key, key_off(bt)), I,
                                      ginv, tabs, g, j, ch, d, smem_raw);
}

// c2out (or null): the reference's packingRLWEs leaves c2 = X^I c + r of the
// merge of (j, I + j) in rlwes[I + j] (answer.cpp:727-731, 821-828); the
// staged entry point returns it there, as [r][comp][ch][N] residues.
template <int ELL, class Sync>
__device__ __forceinline__ void pack_split_inv_body(const uint32_t* __restrict__ in, const uint32_t* __restrict__ part,
                                                    uint32_t* __restrict__ out, int I, const NttTables& tabs, int j,
                                                    int ch, int comp, uint32_t* __restrict__ c2out,
                                                    uint8_t* smem_raw) {
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* S = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);
    const int tid = threadIdx.x;
    const uint32_t q = c_dev.ch[ch].q;
    pdl_launch_dependents();
    stage_twiddles(tws, tabs, ch, NTT_INV);
    pdl_wait();   // the terms come from the previous kernel
    const uint32_t* pj = part + ((size_t)j * 2 + ch) * (ELL + 1) * 2 * kN;
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
        uint32_t sum = 0;
#pragma unroll
        for (int d = 0; d < ELL; d++) sum = addmod(sum, __ldcg(pj + ((size_t)d * 2 + comp) * kN + k), q);
        // a' = -sum_d dig_d key[d].a ;  b' = NTT(temp.b) - sum_d dig_d key[d].b
        S[pidx(tid) + it * kPadStep] = comp == 0 ? negmod(sum, q) : submod(__ldcg(pj + (size_t)ELL * 2 * kN + k), sum, q);
    }
    // c2 = X^I c + r of the level input, loaded ahead of the transform
    const uint32_t* r0 = in + (size_t)j * 4 * kN;
    const uint32_t* cc = in + (size_t)(I + j) * 4 * kN + (comp * 2 + ch) * kN;
    uint32_t c2[kPerThreadG];
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
        const int s = k - I;
        const uint32_t sh = s >= 0 ? __ldcg(cc + s) : negmod(__ldcg(cc + s + kN), q);
        c2[it] = addmod(sh, __ldcg(r0 + (comp * 2 + ch) * kN + k), q);
        if (c2out) c2out[((size_t)(I + j) * 4 + comp * 2 + ch) * kN + k] = c2[it];
    }
    cta_ntt_inverse<Sync>(S, tws, ch);
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
        out[((size_t)j * 4 + comp * 2 + ch) * kN + k] = addmod(S[pidx(tid) + it * kPadStep], c2[it], q);
    }
}

template <int ELL>
__global__ void __launch_bounds__(kNttThreads) k_pack_split_inv(const uint32_t* __restrict__ in,
                                                                const uint32_t* __restrict__ part,
                                                                uint32_t* __restrict__ out, int I, NttTables tabs,
                                                                Batch bt, uint32_t* __restrict__ c2out) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    const int comp = blockIdx.x & 1, ch = (blockIdx.x >> 1) & 1, j = blockIdx.x >> 2;
    pack_split_inv_body<ELL, CtaSync>(shifted(in, ws_off(bt)), shifted(part, ws_off(bt)), shifted(out, ws_off(bt)), I,
                                      tabs, j, ch, comp, shifted(c2out, ws_off(bt)), smem_raw);
}

// The external product after first_dim is in coefficient form in P[comp * 2 +
// prime] (both primes, as the decomposition needs the composed word): signed
// digits of a and b, their transforms on prime ch, init (or 0) + sum_row
// row * rgsw[row], inverse transform, into ext [comp][ch][N].  rgsw, init and
// ext point at the query's key slot and its polynomial r.
template <int ELL, class Sync>
__device__ __forceinline__ void ext_tail(uint32_t* P, uint2* tws, const uint32_t* __restrict__ rgsw,
                                         const uint32_t* __restrict__ init, uint32_t* __restrict__ ext,
                                         const NttTables& tabs, const GadgetS& g, int ch) {
    const int tid = threadIdx.x;
    // signed digits of a and b (rows comp * ELL + t), residues of this prime
    uint32_t dres[kPerThreadG][2 * ELL];
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
#pragma unroll
        for (int comp = 0; comp < 2; comp++) {
            int32_t dig[kMaxEll];
            const int pk = pidx(tid) + it * kPadStep;
            decompose_signed(crt_compose_res(P[(comp * 2 + 0) * kPadN + pk], P[(comp * 2 + 1) * kPadN + pk]), kCrtMod, g,
                             dig);
#pragma unroll
            for (int t = 0; t < ELL; t++) dres[it][comp * ELL + t] = signed_to_res(dig[t], ch ? kQ2 : kQ1);
        }
    }
    Sync::sync();
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++)
#pragma unroll
        for (int row = 0; row < 2 * ELL; row++) P[row * kPadN + pidx(tid) + it * kPadStep] = dres[it][row];
    stage_twiddles(tws, tabs, ch, NTT_FWD);
    cta_ntt_forward_m<2 * ELL, Sync, true>(P, kPadN, tws, ch);   // digits in [0, 4q), for the exact sum below
    const ChanConst cq = c_dev.ch[ch];
    uint32_t outv[kPerThreadG][2];
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
#pragma unroll
        for (int comp = 0; comp < 2; comp++) {
            uint64_t s = 0;
#pragma unroll
            for (int row = 0; row < 2 * ELL; row++)
                mad_wide(s, P[row * kPadN + pidx(tid) + it * kPadStep], __ldg(rgsw + ((row * 2 + comp) * 2 + ch) * kN + k));
            const uint32_t m = mod_crt(s, ch);
            outv[it][comp] = init ? addmod(__ldcg(init + (size_t)(comp * 2 + ch) * kN + k), m, cq.q) : m;
        }
    }
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int pk = pidx(tid) + it * kPadStep;
        P[pk] = outv[it][0];        // only this thread reads this slot of rows 0, 1
        P[kPadN + pk] = outv[it][1];
    }
    stage_twiddles(tws, tabs, ch, NTT_INV);   // the forward transforms ended with a barrier
    cta_ntt_inverse_m<2, Sync>(P, kPadN, tws, ch);
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++) {
        const int k = tid + it * kNttThreads;
#pragma unroll
        for (int comp = 0; comp < 2; comp++)
            ext[(size_t)(comp * 2 + ch) * kN + k] = P[comp * kPadN + pidx(tid) + it * kPadStep];
    }
}

// ---------------------------------------------------------------------------
// fused external product: one CTA per (r, prime ch) runs externalProduct
// (lwe.cpp:761-808) in shared memory:
//   INTT(first_dim) (both primes, to compose) -> decompose_rlwe (2 ell rows)
//   -> row transforms -> init + sum_row row * rgsw[row] -> INTT
constexpr int kExtPolys = 4;
constexpr int kExtSmem = kN * 8 + kExtPolys * kPadN * 4;

template <int ELL>
__global__ void __launch_bounds__(kNttThreads) k_ext_fused(const uint32_t* __restrict__ first_dim,
                                                           const uint32_t* __restrict__ rgsw,
                                                           const uint32_t* __restrict__ init,
                                                           uint32_t* __restrict__ ext,
                                                           uint32_t* __restrict__ coef_out, NttTables tabs,
                                                           GadgetS g, Batch bt) {
    static_assert(2 * ELL <= kExtPolys, "shared-memory polynomials");
    extern __shared__ __align__(16) uint8_t smem_raw[];
    first_dim = shifted(first_dim, ws_off(bt));
    init = shifted(init, ws_off(bt));
    ext = shifted(ext, ws_off(bt));
    coef_out = shifted(coef_out, ws_off(bt));
    rgsw = shifted(rgsw, key_off(bt));
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* P = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);   // [4][N]
    const int r = blockIdx.x >> 1, ch = blockIdx.x & 1;
    const uint32_t* fd = first_dim + (size_t)r * 4 * kN;          // [comp][prime][N]
    pdl_launch_dependents();
    // first_dim to coefficient form, all four polynomials (P[comp * 2 + prime])
#pragma unroll
    for (int pch = 0; pch < 2; pch++) {
        if (pch) __syncthreads();
        stage_twiddles(tws, tabs, pch, NTT_INV);
        pdl_wait();   // the first-dimension results come from the previous kernel
#pragma unroll
        for (int comp = 0; comp < 2; comp++) {
            poly_to_smem(P + (comp * 2 + pch) * kPadN, fd + (comp * 2 + pch) * kN);
        }
        cta_ntt_inverse_m<2>(P + pch * kPadN, 2 * kPadN, tws, pch);   // a and b of this prime
    }
    if (coef_out && ch == 0) {
#pragma unroll
        for (int i = 0; i < 4; i++) poly_from_smem(coef_out + ((size_t)r * 4 + i) * kN, P + i * kPadN);
    }
    ext_tail<ELL, CtaSync>(P, tws, rgsw, init ? init + (size_t)r * 4 * kN : nullptr, ext + (size_t)r * 4 * kN, tabs, g,
                           ch);
}

}  // namespace kspir
