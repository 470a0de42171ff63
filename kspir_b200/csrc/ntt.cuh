// CTA-level negacyclic NTT of length 4096 on one residue channel, operating on
// a shared-memory array, so every kernel fuses its transforms with their
// producers and consumers.
//
// Order and root follow HEXL as the reference uses it: the forward transform
// maps natural order to bit-reversed order, slot j holding
// sum_k x_k psi^((2 bitrev(j) + 1) k)  (reference utils.cpp:1473-1478), and the
// inverse includes N^-1.  Outputs are canonical.
//
// 512 threads, one radix-8 unit (8 elements, three butterfly layers) per
// thread per pass: four passes and four __syncthreads per transform.  Harvey
// lazy butterflies on 32-bit words (q < 2^28, values < 4q < 2^30) with Shoup
// twiddles.  The twiddles of one direction of one channel are staged into
// shared memory first (stage_twiddles) as uint2 {w, floor(w 2^32 / q)}.
//
// Shared-memory layout.  A polynomial occupies kPadN words: coefficient (or
// slot) i sits at pidx(i) = i + 4 (i / 32).  With that padding the element
// pattern of every pass (strides 512, 64 and 8 words, then eight contiguous
// words read as two 16-byte vectors) hits 32 distinct banks per warp access,
// and the position of element t of a thread's unit is pidx(base) plus a
// compile-time offset, so the padding costs no address arithmetic.
//
// Device table layout per channel: uint2 tw[2][N] (forward, inverse), entry
// m + i of level m = 2^l (root^brv(m + i) and its Shoup companion) stored
// "k-major" within its pass: for the pass p = l / 3 with unit count
// m0 = 8^p, level 2 m0 index 2 i0 + k sits at 2 m0 + k m0 + i0 and level 4 m0
// index 4 i0 + k at 4 m0 + k m0 + i0, so the twiddles a warp reads in one
// load are consecutive (tw_layout_pos gives the position).
#pragma once

#include "common.cuh"

namespace kspir {

constexpr int kNttThreads = 512;
constexpr int kPadN = kN + kN / 8;      // padded length of a polynomial in shared memory
constexpr int kPadStep = 576;           // pidx(i + 512) - pidx(i)

__host__ __device__ __forceinline__ int pidx(int i) { return i + ((i >> 5) << 2); }

// position of twiddle-table index idx (1 <= idx < N) in the k-major layout
__host__ __device__ inline int tw_layout_pos(int idx) {
    if (idx <= 0) return 0;
    int l = 0;
    while ((2 << l) <= idx) l++;
    const int m = 1 << l, i = idx - m, r = l % 3, m0 = 1 << (3 * (l / 3));
    if (r == 0) return idx;
    if (r == 1) return m + (i & 1) * m0 + (i >> 1);
    return m + (i & 3) * m0 + (i >> 2);
}

struct NttTables {
    const uint2* tw[CH_COUNT];   // [2][N] per channel
};

// Barrier of the 512 threads that run a transform.  A stand-alone kernel
// synchronises its whole CTA; the fused answer kernel (k_answer.cuh) runs its
// transforms in a 512-thread warp group beside the scan warps and uses a named
// barrier (KsSync there).
struct CtaSync {
    __device__ __forceinline__ static void sync() { __syncthreads(); }
};

enum NttDir : int { NTT_FWD = 0, NTT_INV = 1 };

// Copies the twiddles of (channel, direction) into shared memory.  The caller
// synchronises (the transforms start with __syncthreads).
// The device table of (ch, dir); its layout is the staged one, so a kernel
// may also run its transforms on it directly (reads through L1).
__device__ __forceinline__ const uint2* twiddle_table(const NttTables& tabs, int ch, int dir) {
    // a select chain, not tabs.tw[ch]: a run-time index into a kernel
    // parameter array makes the compiler copy the array to local memory
    const uint2* t = ch == 0 ? tabs.tw[0] : ch == 1 ? tabs.tw[1] : ch == 2 ? tabs.tw[2] : ch == 3 ? tabs.tw[3]
                   : ch == 4 ? tabs.tw[4] : ch == 5 ? tabs.tw[5] : tabs.tw[6];
    return t + (size_t)dir * kN;
}

__device__ __forceinline__ void stage_twiddles(uint2* tws, const NttTables& tabs, int ch, int dir) {
    const uint4* g = reinterpret_cast<const uint4*>(twiddle_table(tabs, ch, dir));
    uint4* s = reinterpret_cast<uint4*>(tws);
#pragma unroll
    for (int k = threadIdx.x; k < kN / 2; k += kNttThreads) s[k] = __ldg(g + k);
}

// offset of element t of a radix-8 unit from pidx(unit base), pass P
template <int P>
__device__ __forceinline__ constexpr int unit_off(int t) {
    return P == 0 ? 576 * t : P == 1 ? 72 * t : P == 2 ? 8 * t + 4 * (t >> 2) : t;
}

template <int P>
__device__ __forceinline__ void unit_load(const uint32_t* s, int b, uint32_t* x) {
    if (P == 3) {
        const uint4 a = *reinterpret_cast<const uint4*>(s + b);
        const uint4 c = *reinterpret_cast<const uint4*>(s + b + 4);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w; x[4] = c.x; x[5] = c.y; x[6] = c.z; x[7] = c.w;
    } else {
#pragma unroll
        for (int t = 0; t < 8; t++) x[t] = s[b + unit_off<P>(t)];
    }
}

template <int P>
__device__ __forceinline__ void unit_store(uint32_t* s, int b, const uint32_t* x) {
    if (P == 3) {
        *reinterpret_cast<uint4*>(s + b) = make_uint4(x[0], x[1], x[2], x[3]);
        *reinterpret_cast<uint4*>(s + b + 4) = make_uint4(x[4], x[5], x[6], x[7]);
    } else {
#pragma unroll
        for (int t = 0; t < 8; t++) s[b + unit_off<P>(t)] = x[t];
    }
}

// x - m if x >= m else x, for x < 2m < 2^32: one subtraction and an unsigned
// minimum (x - m wraps above x when x < m)
__device__ __forceinline__ uint32_t sub_if_ge(uint32_t x, uint32_t m) { return umin(x, x - m); }

__device__ __forceinline__ void fwd_bfly(uint32_t& X, uint32_t& Y, uint2 w, uint32_t q, uint32_t q2) {
    uint32_t x = sub_if_ge(X, q2);
    uint32_t t = shoup_lazy(Y, w.x, w.y, q);
    X = x + t;
    Y = x - t + q2;
}

__device__ __forceinline__ void inv_bfly(uint32_t& X, uint32_t& Y, uint2 w, uint32_t q, uint32_t q2) {
    uint32_t s = sub_if_ge(X + Y, q2);
    uint32_t d = shoup_lazy(X - Y + q2, w.x, w.y, q);
    X = s;
    Y = d;
}

// One forward pass over M polynomials (s + m * stride): thread u's radix-8 unit
// of each, three butterfly layers, no barrier inside (units are disjoint).
// LAZY: the last pass leaves its outputs in [0, 4q) instead of canonical.
template <int P, int M, bool LAZY = false>
__device__ __forceinline__ void fwd_pass(uint32_t* s, int stride, const uint2* tws, uint32_t q, uint32_t q2, int u) {
    constexpr int lq = 9 - 3 * P, q8 = 1 << lq, m0 = 1 << (3 * P);
    const int i0 = u >> lq, j = u & (q8 - 1);
    const int b = pidx(i0 * 8 * q8 + j);
    const uint2 wa = tws[m0 + i0];
    const uint2 wb0 = tws[2 * m0 + i0], wb1 = tws[3 * m0 + i0];
    const uint2 wc0 = tws[4 * m0 + i0], wc1 = tws[5 * m0 + i0], wc2 = tws[6 * m0 + i0], wc3 = tws[7 * m0 + i0];
    uint32_t x[M][8];
#pragma unroll
    for (int m = 0; m < M; m++) unit_load<P>(s + m * stride, b, x[m]);
#pragma unroll
    for (int m = 0; m < M; m++) {
        if (P == 0) {
            // the first layer: inputs are below 2q, so X needs no reduction
            // (X + t < 4q and X - t + 2q is in (0, 4q))
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const uint32_t tw = shoup_lazy(x[m][t + 4], wa.x, wa.y, q);
                x[m][t + 4] = x[m][t] - tw + q2;
                x[m][t] = x[m][t] + tw;
            }
        } else {
#pragma unroll
            for (int t = 0; t < 4; t++) fwd_bfly(x[m][t], x[m][t + 4], wa, q, q2);
        }
        fwd_bfly(x[m][0], x[m][2], wb0, q, q2);
        fwd_bfly(x[m][1], x[m][3], wb0, q, q2);
        fwd_bfly(x[m][4], x[m][6], wb1, q, q2);
        fwd_bfly(x[m][5], x[m][7], wb1, q, q2);
        fwd_bfly(x[m][0], x[m][1], wc0, q, q2);
        fwd_bfly(x[m][2], x[m][3], wc1, q, q2);
        fwd_bfly(x[m][4], x[m][5], wc2, q, q2);
        fwd_bfly(x[m][6], x[m][7], wc3, q, q2);
        if (P == 3 && !LAZY) {
#pragma unroll
            for (int t = 0; t < 8; t++) {
                x[m][t] = sub_if_ge(sub_if_ge(x[m][t], q2), q);
            }
        }
    }
#pragma unroll
    for (int m = 0; m < M; m++) unit_store<P>(s + m * stride, b, x[m]);
}

template <int P, int M>
__device__ __forceinline__ void inv_pass(uint32_t* s, int stride, const uint2* tws, uint32_t q, uint32_t q2,
                                         uint32_t ni, uint32_t nip, int u, int ch) {
    constexpr int lq = 9 - 3 * P, q8 = 1 << lq, m0 = 1 << (3 * P);
    const int i0 = u >> lq, j = u & (q8 - 1);
    const int b = pidx(i0 * 8 * q8 + j);
    const uint2 wa = tws[m0 + i0];
    const uint2 wb0 = tws[2 * m0 + i0], wb1 = tws[3 * m0 + i0];
    const uint2 wc0 = tws[4 * m0 + i0], wc1 = tws[5 * m0 + i0], wc2 = tws[6 * m0 + i0], wc3 = tws[7 * m0 + i0];
    uint32_t x[M][8];
#pragma unroll
    for (int m = 0; m < M; m++) unit_load<P>(s + m * stride, b, x[m]);
#pragma unroll
    for (int m = 0; m < M; m++) {
        inv_bfly(x[m][0], x[m][1], wc0, q, q2);
        inv_bfly(x[m][2], x[m][3], wc1, q, q2);
        inv_bfly(x[m][4], x[m][5], wc2, q, q2);
        inv_bfly(x[m][6], x[m][7], wc3, q, q2);
        inv_bfly(x[m][0], x[m][2], wb0, q, q2);
        inv_bfly(x[m][1], x[m][3], wb0, q, q2);
        inv_bfly(x[m][4], x[m][6], wb1, q, q2);
        inv_bfly(x[m][5], x[m][7], wb1, q, q2);
        if (P == 0) {
            // the last layer with N^-1 folded in (its one twiddle wa times
            // N^-1 is a per-channel constant): X + Y and X - Y each take one
            // product and come out canonical
            const ChanConst& cc = c_dev.ch[ch];
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const uint32_t X = x[m][t], Y = x[m][t + 4];
                x[m][t] = shoup_mul(X + Y, ni, nip, q);
                x[m][t + 4] = shoup_mul(X - Y + q2, cc.ninv_w, cc.ninv_w_p, q);
            }
        } else {
#pragma unroll
            for (int t = 0; t < 4; t++) inv_bfly(x[m][t], x[m][t + 4], wa, q, q2);
        }
    }
#pragma unroll
    for (int m = 0; m < M; m++) unit_store<P>(s + m * stride, b, x[m]);
}

// Forward transforms of M padded polynomials s + m * stride of channel ch in
// lockstep (one barrier per pass for all of them); input in [0, 2q)
// (canonical inputs are fine), output canonical -- or, with LAZY, in [0, 4q)
// for consumers that only multiply-accumulate and reduce exactly (the
// canonical pass costs two minima per coefficient, 6 % of a transform).
// tws holds the forward twiddles of ch.
template <int M, class Sync = CtaSync, bool LAZY = false>
__device__ __forceinline__ void cta_ntt_forward_m(uint32_t* s, int stride, const uint2* tws, int ch) {
    const uint32_t q = c_dev.ch[ch].q, q2 = c_dev.ch[ch].two_q;
    const int u = threadIdx.x;
    Sync::sync();
    fwd_pass<0, M>(s, stride, tws, q, q2, u);
    Sync::sync();
    fwd_pass<1, M>(s, stride, tws, q, q2, u);
    Sync::sync();
    fwd_pass<2, M>(s, stride, tws, q, q2, u);
    Sync::sync();
    fwd_pass<3, M, LAZY>(s, stride, tws, q, q2, u);
    Sync::sync();
}

// x in [0, 4q) to canonical
__device__ __forceinline__ uint32_t canon4q(uint32_t x, uint32_t q) { return sub_if_ge(sub_if_ge(x, 2 * q), q); }

// Inverse transforms (include N^-1); input in [0, 2q) (canonical inputs are
// fine), output canonical.  tws holds the inverse twiddles of ch.
template <int M, class Sync = CtaSync>
__device__ __forceinline__ void cta_ntt_inverse_m(uint32_t* s, int stride, const uint2* tws, int ch) {
    const uint32_t q = c_dev.ch[ch].q, q2 = c_dev.ch[ch].two_q;
    const uint32_t ni = c_dev.ch[ch].ninv, nip = c_dev.ch[ch].ninv_p;
    const int u = threadIdx.x;
    Sync::sync();
    inv_pass<3, M>(s, stride, tws, q, q2, ni, nip, u, ch);
    Sync::sync();
    inv_pass<2, M>(s, stride, tws, q, q2, ni, nip, u, ch);
    Sync::sync();
    inv_pass<1, M>(s, stride, tws, q, q2, ni, nip, u, ch);
    Sync::sync();
    inv_pass<0, M>(s, stride, tws, q, q2, ni, nip, u, ch);
    Sync::sync();
}

template <class Sync = CtaSync, bool LAZY = false>
__device__ __forceinline__ void cta_ntt_forward(uint32_t* s, const uint2* tws, int ch) {
    cta_ntt_forward_m<1, Sync, LAZY>(s, kPadN, tws, ch);
}
template <class Sync = CtaSync>
__device__ __forceinline__ void cta_ntt_inverse(uint32_t* s, const uint2* tws, int ch) {
    cta_ntt_inverse_m<1, Sync>(s, kPadN, tws, ch);
}

// Copies of whole polynomials between global memory (natural order) and a
// padded shared-memory polynomial; 16-byte vectors.  The loads bypass L1
// (ld.global.cg): the source is usually the previous kernel's output, and a
// kernel started early by programmatic dependent launch must not hit lines
// an overlapping kernel left in L1.
__device__ __forceinline__ void poly_to_smem(uint32_t* s, const uint32_t* __restrict__ g) {
    const uint4* g4 = reinterpret_cast<const uint4*>(g);
#pragma unroll
    for (int k = threadIdx.x; k < kN / 4; k += kNttThreads) *reinterpret_cast<uint4*>(s + pidx(4 * k)) = __ldcg(g4 + k);
}
__device__ __forceinline__ void poly_from_smem(uint32_t* __restrict__ g, const uint32_t* s) {
    uint4* g4 = reinterpret_cast<uint4*>(g);
#pragma unroll
    for (int k = threadIdx.x; k < kN / 4; k += kNttThreads) g4[k] = *reinterpret_cast<const uint4*>(s + pidx(4 * k));
}

}  // namespace kspir
