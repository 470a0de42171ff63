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
// Device table layout per channel: uint2 tw[2][N]; tw[0][k] = psi^brv(k),
// tw[1][k] = psi^-brv(k), each with its Shoup companion.
#pragma once

#include "common.cuh"

namespace kspir {

constexpr int kNttThreads = 512;

struct NttTables {
    const uint2* tw[CH_COUNT];   // [2][N] per channel
};

enum NttDir : int { NTT_FWD = 0, NTT_INV = 1 };

// Copies the twiddles of (channel, direction) into shared memory.  The caller
// synchronises (the transforms start with __syncthreads).
__device__ __forceinline__ void stage_twiddles(uint2* tws, const NttTables& tabs, int ch, int dir) {
    const uint4* g = reinterpret_cast<const uint4*>(tabs.tw[ch] + (size_t)dir * kN);
    uint4* s = reinterpret_cast<uint4*>(tws);
#pragma unroll
    for (int k = threadIdx.x; k < kN / 2; k += kNttThreads) s[k] = __ldg(g + k);
}

// the 8 elements of a radix-8 unit; contiguous (one 32-byte run) when q8 == 1
__device__ __forceinline__ void load8(const uint32_t* s, int base, int q8, uint32_t* x) {
    if (q8 == 1) {
        const uint4 a = *reinterpret_cast<const uint4*>(s + base);
        const uint4 b = *reinterpret_cast<const uint4*>(s + base + 4);
        x[0] = a.x; x[1] = a.y; x[2] = a.z; x[3] = a.w; x[4] = b.x; x[5] = b.y; x[6] = b.z; x[7] = b.w;
    } else {
#pragma unroll
        for (int t = 0; t < 8; t++) x[t] = s[base + t * q8];
    }
}

__device__ __forceinline__ void store8(uint32_t* s, int base, int q8, const uint32_t* x) {
    if (q8 == 1) {
        *reinterpret_cast<uint4*>(s + base) = make_uint4(x[0], x[1], x[2], x[3]);
        *reinterpret_cast<uint4*>(s + base + 4) = make_uint4(x[4], x[5], x[6], x[7]);
    } else {
#pragma unroll
        for (int t = 0; t < 8; t++) s[base + t * q8] = x[t];
    }
}

__device__ __forceinline__ void fwd_bfly(uint32_t& X, uint32_t& Y, uint2 w, uint32_t q, uint32_t q2) {
    uint32_t x = X >= q2 ? X - q2 : X;
    uint32_t t = shoup_lazy(Y, w.x, w.y, q);
    X = x + t;
    Y = x - t + q2;
}

__device__ __forceinline__ void inv_bfly(uint32_t& X, uint32_t& Y, uint2 w, uint32_t q, uint32_t q2) {
    uint32_t s = X + Y;
    s = s >= q2 ? s - q2 : s;
    uint32_t d = shoup_lazy(X - Y + q2, w.x, w.y, q);
    X = s;
    Y = d;
}

// Forward transform of s[0..N) in place; input in [0, 4q) (canonical inputs are
// fine), output canonical.  tws holds the forward twiddles of `ch`.
__device__ __forceinline__ void cta_ntt_forward(uint32_t* s, const uint2* tws, int ch) {
    const uint32_t q = c_dev.ch[ch].q, q2 = c_dev.ch[ch].two_q;
    const int u = threadIdx.x;
    __syncthreads();
#pragma unroll
    for (int p = 0; p < 4; p++) {
        const int lq = 9 - 3 * p;             // log2 of the element stride within a unit
        const int q8 = 1 << lq;
        const int m0 = 1 << (3 * p);
        const int i0 = u >> lq, j = u & (q8 - 1);
        const int base = i0 * 8 * q8 + j;
        uint32_t x[8];
        load8(s, base, q8, x);
        const uint2 wa = tws[m0 + i0];
        const uint2 wb0 = tws[2 * m0 + 2 * i0], wb1 = tws[2 * m0 + 2 * i0 + 1];
        const uint2 wc0 = tws[4 * m0 + 4 * i0], wc1 = tws[4 * m0 + 4 * i0 + 1];
        const uint2 wc2 = tws[4 * m0 + 4 * i0 + 2], wc3 = tws[4 * m0 + 4 * i0 + 3];
#pragma unroll
        for (int t = 0; t < 4; t++) fwd_bfly(x[t], x[t + 4], wa, q, q2);
        fwd_bfly(x[0], x[2], wb0, q, q2);
        fwd_bfly(x[1], x[3], wb0, q, q2);
        fwd_bfly(x[4], x[6], wb1, q, q2);
        fwd_bfly(x[5], x[7], wb1, q, q2);
        fwd_bfly(x[0], x[1], wc0, q, q2);
        fwd_bfly(x[2], x[3], wc1, q, q2);
        fwd_bfly(x[4], x[5], wc2, q, q2);
        fwd_bfly(x[6], x[7], wc3, q, q2);
        if (p == 3) {
#pragma unroll
            for (int t = 0; t < 8; t++) {
                uint32_t v = x[t] >= q2 ? x[t] - q2 : x[t];
                x[t] = v >= q ? v - q : v;
            }
        }
        // the units of one pass are disjoint: write back without a barrier
        store8(s, base, q8, x);
        __syncthreads();
    }
}

// Inverse transform of s[0..N) in place (includes N^-1); input in [0, 2q)
// (canonical inputs are fine), output canonical.  tws holds the inverse
// twiddles of `ch`.
__device__ __forceinline__ void cta_ntt_inverse(uint32_t* s, const uint2* tws, int ch) {
    const uint32_t q = c_dev.ch[ch].q, q2 = c_dev.ch[ch].two_q;
    const uint32_t ni = c_dev.ch[ch].ninv, nip = c_dev.ch[ch].ninv_p;
    const int u = threadIdx.x;
    __syncthreads();
#pragma unroll
    for (int p = 3; p >= 0; p--) {
        const int lq = 9 - 3 * p;
        const int q8 = 1 << lq;
        const int m0 = 1 << (3 * p);
        const int i0 = u >> lq, j = u & (q8 - 1);
        const int base = i0 * 8 * q8 + j;
        uint32_t x[8];
        load8(s, base, q8, x);
        const uint2 wa = tws[m0 + i0];
        const uint2 wb0 = tws[2 * m0 + 2 * i0], wb1 = tws[2 * m0 + 2 * i0 + 1];
        const uint2 wc0 = tws[4 * m0 + 4 * i0], wc1 = tws[4 * m0 + 4 * i0 + 1];
        const uint2 wc2 = tws[4 * m0 + 4 * i0 + 2], wc3 = tws[4 * m0 + 4 * i0 + 3];
        inv_bfly(x[0], x[1], wc0, q, q2);
        inv_bfly(x[2], x[3], wc1, q, q2);
        inv_bfly(x[4], x[5], wc2, q, q2);
        inv_bfly(x[6], x[7], wc3, q, q2);
        inv_bfly(x[0], x[2], wb0, q, q2);
        inv_bfly(x[1], x[3], wb0, q, q2);
        inv_bfly(x[4], x[6], wb1, q, q2);
        inv_bfly(x[5], x[7], wb1, q, q2);
#pragma unroll
        for (int t = 0; t < 4; t++) inv_bfly(x[t], x[t + 4], wa, q, q2);
        if (p == 0) {
#pragma unroll
            for (int t = 0; t < 8; t++) x[t] = shoup_mul(x[t], ni, nip, q);
        }
        store8(s, base, q8, x);
        __syncthreads();
    }
}

// M polynomials of the same channel, s + m * stride (m < M), transformed in
// lockstep: one barrier per pass for all of them and M independent radix-8
// units per thread, which hides the butterfly and shared-memory latencies a
// single transform exposes.
template <int M>
__device__ __forceinline__ void cta_ntt_forward_m(uint32_t* s, int stride, const uint2* tws, int ch) {
    const uint32_t q = c_dev.ch[ch].q, q2 = c_dev.ch[ch].two_q;
    const int u = threadIdx.x;
    __syncthreads();
#pragma unroll
    for (int p = 0; p < 4; p++) {
        const int lq = 9 - 3 * p;
        const int q8 = 1 << lq;
        const int m0 = 1 << (3 * p);
        const int i0 = u >> lq, j = u & (q8 - 1);
        const int base = i0 * 8 * q8 + j;
        const uint2 wa = tws[m0 + i0];
        const uint2 wb0 = tws[2 * m0 + 2 * i0], wb1 = tws[2 * m0 + 2 * i0 + 1];
        const uint2 wc0 = tws[4 * m0 + 4 * i0], wc1 = tws[4 * m0 + 4 * i0 + 1];
        const uint2 wc2 = tws[4 * m0 + 4 * i0 + 2], wc3 = tws[4 * m0 + 4 * i0 + 3];
        uint32_t x[M][8];
#pragma unroll
        for (int m = 0; m < M; m++) load8(s + m * stride, base, q8, x[m]);
#pragma unroll
        for (int m = 0; m < M; m++) {
#pragma unroll
            for (int t = 0; t < 4; t++) fwd_bfly(x[m][t], x[m][t + 4], wa, q, q2);
            fwd_bfly(x[m][0], x[m][2], wb0, q, q2);
            fwd_bfly(x[m][1], x[m][3], wb0, q, q2);
            fwd_bfly(x[m][4], x[m][6], wb1, q, q2);
            fwd_bfly(x[m][5], x[m][7], wb1, q, q2);
            fwd_bfly(x[m][0], x[m][1], wc0, q, q2);
            fwd_bfly(x[m][2], x[m][3], wc1, q, q2);
            fwd_bfly(x[m][4], x[m][5], wc2, q, q2);
            fwd_bfly(x[m][6], x[m][7], wc3, q, q2);
            if (p == 3) {
#pragma unroll
                for (int t = 0; t < 8; t++) {
                    uint32_t v = x[m][t] >= q2 ? x[m][t] - q2 : x[m][t];
                    x[m][t] = v >= q ? v - q : v;
                }
            }
        }
#pragma unroll
        for (int m = 0; m < M; m++) store8(s + m * stride, base, q8, x[m]);
        __syncthreads();
    }
}

template <int M>
__device__ __forceinline__ void cta_ntt_inverse_m(uint32_t* s, int stride, const uint2* tws, int ch) {
    const uint32_t q = c_dev.ch[ch].q, q2 = c_dev.ch[ch].two_q;
    const uint32_t ni = c_dev.ch[ch].ninv, nip = c_dev.ch[ch].ninv_p;
    const int u = threadIdx.x;
    __syncthreads();
#pragma unroll
    for (int p = 3; p >= 0; p--) {
        const int lq = 9 - 3 * p;
        const int q8 = 1 << lq;
        const int m0 = 1 << (3 * p);
        const int i0 = u >> lq, j = u & (q8 - 1);
        const int base = i0 * 8 * q8 + j;
        const uint2 wa = tws[m0 + i0];
        const uint2 wb0 = tws[2 * m0 + 2 * i0], wb1 = tws[2 * m0 + 2 * i0 + 1];
        const uint2 wc0 = tws[4 * m0 + 4 * i0], wc1 = tws[4 * m0 + 4 * i0 + 1];
        const uint2 wc2 = tws[4 * m0 + 4 * i0 + 2], wc3 = tws[4 * m0 + 4 * i0 + 3];
        uint32_t x[M][8];
#pragma unroll
        for (int m = 0; m < M; m++) load8(s + m * stride, base, q8, x[m]);
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
#pragma unroll
            for (int t = 0; t < 4; t++) inv_bfly(x[m][t], x[m][t + 4], wa, q, q2);
            if (p == 0) {
#pragma unroll
                for (int t = 0; t < 8; t++) x[m][t] = shoup_mul(x[m][t], ni, nip, q);
            }
        }
#pragma unroll
        for (int m = 0; m < M; m++) store8(s + m * stride, base, q8, x[m]);
        __syncthreads();
    }
}

}  // namespace kspir
