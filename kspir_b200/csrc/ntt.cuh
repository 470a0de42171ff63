// CTA-level negacyclic NTT of length 4096 on one residue channel, operating on
// a shared-memory array.  Every kernel that needs a transform calls these so
// the transform is fused with its producer and consumer.
//
// Order and root follow HEXL as the reference uses it: the forward transform
// maps natural order to bit-reversed order, slot j holding
// sum_k x_k psi^((2 bitrev(j) + 1) k)  (reference utils.cpp:1473-1478), and the
// inverse includes N^-1.  Outputs are canonical.
//
// Radix-4 passes (two butterfly layers per __syncthreads) of Harvey lazy
// butterflies with Shoup twiddles.  Twiddle tables (per channel, in global
// memory, read through the read-only path):
//   tw[0*N + k] = psi^brv(k)      tw[1*N + k] = Shoup companion
//   tw[2*N + k] = psi^-brv(k)     tw[3*N + k] = Shoup companion
#pragma once

#include "common.cuh"

namespace kspir {

struct NttTables {
    const uint32_t* tw[CH_COUNT];   // 4*N words per channel
};

// Forward transform of s[0..N) in place.  Input in [0, 4q) (canonical inputs
// are fine), output canonical.  T = blockDim.x (a multiple of 32, <= 1024).
template <int T>
__device__ __forceinline__ void cta_ntt_forward(uint32_t* s, const uint32_t* __restrict__ tw, int ch) {
    const uint32_t q = c_dev.ch[ch].q, q2 = c_dev.ch[ch].two_q;
    const uint32_t* __restrict__ w = tw;
    const uint32_t* __restrict__ wp = tw + kN;
    __syncthreads();
#pragma unroll 1
    for (int m = 1; m < kN; m <<= 2) {
        const int h = kN / (2 * m);         // half-size of layer m
        const int hh = h >> 1;               // half-size of layer 2m
        const int lg_hh = __ffs(hh) - 1;
#pragma unroll
        for (int u = threadIdx.x; u < kN / 4; u += T) {
            const int i = u >> lg_hh, j = u & (hh - 1);
            const int e0 = 2 * i * h + j;
            const uint32_t W1 = __ldg(w + m + i), W1p = __ldg(wp + m + i);
            const uint32_t W2 = __ldg(w + 2 * m + 2 * i), W2p = __ldg(wp + 2 * m + 2 * i);
            const uint32_t W3 = __ldg(w + 2 * m + 2 * i + 1), W3p = __ldg(wp + 2 * m + 2 * i + 1);
            uint32_t x0 = s[e0], x1 = s[e0 + hh], x2 = s[e0 + h], x3 = s[e0 + h + hh];
            // layer m: (x0, x2), (x1, x3) with W1
            if (x0 >= q2) x0 -= q2;
            if (x1 >= q2) x1 -= q2;
            uint32_t t2 = shoup_lazy(x2, W1, W1p, q);
            uint32_t t3 = shoup_lazy(x3, W1, W1p, q);
            uint32_t y0 = x0 + t2, y2 = x0 - t2 + q2;
            uint32_t y1 = x1 + t3, y3 = x1 - t3 + q2;
            // layer 2m: (y0, y1) with W2, (y2, y3) with W3
            if (y0 >= q2) y0 -= q2;
            if (y2 >= q2) y2 -= q2;
            uint32_t t1 = shoup_lazy(y1, W2, W2p, q);
            uint32_t t3b = shoup_lazy(y3, W3, W3p, q);
            s[e0] = y0 + t1;
            s[e0 + hh] = y0 - t1 + q2;
            s[e0 + h] = y2 + t3b;
            s[e0 + h + hh] = y2 - t3b + q2;
        }
        __syncthreads();
    }
#pragma unroll
    for (int k = threadIdx.x; k < kN; k += T) {
        uint32_t x = s[k];
        if (x >= q2) x -= q2;
        if (x >= q) x -= q;
        s[k] = x;
    }
    __syncthreads();
}

// Inverse transform of s[0..N) in place (includes N^-1).  Input in [0, 2q)
// (canonical inputs are fine), output canonical.
template <int T>
__device__ __forceinline__ void cta_ntt_inverse(uint32_t* s, const uint32_t* __restrict__ tw, int ch) {
    const uint32_t q = c_dev.ch[ch].q, q2 = c_dev.ch[ch].two_q;
    const uint32_t* __restrict__ w = tw + 2 * kN;
    const uint32_t* __restrict__ wp = tw + 3 * kN;
    __syncthreads();
#pragma unroll 1
    for (int m = kN / 2; m >= 2; m >>= 2) {
        const int h = kN / (2 * m);          // half-size of layer m; layer m/2 has 2h
        const int lg_h = __ffs(h) - 1;
#pragma unroll
        for (int u = threadIdx.x; u < kN / 4; u += T) {
            const int i = u >> lg_h, j = u & (h - 1);
            const int e0 = 4 * i * h + j;
            const uint32_t Wa = __ldg(w + m + 2 * i), Wap = __ldg(wp + m + 2 * i);
            const uint32_t Wb = __ldg(w + m + 2 * i + 1), Wbp = __ldg(wp + m + 2 * i + 1);
            const uint32_t Wc = __ldg(w + m / 2 + i), Wcp = __ldg(wp + m / 2 + i);
            uint32_t x0 = s[e0], x1 = s[e0 + h], x2 = s[e0 + 2 * h], x3 = s[e0 + 3 * h];
            // layer m: (x0, x1) with Wa, (x2, x3) with Wb
            uint32_t y0 = x0 + x1; if (y0 >= q2) y0 -= q2;
            uint32_t y1 = shoup_lazy(x0 - x1 + q2, Wa, Wap, q);
            uint32_t y2 = x2 + x3; if (y2 >= q2) y2 -= q2;
            uint32_t y3 = shoup_lazy(x2 - x3 + q2, Wb, Wbp, q);
            // layer m/2: (y0, y2), (y1, y3) with Wc
            uint32_t z0 = y0 + y2; if (z0 >= q2) z0 -= q2;
            uint32_t z2 = shoup_lazy(y0 - y2 + q2, Wc, Wcp, q);
            uint32_t z1 = y1 + y3; if (z1 >= q2) z1 -= q2;
            uint32_t z3 = shoup_lazy(y1 - y3 + q2, Wc, Wcp, q);
            s[e0] = z0; s[e0 + h] = z1; s[e0 + 2 * h] = z2; s[e0 + 3 * h] = z3;
        }
        __syncthreads();
    }
    const uint32_t ni = c_dev.ch[ch].ninv, nip = c_dev.ch[ch].ninv_p;
#pragma unroll
    for (int k = threadIdx.x; k < kN; k += T) s[k] = shoup_mul(s[k], ni, nip, q);
    __syncthreads();
}

}  // namespace kspir
