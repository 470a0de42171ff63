// The first-dimension database scan (reference fastMultiplyQueryByDatabaseDim1InvCRT,
// crt.cpp:643-856), as a persistent HBM-streaming kernel.
//
// Database word DB[r][z][i][k] = (v mod q1) | (v mod q2) << 32 (database_tocrt,
// crt.cpp:859-885); cipherbuf[z][k] = (a_k, b_k) packed the same way
// (reorientCipher).  For every sub-database r, NTT slot z and giant row i:
//   a_lo = sum_k lo(DB) * lo(a_k)      a_hi = sum_k hi(DB) * hi(a_k)
//   b_lo = sum_k lo(DB) * lo(b_k)      b_hi = sum_k hi(DB) * hi(b_k)
// exact 64-bit sums (products < 2^56, N1 <= 128 terms -> < 2^63), and the
// reference composes out = crt_compose(a_lo, a_hi), which is the canonical
// crtMod value with residues (a_lo mod q1, a_hi mod q2).  The kernel stores
// those residues directly: sout[r][i][comp][ch][z].
//
// Data movement: one 16 KiB slab DB[r][z] (N2 x N1 words) plus the 16*N1-byte
// cipherbuf row z per work item, brought in by 1-D bulk copies (TMA engine)
// into an NST-deep shared-memory ring; a producer warp issues, 8 consumer warps
// (4 groups of 64 threads, one item per group) multiply-accumulate with
// IMAD.WIDE and reduce across the TPR = N1/32 threads that share a row.
#pragma once

#include "common.cuh"
#include "ptx.cuh"

namespace kspir {

constexpr int kScanThreads = 288;            // 8 consumer warps + 1 producer warp
constexpr int kScanStages = 8;
constexpr int kScanGroups = 4;
constexpr uint64_t kWaitLimitNs = 2000000000ull;   // 2 s per bounded wait

template <int N1>
struct ScanCfg {
    static constexpr int N2 = kN / 2 / N1;
    static constexpr int TPR = N1 / 32;                 // threads per row
    static constexpr int SLAB = kN / 2 * 8;             // DB bytes per item
    static constexpr int QSLAB = 2 * N1 * 8;            // cipherbuf bytes per item
    static constexpr int STAGE = SLAB + QSLAB;
    static constexpr int SMEM = kScanStages * STAGE + 2 * kScanStages * 8;
};

template <int N1>
__global__ void __launch_bounds__(kScanThreads, 1)
    k_scan(const uint64_t* __restrict__ db, const uint64_t* __restrict__ cbuf, uint32_t* __restrict__ sout,
           int R, int* __restrict__ err) {
    using C = ScanCfg<N1>;
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + kScanStages * C::STAGE);
    uint64_t* empty = full + kScanStages;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int s = 0; s < kScanStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 2);   // the two consumer warps of the owning group
        }
        fence_mbar_init();
    }
    __syncthreads();

    const long total = (long)R * kN;
    const long nloc = blockIdx.x < total ? (total - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    if (warp == 8) {
        // producer
        if (lane == 0) {
            long issued = 0;
            for (long j = 0; j < nloc; j++) {
                const int s = (int)(j % kScanStages);
                if (j >= kScanStages) {
                    const uint32_t par = (uint32_t)((j / kScanStages - 1) & 1);
                    if (!mbar_wait_bounded(&empty[s], par, kWaitLimitNs)) {
                        atomicOr(err, 1);
                        break;
                    }
                }
                const long it = blockIdx.x + j * gridDim.x;
                const long r = it / kN, z = it % kN;
                uint8_t* st = smem + (size_t)s * C::STAGE;
                mbar_arrive_expect_tx(&full[s], C::STAGE);
                bulk_g2s(st, db + ((size_t)r * kN + z) * (kN / 2), C::SLAB, &full[s]);
                bulk_g2s(st + C::SLAB, cbuf + (size_t)z * 2 * N1, C::QSLAB, &full[s]);
                issued = j + 1;
            }
            // never leave the CTA with copies in flight into its shared memory
            const long first = issued > kScanStages ? issued - kScanStages : 0;
            for (long j = first; j < issued; j++)
                if (!mbar_wait_bounded(&full[j % kScanStages], (uint32_t)((j / kScanStages) & 1), kWaitLimitNs))
                    atomicOr(err, 4);
        }
        return;
    }

    // consumers
    const int g = warp >> 1;              // slab group
    const int t = tid & 63;               // thread within group
    const int i = t / C::TPR;             // giant row
    const int qd = t % C::TPR;            // quarter within row
    for (long j = g; j < nloc; j += kScanGroups) {
        const int s = (int)(j % kScanStages);
        if (!mbar_wait_bounded(&full[s], (uint32_t)((j / kScanStages) & 1), kWaitLimitNs)) {
            atomicOr(err, 2);
            break;
        }
        const uint8_t* st = smem + (size_t)s * C::STAGE;
        const uint64_t* D = reinterpret_cast<const uint64_t*>(st) + (size_t)i * N1;
        const uint64_t* Qs = reinterpret_cast<const uint64_t*>(st + C::SLAB);
        uint64_t alo = 0, ahi = 0, blo = 0, bhi = 0;
#pragma unroll
        for (int m = 0; m < 16; m++) {
            // 16-byte chunk of the row, rotated by the row index so that the
            // lanes of different rows hit different banks
            const int kc = qd + C::TPR * ((m + i) & 15);
            const uint4 w = *reinterpret_cast<const uint4*>(D + 2 * kc);
            const uint4 qa = *reinterpret_cast<const uint4*>(Qs + 4 * kc);
            const uint4 qb = *reinterpret_cast<const uint4*>(Qs + 4 * kc + 2);
            alo += (uint64_t)w.x * qa.x;
            alo += (uint64_t)w.z * qb.x;
            ahi += (uint64_t)w.y * qa.y;
            ahi += (uint64_t)w.w * qb.y;
            blo += (uint64_t)w.x * qa.z;
            blo += (uint64_t)w.z * qb.z;
            bhi += (uint64_t)w.y * qa.w;
            bhi += (uint64_t)w.w * qb.w;
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
#pragma unroll
        for (int off = 1; off < C::TPR; off <<= 1) {
            alo += __shfl_xor_sync(0xffffffffu, alo, off);
            ahi += __shfl_xor_sync(0xffffffffu, ahi, off);
            blo += __shfl_xor_sync(0xffffffffu, blo, off);
            bhi += __shfl_xor_sync(0xffffffffu, bhi, off);
        }
        const long it = blockIdx.x + j * gridDim.x;
        const long r = it / kN, z = it % kN;
        uint32_t* o = sout + ((size_t)(r * C::N2 + i) * 4) * kN + z;
        for (int oi = qd; oi < 4; oi += C::TPR) {
            uint32_t v;
            if (oi == 0) v = mod_q1(alo);
            else if (oi == 1) v = mod_q2(ahi);
            else if (oi == 2) v = mod_q1(blo);
            else v = mod_q2(bhi);
            o[(size_t)oi * kN] = v;   // [comp][ch]: 0 = a q1, 1 = a q2, 2 = b q1, 3 = b q2
        }
    }
}

}  // namespace kspir
