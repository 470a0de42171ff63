// The first-dimension database scan (reference fastMultiplyQueryByDatabaseDim1InvCRT,
// crt.cpp:643-856), as a persistent HBM-streaming kernel.
//
// Database word DB[r][z][i][k] = (v mod q1) | (v mod q2) << 32 (database_tocrt,
// crt.cpp:859-885); cipherbuf[z][k] = (a_k, b_k) packed the same way
// (reorientCipher).  For every sub-database r, NTT slot z and giant row i:
//   a_lo = sum_k lo(DB) * lo(a_k)      a_hi = sum_k hi(DB) * hi(a_k)
//   b_lo = sum_k lo(DB) * lo(b_k)      b_hi = sum_k hi(DB) * hi(b_k)
// exact 64-bit sums (products < 2^56, N1 <= 512 terms; any wrap mod 2^64 is
// the reference's too), and the reference composes out = crt_compose(a_lo,
// a_hi), which is the canonical crtMod value with residues (a_lo mod q1,
// a_hi mod q2).  The kernel stores those residues in the blocked layout of
// sout_idx (row r * N2 + i, cv = comp * 2 + ch).
//
// Data movement: one 16 KiB slab DB[r][z] (N2 x N1 words) plus the 16*N1-byte
// cipherbuf row z per work item, brought in by 1-D bulk copies (TMA engine,
// no multicast) into an NST-deep shared-memory ring (12 stages at N1 = 128);
// one producer warp issues, CONS consumer warps each take one item at a time.
//
// Consumer mapping (one warp per slab): lane = 8 * r + c covers rows
// {r, r+4, ...} and 16-byte chunks {c, c+8, ...}.  Eight lanes of a row read
// 128 contiguous bytes of it (no bank conflicts), the four lanes that share a
// chunk read the same cipherbuf bytes (broadcast), and each cipherbuf chunk is
// loaded once per lane and reused across its rows.  The 4*RPL partial sums of
// a lane are reduced across the eight lanes of its row by a transpose-reduce
// (each shuffle level hands over half of the values), which leaves every lane
// holding 4*RPL/8 finished outputs.
#pragma once

#include "common.cuh"
#include "ptx.cuh"

namespace kspir {

constexpr uint64_t kWaitLimitNs = 2000000000ull;     // 2 s per bounded wait

// Stage ownership: consumer warp w takes items w, w + CONS, ... and stage
// j % NST with NST a multiple of CONS, so every stage belongs to one warp and
// that warp never waits more than one phase ahead of the barrier (an mbarrier
// parity wait cannot tell phase u-1 from u+1).

// Ring shapes of the single-query scan, measured on B200 with a 1 GiB
// database (consumer warps x stages of 18 KiB, 148 CTAs): 4 x 8 0.156 ms
// (6.9 TB/s), 6 x 6 0.176 ms, 6 x 12 0.176 ms, 4 x 4 0.214 ms.  The default
// (streaming) shape is 4 x 8: 148 KiB of shared memory, which leaves room on
// the SM for a baby-step or transform CTA of a concurrent answer.  The sharing
// shape (ScanShare) is 6 x 6: 110 KiB, slower alone but leaving room for a
// giant-step or external-product CTA (107 KiB) beside it, which pays when
// several answers are in flight.
template <int N1, int CONS_ = 4, int NST_ = 8>
struct ScanCfg {
    static constexpr int N2 = kN / 2 / N1;
    static constexpr int CHUNKS = N1 / 2;               // 16-byte chunks per row
    static constexpr int RPL = N2 / 4;                  // rows per lane
    static constexpr int CPL = CHUNKS / 8;              // chunks per lane
    static constexpr int SLAB = kN / 2 * 8;             // DB bytes per item
    static constexpr int QSLAB = 2 * N1 * 8;            // cipherbuf bytes per item
    static constexpr int STAGE = SLAB + QSLAB;
    static constexpr int CONS = CONS_;                  // consumer warps
    static constexpr int NST = NST_;                    // ring stages, a multiple of CONS
    static constexpr int THREADS = 32 * (CONS + 1);
    static constexpr int SMEM = NST * STAGE + 2 * NST * 8;
    static_assert(NST % CONS == 0, "stages must be owned by one consumer warp each");
    static_assert(SMEM <= 227 * 1024, "shared memory budget");
    static constexpr int NV = 4 * RPL;                  // partial sums per lane
    static constexpr int NOUT = NV / 8;                 // finished outputs per lane
    static_assert(RPL >= 2 && CPL >= 1, "N1 must be in [64, 256]");
};

template <int N1>
struct ScanShare {   // 6 x 6 where a 107 KiB CTA still fits beside it (N1 <= 128)
    static constexpr int CONS = N1 <= 128 ? 6 : 4;
    static constexpr int NST = N1 <= 128 ? 6 : 8;
    using Cfg = ScanCfg<N1, CONS, NST>;
};

// The multiply-accumulate of one work item by one warp: the slab DB[r][z]
// and cipherbuf row z in shared memory at `st` -> the lane's 4 * RPL partial
// sums v[o], o = 4 * rr + comp_ch (0 = a q1 (lo), 1 = a q2 (hi), 2 = b q1,
// 3 = b q2) of rows lr + 4 rr.
template <int N1>
__device__ __forceinline__ void scan_item_mac(const uint8_t* st, int lane, uint64_t* v) {
    using C = ScanCfg<N1>;
    const int lr = lane >> 3;    // row lane 0..3
    const int lc = lane & 7;     // chunk lane 0..7
    const uint4* D4 = reinterpret_cast<const uint4*>(st);             // [N2][CHUNKS] chunks of 2 words
    const uint4* Q4 = reinterpret_cast<const uint4*>(st + C::SLAB);   // [N1] (a_k, b_k) pairs
#pragma unroll
    for (int o = 0; o < C::NV; o++) v[o] = 0;
#pragma unroll
    for (int cc = 0; cc < C::CPL; cc++) {
        const int kc = lc + 8 * cc;                   // chunk = words 2kc, 2kc+1
        const uint4 qa = Q4[2 * kc];                  // (a_2kc, b_2kc)
        const uint4 qb = Q4[2 * kc + 1];              // (a_2kc+1, b_2kc+1)
#pragma unroll
        for (int rr = 0; rr < C::RPL; rr++) {
            const uint4 w = D4[(lr + 4 * rr) * C::CHUNKS + kc];
            mad_wide(v[4 * rr + 0], w.x, qa.x);
            mad_wide(v[4 * rr + 0], w.z, qb.x);
            mad_wide(v[4 * rr + 1], w.y, qa.y);
            mad_wide(v[4 * rr + 1], w.w, qb.y);
            mad_wide(v[4 * rr + 2], w.x, qa.z);
            mad_wide(v[4 * rr + 2], w.z, qb.z);
            mad_wide(v[4 * rr + 3], w.y, qa.w);
            mad_wide(v[4 * rr + 3], w.w, qb.w);
        }
    }
}

// Transpose-reduce over the chunk lanes (offsets 4, 2, 1: at each level the
// lane keeps the half of its values selected by its lane bit and adds the
// partner's copy of that half), then the residues of the lane's finished
// outputs into the scan output of sub-database r, slot z.
template <int N1>
__device__ __forceinline__ void scan_item_store(uint64_t* v, int lane, int r, int z, int R, uint32_t* sout) {
    using C = ScanCfg<N1>;
    const int lr = lane >> 3, lc = lane & 7;
#pragma unroll
    for (int lvl = 0; lvl < 3; lvl++) {
        const int d = 4 >> lvl;
        const int hs = C::NV >> (lvl + 1);
        const bool upper = (lc & d) != 0;
#pragma unroll
        for (int i = 0; i < hs; i++) {
            const uint64_t send = upper ? v[i] : v[i + hs];
            const uint64_t keep = upper ? v[i + hs] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, d);
        }
    }
    // lane lc now holds outputs o = NOUT * lc + t
#pragma unroll
    for (int t = 0; t < C::NOUT; t++) {
        const int o = C::NOUT * lc + t;
        const int i = lr + 4 * (o >> 2), cv = o & 3;
        const uint32_t res = (cv & 1) ? mod_q2(v[t]) : mod_q1(v[t]);
        sout[sout_idx(r * C::N2 + i, cv, z, R * C::N2)] = res;
    }
}

// Failure injection for the tests of the bounded waits (kspir_debug_scan_fault):
// `limit_ns` replaces the 2 s limit of every wait, and CTA 0's producer
// issues no copy for its local item `skip` (-1: none), so the consumer of that
// stage waits for bytes that never come, gives up after limit_ns, records the
// error and stops; the producer then gives up waiting for the stage to be
// released, and drains the copies it did issue before the CTA exits.
template <int N1, int CONS = 4, int NST = 8>
__global__ void __launch_bounds__(ScanCfg<N1, CONS, NST>::THREADS, 1)
    k_scan(const uint64_t* __restrict__ db, const uint64_t* __restrict__ cbuf, uint32_t* __restrict__ sout,
           int R, int* __restrict__ err, uint64_t limit_ns, long skip) {
    using C = ScanCfg<N1, CONS, NST>;
    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + C::NST * C::STAGE);
    uint64_t* empty = full + C::NST;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (tid == 0) {
        for (int s = 0; s < C::NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);   // the consuming warp
        }
        fence_mbar_init();
    }
    __syncthreads();

    const long total = (long)R * kN;
    const long nloc = blockIdx.x < total ? (total - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;

    if (warp == C::CONS) {
        // producer
        if (lane == 0) {
            const uint64_t pol_db = l2_policy_evict_first(), pol_cb = l2_policy_evict_last();
            const long skip_j = blockIdx.x == 0 ? skip : -1;
            long issued = 0;
            for (long j = 0; j < nloc; j++) {
                const int s = (int)(j % C::NST);
                if (j >= C::NST) {
                    const uint32_t par = (uint32_t)((j / C::NST - 1) & 1);
                    if (!mbar_wait_bounded(&empty[s], par, limit_ns)) {
                        atomicOr(err, 1);
                        break;
                    }
                }
                issued = j + 1;
                if (j == skip_j) continue;   // injected failure: nothing arrives on full[s]
                const long it = blockIdx.x + j * gridDim.x;
                const long r = it / kN, z = it % kN;
                uint8_t* st = smem + (size_t)s * C::STAGE;
                mbar_arrive_expect_tx(&full[s], C::STAGE);
                // the database streams through L2 once (evict first); the 8 MiB
                // cipherbuf is read again for every sub-database (evict last)
                bulk_g2s_hint(st, db + ((size_t)r * kN + z) * (kN / 2), C::SLAB, &full[s], pol_db);
                bulk_g2s_hint(st + C::SLAB, cbuf + (size_t)z * 2 * N1, C::QSLAB, &full[s], pol_cb);
            }
            // never leave the CTA with copies in flight into its shared memory
            const long first = issued > C::NST ? issued - C::NST : 0;
            for (long j = first; j < issued; j++)
                if (j != skip_j && !mbar_wait_bounded(&full[j % C::NST], (uint32_t)((j / C::NST) & 1), limit_ns))
                    atomicOr(err, 4);
        }
        return;
    }

    // consumers
    for (long j = warp; j < nloc; j += C::CONS) {
        const int s = (int)(j % C::NST);
        if (!mbar_wait_bounded(&full[s], (uint32_t)((j / C::NST) & 1), limit_ns)) {
            atomicOr(err, 2);
            break;
        }
        uint64_t v[C::NV];
        scan_item_mac<N1>(smem + (size_t)s * C::STAGE, lane, v);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        const long it = blockIdx.x + j * gridDim.x;
        scan_item_store<N1>(v, lane, (int)(it / kN), (int)(it % kN), R, sout);
    }
}

}  // namespace kspir
