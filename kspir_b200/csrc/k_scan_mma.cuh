// Batched database scan on the tensor cores (tcgen05.mma, kind::i8).
//
// For B queries the first-dimension scan (reference
// fastMultiplyQueryByDatabaseDim1InvCRT, crt.cpp:643-856) is, per NTT slot z
// and prime ch, a product of the database slice [r*N2 rows][N1] with the B
// queries' rotation residues [N1][2 comp x B]:
//   out[row][comp][b] = sum_k db_ch[z][row][k] * cb_ch[b][z][k][comp]
// summed exactly in 64 bits (the reference's unreduced sums) and then reduced
// mod q_ch.  Both operands are residues below 2^32, split into four 8-bit limbs
// (db limb la, query limb lb), so one u8 x u8 -> s32 MMA per (la, lb) pair
// gives exact partial sums (K = N1 = 128 terms of at most 255^2 stay below
// 2^23, far from the 2^31 bound of the s32 accumulator), and
//   sum = sum_{la,lb} P[la][lb] << 8 (la + lb)      (mod 2^64, as in the reference)
//
// Tiles.  One MMA M = 128, N = 8 BT, K = 128 bytes (four K = 32 steps) puts
// all 16 limb products of 32 database rows x BT queries x 2 components into
// TMEM.  The row and column orders are chosen for the TMEM load shape
// 16x256b, which hands each thread two lanes 8 apart and two adjacent columns
// of every 8-column chunk: database tile row m = 32 (j / 8) + 8 la + j % 8 and
// query tile row n = 16 (g / 4) + 8 (lb / 2) + 2 (g % 4) + lb % 2 for query
// group g = comp * BT + b.  Two loads (lanes +0 and +16 of the warp's quarter)
// then give one thread all 16 products of one (row, group), folded with
// integer adds and three wide multiply-adds; no data crosses lanes.
//
// Both operands are stored in HBM already in the K-major 128-byte-swizzle
// layout of shared memory, so each tile arrives with one 1-D bulk copy (TMA
// engine, no multicast) at a 1 KiB-aligned stage.
//
// Work: a unit is (ZB consecutive NTT slots, prime, query tile); its ZB query
// tiles stay resident while the database tiles stream through a ring in the
// order (row group g, slot).  The epilogue keeps the ZB results of one
// (row, component, query) in registers and writes them as 16-byte pieces of
// the blocked scan output (sout_idx), where the eight row lanes of a query
// cover two 128-byte lines.
//
// Warp roles: warp 0 producer (one lane), warp 1 TMEM allocation and MMA issue
// (one lane), warps 2.. epilogue (warp w reads TMEM lanes 32 (w % 4) .. and a
// 1/PARTS share of the 16-column chunks).  Every wait is bounded; on a timeout
// the warp sets the error word and leaves its loop, the producer waits for its
// own copies in flight, the MMA lane for its own MMAs, and TMEM is freed.
#pragma once

#include "common.cuh"
#include "pipeline.cuh"
#include "ptx.cuh"

namespace kspir {

// byte offset of (row, k) in a K-major tile of 128-byte rows under the 128-byte
// swizzle: 8-row groups of 1 KiB, 16-byte chunk index XOR (row mod 8)
__host__ __device__ __forceinline__ uint32_t sw128_off(int row, int k) {
    return (uint32_t)((row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 4) ^ row) & 7) << 4) + (k & 15));
}

constexpr int kMmaK = 128;              // K bytes per tile row (N1 = 128)
constexpr int kATile = 128 * kMmaK;     // database tile: 32 rows x 4 limbs
constexpr int kMmaSmemLimit = 232448;   // 227 KiB opt-in per block
constexpr uint64_t kMmaWaitNs = 2000000000ull;

template <int BT>
struct MmaCfg {
    static_assert(BT == 4 || BT == 8 || BT == 16 || BT == 32, "query tile");
    static constexpr int N = 8 * BT;                  // MMA N = TMEM columns per accumulator
    static constexpr int ZB = BT == 32 ? 4 : 8;       // NTT slots per unit
    static constexpr int BTILE = N * kMmaK;
    static constexpr int NTB = N >= 256 ? 2 : 4;      // TMEM accumulators (512 columns allocated)
    static constexpr int BAR_BYTES = 512;
    static constexpr int NA_FIT = (kMmaSmemLimit - 1024 - BAR_BYTES - ZB * BTILE) / kATile;
    static constexpr int NA = NA_FIT < 6 ? NA_FIT : 6;  // database-tile ring
    static constexpr int SMEM = 1024 + ZB * BTILE + NA * kATile + BAR_BYTES;
    static constexpr int CHUNKS = N / 16;             // 16-column chunks = 4 query groups each
    static constexpr int PARTS = CHUNKS < 4 ? CHUNKS : 4;   // epilogue warps per TMEM quarter
    static constexpr int CPW = CHUNKS / PARTS;        // chunks (outputs per lane) per epilogue warp
    static constexpr int LDB = CPW < 2 ? CPW : 2;     // outputs whose TMEM loads share one wait
    static constexpr int EPI = 4 * PARTS;             // epilogue warps
    static constexpr int THREADS = 32 * (2 + EPI);
    static_assert(NA >= 2 && SMEM <= kMmaSmemLimit, "shared memory budget");
    static_assert(NTB * N <= 512, "TMEM columns");
};

// tile row of database row j (0..31) limb la, and of query group g limb lb
__host__ __device__ __forceinline__ int mma_arow(int j, int la) { return 32 * (j >> 3) + 8 * la + (j & 7); }
__host__ __device__ __forceinline__ int mma_brow(int g, int lb) {
    return 16 * (g >> 2) + 8 * (lb >> 1) + 2 * (g & 3) + (lb & 1);
}

// instruction descriptor: u8 x u8 -> s32, A and B K-major, M = 128
__host__ __device__ constexpr uint32_t mma_idesc_u8(int n) {
    return (2u << 4) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

// shared-memory descriptor of a K-major 128-byte-swizzled tile at smem address a
__device__ __forceinline__ uint64_t mma_sdesc_sw128(uint32_t a) {
    return (uint64_t)((a & 0x3FFFF) >> 4) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ void mma_u8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// 16x256b, 2 repetitions: 16 lanes x 16 columns; thread t receives lanes
// L = base + t / 4 and L + 8, columns c = 2 (t % 4) + {0, 1} of each 8-column
// repetition: v = {(L,c), (L,c+1), (L+8,c), (L+8,c+1)} x 2 repetitions
__device__ __forceinline__ void tmem_ld_16x256b_x2(uint32_t taddr, uint32_t (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.16x256b.x2.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

struct ScanMmaArgs {
    const uint8_t* dbop;     // [N][2 ch][G][kATile]
    const uint8_t* qop;      // [N][2 ch][QT][BTILE]
    uint32_t* sout0;         // scan output of workspace slot 0 (slots at ws_bytes)
    size_t ws_bytes;
    int slot0, nq, QT, G, rows;   // rows = r * N2
    int* err;
};

template <int BT>
__global__ void __launch_bounds__(MmaCfg<BT>::THREADS, 1) k_scan_mma(ScanMmaArgs a) {
    using C = MmaCfg<BT>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* btiles = smem;                          // [ZB][BTILE]
    uint8_t* atiles = smem + C::ZB * C::BTILE;       // [NA][kATile]
    uint64_t* bars = reinterpret_cast<uint64_t*>(atiles + C::NA * kATile);
    uint64_t* a_full = bars;
    uint64_t* a_empty = a_full + C::NA;
    uint64_t* b_full = a_empty + C::NA;
    uint64_t* b_empty = b_full + C::ZB;
    uint64_t* t_full = b_empty + C::ZB;
    uint64_t* t_empty = t_full + C::NTB;
    uint64_t* done = t_empty + C::NTB;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
        for (int s = 0; s < C::NA; s++) { mbar_init(&a_full[s], 1); mbar_init(&a_empty[s], 1); }
        for (int s = 0; s < C::ZB; s++) { mbar_init(&b_full[s], 1); mbar_init(&b_empty[s], 1); }
        for (int s = 0; s < C::NTB; s++) { mbar_init(&t_full[s], 1); mbar_init(&t_empty[s], C::EPI); }
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_addr(tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    const int QT = a.QT, G = a.G;
    const int units = (kN / C::ZB) * 2 * QT;

    if (warp == 0) {
        // producer
        if (lane == 0) {
            long ia = 0;
            int tu = 0;
            int bl[C::ZB];   // query-tile copies issued per slot
            for (int zi = 0; zi < C::ZB; zi++) bl[zi] = 0;
            bool ok = true;
            for (int u = blockIdx.x; u < units && ok; u += gridDim.x, tu++) {
                const int qt = u % QT, ch = (u / QT) & 1, z0 = (u / QT >> 1) * C::ZB;
                for (int g = 0; g < G && ok; g++)
                    for (int zi = 0; zi < C::ZB && ok; zi++) {
                        const int z = z0 + zi;
                        if (g == 0) {
                            if (tu > 0 && !mbar_wait_bounded(&b_empty[zi], (uint32_t)((tu - 1) & 1), kMmaWaitNs)) {
                                atomicOr(a.err, 8); ok = false; break;
                            }
                            mbar_arrive_expect_tx(&b_full[zi], C::BTILE);
                            bulk_g2s(btiles + zi * C::BTILE, a.qop + (((size_t)z * 2 + ch) * QT + qt) * C::BTILE,
                                     C::BTILE, &b_full[zi]);
                            bl[zi]++;
                        }
                        const int sa = (int)(ia % C::NA);
                        if (ia >= C::NA && !mbar_wait_bounded(&a_empty[sa], (uint32_t)((ia / C::NA - 1) & 1), kMmaWaitNs)) {
                            atomicOr(a.err, 8); ok = false; break;
                        }
                        mbar_arrive_expect_tx(&a_full[sa], kATile);
                        bulk_g2s(atiles + sa * kATile, a.dbop + (((size_t)z * 2 + ch) * G + g) * kATile, kATile,
                                 &a_full[sa]);
                        ia++;
                    }
            }
            // never leave with copies in flight into shared memory
            for (long j = ia > C::NA ? ia - C::NA : 0; j < ia; j++)
                if (!mbar_wait_bounded(&a_full[j % C::NA], (uint32_t)((j / C::NA) & 1), kMmaWaitNs)) atomicOr(a.err, 16);
            for (int zi = 0; zi < C::ZB; zi++)
                if (bl[zi] > 0 && !mbar_wait_bounded(&b_full[zi], (uint32_t)((bl[zi] - 1) & 1), kMmaWaitNs))
                    atomicOr(a.err, 16);
        }
    } else if (warp == 1) {
        // MMA issue
        if (lane == 0) {
            const uint32_t idesc = mma_idesc_u8(C::N);
            const uint32_t abase = smem_addr(atiles), bbase = smem_addr(btiles);
            long ia = 0, tc = 0;
            int tu = 0;
            bool ok = true;
            for (int u = blockIdx.x; u < units && ok; u += gridDim.x, tu++) {
                for (int g = 0; g < G && ok; g++)
                    for (int zi = 0; zi < C::ZB; zi++) {
                        if (g == 0 && !mbar_wait_bounded(&b_full[zi], (uint32_t)(tu & 1), kMmaWaitNs)) {
                            atomicOr(a.err, 32); ok = false; break;
                        }
                        const int sa = (int)(ia % C::NA);
                        if (!mbar_wait_bounded(&a_full[sa], (uint32_t)((ia / C::NA) & 1), kMmaWaitNs)) {
                            atomicOr(a.err, 32); ok = false; break;
                        }
                        const int tb = (int)(tc % C::NTB);
                        if (tc >= C::NTB &&
                            !mbar_wait_bounded(&t_empty[tb], (uint32_t)((tc / C::NTB - 1) & 1), kMmaWaitNs)) {
                            atomicOr(a.err, 32); ok = false; break;
                        }
                        tc_fence_after();
                        const uint64_t ad = mma_sdesc_sw128(abase + sa * kATile);
                        const uint64_t bd = mma_sdesc_sw128(bbase + zi * C::BTILE);
#pragma unroll
                        for (int kk = 0; kk < kMmaK / 32; kk++)
                            mma_u8(tmem + tb * C::N, ad + 2 * kk, bd + 2 * kk, idesc, kk > 0);
                        mma_commit(&a_empty[sa]);
                        if (g == G - 1) mma_commit(&b_empty[zi]);
                        mma_commit(&t_full[tb]);
                        ia++;
                        tc++;
                    }
            }
            mma_commit(done);
            if (!mbar_wait_bounded(done, 0, kMmaWaitNs)) atomicOr(a.err, 64);
        }
    } else {
        // epilogue: warp (quarter q, part p) owns TMEM lanes 32q.. and chunks p*CPW ..
        const int quarter = warp & 3, part = (warp - 2) >> 2;
        const int j3 = lane >> 2, gq = lane & 3;
        const int jrow = 8 * quarter + j3;   // database row within the 32-row tile
        const uint32_t tq = tmem + ((uint32_t)(32 * quarter) << 16) + part * C::CPW * 16;
        long tc = 0;
        bool ok = true;
        uint32_t ob[C::ZB][C::CPW];
        for (int u = blockIdx.x; u < units && ok; u += gridDim.x) {
            const int qt = u % QT, ch = (u / QT) & 1, z0 = (u / QT >> 1) * C::ZB;
            const uint32_t q = ch ? kQ2 : kQ1;
            const uint32_t mu1 = ch ? (uint32_t)((1ull << 59) / kQ2) : (uint32_t)((1ull << 59) / kQ1);
            const uint32_t c32 = ch ? (uint32_t)((1ull << 32) % kQ2) : (uint32_t)((1ull << 32) % kQ1);
            const uint32_t mu2 = ch ? (uint32_t)((1ull << 57) / kQ2) : (uint32_t)((1ull << 57) / kQ1);
            for (int g = 0; g < G && ok; g++) {
#pragma unroll
                for (int zi = 0; zi < C::ZB; zi++) {
                    const int tb = (int)(tc % C::NTB);
                    // warp-uniform outcome: tcgen05.ld below needs the whole warp
                    const bool got = mbar_wait_bounded(&t_full[tb], (uint32_t)((tc / C::NTB) & 1), kMmaWaitNs);
                    if (!__all_sync(0xffffffffu, got)) {
                        if (lane == 0) atomicOr(a.err, 128);
                        ok = false;
                        break;
                    }
                    tc_fence_after();
#pragma unroll
                    for (int c0 = 0; c0 < C::CPW; c0 += C::LDB) {
                        // LDB outputs per wait: their loads overlap
                        uint32_t lo[C::LDB][8], hi[C::LDB][8];   // limbs la 0,1 and la 2,3
#pragma unroll
                        for (int c1 = 0; c1 < C::LDB; c1++) {
                            const uint32_t col = tq + tb * C::N + (c0 + c1) * 16;
                            tmem_ld_16x256b_x2(col, lo[c1]);
                            tmem_ld_16x256b_x2(col + (16u << 16), hi[c1]);
                        }
                        tmem_wait_ld();
#pragma unroll
                        for (int c1 = 0; c1 < C::LDB; c1++) {
                            const uint32_t* L = lo[c1];
                            const uint32_t* H = hi[c1];
                            // v[la][lb]: L = {00, 01, 10, 11, 02, 03, 12, 13}, H likewise for la + 2
                            const uint32_t t1 = L[1] + L[2];
                            const uint32_t t2 = L[4] + L[3] + H[0];
                            const uint32_t t3 = L[5] + L[6] + H[1] + H[2];
                            const uint32_t t4 = L[7] + H[4] + H[3];
                            const uint32_t t5 = H[5] + H[6];
                            uint64_t x = L[0];
                            mad_wide(x, t1, 1u << 8);
                            mad_wide(x, t2, 1u << 16);
                            mad_wide(x, t3, 1u << 24);
                            const uint32_t xh = t4 + (t5 << 8) + (H[7] << 16);   // weights 2^32.. (mod 2^64)
                            x += (uint64_t)xh << 32;
                            ob[zi][c0 + c1] = mod28(x, q, mu1, c32, mu2);
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&t_empty[tb]);
                    tc++;
                }
                if (!ok) break;
                const int row = 32 * g + jrow;
                if (row < a.rows) {
#pragma unroll
                    for (int c = 0; c < C::CPW; c++) {
                        const int grp = 4 * (part * C::CPW + c) + gq;   // comp * BT + b
                        const int comp = grp / BT, bq = qt * BT + grp % BT;
                        if (bq < a.nq) {
                            uint32_t* so = reinterpret_cast<uint32_t*>(reinterpret_cast<char*>(a.sout0) +
                                                                       (size_t)(a.slot0 + bq) * a.ws_bytes);
                            // four consecutive slots per 16-byte store; the eight
                            // row lanes of this query cover two 128-byte lines
#pragma unroll
                            for (int z4 = 0; z4 < C::ZB; z4 += 4)
                                *reinterpret_cast<uint4*>(so + sout_idx(row, comp * 2 + ch, z0 + z4, a.rows)) =
                                    make_uint4(ob[z4][c], ob[z4 + 1][c], ob[z4 + 2][c], ob[z4 + 3][c]);
                        }
                    }
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        __syncwarp();
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
    }
}

// Query operand of a batch: qop[z][ch][qt] tiles of 8 BT rows
// n = mma_brow(comp * BT + b, lb), byte k = limb lb of the prime-ch residue of
// entry (k, comp) of slot z of the cipherbuf of query qt * BT + b (workspace
// slot slot0 + that); queries past nq are zero.  Built from the
// rotation-major cipherbuf (cipherbuf_rm_idx: u32 [k][comp][ch][z]), a
// transpose: one CTA per (block of 32 slots, query slot qt * BT + b).  The
// CTA loads the 512 rows (k, comp, ch) of its slots
// (128 contiguous bytes each) into shared memory, column zz stored at
// zz ^ 4 (k / 16) so that the reads below hit 32 distinct banks, then each
// thread takes slot zz, 16-entry chunk c and component comp of both primes: 16 words,
// byte-transposed into the 4 limb rows' 16-byte chunks (eight threads write
// the 128 bytes of one tile row).
constexpr int kSplitZ = 32;
constexpr int kSplitThreads = 512;
constexpr int kSplitSmem = kMmaK * 4 * kSplitZ * 4;   // 64 KiB

template <int BT>
__global__ void __launch_bounds__(kSplitThreads) k_qop_split_rm(const uint32_t* __restrict__ cb0, size_t ws_bytes,
                                                               int slot0, int nq, int QT, uint8_t* __restrict__ qop) {
    using C = MmaCfg<BT>;
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint32_t* V = reinterpret_cast<uint32_t*>(smem_raw);   // [512 rows][32 columns]
    const int z0 = blockIdx.x * kSplitZ;
    const int bq = blockIdx.y;                              // qt * BT + b
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool live = bq < nq;
    if (live) {
        const uint32_t* cb = reinterpret_cast<const uint32_t*>(reinterpret_cast<const char*>(cb0) +
                                                              (size_t)(slot0 + bq) * ws_bytes);
        constexpr int W = kSplitThreads / 32;
#pragma unroll 32
        for (int row = warp; row < kMmaK * 4; row += W)
            V[row * kSplitZ + (lane ^ (4 * ((row >> 6) & 7)))] = __ldg(cb + (size_t)row * kN + z0 + lane);
        __syncthreads();
    }
    const int c = tid & 7;                                  // 16-entry chunk of k
    const int zz = 4 * (warp & 7) + ((tid >> 3) & 3);
    const int comp = warp >> 3;                             // warps 0-7: a, 8-15: b
    const int z = z0 + zz;
    const int qt = bq / BT, b = bq % BT;
#pragma unroll
    for (int ch = 0; ch < 2; ch++) {
        const int cv = comp * 2 + ch;
        uint32_t w[4][4];   // [limb][word]
#pragma unroll
        for (int g = 0; g < 4; g++) {
            uint32_t v[4];
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const int row = (16 * c + 4 * g + t) * 4 + cv;
                v[t] = live ? V[row * kSplitZ + (zz ^ (4 * c))] : 0u;
            }
            // 4 x 4 byte transpose: word g of limb lb = byte lb of v[0..3]
            const uint32_t t0 = __byte_perm(v[0], v[1], 0x5140), t1 = __byte_perm(v[0], v[1], 0x7362);
            const uint32_t t2 = __byte_perm(v[2], v[3], 0x5140), t3 = __byte_perm(v[2], v[3], 0x7362);
            w[0][g] = __byte_perm(t0, t2, 0x5410);
            w[1][g] = __byte_perm(t0, t2, 0x7632);
            w[2][g] = __byte_perm(t1, t3, 0x5410);
            w[3][g] = __byte_perm(t1, t3, 0x7632);
        }
        uint8_t* tile = qop + (((size_t)z * 2 + ch) * QT + qt) * C::BTILE;
#pragma unroll
        for (int lb = 0; lb < 4; lb++)
            *reinterpret_cast<uint4*>(tile + sw128_off(mma_brow(comp * BT + b, lb), 16 * c)) =
                make_uint4(w[lb][0], w[lb][1], w[lb][2], w[lb][3]);
    }
}

// Database operand: dbop[z][ch][g] tiles of 128 rows m = mma_arow(j, la), byte k =
// limb la of the prime-ch half of datacrt word [r][z][i][k] with
// r * N2 + i = 32 g + j (rows past r * N2 are zero).  One thread per
// (z, ch, g, j, la, 16-byte chunk).  Runs once per database upload.
__global__ void k_dbop_build(const uint64_t* __restrict__ db, uint8_t* __restrict__ dbop, int R, int N2, int G) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long total = (long)kN * 2 * G * 128 * 8;
    if (idx >= total) return;
    const int c = (int)(idx & 7);
    const int jl = (int)((idx >> 3) & 127);     // 4 j + la
    const long zcg = idx >> 10;                 // (z * 2 + ch) * G + g
    const int g = (int)(zcg % G);
    const int ch = (int)((zcg / G) & 1);
    const int z = (int)(zcg / G / 2);
    const int row = 32 * g + (jl >> 2), la = jl & 3;
    const int m = mma_arow(jl >> 2, la);
    uint32_t pk[4] = {0, 0, 0, 0};
    if (row < R * N2) {
        const int r = row / N2, i = row % N2;
        const uint64_t* src = db + (((size_t)r * kN + z) * N2 + i) * kMmaK + 16 * c;
#pragma unroll
        for (int q4 = 0; q4 < 4; q4++) {
            uint32_t x = 0;
#pragma unroll
            for (int t = 0; t < 4; t++) {
                const uint64_t wv = __ldg(src + 4 * q4 + t);
                const uint32_t h = ch ? (uint32_t)(wv >> 32) : (uint32_t)wv;
                x |= ((h >> (8 * la)) & 255u) << (8 * t);
            }
            pk[q4] = x;
        }
    }
    *reinterpret_cast<uint4*>(dbop + (size_t)zcg * kATile + sw128_off(m, 16 * c)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
}

}  // namespace kspir
