// Database preprocessing on the device: the reference's database_tobsgsntt
// followed by database_tocrt (twosteps.cpp:42-179, crt.cpp:859-885), for every
// sub-database at once.
//
// Reference steps for sub-database `data` ([N][N/2] words < bsgsp = 65537):
//   1. diagonal rearrangement into rows R < N/2 (twosteps.cpp:64-74):
//        D[R][j]       = data[(j - R + N/2) mod N/2][j]          j < N/2
//        D[R][N-1-j]   = data[N-1 - ((j - R + N/2) mod N/2)][j]
//   2. slot permutation of row R = k N1 + i (twosteps.cpp:104-118):
//        temp[query_encode[j]] = D[R][j];  row[j] = temp[perm[i][j]]
//      i.e. row[j] = D[R][G_i[j]] with G_i = query_encode^-1 o perm[i]
//      (the host builds the table G);
//   3. inverse NTT mod bsgsp (HEXL, minimal root), lift to signed
//      (v > bsgsp/2: v + crtMod - bsgsp), forward NTT mod crtMod with
//      root_of_unity_crt (twosteps.cpp:156-176);
//   4. datacrt[z * N/2 + R] = (x mod q1) | (x mod q2) << 32 for slot z of row R
//      (crt.cpp:868-880).
// Steps 3-4 run per prime: the NTT mod crtMod reduced mod q1 (q2) is the NTT
// mod q1 (q2) of the lifted input reduced mod q1 (q2) with root_of_unity_crt
// mod q1 (q2), and the lifted value v + crtMod - bsgsp is v + q - bsgsp mod q.
//
// One CTA transforms four consecutive rows in lockstep, so that its output
// words for one slot (rows R..R+3, 32 bytes) fill a whole sector of datacrt.
#pragma once

#include "common.cuh"
#include "ntt.cuh"

namespace kspir {

constexpr int kDbRowsPerCta = 4;
// twiddles of one (channel, direction) + 4 polynomials mod q1 + 4 mod q2
constexpr int kDbRowsSmem = kN * 8 + 2 * kDbRowsPerCta * kPadN * 4;

// Entry D[R][c] of the diagonal rearrangement of one sub-database.
__device__ __forceinline__ size_t db_diag_index(int R, int c) {
    constexpr int H = kN / 2;
    if (c < H) return (size_t)((c - R + H) & (H - 1)) * H + c;
    const int j = kN - 1 - c;
    return (size_t)(kN - 1 - ((j - R + H) & (H - 1))) * H + j;
}

// grid (N/2 / 4, sub-databases), 512 threads.
//   raw   [sub][N][N/2] words < bsgsp (validated by the caller)
//   gtab  [N1][N] gather table G
//   out   [sub][N][N/2] datacrt words (database_tocrt applied)
//   rows  ROWS: also [sub][N/2][N] rows mod crtMod, database_tobsgsntt's own
//         output (its `result`)
template <bool ROWS>
__global__ void __launch_bounds__(kNttThreads, 1)
k_db_rows(const uint64_t* __restrict__ raw, const uint16_t* __restrict__ gtab, uint64_t* __restrict__ out,
          uint64_t* __restrict__ rows, int N1, NttTables tabs) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint8_t* smem = smem_raw;
    uint2* tws = reinterpret_cast<uint2*>(smem);
    uint32_t* s1 = reinterpret_cast<uint32_t*>(smem + kN * 8);    // 4 rows, mod p then mod q1
    uint32_t* s2 = s1 + kDbRowsPerCta * kPadN;                    // 4 rows, mod q2
    const int R0 = blockIdx.x * kDbRowsPerCta;
    const size_t sub = (size_t)blockIdx.y * kN * (kN / 2);
    const uint64_t* data = raw + sub;

    stage_twiddles(tws, tabs, CH_P, NTT_INV);
#pragma unroll
    for (int t = 0; t < kDbRowsPerCta; t++) {
        const int R = R0 + t;
        const uint16_t* g = gtab + (size_t)(R % N1) * kN;
        for (int m = threadIdx.x; m < kN; m += kNttThreads)
            s1[t * kPadN + pidx(m)] = (uint32_t)__ldg(data + db_diag_index(R, __ldg(g + m)));
    }
    cta_ntt_inverse_m<kDbRowsPerCta>(s1, kPadN, tws, CH_P);

    // lift to signed and split per prime; the forward twiddles of q1 replace p's
    const uint32_t q1 = c_dev.ch[CH_Q1].q, q2 = c_dev.ch[CH_Q2].q;
    constexpr uint32_t half = kP / 2;
    for (int k = threadIdx.x; k < kDbRowsPerCta * kPadN; k += kNttThreads) {
        const uint32_t v = s1[k];
        s1[k] = v > half ? v + (q1 - kP) : v;
        s2[k] = v > half ? v + (q2 - kP) : v;
    }
    __syncthreads();
    stage_twiddles(tws, tabs, CH_Q1, NTT_FWD);
    cta_ntt_forward_m<kDbRowsPerCta>(s1, kPadN, tws, CH_Q1);
    stage_twiddles(tws, tabs, CH_Q2, NTT_FWD);
    cta_ntt_forward_m<kDbRowsPerCta>(s2, kPadN, tws, CH_Q2);

    if (ROWS) {
        // the canonical value mod crtMod of each slot, row by row (coalesced)
#pragma unroll
        for (int t = 0; t < kDbRowsPerCta; t++) {
            uint64_t* o = rows + sub + (size_t)(R0 + t) * kN;
            for (int z = threadIdx.x; z < kN; z += kNttThreads)
                o[z] = crt_compose_res(s1[t * kPadN + pidx(z)], s2[t * kPadN + pidx(z)]);
        }
    }
    // slot z of rows R0..R0+3: one 32-byte sector at datacrt[z * N/2 + R0]
    uint64_t* o = out + sub + R0;
    for (int z = threadIdx.x; z < kN; z += kNttThreads) {
        const int pz = pidx(z);
        ulonglong2 a, b;
        a.x = s1[pz] | (uint64_t)s2[pz] << 32;
        a.y = s1[kPadN + pz] | (uint64_t)s2[kPadN + pz] << 32;
        b.x = s1[2 * kPadN + pz] | (uint64_t)s2[2 * kPadN + pz] << 32;
        b.y = s1[3 * kPadN + pz] | (uint64_t)s2[3 * kPadN + pz] << 32;
        ulonglong2* d = reinterpret_cast<ulonglong2*>(o + (size_t)z * (kN / 2));
        d[0] = a;
        d[1] = b;
    }
}

// database_tocrt alone (crt.cpp:859-885) on rows mod crtMod of one or more
// sub-databases: datacrt[z][R] = (x mod q1) | (x mod q2) << 32 for
// x = rows[R][z], any 64-bit x (the reference's Barrett reduction is exact
// for every 64-bit input).  32 x 32 tiles through shared memory; grid
// (N / 32, N/2 / 32, sub-databases), 32 x 8 threads.
__global__ void k_db_tocrt(const uint64_t* __restrict__ rows, uint64_t* __restrict__ datacrt) {
    __shared__ uint64_t tile[32][33];
    const size_t sub = (size_t)blockIdx.z * kN * (kN / 2);
    const int z0 = blockIdx.x * 32, R0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int i = ty; i < 32; i += 8) {
        const uint64_t x = rows[sub + (size_t)(R0 + i) * kN + z0 + tx];
        tile[i][tx] = mod_q1(x) | (uint64_t)mod_q2(x) << 32;
    }
    __syncthreads();
#pragma unroll
    for (int i = ty; i < 32; i += 8) datacrt[sub + (size_t)(z0 + i) * (kN / 2) + R0 + tx] = tile[tx][i];
}

}  // namespace kspir
