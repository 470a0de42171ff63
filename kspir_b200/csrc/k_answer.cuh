// The whole single-query online answer (reference tests/test-pir.cpp:110-116:
// matrix_vector_mul_bsgs_rns_crt_large -> externalProduct x r -> packingRLWEs)
// as ONE persistent cooperative kernel, so that the key switches overlap the
// database scan instead of running before and after it.
//
// As separate kernels, the scan streams the database (1 GiB at r = 16) at HBM
// speed on every SM, and the key switches around it -- baby steps before,
// giant steps, external products and the packing tree after -- run one
// kernel after another.  They are chains of dependent 4096-point transforms
// whose latency, not throughput, sets their time, so most of the GPU idles
// while they run.  Here each SM runs one CTA of two warp groups:
//   * the scan group (one producer warp, SCAN_WARPS consumer warps) streams
//     the database slabs through a shared-memory ring with 1-D bulk copies and
//     computes exactly what k_scan computes (crt.cpp:643-856), sub-database by
//     sub-database in the order the packing tree consumes them;
//   * the key-switch group (512 threads) takes tasks from one queue shared by
//     every CTA: the query's digits and transforms and the baby-step
//     rotations (twosteps.cpp:937-1204, 1386-1403) first, then, as soon as a
//     sub-database's scan is complete, its giant-step key switches
//     (twosteps.cpp:599-677) and external products (lwe.cpp:761-808), and the
//     merges of the packing tree (answer.cpp:720-835) as their inputs complete,
//     and last the response words.
// The grid is one CTA per SM, launched cooperatively, so every CTA is
// resident and a task may wait for another CTA's progress.  The queue holds
// every task after all the tasks it depends on (the host checks this when it
// builds the queue), so every wait ends; each wait is bounded as well
// (limit_ns): a wait that runs out records an error word and raises the
// abort flag that every other wait polls, and the kernel returns.
//
// Dependencies are counters in global memory, zeroed by k_fa_reset before the
// launch.  A task's group writes its results, meets at its barrier, and one
// thread publishes them with a fence and an atomic increment; a waiting
// thread polls with an acquire load before its group reads.  Data produced
// inside the kernel is read through L2 (ld.global.cg) or by bulk copies after
// a proxy fence, never from a possibly stale L1 line.
//
// The values are those of the separate kernels: the same device functions
// compute them.  Only the giant steps differ in form: each adds its terms into
// a per-sub-database accumulator (u32 sums of at most N2 - 1 = 15 canonical
// residues, exact) instead of rewriting the scan-output row it read, and the
// external product adds the scan's row 0 and reduces.
#pragma once

#include "k_baby.cuh"
#include "k_query.cuh"
#include "k_scan.cuh"
#include "k_second.cuh"
#include "k_util.cuh"

namespace kspir {

// named barrier 1 of the key-switch group (warps 0-15); barrier 0 is the CTA's
struct KsSync {
    __device__ __forceinline__ static void sync() { asm volatile("bar.sync 1, 512;" ::: "memory"); }
};

enum FaTaskType : uint8_t {
    FT_PREP = 0,      // b = chunk of 512 query coefficients
    FT_QNTT,          // b = job of the query segment (digits, b, modswitched query -> cipherbuf column 0)
    FT_ROT1,          // b = key index ki, a = comp: rotation 1 + ki from the query
    FT_INTER_NTT,     // b = job: the intermediate rotation's a to coefficient form
    FT_INTER_DEC,     // b = chunk: its digits
    FT_DIG1,          // b = job: the digit transforms
    FT_ROT2,          // b = ki, a = comp: rotation N1/2 + ki from the intermediate
    FT_GIANT,         // b = sub-database r, c = giant row (1..N2-1)
    FT_EXT,           // b = r, a = prime
    FT_PFWD,          // a = level, b = pair j, c = prime, d = digit (ELL: temp.b)
    FT_PINV,          // a = level, b = pair j, c = prime, d = comp
    FT_COMPOSE,       // the response words
};

struct FaTask {
    uint8_t type, a;
    uint16_t b, c, d;
};

// counter words (k_fa_reset zeroes 16 + 6 R of them)
enum : int {
    FC_HEAD = 0, FC_ABORT, FC_PREP, FC_QNTT, FC_ROT1, FC_INTER_ROT, FC_INTER_NTT, FC_INTER_DEC, FC_DIG1, FC_ROT2,
    FC_ZERO, FC_COMPOSE, FC_PER_R = 16,   // then scan [R], giant [R], ext [R], fwd [2R], merge [R]
};
__host__ __device__ __forceinline__ int fa_counter_words(int R) { return FC_PER_R + 6 * R; }

// device timestamps of one answer (ns of %globaltimer): fields kept as maxima,
// minima stored complemented (max of ~t)
enum : int { FT_T_START = 0, FT_T_HEAD, FT_T_SCAN0, FT_T_SCAN1, FT_T_GIANT, FT_T_EXT, FT_T_END, FT_T_COUNT = 8 };

constexpr int kFaPrepChunks = kN / kNttThreads;   // 8
constexpr int kFaKsSmem = kN * 8 + 4 * kPadN * 4;  // twiddles + four padded polynomials

template <int N1, int SCAN_WARPS>
struct FaCfg {
    using SC = ScanCfg<N1>;
    static constexpr int CONS = SCAN_WARPS;
    static constexpr int NST = SCAN_WARPS;                 // each consumer warp owns one stage
    static constexpr int THREADS = kNttThreads + 32 * (CONS + 1);
    static constexpr int RING = NST * SC::STAGE;
    static constexpr int SMEM = kFaKsSmem + RING + 2 * NST * 8;
    static_assert(SMEM <= 227 * 1024, "shared memory budget");
};

struct FaArgs {
    Workspace w;              // slot-0 workspace (shifted by bt)
    ClientKeysDev keys;       // slot-0 keys (shifted by bt's client)
    Batch bt;
    NttTables tabs;
    PathGadgets gad;
    BabyArgs a1, a2;          // first / second half of the rotations (reference cipherbuf layout)
    const NttJob* jobs;
    int seg_q, n_q, seg_inter, seg_dig1;
    int inter_idx;            // key index of the intermediate rotation
    const uint16_t* sigma_giant;
    const uint64_t* db;
    int R, N1, levels;
    const FaTask* tasks;
    int ntasks;
    int* cnt;                 // counter words
    uint32_t* acc;            // giant-step accumulators [R][4][N]
    unsigned long long* times;   // [FT_T_COUNT]
    uint64_t limit_ns;
    long skip;                // failure injection: CTA 0's producer skips this local item (-1: none)
    int* err;                 // the slot's error word
};

// The shape of a fused answer's task graph (host and device).
struct FaShape {
    int R, N1, levels, n_q, inter_idx, ctas;
};

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fa_abort(const FaArgs& A, int code) {
    atomicOr(A.err, code);
    atomicExch(A.cnt + FC_ABORT, 1);
}

__device__ __forceinline__ bool fa_aborted(const FaArgs& A) {
    return *reinterpret_cast<volatile const int*>(A.cnt + FC_ABORT) != 0;
}

// One thread waits until counter `idx` reaches `target`: false on abort or
// when limit_ns runs out (which raises the abort).  Not inlined, and given
// plain values, so the kernel's argument block is not copied to the stack.
__device__ __noinline__ bool fa_wait_counter(int* cnt, int idx, int target, uint64_t limit_ns, int* err) {
    const int* c = cnt + idx;
    if (ld_acquire_gpu(c) >= target) return true;
    const uint64_t t0 = globaltimer_ns();
    // exponential backoff from 64 ns to 2 us: a waiter polls L2, which the
    // database stream is saturating
    for (unsigned ns = 64;; ns = ns < 2048 ? 2 * ns : ns) {
        __nanosleep(ns);
        if (ld_acquire_gpu(c) >= target) return true;
        if (*reinterpret_cast<volatile const int*>(cnt + FC_ABORT)) return false;
        if (globaltimer_ns() - t0 > limit_ns) {
            atomicOr(err, 8);
            atomicExch(cnt + FC_ABORT, 1);
            return false;
        }
    }
}

__device__ __forceinline__ bool fa_wait(const FaArgs& A, int idx, int target) {
    return fa_wait_counter(A.cnt, idx, target, A.limit_ns, A.err);
}

// mbarrier phase wait of the scan group, bounded and abortable
__device__ __forceinline__ bool fa_mbar_wait(const FaArgs& A, uint64_t* bar, uint32_t parity, int code) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 1;; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0) {
            if (fa_aborted(A)) return false;
            if (globaltimer_ns() - t0 > A.limit_ns) {
                fa_abort(A, code);
                return false;
            }
        }
    }
}

__device__ __forceinline__ void fa_signal(int* c, int v) {
    __threadfence();
    atomicAdd(c, v);
}

__device__ __forceinline__ void fa_time_max(const FaArgs& A, int f) {
    atomicMax(A.times + f, (unsigned long long)globaltimer_ns());
}
__device__ __forceinline__ void fa_time_min(const FaArgs& A, int f) {
    atomicMax(A.times + f, ~(unsigned long long)globaltimer_ns());
}

// sub-database scanned at position t: bit reversal of t over log2 R bits, so
// that the subtrees of the packing tree complete one after another
__host__ __device__ __forceinline__ int fa_scan_order(int t, int levels) {
    int x = 0;
    for (int b = 0; b < levels; b++) x |= ((t >> b) & 1) << (levels - 1 - b);
    return x;
}

// g^-1 mod 2N for odd g (the group of units mod 2N = 8192 has order 2048)
__device__ __forceinline__ uint32_t inv_mod_2n_dev(uint32_t g) {
    uint32_t r = 1, b = g & (2 * kN - 1);
    for (uint32_t e = 2047; e; e >>= 1) {
        if (e & 1) r = (r * b) & (2 * kN - 1);
        b = (b * b) & (2 * kN - 1);
    }
    return r;
}

// level lv of the packing tree reads ext (levels - 1 - lv even) or ext2
__device__ __forceinline__ bool fa_level_reads_ext(int levels, int lv) { return ((levels - 1 - lv) & 1) == 0; }

// ---------------------------------------------------------------------------
// tasks of the key-switch group (all 512 threads, uniform control flow)

template <bool INVERSE>
__device__ __forceinline__ void fa_ntt_job(const FaArgs& A, NttJob jb, uint8_t* smem) {
    uint2* tws = reinterpret_cast<uint2*>(smem);
    uint32_t* s = reinterpret_cast<uint32_t*>(smem + kN * 8);
    jb.src = shifted(jb.src, ws_off(A.bt));
    jb.dst = shifted(jb.dst, ws_off(A.bt));
    stage_twiddles(tws, A.tabs, jb.ch, INVERSE ? NTT_INV : NTT_FWD);
    ntt_job_run<INVERSE, KsSync>(jb, tws, s);
}

// one rotation (key index ki, component comp), both primes: k_baby_pair's work
__device__ __forceinline__ void fa_rotation(const FaArgs& A, const BabyArgs& a, int ki, int comp, uint8_t* smem) {
    uint2* tws = reinterpret_cast<uint2*>(smem);
    uint32_t* S = reinterpret_cast<uint32_t*>(smem + kN * 8);
    uint32_t* S2 = S + kPadN;
    BabyRot R;
    stage_twiddles(tws, A.tabs, CH_BS, NTT_INV);
    baby_setup<3>(R, a, A.keys, A.bt, ki, comp);
    baby_bs_part<3, KsSync>(R, a, S, tws, true);
#pragma unroll
    for (int it = 0; it < kPerThread; it++) S2[pidx(R.tid) + it * kPadStep] = S[pidx(R.tid) + it * kPadStep];
    baby_crt_part<3, KsSync>(R, a, S, tws, A.tabs, 0);
    baby_crt_part<3, KsSync>(R, a, S2, tws, A.tabs, 1);
}

// giant step (r, c): the key switch of evalAutoRNSCRT for output row c of
// sub-database r (twosteps.cpp:612-672), as k_giant_fused computes it: the
// terms are added into acc[r].
template <int ELL>
__device__ __forceinline__ void fa_giant(const FaArgs& A, int r, int c, uint8_t* smem) {
    uint2* tws = reinterpret_cast<uint2*>(smem);
    uint32_t* P = reinterpret_cast<uint32_t*>(smem + kN * 8);   // [4][N]
    const int N1 = A.N1, N2 = kN / 2 / N1;
    const int rows = A.R * N2, row = r * N2 + c;
    const int tid = threadIdx.x;
    const uint32_t* sout = shifted(A.w.sout, ws_off(A.bt));
    const uint32_t* gkeys = shifted(A.keys.giant, key_off(A.bt));
    uint32_t* acc = A.acc + (size_t)r * 4 * kN;
#pragma unroll
    for (int ch = 0; ch < 2; ch++) {
        stage_twiddles(tws, A.tabs, ch, NTT_INV);
#pragma unroll
        for (int k = tid; k < kN / 4; k += kNttThreads)
            *reinterpret_cast<uint4*>(P + ch * kPadN + pidx(4 * k)) =
                __ldcg(reinterpret_cast<const uint4*>(sout + sout_idx(row, 0 * 2 + ch, 4 * k, rows)));
        cta_ntt_inverse<KsSync>(P + ch * kPadN, tws, ch);
    }
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
        decompose_b(v, kCrtMod, A.gad.giant, dig);
#pragma unroll
        for (int j = 0; j < ELL; j++) {
            dres[it][j][0] = signed_to_res(dig[j], kQ1);
            dres[it][j][1] = signed_to_res(dig[j], kQ2);
        }
    }
    KsSync::sync();
#pragma unroll
    for (int it = 0; it < kPerThreadG; it++)
#pragma unroll
        for (int j = 0; j < ELL; j++)
#pragma unroll
            for (int ch = 0; ch < 2; ch++) P[(j * 2 + ch) * kPadN + pidx(tid) + it * kPadStep] = dres[it][j][ch];
    const uint32_t* key = gkeys + (size_t)(c - 1) * ELL * 2 * 2 * kN;   // [ELL][2 comp][2 ch][N]
    const uint16_t* sig = A.sigma_giant + (size_t)(c - 1) * kN;
#pragma unroll 1
    for (int ch = 0; ch < 2; ch++) {
        KsSync::sync();
        stage_twiddles(tws, A.tabs, ch, NTT_FWD);
        cta_ntt_forward_m<ELL, KsSync>(P + ch * kPadN, 2 * kPadN, tws, ch);
        const uint32_t q = c_dev.ch[ch].q;
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
            atomicAdd(acc + (size_t)(0 * 2 + ch) * kN + k, negmod(mod_crt(sa, ch), q));
            atomicAdd(acc + (size_t)(1 * 2 + ch) * kN + k, addmod(bv, negmod(mod_crt(sb, ch), q), q));
        }
    }
}

// external product of sub-database r on prime ch: the first-dimension result
// is (acc[r] + scan row 0) mod q (k_giant_finish's sum); the task of prime 0
// also keeps it (NTT form) in the workspace's result for the diagnostics.
__device__ __forceinline__ void fa_ext(const FaArgs& A, int r, int ch, uint8_t* smem) {
    uint2* tws = reinterpret_cast<uint2*>(smem);
    uint32_t* P = reinterpret_cast<uint32_t*>(smem + kN * 8);
    const int N2 = kN / 2 / A.N1, rows = A.R * N2, row0 = r * N2;
    const int tid = threadIdx.x;
    const size_t wo = ws_off(A.bt);
    const uint32_t* sout = shifted(A.w.sout, wo);
    const uint32_t* acc = A.acc + (size_t)r * 4 * kN;
    uint32_t* result = shifted(A.w.result, wo) + (size_t)r * 4 * kN;
#pragma unroll
    for (int pch = 0; pch < 2; pch++) {
        const ChanConst cq = c_dev.ch[pch];
        stage_twiddles(tws, A.tabs, pch, NTT_INV);
#pragma unroll
        for (int comp = 0; comp < 2; comp++) {
            const int cv = comp * 2 + pch;
#pragma unroll
            for (int k4 = tid; k4 < kN / 4; k4 += kNttThreads) {
                const uint4 a4 = __ldcg(reinterpret_cast<const uint4*>(acc + (size_t)cv * kN) + k4);
                const uint4 s4 = __ldcg(reinterpret_cast<const uint4*>(sout + sout_idx(row0, cv, 4 * k4, rows)));
                uint4 v;
                v.x = reduce64((uint64_t)a4.x + s4.x, cq.q, cq.barrett);
                v.y = reduce64((uint64_t)a4.y + s4.y, cq.q, cq.barrett);
                v.z = reduce64((uint64_t)a4.z + s4.z, cq.q, cq.barrett);
                v.w = reduce64((uint64_t)a4.w + s4.w, cq.q, cq.barrett);
                *reinterpret_cast<uint4*>(P + cv * kPadN + pidx(4 * k4)) = v;
                if (ch == 0) reinterpret_cast<uint4*>(result + (size_t)cv * kN)[k4] = v;
            }
        }
        cta_ntt_inverse_m<2, KsSync>(P + pch * kPadN, 2 * kPadN, tws, pch);
    }
    const uint32_t* rgsw = shifted(A.keys.rgsw, key_off(A.bt));
    uint32_t* ext = shifted(A.w.ext, wo) + (size_t)r * 4 * kN;
    ext_tail<2, KsSync>(P, tws, rgsw, nullptr, ext, A.tabs, A.gad.ext, ch);
}

__device__ __forceinline__ void fa_pack_fwd(const FaArgs& A, int lv, int j, int ch, int d, uint8_t* smem) {
    const int I = 1 << lv;
    const size_t wo = ws_off(A.bt);
    const uint32_t* in = shifted(fa_level_reads_ext(A.levels, lv) ? A.w.ext : A.w.ext2, wo);
    const uint32_t* key = shifted(A.keys.packing, key_off(A.bt)) + (size_t)lv * A.gad.pack.ell * 4 * kN;
    const uint32_t ginv = inv_mod_2n_dev((uint32_t)(kN / I + 1));
    pack_split_fwd_body<4, KsSync>(in, shifted(A.w.pkpart, wo), key, I, ginv, A.tabs, A.gad.pack, j, ch, d, smem);
}

__device__ __forceinline__ void fa_pack_inv(const FaArgs& A, int lv, int j, int ch, int comp, uint8_t* smem) {
    const int I = 1 << lv;
    const size_t wo = ws_off(A.bt);
    const bool from_ext = fa_level_reads_ext(A.levels, lv);
    const uint32_t* in = shifted(from_ext ? A.w.ext : A.w.ext2, wo);
    uint32_t* out = shifted(from_ext ? A.w.ext2 : A.w.ext, wo);
    pack_split_inv_body<4, KsSync>(in, shifted(A.w.pkpart, wo), out, I, A.tabs, j, ch, comp, nullptr, smem);
}

// the response words: the packing tree's output (or ext for r = 1) composed
__device__ __forceinline__ void fa_compose(const FaArgs& A) {
    const size_t wo = ws_off(A.bt);
    // after `levels` merges the output sits in ext2 for an odd count, ext for even
    const uint32_t* res = shifted((A.levels & 1) ? A.w.ext2 : A.w.ext, wo);
    uint64_t* resp = A.w.resp64 + (size_t)batch_slot(A.bt) * 2 * kN;
    for (int idx = threadIdx.x; idx < 2 * kN; idx += kNttThreads) {
        const uint32_t* p = res + (size_t)(idx / kN) * 2 * kN;
        const int k = idx % kN;
        resp[idx] = crt_compose_res(__ldcg(p + k), __ldcg(p + kN + k));
    }
}

// counter and target of the dependencies of a task (up to two)
__host__ __device__ __forceinline__ int fa_deps(const FaShape& A, const FaTask& t, int* idx, int* target) {
    const int R = A.R, N2 = kN / 2 / A.N1, L = A.levels;
    const int fc_scan = FC_PER_R, fc_giant = fc_scan + R, fc_ext = fc_giant + R, fc_fwd = fc_ext + R,
              fc_merge = fc_fwd + 2 * R;
    switch (t.type) {
        case FT_PREP: return 0;
        case FT_QNTT: idx[0] = FC_PREP; target[0] = kFaPrepChunks; return 1;
        case FT_ROT1: idx[0] = FC_QNTT; target[0] = A.n_q; return 1;
        case FT_INTER_NTT: idx[0] = FC_INTER_ROT; target[0] = 2; return 1;
        case FT_INTER_DEC: idx[0] = FC_INTER_NTT; target[0] = 2; return 1;
        case FT_DIG1: idx[0] = FC_INTER_DEC; target[0] = kFaPrepChunks; return 1;
        case FT_ROT2: idx[0] = FC_DIG1; target[0] = 9; return 1;
        case FT_GIANT:
            idx[0] = fc_scan + t.b; target[0] = kN;
            idx[1] = FC_ZERO; target[1] = A.ctas;
            return 2;
        case FT_EXT: idx[0] = fc_giant + t.b; target[0] = N2 - 1; return 1;
        case FT_PFWD: {
            const int I = 1 << t.a, j = t.b;
            if (t.a == L - 1) {
                idx[0] = fc_ext + j; target[0] = 2;
                idx[1] = fc_ext + j + I; target[1] = 2;
            } else {
                idx[0] = fc_merge + 2 * I + j; target[0] = 4;
                idx[1] = fc_merge + 3 * I + j; target[1] = 4;
            }
            return 2;
        }
        case FT_PINV: idx[0] = fc_fwd + ((1 << t.a) + t.b) * 2 + t.c; target[0] = 5; return 1;
        case FT_COMPOSE:
            if (L == 0) { idx[0] = fc_ext; target[0] = 2; }
            else { idx[0] = fc_merge + 1; target[0] = 4; }
            return 1;
    }
    return 0;
}

// counter a finished task increments (a second one for the intermediate rotation)
__host__ __device__ __forceinline__ int fa_done(const FaShape& A, const FaTask& t, int* second) {
    const int R = A.R;
    const int fc_scan = FC_PER_R, fc_giant = fc_scan + R, fc_ext = fc_giant + R, fc_fwd = fc_ext + R,
              fc_merge = fc_fwd + 2 * R;
    *second = -1;
    switch (t.type) {
        case FT_PREP: return FC_PREP;
        case FT_QNTT: return FC_QNTT;
        case FT_ROT1:
            if (t.b == A.inter_idx) *second = FC_INTER_ROT;
            return FC_ROT1;
        case FT_INTER_NTT: return FC_INTER_NTT;
        case FT_INTER_DEC: return FC_INTER_DEC;
        case FT_DIG1: return FC_DIG1;
        case FT_ROT2: return FC_ROT2;
        case FT_GIANT: return fc_giant + t.b;
        case FT_EXT: return fc_ext + t.b;
        case FT_PFWD: return fc_fwd + ((1 << t.a) + t.b) * 2 + t.c;
        case FT_PINV: return fc_merge + (1 << t.a) + t.b;
        default: return FC_COMPOSE;
    }
}

__device__ __forceinline__ FaShape fa_shape(const FaArgs& A) {
    return FaShape{A.R, A.N1, A.levels, A.n_q, A.inter_idx, (int)gridDim.x};
}

__device__ __forceinline__ void fa_run(const FaArgs& A, const FaTask& t, uint8_t* smem) {
    switch (t.type) {
        case FT_PREP: query_prep_one(ws_at(A.w, A.bt), A.gad.baby, t.b * kNttThreads + threadIdx.x); break;
        case FT_QNTT: fa_ntt_job<false>(A, A.jobs[A.seg_q + t.b], smem); break;
        case FT_ROT1: fa_rotation(A, A.a1, t.b, t.a, smem); break;
        case FT_INTER_NTT: fa_ntt_job<true>(A, A.jobs[A.seg_inter + t.b], smem); break;
        case FT_INTER_DEC: inter_decomp_one(ws_at(A.w, A.bt), A.gad.baby, t.b * kNttThreads + threadIdx.x); break;
        case FT_DIG1: fa_ntt_job<false>(A, A.jobs[A.seg_dig1 + t.b], smem); break;
        case FT_ROT2: fa_rotation(A, A.a2, t.b, t.a, smem); break;
        case FT_GIANT: fa_giant<2>(A, t.b, t.c, smem); break;
        case FT_EXT: fa_ext(A, t.b, t.a, smem); break;
        case FT_PFWD: fa_pack_fwd(A, t.a, t.b, t.c, t.d, smem); break;
        case FT_PINV: fa_pack_inv(A, t.a, t.b, t.c, t.d, smem); break;
        default: fa_compose(A); break;
    }
}

__device__ __forceinline__ void fa_key_switch_group(const FaArgs& A, uint8_t* smem, int* s_task, int* s_go) {
    const int tid = threadIdx.x;
    if (tid == 0) fa_time_min(A, FT_T_START);
    for (;;) {
        if (tid == 0) {
            const int t = atomicAdd(A.cnt + FC_HEAD, 1);
            int go = 0;
            if (t < A.ntasks && !fa_aborted(A)) {
                const FaTask tk = A.tasks[t];
                int idx[2], target[2];
                const int n = fa_deps(fa_shape(A), tk, idx, target);
                go = 1;
                for (int i = 0; i < n && go; i++) go = fa_wait(A, idx[i], target[i]) ? 1 : 0;
            }
            *s_task = t;
            *s_go = go;
        }
        KsSync::sync();
        const int t = *s_task, go = *s_go;
        if (t >= A.ntasks || !go) break;   // the same for every thread of the group
        const FaTask tk = A.tasks[t];
        fa_run(A, tk, smem);
        KsSync::sync();   // the task's results are written and its shared memory is free
        if (tid == 0) {
            int second;
            const int c = fa_done(fa_shape(A), tk, &second);
            __threadfence();
            atomicAdd(A.cnt + c, 1);
            if (second >= 0) atomicAdd(A.cnt + second, 1);
            if (tk.type == FT_ROT2) fa_time_max(A, FT_T_HEAD);
            else if (tk.type == FT_GIANT) fa_time_max(A, FT_T_GIANT);
            else if (tk.type == FT_EXT) fa_time_max(A, FT_T_EXT);
            else if (tk.type == FT_COMPOSE) fa_time_max(A, FT_T_END);
        }
    }
}

// The scan group: k_scan's producer and consumers over this CTA's items
// it = blockIdx.x + j gridDim.x, item it covering NTT slot it % N of
// sub-database fa_scan_order(it / N).  The producer warp first zeroes this
// CTA's share of the giant-step accumulators; the producer then waits for the
// rotated-query buffer (all N1 columns) before its first copy.
template <int N1, int CONS>
__device__ __forceinline__ void fa_scan_group(const FaArgs& A, uint8_t* ring, uint64_t* full, uint64_t* empty,
                                              int stid) {
    using SC = ScanCfg<N1>;
    constexpr int NST = CONS;
    const int warp = stid >> 5, lane = stid & 31;
    const long total = (long)A.R * kN;
    const long nloc = (total - blockIdx.x + gridDim.x - 1) / gridDim.x;
    const int N1h = N1 / 2;
    if (warp == CONS) {
        const size_t n = (size_t)A.R * 4 * kN, per = (n + gridDim.x - 1) / gridDim.x;
        const size_t lo = (size_t)blockIdx.x * per, hi = lo + per < n ? lo + per : n;
        for (size_t i = lo + lane; i < hi; i += 32) A.acc[i] = 0;
        __syncwarp();
        if (lane == 0) fa_signal(A.cnt + FC_ZERO, 1);
        if (lane != 0) return;
        const bool ok =
            fa_wait(A, FC_QNTT, A.n_q) && fa_wait(A, FC_ROT1, 2 * (N1h - 1)) && fa_wait(A, FC_ROT2, 2 * N1h);
        // the rotations were written by generic stores of other CTAs; the bulk
        // copies below read them through the async proxy
        asm volatile("fence.proxy.async.global;" ::: "memory");
        const uint64_t pol_db = l2_policy_evict_first(), pol_cb = l2_policy_evict_last();
        const uint64_t* cbuf = shifted(A.w.cipherbuf, ws_off(A.bt));
        const long skip_j = blockIdx.x == 0 ? A.skip : -1;
        long issued = 0;
        if (ok) {
            fa_time_min(A, FT_T_SCAN0);
            for (long j = 0; j < nloc; j++) {
                const int s = (int)(j % NST);
                if (j >= NST && !fa_mbar_wait(A, &empty[s], (uint32_t)((j / NST - 1) & 1), 1)) break;
                issued = j + 1;
                if (j == skip_j) continue;   // injected failure: nothing arrives on full[s]
                const long it = blockIdx.x + j * gridDim.x;
                const long r = fa_scan_order((int)(it / kN), A.levels), z = it % kN;
                uint8_t* st = ring + (size_t)s * SC::STAGE;
                mbar_arrive_expect_tx(&full[s], SC::STAGE);
                bulk_g2s_hint(st, A.db + ((size_t)r * kN + z) * (kN / 2), SC::SLAB, &full[s], pol_db);
                bulk_g2s_hint(st + SC::SLAB, cbuf + (size_t)z * 2 * N1, SC::QSLAB, &full[s], pol_cb);
            }
        }
        // never leave the CTA with copies in flight into its shared memory
        const long first = issued > NST ? issued - NST : 0;
        for (long j = first; j < issued; j++)
            if (j != skip_j && !mbar_wait_bounded(&full[j % NST], (uint32_t)((j / NST) & 1), A.limit_ns))
                atomicOr(A.err, 4);
        return;
    }
    // consumers
    uint32_t* sout = shifted(A.w.sout, ws_off(A.bt));
    int cur_r = -1, count = 0;
    for (long j = warp; j < nloc; j += CONS) {
        const long it = blockIdx.x + j * gridDim.x;
        const int r = fa_scan_order((int)(it / kN), A.levels), z = (int)(it % kN);
        if (r != cur_r) {   // this warp is done with sub-database cur_r: publish its items
            if (count) {
                __syncwarp();
                if (lane == 0) fa_signal(A.cnt + FC_PER_R + cur_r, count);
            }
            cur_r = r;
            count = 0;
        }
        const int s = (int)(j % NST);
        if (!fa_mbar_wait(A, &full[s], (uint32_t)((j / NST) & 1), 2)) break;
        uint64_t v[SC::NV];
        scan_item_mac<N1>(ring + (size_t)s * SC::STAGE, lane, v);
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        scan_item_store<N1>(v, lane, r, z, A.R, sout);
        count++;
    }
    if (count) {
        __syncwarp();
        if (lane == 0) {
            fa_signal(A.cnt + FC_PER_R + cur_r, count);
            fa_time_max(A, FT_T_SCAN1);
        }
    }
}

template <int N1, int CONS>
__global__ void __launch_bounds__(FaCfg<N1, CONS>::THREADS, 1) k_answer(const FaArgs A) {
    using F = FaCfg<N1, CONS>;
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ int s_task, s_go;
    uint8_t* ring = smem + kFaKsSmem;
    uint64_t* full = reinterpret_cast<uint64_t*>(ring + F::RING);
    uint64_t* empty = full + F::NST;
    if (threadIdx.x == 0) {
        for (int s = 0; s < F::NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x < kNttThreads) fa_key_switch_group(A, smem, &s_task, &s_go);
    else fa_scan_group<N1, CONS>(A, ring, full, empty, threadIdx.x - kNttThreads);
}

// Before each fused answer: the client of the slot, and zeroed counters and
// timestamps.
__global__ void k_fa_reset(int* client_of, int slot, int client, int* cnt, int words, unsigned long long* times) {
    for (int i = threadIdx.x; i < words; i += blockDim.x) cnt[i] = 0;
    if (threadIdx.x < FT_T_COUNT) times[threadIdx.x] = 0;
    if (threadIdx.x == 0) client_of[slot] = client;
}

}  // namespace kspir
