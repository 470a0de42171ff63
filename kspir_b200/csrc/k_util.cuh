// Generic building blocks: batched transforms driven by job lists, residue
// composition into 64-bit words, and small element-wise helpers.
#pragma once

#include "common.cuh"
#include "ntt.cuh"
#include "pipeline.cuh"
#include "ptx.cuh"

namespace kspir {

// One transform: read N residues from src (stride 1), transform on channel
// `ch`, write to dst[k * dst_stride] (dst may equal src).
struct NttJob {
    const uint32_t* src;
    uint32_t* dst;
    int32_t ch;
    int32_t dst_stride;
};

// dynamic shared memory: 32 KiB twiddles + one padded polynomial
constexpr int kNttJobSmem = kN * 8 + kPadN * 4;

// The transform of one job whose twiddles are staged in tws (the caller
// synchronises nothing: the transform starts with a barrier).
template <bool INVERSE, class Sync>
__device__ __forceinline__ void ntt_job_run(const NttJob& jb, const uint2* tws, uint32_t* s) {
    poly_to_smem(s, jb.src);
    if (INVERSE) cta_ntt_inverse<Sync>(s, tws, jb.ch);
    else cta_ntt_forward<Sync>(s, tws, jb.ch);
    if (jb.dst_stride == 1) {
        poly_from_smem(jb.dst, s);
    } else {
        for (int k = threadIdx.x; k < kN; k += kNttThreads) jb.dst[(size_t)k * jb.dst_stride] = s[pidx(k)];
    }
}

template <bool INVERSE>
__global__ void __launch_bounds__(kNttThreads) k_ntt_jobs(const NttJob* __restrict__ jobs, NttTables tabs, Batch bt) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    uint2* tws = reinterpret_cast<uint2*>(smem_raw);
    uint32_t* s = reinterpret_cast<uint32_t*>(smem_raw + kN * 8);
    pdl_launch_dependents();
    NttJob jb = jobs[blockIdx.x];
    jb.src = shifted(jb.src, ws_off(bt));   // job lists address workspace slot 0
    jb.dst = shifted(jb.dst, ws_off(bt));
    stage_twiddles(tws, tabs, jb.ch, INVERSE ? NTT_INV : NTT_FWD);
    pdl_wait();
    ntt_job_run<INVERSE, CtaSync>(jb, tws, s);
}

// words[p][k] = canonical crtMod value of residues (res[p][0][k], res[p][1][k])
// for `polys` consecutive [2][N] residue polynomials.
__global__ void k_compose_words(const uint32_t* __restrict__ res, uint64_t* __restrict__ words, int polys) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= polys * kN) return;
    int p = idx / kN, k = idx % kN;
    const uint32_t* r = res + (size_t)p * 2 * kN;
    words[idx] = crt_compose_res(r[k], r[kN + k]);
}

// Response words of every query of a batch: resp64 of its slot = canonical
// words of the two residue polynomials `res` (a workspace pointer of slot 0).
__global__ void k_compose_resp(const uint32_t* __restrict__ res, Workspace w, Batch bt) {
    pdl_launch_dependents();
    pdl_wait();
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= 2 * kN) return;
    const uint32_t* r = shifted(res, ws_off(bt)) + (size_t)(idx / kN) * 2 * kN;
    const int k = idx % kN;
    w.resp64[(size_t)batch_slot(bt) * 2 * kN + idx] = crt_compose_res(__ldcg(r + k), __ldcg(r + kN + k));
}

// res[p][ch][k] = words[p][k] mod q_ch (ch = q1, q2) for `polys` polynomials.
__global__ void k_split_words(const uint64_t* __restrict__ words, uint32_t* __restrict__ res, int polys) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= polys * kN) return;
    int p = idx / kN, k = idx % kN;
    uint64_t v = words[idx];
    uint32_t* r = res + (size_t)p * 2 * kN;
    r[k] = mod_q1(v);
    r[kN + k] = mod_q2(v);
}

// Client keys from reference words (layouts of include/kspir_b200.h) into a
// key slot's residues: baby rows 0-2 mod crtMod -> baby_crt (both primes),
// rows 3-5 mod bsMod -> baby_bs; giant, packing and RGSW -> both primes.  The
// words were checked canonical when they were registered.
__global__ void k_keys_from_words(const uint64_t* __restrict__ baby, const uint64_t* __restrict__ giant,
                                  const uint64_t* __restrict__ packing, const uint64_t* __restrict__ rgsw,
                                  uint32_t* __restrict__ baby_crt, uint32_t* __restrict__ baby_bs,
                                  uint32_t* __restrict__ giant_res, uint32_t* __restrict__ packing_res,
                                  uint32_t* __restrict__ rgsw_res, int nbaby, int ngiant, int npack) {
    // polynomial index over [baby: nbaby * 6 * 2][giant: ngiant][packing: npack][rgsw: 8]
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long nb = (long)nbaby * 12, total = nb + ngiant + npack + 8;
    if (idx >= total * kN) return;
    const int k = (int)(idx % kN);
    long p = idx / kN;
    if (p < nb) {
        const long i = p / 12, j = (p / 2) % 6, comp = p % 2;
        const uint64_t v = baby[p * kN + k];
        if (j < 3) {
            uint32_t* d = baby_crt + (((i * 3 + j) * 2 + comp) * 2) * kN;
            d[k] = mod_q1(v);
            d[kN + k] = mod_q2(v);
        } else {
            baby_bs[((i * 3 + j - 3) * 2 + comp) * kN + k] = (uint32_t)v;
        }
        return;
    }
    p -= nb;
    const uint64_t* src;
    uint32_t* dst;
    if (p < ngiant) { src = giant; dst = giant_res; }
    else if ((p -= ngiant) < npack) { src = packing; dst = packing_res; }
    else { p -= npack; src = rgsw; dst = rgsw_res; }
    const uint64_t v = src[p * kN + k];
    dst[(p * 2) * kN + k] = mod_q1(v);
    dst[(p * 2 + 1) * kN + k] = mod_q2(v);
}

// Validation of caller words: flags[0] |= 1 when some word is >= its modulus.
__global__ void k_check_canonical(const uint64_t* __restrict__ words, size_t n, uint64_t modulus,
                                  int* __restrict__ flag) {
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; i < n; i += (size_t)gridDim.x * blockDim.x)
        if (words[i] >= modulus) atomicOr(flag, 1);
}

}  // namespace kspir
