// Query-side element-wise kernels of the baby steps.
#pragma once

#include "pipeline.cuh"
#include "ptx.cuh"

namespace kspir {

// Per coefficient k of the caller's query (coefficient form, reference
// encrypt.cpp:488-493):
//  * digits of decompose_bsgs(query a mod crtMod, query a mod bsMod)
//    (evalAutoSRNSFirst, twosteps.cpp:960-968), as residues of q1, q2, bs;
//  * query b as residues (its crt transform feeds the hoisted b terms);
//  * the RNS modswitch of the query itself, (x_crt - x_bs) * bsMod^-1 mod
//    crtMod (twosteps.cpp:1073-1086), as residues before its transform.
// k < N; ws is already the query's workspace slot.
__device__ __forceinline__ void query_prep_one(const Workspace& ws, const GadgetBsgs& g, int k) {
    const uint64_t a_crt = ws.q64[k], b_crt = ws.q64[kN + k];
    const uint32_t a_bs = (uint32_t)ws.q64[2 * kN + k], b_bs = (uint32_t)ws.q64[3 * kN + k];
    int32_t dig[kMaxEll];
    decompose_bsgs(a_crt, a_bs, g, dig);
    for (int j = 0; j < g.ell; j++) {
        ws.dig0[(j * 3 + CH_Q1) * kN + k] = signed_to_res(dig[j], kQ1);
        ws.dig0[(j * 3 + CH_Q2) * kN + k] = signed_to_res(dig[j], kQ2);
        ws.dig0[(j * 3 + CH_BS) * kN + k] = signed_to_res(dig[j], kBsMod);
    }
    const uint32_t bq1 = mod_q1(b_crt), bq2 = mod_q2(b_crt);
    ws.qbn[k] = bq1;
    ws.qbn[kN + k] = bq2;
    ws.qbbs[k] = b_bs;
    const uint32_t aq1 = mod_q1(a_crt), aq2 = mod_q2(a_crt);
    const ChanConst& c1 = c_dev.ch[CH_Q1];
    const ChanConst& c2 = c_dev.ch[CH_Q2];
    ws.col0[0 * kN + k] = shoup_mul(submod(aq1, a_bs, kQ1), c1.bsinv, c1.bsinv_p, kQ1);
    ws.col0[1 * kN + k] = shoup_mul(submod(aq2, a_bs, kQ2), c2.bsinv, c2.bsinv_p, kQ2);
    ws.col0[2 * kN + k] = shoup_mul(submod(bq1, b_bs, kQ1), c1.bsinv, c1.bsinv_p, kQ1);
    ws.col0[3 * kN + k] = shoup_mul(submod(bq2, b_bs, kQ2), c2.bsinv, c2.bsinv_p, kQ2);
}

// Also zeroes the query's giant-step accumulators (acc_words u32 words of
// ws.result, and of ws.ecoef when two_acc): the giant steps of this answer
// add into them.
__global__ void k_query_prep(Workspace ws, GadgetBsgs g, Batch bt, int acc_words, int two_acc) {
    pdl_launch_dependents();
    pdl_wait();
    ws = ws_at(ws, bt);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < kN) query_prep_one(ws, g, k);
    const uint4 z = make_uint4(0, 0, 0, 0);
    for (int i = 4 * k; i < acc_words; i += 4 * kN) {
        *reinterpret_cast<uint4*>(ws.result + i) = z;
        if (two_acc) *reinterpret_cast<uint4*>(ws.ecoef + i) = z;
    }
}

// Digits of the intermediate rotation (evalAutoSRNSSecond, twosteps.cpp:1109-1120):
// decompose_bsgs of its coefficient-form a (crt residues composed to the
// canonical word) and its bsMod part.
__device__ __forceinline__ void inter_decomp_one(const Workspace& ws, const GadgetBsgs& g, int k) {
    const uint64_t a_crt = crt_compose_res(__ldcg(ws.inter_acoef + k), __ldcg(ws.inter_acoef + kN + k));
    const uint32_t a_bs = __ldcg(ws.inter_bs + k);
    int32_t dig[kMaxEll];
    decompose_bsgs(a_crt, a_bs, g, dig);
    for (int j = 0; j < g.ell; j++) {
        ws.dig1[(j * 3 + CH_Q1) * kN + k] = signed_to_res(dig[j], kQ1);
        ws.dig1[(j * 3 + CH_Q2) * kN + k] = signed_to_res(dig[j], kQ2);
        ws.dig1[(j * 3 + CH_BS) * kN + k] = signed_to_res(dig[j], kBsMod);
    }
}

__global__ void k_inter_decomp(Workspace ws, GadgetBsgs g, Batch bt) {
    pdl_launch_dependents();
    pdl_wait();
    ws = ws_at(ws, bt);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < kN) inter_decomp_one(ws, g, k);
}

}  // namespace kspir
