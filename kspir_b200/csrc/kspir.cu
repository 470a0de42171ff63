// kspir_b200: context, device tables, the launch sequence of the online answer,
// and the C ABI of include/kspir_b200.h.  Single translation unit: the kernel
// headers are included here so the __constant__ block is shared without
// relocatable device code.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/kspir_b200.h"
#include "common.cuh"
#include "gadget.cuh"
#include "k_baby.cuh"
#include "k_query.cuh"
#include "k_scan.cuh"
#include "k_second.cuh"
#include "k_util.cuh"
#include "ntt.cuh"
#include "pipeline.cuh"

using namespace kspir;

namespace {

// ---------------------------------------------------------------------------
// host-side number theory

typedef unsigned __int128 hu128;

uint64_t h_powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = (uint64_t)((hu128)r * a % q);
        a = (uint64_t)((hu128)a * a % q);
        e >>= 1;
    }
    return r;
}

uint64_t h_invmod(uint64_t a, uint64_t q) {
    __int128 t = 0, nt = 1, r = q, nr = a % q;
    while (nr) {
        __int128 quo = r / nr, tmp;
        tmp = t - quo * nt; t = nt; nt = tmp;
        tmp = r - quo * nr; r = nr; nr = tmp;
    }
    if (t < 0) t += q;
    return (uint64_t)t;
}

uint32_t h_bitrev12(uint32_t x) {
    uint32_t r = 0;
    for (int i = 0; i < kLogN; i++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

// smallest primitive 2N-th root of unity mod prime q (HEXL MinimalPrimitiveRoot semantics)
uint64_t h_min_root(uint64_t q) {
    uint64_t root = 0;
    for (uint64_t g = 2; g < q; g++) {
        uint64_t c = h_powmod(g, (q - 1) / (2 * kN), q);
        if (h_powmod(c, kN, q) == q - 1) { root = c; break; }
    }
    uint64_t sq = (uint64_t)((hu128)root * root % q), cur = root, best = root;
    for (int i = 0; i < kN; i++) {
        if (cur < best) best = cur;
        cur = (uint64_t)((hu128)cur * sq % q);
    }
    return best;
}

uint32_t shoup32(uint32_t w, uint32_t q) { return (uint32_t)(((uint64_t)w << 32) / q); }

// X -> X^g in the NTT domain: out[j] = in[sigma[j]]
void slot_permutation(uint32_t g, uint16_t* sigma) {
    std::vector<uint32_t> slot_of(kN);
    for (uint32_t j = 0; j < (uint32_t)kN; j++) slot_of[h_bitrev12(j)] = j;   // e = 2*brv(j)+1 -> (e-1)/2 = brv(j)
    for (uint32_t j = 0; j < (uint32_t)kN; j++) {
        uint32_t e = 2 * h_bitrev12(j) + 1;
        uint32_t e2 = (uint32_t)(((uint64_t)g * e) & (2 * kN - 1));
        sigma[j] = (uint16_t)slot_of[(e2 - 1) / 2];
    }
}

uint32_t pow5(uint32_t e) { return (uint32_t)h_powmod(5, e, 2 * kN); }
uint32_t inv_mod_2n(uint32_t g) { return (uint32_t)h_powmod(g, 2047, 2 * kN); }   // group order | 2048

int ilog2i(int v) { int l = 0; while ((1 << l) < v) l++; return l; }

GadgetB make_gadget_b(int ell, uint64_t base, uint64_t bg) {
    GadgetB g;
    g.ell = ell;
    g.base_bits = base ? ilog2i((int)std::min<uint64_t>(base, 1u << 30)) : 0;
    if (base > (1u << 30)) { int b = 0; while ((1ull << b) < base) b++; g.base_bits = b; }
    int gb = 0; while ((1ull << gb) < bg) gb++;
    g.gbits = gb;
    uint64_t off = 0;
    for (int i = 0; i < ell; i++) off += 1ull << (g.base_bits + i * gb);
    off <<= (gb - 1);
    off += base / 2;
    g.offset = off;
    return g;
}

GadgetBsgs make_gadget_bsgs(int ell, uint64_t base, uint64_t bg) {
    GadgetBsgs g;
    g.ell = ell;
    int bb = 0; while (base && (1ull << bb) < base) bb++;
    int gb = 0; while ((1ull << gb) < bg) gb++;
    g.base_bits = bb; g.gbits = gb;
    hu128 off = 0;
    for (int i = 0; i < ell; i++) off += (hu128)1 << (bb + i * gb);
    off <<= (gb - 1);
    off += base / 2;
    g.offset.lo = (uint64_t)off; g.offset.hi = (uint64_t)(off >> 64);
    hu128 M = (hu128)kCrtMod * kBsMod;
    g.M.lo = (uint64_t)M; g.M.hi = (uint64_t)(M >> 64);
    return g;
}

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// ---------------------------------------------------------------------------

struct WsSlot {
    Workspace ws{};
    void* mem = nullptr;
    uint32_t* stage32 = nullptr;   // scratch residues for the staged entry points
    NttJob* jobs = nullptr;        // device job list
    int seg_q = 0, n_q = 0, seg_inter = 0, seg_dig1 = 0;
};

constexpr int kTimingRing = 512;   // per-answer event sets kept for kspir_timing_summary

struct ClientSlot {
    bool loaded = false;
    uint32_t* mem = nullptr;
    ClientKeysDev keys{};
};

}  // namespace

struct kspir_ctx {
    int device = 0;
    kspir_params p{};
    int N1 = 0, N2 = 0, N1h = 0, levels = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    uint64_t* db = nullptr;
    bool db_loaded = false;
    int32_t* perms = nullptr;
    bool perms_loaded = false;
    uint32_t* tw = nullptr;          // [3][4][N]
    uint16_t* sigma_baby = nullptr;  // [N1/2][N]
    uint16_t* sigma_giant = nullptr; // [N2-1][N]
    NttTables ntabs{};
    PathGadgets gad{};
    int nsm = 148;
    std::vector<ClientSlot> clients;
    std::vector<WsSlot> ws;
    // CUDA graphs of the four non-scan phases, per (workspace, client)
    struct PhaseGraphs { bool ready = false; cudaGraphExec_t g[4] = {nullptr, nullptr, nullptr, nullptr}; };
    std::vector<PhaseGraphs> graphs;   // [ws * max_clients + client]
    cudaStream_t capture = nullptr;
    bool use_graphs = true;
    // phase events of recent answers: ring[i][0..5] brackets baby / scan / giant / ext / packing
    std::vector<std::array<cudaEvent_t, 6>> ring;
    long answers = 0;          // answers enqueued since the last kspir_timing_reset
    long launches = 0;         // kernels launched by those answers
    int last_slot = -1;
};

namespace {

thread_local std::string g_thread_err;   // errors without a context (creation)

int set_err(kspir_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    g_thread_err = msg;
    return code;
}

#define KS_CUDA(ctx, call)                                                                   \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess)                                                               \
            return set_err(ctx, e_ == cudaErrorMemoryAllocation ? KSPIR_ERR_OOM : KSPIR_ERR_CUDA, \
                           std::string(#call) + ": " + cudaGetErrorString(e_));              \
    } while (0)

// Every host<->device copy goes through the context's (non-blocking) stream and
// is waited for: a plain cudaMemcpy runs on the legacy stream, which a
// non-blocking stream does not order against, and a pageable host->device
// cudaMemcpy may return before its DMA has landed.
int copy_sync(kspir_ctx* c, void* dst, const void* src, size_t bytes, cudaMemcpyKind kind) {
    KS_CUDA(c, cudaMemcpyAsync(dst, src, bytes, kind, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return KSPIR_OK;
}

#define KS_COPY(ctx, dst, src, bytes, kind)                      \
    do {                                                         \
        int rc_ = copy_sync(ctx, dst, src, bytes, kind);         \
        if (rc_) return rc_;                                     \
    } while (0)

int init_constants(kspir_ctx* c) {
    DevConst dc{};
    const uint32_t qs[3] = {kQ1, kQ2, kBsMod};
    for (int ch = 0; ch < 3; ch++) {
        ChanConst& cc = dc.ch[ch];
        cc.q = qs[ch];
        cc.two_q = 2 * qs[ch];
        cc.barrett = ~0ull / qs[ch];
        cc.ninv = (uint32_t)h_invmod(kN, qs[ch]);
        cc.ninv_p = shoup32(cc.ninv, qs[ch]);
        cc.bsinv = ch < 2 ? (uint32_t)(kBsModInvCrt % qs[ch]) : 0;
        cc.bsinv_p = shoup32(cc.bsinv, qs[ch]);
    }
    dc.q1inv_mod_q2 = (uint32_t)h_invmod(kQ1 % kQ2, kQ2);
    dc.q1inv_mod_q2_p = shoup32(dc.q1inv_mod_q2, kQ2);
    KS_CUDA(c, cudaMemcpyToSymbolAsync(c_dev, &dc, sizeof(dc), 0, cudaMemcpyHostToDevice, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));

    // twiddles: crt channels use root_of_unity_crt (reference crt.h:81) reduced
    // per prime; bsMod uses HEXL's minimal primitive root
    const uint64_t root_crt = 3375402822066082ull;
    const uint64_t roots[3] = {root_crt % kQ1, root_crt % kQ2, h_min_root(kBsMod)};
    // per channel uint2 [2][N]: {psi^brv(k), Shoup} then {psi^-brv(k), Shoup}
    std::vector<uint32_t> tw(3 * 4 * kN);
    for (int ch = 0; ch < 3; ch++) {
        const uint64_t q = qs[ch], psi = roots[ch], pinv = h_invmod(psi, q);
        uint32_t* t = tw.data() + (size_t)ch * 4 * kN;
        for (int k = 0; k < kN; k++) {
            uint32_t e = h_bitrev12(k);
            const uint32_t w = (uint32_t)h_powmod(psi, e, q), iw = (uint32_t)h_powmod(pinv, e, q);
            t[2 * k] = w;
            t[2 * k + 1] = shoup32(w, (uint32_t)q);
            t[2 * kN + 2 * k] = iw;
            t[2 * kN + 2 * k + 1] = shoup32(iw, (uint32_t)q);
        }
    }
    KS_CUDA(c, cudaMalloc(&c->tw, tw.size() * 4));
    KS_COPY(c, c->tw, tw.data(), tw.size() * 4, cudaMemcpyHostToDevice);
    for (int ch = 0; ch < 3; ch++) c->ntabs.tw[ch] = reinterpret_cast<const uint2*>(c->tw + (size_t)ch * 4 * kN);

    std::vector<uint16_t> sb((size_t)c->N1h * kN), sg((size_t)std::max(1, c->N2 - 1) * kN);
    for (int i = 0; i < c->N1h; i++) slot_permutation(pow5(i + 1), sb.data() + (size_t)i * kN);
    for (int cc = 1; cc < c->N2; cc++) slot_permutation(pow5((uint32_t)(c->N1 * cc)), sg.data() + (size_t)(cc - 1) * kN);
    KS_CUDA(c, cudaMalloc(&c->sigma_baby, sb.size() * 2));
    KS_COPY(c, c->sigma_baby, sb.data(), sb.size() * 2, cudaMemcpyHostToDevice);
    KS_CUDA(c, cudaMalloc(&c->sigma_giant, sg.size() * 2));
    KS_COPY(c, c->sigma_giant, sg.data(), sg.size() * 2, cudaMemcpyHostToDevice);

    c->gad.baby = make_gadget_bsgs(3, 1u << 20, 1u << 20);
    c->gad.giant = make_gadget_b(2, 1u << 20, 1u << 18);
    c->gad.ext.ell = 2; c->gad.ext.base_bits = 20; c->gad.ext.gbits = 18;
    c->gad.pack = make_gadget_b(4, 0, 1u << 14);
    return KSPIR_OK;
}

// Carves one workspace out of a single allocation and builds its job lists.
int init_workspace(kspir_ctx* c, WsSlot& s) {
    const int r = c->p.r, N2 = c->N2, N1 = c->N1;
    const size_t P = (size_t)kN * 4;   // bytes of one residue poly
    const int half = std::max(1, r / 2);
    struct Part { void** dst; size_t bytes; };
    Workspace& w = s.ws;
    std::vector<Part> parts = {
        {(void**)&w.q64, 4 * kN * 8},
        {(void**)&w.dig0, 9 * P},
        {(void**)&w.qbn, 2 * P},
        {(void**)&w.qbbs, P},
        {(void**)&w.col0, 4 * P},
        {(void**)&w.interA, 2 * P},
        {(void**)&w.interB, 2 * P},
        {(void**)&w.inter_bs, 2 * P},
        {(void**)&w.inter_acoef, 2 * P},
        {(void**)&w.dig1, 9 * P},
        {(void**)&w.cipherbuf, (size_t)kN * N1 * 2 * 8},
        {(void**)&w.sout, (size_t)r * N2 * 4 * P},
        {(void**)&w.result, (size_t)r * 4 * P},
        {(void**)&w.ecoef, (size_t)r * 4 * P},
        {(void**)&w.ext, (size_t)r * 4 * P},
        {(void**)&w.ext2, (size_t)half * 4 * P},
        {(void**)&w.gacc, (size_t)r * 4 * kN * 8},
        {(void**)&w.resp64, 2 * kN * 8},
        {(void**)&w.err, 256},
        {(void**)&s.stage32, (size_t)r * 4 * P},
    };
    size_t total = 0;
    for (auto& pt : parts) total = align_up(total, 256) + pt.bytes;
    KS_CUDA(c, cudaMalloc(&s.mem, total));
    KS_CUDA(c, cudaMemsetAsync(s.mem, 0, total, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    size_t off = 0;
    for (auto& pt : parts) {
        off = align_up(off, 256);
        *pt.dst = (char*)s.mem + off;
        off += pt.bytes;
    }

    std::vector<NttJob> jobs;
    auto add = [&](const uint32_t* src, uint32_t* dst, int ch, int stride) {
        NttJob j; j.src = src; j.dst = dst; j.ch = ch; j.dst_stride = stride; jobs.push_back(j);
    };
    // query: dig0 (9), query b crt (2), modswitched query -> cipherbuf column 0 (4)
    s.seg_q = (int)jobs.size();
    for (int j = 0; j < 3; j++)
        for (int ch = 0; ch < 3; ch++) add(w.dig0 + (j * 3 + ch) * kN, w.dig0 + (j * 3 + ch) * kN, ch, 1);
    for (int ch = 0; ch < 2; ch++) add(w.qbn + ch * kN, w.qbn + ch * kN, ch, 1);
    uint32_t* cb32 = reinterpret_cast<uint32_t*>(w.cipherbuf);
    for (int comp = 0; comp < 2; comp++)
        for (int ch = 0; ch < 2; ch++)
            add(w.col0 + (comp * 2 + ch) * kN, cb32 + 2 * comp + ch, ch, 4 * N1);
    s.n_q = (int)jobs.size() - s.seg_q;
    s.seg_inter = (int)jobs.size();
    for (int ch = 0; ch < 2; ch++) add(w.interA + ch * kN, w.inter_acoef + ch * kN, ch, 1);
    s.seg_dig1 = (int)jobs.size();
    for (int j = 0; j < 3; j++)
        for (int ch = 0; ch < 3; ch++) add(w.dig1 + (j * 3 + ch) * kN, w.dig1 + (j * 3 + ch) * kN, ch, 1);
    KS_CUDA(c, cudaMalloc(&s.jobs, jobs.size() * sizeof(NttJob)));
    KS_COPY(c, s.jobs, jobs.data(), jobs.size() * sizeof(NttJob), cudaMemcpyHostToDevice);
    return KSPIR_OK;
}

inline int blocks_for(long n, int t) { return (int)((n + t - 1) / t); }

// ---------------------------------------------------------------------------
// launch sequence

// baby steps -> cipherbuf (reference evalAutoSRNSSmallKeys + reorientCipher)
void enqueue_baby(kspir_ctx* c, WsSlot& s, const ClientKeysDev& keys, cudaStream_t st) {
    Workspace& w = s.ws;
    k_query_prep<<<kN / 256, 256, 0, st>>>(w, c->gad.baby);
    k_ntt_jobs<false><<<s.n_q, kNttThreads, kNttJobSmem, st>>>(s.jobs + s.seg_q, c->ntabs);
    BabyArgs a1{};
    a1.dig = w.dig0; a1.srcB = w.qbn; a1.srcBbs = w.qbbs; a1.perms = c->perms; a1.sigma = c->sigma_baby;
    a1.cipherbuf = w.cipherbuf; a1.interA = w.interA; a1.interB = w.interB; a1.inter_bs = w.inter_bs;
    a1.N1 = c->N1; a1.col_base = 1; a1.inter_idx = c->N1h - 2;
    if (c->N1h - 1 > 0) k_baby_rot<3><<<(c->N1h - 1) * 4, kNttThreads, kBabySmem, st>>>(a1, keys, c->ntabs);
    k_ntt_jobs<true><<<2, kNttThreads, kNttJobSmem, st>>>(s.jobs + s.seg_inter, c->ntabs);
    k_inter_decomp<<<kN / 256, 256, 0, st>>>(w, c->gad.baby);
    k_ntt_jobs<false><<<9, kNttThreads, kNttJobSmem, st>>>(s.jobs + s.seg_dig1, c->ntabs);
    BabyArgs a2 = a1;
    a2.dig = w.dig1; a2.srcB = w.interB; a2.srcBbs = w.inter_bs + kN;
    a2.col_base = c->N1h; a2.inter_idx = -1;
    k_baby_rot<3><<<c->N1h * 4, kNttThreads, kBabySmem, st>>>(a2, keys, c->ntabs);
}

void enqueue_scan(kspir_ctx* c, WsSlot& s, cudaStream_t st) {
    Workspace& w = s.ws;
    const int R = c->p.r;
    switch (c->N1) {
#define KS_SCAN(n) \
    case n: k_scan<n><<<c->nsm, ScanCfg<n>::THREADS, ScanCfg<n>::SMEM, st>>>(c->db, w.cipherbuf, w.sout, R, w.err); break;
        KS_SCAN(64) KS_SCAN(128) KS_SCAN(256)
#undef KS_SCAN
    }
}

void enqueue_giant(kspir_ctx* c, WsSlot& s, const ClientKeysDev& keys, cudaStream_t st) {
    Workspace& w = s.ws;
    const int R = c->p.r;
    cudaMemsetAsync(w.gacc, 0, (size_t)R * 4 * kN * 8, st);
    if (c->N2 > 1)
        k_giant_fused<2><<<R * (c->N2 - 1), kNttThreads, kGiantSmem, st>>>(w.sout, keys.giant, c->sigma_giant, w.gacc,
                                                                          c->N1, c->ntabs, c->gad.giant);
    k_giant_finish<<<blocks_for((long)R * 4 * kN, 256), 256, 0, st>>>(w.sout, w.gacc, w.result, R, c->N2);
}

// external products of `count` first-dimension results (result -> ext);
// `init` holds NTT-domain accumulators ([count][2][2][N]) or is null for zero;
// coef_out (or null) receives the first-dimension results in coefficient form
void enqueue_ext(kspir_ctx* c, WsSlot& s, const ClientKeysDev& keys, int count, const uint32_t* init,
                 uint32_t* coef_out, cudaStream_t st) {
    Workspace& w = s.ws;
    k_ext_fused<2><<<count * 2, kNttThreads, kExtSmem, st>>>(w.result, keys.rgsw, init, w.ext, coef_out, c->ntabs,
                                                              c->gad.ext);
}

void enqueue_packing(kspir_ctx* c, WsSlot& s, const ClientKeysDev& keys, cudaStream_t st) {
    Workspace& w = s.ws;
    const int pe = c->gad.pack.ell;
    const uint32_t* cur = w.ext;
    for (int lv = c->levels - 1; lv >= 0; lv--) {
        const int I = 1 << lv;
        const uint32_t ginv = inv_mod_2n((uint32_t)(kN / I + 1));
        uint32_t* out = (cur == w.ext) ? w.ext2 : w.ext;
        k_pack_fused<4><<<I * 2, kNttThreads, kPackSmem, st>>>(cur, out, keys.packing + (size_t)lv * pe * 4 * kN, I,
                                                               ginv, c->ntabs, c->gad.pack);
        cur = out;
    }
    k_compose_words<<<2 * kN / 256, 256, 0, st>>>(cur, w.resp64, 2);
}

// kernels launched by one enqueue_answer
long answer_launches(const kspir_ctx* c) {
    // baby 7, scan 1, giant 2, external product 1, packing one per level + compose
    return 7 + 1 + (c->N2 > 1 ? 2 : 1) + 1 + c->levels + 1;
}

// Captures the four non-scan phases of one (workspace, client) pair as CUDA
// graphs (the scan stays a direct launch so its duration is bracketed by the
// per-answer events).  Pointers are fixed for the context's lifetime, so the
// graphs stay valid when keys or the database are re-uploaded.
int build_graphs(kspir_ctx* c, int wsi, int client) {
    auto& pg = c->graphs[(size_t)wsi * c->p.max_clients + client];
    if (pg.ready) return KSPIR_OK;
    WsSlot& s = c->ws[wsi];
    const ClientKeysDev keys = c->clients[client].keys;
    cudaStream_t cs = c->capture;
    for (int ph = 0; ph < 4; ph++) {
        cudaGraph_t g = nullptr;
        KS_CUDA(c, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        if (ph == 0) enqueue_baby(c, s, keys, cs);
        else if (ph == 1) enqueue_giant(c, s, keys, cs);
        else if (ph == 2) enqueue_ext(c, s, keys, c->p.r, nullptr, nullptr, cs);
        else enqueue_packing(c, s, keys, cs);
        KS_CUDA(c, cudaStreamEndCapture(cs, &g));
        cudaError_t e = cudaGraphInstantiate(&pg.g[ph], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return set_err(c, KSPIR_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    pg.ready = true;
    return KSPIR_OK;
}

int enqueue_answer(kspir_ctx* c, int wsi, int client, cudaStream_t st) {
    WsSlot& s = c->ws[wsi];
    const ClientKeysDev& keys = c->clients[client].keys;
    const int slot = (int)(c->answers % kTimingRing);
    auto& ev = c->ring[slot];
    if (c->use_graphs) {
        int rc = build_graphs(c, wsi, client);
        if (rc) return rc;
        auto& pg = c->graphs[(size_t)wsi * c->p.max_clients + client];
        cudaEventRecord(ev[0], st);
        KS_CUDA(c, cudaGraphLaunch(pg.g[0], st));
        cudaEventRecord(ev[1], st);
        enqueue_scan(c, s, st);
        cudaEventRecord(ev[2], st);
        KS_CUDA(c, cudaGraphLaunch(pg.g[1], st));
        cudaEventRecord(ev[3], st);
        KS_CUDA(c, cudaGraphLaunch(pg.g[2], st));
        cudaEventRecord(ev[4], st);
        KS_CUDA(c, cudaGraphLaunch(pg.g[3], st));
        cudaEventRecord(ev[5], st);
    } else {
        cudaEventRecord(ev[0], st);
        enqueue_baby(c, s, keys, st);
        cudaEventRecord(ev[1], st);
        enqueue_scan(c, s, st);
        cudaEventRecord(ev[2], st);
        enqueue_giant(c, s, keys, st);
        cudaEventRecord(ev[3], st);
        enqueue_ext(c, s, keys, c->p.r, nullptr, nullptr, st);
        cudaEventRecord(ev[4], st);
        enqueue_packing(c, s, keys, st);
        cudaEventRecord(ev[5], st);
    }
    c->answers++;
    c->launches += answer_launches(c);
    c->last_slot = slot;
    return KSPIR_OK;
}

bool canonical(const uint64_t* w, size_t n, uint64_t q) {
    for (size_t i = 0; i < n; i++)
        if (w[i] >= q) return false;
    return true;
}

int check_ready(kspir_ctx* c, int client) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    if (client < 0 || client >= (int)c->clients.size()) return set_err(c, KSPIR_ERR_INVALID_ARG, "client slot out of range");
    if (!c->db_loaded) return set_err(c, KSPIR_ERR_NOT_READY, "database not uploaded");
    if (!c->perms_loaded) return set_err(c, KSPIR_ERR_NOT_READY, "permutations not uploaded");
    if (!c->clients[client].loaded) return set_err(c, KSPIR_ERR_NOT_READY, "client keys not uploaded");
    return KSPIR_OK;
}

int finish(kspir_ctx* c, WsSlot& s) {
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    int herr = 0;
    KS_COPY(c, &herr, s.ws.err, sizeof(int), cudaMemcpyDeviceToHost);
    if (herr) {
        cudaMemsetAsync(s.ws.err, 0, sizeof(int), c->stream);
        cudaStreamSynchronize(c->stream);
        return set_err(c, KSPIR_ERR_TIMEOUT, "a bounded device wait gave up (code " + std::to_string(herr) + ")");
    }
    return KSPIR_OK;
}

}  // namespace

// ===========================================================================
// C ABI

extern "C" {

const char* kspir_strerror(int code) {
    switch (code) {
        case KSPIR_OK: return "ok";
        case KSPIR_ERR_INVALID_ARG: return "invalid argument";
        case KSPIR_ERR_CUDA: return "CUDA error";
        case KSPIR_ERR_NOT_READY: return "database, permutations or keys missing";
        case KSPIR_ERR_OOM: return "out of device memory";
        case KSPIR_ERR_TIMEOUT: return "device-side wait timed out";
        case KSPIR_ERR_BUSY: return "no free slot";
        default: return "unknown error";
    }
}

const char* kspir_last_error(const kspir_ctx* ctx) { return ctx ? ctx->err.c_str() : g_thread_err.c_str(); }

int kspir_ctx_create(int device, const kspir_params* params, kspir_ctx** out) {
    if (!params || !out) return KSPIR_ERR_INVALID_ARG;
    const kspir_params p = *params;
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    if (!pow2(p.r) || p.r > 512 || !pow2(p.N1) || p.N1 < 64 || p.N1 > 256 || p.max_clients < 1 ||
        p.max_inflight < 1)
        return KSPIR_ERR_INVALID_ARG;
    std::unique_ptr<kspir_ctx> c(new kspir_ctx());
    c->device = device;
    c->p = p;
    c->N1 = p.N1;
    c->N1h = p.N1 / 2;
    c->N2 = kN / 2 / p.N1;
    c->levels = ilog2i(p.r);
    KS_CUDA(c.get(), cudaSetDevice(device));
    KS_CUDA(c.get(), cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    KS_CUDA(c.get(), cudaStreamCreateWithFlags(&c->capture, cudaStreamNonBlocking));
    if (const char* e = getenv("KSPIR_NO_GRAPHS")) c->use_graphs = !(e[0] == '1');
    KS_CUDA(c.get(), cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_giant_fused<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGiantSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_ext_fused<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kExtSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_pack_fused<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPackSmem));
#define KS_ATTR(n) \
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_scan<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, ScanCfg<n>::SMEM));
    KS_ATTR(64) KS_ATTR(128) KS_ATTR(256)
#undef KS_ATTR
    int rc = init_constants(c.get());
    if (rc) return rc;
    KS_CUDA(c.get(), cudaMalloc(&c->perms, (size_t)p.N1 * kN * 4));
    c->ring.resize(kTimingRing);
    for (auto& evs : c->ring)
        for (auto& e : evs) KS_CUDA(c.get(), cudaEventCreate(&e));
    c->clients.resize(p.max_clients);
    c->ws.resize(p.max_inflight);
    c->graphs.resize((size_t)p.max_inflight * p.max_clients);
    for (auto& s : c->ws) {
        rc = init_workspace(c.get(), s);
        if (rc) return rc;
    }
    *out = c.release();
    return KSPIR_OK;
}

int kspir_ctx_destroy(kspir_ctx* c) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    for (auto& s : c->ws) {
        cudaFree(s.mem);
        cudaFree(s.jobs);
    }
    for (auto& evs : c->ring)
        for (auto& e : evs) if (e) cudaEventDestroy(e);
    for (auto& pg : c->graphs)
        for (auto& g : pg.g) if (g) cudaGraphExecDestroy(g);
    if (c->capture) cudaStreamDestroy(c->capture);
    for (auto& cl : c->clients) cudaFree(cl.mem);
    cudaFree(c->db);
    cudaFree(c->perms);
    cudaFree(c->tw);
    cudaFree(c->sigma_baby);
    cudaFree(c->sigma_giant);
    cudaStreamDestroy(c->stream);
    delete c;
    return KSPIR_OK;
}

int kspir_db_upload(kspir_ctx* c, const uint64_t* datacrt, size_t words) {
    if (!c || !datacrt) return KSPIR_ERR_INVALID_ARG;
    const size_t need = (size_t)c->p.r * kN * (kN / 2);
    if (words != need) return set_err(c, KSPIR_ERR_INVALID_ARG, "database size must be r*N*N/2 words");
    KS_CUDA(c, cudaSetDevice(c->device));
    if (!c->db) KS_CUDA(c, cudaMalloc(&c->db, need * 8));
    KS_COPY(c, c->db, datacrt, need * 8, cudaMemcpyHostToDevice);
    c->db_loaded = true;
    return KSPIR_OK;
}

int kspir_perms_upload(kspir_ctx* c, const int32_t* perms, size_t count) {
    if (!c || !perms) return KSPIR_ERR_INVALID_ARG;
    if (count != (size_t)c->N1 * kN) return set_err(c, KSPIR_ERR_INVALID_ARG, "permutations must be N1*N entries");
    for (size_t i = 0; i < count; i++)
        if (perms[i] < 0 || perms[i] >= kN) return set_err(c, KSPIR_ERR_INVALID_ARG, "permutation entry out of range");
    KS_CUDA(c, cudaSetDevice(c->device));
    KS_COPY(c, c->perms, perms, count * 4, cudaMemcpyHostToDevice);
    c->perms_loaded = true;
    return KSPIR_OK;
}

int kspir_client_keys_upload(kspir_ctx* c, int client, const uint64_t* baby, const uint64_t* giant,
                             const uint64_t* packing, const uint64_t* rgsw) {
    if (!c || client < 0 || client >= (int)c->clients.size() || !baby || !rgsw) return KSPIR_ERR_INVALID_ARG;
    if (c->N2 > 1 && !giant) return KSPIR_ERR_INVALID_ARG;
    if (c->levels > 0 && !packing) return KSPIR_ERR_INVALID_ARG;
    KS_CUDA(c, cudaSetDevice(c->device));
    const size_t nb_poly = (size_t)c->N1h * 3 * 2;                 // crt rows and bs rows each
    const size_t ng_poly = (size_t)(c->N2 - 1) * 2 * 2;
    const size_t np_poly = (size_t)c->levels * 4 * 2;
    const size_t nr_poly = 4 * 2;
    // split baby rows 0-2 (crtMod) and 3-5 (bsMod)
    std::vector<uint64_t> crt_rows(nb_poly * kN), bs_rows(nb_poly * kN);
    for (int i = 0; i < c->N1h; i++)
        for (int j = 0; j < 6; j++)
            for (int comp = 0; comp < 2; comp++) {
                const uint64_t* src = baby + (((size_t)i * 6 + j) * 2 + comp) * kN;
                uint64_t* dst = (j < 3 ? crt_rows.data() : bs_rows.data()) +
                                (((size_t)i * 3 + (j % 3)) * 2 + comp) * kN;
                memcpy(dst, src, kN * 8);
            }
    if (!canonical(crt_rows.data(), crt_rows.size(), kCrtMod) || !canonical(bs_rows.data(), bs_rows.size(), kBsMod) ||
        (giant && !canonical(giant, ng_poly * kN, kCrtMod)) || (packing && !canonical(packing, np_poly * kN, kCrtMod)) ||
        !canonical(rgsw, nr_poly * kN, kCrtMod))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "key word not canonical");

    ClientSlot& cl = c->clients[client];
    const size_t P = (size_t)kN;   // u32 words per residue poly
    const size_t n_baby_crt = nb_poly * 2 * P, n_baby_bs = nb_poly * P;
    const size_t n_giant = ng_poly * 2 * P, n_pack = np_poly * 2 * P, n_rgsw = nr_poly * 2 * P;
    const size_t total = n_baby_crt + n_baby_bs + n_giant + n_pack + n_rgsw;
    if (!cl.mem) KS_CUDA(c, cudaMalloc(&cl.mem, total * 4));
    uint32_t* base = cl.mem;
    cl.keys.baby_crt = base; base += n_baby_crt;
    cl.keys.baby_bs = base; base += n_baby_bs;
    cl.keys.giant = base; base += n_giant;
    cl.keys.packing = base; base += n_pack;
    cl.keys.rgsw = base;

    const size_t stage_words = std::max({nb_poly, ng_poly, np_poly, nr_poly}) * kN;
    uint64_t* stage = nullptr;
    KS_CUDA(c, cudaMalloc(&stage, stage_words * 8));
    auto split = [&](const uint64_t* h, size_t polys, uint32_t* dst) -> int {
        if (!polys) return KSPIR_OK;
        KS_COPY(c, stage, h, polys * kN * 8, cudaMemcpyHostToDevice);
        k_split_words<<<blocks_for((long)polys * kN, 256), 256, 0, c->stream>>>(stage, dst, (int)polys);
        KS_CUDA(c, cudaStreamSynchronize(c->stream));
        return KSPIR_OK;
    };
    int rc = split(crt_rows.data(), nb_poly, const_cast<uint32_t*>(cl.keys.baby_crt));
    if (!rc) rc = split(giant, ng_poly, const_cast<uint32_t*>(cl.keys.giant));
    if (!rc) rc = split(packing, np_poly, const_cast<uint32_t*>(cl.keys.packing));
    if (!rc) rc = split(rgsw, nr_poly, const_cast<uint32_t*>(cl.keys.rgsw));
    if (!rc) {
        std::vector<uint32_t> bs32(bs_rows.size());
        for (size_t i = 0; i < bs_rows.size(); i++) bs32[i] = (uint32_t)bs_rows[i];
        rc = copy_sync(c, const_cast<uint32_t*>(cl.keys.baby_bs), bs32.data(), bs32.size() * 4,
                       cudaMemcpyHostToDevice);
    }
    cudaFree(stage);
    if (rc) return rc;
    cl.loaded = true;
    return KSPIR_OK;
}

int kspir_answer_device(kspir_ctx* c, int client, const uint64_t* d_query, uint64_t* d_response, void* stream) {
    int rc = check_ready(c, client);
    if (rc) return rc;
    if (!d_query || !d_response) return KSPIR_ERR_INVALID_ARG;
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    WsSlot& s = c->ws[0];
    KS_CUDA(c, cudaSetDevice(c->device));
    KS_CUDA(c, cudaMemcpyAsync(s.ws.q64, d_query, 4 * kN * 8, cudaMemcpyDeviceToDevice, st));
    rc = enqueue_answer(c, 0, client, st);
    if (rc) return rc;
    KS_CUDA(c, cudaMemcpyAsync(d_response, s.ws.resp64, 2 * kN * 8, cudaMemcpyDeviceToDevice, st));
    KS_CUDA(c, cudaGetLastError());
    return KSPIR_OK;
}

int kspir_sync(kspir_ctx* c) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    KS_CUDA(c, cudaDeviceSynchronize());
    return finish(c, c->ws[0]);
}

int kspir_answer(kspir_ctx* c, int client, const uint64_t* query, uint64_t* response) {
    int rc = check_ready(c, client);
    if (rc) return rc;
    if (!query || !response) return KSPIR_ERR_INVALID_ARG;
    if (!canonical(query, 2 * kN, kCrtMod) || !canonical(query + 2 * kN, 2 * kN, kBsMod))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "query word not canonical");
    WsSlot& s = c->ws[0];
    KS_CUDA(c, cudaSetDevice(c->device));
    KS_CUDA(c, cudaMemcpyAsync(s.ws.q64, query, 4 * kN * 8, cudaMemcpyHostToDevice, c->stream));
    rc = enqueue_answer(c, 0, client, c->stream);
    if (rc) return rc;
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(response, s.ws.resp64, 2 * kN * 8, cudaMemcpyDeviceToHost, c->stream));
    return finish(c, s);
}

int kspir_last_timing(kspir_ctx* c, float* total_ms, float* phase_ms) {
    if (!c || c->last_slot < 0) return KSPIR_ERR_NOT_READY;
    auto& ev = c->ring[c->last_slot];
    KS_CUDA(c, cudaEventSynchronize(ev[5]));
    float t = 0;
    KS_CUDA(c, cudaEventElapsedTime(&t, ev[0], ev[5]));
    if (total_ms) *total_ms = t;
    if (phase_ms)
        for (int i = 0; i < 5; i++) KS_CUDA(c, cudaEventElapsedTime(&phase_ms[i], ev[i], ev[i + 1]));
    return KSPIR_OK;
}

int kspir_timing_reset(kspir_ctx* c) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    c->answers = 0;
    c->launches = 0;
    c->last_slot = -1;
    return KSPIR_OK;
}

int kspir_timing_summary(kspir_ctx* c, int* answers, long* launches, float* total_ms, float* phase_ms) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    const int n = (int)std::min<long>(c->answers, kTimingRing);
    float tot = 0, ph[5] = {0, 0, 0, 0, 0};
    for (int k = 0; k < n; k++) {
        auto& ev = c->ring[k];
        KS_CUDA(c, cudaEventSynchronize(ev[5]));
        float t = 0;
        KS_CUDA(c, cudaEventElapsedTime(&t, ev[0], ev[5]));
        tot += t;
        for (int i = 0; i < 5; i++) {
            KS_CUDA(c, cudaEventElapsedTime(&t, ev[i], ev[i + 1]));
            ph[i] += t;
        }
    }
    if (answers) *answers = n;
    if (launches) *launches = c->launches;
    if (total_ms) *total_ms = tot;
    if (phase_ms)
        for (int i = 0; i < 5; i++) phase_ms[i] = ph[i];
    return KSPIR_OK;
}

int kspir_matrix_vector_mul_bsgs_rns_crt_large(kspir_ctx* c, int client, uint64_t* query_inout, uint64_t* result) {
    int rc = check_ready(c, client);
    if (rc) return rc;
    if (!query_inout || !result) return KSPIR_ERR_INVALID_ARG;
    if (!canonical(query_inout, 2 * kN, kCrtMod) || !canonical(query_inout + 2 * kN, 2 * kN, kBsMod))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "query word not canonical");
    WsSlot& s = c->ws[0];
    const ClientKeysDev& keys = c->clients[client].keys;
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    KS_CUDA(c, cudaMemcpyAsync(s.ws.q64, query_inout, 4 * kN * 8, cudaMemcpyHostToDevice, st));
    enqueue_baby(c, s, keys, st);
    enqueue_scan(c, s, st);
    enqueue_giant(c, s, keys, st);
    // result words, and the modswitched query (cipherbuf column 0) back into query1[0]
    uint64_t* words = reinterpret_cast<uint64_t*>(s.stage32);
    k_compose_words<<<blocks_for((long)c->p.r * 2 * kN, 256), 256, 0, st>>>(s.ws.result, words, c->p.r * 2);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(result, words, (size_t)c->p.r * 2 * kN * 8, cudaMemcpyDeviceToHost, st));
    rc = finish(c, s);
    if (rc) return rc;
    std::vector<uint64_t> cb((size_t)kN * c->N1 * 2);
    KS_COPY(c, cb.data(), s.ws.cipherbuf, cb.size() * 8, cudaMemcpyDeviceToHost);
    for (int comp = 0; comp < 2; comp++)
        for (int k = 0; k < kN; k++) {
            const uint64_t wv = cb[(size_t)k * c->N1 * 2 + comp];
            const uint64_t r1 = (uint32_t)wv, r2 = wv >> 32;
            // canonical value with these residues (Garner on the host)
            const uint64_t t = (uint64_t)(((hu128)((r2 + kQ2 - r1 % kQ2) % kQ2) * h_invmod(kQ1, kQ2)) % kQ2);
            query_inout[(size_t)comp * kN + k] = r1 + (uint64_t)kQ1 * t;
        }
    return KSPIR_OK;
}

int kspir_external_product(kspir_ctx* c, int client, uint64_t* result, uint64_t* first_dim, int count) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    if (client < 0 || client >= (int)c->clients.size() || !c->clients[client].loaded)
        return set_err(c, KSPIR_ERR_NOT_READY, "client keys not uploaded");
    if (!result || !first_dim || count < 1 || count > c->p.r) return KSPIR_ERR_INVALID_ARG;
    const size_t n = (size_t)count * 2 * kN;
    if (!canonical(result, n, kCrtMod) || !canonical(first_dim, n, kCrtMod))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "ciphertext word not canonical");
    WsSlot& s = c->ws[0];
    const ClientKeysDev& keys = c->clients[client].keys;
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    uint64_t* words = reinterpret_cast<uint64_t*>(s.stage32);     // r*2*N u64 fit in r*4*N u32
    // first_dim -> ws.result residues; the caller's accumulators (NTT domain) -> ws.sout residues
    KS_CUDA(c, cudaMemcpyAsync(words, first_dim, n * 8, cudaMemcpyHostToDevice, st));
    k_split_words<<<blocks_for((long)n, 256), 256, 0, st>>>(words, s.ws.result, count * 2);
    uint32_t* acc = s.ws.sout;   // r*N2*4*N >= count*4*N residues
    KS_CUDA(c, cudaMemcpyAsync(words, result, n * 8, cudaMemcpyHostToDevice, st));
    k_split_words<<<blocks_for((long)n, 256), 256, 0, st>>>(words, acc, count * 2);
    enqueue_ext(c, s, keys, count, acc, s.ws.ecoef, st);
    k_compose_words<<<blocks_for((long)n, 256), 256, 0, st>>>(s.ws.ext, words, count * 2);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(result, words, n * 8, cudaMemcpyDeviceToHost, st));
    int rc = finish(c, s);
    if (rc) return rc;
    k_compose_words<<<blocks_for((long)n, 256), 256, 0, st>>>(s.ws.ecoef, words, count * 2);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(first_dim, words, n * 8, cudaMemcpyDeviceToHost, st));
    return finish(c, s);
}

int kspir_packing_rlwes(kspir_ctx* c, int client, const uint64_t* rlwes, uint64_t* response) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    if (client < 0 || client >= (int)c->clients.size() || !c->clients[client].loaded)
        return set_err(c, KSPIR_ERR_NOT_READY, "client keys not uploaded");
    if (!rlwes || !response) return KSPIR_ERR_INVALID_ARG;
    const size_t n = (size_t)c->p.r * 2 * kN;
    if (!canonical(rlwes, n, kCrtMod)) return set_err(c, KSPIR_ERR_INVALID_ARG, "ciphertext word not canonical");
    WsSlot& s = c->ws[0];
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    uint64_t* words = reinterpret_cast<uint64_t*>(s.stage32);
    KS_CUDA(c, cudaMemcpyAsync(words, rlwes, n * 8, cudaMemcpyHostToDevice, st));
    k_split_words<<<blocks_for((long)n, 256), 256, 0, st>>>(words, s.ws.ext, c->p.r * 2);
    enqueue_packing(c, s, c->clients[client].keys, st);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(response, s.ws.resp64, 2 * kN * 8, cudaMemcpyDeviceToHost, st));
    return finish(c, s);
}

int kspir_permutation_matrix(int32_t* perms, int N1) {
    if (!perms || N1 < 1 || N1 > kN / 2) return KSPIR_ERR_INVALID_ARG;
    std::vector<uint16_t> row(kN);
    for (int i = 0; i < N1; i++) {
        slot_permutation(pow5((uint32_t)i), row.data());
        for (int k = 0; k < kN; k++) perms[(size_t)i * kN + k] = row[k];
    }
    return KSPIR_OK;
}

int kspir_fetch_stage(kspir_ctx* c, int stage, uint64_t* out, size_t words) {
    if (!c || !out) return KSPIR_ERR_INVALID_ARG;
    WsSlot& s = c->ws[0];
    const int R = c->p.r;
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    KS_CUDA(c, cudaStreamSynchronize(st));
    if (stage == KSPIR_STAGE_CIPHERBUF) {
        const size_t n = (size_t)kN * c->N1 * 2;
        if (words != n) return set_err(c, KSPIR_ERR_INVALID_ARG, "size mismatch");
        KS_COPY(c, out, s.ws.cipherbuf, n * 8, cudaMemcpyDeviceToHost);
        return KSPIR_OK;
    }
    const uint32_t* src = nullptr;
    size_t polys = 0;
    if (stage == KSPIR_STAGE_SCAN) { src = s.ws.sout; polys = (size_t)R * c->N2 * 2; }
    else if (stage == KSPIR_STAGE_RESULT) { src = s.ws.result; polys = (size_t)R * 2; }
    else if (stage == KSPIR_STAGE_EXT) { src = s.ws.ext; polys = (size_t)R * 2; }
    else return set_err(c, KSPIR_ERR_INVALID_ARG, "unknown stage");
    if (words != polys * kN) return set_err(c, KSPIR_ERR_INVALID_ARG, "size mismatch");
    uint64_t* tmp = nullptr;
    KS_CUDA(c, cudaMalloc(&tmp, words * 8));
    k_compose_words<<<blocks_for((long)words, 256), 256, 0, st>>>(src, tmp, (int)polys);
    cudaError_t e = cudaMemcpyAsync(out, tmp, words * 8, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    if (e != cudaSuccess) return set_err(c, KSPIR_ERR_CUDA, cudaGetErrorString(e));
    return KSPIR_OK;
}

}  // extern "C"

// ===========================================================================
// External product without any allocation (kspir_external_product_noalloc).
//
// Some callers cannot call cudaMalloc: a plugin inside a host process that owns
// every byte of device memory through its own pool, code that runs while the
// process must not synchronize the device (cudaMalloc/cudaFree can), or a
// runtime that forbids allocation after start-up.  This entry point gives them
// the external product with no allocation of any kind: its scratch is the
// file-scope array below, which every GPU that loads this library holds until
// the process exits.  The caller passes its inputs and outputs in device
// memory it already owns.

namespace {

constexpr int kNoAllocMaxCount = 16;   // ciphertexts per call
constexpr size_t kNaPoly = kN;         // u32 words per residue polynomial
// per ciphertext: first_dim residues (4), accumulator residues (4), coefficient
// form (4), digits (8), products (4) = 24 polynomials
constexpr size_t kNaPerCt = 24 * kNaPoly;
constexpr size_t kNaJobsWords = (size_t)kNoAllocMaxCount * 12 * sizeof(NttJob) / 4;
constexpr size_t kNaScratchWords = (size_t)kNoAllocMaxCount * kNaPerCt   // per-ciphertext polynomials
                                   + 16 * kNaPoly                         // RGSW residues [4][2][2][N]
                                   + 64                                   // flag words
                                   + kNaJobsWords;                        // transform job list

// Scratch shared by every call on a device; it keeps the previous call's
// contents.  Twiddle tables of the no-allocation path live beside it.
static __device__ __align__(256) uint32_t g_na_scratch[kNaScratchWords];
static __device__ __align__(256) uint32_t g_na_tw[3 * 4 * kN];

struct NaDevice {
    bool ready = false;
    uint32_t* scratch = nullptr;   // device address of g_na_scratch on this device
    uint32_t* tw = nullptr;        // device address of g_na_tw on this device
};
NaDevice g_na[64];
std::mutex g_na_mutex;

// twiddles psi^brv(k), psi^-brv(k) and Shoup companions, computed on the device
__global__ void k_na_twiddles(uint32_t* tw, uint32_t q0, uint32_t q1, uint32_t q2, uint32_t p0, uint32_t p1,
                              uint32_t p2) {
    const int ch = blockIdx.y;
    const uint32_t q = ch == 0 ? q0 : ch == 1 ? q1 : q2;
    const uint32_t psi = ch == 0 ? p0 : ch == 1 ? p1 : p2;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < kN; k += gridDim.x * blockDim.x) {
        uint32_t e = __brev((uint32_t)k) >> (32 - kLogN);
        auto pw = [&](uint32_t x) {
            uint64_t r = 1, b = psi;
            while (x) {
                if (x & 1) r = r * b % q;
                b = b * b % q;
                x >>= 1;
            }
            return (uint32_t)r;
        };
        uint32_t w = pw(e);
        uint32_t iw = pw((2 * kN - e) % (2 * kN));   // psi^(2N) = 1
        uint32_t* t = tw + (size_t)ch * 4 * kN;   // uint2 [2][N]
        t[2 * k] = w;
        t[2 * k + 1] = (uint32_t)(((uint64_t)w << 32) / q);
        t[2 * kN + 2 * k] = iw;
        t[2 * kN + 2 * k + 1] = (uint32_t)(((uint64_t)iw << 32) / q);
    }
}

// job list for count <= kNoAllocMaxCount: inverse transforms of the first
// kNoAllocMaxCount*4 polynomials, then forward transforms of the digits
__global__ void k_na_jobs(NttJob* jobs, uint32_t* fd_res, uint32_t* ecoef, uint32_t* edig) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < kNoAllocMaxCount * 4) {
        jobs[t].src = fd_res + (size_t)t * kN;
        jobs[t].dst = ecoef + (size_t)t * kN;
        jobs[t].ch = t & 1;
        jobs[t].dst_stride = 1;
    } else if (t < kNoAllocMaxCount * 12) {
        const int u = t - kNoAllocMaxCount * 4;
        jobs[t].src = edig + (size_t)u * kN;
        jobs[t].dst = edig + (size_t)u * kN;
        jobs[t].ch = u & 1;
        jobs[t].dst_stride = 1;
    }
}

struct NaLayout {
    uint32_t *fd_res, *acc_res, *ecoef, *edig, *ext, *rgsw, *flag;
    NttJob* jobs;
};

NaLayout na_layout(uint32_t* s) {
    NaLayout L;
    const size_t M = kNoAllocMaxCount;
    L.fd_res = s;
    L.acc_res = L.fd_res + M * 4 * kNaPoly;
    L.ecoef = L.acc_res + M * 4 * kNaPoly;
    L.edig = L.ecoef + M * 4 * kNaPoly;
    L.ext = L.edig + M * 8 * kNaPoly;
    L.rgsw = L.ext + M * 4 * kNaPoly;
    L.flag = L.rgsw + 16 * kNaPoly;
    L.jobs = reinterpret_cast<NttJob*>(L.flag + 64);
    return L;
}

// Once per device, with that device current: constants, twiddles, job list,
// and the device addresses of the static arrays.
int na_setup(int device, cudaStream_t st) {
    NaDevice& d = g_na[device];
    if (d.ready) return KSPIR_OK;
    if (cudaGetSymbolAddress((void**)&d.scratch, g_na_scratch) != cudaSuccess) return KSPIR_ERR_CUDA;
    if (cudaGetSymbolAddress((void**)&d.tw, g_na_tw) != cudaSuccess) return KSPIR_ERR_CUDA;
    DevConst dc{};
    const uint32_t qs[3] = {kQ1, kQ2, kBsMod};
    for (int ch = 0; ch < 3; ch++) {
        ChanConst& cc = dc.ch[ch];
        cc.q = qs[ch];
        cc.two_q = 2 * qs[ch];
        cc.barrett = ~0ull / qs[ch];
        cc.ninv = (uint32_t)h_invmod(kN, qs[ch]);
        cc.ninv_p = shoup32(cc.ninv, qs[ch]);
        cc.bsinv = ch < 2 ? (uint32_t)(kBsModInvCrt % qs[ch]) : 0;
        cc.bsinv_p = shoup32(cc.bsinv, qs[ch]);
    }
    dc.q1inv_mod_q2 = (uint32_t)h_invmod(kQ1 % kQ2, kQ2);
    dc.q1inv_mod_q2_p = shoup32(dc.q1inv_mod_q2, kQ2);
    if (cudaMemcpyToSymbolAsync(c_dev, &dc, sizeof(dc), 0, cudaMemcpyHostToDevice, st) != cudaSuccess)
        return KSPIR_ERR_CUDA;
    const uint64_t root_crt = 3375402822066082ull;
    k_na_twiddles<<<dim3(16, 3), 256, 0, st>>>(d.tw, kQ1, kQ2, kBsMod, (uint32_t)(root_crt % kQ1),
                                              (uint32_t)(root_crt % kQ2), (uint32_t)h_min_root(kBsMod));
    NaLayout L = na_layout(d.scratch);
    k_na_jobs<<<1, kNoAllocMaxCount * 12, 0, st>>>(L.jobs, L.fd_res, L.ecoef, L.edig);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) return KSPIR_ERR_CUDA;
    d.ready = true;
    return KSPIR_OK;
}

}  // namespace

extern "C" int kspir_external_product_noalloc(int device, const uint64_t* d_rgsw, uint64_t* d_result,
                                              uint64_t* d_first_dim, int count, void* stream) {
    if (device < 0 || device >= 64 || !d_rgsw || !d_result || !d_first_dim) return KSPIR_ERR_INVALID_ARG;
    if (count < 1 || count > kNoAllocMaxCount) return KSPIR_ERR_INVALID_ARG;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return KSPIR_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return KSPIR_ERR_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = KSPIR_OK;
    {
        std::lock_guard<std::mutex> lock(g_na_mutex);
        rc = na_setup(device, st);
    }
    if (rc == KSPIR_OK) {
        const NaDevice& d = g_na[device];
        NaLayout L = na_layout(d.scratch);
        NttTables tabs;
        for (int ch = 0; ch < 3; ch++) tabs.tw[ch] = reinterpret_cast<const uint2*>(d.tw + (size_t)ch * 4 * kN);
        GadgetS g;
        g.ell = 2; g.base_bits = 20; g.gbits = 18;   // RGSW of test-pir.cpp:71
        const size_t n = (size_t)count * 2 * kN;
        cudaMemsetAsync(L.flag, 0, 64 * 4, st);   // the flag must start at zero on every call
        k_check_canonical<<<64, 256, 0, st>>>(d_result, n, kCrtMod, (int*)L.flag);
        k_check_canonical<<<64, 256, 0, st>>>(d_first_dim, n, kCrtMod, (int*)L.flag);
        k_check_canonical<<<16, 256, 0, st>>>(d_rgsw, 8 * (size_t)kN, kCrtMod, (int*)L.flag);
        k_split_words<<<blocks_for((long)n, 256), 256, 0, st>>>(d_first_dim, L.fd_res, count * 2);
        k_split_words<<<blocks_for((long)n, 256), 256, 0, st>>>(d_result, L.acc_res, count * 2);
        k_split_words<<<blocks_for(8L * kN, 256), 256, 0, st>>>(d_rgsw, L.rgsw, 8);
        k_ntt_jobs<true><<<count * 4, kNttThreads, kNttJobSmem, st>>>(L.jobs, tabs);
        k_ext_decomp<<<blocks_for((long)count * kN, 256), 256, 0, st>>>(L.ecoef, L.edig, count, g);
        k_ntt_jobs<false><<<count * 8, kNttThreads, kNttJobSmem, st>>>(L.jobs + kNoAllocMaxCount * 4, tabs);
        k_ext_mac_intt<<<count * 4, kNttThreads, kMacSmem, st>>>(L.edig, L.rgsw, L.acc_res, L.ext, 4, tabs);
        int flag = 0;
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(&flag, L.flag, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = KSPIR_ERR_CUDA;
        } else if (flag) {
            rc = KSPIR_ERR_INVALID_ARG;   // outputs left untouched
        } else {
            k_compose_words<<<blocks_for((long)n, 256), 256, 0, st>>>(L.ext, d_result, count * 2);
            k_compose_words<<<blocks_for((long)n, 256), 256, 0, st>>>(L.ecoef, d_first_dim, count * 2);
            if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) rc = KSPIR_ERR_CUDA;
        }
    }
    cudaSetDevice(prev);
    return rc;
}
