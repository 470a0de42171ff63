// kspir_b200: context, device tables, the launch sequence of the online answer,
// and the C ABI of include/kspir_b200.h.  Single translation unit: the kernel
// headers are included here so the __constant__ block is shared without
// relocatable device code.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/kspir_b200.h"
#include "common.cuh"
#include "gadget.cuh"
#include "k_baby.cuh"
#include "k_client.cuh"
#include "k_db.cuh"
#include "formats.cuh"
#include "k_query.cuh"
#include "k_scan.cuh"
#include "k_scan_mma.cuh"
#include "k_second.cuh"
#include "k_util.cuh"
#include "k_answer.cuh"
#include "k_offline.cuh"
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

// Gather table of the database preprocessing: row R = k N1 + i of the
// rearranged database takes entry G_i[j] of its diagonal row, where
// G_i = query_encode^-1 o perm[i] (reference twosteps.cpp:104-118).
// query_encode[t] = brv((rot_t - 1) / 2) with rot_t = 5^t mod 2N for t < N/2
// and rot_{N-1-t} = -5^t mod 2N (utils.cpp:1473-1512, :1657-1675); perm[i] is
// the slot permutation of X -> X^(5^i) (compute_permutation_matrix,
// utils.cpp:1585-1619).
// query_encode[t] (utils.cpp:1657-1675): brv((rot_t - 1) / 2), rot_t = 5^t mod 2N
// for t < N/2 and rot_{N-1-t} = -5^t mod 2N
std::vector<int32_t> query_encode_table() {
    std::vector<int32_t> qe(kN);
    for (uint32_t t = 0; t < (uint32_t)kN / 2; t++) {
        const uint32_t rot = pow5(t);
        qe[t] = (int32_t)h_bitrev12((rot - 1) / 2);
        qe[kN - 1 - t] = (int32_t)h_bitrev12((2 * kN - rot - 1) / 2);
    }
    return qe;
}

std::vector<uint16_t> db_gather_table(int N1) {
    std::vector<uint16_t> inv_qe(kN), perm(kN), g((size_t)N1 * kN);
    for (uint32_t t = 0; t < (uint32_t)kN / 2; t++) {
        const uint32_t rot = pow5(t);
        inv_qe[h_bitrev12((rot - 1) / 2)] = (uint16_t)t;
        inv_qe[h_bitrev12((2 * kN - rot - 1) / 2)] = (uint16_t)(kN - 1 - t);
    }
    for (int i = 0; i < N1; i++) {
        slot_permutation(pow5((uint32_t)i), perm.data());
        for (int j = 0; j < kN; j++) g[(size_t)i * kN + j] = inv_qe[perm[j]];
    }
    return g;
}
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

constexpr int kTimingRing = 512;   // event sets of recent launches kept for kspir_timing_summary
// workspace slots (and streams) single answers rotate over: answers in
// different slots overlap on the device
#ifndef KSPIR_SINGLE_SLOTS
#define KSPIR_SINGLE_SLOTS 8
#endif
constexpr int kSingleSlots = KSPIR_SINGLE_SLOTS;
constexpr int kMaxBatch = 256;     // queries per launch

struct ClientList {
    int n;
    int id[kMaxBatch];
};

// client_of[slot0 + i] = key slot of query i of a launch (read by the kernels)
__global__ void k_set_clients(int* client_of, int slot0, ClientList cl) {
    const int i = threadIdx.x;
    if (i < cl.n) client_of[slot0 + i] = cl.id[i];
}

// scan-stage residues back to the [row][comp][ch][N] polynomial layout
__global__ void k_unblock_sout(const uint32_t* __restrict__ sout, uint32_t* __restrict__ out, int rows) {
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)rows * 4 * kN) return;
    const int z = (int)(idx % kN), cv = (int)((idx / kN) % 4), row = (int)(idx / (4 * kN));
    out[idx] = sout[sout_idx(row, cv, z, rows)];
}

// database-scan variants (chosen per batch size by kspir_tune_batch)
enum ScanKind { SCAN_CUDA = 0, SCAN_MMA4 = 1, SCAN_MMA8 = 2, SCAN_MMA16 = 3, SCAN_MMA32 = 4, SCAN_KINDS = 5 };
int scan_bt(int kind) { return kind == SCAN_MMA4 ? 4 : kind == SCAN_MMA8 ? 8 : kind == SCAN_MMA16 ? 16 : 32; }

}  // namespace

struct kspir_ctx {
    int device = 0;
    kspir_params p{};
    int N1 = 0, N2 = 0, N1h = 0, levels = 0;
    cudaStream_t stream = nullptr;
    uint64_t* db = nullptr;
    bool db_loaded = false;
    bool mma = false;                 // batched tensor-core scan enabled (N1 = 128, several slots)
    uint16_t* dbg = nullptr;          // gather table of the database preprocessing [N1][N]
    int* dbflag = nullptr;            // its validation word
    // one-sub-database preprocessing calls (kspir_database_*): device raw,
    // rows and datacrt; pinned host staging and the last rows returned
    uint64_t* prep_dev = nullptr;
    uint64_t* prep_host = nullptr;
    bool prep_rows_valid = false;
    // client-side helpers: query_encode [N] int32, the message scaling table [p]
    int32_t* cl_qenc = nullptr;
    uint64_t* cl_dm = nullptr;
    // device buffers of the client calls, kept between calls (grown on
    // demand): a cudaFree per call would synchronise the whole device
    uint8_t* cl_scratch = nullptr;
    size_t cl_scratch_bytes = 0;
    uint8_t* dbop = nullptr;          // its database operand [N][2][G] tiles
    int G = 0;
    uint8_t* qop = nullptr;           // its query operand: launch at slot0 uses qop_at(slot0)
    int32_t* perms = nullptr;
    bool perms_loaded = false;
    uint32_t* tw = nullptr;           // [3][4][N]
    uint16_t* sigma_baby = nullptr;   // [N1/2][N]
    uint16_t* sigma_giant = nullptr;  // [N2-1][N]
    NttTables ntabs{};
    PathGadgets gad{};
    int nsm = 148;
    int scan_ctas = 148;      // CTAs of the single-query scan (KSPIR_SCAN_CTAS, default every SM)
    // workspaces: slot s is slot 0's layout shifted by s * ws_bytes
    void* ws_mem = nullptr;
    size_t ws_bytes = 0;
    Workspace ws0{};
    uint64_t* bq64 = nullptr;         // [slots][4][N] query words
    uint64_t* bresp = nullptr;        // [slots][2][N] response words
    int* errs = nullptr;              // [slots][kErrStride]
    int* errs_host = nullptr;         // pinned copy read back by finish()
    int* client_of = nullptr;         // [slots]
    uint32_t* stage32 = nullptr;      // [r][4][N] residues for the staged entry points
    NttJob* jobs = nullptr;           // transform job lists of slot 0
    int seg_q = 0, seg_q_rm = 0, n_q = 0, seg_inter = 0, seg_dig1 = 0;
    // client keys: key slot k is slot 0's layout shifted by k * key_bytes
    uint32_t* key_mem = nullptr;
    size_t key_bytes = 0;
    ClientKeysDev keys0{};
    std::vector<char> key_loaded;
    // CUDA graphs of the four non-scan phases per (slot0, queries)
    struct PhaseGraphs { cudaGraphExec_t g[4] = {nullptr, nullptr, nullptr, nullptr}; };
    std::map<std::pair<int, int>, PhaseGraphs> graphs;
    cudaStream_t capture = nullptr;
    bool use_graphs = true;
    bool use_pdl = true;              // programmatic dependent launch inside the phases
    std::map<int, int> scan_choice;   // queries per launch -> ScanKind
    int last_kind = 0;                // scan variant of the last answer launch
    // events of recent launches: ring[i][0..5] brackets baby / scan / giant / ext / packing
    std::vector<std::array<cudaEvent_t, 6>> ring;
    std::vector<int> ring_nq;
    long enqueues = 0;        // launches since the last kspir_timing_reset
    long answers = 0;         // queries of those launches
    long launches = 0;        // kernels launched by them
    int last_slot = -1;
    // failure injection of the tests (kspir_debug_scan_fault): the limit of
    // every bounded wait of the database scan, and a local item of CTA 0 whose
    // copy the next CUDA-core scan does not issue (-1: none)
    uint64_t wait_limit_ns = kWaitLimitNs;
    long scan_skip = -1;
    // the fused single answer (k_answer.cuh): task list, counters, giant-step
    // accumulators and per-launch device timestamps ([kTimingRing][8])
    bool fused_ok = false;    // built for this context
    bool fused = false;       // single answers use it
    FaTask* fa_tasks = nullptr;
    int fa_ntasks = 0;
    int* fa_cnt = nullptr;
    uint32_t* fa_acc = nullptr;
    unsigned long long* fa_times = nullptr;
    std::vector<char> ring_fused;
    // single answers rotate over the first single_slots workspace slots, so
    // answers issued on different streams (or by different host threads)
    // overlap; each slot's last answer is marked by slot_done (waited for
    // before reuse).  A host-buffer answer owns its slot (slot_busy) from its
    // enqueue until it has read its response, runs on the slot's stream and
    // waits for host_done outside the mutex; its error word lands in
    // single_errs[slot] (pinned).
    int single_slots = 1;
    int next_single = 0;
    std::vector<cudaEvent_t> slot_done;
    std::vector<cudaEvent_t> host_done;
    std::vector<cudaStream_t> slot_stream;
    std::vector<char> slot_used;
    std::vector<char> slot_busy;
    std::vector<cudaStream_t> slot_last_stream;   // stream of each slot's last answer
    int* single_errs = nullptr;
    std::condition_variable slot_cv;
    std::mutex mu;            // serialises enqueues from several host threads
};

namespace {

thread_local std::string g_thread_err;   // the calling thread's last error text

// Error text is kept per host thread (like errno): several threads may call
// into one context at once.
int set_err(kspir_ctx*, int code, const std::string& msg) {
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

template <class T>
T* host_shift(T* p, size_t off) {
    return p ? reinterpret_cast<T*>(reinterpret_cast<char*>(const_cast<typename std::remove_const<T>::type*>(p)) + off)
             : p;
}

// host copy of ws_at: the buffers of workspace slot s
Workspace ws_host(const kspir_ctx* c, int s) {
    Workspace w = c->ws0;
    const size_t off = (size_t)s * c->ws_bytes;
    w.q64 += (size_t)s * 4 * kN;
    w.resp64 += (size_t)s * 2 * kN;
    w.dig0 = host_shift(w.dig0, off);
    w.qbn = host_shift(w.qbn, off);
    w.qbbs = host_shift(w.qbbs, off);
    w.col0 = host_shift(w.col0, off);
    w.interA = host_shift(w.interA, off);
    w.interB = host_shift(w.interB, off);
    w.inter_bs = host_shift(w.inter_bs, off);
    w.inter_acoef = host_shift(w.inter_acoef, off);
    w.dig1 = host_shift(w.dig1, off);
    w.cipherbuf = host_shift(w.cipherbuf, off);
    w.sout = host_shift(w.sout, off);
    w.result = host_shift(w.result, off);
    w.ecoef = host_shift(w.ecoef, off);
    w.ext = host_shift(w.ext, off);
    w.ext2 = host_shift(w.ext2, off);
    w.pkpart = host_shift(w.pkpart, off);
    w.err += (size_t)s * kErrStride;
    return w;
}

ClientKeysDev keys_host(const kspir_ctx* c, int k) {
    ClientKeysDev d = c->keys0;
    const size_t off = (size_t)k * c->key_bytes;
    d.baby_crt = host_shift(d.baby_crt, off);
    d.baby_bs = host_shift(d.baby_bs, off);
    d.giant = host_shift(d.giant, off);
    d.packing = host_shift(d.packing, off);
    d.rgsw = host_shift(d.rgsw, off);
    return d;
}

Batch batch_of(const kspir_ctx* c, int slot0) {
    Batch b;
    b.ws_bytes = c->ws_bytes;
    b.key_bytes = c->key_bytes;
    b.client_of = c->client_of;
    b.slot0 = slot0;
    return b;
}

// the channel moduli, in Chan order
const uint32_t kChanQ[CH_COUNT] = {kQ1, kQ2, kBsMod, kP, kBsMod, kAuxMod, kAuxMod};
const uint64_t kRootCrt = 3375402822066082ull;     // root_of_unity_crt, crt.h:81
const uint64_t kRootCrtBa = 1486445687605966ull;   // root_of_unity_crt_bamod, crt.h:82

// the transform root psi of each channel: crt channels use root_of_unity_crt
// (reference crt.h:81) reduced per prime; bsMod and p use HEXL's minimal
// primitive root
uint64_t chan_root(int ch) {
    switch (ch) {
        case CH_Q1: return kRootCrt % kQ1;
        case CH_Q2: return kRootCrt % kQ2;
        case CH_BA_BS: return kRootCrtBa % kBsMod;
        case CH_BA_AUX: return kRootCrtBa % kAuxMod;
        default: return h_min_root(kChanQ[ch]);
    }
}

// every per-channel constant of c_dev (also written by the allocation-free set-up)
DevConst make_dev_const() {
    DevConst dc{};
    for (int ch = 0; ch < CH_COUNT; ch++) {
        ChanConst& cc = dc.ch[ch];
        const uint32_t q = kChanQ[ch];
        cc.q = q;
        cc.two_q = 2 * q;
        cc.barrett = ~0ull / q;
        cc.ninv = (uint32_t)h_invmod(kN, q);
        cc.ninv_p = shoup32(cc.ninv, q);
        // the last inverse layer's single twiddle is entry 1 of the inverse
        // table: psi^-brv(1) = psi^-(N/2); folding N^-1 into it saves one
        // multiplication per butterfly of that layer
        const uint64_t iw1 = h_powmod(h_invmod(chan_root(ch), q), h_bitrev12(1), q);
        cc.ninv_w = (uint32_t)(iw1 * cc.ninv % q);
        cc.ninv_w_p = shoup32(cc.ninv_w, q);
        cc.bsinv = ch < 2 ? (uint32_t)(kBsModInvCrt % q) : 0;
        cc.bsinv_p = shoup32(cc.bsinv, q);
    }
    dc.q1inv_mod_q2 = (uint32_t)h_invmod(kQ1 % kQ2, kQ2);
    dc.q1inv_mod_q2_p = shoup32(dc.q1inv_mod_q2, kQ2);
    return dc;
}

int init_constants(kspir_ctx* c) {
    const DevConst dc = make_dev_const();
    KS_CUDA(c, cudaMemcpyToSymbolAsync(c_dev, &dc, sizeof(dc), 0, cudaMemcpyHostToDevice, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));

    // twiddles: crt channels use root_of_unity_crt (reference crt.h:81) reduced
    // per prime; bsMod and p use HEXL's minimal primitive root
    uint64_t roots[CH_COUNT];
    for (int ch = 0; ch < CH_COUNT; ch++) roots[ch] = chan_root(ch);
    // per channel uint2 [2][N]: {psi^brv(k), Shoup} then {psi^-brv(k), Shoup}, k-major order
    std::vector<uint32_t> tw((size_t)CH_COUNT * 4 * kN);
    for (int ch = 0; ch < CH_COUNT; ch++) {
        const uint64_t q = kChanQ[ch], psi = roots[ch], pinv = h_invmod(psi, q);
        uint32_t* t = tw.data() + (size_t)ch * 4 * kN;
        for (int k = 0; k < kN; k++) {
            uint32_t e = h_bitrev12(k);
            const uint32_t w = (uint32_t)h_powmod(psi, e, q), iw = (uint32_t)h_powmod(pinv, e, q);
            const int pos = tw_layout_pos(k);   // the transforms read the k-major layout
            t[2 * pos] = w;
            t[2 * pos + 1] = shoup32(w, (uint32_t)q);
            t[2 * kN + 2 * pos] = iw;
            t[2 * kN + 2 * pos + 1] = shoup32(iw, (uint32_t)q);
        }
    }
    KS_CUDA(c, cudaMalloc(&c->tw, tw.size() * 4));
    KS_COPY(c, c->tw, tw.data(), tw.size() * 4, cudaMemcpyHostToDevice);
    for (int ch = 0; ch < CH_COUNT; ch++) c->ntabs.tw[ch] = reinterpret_cast<const uint2*>(c->tw + (size_t)ch * 4 * kN);

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

// Carves the workspace slots (slot 0's layout repeated at ws_bytes) and the
// slot-indexed arrays, and builds slot 0's transform job lists.
int init_workspaces(kspir_ctx* c) {
    const int r = c->p.r, N2 = c->N2, N1 = c->N1, S = c->p.max_inflight;
    const size_t P = (size_t)kN * 4;   // bytes of one residue poly
    const int half = std::max(1, r / 2);
    struct Part { void** dst; size_t bytes; };
    Workspace& w = c->ws0;
    std::vector<Part> parts = {
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
        {(void**)&w.pkpart, (size_t)half * kPackPartPolys * P},
    };
    size_t total = 0;
    for (auto& pt : parts) total = align_up(total, 256) + pt.bytes;
    c->ws_bytes = align_up(total, 4096);
    KS_CUDA(c, cudaMalloc(&c->ws_mem, c->ws_bytes * S));
    KS_CUDA(c, cudaMemsetAsync(c->ws_mem, 0, c->ws_bytes * S, c->stream));
    size_t off = 0;
    for (auto& pt : parts) {
        off = align_up(off, 256);
        *pt.dst = (char*)c->ws_mem + off;
        off += pt.bytes;
    }
    KS_CUDA(c, cudaMalloc(&c->bq64, (size_t)S * 4 * kN * 8));
    KS_CUDA(c, cudaMalloc(&c->bresp, (size_t)S * 2 * kN * 8));
    KS_CUDA(c, cudaMalloc(&c->errs, (size_t)S * kErrStride * 4));
    KS_CUDA(c, cudaMemsetAsync(c->errs, 0, (size_t)S * kErrStride * 4, c->stream));
    KS_CUDA(c, cudaHostAlloc(&c->errs_host, (size_t)S * kErrStride * 4, cudaHostAllocDefault));
    KS_CUDA(c, cudaMalloc(&c->client_of, (size_t)S * 4));
    KS_CUDA(c, cudaMemsetAsync(c->client_of, 0, (size_t)S * 4, c->stream));
    KS_CUDA(c, cudaMalloc(&c->stage32, (size_t)r * 4 * P));
    w.q64 = c->bq64;
    w.resp64 = c->bresp;
    w.err = c->errs;

    std::vector<NttJob> jobs;
    auto add = [&](const uint32_t* src, uint32_t* dst, int ch, int stride) {
        NttJob j; j.src = src; j.dst = dst; j.ch = ch; j.dst_stride = stride; jobs.push_back(j);
    };
    // query: dig0 (9), query b crt (2), modswitched query -> cipherbuf column 0 (4);
    // a second copy writes column 0 of the rotation-major cipherbuf
    uint32_t* cb32 = reinterpret_cast<uint32_t*>(w.cipherbuf);
    for (int rm = 0; rm < 2; rm++) {
        (rm ? c->seg_q_rm : c->seg_q) = (int)jobs.size();
        for (int j = 0; j < 3; j++)
            for (int ch = 0; ch < 3; ch++) add(w.dig0 + (j * 3 + ch) * kN, w.dig0 + (j * 3 + ch) * kN, ch, 1);
        for (int ch = 0; ch < 2; ch++) add(w.qbn + ch * kN, w.qbn + ch * kN, ch, 1);
        for (int comp = 0; comp < 2; comp++)
            for (int ch = 0; ch < 2; ch++) {
                if (rm) add(w.col0 + (comp * 2 + ch) * kN, cb32 + cipherbuf_rm_idx(0, comp, ch, 0), ch, 1);
                else add(w.col0 + (comp * 2 + ch) * kN, cb32 + 2 * comp + ch, ch, 4 * N1);
            }
        c->n_q = (int)jobs.size() - (rm ? c->seg_q_rm : c->seg_q);
    }
    c->seg_inter = (int)jobs.size();
    for (int ch = 0; ch < 2; ch++) add(w.interA + ch * kN, w.inter_acoef + ch * kN, ch, 1);
    c->seg_dig1 = (int)jobs.size();
    for (int j = 0; j < 3; j++)
        for (int ch = 0; ch < 3; ch++) add(w.dig1 + (j * 3 + ch) * kN, w.dig1 + (j * 3 + ch) * kN, ch, 1);
    KS_CUDA(c, cudaMalloc(&c->jobs, jobs.size() * sizeof(NttJob)));
    KS_COPY(c, c->jobs, jobs.data(), jobs.size() * sizeof(NttJob), cudaMemcpyHostToDevice);
    return KSPIR_OK;
}

// Key slot layout (u32 residue words) and the single allocation of all slots.
int init_key_slots(kspir_ctx* c) {
    const size_t P = (size_t)kN;
    const size_t nb_poly = (size_t)c->N1h * 3 * 2;
    const size_t ng_poly = (size_t)std::max(0, c->N2 - 1) * 2 * 2;
    const size_t np_poly = (size_t)c->levels * 4 * 2;
    const size_t nr_poly = 4 * 2;
    const size_t n_baby_crt = nb_poly * 2 * P, n_baby_bs = nb_poly * P;
    const size_t n_giant = ng_poly * 2 * P, n_pack = np_poly * 2 * P, n_rgsw = nr_poly * 2 * P;
    const size_t words = n_baby_crt + n_baby_bs + n_giant + n_pack + n_rgsw;
    c->key_bytes = align_up(words * 4, 4096);
    KS_CUDA(c, cudaMalloc(&c->key_mem, c->key_bytes * c->p.max_clients));
    uint32_t* base = c->key_mem;
    c->keys0.baby_crt = base; base += n_baby_crt;
    c->keys0.baby_bs = base; base += n_baby_bs;
    c->keys0.giant = base; base += n_giant;
    c->keys0.packing = base; base += n_pack;
    c->keys0.rgsw = base;
    c->key_loaded.assign(c->p.max_clients, 0);
    return KSPIR_OK;
}

inline int blocks_for(long n, int t) { return (int)((n + t - 1) / t); }

constexpr int kPackSplitMaxBatch = 4;   // batches up to this size pack with the split (latency) kernels

// ---------------------------------------------------------------------------
// launch sequence of `nq` queries in workspace slots slot0 .. slot0 + nq - 1
// (blockIdx.y of every kernel is the query)

// baby steps -> cipherbuf (reference evalAutoSRNSSmallKeys + reorientCipher)
// Launches a kernel of an answer phase.  With pdl (and c->use_pdl) the launch
// carries the programmatic-serialization attribute: the kernel may start
// while the previous one in the stream finishes, stage its twiddles, and wait
// in pdl_wait() (every phase kernel calls it) for the data.  Measured on a
// single answer: the packing levels gain 7 us (0.101 -> 0.094 ms), while the
// baby and giant steps lose 2-3 us and batches of 8 and 64 lose 4-6 %, so only
// the packing of small batches uses it.
template <typename... KArgs, typename... Args>
void launch(const kspir_ctx* c, bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
            cudaStream_t st, Args... args) {
    if (!pdl || !c->use_pdl) {
        kern<<<grid, block, smem, st>>>(args...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

// the giant steps of a sub-database need a second u32 accumulator
bool giant_two_acc(const kspir_ctx* c) { return c->N2 - 1 > kGiantTermsPerAcc; }

// rm: write the cipherbuf rotation-major (the tensor-core scans read that one)
void enqueue_baby(kspir_ctx* c, int slot0, int nq, bool rm, cudaStream_t st) {
    const Workspace& w = c->ws0;
    const Batch bt = batch_of(c, slot0);
    launch(c, false, k_query_prep, dim3(kN / 256, nq), 256, 0, st, w, c->gad.baby, bt, c->p.r * 4 * kN,
           giant_two_acc(c) ? 1 : 0);
    launch(c, false, k_ntt_jobs<false>, dim3(c->n_q, nq), kNttThreads, kNttJobSmem, st,
           (const NttJob*)(c->jobs + (rm ? c->seg_q_rm : c->seg_q)), c->ntabs, bt);
    BabyArgs a1{};
    a1.cb_rm = rm ? 1 : 0;
    a1.dig = w.dig0; a1.srcB = w.qbn; a1.srcBbs = w.qbbs; a1.perms = c->perms; a1.sigma = c->sigma_baby;
    a1.cipherbuf = w.cipherbuf; a1.interA = w.interA; a1.interB = w.interB; a1.inter_bs = w.inter_bs;
    a1.N1 = c->N1; a1.col_base = 1; a1.inter_idx = c->N1h - 2;
    // one CTA per (rotation, component), also for a single query: with the
    // minimum-form reductions its six transforms per rotation beat the
    // four-CTA shape (eight transforms) on one answer (0.399 against
    // 0.403 ms) and on overlapped answers (0.229 against 0.235 ms)
    auto rot = [&](const BabyArgs& args, int nrot) {
        if (nrot <= 0) return;
        launch(c, false, k_baby_pair<3, 2>, dim3(nrot * 2, nq), kNttThreads, kBabyPairSmem, st, args, c->keys0, c->ntabs,
               bt);
    };
    rot(a1, c->N1h - 1);
    launch(c, false, k_ntt_jobs<true>, dim3(2, nq), kNttThreads, kNttJobSmem, st, (const NttJob*)(c->jobs + c->seg_inter),
           c->ntabs, bt);
    launch(c, false, k_inter_decomp, dim3(kN / 256, nq), 256, 0, st, w, c->gad.baby, bt);
    launch(c, false, k_ntt_jobs<false>, dim3(9, nq), kNttThreads, kNttJobSmem, st, (const NttJob*)(c->jobs + c->seg_dig1),
           c->ntabs, bt);
    BabyArgs a2 = a1;
    a2.dig = w.dig1; a2.srcB = w.interB; a2.srcBbs = w.inter_bs + kN;
    a2.col_base = c->N1h; a2.inter_idx = -1;
    rot(a2, c->N1h);
}

int scan_kind_for(kspir_ctx* c, int nq) {
    if (!c->mma) return SCAN_CUDA;
    auto it = c->scan_choice.find(nq);
    if (it != c->scan_choice.end()) return it->second;
    if (nq == 1) return SCAN_CUDA;
    return nq >= 16 ? SCAN_MMA16 : nq >= 8 ? SCAN_MMA8 : SCAN_MMA4;
}

long scan_launches(const kspir_ctx* c, int kind, int nq) { return kind == SCAN_CUDA ? nq : 2; }

// Query-operand region of a launch starting at workspace slot slot0: 8 MiB per
// slot, so launches on disjoint 32-aligned slot ranges (serving lanes) never
// share it.
uint8_t* qop_at(kspir_ctx* c, int slot0) { return c->qop + (size_t)slot0 * kN * 2 * 8 * kMmaK; }

template <int BT>
void launch_scan_mma(kspir_ctx* c, int slot0, int nq, cudaStream_t st) {
    using C = MmaCfg<BT>;
    const int QT = (nq + BT - 1) / BT;
    uint8_t* qop = qop_at(c, slot0);
    // the baby steps wrote this launch's cipherbufs rotation-major
    k_qop_split_rm<BT><<<dim3(kN / kSplitZ, QT * BT), kSplitThreads, kSplitSmem, st>>>(
        reinterpret_cast<const uint32_t*>(c->ws0.cipherbuf), c->ws_bytes, slot0, nq, QT, qop);
    ScanMmaArgs a;
    a.dbop = c->dbop;
    a.qop = qop;
    a.sout0 = c->ws0.sout;
    a.ws_bytes = c->ws_bytes;
    a.slot0 = slot0;
    a.nq = nq;
    a.QT = QT;
    a.G = c->G;
    a.rows = c->p.r * c->N2;
    a.err = c->errs + (size_t)slot0 * kErrStride;
    const int units = (kN / C::ZB) * 2 * QT;
    k_scan_mma<BT><<<std::min(c->nsm, units), C::THREADS, C::SMEM, st>>>(a);
}

// `share`: another single answer runs beside this one, so the CUDA-core scan
// takes the ring shape that leaves room for that answer's key-switch CTAs.
void enqueue_scan(kspir_ctx* c, int slot0, int nq, int kind, cudaStream_t st, bool share = false) {
    const int R = c->p.r;
    if (kind == SCAN_CUDA) {
        for (int q = 0; q < nq; q++) {
            const Workspace w = ws_host(c, slot0 + q);
            switch (c->N1) {
#define KS_SCAN(n)                                                                                           \
    case n:                                                                                                  \
        if (share) {                                                                                         \
            using SC = typename ScanShare<n>::Cfg;                                                           \
            k_scan<n, SC::CONS, SC::NST><<<c->scan_ctas, SC::THREADS, SC::SMEM, st>>>(                        \
                c->db, w.cipherbuf, w.sout, R, w.err, c->wait_limit_ns, c->scan_skip);                        \
        } else {                                                                                             \
            k_scan<n><<<c->scan_ctas, ScanCfg<n>::THREADS, ScanCfg<n>::SMEM, st>>>(                          \
                c->db, w.cipherbuf, w.sout, R, w.err, c->wait_limit_ns, c->scan_skip);                        \
        }                                                                                                    \
        break;
                KS_SCAN(64) KS_SCAN(128) KS_SCAN(256)
#undef KS_SCAN
            }
            c->scan_skip = -1;   // an injected failure applies to one scan launch
        }
        return;
    }
    switch (scan_bt(kind)) {
        case 4: launch_scan_mma<4>(c, slot0, nq, st); break;
        case 8: launch_scan_mma<8>(c, slot0, nq, st); break;
        case 16: launch_scan_mma<16>(c, slot0, nq, st); break;
        default: launch_scan_mma<32>(c, slot0, nq, st); break;
    }
}

// The giant steps add into result (and, past kGiantTermsPerAcc steps per
// sub-database, ecoef as the second accumulator), which the answer's
// k_query_prep (enqueue_baby) has zeroed.
void enqueue_giant(kspir_ctx* c, int slot0, int nq, cudaStream_t st) {
    const Workspace& w = c->ws0;
    const Batch bt = batch_of(c, slot0);
    const int R = c->p.r;
    uint32_t* acc1 = giant_two_acc(c) ? w.ecoef : nullptr;
    if (c->N2 > 1)
        launch(c, false, k_giant_fused<2>, dim3(R * (c->N2 - 1), nq), kNttThreads, kGiantSmem, st,
               (const uint32_t*)w.sout, w.result, acc1, (const uint32_t*)c->keys0.giant,
               (const uint16_t*)c->sigma_giant, c->N1, c->ntabs, c->gad.giant, R, bt);
    launch(c, false, k_giant_finish, dim3(blocks_for((long)R * 4 * (kN / 4), 256), nq), 256, 0, st, (const uint32_t*)w.sout,
           w.result, (const uint32_t*)acc1, R, c->N2, bt);
}

// external products of `count` first-dimension results (result -> ext);
// `init` holds NTT-domain accumulators ([count][2][2][N], slot-0 workspace
// address) or is null for zero; coef_out (or null) receives the
// first-dimension results in coefficient form
void enqueue_ext(kspir_ctx* c, int slot0, int nq, int count, const uint32_t* init, uint32_t* coef_out,
                 cudaStream_t st) {
    const Workspace& w = c->ws0;
    launch(c, false, k_ext_fused<2>, dim3(count * 2, nq), kNttThreads, kExtSmem, st, (const uint32_t*)w.result,
           (const uint32_t*)c->keys0.rgsw, init, w.ext, coef_out, c->ntabs, c->gad.ext, batch_of(c, slot0));
}

// c2out (or null; split kernels only): receives each merge's X^I c + r, the
// words the reference's packingRLWEs leaves in rlwes[I + j]
void enqueue_packing(kspir_ctx* c, int slot0, int nq, cudaStream_t st, uint32_t* c2out = nullptr) {
    const Workspace& w = c->ws0;
    const Batch bt = batch_of(c, slot0);
    const int pe = c->gad.pack.ell;
    const uint32_t* cur = w.ext;
    for (int lv = c->levels - 1; lv >= 0; lv--) {
        const int I = 1 << lv;
        const uint32_t ginv = inv_mod_2n((uint32_t)(kN / I + 1));
        uint32_t* out = (cur == w.ext) ? w.ext2 : w.ext;
        const uint32_t* key = c->keys0.packing + (size_t)lv * pe * 4 * kN;
        if (nq <= kPackSplitMaxBatch) {   // latency: one transform per CTA
            launch(c, true, k_pack_split_fwd<4>, dim3(I * 2 * 5, nq), kNttThreads, kPackSplitSmem, st, cur, w.pkpart, key, I,
                   ginv, c->ntabs, c->gad.pack, bt);
            launch(c, true, k_pack_split_inv<4>, dim3(I * 4, nq), kNttThreads, kPackSplitSmem, st, cur,
                   (const uint32_t*)w.pkpart, out, I, c->ntabs, bt, c2out);
        } else {                          // throughput: the whole level per CTA pair
            launch(c, false, k_pack_fused<4>, dim3(I * 2, nq), kNttThreads, kPackSmem, st, cur, out, key, I, ginv, c->ntabs,
                   c->gad.pack, bt);
        }
        cur = out;
    }
    launch(c, nq <= kPackSplitMaxBatch, k_compose_resp, dim3(2 * kN / 256, nq), 256, 0, st, cur, w, bt);
}

// kernels launched by one enqueue_answer
long answer_launches(const kspir_ctx* c, int kind, int nq) {
    // clients 1, baby 7, scan, giant 2, external product 1, packing one or two per level + compose
    const int per_level = nq <= kPackSplitMaxBatch ? 2 : 1;
    return 1 + 7 + scan_launches(c, kind, nq) + (c->N2 > 1 ? 2 : 1) + 1 + per_level * c->levels + 1;
}

// Captures the four non-scan phases of (slot0, nq) as CUDA graphs (the scan
// stays a direct launch so its duration is bracketed by the per-launch
// events).  Pointers are fixed for the context's lifetime and the key slot of
// each query is read from client_of at run time, so the graphs stay valid for
// any clients and across key or database uploads.
int build_graphs(kspir_ctx* c, int slot0, int nq, bool rm, kspir_ctx::PhaseGraphs** out) {
    auto key = std::make_pair(slot0, nq * 2 + (rm ? 1 : 0));
    auto it = c->graphs.find(key);
    if (it != c->graphs.end()) { *out = &it->second; return KSPIR_OK; }
    kspir_ctx::PhaseGraphs pg;
    cudaStream_t cs = c->capture;
    for (int ph = 0; ph < 4; ph++) {
        cudaGraph_t g = nullptr;
        KS_CUDA(c, cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        if (ph == 0) enqueue_baby(c, slot0, nq, rm, cs);
        else if (ph == 1) enqueue_giant(c, slot0, nq, cs);
        else if (ph == 2) enqueue_ext(c, slot0, nq, c->p.r, nullptr, nullptr, cs);
        else enqueue_packing(c, slot0, nq, cs);
        KS_CUDA(c, cudaStreamEndCapture(cs, &g));
        cudaError_t e = cudaGraphInstantiate(&pg.g[ph], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return set_err(c, KSPIR_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    }
    auto res = c->graphs.emplace(key, pg);
    *out = &res.first->second;
    return KSPIR_OK;
}

// The fused single answer of workspace slot 0 (k_answer.cuh): reset of its
// counters, then one cooperative launch of one CTA per SM.
FaArgs fa_args(const kspir_ctx* c, int ring_slot) {
    FaArgs A{};
    const Workspace& w = c->ws0;
    A.w = w;
    A.keys = c->keys0;
    A.bt = batch_of(c, 0);
    A.tabs = c->ntabs;
    A.gad = c->gad;
    BabyArgs a1{};
    a1.cb_rm = 0;
    a1.dig = w.dig0; a1.srcB = w.qbn; a1.srcBbs = w.qbbs; a1.perms = c->perms; a1.sigma = c->sigma_baby;
    a1.cipherbuf = w.cipherbuf; a1.interA = w.interA; a1.interB = w.interB; a1.inter_bs = w.inter_bs;
    a1.N1 = c->N1; a1.col_base = 1; a1.inter_idx = c->N1h - 2;
    BabyArgs a2 = a1;
    a2.dig = w.dig1; a2.srcB = w.interB; a2.srcBbs = w.inter_bs + kN;
    a2.col_base = c->N1h; a2.inter_idx = -1;
    A.a1 = a1;
    A.a2 = a2;
    A.jobs = c->jobs;
    A.seg_q = c->seg_q;
    A.n_q = c->n_q;
    A.seg_inter = c->seg_inter;
    A.seg_dig1 = c->seg_dig1;
    A.inter_idx = c->N1h - 2;
    A.sigma_giant = c->sigma_giant;
    A.db = c->db;
    A.R = c->p.r;
    A.N1 = c->N1;
    A.levels = c->levels;
    A.tasks = c->fa_tasks;
    A.ntasks = c->fa_ntasks;
    A.cnt = c->fa_cnt;
    A.acc = c->fa_acc;
    A.times = c->fa_times + (size_t)ring_slot * FT_T_COUNT;
    A.limit_ns = c->wait_limit_ns;
    A.skip = c->scan_skip;
    A.err = c->errs;
    return A;
}

constexpr int kFaScanWarps = 6;

int enqueue_fused(kspir_ctx* c, int client, cudaStream_t st, int ring_slot) {
    k_fa_reset<<<1, 256, 0, st>>>(c->client_of, 0, client, c->fa_cnt, fa_counter_words(c->p.r),
                                  c->fa_times + (size_t)ring_slot * FT_T_COUNT);
    const FaArgs A = fa_args(c, ring_slot);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(c->nsm);
    cfg.blockDim = dim3(FaCfg<128, kFaScanWarps>::THREADS);
    cfg.dynamicSmemBytes = FaCfg<128, kFaScanWarps>::SMEM;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    KS_CUDA(c, cudaLaunchKernelEx(&cfg, k_answer<128, kFaScanWarps>, A));
    c->scan_skip = -1;   // an injected failure applies to one launch
    return KSPIR_OK;
}

// allow_fused: a single answer of slot 0 through the public single-answer
// calls may run as the fused kernel (batches and serving lanes never do)
int enqueue_answer(kspir_ctx* c, int slot0, int nq, const int* clients, cudaStream_t st, bool allow_fused = false,
                   bool share = false) {
    const int slot = (int)(c->enqueues % kTimingRing);
    auto& ev = c->ring[slot];
    if (allow_fused && c->fused && nq == 1 && slot0 == 0) {
        c->last_kind = SCAN_CUDA;
        cudaEventRecord(ev[0], st);
        int rc = enqueue_fused(c, clients[0], st, slot);
        if (rc) return rc;
        for (int i = 1; i < 6; i++) cudaEventRecord(ev[i], st);
        c->ring_nq[slot] = 1;
        c->ring_fused[slot] = 1;
        c->enqueues++;
        c->answers += 1;
        c->launches += 2;
        c->last_slot = slot;
        return KSPIR_OK;
    }
    c->ring_fused[slot] = 0;
    ClientList cl;
    cl.n = nq;
    for (int i = 0; i < nq; i++) cl.id[i] = clients[i];
    k_set_clients<<<1, kMaxBatch, 0, st>>>(c->client_of, slot0, cl);
    const int kind = scan_kind_for(c, nq);
    c->last_kind = kind;
    if (c->use_graphs) {
        kspir_ctx::PhaseGraphs* pg = nullptr;
        int rc = build_graphs(c, slot0, nq, kind != SCAN_CUDA, &pg);
        if (rc) return rc;
        cudaEventRecord(ev[0], st);
        KS_CUDA(c, cudaGraphLaunch(pg->g[0], st));
        cudaEventRecord(ev[1], st);
        enqueue_scan(c, slot0, nq, kind, st, share);
        cudaEventRecord(ev[2], st);
        KS_CUDA(c, cudaGraphLaunch(pg->g[1], st));
        cudaEventRecord(ev[3], st);
        KS_CUDA(c, cudaGraphLaunch(pg->g[2], st));
        cudaEventRecord(ev[4], st);
        KS_CUDA(c, cudaGraphLaunch(pg->g[3], st));
        cudaEventRecord(ev[5], st);
    } else {
        cudaEventRecord(ev[0], st);
        enqueue_baby(c, slot0, nq, kind != SCAN_CUDA, st);
        cudaEventRecord(ev[1], st);
        enqueue_scan(c, slot0, nq, kind, st, share);
        cudaEventRecord(ev[2], st);
        enqueue_giant(c, slot0, nq, st);
        cudaEventRecord(ev[3], st);
        enqueue_ext(c, slot0, nq, c->p.r, nullptr, nullptr, st);
        cudaEventRecord(ev[4], st);
        enqueue_packing(c, slot0, nq, st);
        cudaEventRecord(ev[5], st);
    }
    c->ring_nq[slot] = nq;
    c->enqueues++;
    c->answers += nq;
    c->launches += answer_launches(c, kind, nq);
    c->last_slot = slot;
    return KSPIR_OK;
}

bool canonical(const uint64_t* w, size_t n, uint64_t q) {
    for (size_t i = 0; i < n; i++)
        if (w[i] >= q) return false;
    return true;
}

int check_base(kspir_ctx* c) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    if (!c->db_loaded) return set_err(c, KSPIR_ERR_NOT_READY, "database not uploaded");
    if (!c->perms_loaded) return set_err(c, KSPIR_ERR_NOT_READY, "permutations not uploaded");
    return KSPIR_OK;
}

int check_client(kspir_ctx* c, int client) {
    if (client < 0 || client >= c->p.max_clients) return set_err(c, KSPIR_ERR_INVALID_ARG, "client slot out of range");
    if (!c->key_loaded[client]) return set_err(c, KSPIR_ERR_NOT_READY, "client keys not uploaded");
    return KSPIR_OK;
}

int check_ready(kspir_ctx* c, int client) {
    int rc = check_base(c);
    return rc ? rc : check_client(c, client);
}

// Waits for the work enqueued on the context stream and collects the error
// words of slots [slot0, slot0 + nq) with it (one synchronisation).
int finish(kspir_ctx* c, int slot0, int nq) {
    const size_t bytes = (size_t)nq * kErrStride * 4;
    KS_CUDA(c, cudaMemcpyAsync(c->errs_host + (size_t)slot0 * kErrStride, c->errs + (size_t)slot0 * kErrStride, bytes,
                               cudaMemcpyDeviceToHost, c->stream));
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    const int* e = c->errs_host + (size_t)slot0 * kErrStride;
    int herr = 0;
    for (int q = 0; q < nq; q++) herr |= e[(size_t)q * kErrStride];
    if (herr) {
        cudaMemsetAsync(c->errs + (size_t)slot0 * kErrStride, 0, bytes, c->stream);
        cudaStreamSynchronize(c->stream);
        return set_err(c, KSPIR_ERR_TIMEOUT, "a bounded device wait gave up (code " + std::to_string(herr) + ")");
    }
    return KSPIR_OK;
}

// Orders `st` after every device-buffer single answer still using a workspace
// slot (they may run on other streams).
int wait_singles(kspir_ctx* c, cudaStream_t st) {
    for (int i = 0; i < c->single_slots; i++)
        if (c->slot_used[i]) KS_CUDA(c, cudaStreamWaitEvent(st, c->slot_done[i], 0));
    return KSPIR_OK;
}

// Marks every single-answer slot as used by work just enqueued on `st`, so a
// later device-buffer single answer (on any stream) is ordered after it.
int mark_singles(kspir_ctx* c, cudaStream_t st) {
    for (int i = 0; i < c->single_slots; i++) {
        KS_CUDA(c, cudaEventRecord(c->slot_done[i], st));
        c->slot_used[i] = 1;
        c->slot_last_stream[i] = st;
    }
    return KSPIR_OK;
}

// Chooses the workspace slot of a single answer; `lk` holds c->mu.  The fused
// answer has one set of counters and always runs in slot 0.  A host-buffer
// answer (`host`) waits until a slot no other host call owns is free; a
// device-buffer answer prefers such a slot but takes the next one otherwise
// (the slot events order it after the owner on the device).
int pick_slot(kspir_ctx* c, std::unique_lock<std::mutex>& lk, bool host) {
    for (;;) {
        const int n = c->fused ? 1 : c->single_slots;
        for (int k = 0; k < n; k++) {
            const int s = (c->next_single + k) % n;
            if (!c->slot_busy[s]) {
                c->next_single = (s + 1) % c->single_slots;
                return s;
            }
        }
        if (!host) {
            const int s = c->fused ? 0 : c->next_single;
            c->next_single = (s + 1) % c->single_slots;
            return s;
        }
        c->slot_cv.wait(lk);
    }
}

// A host call's ownership of a single-answer slot; released (and the waiting
// host calls woken) when it goes out of scope with c->mu held.
struct SlotHold {
    kspir_ctx* c;
    int slot;
    ~SlotHold() {
        c->slot_busy[slot] = 0;
        c->slot_cv.notify_all();
    }
};

// Whether a single answer in another slot, on another stream, may still be
// running when this one (slot `self`, stream `st`) starts: then the scan takes
// the sharing ring shape.  Answers on the same stream run one after another
// and keep the streaming shape.
bool singles_beside(kspir_ctx* c, int self, cudaStream_t st) {
    for (int i = 0; i < c->single_slots; i++) {
        if (i == self || !c->slot_used[i] || c->slot_last_stream[i] == st) continue;
        if (c->slot_busy[i] || cudaEventQuery(c->slot_done[i]) == cudaErrorNotReady) return true;
    }
    return false;
}

// the tensor-core database operand, rebuilt from the resident database
int build_dbop(kspir_ctx* c) {
    if (!c->mma) return KSPIR_OK;
    const size_t bytes = (size_t)kN * 2 * c->G * kATile;
    if (!c->dbop) KS_CUDA(c, cudaMalloc(&c->dbop, bytes));
    k_dbop_build<<<blocks_for((long)kN * 2 * c->G * 128 * 8, 256), 256, 0, c->stream>>>(c->db, c->dbop, c->p.r, c->N2,
                                                                                        c->G);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaStreamSynchronize(c->stream));
    return KSPIR_OK;
}

// The task queue of the fused answer (k_answer.cuh).  Every task comes after
// the tasks it depends on; the tail (giant steps, external products, packing
// merges) is sorted by when its inputs complete: the scan position of the
// last sub-database it needs (the scan runs in fa_scan_order), then its depth.
std::vector<FaTask> build_fa_tasks(const kspir_ctx* c) {
    std::vector<FaTask> t;
    auto add = [&](int type, int a, int b, int cc = 0, int d = 0) {
        FaTask x;
        x.type = (uint8_t)type; x.a = (uint8_t)a; x.b = (uint16_t)b; x.c = (uint16_t)cc; x.d = (uint16_t)d;
        t.push_back(x);
    };
    const int R = c->p.r, N2 = c->N2, L = c->levels, N1h = c->N1h, inter = N1h - 2;
    for (int b = 0; b < kFaPrepChunks; b++) add(FT_PREP, 0, b);
    for (int b = 0; b < c->n_q; b++) add(FT_QNTT, 0, b);
    for (int comp = 0; comp < 2; comp++) add(FT_ROT1, comp, inter);
    for (int b = 0; b < 2; b++) add(FT_INTER_NTT, 0, b);
    for (int b = 0; b < kFaPrepChunks; b++) add(FT_INTER_DEC, 0, b);
    for (int b = 0; b < 9; b++) add(FT_DIG1, 0, b);
    for (int ki = 0; ki < N1h - 1; ki++)
        if (ki != inter)
            for (int comp = 0; comp < 2; comp++) add(FT_ROT1, comp, ki);
    for (int ki = 0; ki < N1h; ki++)
        for (int comp = 0; comp < 2; comp++) add(FT_ROT2, comp, ki);
    std::vector<int> pos(R);
    for (int x = 0; x < R; x++) pos[fa_scan_order(x, L)] = x;   // pos[sub-database] = scan position
    struct Keyed { int k0, k1, k2; FaTask task; };
    std::vector<Keyed> tail;
    auto push = [&](int k0, int k1, int k2, int type, int a, int b, int cc = 0, int d = 0) {
        FaTask x;
        x.type = (uint8_t)type; x.a = (uint8_t)a; x.b = (uint16_t)b; x.c = (uint16_t)cc; x.d = (uint16_t)d;
        tail.push_back(Keyed{k0, k1, k2, x});
    };
    for (int r = 0; r < R; r++) {
        for (int cg = 1; cg < N2; cg++) push(pos[r], 0, cg, FT_GIANT, 0, r, cg);
        for (int ch = 0; ch < 2; ch++) push(pos[r], 1, ch, FT_EXT, ch, r);
    }
    for (int lv = L - 1; lv >= 0; lv--) {
        const int I = 1 << lv;
        for (int j = 0; j < I; j++) {
            int last = 0;
            for (int x = j; x < R; x += I) last = std::max(last, pos[x]);
            const int depth = 2 + 2 * (L - 1 - lv);
            for (int ch = 0; ch < 2; ch++)
                for (int d = 0; d <= 4; d++) push(last, depth, ch * 8 + d, FT_PFWD, lv, j, ch, d);
            for (int ch = 0; ch < 2; ch++)
                for (int comp = 0; comp < 2; comp++) push(last, depth + 1, ch * 2 + comp, FT_PINV, lv, j, ch, comp);
        }
    }
    std::stable_sort(tail.begin(), tail.end(), [](const Keyed& x, const Keyed& y) {
        return x.k0 != y.k0 ? x.k0 < y.k0 : x.k1 != y.k1 ? x.k1 < y.k1 : x.k2 < y.k2;
    });
    for (auto& k : tail) t.push_back(k.task);
    add(FT_COMPOSE, 0, 0);
    return t;
}

// Runs the queue in order on the host with the kernel's own dependency rules
// (the scan completes once every rotation has): every task must find its
// inputs complete when it is dequeued, so no wait of the kernel can depend on
// a task behind it.  Returns the index of the first task that fails, or -1.
int fa_check_order(const std::vector<FaTask>& tasks, const FaShape& sh) {
    std::vector<int> cnt(fa_counter_words(sh.R), 0);
    cnt[FC_ZERO] = sh.ctas;
    for (size_t i = 0; i < tasks.size(); i++) {
        int idx[2], target[2];
        const int n = fa_deps(sh, tasks[i], idx, target);
        for (int d = 0; d < n; d++)
            if (idx[d] < 0 || idx[d] >= (int)cnt.size() || cnt[idx[d]] < target[d]) return (int)i;
        int second;
        const int c = fa_done(sh, tasks[i], &second);
        cnt[c]++;
        if (second >= 0) cnt[second]++;
        if (cnt[FC_QNTT] >= sh.n_q && cnt[FC_ROT1] >= 2 * (sh.N1 / 2 - 1) && cnt[FC_ROT2] >= sh.N1)
            for (int r = 0; r < sh.R; r++) cnt[FC_PER_R + r] = kN;
    }
    return cnt[FC_COMPOSE] == 1 ? -1 : (int)tasks.size();
}

// The fused single answer needs N1 = 128, a device that launches cooperative
// kernels, and one CTA of k_answer per SM.  Single answers use it when
// KSPIR_FUSED=1 or kspir_set_fused turns it on.
int init_fused(kspir_ctx* c) {
    if (c->N1 != 128) return KSPIR_OK;
    int coop = 0;
    KS_CUDA(c, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, c->device));
    if (!coop) return KSPIR_OK;
    using F = FaCfg<128, kFaScanWarps>;
    KS_CUDA(c, cudaFuncSetAttribute(k_answer<128, kFaScanWarps>, cudaFuncAttributeMaxDynamicSharedMemorySize, F::SMEM));
    int per_sm = 0;
    KS_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_answer<128, kFaScanWarps>, F::THREADS, F::SMEM));
    if (per_sm < 1) return KSPIR_OK;
    const std::vector<FaTask> tasks = build_fa_tasks(c);
    const int bad = fa_check_order(tasks, FaShape{c->p.r, c->N1, c->levels, c->n_q, c->N1h - 2, c->nsm});
    if (bad >= 0)
        return set_err(c, KSPIR_ERR_INVALID_ARG, "fused answer: task " + std::to_string(bad) + " out of order");
    c->fa_ntasks = (int)tasks.size();
    KS_CUDA(c, cudaMalloc(&c->fa_tasks, tasks.size() * sizeof(FaTask)));
    KS_COPY(c, c->fa_tasks, tasks.data(), tasks.size() * sizeof(FaTask), cudaMemcpyHostToDevice);
    KS_CUDA(c, cudaMalloc(&c->fa_cnt, (size_t)fa_counter_words(c->p.r) * 4));
    KS_CUDA(c, cudaMalloc(&c->fa_acc, (size_t)c->p.r * 4 * kN * 4));
    KS_CUDA(c, cudaMalloc(&c->fa_times, (size_t)kTimingRing * FT_T_COUNT * 8));
    KS_CUDA(c, cudaMemsetAsync(c->fa_times, 0, (size_t)kTimingRing * FT_T_COUNT * 8, c->stream));
    c->fused_ok = true;
    if (const char* e = getenv("KSPIR_FUSED")) c->fused = e[0] == '1';
    return KSPIR_OK;
}

template <int BT>
int mma_attr(kspir_ctx* c) {
    KS_CUDA(c, cudaFuncSetAttribute(k_scan_mma<BT>, cudaFuncAttributeMaxDynamicSharedMemorySize, MmaCfg<BT>::SMEM));
    KS_CUDA(c, cudaFuncSetAttribute(k_qop_split_rm<BT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kSplitSmem));
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
        case KSPIR_ERR_BUSY: return "busy: requests in flight";
        case KSPIR_ERR_IO: return "file or format error";
        default: return "unknown error";
    }
}

const char* kspir_last_error(const kspir_ctx*) { return g_thread_err.c_str(); }

int kspir_ctx_create(int device, const kspir_params* params, kspir_ctx** out) {
    if (!params || !out) return KSPIR_ERR_INVALID_ARG;
    const kspir_params p = *params;
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    if (!pow2(p.r) || p.r > 512 || !pow2(p.N1) || p.N1 < 64 || p.N1 > 256 || p.max_clients < 1 ||
        p.max_inflight < 1 || p.max_inflight > 4096)
        return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "invalid parameters");
    std::unique_ptr<kspir_ctx> c(new kspir_ctx());
    c->device = device;
    c->p = p;
    c->N1 = p.N1;
    c->N1h = p.N1 / 2;
    c->N2 = kN / 2 / p.N1;
    c->levels = ilog2i(p.r);
    c->mma = (p.N1 == kMmaK && p.max_inflight >= 2);
    c->G = (p.r * c->N2 + 31) / 32;
    KS_CUDA(c.get(), cudaSetDevice(device));
    KS_CUDA(c.get(), cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    KS_CUDA(c.get(), cudaStreamCreateWithFlags(&c->capture, cudaStreamNonBlocking));
    if (const char* e = getenv("KSPIR_NO_GRAPHS")) c->use_graphs = !(e[0] == '1');
    if (const char* e = getenv("KSPIR_NO_PDL")) c->use_pdl = !(e[0] == '1');
    KS_CUDA(c.get(), cudaDeviceGetAttribute(&c->nsm, cudaDevAttrMultiProcessorCount, device));
    c->scan_ctas = c->nsm;
    if (const char* e = getenv("KSPIR_SCAN_CTAS")) c->scan_ctas = std::max(1, std::min(c->nsm, atoi(e)));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_baby_pair<3, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBabyPairSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_client_query, cudaFuncAttributeMaxDynamicSharedMemorySize, kClientSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_client_decrypt, cudaFuncAttributeMaxDynamicSharedMemorySize, kClientSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_db_rows<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDbRowsSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_db_rows<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kDbRowsSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_ntt_jobs<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kNttJobSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_ntt_jobs<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kNttJobSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_giant_fused<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGiantSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_ext_fused<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kExtSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_pack_fused<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPackSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_pack_split_fwd<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPackSplitSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_pack_split_inv<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kPackSplitSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_off_keyswitch, cudaFuncAttributeMaxDynamicSharedMemorySize, kOffSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_off_intt_key, cudaFuncAttributeMaxDynamicSharedMemorySize, kNttJobSmem));
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_off_modswitch, cudaFuncAttributeMaxDynamicSharedMemorySize, kNttJobSmem));
#define KS_ATTR(n)                                                                                         \
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_scan<n>, cudaFuncAttributeMaxDynamicSharedMemorySize, ScanCfg<n>::SMEM)); \
    KS_CUDA(c.get(), cudaFuncSetAttribute(k_scan<n, ScanShare<n>::CONS, ScanShare<n>::NST>,                     \
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, ScanShare<n>::Cfg::SMEM));
    KS_ATTR(64) KS_ATTR(128) KS_ATTR(256)
#undef KS_ATTR
    int rc = KSPIR_OK;
    if (c->mma) {
        if (!rc) rc = mma_attr<4>(c.get());
        if (!rc) rc = mma_attr<8>(c.get());
        if (!rc) rc = mma_attr<16>(c.get());
        if (!rc) rc = mma_attr<32>(c.get());
        if (rc) return rc;
        const size_t qslots = align_up((size_t)p.max_inflight, 32) + 32;   // a launch may round up by a tile
        KS_CUDA(c.get(), cudaMalloc(&c->qop, (size_t)kN * 2 * qslots * 8 * kMmaK));
    }
    rc = init_constants(c.get());
    if (rc) return rc;
    KS_CUDA(c.get(), cudaMalloc(&c->perms, (size_t)p.N1 * kN * 4));
    c->ring.resize(kTimingRing);
    c->ring_nq.assign(kTimingRing, 0);
    for (auto& evs : c->ring)
        for (auto& e : evs) KS_CUDA(c.get(), cudaEventCreate(&e));
    c->single_slots = std::min(p.max_inflight, kSingleSlots);
    c->slot_done.assign(c->single_slots, nullptr);
    c->host_done.assign(c->single_slots, nullptr);
    c->slot_stream.assign(c->single_slots, nullptr);
    c->slot_used.assign(c->single_slots, 0);
    c->slot_busy.assign(c->single_slots, 0);
    c->slot_last_stream.assign(c->single_slots, nullptr);
    for (int i = 0; i < c->single_slots; i++) {
        KS_CUDA(c.get(), cudaEventCreateWithFlags(&c->slot_done[i], cudaEventDisableTiming));
        KS_CUDA(c.get(), cudaEventCreateWithFlags(&c->host_done[i], cudaEventDisableTiming));
        KS_CUDA(c.get(), cudaStreamCreateWithFlags(&c->slot_stream[i], cudaStreamNonBlocking));
    }
    KS_CUDA(c.get(), cudaHostAlloc(&c->single_errs, (size_t)c->single_slots * 4, cudaHostAllocDefault));
    rc = init_key_slots(c.get());
    if (rc) return rc;
    rc = init_workspaces(c.get());
    if (rc) return rc;
    c->ring_fused.assign(kTimingRing, 0);
    rc = init_fused(c.get());
    if (rc) return rc;
    KS_CUDA(c.get(), cudaStreamSynchronize(c->stream));
    *out = c.release();
    return KSPIR_OK;
}

int kspir_ctx_destroy(kspir_ctx* c) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    cudaDeviceSynchronize();
    for (auto& evs : c->ring)
        for (auto& e : evs) if (e) cudaEventDestroy(e);
    for (auto& e : c->slot_done) if (e) cudaEventDestroy(e);
    for (auto& e : c->host_done) if (e) cudaEventDestroy(e);
    for (auto& st : c->slot_stream) if (st) cudaStreamDestroy(st);
    if (c->single_errs) cudaFreeHost(c->single_errs);
    for (auto& kv : c->graphs)
        for (auto& g : kv.second.g) if (g) cudaGraphExecDestroy(g);
    if (c->capture) cudaStreamDestroy(c->capture);
    cudaFree(c->ws_mem);
    cudaFree(c->jobs);
    cudaFree(c->bq64);
    cudaFree(c->bresp);
    cudaFree(c->errs);
    if (c->errs_host) cudaFreeHost(c->errs_host);
    cudaFree(c->client_of);
    cudaFree(c->stage32);
    cudaFree(c->key_mem);
    cudaFree(c->db);
    cudaFree(c->dbg);
    cudaFree(c->dbflag);
    cudaFree(c->prep_dev);
    cudaFree(c->cl_qenc);
    cudaFree(c->cl_dm);
    cudaFree(c->cl_scratch);
    if (c->prep_host) cudaFreeHost(c->prep_host);
    cudaFree(c->dbop);
    cudaFree(c->qop);
    cudaFree(c->fa_tasks);
    cudaFree(c->fa_cnt);
    cudaFree(c->fa_acc);
    cudaFree(c->fa_times);
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
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    if (!c->db) KS_CUDA(c, cudaMalloc(&c->db, need * 8));
    KS_COPY(c, c->db, datacrt, need * 8, cudaMemcpyHostToDevice);
    int rc = build_dbop(c);
    if (rc) return rc;
    c->db_loaded = true;
    return KSPIR_OK;
}

namespace {
// Validates the raw database on the device, then overwrites the resident one
// with its preprocessed form (k_db_rows), caller holds the lock.
// the gather table of the context's N1 and the validation word, built once
int ensure_db_tables(kspir_ctx* c) {
    if (c->dbg) return KSPIR_OK;
    const std::vector<uint16_t> g = db_gather_table(c->N1);
    KS_CUDA(c, cudaMalloc(&c->dbflag, sizeof(int)));
    KS_CUDA(c, cudaMalloc(&c->dbg, g.size() * 2));
    KS_COPY(c, c->dbg, g.data(), g.size() * 2, cudaMemcpyHostToDevice);
    return KSPIR_OK;
}

// 1 when some of the n raw words is >= bsgsp (synchronises)
int db_words_invalid(kspir_ctx* c, const uint64_t* d_raw, size_t n, int* bad) {
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaMemsetAsync(c->dbflag, 0, sizeof(int), st));
    k_check_canonical<<<c->nsm * 8, 256, 0, st>>>(d_raw, n, kP, c->dbflag);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(bad, c->dbflag, sizeof(int), cudaMemcpyDeviceToHost, st));
    KS_CUDA(c, cudaStreamSynchronize(st));
    return KSPIR_OK;
}

int db_preprocess_dev(kspir_ctx* c, const uint64_t* d_raw, float* device_ms) {
    const int r = c->p.r;
    const size_t words = (size_t)r * kN * (kN / 2);
    cudaStream_t st = c->stream;
    int rc0 = ensure_db_tables(c);
    if (rc0) return rc0;
    if (!c->db) KS_CUDA(c, cudaMalloc(&c->db, words * 8));
    cudaEvent_t ev[2] = {nullptr, nullptr};
    if (device_ms) {
        KS_CUDA(c, cudaEventCreate(&ev[0]));
        KS_CUDA(c, cudaEventCreate(&ev[1]));
        KS_CUDA(c, cudaEventRecord(ev[0], st));
    }
    int bad = 0;
    rc0 = db_words_invalid(c, d_raw, words, &bad);
    if (rc0) return rc0;
    if (bad) {
        if (device_ms) { cudaEventDestroy(ev[0]); cudaEventDestroy(ev[1]); }
        return set_err(c, KSPIR_ERR_INVALID_ARG, "database entries must be below bsgsp = 65537");
    }
    c->db_loaded = false;
    k_db_rows<false><<<dim3(kN / 2 / kDbRowsPerCta, r), kNttThreads, kDbRowsSmem, st>>>(d_raw, c->dbg, c->db,
                                                                                          nullptr, c->N1, c->ntabs);
    KS_CUDA(c, cudaGetLastError());
    int rc = build_dbop(c);   // synchronises
    if (rc) return rc;
    if (device_ms) {
        KS_CUDA(c, cudaEventRecord(ev[1], st));
        KS_CUDA(c, cudaEventSynchronize(ev[1]));
        KS_CUDA(c, cudaEventElapsedTime(device_ms, ev[0], ev[1]));
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
    }
    KS_CUDA(c, cudaStreamSynchronize(st));
    c->db_loaded = true;
    return KSPIR_OK;
}
}  // namespace

int kspir_db_preprocess(kspir_ctx* c, const uint64_t* data, size_t words, float* device_ms) {
    if (!c || !data) return KSPIR_ERR_INVALID_ARG;
    const size_t need = (size_t)c->p.r * kN * (kN / 2);
    if (words != need) return set_err(c, KSPIR_ERR_INVALID_ARG, "raw database must be r*N*N/2 words");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    uint64_t* d_raw = nullptr;
    KS_CUDA(c, cudaMalloc(&d_raw, need * 8));
    int rc = copy_sync(c, d_raw, data, need * 8, cudaMemcpyHostToDevice);
    if (!rc) rc = db_preprocess_dev(c, d_raw, device_ms);
    cudaFree(d_raw);
    return rc;
}

int kspir_db_preprocess_device(kspir_ctx* c, const uint64_t* d_data, size_t words, float* device_ms) {
    if (!c || !d_data) return KSPIR_ERR_INVALID_ARG;
    if (words != (size_t)c->p.r * kN * (kN / 2))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "raw database must be r*N*N/2 words");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    return db_preprocess_dev(c, d_data, device_ms);
}

namespace {
constexpr size_t kSubWords = (size_t)kN * (kN / 2);

int ensure_prep_buffers(kspir_ctx* c) {
    if (!c->prep_dev) KS_CUDA(c, cudaMalloc(&c->prep_dev, 3 * kSubWords * 8));
    if (!c->prep_host) KS_CUDA(c, cudaHostAlloc(&c->prep_host, 2 * kSubWords * 8, cudaHostAllocDefault));
    return KSPIR_OK;
}
}  // namespace

int kspir_database_tobsgsntt(kspir_ctx* c, const uint64_t* data, uint64_t* result) {
    if (!c || !data || !result) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    int rc = ensure_db_tables(c);
    if (!rc) rc = ensure_prep_buffers(c);
    if (rc) return rc;
    c->prep_rows_valid = false;
    uint64_t* d_raw = c->prep_dev;
    uint64_t* d_rows = c->prep_dev + kSubWords;
    uint64_t* d_crt = c->prep_dev + 2 * kSubWords;
    uint64_t* h_in = c->prep_host;
    uint64_t* h_rows = c->prep_host + kSubWords;
    memcpy(h_in, data, kSubWords * 8);
    KS_COPY(c, d_raw, h_in, kSubWords * 8, cudaMemcpyHostToDevice);
    int bad = 0;
    rc = db_words_invalid(c, d_raw, kSubWords, &bad);
    if (rc) return rc;
    if (bad) return set_err(c, KSPIR_ERR_INVALID_ARG, "database entries must be below bsgsp = 65537");
    // the datacrt comes out of the same pass and stays on the device for a
    // database_tocrt of exactly these rows
    k_db_rows<true><<<dim3(kN / 2 / kDbRowsPerCta, 1), kNttThreads, kDbRowsSmem, c->stream>>>(
        d_raw, c->dbg, d_crt, d_rows, c->N1, c->ntabs);
    KS_CUDA(c, cudaGetLastError());
    KS_COPY(c, h_rows, d_rows, kSubWords * 8, cudaMemcpyDeviceToHost);
    memcpy(result, h_rows, kSubWords * 8);
    c->prep_rows_valid = true;
    return KSPIR_OK;
}

int kspir_database_tocrt(kspir_ctx* c, const uint64_t* data_ntt, uint64_t* datacrt) {
    if (!c || !data_ntt || !datacrt) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    int rc = ensure_prep_buffers(c);
    if (rc) return rc;
    uint64_t* d_rows = c->prep_dev + kSubWords;
    uint64_t* d_crt = c->prep_dev + 2 * kSubWords;
    uint64_t* h_in = c->prep_host;
    // rows equal to the last database_tobsgsntt output (compared, not
    // assumed): its datacrt is already on the device
    if (!(c->prep_rows_valid && memcmp(data_ntt, c->prep_host + kSubWords, kSubWords * 8) == 0)) {
        c->prep_rows_valid = false;
        memcpy(h_in, data_ntt, kSubWords * 8);
        KS_COPY(c, d_rows, h_in, kSubWords * 8, cudaMemcpyHostToDevice);
        k_db_tocrt<<<dim3(kN / 32, kN / 2 / 32, 1), dim3(32, 8), 0, c->stream>>>(d_rows, d_crt);
        KS_CUDA(c, cudaGetLastError());
    }
    KS_COPY(c, h_in, d_crt, kSubWords * 8, cudaMemcpyDeviceToHost);
    memcpy(datacrt, h_in, kSubWords * 8);
    return KSPIR_OK;
}

// ---------------------------------------------------------------------------
// client side (k_client.cuh)

}  // extern "C"

namespace {
// a small secret word: s < B or s > crtMod - B, B = bsMod / 2 (the centred
// lift into bsMod, guass_to_modulus, is then meaningful)
bool small_secret(const uint64_t* s, size_t n) {
    for (size_t i = 0; i < n; i++)
        if (!(s[i] < kBsMod / 2 || (s[i] < kCrtMod && s[i] > kCrtMod - kBsMod / 2))) return false;
    return true;
}

int ensure_client_tables(kspir_ctx* c) {
    if (c->cl_dm) return KSPIR_OK;
    const std::vector<int32_t> qe = query_encode_table();
    // the reference's own expression, twosteps.cpp:303, as it compiles: a
    // long double quotient (x87 on the host here too) through the C library's
    // round(double)
    std::vector<uint64_t> dm(kP);
    for (uint64_t me = 0; me < kP; me++) dm[me] = (uint64_t)::round((double)((long double)me * kCrtMod / kP));
    KS_CUDA(c, cudaMalloc(&c->cl_qenc, kN * 4));
    KS_CUDA(c, cudaMalloc(&c->cl_dm, kP * 8));
    KS_COPY(c, c->cl_qenc, qe.data(), kN * 4, cudaMemcpyHostToDevice);
    KS_COPY(c, c->cl_dm, dm.data(), kP * 8, cudaMemcpyHostToDevice);
    return KSPIR_OK;
}

// one device allocation carved into pieces (16-byte aligned)
struct Carve {
    uint8_t* base = nullptr;
    size_t off = 0;
    template <class T>
    T* take(size_t count) {
        T* p = reinterpret_cast<T*>(base + off);
        off += (count * sizeof(T) + 255) & ~(size_t)255;
        return p;
    }
};

// The context's client scratch, at least `bytes` long (caller holds c->mu).
int client_scratch(kspir_ctx* c, size_t bytes, uint8_t** out) {
    if (c->cl_scratch_bytes < bytes) {
        KS_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->cl_scratch);
        c->cl_scratch = nullptr;
        c->cl_scratch_bytes = 0;
        KS_CUDA(c, cudaMalloc(&c->cl_scratch, bytes));
        c->cl_scratch_bytes = bytes;
    }
    *out = c->cl_scratch;
    return KSPIR_OK;
}
}  // namespace

// ---------------------------------------------------------------------------
// Offline key derivation (k_offline.cuh)

namespace {

CrtRef make_crt_ref(uint64_t m1, uint64_t m2) {
    CrtRef c;
    const hu128 M = (hu128)m1 * m2;
    const hu128 two128 = (~(hu128)0 % M + 1) % M;   // 2^128 mod M
    c.M.lo = (uint64_t)M; c.M.hi = (uint64_t)(M >> 64);
    c.two128.lo = (uint64_t)two128; c.two128.hi = (uint64_t)(two128 >> 64);
    c.qi1 = m2; c.qinv1 = h_invmod(m2 % m1, m1);   // term of x1: m2 * (m2^-1 mod m1)
    c.qi2 = m1; c.qinv2 = h_invmod(m1 % m2, m2);   // term of x2: m1 * (m1^-1 mod m2)
    return c;
}

OffGadget make_off_gadget(int ell, int base_bits, int gbits) {
    OffGadget g;
    g.ell = ell; g.base_bits = base_bits; g.gbits = gbits;
    hu128 off = 0;
    for (int i = 0; i < ell; i++) off += (hu128)1 << (base_bits + i * gbits);
    off <<= (gbits - 1);
    off += base_bits ? ((hu128)1 << (base_bits - 1)) : 0;   // base / 2
    g.offset.lo = (uint64_t)off; g.offset.hi = (uint64_t)(off >> 64);
    return g;
}

// One chain: entries e = 1..E of keys (device words [E + 1][6][2][N]; entry 1
// = the automorphism key as generated), links e -> e + 1 for e = 1..E-1; the
// first link reads entry 1 in coefficient form from entry 0.
int run_offline_chain(kspir_ctx* c, const OffChain& ch, uint64_t* keys, int E, const uint32_t* okey, uint32_t* kres,
                      uint32_t* dig, uint32_t* bres, uint32_t* res, uint32_t p1inv) {
    cudaStream_t st = c->stream;
    const size_t key_words = (size_t)6 * 2 * kN;
    k_off_key_residues<<<blocks_for(6L * 2 * kN, 256), 256, 0, st>>>(keys + key_words, kres, 6, kOffRows, ch);
    k_off_intt_key<<<dim3(2, 2, 6), kNttThreads, kNttJobSmem, st>>>(kres, res, c->ntabs, ch);
    k_off_compose<<<dim3(kN / 256, 2, kOffRows), 256, 0, st>>>(res, keys, ch, p1inv);
    for (int e = 1; e < E; e++) {
        const uint64_t* in = keys + (size_t)(e == 1 ? 0 : e) * key_words;
        k_off_decomp<<<dim3(kN / 256, kOffRows), 256, 0, st>>>(in, dig, bres, ch);
        k_off_keyswitch<<<dim3(2 + ch.nch2, kOffRows), kNttThreads, kOffSmem, st>>>(dig, bres, okey, res, c->ntabs, ch);
        k_off_compose<<<dim3(kN / 256, 2, kOffRows), 256, 0, st>>>(res, keys + (size_t)(e + 1) * key_words, ch, p1inv);
    }
    KS_CUDA(c, cudaGetLastError());
    return KSPIR_OK;
}

}  // namespace

extern "C" int kspir_gen_autokey_from_offline(kspir_ctx* c, const uint64_t* offline1, const uint64_t* offline2,
                                              const uint64_t* auto1, const uint64_t* auto2, uint64_t* chain1,
                                              uint64_t* chain2, uint64_t* baby_out, uint64_t* giant_out,
                                              float* device_ms) {
    if (!c || !offline1 || !offline2 || !auto1 || !auto2) return KSPIR_ERR_INVALID_ARG;
    const int N1 = c->N1, N2 = c->N2;
    if (N2 < 2) return set_err(c, KSPIR_ERR_INVALID_ARG, "offline derivation needs N2 >= 2");
    const uint64_t kBa = (uint64_t)kBsMod * kAuxMod;
    const size_t P2 = (size_t)2 * kN;   // words of one RLWE
    // inputs: crtMod rows, then rows of the second modulus
    if (!canonical(offline1, 5 * P2, kCrtMod) || !canonical(offline1 + 5 * P2, 5 * P2, kBa) ||
        !canonical(offline2, 5 * P2, kCrtMod) || !canonical(offline2 + 5 * P2, 5 * P2, kAuxMod) ||
        !canonical(auto1, 3 * P2, kCrtMod) || !canonical(auto1 + 3 * P2, 3 * P2, kBa) ||
        !canonical(auto2, 3 * P2, kCrtMod) || !canonical(auto2 + 3 * P2, 3 * P2, kAuxMod))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "key word not canonical");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    cudaStream_t st = c->stream;

    OffChain baby{};
    baby.nch2 = 2; baby.ch2[0] = CH_BA_BS; baby.ch2[1] = CH_BA_AUX; baby.m2 = kBa;
    baby.ginv = inv_mod_2n(5);
    baby.crt = make_crt_ref(kCrtMod, kBa);
    baby.g = make_off_gadget(5, 18, 18);           // offlineKey1: ellnum 5, base 2^18, Bg 2^18
    OffChain giant{};
    giant.nch2 = 1; giant.ch2[0] = CH_AUX; giant.ch2[1] = CH_AUX; giant.m2 = kAuxMod;
    giant.ginv = inv_mod_2n(pow5((uint32_t)N1));
    giant.crt = make_crt_ref(kCrtMod, kAuxMod);
    giant.g = make_off_gadget(5, 14, 14);          // offlineKey2: ellnum 5, base 2^14, Bg 2^14
    const uint32_t p1inv = (uint32_t)h_invmod(kBsMod, kAuxMod);
    const uint64_t aux_inv = h_invmod(kAuxMod % kCrtMod, kCrtMod);   // auxModInv

    // device buffers, carved from the context's scratch allocation
    const size_t key_words = 6 * P2;
    const size_t n_keys1 = (size_t)N1 * key_words, n_keys2 = (size_t)N2 * key_words;
    const size_t n_okey = (size_t)10 * 2 * 4 * kN, n_kres = (size_t)6 * 2 * 4 * kN;
    const size_t n_dig = (size_t)kOffRows * kOffEll * 4 * kN, n_bres = (size_t)kOffRows * 4 * kN;
    const size_t n_res = (size_t)kOffRows * 4 * 2 * kN;
    const size_t n_ms = (size_t)(N1 - 1 + N2 - 1) * kOffRows * 2 * 2 * kN;
    const size_t n_msw = (size_t)(N1 - 1 + N2 - 1) * kOffRows * P2;
    const size_t bytes = (n_keys1 + n_keys2 + 2 * 10 * P2 + n_msw) * 8 +
                         (2 * n_okey + n_kres + n_dig + n_bres + n_res + n_ms) * 4 + 64 * 256;
    uint8_t* base = nullptr;
    int rc = client_scratch(c, bytes, &base);
    if (rc) return rc;
    Carve cv;
    cv.base = base;
    uint64_t* keys1 = cv.take<uint64_t>(n_keys1);
    uint64_t* keys2 = cv.take<uint64_t>(n_keys2);
    uint64_t* off_w = cv.take<uint64_t>(2 * 10 * P2);
    uint64_t* msw = cv.take<uint64_t>(n_msw);
    uint32_t* okey1 = cv.take<uint32_t>(n_okey);
    uint32_t* okey2 = cv.take<uint32_t>(n_okey);
    uint32_t* kres = cv.take<uint32_t>(n_kres);
    uint32_t* dig = cv.take<uint32_t>(n_dig);
    uint32_t* bres = cv.take<uint32_t>(n_bres);
    uint32_t* res = cv.take<uint32_t>(n_res);
    uint32_t* ms = cv.take<uint32_t>(n_ms);

    cudaEvent_t e0, e1;
    KS_CUDA(c, cudaEventCreate(&e0));
    KS_CUDA(c, cudaEventCreate(&e1));
    KS_CUDA(c, cudaMemcpyAsync(keys1 + key_words, auto1, key_words * 8, cudaMemcpyHostToDevice, st));
    KS_CUDA(c, cudaMemcpyAsync(keys2 + key_words, auto2, key_words * 8, cudaMemcpyHostToDevice, st));
    KS_CUDA(c, cudaMemcpyAsync(off_w, offline1, 10 * P2 * 8, cudaMemcpyHostToDevice, st));
    KS_CUDA(c, cudaMemcpyAsync(off_w + 10 * P2, offline2, 10 * P2 * 8, cudaMemcpyHostToDevice, st));
    KS_CUDA(c, cudaEventRecord(e0, st));
    k_off_key_residues<<<blocks_for(10L * 2 * kN, 256), 256, 0, st>>>(off_w, okey1, 10, kOffEll, baby);
    k_off_key_residues<<<blocks_for(10L * 2 * kN, 256), 256, 0, st>>>(off_w + 10 * P2, okey2, 10, kOffEll, giant);
    rc = run_offline_chain(c, baby, keys1, N1 - 1, okey1, kres, dig, bres, res, p1inv);
    if (!rc) rc = run_offline_chain(c, giant, keys2, N2 - 1, okey2, kres, dig, bres, res, p1inv);
    if (!rc) {
        // the modulus switch of every key of both chains (entries 1..): the
        // baby keys' words, then the giant keys' words
        uint32_t* ms2 = ms + (size_t)(N1 - 1) * kOffRows * 2 * 2 * kN;
        uint64_t* msw2 = msw + (size_t)(N1 - 1) * kOffRows * P2;
        k_off_modswitch<<<(N1 - 1) * 4 * kOffRows, kNttThreads, kNttJobSmem, st>>>(keys1 + key_words, ms, aux_inv,
                                                                                  c->ntabs);
        k_off_modswitch<<<(N2 - 1) * 4 * kOffRows, kNttThreads, kNttJobSmem, st>>>(keys2 + key_words, ms2, aux_inv,
                                                                                  c->ntabs);
        k_compose_words<<<blocks_for((long)(N1 - 1 + N2 - 1) * kOffRows * 2 * kN, 256), 256, 0, st>>>(
            ms, msw, (N1 - 1 + N2 - 1) * kOffRows * 2);
        KS_CUDA(c, cudaEventRecord(e1, st));
        KS_CUDA(c, cudaGetLastError());
        std::vector<uint64_t> w((size_t)(N1 - 1) * kOffRows * P2);
        KS_COPY(c, w.data(), msw, w.size() * 8, cudaMemcpyDeviceToHost);
        if (baby_out)
            for (int e = 0; e < N1 - 1; e++) {
                uint64_t* o = baby_out + (size_t)e * key_words;
                memcpy(o, w.data() + (size_t)e * kOffRows * P2, kOffRows * P2 * 8);
                memset(o + kOffRows * P2, 0, kOffRows * P2 * 8);   // the bsMod rows come out zero
            }
        if (giant_out) KS_COPY(c, giant_out, msw2, (size_t)(N2 - 1) * kOffRows * P2 * 8, cudaMemcpyDeviceToHost);
        if (chain1 && N1 > 2)
            KS_COPY(c, chain1, keys1 + 2 * key_words, (size_t)(N1 - 2) * key_words * 8, cudaMemcpyDeviceToHost);
        if (chain2 && N2 > 2)
            KS_COPY(c, chain2, keys2 + 2 * key_words, (size_t)(N2 - 2) * key_words * 8, cudaMemcpyDeviceToHost);
        float ms_ = 0;
        KS_CUDA(c, cudaEventElapsedTime(&ms_, e0, e1));
        if (device_ms) *device_ms = ms_;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
}

extern "C" {

int kspir_client_queries(kspir_ctx* c, int n, const uint64_t* secrets, const uint32_t* rows, uint64_t seed,
                         uint64_t* queries) {
    if (!c || n < 1 || n > 65535 || !secrets || !rows || !queries) return KSPIR_ERR_INVALID_ARG;
    for (int i = 0; i < n; i++)
        if (rows[i] >= (uint32_t)kN / 2) return set_err(c, KSPIR_ERR_INVALID_ARG, "row must be below N/2");
    if (!small_secret(secrets, (size_t)n * kN)) return set_err(c, KSPIR_ERR_INVALID_ARG, "secret words must be small");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    int rc = ensure_client_tables(c);
    if (rc) return rc;
    const size_t sw = (size_t)n * kN, qw = (size_t)n * 4 * kN, rw = (size_t)n * 6 * kN;
    Carve cv;
    if ((rc = client_scratch(c, sw * 8 + qw * 8 + rw * 4 + (size_t)n * 4 + 1024, &cv.base))) return rc;
    uint64_t* d_s = cv.take<uint64_t>(sw);
    uint64_t* d_q = cv.take<uint64_t>(qw);
    uint32_t* d_res = cv.take<uint32_t>(rw);
    uint32_t* d_rows = cv.take<uint32_t>(n);
    rc = copy_sync(c, d_s, secrets, sw * 8, cudaMemcpyHostToDevice);
    if (!rc) rc = copy_sync(c, d_rows, rows, (size_t)n * 4, cudaMemcpyHostToDevice);
    if (!rc) {
        ClientQueryArgs qa{d_s, d_rows, c->cl_qenc, c->cl_dm, seed, d_res};
        k_client_query<<<dim3(3, n), kNttThreads, kClientSmem, c->stream>>>(qa, c->ntabs);
        k_client_query_words<<<blocks_for((long)n * 2 * kN, 256), 256, 0, c->stream>>>(d_res, d_q, n);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = set_err(c, KSPIR_ERR_CUDA, std::string("client query: ") + cudaGetErrorString(e));
    }
    if (!rc) rc = copy_sync(c, queries, d_q, qw * 8, cudaMemcpyDeviceToHost);
    return rc;
}

int kspir_client_decrypt(kspir_ctx* c, int n, const uint64_t* secrets, const uint64_t* responses, int r,
                         uint64_t* messages) {
    if (!c || n < 1 || n > 65535 || !secrets || !responses || !messages || r < 1 || r > 4096 || (r & (r - 1)))
        return KSPIR_ERR_INVALID_ARG;
    if (!canonical(secrets, (size_t)n * kN, kCrtMod) || !canonical(responses, (size_t)n * 2 * kN, kCrtMod))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "word not canonical");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    // QInv(r, crtMod) (utils.cpp:118-190) is r^-1 mod crtMod for every r of its
    // table; it has no entry for 128 (and returns 0 there)
    const uint64_t qinv = (uint64_t)h_invmod((uint64_t)r % kCrtMod, kCrtMod);
    const size_t sw = (size_t)n * kN, rw = (size_t)n * 2 * kN;
    Carve cv;
    int rc = client_scratch(c, sw * 8 + rw * 8 + rw * 4 + sw * 8 + 1024, &cv.base);
    if (rc) return rc;
    uint64_t* d_s = cv.take<uint64_t>(sw);
    uint64_t* d_r = cv.take<uint64_t>(rw);
    uint32_t* d_res = cv.take<uint32_t>(rw);
    uint64_t* d_m = cv.take<uint64_t>(sw);
    rc = copy_sync(c, d_s, secrets, sw * 8, cudaMemcpyHostToDevice);
    if (!rc) rc = copy_sync(c, d_r, responses, rw * 8, cudaMemcpyHostToDevice);
    if (!rc) {
        k_client_decrypt<<<dim3(2, n), kNttThreads, kClientSmem, c->stream>>>(d_s, d_r, qinv, d_res, c->ntabs);
        k_client_round<<<blocks_for((long)n * kN, 256), 256, 0, c->stream>>>(d_res, d_m, n);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) rc = set_err(c, KSPIR_ERR_CUDA, std::string("client decrypt: ") + cudaGetErrorString(e));
    }
    if (!rc) rc = copy_sync(c, messages, d_m, sw * 8, cudaMemcpyDeviceToHost);
    return rc;
}

int kspir_db_download(kspir_ctx* c, uint64_t* datacrt, size_t words) {
    if (!c || !datacrt) return KSPIR_ERR_INVALID_ARG;
    const size_t need = (size_t)c->p.r * kN * (kN / 2);
    if (words != need) return set_err(c, KSPIR_ERR_INVALID_ARG, "database size must be r*N*N/2 words");
    if (!c->db_loaded) return set_err(c, KSPIR_ERR_NOT_READY, "database not uploaded");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    KS_COPY(c, datacrt, c->db, need * 8, cudaMemcpyDeviceToHost);
    return KSPIR_OK;
}

// ---------------------------------------------------------------------------
// wire and file formats (formats.cuh)

}  // extern "C"

namespace {
bool shape_ok(int r, int N1) {
    auto pow2 = [](int v) { return v > 0 && (v & (v - 1)) == 0; };
    return pow2(r) && r <= 512 && pow2(N1) && N1 >= 64 && N1 <= 256;
}

// per-word byte width of each row of the key payload, in payload order, with
// the array it comes from and the modulus its words are below
template <class F>
void key_rows(int r, int N1, F&& f) {
    const int N2 = kN / 2 / N1, levels = log2_ceil(r);
    for (int i = 0; i < N1 / 2; i++)
        for (int j = 0; j < 6; j++)
            for (int comp = 0; comp < 2; comp++)
                f(0, (((size_t)i * 6 + j) * 2 + comp) * kN, j < 3 ? 7 : 3, j < 3 ? kCrtMod : (uint64_t)kBsMod);
    for (size_t k = 0; k < (size_t)(N2 - 1) * 2 * 2; k++) f(1, k * kN, 7, kCrtMod);
    for (size_t k = 0; k < (size_t)levels * 4 * 2; k++) f(2, k * kN, 7, kCrtMod);
    for (size_t k = 0; k < 4 * 2; k++) f(3, k * kN, 7, kCrtMod);
}
}  // namespace

extern "C" {

size_t kspir_key_bundle_bytes(int r, int N1) {
    return shape_ok(r, N1) ? kFileHeader + key_payload_bytes(r, N1) : 0;
}

int kspir_key_bundle_write(int r, int N1, const uint64_t* baby, const uint64_t* giant, const uint64_t* packing,
                           const uint64_t* rgsw, uint8_t* out, size_t out_bytes) {
    if (!shape_ok(r, N1) || !baby || !rgsw || !out) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "invalid arguments");
    if ((kN / 2 / N1 > 1 && !giant) || (r > 1 && !packing)) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "missing key array");
    if (out_bytes != kspir_key_bundle_bytes(r, N1)) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "bundle size");
    const uint64_t* src[4] = {baby, giant, packing, rgsw};
    bool ok = true;
    key_rows(r, N1, [&](int a, size_t off, int, uint64_t q) { ok = ok && canonical(src[a] + off, kN, q); });
    if (!ok) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "key word not canonical");
    uint8_t* p = out + kFileHeader;
    key_rows(r, N1, [&](int a, size_t off, int width, uint64_t) {
        pack_words(src[a] + off, kN, width, p);
        p += (size_t)kN * width;
    });
    FileHeader h{};
    memcpy(h.magic, kKeyMagic, 8);
    h.version = kFormatVersion;
    h.n = kN;
    h.r = (uint32_t)r;
    h.n1 = (uint32_t)N1;
    h.payload_bytes = key_payload_bytes(r, N1);
    h.checksum = payload_checksum(out + kFileHeader, h.payload_bytes);
    memcpy(out, &h, sizeof(h));
    return KSPIR_OK;
}

int kspir_key_bundle_read(const uint8_t* bundle, size_t bytes, int r, int N1, uint64_t* baby, uint64_t* giant,
                          uint64_t* packing, uint64_t* rgsw) {
    if (!shape_ok(r, N1) || !bundle || !baby || !rgsw) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "invalid arguments");
    if ((kN / 2 / N1 > 1 && !giant) || (r > 1 && !packing)) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "missing key array");
    FileHeader h;
    if (bytes < sizeof(h)) return set_err(nullptr, KSPIR_ERR_IO, "key bundle truncated");
    memcpy(&h, bundle, sizeof(h));
    if (memcmp(h.magic, kKeyMagic, 8) != 0 || h.version != kFormatVersion || h.n != (uint32_t)kN)
        return set_err(nullptr, KSPIR_ERR_IO, "not a key bundle of this format version");
    if (h.r != (uint32_t)r || h.n1 != (uint32_t)N1) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "key bundle for another (r, N1)");
    if (h.payload_bytes != key_payload_bytes(r, N1) || bytes != kFileHeader + h.payload_bytes)
        return set_err(nullptr, KSPIR_ERR_IO, "key bundle size");
    if (payload_checksum(bundle + kFileHeader, h.payload_bytes) != h.checksum)
        return set_err(nullptr, KSPIR_ERR_IO, "key bundle checksum mismatch");
    uint64_t* dst[4] = {baby, giant, packing, rgsw};
    const uint8_t* p = bundle + kFileHeader;
    bool ok = true;
    key_rows(r, N1, [&](int a, size_t off, int width, uint64_t q) {
        unpack_words(p, kN, width, dst[a] + off);
        ok = ok && canonical(dst[a] + off, kN, q);
        p += (size_t)kN * width;
    });
    return ok ? KSPIR_OK : set_err(nullptr, KSPIR_ERR_INVALID_ARG, "key word not canonical");
}

int kspir_client_keys_upload_bundle(kspir_ctx* c, int client, const uint8_t* bundle, size_t bytes) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    const int r = c->p.r, N1 = c->N1;
    std::vector<uint64_t> baby((size_t)(N1 / 2) * 6 * 2 * kN), giant((size_t)(c->N2 - 1) * 2 * 2 * kN),
        packing((size_t)c->levels * 4 * 2 * kN), rgsw((size_t)4 * 2 * kN);
    int rc = kspir_key_bundle_read(bundle, bytes, r, N1, baby.data(), giant.empty() ? nullptr : giant.data(),
                                   packing.empty() ? nullptr : packing.data(), rgsw.data());
    if (rc) return set_err(c, rc, g_thread_err);
    return kspir_client_keys_upload(c, client, baby.data(), giant.empty() ? nullptr : giant.data(),
                                    packing.empty() ? nullptr : packing.data(), rgsw.data());
}

int kspir_query_pack(const uint64_t* query, uint8_t* out) {
    if (!query || !out) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "null pointer");
    if (!canonical(query, 2 * kN, kCrtMod) || !canonical(query + 2 * kN, 2 * kN, kBsMod))
        return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "query word not canonical");
    pack_words(query, 2 * kN, 7, out + kWireHeader);
    pack_words(query + 2 * kN, 2 * kN, 3, out + kWireHeader + (size_t)2 * kN * 7);
    WireHeader h{};
    memcpy(h.magic, kWireMagic, 4);
    h.version = (uint16_t)kFormatVersion;
    h.kind = 1;
    h.checksum = payload_checksum(out + kWireHeader, kQueryWireBytes - kWireHeader);
    memcpy(out, &h, sizeof(h));
    return KSPIR_OK;
}

int kspir_response_pack(const uint64_t* response, uint8_t* out) {
    if (!response || !out) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "null pointer");
    if (!canonical(response, 2 * kN, kCrtMod)) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "response word not canonical");
    pack_words(response, 2 * kN, 7, out + kWireHeader);
    WireHeader h{};
    memcpy(h.magic, kWireMagic, 4);
    h.version = (uint16_t)kFormatVersion;
    h.kind = 2;
    h.checksum = payload_checksum(out + kWireHeader, kResponseWireBytes - kWireHeader);
    memcpy(out, &h, sizeof(h));
    return KSPIR_OK;
}

namespace {
int wire_check(const uint8_t* in, size_t bytes, uint16_t kind, size_t want) {
    if (!in) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "null pointer");
    WireHeader h;
    if (bytes != want) return set_err(nullptr, KSPIR_ERR_IO, "wire message size");
    memcpy(&h, in, sizeof(h));
    if (memcmp(h.magic, kWireMagic, 4) != 0 || h.version != kFormatVersion || h.kind != kind)
        return set_err(nullptr, KSPIR_ERR_IO, "not a wire message of this kind and format version");
    if (payload_checksum(in + kWireHeader, want - kWireHeader) != h.checksum)
        return set_err(nullptr, KSPIR_ERR_IO, "wire message checksum mismatch");
    return KSPIR_OK;
}
}  // namespace

int kspir_query_unpack(const uint8_t* in, size_t bytes, uint64_t* query) {
    if (!query) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "null pointer");
    int rc = wire_check(in, bytes, 1, kQueryWireBytes);
    if (rc) return rc;
    unpack_words(in + kWireHeader, 2 * kN, 7, query);
    unpack_words(in + kWireHeader + (size_t)2 * kN * 7, 2 * kN, 3, query + 2 * kN);
    if (!canonical(query, 2 * kN, kCrtMod) || !canonical(query + 2 * kN, 2 * kN, kBsMod))
        return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "query word not canonical");
    return KSPIR_OK;
}

int kspir_response_unpack(const uint8_t* in, size_t bytes, uint64_t* response) {
    if (!response) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "null pointer");
    int rc = wire_check(in, bytes, 2, kResponseWireBytes);
    if (rc) return rc;
    unpack_words(in + kWireHeader, 2 * kN, 7, response);
    if (!canonical(response, 2 * kN, kCrtMod)) return set_err(nullptr, KSPIR_ERR_INVALID_ARG, "response word not canonical");
    return KSPIR_OK;
}

namespace {
// checksum of the n words at d on the device (synchronises)
int device_checksum(kspir_ctx* c, const uint64_t* d, size_t n, uint64_t* out) {
    unsigned long long* acc = nullptr;
    KS_CUDA(c, cudaMalloc(&acc, sizeof(*acc)));
    int rc = KSPIR_OK;
    cudaError_t e = cudaMemsetAsync(acc, 0, sizeof(*acc), c->stream);
    if (e == cudaSuccess) {
        k_words_checksum<<<c->nsm * 8, 256, 0, c->stream>>>(d, n, acc);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, acc, sizeof(*acc), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) rc = set_err(c, KSPIR_ERR_CUDA, std::string("database checksum: ") + cudaGetErrorString(e));
    cudaFree(acc);
    return rc;
}
}  // namespace

int kspir_db_save(kspir_ctx* c, const char* path) {
    if (!c || !path) return KSPIR_ERR_INVALID_ARG;
    if (!c->db_loaded) return set_err(c, KSPIR_ERR_NOT_READY, "database not uploaded");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    const size_t words = (size_t)c->p.r * kN * (kN / 2);
    FileHeader h{};
    memcpy(h.magic, kDbMagic, 8);
    h.version = kFormatVersion;
    h.n = kN;
    h.r = (uint32_t)c->p.r;
    h.n1 = (uint32_t)c->N1;
    h.payload_bytes = words * 8;
    int rc = device_checksum(c, c->db, words, &h.checksum);
    if (rc) return rc;
    FILE* f = fopen(path, "wb");
    if (!f) return set_err(c, KSPIR_ERR_IO, std::string("cannot create ") + path);
    bool ok = fwrite(&h, sizeof(h), 1, f) == 1;
    // through a pinned staging buffer, 64 MiB at a time
    const size_t chunk = (size_t)8 << 20;
    uint64_t* stage = nullptr;
    if (ok && cudaHostAlloc(&stage, chunk * 8, cudaHostAllocDefault) != cudaSuccess) ok = false;
    for (size_t off = 0; ok && off < words; off += chunk) {
        const size_t n = std::min(chunk, words - off);
        ok = cudaMemcpyAsync(stage, c->db + off, n * 8, cudaMemcpyDeviceToHost, c->stream) == cudaSuccess &&
             cudaStreamSynchronize(c->stream) == cudaSuccess && fwrite(stage, 8, n, f) == n;
    }
    if (stage) cudaFreeHost(stage);
    ok = (fclose(f) == 0) && ok;
    return ok ? KSPIR_OK : set_err(c, KSPIR_ERR_IO, std::string("writing ") + path);
}

int kspir_db_load(kspir_ctx* c, const char* path) {
    if (!c || !path) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    const size_t words = (size_t)c->p.r * kN * (kN / 2);
    FILE* f = fopen(path, "rb");
    if (!f) return set_err(c, KSPIR_ERR_IO, std::string("cannot open ") + path);
    FileHeader h;
    int rc = KSPIR_OK;
    if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, kDbMagic, 8) != 0 || h.version != kFormatVersion ||
        h.n != (uint32_t)kN)
        rc = set_err(c, KSPIR_ERR_IO, std::string(path) + ": not a database file of this format version");
    else if (h.r != (uint32_t)c->p.r || h.n1 != (uint32_t)c->N1 || h.payload_bytes != words * 8)
        rc = set_err(c, KSPIR_ERR_INVALID_ARG, std::string(path) + ": database of another (r, N1)");
    // into a fresh device buffer: the resident database changes only once the
    // whole file has arrived and its checksum matches
    uint64_t* d = nullptr;
    uint64_t* stage = nullptr;
    const size_t chunk = (size_t)8 << 20;
    if (!rc && cudaMalloc(&d, words * 8) != cudaSuccess) rc = set_err(c, KSPIR_ERR_OOM, "database buffer");
    if (!rc && cudaHostAlloc(&stage, chunk * 8, cudaHostAllocDefault) != cudaSuccess)
        rc = set_err(c, KSPIR_ERR_OOM, "staging buffer");
    for (size_t off = 0; !rc && off < words; off += chunk) {
        const size_t n = std::min(chunk, words - off);
        if (fread(stage, 8, n, f) != n) rc = set_err(c, KSPIR_ERR_IO, std::string(path) + ": truncated");
        else if (cudaMemcpyAsync(d + off, stage, n * 8, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
                 cudaStreamSynchronize(c->stream) != cudaSuccess)
            rc = set_err(c, KSPIR_ERR_CUDA, "database upload");
    }
    fclose(f);
    if (stage) cudaFreeHost(stage);
    uint64_t sum = 0;
    if (!rc) rc = device_checksum(c, d, words, &sum);
    if (!rc && sum != h.checksum) rc = set_err(c, KSPIR_ERR_IO, std::string(path) + ": checksum mismatch");
    if (rc) {
        cudaFree(d);
        return rc;
    }
    cudaFree(c->db);
    c->db = d;
    c->db_loaded = false;
    rc = build_dbop(c);
    if (rc) return rc;
    c->db_loaded = true;
    return KSPIR_OK;
}

int kspir_perms_upload(kspir_ctx* c, const int32_t* perms, size_t count) {
    if (!c || !perms) return KSPIR_ERR_INVALID_ARG;
    if (count != (size_t)c->N1 * kN) return set_err(c, KSPIR_ERR_INVALID_ARG, "permutations must be N1*N entries");
    for (size_t i = 0; i < count; i++)
        if (perms[i] < 0 || perms[i] >= kN) return set_err(c, KSPIR_ERR_INVALID_ARG, "permutation entry out of range");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    KS_COPY(c, c->perms, perms, count * 4, cudaMemcpyHostToDevice);
    c->perms_loaded = true;
    return KSPIR_OK;
}

int kspir_client_keys_upload(kspir_ctx* c, int client, const uint64_t* baby, const uint64_t* giant,
                             const uint64_t* packing, const uint64_t* rgsw) {
    if (!c || client < 0 || client >= c->p.max_clients || !baby || !rgsw) return KSPIR_ERR_INVALID_ARG;
    if (c->N2 > 1 && !giant) return KSPIR_ERR_INVALID_ARG;
    if (c->levels > 0 && !packing) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
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

    const ClientKeysDev keys = keys_host(c, client);
    const size_t stage_words = std::max({nb_poly, ng_poly, np_poly, nr_poly}) * kN;
    uint64_t* stage = nullptr;
    KS_CUDA(c, cudaMalloc(&stage, stage_words * 8));
    auto split = [&](const uint64_t* h, size_t polys, const uint32_t* dst) -> int {
        if (!polys) return KSPIR_OK;
        KS_COPY(c, stage, h, polys * kN * 8, cudaMemcpyHostToDevice);
        k_split_words<<<blocks_for((long)polys * kN, 256), 256, 0, c->stream>>>(stage, const_cast<uint32_t*>(dst),
                                                                              (int)polys);
        KS_CUDA(c, cudaStreamSynchronize(c->stream));
        return KSPIR_OK;
    };
    c->key_loaded[client] = 0;
    int rc = split(crt_rows.data(), nb_poly, keys.baby_crt);
    if (!rc) rc = split(giant, ng_poly, keys.giant);
    if (!rc) rc = split(packing, np_poly, keys.packing);
    if (!rc) rc = split(rgsw, nr_poly, keys.rgsw);
    if (!rc) {
        std::vector<uint32_t> bs32(bs_rows.size());
        for (size_t i = 0; i < bs_rows.size(); i++) bs32[i] = (uint32_t)bs_rows[i];
        rc = copy_sync(c, const_cast<uint32_t*>(keys.baby_bs), bs32.data(), bs32.size() * 4, cudaMemcpyHostToDevice);
    }
    cudaFree(stage);
    if (rc) return rc;
    c->key_loaded[client] = 1;
    return KSPIR_OK;
}

int kspir_answer_device(kspir_ctx* c, int client, const uint64_t* d_query, uint64_t* d_response, void* stream) {
    int rc = check_ready(c, client);
    if (rc) return rc;
    if (!d_query || !d_response) return KSPIR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(c->mu);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    const int slot = pick_slot(c, lk, false);
    const bool share = singles_beside(c, slot, st);
    if (c->slot_used[slot]) KS_CUDA(c, cudaStreamWaitEvent(st, c->slot_done[slot], 0));
    KS_CUDA(c, cudaMemcpyAsync(c->bq64 + (size_t)slot * 4 * kN, d_query, 4 * kN * 8, cudaMemcpyDeviceToDevice, st));
    rc = enqueue_answer(c, slot, 1, &client, st, true, share);
    if (rc) return rc;
    KS_CUDA(c, cudaMemcpyAsync(d_response, c->bresp + (size_t)slot * 2 * kN, 2 * kN * 8, cudaMemcpyDeviceToDevice, st));
    KS_CUDA(c, cudaEventRecord(c->slot_done[slot], st));
    c->slot_used[slot] = 1;
    c->slot_last_stream[slot] = st;
    KS_CUDA(c, cudaGetLastError());
    return KSPIR_OK;
}

int kspir_sync(kspir_ctx* c) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    KS_CUDA(c, cudaDeviceSynchronize());
    return finish(c, 0, c->p.max_inflight);
}

int kspir_debug_scan_fault(kspir_ctx* c, int64_t wait_limit_ns, long skip_item) {
    if (!c || skip_item < -1) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    c->wait_limit_ns = wait_limit_ns > 0 ? (uint64_t)wait_limit_ns : kWaitLimitNs;
    c->scan_skip = skip_item;
    return KSPIR_OK;
}

int kspir_answer(kspir_ctx* c, int client, const uint64_t* query, uint64_t* response) {
    int rc = check_ready(c, client);
    if (rc) return rc;
    if (!query || !response) return KSPIR_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    const int slot = pick_slot(c, lk, true);
    c->slot_busy[slot] = 1;
    SlotHold hold{c, slot};
    cudaStream_t st = c->slot_stream[slot];
    const bool share = singles_beside(c, slot, st);
    if (c->slot_used[slot]) KS_CUDA(c, cudaStreamWaitEvent(st, c->slot_done[slot], 0));
    KS_CUDA(c, cudaMemcpyAsync(c->bq64 + (size_t)slot * 4 * kN, query, 4 * kN * 8, cudaMemcpyHostToDevice, st));
    rc = enqueue_answer(c, slot, 1, &client, st, true, share);
    if (rc) return rc;
    KS_CUDA(c, cudaGetLastError());
    // the query is validated while the device answers it; a non-canonical one
    // is reported before anything reaches the caller's response buffer
    const bool ok = canonical(query, 2 * kN, kCrtMod) && canonical(query + 2 * kN, 2 * kN, kBsMod);
    if (ok) {
        KS_CUDA(c, cudaMemcpyAsync(response, c->bresp + (size_t)slot * 2 * kN, 2 * kN * 8, cudaMemcpyDeviceToHost, st));
        KS_CUDA(c, cudaMemcpyAsync(c->single_errs + slot, c->errs + (size_t)slot * kErrStride, 4,
                                   cudaMemcpyDeviceToHost, st));
    }
    KS_CUDA(c, cudaEventRecord(c->slot_done[slot], st));
    KS_CUDA(c, cudaEventRecord(c->host_done[slot], st));
    c->slot_used[slot] = 1;
    c->slot_last_stream[slot] = st;
    // other host calls enqueue while this one waits for its answer
    lk.unlock();
    const cudaError_t e = cudaEventSynchronize(c->host_done[slot]);
    lk.lock();
    if (e != cudaSuccess) return set_err(c, KSPIR_ERR_CUDA, cudaGetErrorString(e));
    if (!ok) return set_err(c, KSPIR_ERR_INVALID_ARG, "query word not canonical");
    if (const int herr = c->single_errs[slot]) {
        KS_CUDA(c, cudaMemsetAsync(c->errs + (size_t)slot * kErrStride, 0, kErrStride * 4, st));
        KS_CUDA(c, cudaStreamSynchronize(st));
        return set_err(c, KSPIR_ERR_TIMEOUT, "a bounded device wait gave up (code " + std::to_string(herr) + ")");
    }
    return KSPIR_OK;
}

int kspir_answer_batch_device(kspir_ctx* c, int n, const int32_t* clients, const uint64_t* d_queries,
                              uint64_t* d_responses, void* stream) {
    int rc = check_base(c);
    if (rc) return rc;
    if (n < 1 || n > c->p.max_inflight || n > kMaxBatch || !clients || !d_queries || !d_responses)
        return set_err(c, KSPIR_ERR_INVALID_ARG, "batch size out of range or null pointer");
    for (int i = 0; i < n; i++)
        if ((rc = check_client(c, clients[i]))) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaStream_t st = stream ? (cudaStream_t)stream : c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, st)) return wrc;
    KS_CUDA(c, cudaMemcpyAsync(c->bq64, d_queries, (size_t)n * 4 * kN * 8, cudaMemcpyDeviceToDevice, st));
    rc = enqueue_answer(c, 0, n, clients, st);
    if (rc) return rc;
    KS_CUDA(c, cudaMemcpyAsync(d_responses, c->bresp, (size_t)n * 2 * kN * 8, cudaMemcpyDeviceToDevice, st));
    KS_CUDA(c, cudaGetLastError());
    return mark_singles(c, st);
}

int kspir_answer_batch(kspir_ctx* c, int n, const int32_t* clients, const uint64_t* queries, uint64_t* responses) {
    int rc = check_base(c);
    if (rc) return rc;
    if (n < 1 || n > c->p.max_inflight || n > kMaxBatch || !clients || !queries || !responses)
        return set_err(c, KSPIR_ERR_INVALID_ARG, "batch size out of range or null pointer");
    for (int i = 0; i < n; i++)
        if ((rc = check_client(c, clients[i]))) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    KS_CUDA(c, cudaMemcpyAsync(c->bq64, queries, (size_t)n * 4 * kN * 8, cudaMemcpyHostToDevice, c->stream));
    rc = enqueue_answer(c, 0, n, clients, c->stream);
    if (rc) return rc;
    KS_CUDA(c, cudaGetLastError());
    // the queries are validated while the device answers them; a
    // non-canonical word is reported before anything reaches `responses`
    for (int i = 0; i < n; i++) {
        const uint64_t* q = queries + (size_t)i * 4 * kN;
        if (!canonical(q, 2 * kN, kCrtMod) || !canonical(q + 2 * kN, 2 * kN, kBsMod)) {
            KS_CUDA(c, cudaStreamSynchronize(c->stream));
            return set_err(c, KSPIR_ERR_INVALID_ARG, "query word not canonical");
        }
    }
    KS_CUDA(c, cudaMemcpyAsync(responses, c->bresp, (size_t)n * 2 * kN * 8, cudaMemcpyDeviceToHost, c->stream));
    return finish(c, 0, n);
}

int kspir_tune_batch(kspir_ctx* c, int n, int* kind_out, float* ms_out) {
    int rc = check_base(c);
    if (rc) return rc;
    if (n < 1 || n > c->p.max_inflight || n > kMaxBatch) return set_err(c, KSPIR_ERR_INVALID_ARG, "batch size");
    std::lock_guard<std::mutex> lk(c->mu);
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    cudaEvent_t e0, e1;
    KS_CUDA(c, cudaEventCreate(&e0));
    KS_CUDA(c, cudaEventCreate(&e1));
    int best = SCAN_CUDA;
    float best_ms = 1e30f;
    for (int kind = 0; kind < SCAN_KINDS; kind++) {
        if (kind != SCAN_CUDA && !c->mma) continue;
        if (kind != SCAN_CUDA && scan_bt(kind) > 4 && (n + 3) / 4 * 4 < scan_bt(kind) / 2) continue;   // mostly padding
        float ms_min = 1e30f;
        for (int rep = 0; rep < 4; rep++) {
            cudaEventRecord(e0, c->stream);
            enqueue_scan(c, 0, n, kind, c->stream);
            cudaEventRecord(e1, c->stream);
            KS_CUDA(c, cudaEventSynchronize(e1));
            float ms = 0;
            KS_CUDA(c, cudaEventElapsedTime(&ms, e0, e1));
            if (rep > 0) ms_min = std::min(ms_min, ms);   // first run warms up
        }
        if (ms_min < best_ms) { best_ms = ms_min; best = kind; }
        if (ms_out) ms_out[kind] = ms_min;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    rc = finish(c, 0, n);
    if (rc) return rc;
    c->scan_choice[n] = best;
    if (kind_out) *kind_out = best;
    return KSPIR_OK;
}

int kspir_set_scan_kind(kspir_ctx* c, int n, int kind) {
    if (!c || n < 1 || kind < -1 || kind >= SCAN_KINDS) return KSPIR_ERR_INVALID_ARG;
    if (kind > SCAN_CUDA && !c->mma) return set_err(c, KSPIR_ERR_INVALID_ARG, "tensor-core scan not enabled");
    std::lock_guard<std::mutex> lk(c->mu);
    if (kind < 0) c->scan_choice.erase(n);
    else c->scan_choice[n] = kind;
    return KSPIR_OK;
}

int kspir_get_scan_kind(kspir_ctx* c, int n) { return c ? scan_kind_for(c, n) : KSPIR_ERR_INVALID_ARG; }

namespace {
// Phase split of a fused answer from its device timestamps: the segments of its
// critical path (query side up to the scan start or the last rotation, the
// scan, and what the giant steps, external products and packing add after
// the scan ends).
void fused_phases(const unsigned long long* t, float* ph) {
    const double start = (double)~t[FT_T_START], scan0 = (double)~t[FT_T_SCAN0];
    const double head = (double)t[FT_T_HEAD], scan1 = (double)t[FT_T_SCAN1], giant = (double)t[FT_T_GIANT],
                 ext = (double)t[FT_T_EXT], end = (double)t[FT_T_END];
    auto ms = [](double a, double b) { return (float)(b > a ? (b - a) * 1e-6 : 0.0); };
    ph[0] = ms(start, std::min(head, scan0));
    ph[1] = ms(scan0, scan1);
    ph[2] = ms(scan1, giant);
    ph[3] = ms(std::max(scan1, giant), ext);
    ph[4] = ms(std::max(scan1, ext), end);
}

int phases_of(kspir_ctx* c, int slot, float* ph) {
    auto& ev = c->ring[slot];
    KS_CUDA(c, cudaEventSynchronize(ev[5]));
    if (!c->ring_fused[slot]) {
        for (int i = 0; i < 5; i++) KS_CUDA(c, cudaEventElapsedTime(&ph[i], ev[i], ev[i + 1]));
        return KSPIR_OK;
    }
    unsigned long long t[FT_T_COUNT];
    KS_CUDA(c, cudaMemcpy(t, c->fa_times + (size_t)slot * FT_T_COUNT, sizeof(t), cudaMemcpyDeviceToHost));
    fused_phases(t, ph);
    return KSPIR_OK;
}
}  // namespace

int kspir_last_timing(kspir_ctx* c, float* total_ms, float* phase_ms) {
    if (!c || c->last_slot < 0) return KSPIR_ERR_NOT_READY;
    auto& ev = c->ring[c->last_slot];
    KS_CUDA(c, cudaEventSynchronize(ev[5]));
    float t = 0;
    KS_CUDA(c, cudaEventElapsedTime(&t, ev[0], ev[5]));
    if (total_ms) *total_ms = t;
    if (phase_ms) return phases_of(c, c->last_slot, phase_ms);
    return KSPIR_OK;
}

int kspir_set_fused(kspir_ctx* c, int enable) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    if (enable && !c->fused_ok) return set_err(c, KSPIR_ERR_NOT_READY, "fused answer not available on this context");
    std::lock_guard<std::mutex> lk(c->mu);
    c->fused = enable != 0;
    return KSPIR_OK;
}

int kspir_get_fused(const kspir_ctx* c) { return c ? (c->fused ? 1 : 0) : KSPIR_ERR_INVALID_ARG; }

int kspir_timing_reset(kspir_ctx* c) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    c->enqueues = 0;
    c->answers = 0;
    c->launches = 0;
    c->last_slot = -1;
    return KSPIR_OK;
}

int kspir_timing_summary(kspir_ctx* c, int* answers, long* launches, float* total_ms, float* phase_ms) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    const int n = (int)std::min<long>(c->enqueues, kTimingRing);
    float tot = 0, ph[5] = {0, 0, 0, 0, 0};
    int queries = 0;
    for (int k = 0; k < n; k++) {
        auto& ev = c->ring[k];
        KS_CUDA(c, cudaEventSynchronize(ev[5]));
        float t = 0;
        KS_CUDA(c, cudaEventElapsedTime(&t, ev[0], ev[5]));
        tot += t;
        queries += c->ring_nq[k];
        float p[5];
        int rc = phases_of(c, k, p);
        if (rc) return rc;
        for (int i = 0; i < 5; i++) ph[i] += p[i];
    }
    if (answers) *answers = queries;
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
    std::lock_guard<std::mutex> lk(c->mu);
    const Workspace w = ws_host(c, 0);
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    KS_CUDA(c, cudaMemcpyAsync(c->bq64, query_inout, 4 * kN * 8, cudaMemcpyHostToDevice, st));
    k_set_clients<<<1, 32, 0, st>>>(c->client_of, 0, ClientList{1, {client}});
    enqueue_baby(c, 0, 1, false, st);
    enqueue_scan(c, 0, 1, SCAN_CUDA, st);
    enqueue_giant(c, 0, 1, st);
    // result words, and the modswitched query (cipherbuf column 0) back into query1[0]
    uint64_t* words = reinterpret_cast<uint64_t*>(c->stage32);
    k_compose_words<<<blocks_for((long)c->p.r * 2 * kN, 256), 256, 0, st>>>(w.result, words, c->p.r * 2);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(result, words, (size_t)c->p.r * 2 * kN * 8, cudaMemcpyDeviceToHost, st));
    rc = finish(c, 0, 1);
    if (rc) return rc;
    std::vector<uint64_t> cb((size_t)kN * c->N1 * 2);
    KS_COPY(c, cb.data(), w.cipherbuf, cb.size() * 8, cudaMemcpyDeviceToHost);
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
    int rc = check_client(c, client);
    if (rc) return rc;
    if (!result || !first_dim || count < 1 || count > c->p.r) return KSPIR_ERR_INVALID_ARG;
    const size_t n = (size_t)count * 2 * kN;
    if (!canonical(result, n, kCrtMod) || !canonical(first_dim, n, kCrtMod))
        return set_err(c, KSPIR_ERR_INVALID_ARG, "ciphertext word not canonical");
    std::lock_guard<std::mutex> lk(c->mu);
    const Workspace w = ws_host(c, 0);
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    k_set_clients<<<1, 32, 0, st>>>(c->client_of, 0, ClientList{1, {client}});
    uint64_t* words = reinterpret_cast<uint64_t*>(c->stage32);     // r*2*N u64 fit in r*4*N u32
    // first_dim -> ws.result residues; the caller's accumulators (NTT domain) -> ws.sout residues
    KS_CUDA(c, cudaMemcpyAsync(words, first_dim, n * 8, cudaMemcpyHostToDevice, st));
    k_split_words<<<blocks_for((long)n, 256), 256, 0, st>>>(words, w.result, count * 2);
    uint32_t* acc = w.sout;   // r*N2*4*N >= count*4*N residues
    KS_CUDA(c, cudaMemcpyAsync(words, result, n * 8, cudaMemcpyHostToDevice, st));
    k_split_words<<<blocks_for((long)n, 256), 256, 0, st>>>(words, acc, count * 2);
    enqueue_ext(c, 0, 1, count, acc, w.ecoef, st);
    k_compose_words<<<blocks_for((long)n, 256), 256, 0, st>>>(w.ext, words, count * 2);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(result, words, n * 8, cudaMemcpyDeviceToHost, st));
    rc = finish(c, 0, 1);
    if (rc) return rc;
    k_compose_words<<<blocks_for((long)n, 256), 256, 0, st>>>(w.ecoef, words, count * 2);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(first_dim, words, n * 8, cudaMemcpyDeviceToHost, st));
    return finish(c, 0, 1);
}

int kspir_packing_rlwes(kspir_ctx* c, int client, uint64_t* rlwes, uint64_t* response) {
    if (!c) return KSPIR_ERR_INVALID_ARG;
    int rc = check_client(c, client);
    if (rc) return rc;
    if (!rlwes || !response) return KSPIR_ERR_INVALID_ARG;
    const int R = c->p.r;
    const size_t n = (size_t)R * 2 * kN;
    if (!canonical(rlwes, n, kCrtMod)) return set_err(c, KSPIR_ERR_INVALID_ARG, "ciphertext word not canonical");
    std::lock_guard<std::mutex> lk(c->mu);
    const Workspace w = ws_host(c, 0);
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    k_set_clients<<<1, 32, 0, st>>>(c->client_of, 0, ClientList{1, {client}});
    uint64_t* words = reinterpret_cast<uint64_t*>(c->stage32);
    KS_CUDA(c, cudaMemcpyAsync(words, rlwes, n * 8, cudaMemcpyHostToDevice, st));
    k_split_words<<<blocks_for((long)n, 256), 256, 0, st>>>(words, w.ext, R * 2);
    // rlwes[I + j] of every merge, as the reference leaves them (residues in
    // the scan-output region, which the packing does not use)
    uint32_t* c2 = w.sout;
    enqueue_packing(c, 0, 1, st, c2);
    KS_CUDA(c, cudaGetLastError());
    KS_CUDA(c, cudaMemcpyAsync(response, c->bresp, 2 * kN * 8, cudaMemcpyDeviceToHost, st));
    if (R > 1) {
        k_compose_words<<<blocks_for((long)(R - 1) * 2 * kN, 256), 256, 0, st>>>(c2 + 4 * kN, words + 2 * kN,
                                                                                (R - 1) * 2);
        KS_CUDA(c, cudaGetLastError());
        KS_CUDA(c, cudaMemcpyAsync(rlwes + 2 * kN, words + 2 * kN, (size_t)(R - 1) * 2 * kN * 8, cudaMemcpyDeviceToHost,
                                   st));
    }
    rc = finish(c, 0, 1);
    if (rc) return rc;
    memcpy(rlwes, response, 2 * kN * 8);   // rlwes[0] ends as the packed result
    return KSPIR_OK;
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

int kspir_fetch_stage_slot(kspir_ctx* c, int slot, int stage, uint64_t* out, size_t words) {
    if (!c || !out || slot < 0 || slot >= c->p.max_inflight) return KSPIR_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(c->mu);
    const Workspace w = ws_host(c, slot);
    const int R = c->p.r;
    cudaStream_t st = c->stream;
    KS_CUDA(c, cudaSetDevice(c->device));
    if (int wrc = wait_singles(c, c->stream)) return wrc;
    KS_CUDA(c, cudaStreamSynchronize(st));
    if (stage == KSPIR_STAGE_CIPHERBUF) {
        const size_t n = (size_t)kN * c->N1 * 2;
        if (words != n) return set_err(c, KSPIR_ERR_INVALID_ARG, "size mismatch");
        KS_COPY(c, out, w.cipherbuf, n * 8, cudaMemcpyDeviceToHost);
        if (c->last_kind != SCAN_CUDA) {
            // the tensor-core scans' launches write it rotation-major: back to [N][N1][2]
            std::vector<uint32_t> rm(2 * n);
            memcpy(rm.data(), out, n * 8);
            for (int k = 0; k < c->N1; k++)
                for (int comp = 0; comp < 2; comp++)
                    for (int z = 0; z < kN; z++)
                        out[((size_t)z * c->N1 + k) * 2 + comp] =
                            rm[cipherbuf_rm_idx(k, comp, 0, z)] | (uint64_t)rm[cipherbuf_rm_idx(k, comp, 1, z)] << 32;
        }
        return KSPIR_OK;
    }
    const uint32_t* src = nullptr;
    size_t polys = 0;
    if (stage == KSPIR_STAGE_SCAN) { src = w.sout; polys = (size_t)R * c->N2 * 2; }
    else if (stage == KSPIR_STAGE_RESULT) { src = w.result; polys = (size_t)R * 2; }
    else if (stage == KSPIR_STAGE_EXT) { src = w.ext; polys = (size_t)R * 2; }
    else return set_err(c, KSPIR_ERR_INVALID_ARG, "unknown stage");
    if (words != polys * kN) return set_err(c, KSPIR_ERR_INVALID_ARG, "size mismatch");
    uint64_t* tmp = nullptr;
    uint32_t* flat = nullptr;
    KS_CUDA(c, cudaMalloc(&tmp, words * 8));
    cudaError_t e = cudaSuccess;
    if (stage == KSPIR_STAGE_SCAN) {
        e = cudaMalloc(&flat, words * 8);
        if (e == cudaSuccess) {
            k_unblock_sout<<<blocks_for((long)R * c->N2 * 4 * kN, 256), 256, 0, st>>>(src, flat, R * c->N2);
            src = flat;
        }
    }
    if (e == cudaSuccess) {
        k_compose_words<<<blocks_for((long)words, 256), 256, 0, st>>>(src, tmp, (int)polys);
        e = cudaMemcpyAsync(out, tmp, words * 8, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tmp);
    cudaFree(flat);
    if (e != cudaSuccess) return set_err(c, KSPIR_ERR_CUDA, cudaGetErrorString(e));
    return KSPIR_OK;
}

int kspir_fetch_stage(kspir_ctx* c, int stage, uint64_t* out, size_t words) {
    return kspir_fetch_stage_slot(c, 0, stage, out, words);
}

}  // extern "C"

#include "server.cuh"

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
        uint32_t* t = tw + (size_t)ch * 4 * kN;   // uint2 [2][N], k-major layout
        const int pos = tw_layout_pos(k);
        t[2 * pos] = w;
        t[2 * pos + 1] = (uint32_t)(((uint64_t)w << 32) / q);
        t[2 * kN + 2 * pos] = iw;
        t[2 * kN + 2 * pos + 1] = (uint32_t)(((uint64_t)iw << 32) / q);
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
    if (cudaFuncSetAttribute(k_ntt_jobs<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kNttJobSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_ntt_jobs<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kNttJobSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_ext_mac_intt, cudaFuncAttributeMaxDynamicSharedMemorySize, kMacSmem) != cudaSuccess)
        return KSPIR_ERR_CUDA;
    const DevConst dc = make_dev_const();   // the same constants a context writes
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
        k_ntt_jobs<true><<<count * 4, kNttThreads, kNttJobSmem, st>>>(L.jobs, tabs, Batch{});
        k_ext_decomp<<<blocks_for((long)count * kN, 256), 256, 0, st>>>(L.ecoef, L.edig, count, g);
        k_ntt_jobs<false><<<count * 8, kNttThreads, kNttJobSmem, st>>>(L.jobs + kNoAllocMaxCount * 4, tabs, Batch{});
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
