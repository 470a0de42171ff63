// Device-side layouts shared by the answer kernels.
//
// Residue polynomials are u32 [channel][N]; a value mod crtMod has channels
// (q1, q2), a value mod bsMod the single channel bs.  Every per-query buffer
// lives in one Workspace so several queries can be in flight at once.
#pragma once

#include <type_traits>

#include "common.cuh"
#include "gadget.cuh"

namespace kspir {

// Client key material, converted to residues at upload.
//   baby_crt [N1/2][3][2 comp][2 ch][N]    (reference keyMap[5^i][0..2], lwe.h:381-466)
//   baby_bs  [N1/2][3][2 comp][N]          (keyMap[5^i][3..5], mod bsMod)
//   giant    [N2-1][2][2 comp][2 ch][N]    (keyMap[5^(N1 c)])
//   packing  [log2 r][4][2 comp][2 ch][N]  (AutoKey keyMap[N/2^l + 1])
//   rgsw     [4][2 comp][2 ch][N]          (RGSWCiphertext a[j], b[j])
struct ClientKeysDev {
    const uint32_t* baby_crt;
    const uint32_t* baby_bs;
    const uint32_t* giant;
    const uint32_t* packing;
    const uint32_t* rgsw;
};

// Database-scan output layout: a 128-byte line holds 8 consecutive NTT slots
// of 4 consecutive rows (one 32-byte sector per row):
//   sout[z / 8][row / 4][comp * 2 + ch][row % 4][z % 8],  row = r * N2 + i
// A giant step reads and rewrites its own row in whole sectors, and the
// batched scan's epilogue (four slots per thread, eight row lanes per query)
// writes two lines per query and store instead of eight (rows = r * N2 is a
// multiple of 4).
constexpr int kZBlock = 8;
__host__ __device__ __forceinline__ size_t sout_idx(int row, int cv, int z, int rows) {
    return ((((size_t)(z >> 3) * (rows >> 2) + (row >> 2)) * 4 + cv) * 4 + (row & 3)) * kZBlock + (z & 7);
}

struct Workspace {
    uint64_t* q64;          // [4][N] query words: crt a, crt b, bs a, bs b (coefficient form)
    uint32_t* dig0;         // [3][3 ch][N] decompose_bsgs(query a) digits -> NTT form
    uint32_t* qbn;          // [2 ch][N] query b mod q1/q2 -> NTT form
    uint32_t* qbbs;         // [N] query b mod bsMod, coefficient form
    uint32_t* col0;         // [2 comp][2 ch][N] modswitched query, coefficient form (scratch)
    uint32_t* interA;       // [2 ch][N] rotation N1/2-1, a, before modswitch, NTT form
    uint32_t* interB;       // [2 ch][N] rotation N1/2-1, b, NTT form of the coefficient-form sum
    uint32_t* inter_bs;     // [2 comp][N] rotation N1/2-1 mod bsMod, coefficient form
    uint32_t* inter_acoef;  // [2 ch][N] interA, coefficient form
    uint32_t* dig1;         // [3][3 ch][N] digits of the intermediate -> NTT form
    uint64_t* cipherbuf;    // [N][N1][2] reference reorientCipher layout (twosteps.cpp:1386)
    uint32_t* sout;         // DB-scan outputs, NTT form, layout of sout_idx (r * N2 rows)
    uint32_t* result;       // [r][2 comp][2 ch][N] first-dimension results, NTT form (the
                            // giant steps' accumulator until k_giant_finish)
    uint32_t* ecoef;        // [r][2 comp][2 ch][N] result, coefficient form
    uint32_t* ext;          // [r][2 comp][2 ch][N] external products, coefficient form
    uint32_t* ext2;         // [r/2][2 comp][2 ch][N] packing levels ping-pong with ext
    uint32_t* pkpart;       // [r/2][2 ch][5][2 comp][N] terms of a split packing level
    uint64_t* resp64;       // [2][N] response words
    int* err;               // device error word (bounded waits), slot-indexed array
};
constexpr int kErrStride = 64;   // ints between the error words of two slots

// Batch addressing.  Query q of a launch (blockIdx.y) runs in workspace slot
// slot0 + q.  Every workspace slot is a copy of slot 0's layout at a fixed byte
// stride, every client key slot a copy of slot 0's at another, so a kernel
// reaches its query's buffers by shifting slot-0 pointers.  The query words,
// response words and error words live in slot-indexed arrays (one host copy
// per batch).
struct Batch {
    size_t ws_bytes;        // stride between workspace slots
    size_t key_bytes;       // stride between client key slots
    const int* client_of;   // [slots] client key slot serving each workspace slot
    int slot0;
};

template <class T>
__device__ __forceinline__ T* shifted(T* p, size_t off) {
    return p ? reinterpret_cast<T*>(reinterpret_cast<char*>(const_cast<typename std::remove_const<T>::type*>(p)) + off)
             : p;
}

__device__ __forceinline__ int batch_slot(const Batch& b) { return b.slot0 + (int)blockIdx.y; }

__device__ __forceinline__ Workspace ws_at(Workspace w, const Batch& b) {
    const int s = batch_slot(b);
    const size_t off = (size_t)s * b.ws_bytes;
    w.q64 += (size_t)s * 4 * kN;
    w.resp64 += (size_t)s * 2 * kN;
    w.dig0 = shifted(w.dig0, off);
    w.qbn = shifted(w.qbn, off);
    w.qbbs = shifted(w.qbbs, off);
    w.col0 = shifted(w.col0, off);
    w.interA = shifted(w.interA, off);
    w.interB = shifted(w.interB, off);
    w.inter_bs = shifted(w.inter_bs, off);
    w.inter_acoef = shifted(w.inter_acoef, off);
    w.dig1 = shifted(w.dig1, off);
    w.cipherbuf = shifted(w.cipherbuf, off);
    w.sout = shifted(w.sout, off);
    w.result = shifted(w.result, off);
    w.ecoef = shifted(w.ecoef, off);
    w.ext = shifted(w.ext, off);
    w.ext2 = shifted(w.ext2, off);
    w.pkpart = shifted(w.pkpart, off);
    w.err += (size_t)s * kErrStride;
    return w;
}

__device__ __forceinline__ size_t ws_off(const Batch& b) { return (size_t)batch_slot(b) * b.ws_bytes; }
__device__ __forceinline__ size_t key_off(const Batch& b) {
    return (size_t)__ldg(b.client_of + batch_slot(b)) * b.key_bytes;
}

__device__ __forceinline__ ClientKeysDev keys_at(ClientKeysDev k, const Batch& b) {
    const size_t off = key_off(b);
    k.baby_crt = shifted(k.baby_crt, off);
    k.baby_bs = shifted(k.baby_bs, off);
    k.giant = shifted(k.giant, off);
    k.packing = shifted(k.packing, off);
    k.rgsw = shifted(k.rgsw, off);
    return k;
}

// Gadget parameters of the path (reference defaults; lwe.h:391-404, test-pir.cpp:71, :88).
struct PathGadgets {
    GadgetBsgs baby;   // ell 3, base 2^20, Bg 2^20
    GadgetB giant;     // ell 2, base 2^20, Bg 2^18
    GadgetS ext;       // ell 2, base 2^20, Bg 2^18 (signed)
    GadgetB pack;      // ell 4, base 0,    Bg 2^14
};

}  // namespace kspir
