// Device-side layouts shared by the answer kernels.
//
// Residue polynomials are u32 [channel][N]; a value mod crtMod has channels
// (q1, q2), a value mod bsMod the single channel bs.  Every per-query buffer
// lives in one Workspace so several queries can be in flight at once.
#pragma once

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
    uint32_t* sout;         // [r][N2][2 comp][2 ch][N] DB-scan outputs, NTT form
    uint32_t* result;       // [r][2 comp][2 ch][N] first-dimension results, NTT form
    uint32_t* ecoef;        // [r][2 comp][2 ch][N] result, coefficient form
    uint32_t* ext;          // [r][2 comp][2 ch][N] external products, coefficient form
    uint32_t* ext2;         // [r/2][2 comp][2 ch][N] packing levels ping-pong with ext
    unsigned long long* gacc;  // [r][2 comp][2 ch][N] giant-step accumulators
    uint64_t* resp64;       // [2][N] response words
    int* err;               // device error word (bounded waits)
};

// Gadget parameters of the path (reference defaults; lwe.h:391-404, test-pir.cpp:71, :88).
struct PathGadgets {
    GadgetBsgs baby;   // ell 3, base 2^20, Bg 2^20
    GadgetB giant;     // ell 2, base 2^20, Bg 2^18
    GadgetS ext;       // ell 2, base 2^20, Bg 2^18 (signed)
    GadgetB pack;      // ell 4, base 0,    Bg 2^14
};

}  // namespace kspir
