// The reference's three server-answer functions, implemented over the C ABI
// of libkspir_b200 so that a program written against the reference (for
// example its tests/test-pir.cpp) runs its online answer on the GPU unchanged:
//
//   matrix_vector_mul_bsgs_rns_crt_large   reference src/twosteps.h:55-57
//   externalProduct                        reference src/lwe.h:292
//   packingRLWEs                           reference src/answer.h:79-80
//
// and the server preprocessing that builds the database those answers read:
//
//   database_tobsgsntt                     reference src/twosteps.h:19-20
//   database_tocrt                         reference src/crt.h:133
//
// Same signatures, argument meaning and in-place effects as the reference:
// input[0] is modswitched in place to NTT form and result[j] comes back in NTT
// form; externalProduct accumulates into `result` and returns both `result`
// and `firstDim` in coefficient form; packingRLWEs writes the packed response
// in coefficient form and leaves `rlwes` as the reference does (rlwes[0] =
// the response, rlwes[I + j] = X^I rlwes[I + j] + rlwes[j] of each merge).
//
// The database, permutations and key words stay resident on the device
// between calls.  Every call gathers the words of the key objects and of the
// permutations and compares them with the resident copy, so an object
// rewritten in place, or a new one built where a freed one lived, is uploaded
// again.  The database (1 GiB at r = 16) is recognised by its address and a
// fingerprint of 4096 words spread over it, which any re-preprocessing
// changes; a caller that edits a few datacrt words in place calls
// kspir_dropin_invalidate() before the next answer.
// The reference's functions return void and check only with assert; an error
// of the library here prints its message and aborts likewise.
//
// Built against the reference's headers, so it needs the reference tree:
// oracle/Makefile target `testpir-gpu` links it with the reference's objects.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "answer.h"
#include "crt.h"
#include "lwe.h"
#include "twosteps.h"

#include "kspir_b200.h"

namespace {

constexpr int kPoly = KSPIR_N;

struct Session {
    kspir_ctx* ctx = nullptr;
    int r = 0, N1 = 0;
    const uint64_t* db = nullptr;
    std::vector<uint64_t> db_sample;   // fingerprint of the resident database
    std::vector<int32_t> perms;        // resident permutations (empty: none)
    std::vector<uint64_t> baby, giant, packing, rgsw;   // words of client slot 0
    bool keys_uploaded = false;
};
Session g;

constexpr size_t kDbSample = 4096;

std::vector<uint64_t> db_fingerprint(const uint64_t* data, size_t words) {
    std::vector<uint64_t> f(kDbSample);
    for (size_t i = 0; i < kDbSample; i++) f[i] = data[i * (words - 1) / (kDbSample - 1)];
    return f;
}

// dst (the resident copy) := src; true if any word differed
bool gather(uint64_t* dst, const uint64_t* src, size_t words) {
    if (memcmp(dst, src, words * 8) == 0) return false;
    memcpy(dst, src, words * 8);
    return true;
}

void check(const char* what, int rc) {
    if (rc == KSPIR_OK) return;
    fprintf(stderr, "kspir_b200: %s: %s (%s)\n", what, kspir_strerror(rc),
            kspir_last_error(g.ctx ? g.ctx : nullptr));
    abort();
}

int log2i(int v) {
    int l = 0;
    while ((1 << l) < v) l++;
    return l;
}

uint32_t pow5_mod2n(long e) {
    uint64_t r = 1, b = 5, m = 2 * (uint64_t)kPoly;
    while (e > 0) {
        if (e & 1) r = r * b % m;
        b = b * b % m;
        e >>= 1;
    }
    return (uint32_t)r;
}

void put_rlwe(uint64_t* dst, const RlweCiphertext& c) {
    memcpy(dst, c.a.data(), kPoly * 8);
    memcpy(dst + kPoly, c.b.data(), kPoly * 8);
}

bool gather_rlwe(uint64_t* dst, const RlweCiphertext& c) {
    const bool ca = gather(dst, c.a.data(), kPoly);
    const bool cb = gather(dst + kPoly, c.b.data(), kPoly);
    return ca || cb;
}

void get_rlwe(RlweCiphertext& c, const uint64_t* src) {
    c.a.assign(src, src + kPoly);
    c.b.assign(src + kPoly, src + 2 * kPoly);
}

// a context for (r, N1); the key words start as zeros until their objects arrive
void ensure(int r, int N1) {
    if (g.ctx && g.r == r && g.N1 == N1) return;
    if (g.ctx) kspir_ctx_destroy(g.ctx);
    g = Session();
    kspir_params p;
    p.r = r;
    p.N1 = N1;
    p.max_clients = 1;
    p.max_inflight = 1;
    check("kspir_ctx_create", kspir_ctx_create(0, &p, &g.ctx));
    g.r = r;
    g.N1 = N1;
    const int N2 = kPoly / 2 / N1;
    g.baby.assign((size_t)(N1 / 2) * 6 * 2 * kPoly, 0);
    g.giant.assign((size_t)(N2 - 1) * 2 * 2 * kPoly, 0);
    g.packing.assign((size_t)log2i(r) * 4 * 2 * kPoly, 0);
    g.rgsw.assign((size_t)4 * 2 * kPoly, 0);
}

void upload_keys(bool changed) {
    if (!changed && g.keys_uploaded) return;
    check("kspir_client_keys_upload",
          kspir_client_keys_upload(g.ctx, 0, g.baby.data(), g.giant.empty() ? nullptr : g.giant.data(),
                                   g.packing.empty() ? nullptr : g.packing.data(), g.rgsw.data()));
    g.keys_uploaded = true;
}

// The preprocessing runs in a context of its own (one sub-database at a time,
// N1 of the call), so it never disturbs the answer session's resident data.
struct PrepSession {
    kspir_ctx* ctx = nullptr;
    int N1 = 0;
    std::vector<uint64_t> in, out;   // flat copies of one sub-database
};
PrepSession gp;

void ensure_prep(int N1) {
    if (gp.ctx && gp.N1 == N1) return;
    if (gp.ctx) kspir_ctx_destroy(gp.ctx);
    gp.ctx = nullptr;
    kspir_params p;
    p.r = 1;
    p.N1 = N1;
    p.max_clients = 1;
    p.max_inflight = 1;
    int rc = kspir_ctx_create(0, &p, &gp.ctx);
    if (rc != KSPIR_OK) {
        fprintf(stderr, "kspir_b200: kspir_ctx_create: %s (%s)\n", kspir_strerror(rc), kspir_last_error(nullptr));
        abort();
    }
    gp.N1 = N1;
    gp.in.resize((size_t)kPoly * (kPoly / 2));
    gp.out.resize((size_t)kPoly * (kPoly / 2));
}

void check_prep(const char* what, int rc) {
    if (rc == KSPIR_OK) return;
    fprintf(stderr, "kspir_b200: %s: %s (%s)\n", what, kspir_strerror(rc), kspir_last_error(gp.ctx));
    abort();
}

}  // namespace

void database_tobsgsntt(std::vector<std::vector<uint64_t> >& result, std::vector<std::vector<uint64_t> >& data,
                        uint64_t modulus, int32_t N1) {
    // the reference lifts to modulus and transforms mod crtMod (USE_CRTMOD):
    // the device path implements the combination the reference's callers use
    if (modulus != crtMod) {
        fprintf(stderr, "kspir_b200: database_tobsgsntt: only modulus = crtMod is supported\n");
        abort();
    }
    ensure_prep(N1);
    const size_t H = kPoly / 2;
    for (size_t i = 0; i < (size_t)kPoly; i++) memcpy(gp.in.data() + i * H, data[i].data(), H * 8);
    check_prep("kspir_database_tobsgsntt", kspir_database_tobsgsntt(gp.ctx, gp.in.data(), gp.out.data()));
    for (size_t i = 0; i < H; i++) memcpy(result[i].data(), gp.out.data() + i * kPoly, kPoly * 8);
}

void database_tocrt(uint64_t* datacrt, std::vector<std::vector<uint64_t> >& data_ntt, int32_t N1) {
    ensure_prep(N1);
    const size_t H = kPoly / 2;
    for (size_t i = 0; i < H; i++) memcpy(gp.in.data() + i * kPoly, data_ntt[i].data(), kPoly * 8);
    check_prep("kspir_database_tocrt", kspir_database_tocrt(gp.ctx, gp.in.data(), datacrt));
}

void matrix_vector_mul_bsgs_rns_crt_large(std::vector<RlweCiphertext>& result, std::vector<RlweCiphertext>& input,
                                          uint64_t* data, const AutoKeyBSGSRNS& autoKey, const int32_t N1,
                                          std::vector<std::vector<int32_t> >& permutations, int32_t r) {
    ensure(r, N1);
    const int N2 = kPoly / 2 / N1;
    const size_t db_words = (size_t)r * kPoly * (kPoly / 2);
    std::vector<uint64_t> fp = db_fingerprint(data, db_words);
    if (g.db != data || g.db_sample != fp) {
        check("kspir_db_upload", kspir_db_upload(g.ctx, data, db_words));
        g.db = data;
        g.db_sample.swap(fp);
    }
    std::vector<int32_t> flat((size_t)N1 * kPoly);
    for (int i = 0; i < N1; i++) memcpy(flat.data() + (size_t)i * kPoly, permutations[i].data(), kPoly * 4);
    if (flat != g.perms) {
        check("kspir_perms_upload", kspir_perms_upload(g.ctx, flat.data(), flat.size()));
        g.perms.swap(flat);
    }
    // baby keys keyMap[5^i], i = 1..N1/2 (six RLWEs each: crtMod rows, then bsMod
    // rows); giant keys keyMap[5^(N1 c)], c = 1..N2-1 (two RLWEs each)
    bool changed = false;
    for (int i = 1; i <= N1 / 2; i++) {
        const std::vector<RlweCiphertext>& v = autoKey.keyMap.at((int32_t)pow5_mod2n(i));
        for (int j = 0; j < 6; j++)
            changed |= gather_rlwe(g.baby.data() + ((size_t)(i - 1) * 6 + j) * 2 * kPoly, v[j]);
    }
    for (int c = 1; c < N2; c++) {
        const std::vector<RlweCiphertext>& v = autoKey.keyMap.at((int32_t)pow5_mod2n((long)N1 * c));
        for (int j = 0; j < 2; j++) changed |= gather_rlwe(g.giant.data() + ((size_t)(c - 1) * 2 + j) * 2 * kPoly, v[j]);
    }
    upload_keys(changed);
    std::vector<uint64_t> q(4 * kPoly), res((size_t)r * 2 * kPoly);
    put_rlwe(q.data(), input[0]);
    put_rlwe(q.data() + 2 * kPoly, input[1]);
    check("kspir_matrix_vector_mul_bsgs_rns_crt_large",
          kspir_matrix_vector_mul_bsgs_rns_crt_large(g.ctx, 0, q.data(), res.data()));
    for (int j = 0; j < r; j++) {
        get_rlwe(result[j], res.data() + (size_t)j * 2 * kPoly);
        result[j].setIsNtt(true);
    }
    get_rlwe(input[0], q.data());
    input[0].setIsNtt(true);
}

void externalProduct(RlweCiphertext& result, RlweCiphertext& firstDim, const RGSWCiphertext& query) {
    if (!g.ctx) ensure(1, 128);
    bool changed = false;
    for (int j = 0; j < 4; j++) {
        changed |= gather(g.rgsw.data() + (size_t)j * 2 * kPoly, query.a[j].data(), kPoly);
        changed |= gather(g.rgsw.data() + (size_t)j * 2 * kPoly + kPoly, query.b[j].data(), kPoly);
    }
    upload_keys(changed);
    std::vector<uint64_t> acc(2 * kPoly), fd(2 * kPoly);
    put_rlwe(acc.data(), result);
    put_rlwe(fd.data(), firstDim);
    check("kspir_external_product", kspir_external_product(g.ctx, 0, acc.data(), fd.data(), 1));
    get_rlwe(result, acc.data());
    get_rlwe(firstDim, fd.data());
    result.setIsNtt(false);
    firstDim.setIsNtt(false);
}

void packingRLWEs(RlweCiphertext& result, std::vector<RlweCiphertext>& rlwes, const AutoKey& autokey) {
    const int r = (int)rlwes.size();
    if (!g.ctx || g.r != r) ensure(r, g.N1 ? g.N1 : 128);
    // keyMap[N/2^l + 1], l = 0..log2 r - 1, four RLWEs each
    bool changed = false;
    for (int l = 0; l < log2i(r); l++) {
        const std::vector<RlweCiphertext>& v = autokey.keyMap.at(kPoly / (1 << l) + 1);
        for (int j = 0; j < 4; j++) changed |= gather_rlwe(g.packing.data() + ((size_t)l * 4 + j) * 2 * kPoly, v[j]);
    }
    upload_keys(changed);
    std::vector<uint64_t> in((size_t)r * 2 * kPoly), out(2 * kPoly);
    for (int j = 0; j < r; j++) put_rlwe(in.data() + (size_t)j * 2 * kPoly, rlwes[j]);
    check("kspir_packing_rlwes", kspir_packing_rlwes(g.ctx, 0, in.data(), out.data()));
    get_rlwe(result, out.data());
    result.setIsNtt(false);
    // rlwes left as the reference's packing tree leaves them (answer.cpp:821-828)
    for (int j = 0; j < r; j++) {
        get_rlwe(rlwes[j], in.data() + (size_t)j * 2 * kPoly);
        rlwes[j].setIsNtt(false);
    }
}

// Not a reference function: forgets the resident database fingerprint, the
// permutations and the key words, so the next call uploads them again (for a
// caller that edited a few datacrt words in place).
extern "C" void kspir_dropin_invalidate(void) {
    g.db = nullptr;
    g.db_sample.clear();
    g.perms.clear();
    g.keys_uploaded = false;
}
