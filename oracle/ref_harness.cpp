// TEST INFRASTRUCTURE ONLY -- part of the CPU oracle, never part of the product.
//
// A C-callable harness around the UNMODIFIED KsPIR reference sources
// (compiled from where they lie by oracle/Makefile, against the HEXL
// restatement in oracle/hexl_shim).  It lets the Python tests
//   * replay tests/test-pir.cpp's whole protocol (same rand() stream, same
//     keygen, same database preprocessing) and read its inputs back out in the
//     flat layout of include/kspir_b200.h, to pin known answers;
//   * run the reference's own answer functions
//       matrix_vector_mul_bsgs_rns_crt_large  (reference src/twosteps.cpp:1527)
//       externalProduct                       (reference src/lwe.cpp:761)
//       packingRLWEs                          (reference src/answer.cpp:800)
//     on caller-supplied inputs, so the CUDA path and the C restatement in
//     oracle/kspir_oracle.c can be compared word for word;
//   * time that answer on the host cores (the "reference" CPU baseline).
//
// Flat layouts (u64 words, N = 4096):
//   query    [2 moduli (crtMod, bsMod)][2 comps (a, b)][N]
//   baby     [N1/2][6 (3 crtMod rows, 3 bsMod rows)][2][N]   index i <-> 5^(i+1) mod 2N
//   giant    [N2-1][2][2][N]                                  index c <-> 5^(N1*(c+1)) mod 2N
//   packing  [log2 r][4][2][N]                                level l <-> N/2^l + 1
//   rgsw     [4][2][N]
//   perms    [N1][N] int32
//   result   [r][2][N] (NTT form), ext [r][2][N] (coefficient form), response [2][N]
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <chrono>
#include <vector>

#include "pir.h"
#include "crt.h"

namespace {

const size_t kPoly = N;

void load_rlwe(RlweCiphertext& c, const uint64_t* p, bool is_ntt) {
    memcpy(c.a.data(), p, kPoly * 8);
    memcpy(c.b.data(), p + kPoly, kPoly * 8);
    c.setIsNtt(is_ntt);
}

void store_rlwe(uint64_t* p, const RlweCiphertext& c) {
    memcpy(p, c.a.data(), kPoly * 8);
    memcpy(p + kPoly, c.b.data(), kPoly * 8);
}

int ilog2(int v) { int l = 0; while ((1 << l) < v) l++; return l; }

// Builds the reference key objects from flat arrays.
struct RefKeys {
    AutoKeyBSGSRNS autoKey{N, crtMod, bsMod};
    AutoKey packingKey{N, crtMod, 4, 0, 0x01 << 14};
    RGSWCiphertext gsw{N, crtMod, 2, 0x01 << 20, 0x01 << 18};

    RefKeys(int r, int N1, const uint64_t* baby, const uint64_t* giant,
            const uint64_t* packing, const uint64_t* rgsw) {
        int N2 = N / 2 / N1;
        for (int i = 1; baby && i <= N1 / 2; i++) {
            std::vector<RlweCiphertext> v(3, RlweCiphertext(N, crtMod));
            for (int j = 0; j < 3; j++) v.push_back(RlweCiphertext(N, bsMod));
            for (int j = 0; j < 6; j++)
                load_rlwe(v[j], baby + ((size_t)(i - 1) * 6 + j) * 2 * kPoly, true);
            autoKey.keyMap.insert(std::make_pair(pow_mod(5, i, 2 * N), v));
        }
        for (int c = 1; giant && c < N2; c++) {
            std::vector<RlweCiphertext> v(2, RlweCiphertext(N, crtMod));
            for (int j = 0; j < 2; j++)
                load_rlwe(v[j], giant + ((size_t)(c - 1) * 2 + j) * 2 * kPoly, true);
            autoKey.keyMap.insert(std::make_pair(pow_mod(5, N1 * c, 2 * N), v));
        }
        int levels = packing ? ilog2(r) : 0;
        for (int l = 0; l < levels; l++) {
            std::vector<RlweCiphertext> v(4, RlweCiphertext(N, crtMod));
            for (int j = 0; j < 4; j++)
                load_rlwe(v[j], packing + ((size_t)l * 4 + j) * 2 * kPoly, true);
            packingKey.keyMap.insert(std::make_pair(N / (1 << l) + 1, v));
        }
        // RGSWCiphertext only marks itself NTT-form inside keyGen (lwe.cpp:297-352),
        // and externalProduct asserts that flag; run keyGen on a throwaway secret
        // with a private rand() state, then overwrite every row.
        {
            Secret junk(crtMod, false);
            gsw.keyGen(junk, 0, true);
        }
        for (int j = 0; j < 4; j++) {
            memcpy(gsw.a[j].data(), rgsw + (size_t)j * 2 * kPoly, kPoly * 8);
            memcpy(gsw.b[j].data(), rgsw + (size_t)j * 2 * kPoly + kPoly, kPoly * 8);
        }
    }
};

// State of one replay of tests/test-pir.cpp.
struct PirState {
    int r = 0, N1 = 0;
    uint32_t target_col = 0, target_packing = 0;
    std::vector<uint64_t> datacrt;
    Secret* key = nullptr;
    std::vector<uint64_t> query, baby, giant, packing, rgsw;
    std::vector<int32_t> perms;
    std::vector<uint64_t> raw;   // the sampled database before preprocessing (kept on request)
};
bool g_keep_raw = false;
PirState g_state;

}  // namespace

extern "C" {

// Replays tests/test-pir.cpp:12-93 (database, query, keys, permutations) after
// srand(seed); seed 1 is the driver's own state (it never calls srand).
int ref_pir_setup(uint32_t seed, int r, int N1) {
    srand(seed);
    PirState& s = g_state;
    delete s.key;
    s = PirState();
    s.r = r; s.N1 = N1;
    int N2 = N / 2 / N1;
    s.key = new Secret(crtMod, false);                      // test-pir.cpp:20
    s.target_col = rand() % (N / 2);                        // :23
    s.target_packing = rand() % r;                          // :24

    size_t num_words = (size_t)N * N / 2;
    s.datacrt.assign(num_words * r, 0);
    std::vector<std::vector<uint64_t> > data(N, std::vector<uint64_t>(N / 2, 0));
    std::vector<std::vector<uint64_t> > data_ntt(N / 2, std::vector<uint64_t>(N, 0));
    std::vector<uint64_t> input_record(N);
    for (int k = 0; k < r; k++) {                           // :46-63
        sample_database_bsgs(data);
        for (size_t i = 0; i < (size_t)N; i += r) data[i + s.target_packing][s.target_col] = i + 1 + k;
        for (size_t i = 0; i < (size_t)N; i++) input_record[i] = data[i][s.target_col];
        inverse_encode(input_record);
        for (size_t i = 0; i < (size_t)N; i++) data[i][s.target_col] = input_record[i];
        if (g_keep_raw) {
            s.raw.resize(num_words * (k + 1));
            for (size_t i = 0; i < (size_t)N; i++)
                memcpy(s.raw.data() + num_words * k + i * (N / 2), data[i].data(), (N / 2) * 8);
        }
        database_tobsgsntt(data_ntt, data, crtMod, N1);
        database_tocrt(s.datacrt.data() + num_words * k, data_ntt, N1);
    }

    std::vector<RlweCiphertext> query1(1, RlweCiphertext(N, crtMod));   // :68-75
    query1.push_back(RlweCiphertext(N, bsMod));
    RGSWCiphertext queryGsw(N, crtMod, 2, 0x01 << 20, 0x01 << 18);
    query_bsgs_rns(query1, *s.key, s.target_col);
    queryGsw.keyGen(*s.key, s.target_packing, true);

    AutoKeyBSGSRNS autoKey(N, crtMod, bsMod);                           // :84-89
    autoKey.bsgsKeyGen(*s.key, N1);
    AutoKey packingKey(N, crtMod, 4, 0, 0x01 << 14);
    packingKey.keyGen(*s.key, r, true);

    std::vector<std::vector<int32_t> > permutations(N1, std::vector<int32_t>(N, 0));   // :92-93
    compute_permutation_matrix(permutations, N1, N);

    s.query.assign(4 * kPoly, 0);
    store_rlwe(s.query.data(), query1[0]);
    store_rlwe(s.query.data() + 2 * kPoly, query1[1]);
    s.baby.assign((size_t)(N1 / 2) * 6 * 2 * kPoly, 0);
    for (int i = 1; i <= N1 / 2; i++) {
        const std::vector<RlweCiphertext>& v = autoKey.keyMap.at(pow_mod(5, i, 2 * N));
        for (int j = 0; j < 6; j++) store_rlwe(s.baby.data() + ((size_t)(i - 1) * 6 + j) * 2 * kPoly, v[j]);
    }
    s.giant.assign((size_t)(N2 - 1) * 2 * 2 * kPoly, 0);
    for (int c = 1; c < N2; c++) {
        const std::vector<RlweCiphertext>& v = autoKey.keyMap.at(pow_mod(5, N1 * c, 2 * N));
        for (int j = 0; j < 2; j++) store_rlwe(s.giant.data() + ((size_t)(c - 1) * 2 + j) * 2 * kPoly, v[j]);
    }
    int levels = ilog2(r);
    s.packing.assign((size_t)levels * 4 * 2 * kPoly, 0);
    for (int l = 0; l < levels; l++) {
        const std::vector<RlweCiphertext>& v = packingKey.keyMap.at(N / (1 << l) + 1);
        for (int j = 0; j < 4; j++) store_rlwe(s.packing.data() + ((size_t)l * 4 + j) * 2 * kPoly, v[j]);
    }
    s.rgsw.assign(4 * 2 * kPoly, 0);
    for (int j = 0; j < 4; j++) {
        memcpy(s.rgsw.data() + (size_t)j * 2 * kPoly, queryGsw.a[j].data(), kPoly * 8);
        memcpy(s.rgsw.data() + (size_t)j * 2 * kPoly + kPoly, queryGsw.b[j].data(), kPoly * 8);
    }
    s.perms.assign((size_t)N1 * kPoly, 0);
    for (int i = 0; i < N1; i++) memcpy(s.perms.data() + (size_t)i * kPoly, permutations[i].data(), kPoly * 4);
    return 0;
}

// The test-pir secret in coefficient form mod crtMod (Secret::data).
void ref_pir_get_secret(uint64_t* s) {
    if (g_state.key->isNttForm()) g_state.key->toCoeffForm();
    std::vector<uint64_t> d = g_state.key->getData();
    memcpy(s, d.data(), kPoly * 8);
}

// decrypt_bsgs_total (twosteps.cpp:388-418) of a coefficient-form response
// under the test-pir secret with packing number r.
void ref_pir_decrypt_r(const uint64_t* response, int r, uint64_t* message) {
    RlweCiphertext c(N, crtMod);
    load_rlwe(c, response, false);
    std::vector<uint64_t> m(N);
    decrypt_bsgs_total(m, c, *g_state.key, r);
    memcpy(message, m.data(), kPoly * 8);
}

// Keep (1) the sampled database of the next ref_pir_setup before preprocessing.
void ref_pir_keep_raw(int keep) { g_keep_raw = keep != 0; }

// The kept database: [r][N][N/2], data[i][j] of sub-database k at (k N + i) N/2 + j.
void ref_pir_get_raw(uint64_t* raw) {
    if (raw && !g_state.raw.empty()) memcpy(raw, g_state.raw.data(), g_state.raw.size() * 8);
}

// database_tobsgsntt + database_tocrt of every sub-database, as
// tests/test-pir.cpp:59-60 calls them: raw [r][N][N/2] -> datacrt [r][N][N/2].
void ref_db_preprocess(const uint64_t* raw, int r, int N1, uint64_t* datacrt) {
    const size_t num_words = (size_t)N * N / 2;
    std::vector<std::vector<uint64_t> > data(N, std::vector<uint64_t>(N / 2, 0));
    std::vector<std::vector<uint64_t> > data_ntt(N / 2, std::vector<uint64_t>(N, 0));
    for (int k = 0; k < r; k++) {
        for (size_t i = 0; i < (size_t)N; i++)
            memcpy(data[i].data(), raw + num_words * k + i * (N / 2), (N / 2) * 8);
        database_tobsgsntt(data_ntt, data, crtMod, N1);
        database_tocrt(datacrt + num_words * k, data_ntt, N1);
    }
}

// database_tobsgsntt alone: raw [N][N/2] -> rows [N/2][N] (its `result`).
void ref_database_tobsgsntt(const uint64_t* raw, int N1, uint64_t* rows) {
    std::vector<std::vector<uint64_t> > data(N, std::vector<uint64_t>(N / 2, 0));
    std::vector<std::vector<uint64_t> > data_ntt(N / 2, std::vector<uint64_t>(N, 0));
    for (size_t i = 0; i < (size_t)N; i++) memcpy(data[i].data(), raw + i * (N / 2), (N / 2) * 8);
    database_tobsgsntt(data_ntt, data, crtMod, N1);
    for (size_t i = 0; i < (size_t)N / 2; i++) memcpy(rows + i * N, data_ntt[i].data(), N * 8);
}

// database_tocrt alone: rows [N/2][N] -> datacrt [N][N/2].
void ref_database_tocrt(const uint64_t* rows, int N1, uint64_t* datacrt) {
    std::vector<std::vector<uint64_t> > data_ntt(N / 2, std::vector<uint64_t>(N, 0));
    for (size_t i = 0; i < (size_t)N / 2; i++) memcpy(data_ntt[i].data(), rows + i * N, N * 8);
    database_tocrt(datacrt, data_ntt, N1);
}

void ref_pir_target(uint32_t* col, uint32_t* packing_slot) {
    *col = g_state.target_col;
    *packing_slot = g_state.target_packing;
}

void ref_pir_get_inputs(uint64_t* datacrt, uint64_t* query, uint64_t* baby, uint64_t* giant,
                        uint64_t* packing, uint64_t* rgsw, int32_t* perms) {
    const PirState& s = g_state;
    if (datacrt) memcpy(datacrt, s.datacrt.data(), s.datacrt.size() * 8);
    if (query) memcpy(query, s.query.data(), s.query.size() * 8);
    if (baby) memcpy(baby, s.baby.data(), s.baby.size() * 8);
    if (giant) memcpy(giant, s.giant.data(), s.giant.size() * 8);
    if (packing) memcpy(packing, s.packing.data(), s.packing.size() * 8);
    if (rgsw) memcpy(rgsw, s.rgsw.data(), s.rgsw.size() * 8);
    if (perms) memcpy(perms, s.perms.data(), s.perms.size() * 4);
}

// decrypt_bsgs_total (twosteps.cpp:388-418) of a coefficient-form response.
void ref_pir_decrypt(const uint64_t* response, uint64_t* message) {
    RlweCiphertext c(N, crtMod);
    load_rlwe(c, response, false);
    std::vector<uint64_t> m(N);
    decrypt_bsgs_total(m, c, *g_state.key, g_state.r);
    memcpy(message, m.data(), kPoly * 8);
}

// The server's online answer, test-pir.cpp:110-116, on caller-supplied inputs.
// query is read (and, like the reference, modswitched in a private copy).
// bsgs_out / ext_out may be null; seconds receives the wall time of the three calls.
int ref_answer(const uint64_t* datacrt, int r, int N1, const uint64_t* query,
               const uint64_t* baby, const uint64_t* giant, const uint64_t* packing,
               const uint64_t* rgsw, const int32_t* perms, uint64_t* response,
               uint64_t* bsgs_out, uint64_t* ext_out, double* seconds) {
    RefKeys keys(r, N1, baby, giant, packing, rgsw);
    std::vector<std::vector<int32_t> > permutations(N1, std::vector<int32_t>(N, 0));
    for (int i = 0; i < N1; i++) memcpy(permutations[i].data(), perms + (size_t)i * kPoly, kPoly * 4);
    std::vector<RlweCiphertext> query1(1, RlweCiphertext(N, crtMod));
    query1.push_back(RlweCiphertext(N, bsMod));
    load_rlwe(query1[0], query, false);
    load_rlwe(query1[1], query + 2 * kPoly, false);
    std::vector<RlweCiphertext> result(r, RlweCiphertext(N, crtMod));
    RlweCiphertext result_output(N, crtMod);
    std::vector<RlweCiphertext> ext_rlwes;
    for (int i = 0; i < r; i++) ext_rlwes.push_back(RlweCiphertext(N, crtMod));
    uint64_t* data = const_cast<uint64_t*>(datacrt);

    auto start = std::chrono::high_resolution_clock::now();
    matrix_vector_mul_bsgs_rns_crt_large(result, query1, data, keys.autoKey, N1, permutations, r);
    if (bsgs_out)
        for (int j = 0; j < r; j++) store_rlwe(bsgs_out + (size_t)j * 2 * kPoly, result[j]);
    for (int j = 0; j < r; j++) externalProduct(ext_rlwes[j], result[j], keys.gsw);
    if (ext_out)
        for (int j = 0; j < r; j++) store_rlwe(ext_out + (size_t)j * 2 * kPoly, ext_rlwes[j]);
    packingRLWEs(result_output, ext_rlwes, keys.packingKey);
    auto stop = std::chrono::high_resolution_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(stop - start).count();
    store_rlwe(response, result_output);
    return 0;
}

// matrix_vector_mul_bsgs_rns_crt_large alone.  query_inout is modswitched in
// place exactly as the reference does to its input (twosteps.cpp:1073-1086).
int ref_matrix_vector_mul(const uint64_t* datacrt, int r, int N1, uint64_t* query_inout,
                          const uint64_t* baby, const uint64_t* giant, const int32_t* perms,
                          uint64_t* result) {
    uint64_t dummy_pk[1] = {0};
    std::vector<uint64_t> rgsw(4 * 2 * kPoly, 0);
    RefKeys keys(1, N1, baby, giant, dummy_pk, rgsw.data());
    std::vector<std::vector<int32_t> > permutations(N1, std::vector<int32_t>(N, 0));
    for (int i = 0; i < N1; i++) memcpy(permutations[i].data(), perms + (size_t)i * kPoly, kPoly * 4);
    std::vector<RlweCiphertext> query1(1, RlweCiphertext(N, crtMod));
    query1.push_back(RlweCiphertext(N, bsMod));
    load_rlwe(query1[0], query_inout, false);
    load_rlwe(query1[1], query_inout + 2 * kPoly, false);
    std::vector<RlweCiphertext> res(r, RlweCiphertext(N, crtMod));
    matrix_vector_mul_bsgs_rns_crt_large(res, query1, const_cast<uint64_t*>(datacrt),
                                         keys.autoKey, N1, permutations, r);
    for (int j = 0; j < r; j++) store_rlwe(result + (size_t)j * 2 * kPoly, res[j]);
    store_rlwe(query_inout, query1[0]);
    store_rlwe(query_inout + 2 * kPoly, query1[1]);
    return 0;
}

// externalProduct alone: ext_inout += g^-1(first_dim) * rgsw, first_dim is
// NTT form on entry and (like the reference) coefficient form on exit.
int ref_external_product(uint64_t* ext_inout, uint64_t* first_dim_inout, const uint64_t* rgsw) {
    uint64_t dummy[1] = {0};
    RefKeys keys(1, 128, nullptr, nullptr, dummy, rgsw);
    RlweCiphertext res(N, crtMod), fd(N, crtMod);
    load_rlwe(res, ext_inout, false);
    load_rlwe(fd, first_dim_inout, true);
    externalProduct(res, fd, keys.gsw);
    store_rlwe(ext_inout, res);
    store_rlwe(first_dim_inout, fd);
    return 0;
}

// packingRLWEs alone on r coefficient-form ciphertexts (rlwes_inout is overwritten).
int ref_packing(uint64_t* rlwes_inout, int r, const uint64_t* packing, uint64_t* response) {
    std::vector<uint64_t> rgsw(4 * 2 * kPoly, 0);
    RefKeys keys(r, 128, nullptr, nullptr, packing, rgsw.data());
    std::vector<RlweCiphertext> rl;
    for (int i = 0; i < r; i++) {
        rl.push_back(RlweCiphertext(N, crtMod));
        load_rlwe(rl.back(), rlwes_inout + (size_t)i * 2 * kPoly, false);
    }
    RlweCiphertext out(N, crtMod);
    packingRLWEs(out, rl, keys.packingKey);
    for (int i = 0; i < r; i++) store_rlwe(rlwes_inout + (size_t)i * 2 * kPoly, rl[i]);
    store_rlwe(response, out);
    return 0;
}

// fastMultiplyQueryByDatabaseDim1InvCRT (crt.cpp:643) on one sub-database.
void ref_scan(const uint64_t* db, const uint64_t* cipherbuf, int N1, uint64_t* out /* [N2][2N] */) {
    int N2 = N / 2 / N1;
    std::vector<std::vector<uint64_t> > output(N2, std::vector<uint64_t>(2 * N, 0));
    fastMultiplyQueryByDatabaseDim1InvCRT(output, db, cipherbuf, N1, N2);
    for (int i = 0; i < N2; i++) memcpy(out + (size_t)i * 2 * kPoly, output[i].data(), 2 * kPoly * 8);
}

uint64_t ref_crt_compose(uint64_t x, uint64_t y) { return crt_compose(x, y); }

void ref_permutation_matrix(int32_t* perms, int N1) {
    std::vector<std::vector<int32_t> > p(N1, std::vector<int32_t>(N, 0));
    compute_permutation_matrix(p, N1, N);
    for (int i = 0; i < N1; i++) memcpy(perms + (size_t)i * kPoly, p[i].data(), kPoly * 4);
}

// HEXL-shim transforms, exposed so the oracle's own NTT can be compared.
void ref_ntt(uint64_t* data, uint64_t modulus, int inverse) {
    intel::hexl::NTT t = modulus == crtMod ? intel::hexl::NTT(N, crtMod, root_of_unity_crt)
                                           : intel::hexl::NTT(N, modulus);
    if (inverse) t.ComputeInverse(data, data, 1, 1);
    else t.ComputeForward(data, data, 1, 1);
}

void ref_decompose_bsgs(const uint64_t* a_crt, const uint64_t* a_bs, uint64_t* d_crt, uint64_t* d_bs) {
    std::vector<std::vector<uint64_t> > r1(3, std::vector<uint64_t>(N)), r2(3, std::vector<uint64_t>(N));
    std::vector<uint64_t> i1(a_crt, a_crt + N), i2(a_bs, a_bs + N);
    decompose_bsgs(r1, r2, i1, i2, 3, 0x01 << 20, 0x01 << 20);
    for (int j = 0; j < 3; j++) {
        memcpy(d_crt + (size_t)j * kPoly, r1[j].data(), kPoly * 8);
        memcpy(d_bs + (size_t)j * kPoly, r2[j].data(), kPoly * 8);
    }
}

void ref_decompose(const uint64_t* in, int ellnum, uint64_t base, uint64_t bg, uint64_t* out) {
    std::vector<std::vector<uint64_t> > r(ellnum, std::vector<uint64_t>(N));
    std::vector<uint64_t> i1(in, in + N);
    decompose(r, i1, ellnum, base, bg, crtMod);
    for (int j = 0; j < ellnum; j++) memcpy(out + (size_t)j * kPoly, r[j].data(), kPoly * 8);
}

void ref_decompose_rlwe(const uint64_t* a, const uint64_t* b, int ellnum, uint64_t base, uint64_t bg,
                        uint64_t* out) {
    std::vector<std::vector<uint64_t> > r(2 * ellnum, std::vector<uint64_t>(N));
    std::vector<uint64_t> i1(a, a + N), i2(b, b + N);
    decompose_rlwe(r, i1, i2, ellnum, base, bg, crtMod);
    for (int j = 0; j < 2 * ellnum; j++) memcpy(out + (size_t)j * kPoly, r[j].data(), kPoly * 8);
}

// ---------------------------------------------------------------------------
// Offline key derivation (reference genAutoKeyFromOffline, twosteps.cpp:1749-1864,
// evalAutoRNSKey :1587-1743) with the key parameters of
// tests/test-two-steps-key.cpp:149-155.  The caller supplies the four input
// keys (any words canonical for their moduli: the derivation is arithmetic on
// them; the test's own key generation needs HEXL's default NTT root for the
// composite crtBaMod, which HEXL draws at random).  Layouts (u64 words):
//   offline1 [10][2][N]  offlineKey1.keyMap[5]: rows 0-4 mod crtMod, 5-9 mod crtBaMod, NTT form
//   offline2 [10][2][N]  offlineKey2.keyMap[5^N1]: rows 0-4 mod crtMod, 5-9 mod auxMod
//   auto1    [6][2][N]   autoKey1.keyMap[5]: rows 0-2 mod crtMod, 3-5 mod crtBaMod
//   auto2    [6][2][N]   autoKey2.keyMap[5^N1]: rows 0-2 mod crtMod, 3-5 mod auxMod
//   chain1   [N1-2][6][2][N]  autoKey1.keyMap[5^i], i = 2..N1-1, after the derivation
//   chain2   [N2-2][6][2][N]  autoKey2.keyMap[5^(N1 i)], i = 2..N2-1
//   baby_out [N1-1][6][2][N]  result.keyMap[5^i], i = 1..N1-1
//   giant_out [N2-1][3][2][N] result.keyMap[5^(N1 i)], i = 1..N2-1

namespace {

// (params.h defines `ell` as a macro: the row count is `rows` here)
std::vector<RlweCiphertext> flat_to_keys(const uint64_t* p, int rows, uint64_t m1, uint64_t m2) {
    std::vector<RlweCiphertext> v(rows, RlweCiphertext(N, m1));
    for (int j = 0; j < rows; j++) v.push_back(RlweCiphertext(N, m2));
    for (int j = 0; j < 2 * rows; j++) load_rlwe(v[j], p + (size_t)j * 2 * kPoly, true);
    return v;
}

void keys_to_flat(uint64_t* p, const std::vector<RlweCiphertext>& v) {
    for (size_t j = 0; j < v.size(); j++) store_rlwe(p + j * 2 * kPoly, v[j]);
}

}  // namespace

// genAutoKeyFromOffline(result, autoKey1, autoKey2, offlineKey1, offlineKey2, N1)
// on key objects rebuilt from the flat inputs (NTT form, as keyGen leaves them).
void ref_gen_autokey_from_offline(int N1, const uint64_t* offline1, const uint64_t* offline2, const uint64_t* auto1,
                                  const uint64_t* auto2, uint64_t* chain1, uint64_t* chain2, uint64_t* baby_out,
                                  uint64_t* giant_out, double* seconds) {
    const int N2 = N / 2 / N1;
    AutoKeyBSGSRNS offlineKey1(N, crtMod, crtBaMod, 5, 0x01 << 18, 0x01 << 18);
    AutoKeyBSGSRNS offlineKey2(N, crtMod, auxMod, 5, 0x01 << 14, 0x01 << 14);
    AutoKeyBSGSRNS autoKey1(N, crtMod, crtBaMod, 3, (0x01 << 20) * auxMod, 0x01 << 20);
    AutoKeyBSGSRNS autoKey2(N, crtMod, auxMod, 3, (0x01 << 11) * auxMod, 0x01 << 15);
    const int32_t i1 = pow_mod(5, 1, 2 * N), iN1 = pow_mod(5, N1, 2 * N);
    offlineKey1.keyMap.insert(std::make_pair(i1, flat_to_keys(offline1, 5, crtMod, crtBaMod)));
    offlineKey2.keyMap.insert(std::make_pair(iN1, flat_to_keys(offline2, 5, crtMod, auxMod)));
    autoKey1.keyMap.insert(std::make_pair(i1, flat_to_keys(auto1, 3, crtMod, crtBaMod)));
    autoKey2.keyMap.insert(std::make_pair(iN1, flat_to_keys(auto2, 3, crtMod, auxMod)));
    AutoKeyBSGSRNS result(N, crtMod, bsMod);
    auto t0 = std::chrono::high_resolution_clock::now();
    genAutoKeyFromOffline(result, autoKey1, autoKey2, offlineKey1, offlineKey2, N1);
    auto t1 = std::chrono::high_resolution_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    for (int i = 2; chain1 && i <= N1 - 1; i++)
        keys_to_flat(chain1 + (size_t)(i - 2) * 6 * 2 * kPoly, autoKey1.keyMap.at(pow_mod(5, i, 2 * N)));
    for (int i = 2; chain2 && i <= N2 - 1; i++)
        keys_to_flat(chain2 + (size_t)(i - 2) * 6 * 2 * kPoly, autoKey2.keyMap.at(pow_mod(5, N1 * i, 2 * N)));
    for (int i = 1; baby_out && i <= N1 - 1; i++)
        keys_to_flat(baby_out + (size_t)(i - 1) * 6 * 2 * kPoly, result.keyMap.at(pow_mod(5, i, 2 * N)));
    for (int i = 1; giant_out && i <= N2 - 1; i++)
        keys_to_flat(giant_out + (size_t)(i - 1) * 3 * 2 * kPoly, result.keyMap.at(pow_mod(5, N1 * i, 2 * N)));
}

}  // extern "C"
