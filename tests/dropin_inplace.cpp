// Test program for the C++ drop-in (kspir_b200/cpp/reference_api.cpp): a
// caller written against the reference rewrites its objects in place between
// answers, at the same addresses, and every answer must follow the new words.
//
// Built by `make -C oracle dropin-inplace` exactly like test-pir-gpu (the
// reference's objects, its answer and preprocessing functions taken from the
// drop-in); run by tests/test_gpu_testpir_dropin.py.  The flow is the
// reference's tests/test-pir.cpp at r = 2 with two records planted in the
// target column: rows i + 0 hold i + 1 + k and rows i + 1 hold
// i + 1 + k + base (i a multiple of r, k the sub-database), so the RGSW query
// for packing slot p decrypts to j + 1 + p * base.
//   1. RGSW for slot 0                 -> expect j + 1
//   2. the same RGSW object re-keyed for slot 1 in place -> expect j + 1 + 5000
//   3. the database rebuilt in place with base 9000   -> expect j + 1 + 9000
//   4. packingRLWEs leaves ext_rlwes[0] equal to the response
#include <stdint.h>
#include <stdlib.h>

#include <cstdio>
#include <vector>

#include "crt.h"
#include "pir.h"

namespace {

const int32_t kR = 2;
const int32_t kN1 = 128;

void build_db(uint64_t* datacrt, uint32_t col, uint64_t base) {
    const size_t num_words = (size_t)N * N / 2;
    std::vector<std::vector<uint64_t> > data(N, std::vector<uint64_t>(N / 2, 0));
    std::vector<std::vector<uint64_t> > data_ntt(N / 2, std::vector<uint64_t>(N, 0));
    std::vector<uint64_t> record(N);
    for (int k = 0; k < kR; k++) {
        sample_database_bsgs(data);
        for (size_t i = 0; i < (size_t)N; i += kR) {
            data[i][col] = i + 1 + k;
            data[i + 1][col] = i + 1 + k + base;
        }
        for (size_t i = 0; i < (size_t)N; i++) record[i] = data[i][col];
        inverse_encode(record);
        for (size_t i = 0; i < (size_t)N; i++) data[i][col] = record[i];
        database_tobsgsntt(data_ntt, data, crtMod, kN1);
        database_tocrt(datacrt + num_words * k, data_ntt, kN1);
    }
}

}  // namespace

int main() {
    srand(7);
    Secret queryKey(crtMod, false);
    const uint32_t col = rand() % (N / 2);
    const size_t num_words = (size_t)N * N / 2;
    uint64_t* datacrt = (uint64_t*)aligned_alloc(64, sizeof(uint64_t) * num_words * kR);
    build_db(datacrt, col, 5000);

    RGSWCiphertext queryGsw(N, crtMod, 2, 0x01 << 20, 0x01 << 18);
    AutoKeyBSGSRNS autoKey(N, crtMod, bsMod);
    autoKey.bsgsKeyGen(queryKey, kN1);
    AutoKey packingKey(N, crtMod, 4, 0, 0x01 << 14);
    packingKey.keyGen(queryKey, kR, true);
    std::vector<std::vector<int32_t> > permutations(kN1, std::vector<int32_t>(N, 0));
    compute_permutation_matrix(permutations, kN1, N);

    int failures = 0;
    auto answer = [&](const char* what, uint64_t offset) {
        std::vector<RlweCiphertext> query1(1, RlweCiphertext(N, crtMod));
        query1.push_back(RlweCiphertext(N, bsMod));
        query_bsgs_rns(query1, queryKey, col);
        std::vector<RlweCiphertext> result(kR, RlweCiphertext(N, crtMod));
        std::vector<RlweCiphertext> ext_rlwes(kR, RlweCiphertext(N, crtMod));
        RlweCiphertext result_output(N, crtMod);
        matrix_vector_mul_bsgs_rns_crt_large(result, query1, datacrt, autoKey, kN1, permutations, kR);
        for (int j = 0; j < kR; j++) externalProduct(ext_rlwes[j], result[j], queryGsw);
        packingRLWEs(result_output, ext_rlwes, packingKey);
        int bad = 0;
        if (ext_rlwes[0].a != result_output.a || ext_rlwes[0].b != result_output.b) {
            printf("%s: rlwes[0] is not the response after packingRLWEs\n", what);
            bad++;
        }
        std::vector<uint64_t> msg(N);
        decrypt_bsgs_total(msg, result_output, queryKey, kR);   // (transforms result_output in place)
        for (int j = 0; j < N; j++)
            if (msg[j] != (uint64_t)j + 1 + offset) bad++;
        printf("%s: msg[0..2] = %lu %lu %lu, expected %lu ..., %d wrong\n", what, (unsigned long)msg[0],
               (unsigned long)msg[1], (unsigned long)msg[2], (unsigned long)(1 + offset), bad);
        failures += bad != 0;
    };

    queryGsw.keyGen(queryKey, 0, true);
    answer("slot 0", 0);
    queryGsw.keyGen(queryKey, 1, true);   // same object, words rewritten in place
    answer("slot 1, RGSW rewritten in place", 5000);
    build_db(datacrt, col, 9000);          // same buffer, new database
    answer("slot 1, database rebuilt in place", 9000);
    free(datacrt);
    if (failures) {
        printf("dropin-inplace: FAILED\n");
        return 1;
    }
    printf("dropin-inplace: ok\n");
    return 0;
}
