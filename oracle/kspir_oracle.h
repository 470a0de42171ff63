/* TEST INFRASTRUCTURE ONLY -- the CPU oracle, never part of the product.
 *
 * Plain-C restatement of the KsPIR reference's online answer
 * (reference tests/test-pir.cpp:110-116), operation for operation, on 64-bit
 * words.  It is the checker for the CUDA path and the "port" CPU baseline.
 * Parity of this restatement with the reference itself is pinned in
 * tests/test_oracle.py against oracle/_ref (the reference compiled from its
 * own sources) and against the committed fixtures in tests/golden/.
 *
 * Layouts are those of include/kspir_b200.h (u64 words, N = 4096):
 *   query   [2 moduli (crtMod, bsMod)][2 (a, b)][N], coefficient form
 *   baby    [N1/2][6][2][N]   rows 0-2 mod crtMod, 3-5 mod bsMod; entry i <-> X -> X^(5^(i+1))
 *   giant   [N2-1][2][2][N]   entry c <-> X -> X^(5^(N1*(c+1)))
 *   packing [log2 r][4][2][N] level l <-> X -> X^(N/2^l + 1)
 *   rgsw    [4][2][N]
 *   perms   [N1][N] int32 (reference utils.cpp:1591 compute_permutation_matrix)
 */
#ifndef KSPIR_ORACLE_H
#define KSPIR_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KO_N 4096
#define KO_Q1 268369921ULL
#define KO_Q2 249561089ULL
#define KO_CRTMOD (KO_Q1 * KO_Q2)
#define KO_BSMOD 16760833ULL
#define KO_P 65537ULL

/* Whole answer: matrix_vector_mul_bsgs_rns_crt_large -> externalProduct x r -> packingRLWEs.
 * bsgs_out ([r][2][N], NTT form) and ext_out ([r][2][N], coefficient form) may be NULL. */
int ko_answer(const uint64_t* datacrt, int r, int N1, const uint64_t* query,
              const uint64_t* baby, const uint64_t* giant, const uint64_t* packing,
              const uint64_t* rgsw, const int32_t* perms, uint64_t* response,
              uint64_t* bsgs_out, uint64_t* ext_out);

/* First dimension.  query_inout is modswitched in place like the reference's
 * input (twosteps.cpp:1073-1086).  cipherbuf_out ([N][2*N1]) may be NULL. */
int ko_matrix_vector_mul(const uint64_t* datacrt, int r, int N1, uint64_t* query_inout,
                         const uint64_t* baby, const uint64_t* giant, const int32_t* perms,
                         uint64_t* result, uint64_t* cipherbuf_out);

/* Giant steps of one sub-database (evalAutoRNSCRT, twosteps.cpp:599-677) on its
 * scan output [N2][2][N] (NTT form, INTT'd in place): result [2][N]. */
int ko_giant_steps(uint64_t* result, uint64_t* output, int N1, const uint64_t* giant);

/* ext_inout += g^-1(first_dim) x rgsw; first_dim goes NTT -> coefficient form in place. */
int ko_external_product(uint64_t* ext_inout, uint64_t* first_dim_inout, const uint64_t* rgsw);

/* Packs r coefficient-form RLWEs (overwritten, as in the reference) into response. */
int ko_packing(uint64_t* rlwes_inout, int r, const uint64_t* packing, uint64_t* response);

/* One sub-database DB scan (crt.cpp:643-856): out [N2][2N]. */
void ko_scan(const uint64_t* db, const uint64_t* cipherbuf, int N1, uint64_t* out);

/* Server preprocessing of one sub-database: database_tobsgsntt then
 * database_tocrt (twosteps.cpp:42-179, crt.cpp:859-885).  raw [N][N/2] words
 * < p (else -1), datacrt [N][N/2]. */
int ko_db_preprocess(const uint64_t* raw, int N1, uint64_t* datacrt);
/* The scaled message of query_bsgs_rns for row t (twosteps.cpp:288-307): dm [N]. */
void ko_query_message(int t, uint64_t* dm);

/* The two steps apart: database_tobsgsntt (raw -> rows [N/2][N] mod crtMod,
 * -1 for a word >= p) and database_tocrt (rows -> datacrt [N][N/2]). */
int ko_database_tobsgsntt(const uint64_t* raw, int N1, uint64_t* rows);
void ko_database_tocrt(const uint64_t* rows, uint64_t* datacrt);

/* HEXL-order negacyclic transforms for modulus in {crtMod, bsMod, p, q1, q2}. */
int ko_ntt_forward(uint64_t* a, uint64_t modulus);
int ko_ntt_inverse(uint64_t* a, uint64_t modulus);
/* The transform's 2N-th root of unity psi for a modulus. */
uint64_t ko_ntt_root(uint64_t modulus);

void ko_decompose_bsgs(const uint64_t* a_crt, const uint64_t* a_bs, int ellnum, uint64_t base,
                       uint64_t bg, uint64_t* d_crt, uint64_t* d_bs);
void ko_decompose(const uint64_t* in, int ellnum, uint64_t base, uint64_t bg, uint64_t modulus,
                  uint64_t* out);
void ko_decompose_rlwe(const uint64_t* a, const uint64_t* b, int ellnum, uint64_t base,
                       uint64_t bg, uint64_t modulus, uint64_t* out);
uint64_t ko_crt_compose(uint64_t x, uint64_t y);
uint64_t ko_barrett_coeff(uint64_t v, int n);
void ko_permutation_matrix(int32_t* perms, int N1);
int ko_pow_mod_index(int a, int b);  /* a^b mod 2N, reference utils.cpp:1446-1459 */

#ifdef __cplusplus
}
#endif

#endif
