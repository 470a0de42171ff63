/*
 * kspir_b200 -- B200-native online answer of the KsPIR single-server PIR.
 *
 * C ABI.  Plain pointers and sizes, int status codes, no exceptions.  Every
 * array uses the word layouts of the reference's own objects (u64 words,
 * N = 4096, values canonical modulo the stated modulus):
 *
 *   datacrt  [r][N][N2][N1]   reference database_tocrt output, src/crt.cpp:859-885
 *                             (word = (v mod q1) | (v mod q2) << 32)
 *   query    [2][2][N]        query1[0] = (a, b) mod crtMod, query1[1] = (a, b) mod bsMod,
 *                             coefficient form (src/twosteps.cpp:279-318, encrypt.cpp:443-495)
 *   perms    [N1][N] int32    compute_permutation_matrix(permutations, N1, N), utils.cpp:1591
 *   baby     [N1/2][6][2][N]  AutoKeyBSGSRNS::keyMap[5^i], i = 1..N1/2 (lwe.h:381-466):
 *                             rows 0-2 mod crtMod, rows 3-5 mod bsMod, each (a, b), NTT form
 *   giant    [N2-1][2][2][N]  AutoKeyBSGSRNS::keyMap[5^(N1*c)], c = 1..N2-1
 *   packing  [log2 r][4][2][N] AutoKey::keyMap[N/2^l + 1], l = 0..log2 r - 1 (lwe.h:175-234)
 *   rgsw     [4][2][N]        RGSWCiphertext rows (a[j], b[j]), j = 0..3 (lwe.h:113-170)
 *   result   [r][2][N]        first-dimension results, NTT form
 *   rlwes    [r][2][N]        external products, coefficient form
 *   response [2][N]           packed response (a, b), coefficient form
 *
 * Gadget parameters are the reference's test-pir configuration: baby steps
 * ell 3 / base 2^20 / Bg 2^20 (lwe.h:391-393), giant steps ell 2 / 2^20 / 2^18
 * (lwe.h:402-404), RGSW ell 2 / 2^20 / 2^18 (test-pir.cpp:71), packing
 * ell 4 / 0 / 2^14 (test-pir.cpp:88).
 *
 * Results are word-for-word those of the reference on the same inputs.
 * Unlike the reference, a query, key or RLWE word that is not canonical is
 * rejected with KSPIR_ERR_INVALID_ARG.
 */
#ifndef KSPIR_B200_H
#define KSPIR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define KSPIR_OK 0
#define KSPIR_ERR_INVALID_ARG -1   /* bad size, pointer, or non-canonical word */
#define KSPIR_ERR_CUDA -2          /* a CUDA call failed (kspir_last_error has the text) */
#define KSPIR_ERR_NOT_READY -3     /* database, permutations or client keys missing */
#define KSPIR_ERR_OOM -4           /* device allocation failed */
#define KSPIR_ERR_TIMEOUT -5       /* a bounded device-side wait gave up */
#define KSPIR_ERR_BUSY -6          /* the server cannot take the call now (client has requests in flight) */
#define KSPIR_ERR_IO -7            /* file error, or a malformed / corrupted container */

#define KSPIR_N 4096

typedef struct kspir_ctx kspir_ctx;

typedef struct kspir_params {
    int32_t r;            /* packing number = number of sub-databases, power of two, 1..512 */
    int32_t N1;           /* baby steps: 64, 128 or 256; N2 = N/2/N1 */
    int32_t max_clients;  /* client key slots held on the device */
    int32_t max_inflight; /* query workspaces = largest batch (1 for the plain path) */
} kspir_params;

/* Context bound to one CUDA device.  Allocates the per-query workspaces. */
int kspir_ctx_create(int device, const kspir_params* params, kspir_ctx** out);
int kspir_ctx_destroy(kspir_ctx* ctx);
const char* kspir_last_error(const kspir_ctx* ctx);   /* the calling thread's last error text (any ctx, or NULL) */
const char* kspir_strerror(int code);

/* Replaces the datacrt argument of matrix_vector_mul_bsgs_rns_crt_large
 * (reference twosteps.h:55-57): the whole preprocessed database, host memory,
 * r * N * N / 2 words, kept resident on the device. */
int kspir_db_upload(kspir_ctx* ctx, const uint64_t* datacrt, size_t words);

/* Server preprocessing on the device: reference database_tobsgsntt followed
 * by database_tocrt (twosteps.h, twosteps.cpp:42-179; crt.cpp:859-885), for
 * every sub-database k < r, as tests/test-pir.cpp:59-60 calls them.
 *   data [r][N][N/2] words, data[k][i][j] = the reference's data[i][j] of
 *        sub-database k; every word < bsgsp = 65537 (HEXL's inverse NTT
 *        input range), else KSPIR_ERR_INVALID_ARG and the resident database is
 *        left as it was.
 * The result becomes the resident database, equal word for word to the
 * datacrt the reference writes (kspir_db_upload of that datacrt is the same
 * state).  device_ms (or NULL) receives the device time of validation and
 * preprocessing.  Host buffer; returns when done. */
int kspir_db_preprocess(kspir_ctx* ctx, const uint64_t* data, size_t words, float* device_ms);

/* Same with the raw database already in device memory. */
int kspir_db_preprocess_device(kspir_ctx* ctx, const uint64_t* d_data, size_t words, float* device_ms);

/* The reference's two preprocessing functions one for one, for one
 * sub-database, on the device (host buffers; the context supplies N1):
 *   kspir_database_tobsgsntt  database_tobsgsntt(result, data, crtMod, N1)
 *       (twosteps.h:19-20, twosteps.cpp:42-179): data [N][N/2] words < 65537
 *       (else KSPIR_ERR_INVALID_ARG), result [N/2][N] rows mod crtMod.
 *   kspir_database_tocrt      database_tocrt(datacrt, data_ntt, N1)
 *       (crt.h:133, crt.cpp:859-885): data_ntt [N/2][N] (any 64-bit words),
 *       datacrt [N][N/2].
 * Neither touches the resident database. */
int kspir_database_tobsgsntt(kspir_ctx* ctx, const uint64_t* data, uint64_t* result);
int kspir_database_tocrt(kspir_ctx* ctx, const uint64_t* data_ntt, uint64_t* datacrt);

/* ------------------------------------------------------------------------
 * Wire and file formats.  The reference has no serialization; these carry the
 * words of its objects (RlweCiphertext lwe.h:48-110: a then b; the key maps
 * flattened as for kspir_client_keys_upload) packed to their moduli: words
 * mod crtMod as 7 little-endian bytes, words mod bsMod as 3.  Each container
 * has a header with a format version and a 64-bit checksum of its payload;
 * a wrong magic, version, size or checksum gives KSPIR_ERR_IO, a word not
 * below its modulus KSPIR_ERR_INVALID_ARG.  Host-only except the database
 * file functions.
 *
 * Client key bundle: 64-byte header + baby (rows 0-2 at 7 bytes, rows 3-5 at
 * 3 bytes per word), giant, packing, rgsw (7 bytes per word); 17.7 MiB at
 * r = 16, N1 = 128 (27.1 MiB as u64 words).  kspir_key_bundle_bytes gives the
 * size (0 for an invalid shape).  kspir_client_keys_upload_bundle =
 * kspir_key_bundle_read + kspir_client_keys_upload. */
size_t kspir_key_bundle_bytes(int r, int N1);
int kspir_key_bundle_write(int r, int N1, const uint64_t* baby, const uint64_t* giant, const uint64_t* packing,
                           const uint64_t* rgsw, uint8_t* out, size_t out_bytes);
int kspir_key_bundle_read(const uint8_t* bundle, size_t bytes, int r, int N1, uint64_t* baby, uint64_t* giant,
                          uint64_t* packing, uint64_t* rgsw);
int kspir_client_keys_upload_bundle(kspir_ctx* ctx, int client, const uint8_t* bundle, size_t bytes);

/* Query and response messages: 16-byte header + packed words.  A query
 * ([2][2][N], crtMod part then bsMod part) is 81,936 bytes (131,072 as u64
 * words), a response ([2][N] mod crtMod) 57,360 bytes (65,536). */
#define KSPIR_QUERY_WIRE_BYTES (16 + 2 * KSPIR_N * 7 + 2 * KSPIR_N * 3)
#define KSPIR_RESPONSE_WIRE_BYTES (16 + 2 * KSPIR_N * 7)
int kspir_query_pack(const uint64_t* query, uint8_t* out);
int kspir_query_unpack(const uint8_t* in, size_t bytes, uint64_t* query);
int kspir_response_pack(const uint64_t* response, uint8_t* out);
int kspir_response_unpack(const uint8_t* in, size_t bytes, uint64_t* response);

/* The resident (preprocessed) database as a file: 64-byte header (r, N1,
 * checksum computed on the device) + the datacrt words, 8 bytes each.
 * kspir_db_load checks the file against the context's (r, N1) and the
 * checksum before it replaces the resident database (a failed load leaves it
 * as it was); it skips the preprocessing on a restart. */
int kspir_db_save(kspir_ctx* ctx, const char* path);
int kspir_db_load(kspir_ctx* ctx, const char* path);

/* ------------------------------------------------------------------------
 * The client side on the device (test clients, load generation).  Host
 * buffers, n queries / responses per call, run on the context's device.
 *
 * kspir_client_queries: query_bsgs_rns (twosteps.cpp:279-318) for each
 *   (secrets[i], rows[i]): secrets [n][N] in coefficient form mod crtMod (the
 *   reference Secret's words; each must be small: below bsMod/2 or above
 *   crtMod - bsMod/2), rows[i] < N/2, queries [n][2][2][N] (the layout of
 *   kspir_answer's query).  Same algebra and message scaling as the
 *   reference; its rand() draws are replaced by Philox4x32-10 keyed by `seed`
 *   (query i uses counter block i), so a query is a deterministic function of
 *   (secret, row, seed, i).
 * kspir_client_decrypt: decrypt_bsgs_total (twosteps.cpp:388-418) of responses
 *   [n][2][N] (coefficient form) under secrets [n][N] for a packing number r
 *   (a power of two up to 4096): messages [n][N].  The reference's
 *   QInv(r, crtMod) has no entry for r = 128 (it returns 0 there); this uses
 *   r^-1 mod crtMod, the value of every entry it has. */
int kspir_client_queries(kspir_ctx* ctx, int n, const uint64_t* secrets, const uint32_t* rows, uint64_t seed,
                         uint64_t* queries);
int kspir_client_decrypt(kspir_ctx* ctx, int n, const uint64_t* secrets, const uint64_t* responses, int r,
                         uint64_t* messages);

/* ------------------------------------------------------------------------
 * Offline key derivation, reference genAutoKeyFromOffline (twosteps.h,
 * twosteps.cpp:1749-1864) with its key switch evalAutoRNSKey
 * (twosteps.cpp:1587-1743), as tests/test-two-steps-key.cpp:140-175 runs it:
 * offline keys offlineKey1 (crtMod, crtBaMod = bsMod * auxMod, ell 5, base
 * 2^18, Bg 2^18) and offlineKey2 (crtMod, auxMod, ell 5, base 2^14, Bg 2^14),
 * automorphism keys autoKey1 (crtMod, crtBaMod) and autoKey2 (crtMod, auxMod),
 * N1 and N2 of the context.  Host buffers of u64 words, NTT form as keyGen
 * leaves the inputs:
 *   offline1  [10][2][N]  offlineKey1.keyMap[5]: rows 0-4 mod crtMod, 5-9 mod crtBaMod
 *   offline2  [10][2][N]  offlineKey2.keyMap[5^N1]: rows 0-4 mod crtMod, 5-9 mod auxMod
 *   auto1     [6][2][N]   autoKey1.keyMap[5]: rows 0-2 mod crtMod, 3-5 mod crtBaMod
 *   auto2     [6][2][N]   autoKey2.keyMap[5^N1]: rows 0-2 mod crtMod, 3-5 mod auxMod
 * Outputs (each may be NULL), word for word the reference's key maps after
 * the call:
 *   chain1    [N1-2][6][2][N]  autoKey1.keyMap[5^i], i = 2..N1-1 (coefficient form)
 *   chain2    [N2-2][6][2][N]  autoKey2.keyMap[5^(N1 i)], i = 2..N2-1
 *   baby_out  [N1-1][6][2][N]  result.keyMap[5^i], i = 1..N1-1 (NTT form)
 *   giant_out [N2-1][3][2][N]  result.keyMap[5^(N1 i)], i = 1..N2-1
 * The reference reads the crtBaMod rows through EltwiseReduceMod with factors
 * (1, 1), which leaves them unreduced, so rows 3-5 of every baby_out key are
 * zero; these are the reference's words, not keys the answer can use.
 * device_ms (or NULL) receives the device time.  Non-canonical input words:
 * KSPIR_ERR_INVALID_ARG. */
int kspir_gen_autokey_from_offline(kspir_ctx* ctx, const uint64_t* offline1, const uint64_t* offline2,
                                   const uint64_t* auto1, const uint64_t* auto2, uint64_t* chain1, uint64_t* chain2,
                                   uint64_t* baby_out, uint64_t* giant_out, float* device_ms);

/* Copies the resident database (datacrt layout, r * N * N / 2 words) to host. */
int kspir_db_download(kspir_ctx* ctx, uint64_t* datacrt, size_t words);

/* Replaces the permutations argument of matrix_vector_mul_bsgs_rns_crt_large
 * (twosteps.h:55-57). */
int kspir_perms_upload(kspir_ctx* ctx, const int32_t* perms, size_t count);

/* Replaces the autoKey (AutoKeyBSGSRNS, twosteps.h:55-57), packing key
 * (AutoKey, answer.h:79-80) and RGSW query (externalProduct, lwe.h:292) of one
 * client, kept resident in slot `client`. */
int kspir_client_keys_upload(kspir_ctx* ctx, int client, const uint64_t* baby, const uint64_t* giant,
                             const uint64_t* packing, const uint64_t* rgsw);

/* The server's online answer, reference tests/test-pir.cpp:110-116
 * (matrix_vector_mul_bsgs_rns_crt_large -> externalProduct x r -> packingRLWEs),
 * host buffers in and out.  The caller's query is not modified.  Blocks until
 * the response is in `response`.  Safe to call from several host threads at
 * once: each call owns one of min(max_inflight, 8) workspace slots and its
 * stream while it runs, and waits for its answer without holding the context,
 * so up to eight concurrent callers' answers overlap on the device (one
 * answer's key switches with another's database scan).  Pinned host buffers
 * let the copies run asynchronously. */
int kspir_answer(kspir_ctx* ctx, int client, const uint64_t* query, uint64_t* response);

/* Same on device buffers (query [2][2][N], response [2][N]), enqueued on
 * `stream` (a cudaStream_t, or NULL for the context's stream); returns once
 * enqueued.  Call kspir_sync to wait and collect device-side errors.
 * Successive calls rotate over the same workspace slots as kspir_answer (each
 * waits, on its stream, for the last answer that used its slot), so answers
 * issued on different streams run at the same time.  With the fused answer on
 * (kspir_set_fused) every single answer uses slot 0. */
int kspir_answer_device(kspir_ctx* ctx, int client, const uint64_t* d_query, uint64_t* d_response, void* stream);
int kspir_sync(kspir_ctx* ctx);

/* Batched answer: n queries of (possibly) different clients in one launch
 * sequence (every kernel covers all n queries; the first-dimension scan reads
 * the database once for the whole batch on the tensor cores when the context
 * has N1 = 128 and max_inflight >= 2).  No reference counterpart as one call:
 * each response equals kspir_answer(clients[i], query i), which equals the
 * reference's test-pir.cpp:110-116 on that query.
 *   queries   [n][2][2][N]   layout of kspir_answer's query
 *   responses [n][2][N]
 * 1 <= n <= min(max_inflight, 256).  Host buffers; returns when done. */
int kspir_answer_batch(kspir_ctx* ctx, int n, const int32_t* clients, const uint64_t* queries, uint64_t* responses);

/* Same on device buffers, enqueued on `stream` (NULL = context stream);
 * returns once enqueued (kspir_sync waits and reports device errors). */
int kspir_answer_batch_device(kspir_ctx* ctx, int n, const int32_t* clients, const uint64_t* d_queries,
                              uint64_t* d_responses, void* stream);

/* Database-scan variant used for a batch of n queries:
 *   0 CUDA-core scan, one database pass per query
 *   1..4 tensor-core scan with query tiles of 4, 8, 16, 32 queries
 * kspir_tune_batch times every variant on the resident database (results are
 * identical by construction; only speed differs), keeps the fastest for n and
 * returns it; ms_out ([5] or NULL) receives each variant's scan time (1e30 for
 * variants not tried).  Do not call while answers are in flight: it uses the
 * workspaces.  kspir_set_scan_kind forces a variant (-1 = back to the
 * default), kspir_get_scan_kind reports the one in use. */
int kspir_tune_batch(kspir_ctx* ctx, int n, int* kind_out, float* ms_out);
int kspir_set_scan_kind(kspir_ctx* ctx, int n, int kind);
int kspir_get_scan_kind(kspir_ctx* ctx, int n);

/* Reference matrix_vector_mul_bsgs_rns_crt_large (twosteps.h:55-57,
 * twosteps.cpp:1527-1579) for one client: query_inout is modswitched in place
 * to NTT form mod crtMod exactly like the reference's input[0] (twosteps.cpp:
 * 1073-1086) and result ([r][2][N], NTT form) receives the r first-dimension
 * results.  Host buffers. */
int kspir_matrix_vector_mul_bsgs_rns_crt_large(kspir_ctx* ctx, int client, uint64_t* query_inout,
                                               uint64_t* result);

/* Reference externalProduct (lwe.h:292, lwe.cpp:761-808) for `count`
 * ciphertexts: result[j] += g^-1(first_dim[j]) x RGSW, returned in
 * coefficient form; first_dim ([count][2][N], NTT form) is converted to
 * coefficient form in place, as the reference does.  Host buffers. */
int kspir_external_product(kspir_ctx* ctx, int client, uint64_t* result, uint64_t* first_dim, int count);

/* Reference packingRLWEs (answer.h:79-80, answer.cpp:800-835): packs r
 * coefficient-form RLWEs ([r][2][N]) into response ([2][N], coefficient
 * form).  Host buffers.  rlwes is overwritten as the reference overwrites it
 * (answer.cpp:821-828): rlwes[0] becomes the response and, for each merge of
 * rlwes[j] with rlwes[I + j] (I = r/2, ..., 1; j < I), rlwes[I + j] becomes
 * X^I rlwes[I + j] + rlwes[j] of that level's inputs. */
int kspir_packing_rlwes(kspir_ctx* ctx, int client, uint64_t* rlwes, uint64_t* response);

/* No counterpart in the reference.  The external product of
 * kspir_external_product (reference externalProduct, lwe.cpp:761-808, with
 * the RGSW parameters of test-pir.cpp:71) for callers that cannot allocate
 * device memory -- e.g. a plugin whose host owns all device memory through its
 * own pool, or code that must not trigger the device synchronisation that
 * cudaMalloc/cudaFree can cause.  It calls no cudaMalloc, cudaFree or other
 * allocating routine and needs no kspir_ctx.  All pointers are device memory
 * owned by the caller:
 *   d_rgsw      [4][2][N]       RGSW rows, NTT form
 *   d_result    [count][2][N]   in: NTT-domain accumulators (zero for a fresh
 *                               product); out: results, coefficient form
 *   d_first_dim [count][2][N]   in: NTT form; out: coefficient form
 * count <= KSPIR_NOALLOC_MAX_COUNT; larger counts are rejected with
 * KSPIR_ERR_INVALID_ARG, as are non-canonical words (outputs then untouched).
 * Work is enqueued on `stream` (a cudaStream_t, NULL = the legacy default
 * stream); the call then waits for that stream (cudaStreamSynchronize) and
 * reads a validation word back, so it returns only after its work is done
 * and blocks the calling thread until then.
 * Scratch: a fixed file-scope device array of about 6.3 MiB (plus 192 KiB of
 * transform tables) that every GPU loading this library holds until the
 * process exits.  All calls on a device share it, so calls that overlap on
 * the GPU (other threads, other streams) race and must be serialised by the
 * caller.  The first call on each device also sets that device up (constant
 * tables and the device address of the scratch array); make that first call
 * before any stream capture. */
#define KSPIR_NOALLOC_MAX_COUNT 16
int kspir_external_product_noalloc(int device, const uint64_t* d_rgsw, uint64_t* d_result, uint64_t* d_first_dim,
                                   int count, void* stream);

/* Fills perms ([N1][N] int32) with the matrix the reference's
 * compute_permutation_matrix(permutations, N1, N) builds (utils.cpp:1591-1619):
 * row i is the NTT-slot gather that applies X -> X^(5^i).  No device needed. */
int kspir_permutation_matrix(int32_t* perms, int N1);

/* Device time of the last answer launch (single or batched) in
 * milliseconds, and per-phase split (baby steps, DB scan, giant steps,
 * external products, packing). */
int kspir_last_timing(kspir_ctx* ctx, float* total_ms, float* phase_ms /* [5] or NULL */);

/* Timing of every answer launch since kspir_timing_reset (the most recent
 * 512 launches are kept): the queries they answered, the kernels launched,
 * and the summed device time in milliseconds in total and per phase (same
 * split as kspir_last_timing).  Waits for those launches to finish. */
int kspir_timing_reset(kspir_ctx* ctx);
int kspir_timing_summary(kspir_ctx* ctx, int* answers, long* launches, float* total_ms, float* phase_ms);

/* Diagnostics: copies an intermediate of the last answer out of workspace 0,
 * as reference words (host buffer of exactly the stated size):
 *   KSPIR_STAGE_CIPHERBUF [N][N1][2]  reorientCipher output (twosteps.cpp:1386-1403)
 *   KSPIR_STAGE_SCAN      [r][N2][2][N] fastMultiplyQueryByDatabaseDim1InvCRT outputs
 *                         (recomputed from the slot's reorientCipher output by
 *                         the scan variant of the last launch: the giant steps
 *                         reuse the scan output in place)
 *   KSPIR_STAGE_RESULT    [r][2][N]   first-dimension results (NTT form)
 *   KSPIR_STAGE_EXT       [r][2][N]   external products (coefficient form) */
#define KSPIR_STAGE_CIPHERBUF 0
#define KSPIR_STAGE_SCAN 1
#define KSPIR_STAGE_RESULT 2
#define KSPIR_STAGE_EXT 3
int kspir_fetch_stage(kspir_ctx* ctx, int stage, uint64_t* out, size_t words);
/* Same for the query that ran in workspace slot `slot` (query i of the last
 * batch ran in slot i). */
int kspir_fetch_stage_slot(kspir_ctx* ctx, int slot, int stage, uint64_t* out, size_t words);

/* Failure injection, for tests of the device-side failure detection.  Every
 * wait of the database scan on the device is bounded: a wait that runs out
 * records an error word and the kernel returns, and the call that collects
 * the launch reports KSPIR_ERR_TIMEOUT; the context stays usable.  This sets
 * the limit of those waits (wait_limit_ns <= 0: the default of 2 s) and makes
 * the next CUDA-core database scan (the one of a single answer) skip the copy
 * of local work item `skip_item` of its first CTA (-1: none), so that the
 * wait for it runs out.  No GPU fault is involved: the kernel only waits for
 * bytes that were never requested. */
int kspir_debug_scan_fault(kspir_ctx* ctx, int64_t wait_limit_ns, long skip_item);

/* The single answer as one kernel (kspir_answer and kspir_answer_device on
 * contexts with N1 = 128): one cooperative launch of one CTA per SM in which
 * a 512-thread warp group runs the key switches from a dependency-ordered task
 * queue while the other warps stream the database, so the giant steps,
 * external products and packing merges of sub-databases already scanned
 * overlap the scan of the rest.  Same words as the separate kernels.
 * kspir_set_fused turns it on (1) or off (0): KSPIR_ERR_NOT_READY when the
 * context cannot run it; the environment variable KSPIR_FUSED=1 turns it on
 * at context creation.  kspir_get_fused: 1 on, 0 off. */
int kspir_set_fused(kspir_ctx* ctx, int enable);
int kspir_get_fused(const kspir_ctx* ctx);

/* Bytes of one client's keys in a device key slot (for sizing max_clients
 * from an HBM budget). */
size_t kspir_client_key_bytes(const kspir_ctx* ctx);

/* ------------------------------------------------------------------------
 * Serving loop (no counterpart in the reference): continuous batching of
 * online answers on one context.
 *
 * A worker thread runs `lanes` lanes of `lane_size` workspace slots each
 * (the context needs max_inflight >= lanes * lane_size, with lane_size
 * rounded up to a multiple of 32 when the tensor-core scan is enabled).
 * Whenever a lane is free, the waiting requests (up to lane_size) are
 * admitted as one batch on it while the other lanes' batches still run.
 * Client keys live in caller memory (registered once, kept valid by the
 * caller until the server is destroyed or the client re-registered) and are
 * cached in device key slots: at most key_budget_bytes of them (0 = all the
 * context's slots), least recently used idle clients evicted first.  Each
 * response equals kspir_answer on the same client and query.
 * ------------------------------------------------------------------------ */
typedef struct kspir_server kspir_server;

typedef struct kspir_server_params {
    int32_t lanes;             /* batches in flight at once */
    int32_t lane_size;         /* largest batch (1..256) */
    int64_t key_budget_bytes;  /* HBM for cached client keys; 0 = every key slot of the context */
} kspir_server_params;

typedef struct kspir_server_stats {
    long served;               /* responses delivered since the last reset */
    long batches;              /* batches launched */
    double mean_batch;         /* queries per batch */
    double p50_us, p95_us, p99_us, max_us;   /* submit -> response latency */
    double queries_per_s;      /* served / seconds since the last reset */
    long key_uploads;          /* client key sets brought into device slots */
    long evictions;            /* resident key sets evicted for others */
    int32_t key_slots;         /* device key slots the server may use */
    int32_t max_running_lanes; /* most batches seen running at once */
} kspir_server_stats;

int kspir_server_create(kspir_ctx* ctx, const kspir_server_params* params, kspir_server** out);
int kspir_server_destroy(kspir_server* srv);   /* finishes every submitted request first */
int kspir_server_register_client(kspir_server* srv, int64_t client, const uint64_t* baby, const uint64_t* giant,
                                 const uint64_t* packing, const uint64_t* rgsw);
/* Queues one answer (query [2][2][N] and response [2][N] host buffers, both
 * kept valid until the request completes); *ticket identifies it. */
int kspir_server_submit(kspir_server* srv, int64_t client, const uint64_t* query, uint64_t* response,
                        uint64_t* ticket);
/* 1 = done (the ticket is released), 0 = still running, < 0 = the request
 * failed with that error (released).  kspir_server_wait blocks up to
 * timeout_ms. */
int kspir_server_poll(kspir_server* srv, uint64_t ticket);
int kspir_server_wait(kspir_server* srv, uint64_t ticket, int timeout_ms);
int kspir_server_get_stats(kspir_server* srv, kspir_server_stats* out);
int kspir_server_reset_stats(kspir_server* srv);
/* Submit-to-response latencies (microseconds) of the requests served since
 * the last reset, in completion order: *count receives how many there are,
 * out (or NULL) the first min(capacity, count). */
int kspir_server_latencies(kspir_server* srv, double* out, size_t capacity, size_t* count);

#ifdef __cplusplus
}
#endif

#endif /* KSPIR_B200_H */
