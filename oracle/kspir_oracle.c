/* TEST INFRASTRUCTURE ONLY -- the CPU oracle, never part of the product.
 *
 * Plain-C restatement of the KsPIR reference's online answer, following the
 * reference's own sequence of operations (every function cites the reference
 * file:line it restates).  The HEXL calls of the reference are restated with
 * HEXL's published semantics (see oracle/hexl_shim/hexl/hexl.hpp): negacyclic
 * NTT in bit-reversed order with canonical outputs, and single-correction
 * add/sub.  Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline
 * load this file.
 */
#define _GNU_SOURCE
#include "kspir_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;
typedef __int128 i128;

#define N KO_N
#define Q1 KO_Q1
#define Q2 KO_Q2
#define CRTMOD KO_CRTMOD
#define BSMOD KO_BSMOD

/* reference crt.h:33-34 */
#define BSMOD_INV 51309461009346113ULL /* bsMod^-1 mod crtMod */
#define CRTMOD_INV 3920321ULL          /* crtMod^-1 mod bsMod */
/* reference crt.h:81 */
#define ROOT_CRT 3375402822066082ULL

/* ------------------------------------------------------------------ */
/* modular helpers                                                      */

static inline uint64_t mulhi64(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) >> 64); }

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = (uint64_t)((u128)r * a % q);
        a = (uint64_t)((u128)a * a % q);
        e >>= 1;
    }
    return r;
}

static uint64_t invmod(uint64_t a, uint64_t q) {
    i128 t = 0, nt = 1, r = q, nr = a % q;
    while (nr) {
        i128 quo = r / nr, tmp;
        tmp = t - quo * nt; t = nt; nt = tmp;
        tmp = r - quo * nr; r = nr; nr = tmp;
    }
    if (t < 0) t += q;
    return (uint64_t)t;
}

/* exact (a*b + c) mod q for any 128-bit value, Barrett with mu = floor(2^128/q) */
typedef struct { uint64_t q, mh, ml; } barrett_t;

static barrett_t barrett_make(uint64_t q) {
    barrett_t b;
    u128 mu = (~(u128)0) / q;
    b.q = q; b.mh = (uint64_t)(mu >> 64); b.ml = (uint64_t)mu;
    return b;
}

static inline uint64_t barrett_reduce(const barrett_t* b, u128 z) {
    uint64_t zl = (uint64_t)z, zh = (uint64_t)(z >> 64);
    u128 t = ((u128)zl * b->ml) >> 64;
    t += (u128)zl * b->mh;
    u128 u = (u128)zh * b->ml + (uint64_t)t;
    uint64_t qhat = (uint64_t)(t >> 64) + (uint64_t)(u >> 64) + zh * b->mh;
    uint64_t r = zl - qhat * b->q;
    while (r >= b->q) r -= b->q;
    return r;
}

/* HEXL EltwiseAddMod / EltwiseSubMod semantics (single correction). */
static inline uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    return s >= q ? s - q : s;
}
static inline uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) {
    return a >= b ? a - b : a + q - b;
}

static void vadd(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t q) {
    for (int i = 0; i < N; i++) r[i] = add_mod(a[i], b[i], q);
}
static void vsub(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t q) {
    for (int i = 0; i < N; i++) r[i] = sub_mod(a[i], b[i], q);
}
static void vmul(uint64_t* r, const uint64_t* a, const uint64_t* b, uint64_t q) {
    barrett_t br = barrett_make(q);
    for (int i = 0; i < N; i++) r[i] = barrett_reduce(&br, (u128)a[i] * b[i]);
}
static void vmulc(uint64_t* r, const uint64_t* a, uint64_t c, uint64_t q) {
    barrett_t br = barrett_make(q);
    c %= q;
    for (int i = 0; i < N; i++) r[i] = barrett_reduce(&br, (u128)a[i] * c);
}

/* ------------------------------------------------------------------ */
/* NTT (HEXL order): slot j = sum_k x_k psi^((2 brv(j) + 1) k)           */

typedef struct {
    uint64_t q, psi;
    uint64_t w[N], wp[N], iw[N], iwp[N];
    uint64_t ninv, ninvp;
} ntt_tab_t;

enum { T_CRT, T_BS, T_P, T_Q1, T_Q2, T_COUNT };
static ntt_tab_t g_tab[T_COUNT];

static uint64_t bitrev12(uint64_t x) {
    uint64_t r = 0;
    for (int i = 0; i < 12; i++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* smallest primitive 2N-th root of unity (HEXL MinimalPrimitiveRoot(2N, q)) */
static uint64_t min_root(uint64_t q) {
    uint64_t root = 0;
    for (uint64_t g = 2; g < q; g++) {
        uint64_t c = powmod(g, (q - 1) / (2 * N), q);
        if (powmod(c, N, q) == q - 1) { root = c; break; }
    }
    uint64_t sq = (uint64_t)((u128)root * root % q), cur = root, best = root;
    for (int i = 0; i < N; i++) {
        if (cur < best) best = cur;
        cur = (uint64_t)((u128)cur * sq % q);
    }
    return best;
}

static void tab_init(ntt_tab_t* t, uint64_t q, uint64_t psi) {
    t->q = q; t->psi = psi;
    uint64_t pinv = invmod(psi, q);
    for (int k = 0; k < N; k++) {
        uint64_t e = bitrev12(k);
        t->w[k] = powmod(psi, e, q);
        t->iw[k] = powmod(pinv, e, q);
        t->wp[k] = (uint64_t)(((u128)t->w[k] << 64) / q);
        t->iwp[k] = (uint64_t)(((u128)t->iw[k] << 64) / q);
    }
    t->ninv = invmod(N, q);
    t->ninvp = (uint64_t)(((u128)t->ninv << 64) / q);
}

__attribute__((constructor)) static void ko_init(void) {
    tab_init(&g_tab[T_CRT], CRTMOD, ROOT_CRT);          /* reference crt.h:81 */
    tab_init(&g_tab[T_BS], BSMOD, min_root(BSMOD));     /* HEXL NTT(N, bsMod) */
    tab_init(&g_tab[T_P], KO_P, min_root(KO_P));        /* HEXL NTT(N, bsgsp) */
    tab_init(&g_tab[T_Q1], Q1, ROOT_CRT % Q1);
    tab_init(&g_tab[T_Q2], Q2, ROOT_CRT % Q2);
}

static const ntt_tab_t* tab_for(uint64_t q) {
    for (int i = 0; i < T_COUNT; i++)
        if (g_tab[i].q == q) return &g_tab[i];
    return NULL;
}

static inline uint64_t shoup_lazy(uint64_t x, uint64_t w, uint64_t wp, uint64_t q) {
    return x * w - mulhi64(x, wp) * q;
}

static void ntt_fwd(uint64_t* a, const ntt_tab_t* t) {
    const uint64_t q = t->q, q2 = 2 * q;
    for (int i = 0; i < N; i++) if (a[i] >= q) a[i] %= q;
    for (int m = 1, h = N / 2; m < N; m <<= 1, h >>= 1) {
        for (int i = 0; i < m; i++) {
            uint64_t W = t->w[m + i], Wp = t->wp[m + i];
            uint64_t *X = a + 2 * i * h, *Y = X + h;
            for (int j = 0; j < h; j++) {
                uint64_t x = X[j];
                if (x >= q2) x -= q2;
                uint64_t wy = shoup_lazy(Y[j], W, Wp, q);
                X[j] = x + wy;
                Y[j] = x - wy + q2;
            }
        }
    }
    for (int i = 0; i < N; i++) {
        uint64_t x = a[i];
        if (x >= q2) x -= q2;
        if (x >= q) x -= q;
        a[i] = x;
    }
}

static void ntt_inv(uint64_t* a, const ntt_tab_t* t) {
    const uint64_t q = t->q, q2 = 2 * q;
    for (int i = 0; i < N; i++) if (a[i] >= q) a[i] %= q;
    for (int m = N / 2, h = 1; m >= 1; m >>= 1, h <<= 1) {
        for (int i = 0; i < m; i++) {
            uint64_t W = t->iw[m + i], Wp = t->iwp[m + i];
            uint64_t *X = a + 2 * i * h, *Y = X + h;
            for (int j = 0; j < h; j++) {
                uint64_t x = X[j], y = Y[j];
                uint64_t s = x + y;
                if (s >= q2) s -= q2;
                X[j] = s;
                Y[j] = shoup_lazy(x - y + q2, W, Wp, q);
            }
        }
    }
    for (int i = 0; i < N; i++) {
        uint64_t x = shoup_lazy(a[i], t->ninv, t->ninvp, q);
        if (x >= q) x -= q;
        a[i] = x;
    }
}

int ko_ntt_forward(uint64_t* a, uint64_t modulus) {
    const ntt_tab_t* t = tab_for(modulus);
    if (!t) return -1;
    ntt_fwd(a, t);
    return 0;
}

int ko_ntt_inverse(uint64_t* a, uint64_t modulus) {
    const ntt_tab_t* t = tab_for(modulus);
    if (!t) return -1;
    ntt_inv(a, t);
    return 0;
}

uint64_t ko_ntt_root(uint64_t modulus) {
    const ntt_tab_t* t = tab_for(modulus);
    return t ? t->psi : 0;
}

#define NTT_CRT(a) ntt_fwd((a), &g_tab[T_CRT])
#define INTT_CRT(a) ntt_inv((a), &g_tab[T_CRT])
#define NTT_BS(a) ntt_fwd((a), &g_tab[T_BS])
#define INTT_BS(a) ntt_inv((a), &g_tab[T_BS])

/* ------------------------------------------------------------------ */
/* CRT helpers, reference crt.cpp                                       */

/* barrett_raw_u64 + barrett_coeff, crt.cpp:287-301 */
uint64_t ko_barrett_coeff(uint64_t v, int n) {
    uint64_t ratio = n == 0 ? 68736257792ULL : 73916747789ULL;   /* cr1_p / cr1_b, crt.h:20-21 */
    uint64_t q = n == 0 ? Q1 : Q2;
    uint64_t t = mulhi64(v, ratio);
    uint64_t r = v - t * q;
    return r >= q ? r - q : r;
}

/* barrett_raw_u128, crt.cpp:345-366, with cr0_Q/cr1_Q of crt.cpp:27-28 */
static uint64_t barrett_raw_u128(u128 val, uint64_t c0, uint64_t c1, uint64_t modulus) {
    uint64_t zx = (uint64_t)val, zy = (uint64_t)(val >> 64);
    u128 prod = (u128)zx * c0;
    uint64_t carry = (uint64_t)(prod >> 64);
    u128 t2 = (u128)zx * c1;
    uint64_t tmp1 = (uint64_t)t2 + carry;
    uint64_t tmp3 = (uint64_t)(t2 >> 64) + (tmp1 < (uint64_t)t2);
    t2 = (u128)zy * c0;
    uint64_t old = tmp1;
    tmp1 = tmp1 + (uint64_t)t2;
    carry = (uint64_t)(t2 >> 64) + (tmp1 < old);
    tmp1 = zy * c1 + tmp3 + carry;
    return zx - tmp1 * modulus;
}

/* crt_compose, crt.cpp:368-377 (b_inv_pa_i / pa_inv_b_i of crt.cpp:25-26) */
uint64_t ko_crt_compose(uint64_t x, uint64_t y) {
    const u128 b_inv_pa_i = (u128)163640210ULL * Q2;
    const u128 pa_inv_b_i = (u128)97389680ULL * Q1;
    u128 val = (u128)x * b_inv_pa_i;
    val += (u128)y * pa_inv_b_i;
    uint64_t r = barrett_raw_u128(val, 7906011006380390721ULL, 275ULL, CRTMOD);
    if (r >= CRTMOD) r -= CRTMOD;
    return r;
}

/* fastMultiplyQueryByDatabaseDim1InvCRT, crt.cpp:643-768.  The AVX-512 lanes
 * only reorder exact 64-bit integer sums, so a scalar sum gives the same words. */
void ko_scan(const uint64_t* db, const uint64_t* cipherbuf, int N1, uint64_t* out) {
    int N2 = N / 2 / N1;
    for (int z = 0; z < N; z++) {
        const uint64_t* v = cipherbuf + (size_t)z * 2 * N1;
        const uint64_t* d = db + (size_t)z * N2 * N1;
        for (int i = 0; i < N2; i++) {
            uint64_t a_lo = 0, a_hi = 0, b_lo = 0, b_hi = 0;
            for (int k = 0; k < N1; k++) {
                uint64_t w = d[(size_t)i * N1 + k];
                uint64_t wl = (uint32_t)w, wh = w >> 32;
                uint64_t ca = v[2 * k], cb = v[2 * k + 1];
                a_lo += wl * (uint32_t)ca;
                a_hi += wh * (ca >> 32);
                b_lo += wl * (uint32_t)cb;
                b_hi += wh * (cb >> 32);
            }
            out[(size_t)i * 2 * N + z] = ko_crt_compose(a_lo, a_hi);
            out[(size_t)i * 2 * N + N + z] = ko_crt_compose(b_lo, b_hi);
        }
    }
}

/* ------------------------------------------------------------------ */
/* gadget decompositions, reference utils.cpp                          */

static int ilog2u(uint64_t v) { int l = 0; while (v > 1) { v >>= 1; l++; } return l; }

/* decompose, VARIANT B (DECOMPOSE_VARIANT_A is off, utils.cpp:690), utils.cpp:754-811 */
void ko_decompose(const uint64_t* in, int ellnum, uint64_t base, uint64_t bg, uint64_t modulus,
                  uint64_t* out) {
    int gbits = ilog2u(bg);
    int base_bits = base ? ilog2u(base) : 0;
    int sub = 64 - gbits;
    uint64_t offset = 0;
    for (int i = 0; i < ellnum; i++) offset += (uint64_t)1 << (base_bits + i * gbits);
    offset <<= (gbits - 1);
    offset += base / 2;
    for (int i = 0; i < N; i++) {
        uint64_t d = in[i] + offset;
        if (d > modulus) d -= modulus;      /* note: strict '>' as in the reference */
        d >>= base_bits;
        for (int j = 0; j < ellnum; j++) {
            int64_t r = (int64_t)(d << sub >> sub);
            r -= (int64_t)(bg / 2);
            d >>= gbits;
            out[(size_t)j * N + i] = r >= 0 ? (uint64_t)r : (uint64_t)r + modulus;
        }
    }
}

/* compute_mult_qinvqi_bsgs, utils.cpp:406-432 */
static u128 mult_qinvqi_bsgs(uint64_t input, uint64_t qinv, uint64_t qi) {
    const u128 modulus = (u128)CRTMOD * BSMOD;
    const u128 two128_mod = ((u128)54824ULL << 63) + (u128)1764040975123512121ULL; /* crt.h:91-92 */
    const u128 lowmask = ((u128)1 << 64) - 1;
    u128 factor = (u128)qi * qinv;
    u128 fh = factor >> 64, fl = factor & lowmask;
    u128 temp = (u128)input * fh;
    u128 result = (temp >> 64) * two128_mod % modulus;
    result += (temp << 64) % modulus;
    result += input * fl;
    result %= modulus;
    return result;
}

/* decompose_bsgs, utils.cpp:1120-1189, on crt_inv_bsgs, utils.cpp:516-532 */
void ko_decompose_bsgs(const uint64_t* a_crt, const uint64_t* a_bs, int ellnum, uint64_t base,
                       uint64_t bg, uint64_t* d_crt, uint64_t* d_bs) {
    const u128 modulus = (u128)CRTMOD * BSMOD;
    int gbits = ilog2u(bg);
    int base_bits = base ? ilog2u(base) : 0;
    int sub = 128 - gbits;
    u128 offset = 0;
    for (int i = 0; i < ellnum; i++) offset += (u128)1 << (base_bits + i * gbits);
    offset <<= (gbits - 1);
    offset += base / 2;
    for (int i = 0; i < N; i++) {
        u128 x = mult_qinvqi_bsgs(a_crt[i], BSMOD_INV, BSMOD);
        x += mult_qinvqi_bsgs(a_bs[i], CRTMOD_INV, CRTMOD);
        x %= modulus;
        u128 d = x + offset;
        if (d > modulus) d -= modulus;
        d >>= base_bits;
        for (int j = 0; j < ellnum; j++) {
            int64_t r = (int64_t)(d << sub >> sub);
            r -= (int64_t)(bg / 2);
            d >>= gbits;
            if (r >= 0) {
                d_crt[(size_t)j * N + i] = (uint64_t)r;
                d_bs[(size_t)j * N + i] = (uint64_t)r;
            } else {
                d_crt[(size_t)j * N + i] = (uint64_t)r + CRTMOD;
                d_bs[(size_t)j * N + i] = (uint64_t)r + BSMOD;
            }
        }
    }
}

/* decompose_rlwe, utils.cpp:974-1044 (signed digits, dropped low bits truncated) */
void ko_decompose_rlwe(const uint64_t* a, const uint64_t* b, int ellnum, uint64_t base,
                       uint64_t bg, uint64_t modulus, uint64_t* out) {
    uint64_t half = modulus >> 1;
    int gbits = ilog2u(bg);
    int base_bits = ilog2u(base);
    int sub = 64 - gbits;
    for (int part = 0; part < 2; part++) {
        const uint64_t* in = part ? b : a;
        for (int i = 0; i < N; i++) {
            int64_t d = in[i] > half ? (int64_t)(in[i] - modulus) : (int64_t)in[i];
            d >>= base_bits;
            for (int j = 0; j < ellnum; j++) {
                int64_t r = (int64_t)((uint64_t)d << sub) >> sub;
                d -= r;
                d >>= gbits;
                out[(size_t)(part * ellnum + j) * N + i] = r >= 0 ? (uint64_t)r : (uint64_t)r + modulus;
            }
        }
    }
}

/* ------------------------------------------------------------------ */
/* automorphisms                                                        */

/* pow_mod(int32), utils.cpp:1446-1459: wraps mod 2^32, harmless since 8192 | 2^32 */
int ko_pow_mod_index(int a, int b) {
    uint32_t r = 1;
    for (int i = 0; i < b; i++) r *= (uint32_t)a;
    return (int)(r & (2 * N - 1));
}

/* automorphic_rns, twosteps.cpp:757-783 (canonical negation) */
static void automorphic_rns(uint64_t* res, const uint64_t* in, int index, uint64_t q) {
    for (int i = 0; i < N; i++) {
        uint64_t dst = ((uint64_t)i * (uint64_t)index) & (2 * N - 1);
        if (dst >= N) {
            uint64_t t = q - in[i];
            res[dst - N] = t != q ? t : 0;
        } else {
            res[dst] = in[i];
        }
    }
}

/* the inline automorphism of evalAutoRNSCRT (twosteps.cpp:617-636) and
 * evalAuto (answer.cpp:595-615): negation leaves q for a zero coefficient */
static void automorphic_raw(uint64_t* res, const uint64_t* in, int index, uint64_t q) {
    for (int i = 0; i < N; i++) {
        uint64_t dst = ((uint64_t)i * (uint64_t)index) & (2 * N - 1);
        if (dst >= N) res[dst - N] = q - in[i];
        else res[dst] = in[i];
    }
}

/* ------------------------------------------------------------------ */
/* permutations, utils.cpp:1473-1619                                    */

static void hexl_rotate_indexes(int32_t* hexl_idx, int32_t* rot_idx) {
    memset(hexl_idx, 0, sizeof(int32_t) * N);
    hexl_idx[0] = 1;
    for (int i = 0; (1 << i) < N; i++) {
        int32_t fill = 1 << i, interval = N / fill;
        for (int j = 0; j < fill; j++)
            hexl_idx[j * interval + interval / 2] = hexl_idx[j * interval] * (2 * fill + 1) % (4 * fill);
    }
    rot_idx[0] = 1;
    rot_idx[N - 1] = 2 * N - 1;
    for (int i = 1; i < N / 2; i++) {
        rot_idx[i] = rot_idx[i - 1] * 5 % (2 * N);
        rot_idx[N - 1 - i] = rot_idx[N - 1 - i + 1] * 5 % (2 * N);
    }
}

void ko_permutation_matrix(int32_t* perms, int N1) {
    int32_t* hexl_idx = malloc(sizeof(int32_t) * N);
    int32_t* rot = malloc(sizeof(int32_t) * N);
    int32_t* find = malloc(sizeof(int32_t) * N);
    int32_t* inter = calloc(N, sizeof(int32_t));
    hexl_rotate_indexes(hexl_idx, rot);
    for (int i = 0; i < N; i++) find[hexl_idx[i] >> 1] = i;
    for (int index = 0; index < N1; index++) {
        for (int i = 0; i < N / 2 - index; i++) {
            inter[rot[i] >> 1] = rot[i + index];
            inter[rot[N - 1 - i] >> 1] = rot[N - 1 - i - index];
        }
        for (int i = N / 2 - index; i < N / 2; i++) {
            inter[rot[i] >> 1] = rot[i + index - N / 2];
            inter[rot[N - 1 - i] >> 1] = rot[N - 1 - i - index + N / 2];
        }
        for (int i = 0; i < N; i++)
            perms[(size_t)index * N + i] = find[inter[hexl_idx[i] >> 1] >> 1];
    }
    free(hexl_idx); free(rot); free(find); free(inter);
}

/* ------------------------------------------------------------------ */
/* database preprocessing, twosteps.cpp:42-179 and crt.cpp:859-885      */

/* query_encode, utils.cpp:1657-1675: find_index[rotate_index[i] / 2] */
static void query_encode(int32_t* qe) {
    int32_t* hexl_idx = malloc(sizeof(int32_t) * N);
    int32_t* rot = malloc(sizeof(int32_t) * N);
    int32_t* find = malloc(sizeof(int32_t) * N);
    hexl_rotate_indexes(hexl_idx, rot);
    for (int i = 0; i < N; i++) find[hexl_idx[i] >> 1] = i;
    for (int i = 0; i < N; i++) qe[i] = find[rot[i] / 2];
    free(hexl_idx); free(rot); free(find);
}

int ko_database_tobsgsntt(const uint64_t* raw, int N1, uint64_t* rows) {
    const int H = N / 2, N2 = N / 2 / N1;
    for (size_t i = 0; i < (size_t)N * H; i++)
        if (raw[i] >= KO_P) return -1;
    int32_t* qe = malloc(sizeof(int32_t) * N);
    int32_t* perms = malloc(sizeof(int32_t) * (size_t)N1 * N);
    uint64_t* row = malloc(8 * N);
    uint64_t* tmp = malloc(8 * N);
    query_encode(qe);
    ko_permutation_matrix(perms, N1);
    /* diagonal rearrangement, twosteps.cpp:64-74 */
    for (int i = 0; i < H; i++)
        for (int j = 0; j < H; j++) {
            int rr = (j - i + H) & (H - 1);
            rows[(size_t)i * N + j] = raw[(size_t)rr * H + j];
            rows[(size_t)i * N + N - 1 - j] = raw[(size_t)(N - 1 - rr) * H + j];
        }
    for (int k = 0; k < N2; k++)
        for (int i = 0; i < N1; i++) {
            uint64_t* x = rows + ((size_t)k * N1 + i) * N;
            /* permutation, twosteps.cpp:104-118 */
            for (int j = 0; j < N; j++) tmp[qe[j]] = x[j];
            for (int j = 0; j < N; j++) row[j] = tmp[perms[(size_t)i * N + j]];
            /* encode, twosteps.cpp:156-176 */
            ko_ntt_inverse(row, KO_P);
            for (int j = 0; j < N; j++)
                if (row[j] > KO_P / 2) row[j] += KO_CRTMOD - KO_P;
            ko_ntt_forward(row, KO_CRTMOD);
            memcpy(x, row, 8 * N);
        }
    free(qe); free(perms); free(row); free(tmp);
    return 0;
}

void ko_database_tocrt(const uint64_t* rows, uint64_t* datacrt) {
    /* crt.cpp:868-880 */
    const int H = N / 2;
    for (int z = 0; z < N; z++)
        for (int R = 0; R < H; R++) {
            uint64_t t = rows[(size_t)R * N + z];
            datacrt[(size_t)z * H + R] = ko_barrett_coeff(t, 0) | ko_barrett_coeff(t, 1) << 32;
        }
}

/* The scaled message of query_bsgs_rns (twosteps.cpp:288-307) for row t:
 * m[query_encode[t]] = m[query_encode[N-1-t]] = 1, INTT mod p, then
 * round((long double)me * crtMod / p) as the reference compiles it: the
 * unqualified round there is the C library's round(double), so the long
 * double quotient is first rounded to a double (53-bit mantissa: the scaled
 * words, below 2^56, land on multiples of 4 or 8), then to an integer. */
void ko_query_message(int t, uint64_t* dm) {
    int32_t* qe = malloc(sizeof(int32_t) * N);
    query_encode(qe);
    memset(dm, 0, 8 * N);
    dm[qe[t]] = 1;
    dm[qe[N - 1 - t]] = 1;
    ko_ntt_inverse(dm, KO_P);
    for (int i = 0; i < N; i++) dm[i] = (uint64_t)round((double)((long double)dm[i] * KO_CRTMOD / KO_P));
    free(qe);
}

int ko_db_preprocess(const uint64_t* raw, int N1, uint64_t* datacrt) {
    uint64_t* rows = malloc(8 * (size_t)(N / 2) * N);
    int rc = ko_database_tobsgsntt(raw, N1, rows);
    if (rc == 0) ko_database_tocrt(rows, datacrt);
    free(rows);
    return rc;
}

/* ------------------------------------------------------------------ */
/* first dimension, twosteps.cpp                                        */

#define POLY(p, i) ((p) + (size_t)(i) * N)

/* The hoisted baby steps of one half: evalAutoSRNSFirst (twosteps.cpp:937-1087)
 * when `first`, else evalAutoSRNSSecond (twosteps.cpp:1090-1204).
 *   src_crt / src_bs : [2][N] coefficient-form (a, b) of the rotated source
 *   rot              : [N1-1][2][N] output rotations (mod crtMod, NTT form)
 *   inter_crt/_bs    : (first only) the coefficient-form rotation N1h-1 before modswitch */
static void baby_half(int first, int N1h, uint64_t* src_crt, uint64_t* src_bs, const uint64_t* baby,
                      const int32_t* perms, uint64_t* rot, uint64_t* inter_crt, uint64_t* inter_bs) {
    const int ell = 3;
    const uint64_t base = 1u << 20, bg = 1u << 20;   /* AutoKeyBSGSRNS defaults, lwe.h:391-393 */
    uint64_t* dec = malloc(sizeof(uint64_t) * ell * N);
    uint64_t* dec_aux = malloc(sizeof(uint64_t) * ell * N);
    uint64_t* a1 = malloc(sizeof(uint64_t) * N);
    uint64_t* a2 = malloc(sizeof(uint64_t) * N);
    uint64_t* t1 = malloc(sizeof(uint64_t) * N);
    uint64_t* t2 = malloc(sizeof(uint64_t) * N);
    int nrot = first ? N1h - 1 : N1h;
    uint64_t* aux = calloc((size_t)nrot * 2 * N, sizeof(uint64_t));  /* result_aux, zero */

    ko_decompose_bsgs(src_crt, src_bs, ell, base, bg, dec, dec_aux);
    for (int j = 0; j < ell; j++) {
        NTT_CRT(POLY(dec, j));
        NTT_BS(POLY(dec_aux, j));
    }
    for (int s = 0; s < nrot; s++) {
        int i = s + 1;                          /* rotation index of the key and permutation */
        int dst = first ? s : N1h + s - 1;      /* slot in rot[] */
        const uint64_t* key = baby + (size_t)(i - 1) * 6 * 2 * N;   /* keyMap.at(5^i) */
        const int32_t* perm = perms + (size_t)i * N;
        uint64_t* ra = POLY(rot, 2 * dst);
        uint64_t* rb = POLY(rot, 2 * dst + 1);
        uint64_t* xa = POLY(aux, 2 * s);
        uint64_t* xb = POLY(aux, 2 * s + 1);
        for (int j = 0; j < ell; j++) {
            for (int k = 0; k < N; k++) {
                a1[k] = dec[(size_t)j * N + perm[k]];
                a2[k] = dec_aux[(size_t)j * N + perm[k]];
            }
            vmul(t1, a1, key + (size_t)(2 * j) * N, CRTMOD);
            vmul(t2, a1, key + (size_t)(2 * j + 1) * N, CRTMOD);
            vsub(ra, ra, t1, CRTMOD);
            vsub(rb, rb, t2, CRTMOD);
            vmul(t1, a2, key + (size_t)(2 * (j + ell)) * N, BSMOD);
            vmul(t2, a2, key + (size_t)(2 * (j + ell) + 1) * N, BSMOD);
            vsub(xa, xa, t1, BSMOD);
            vsub(xb, xb, t2, BSMOD);
        }
    }
    /* rns modswitch */
    for (int s = 0; s < nrot; s++) {
        int dst = first ? s : N1h + s - 1;
        uint64_t* ra = POLY(rot, 2 * dst);
        uint64_t* rb = POLY(rot, 2 * dst + 1);
        uint64_t* xa = POLY(aux, 2 * s);
        uint64_t* xb = POLY(aux, 2 * s + 1);
        INTT_CRT(ra); INTT_CRT(rb);
        INTT_BS(xa); INTT_BS(xb);
        int g = ko_pow_mod_index(5, s + 1);
        automorphic_rns(t1, POLY(src_crt, 1), g, CRTMOD);
        automorphic_rns(t2, POLY(src_bs, 1), g, BSMOD);
        vadd(rb, rb, t1, CRTMOD);
        vadd(xb, xb, t2, BSMOD);
        if (first && s == N1h - 2) {
            memcpy(inter_crt, ra, 8 * N); memcpy(inter_crt + N, rb, 8 * N);
            memcpy(inter_bs, xa, 8 * N); memcpy(inter_bs + N, xb, 8 * N);
        }
        vsub(ra, ra, xa, CRTMOD);
        vmulc(ra, ra, BSMOD_INV, CRTMOD);
        NTT_CRT(ra);
        vsub(rb, rb, xb, CRTMOD);
        vmulc(rb, rb, BSMOD_INV, CRTMOD);
        NTT_CRT(rb);
    }
    if (first) {  /* rns modswitch of the input itself, twosteps.cpp:1073-1086 */
        vsub(POLY(src_crt, 0), POLY(src_crt, 0), POLY(src_bs, 0), CRTMOD);
        vmulc(POLY(src_crt, 0), POLY(src_crt, 0), BSMOD_INV, CRTMOD);
        NTT_CRT(POLY(src_crt, 0));
        vsub(POLY(src_crt, 1), POLY(src_crt, 1), POLY(src_bs, 1), CRTMOD);
        vmulc(POLY(src_crt, 1), POLY(src_crt, 1), BSMOD_INV, CRTMOD);
        NTT_CRT(POLY(src_crt, 1));
    }
    free(dec); free(dec_aux); free(a1); free(a2); free(t1); free(t2); free(aux);
}

/* evalAutoRNSCRT, twosteps.cpp:599-677: result += sum_{c>=1} giant-step key switch of output[c].
 * output is [N2][2][N] NTT form and is INTT'd in place for c >= 1 (as the reference does). */
static void eval_auto_rns_crt(uint64_t* result, uint64_t* output, int N2, int N1, const uint64_t* giant) {
    const int ell = 2;
    const uint64_t base = 1u << 20, bg = 1u << 18;   /* lwe.h:402-404 */
    uint64_t* ta = malloc(8 * N);
    uint64_t* tb = malloc(8 * N);
    uint64_t* tmp = malloc(8 * N);
    uint64_t* dec = malloc(8 * (size_t)ell * N);
    for (int c = 1; c < N2; c++) {
        uint64_t* in_a = output + (size_t)c * 2 * N;
        uint64_t* in_b = in_a + N;
        INTT_CRT(in_a);
        INTT_CRT(in_b);
        int index = ko_pow_mod_index(5, N1 * c);
        automorphic_raw(ta, in_a, index, CRTMOD);
        automorphic_raw(tb, in_b, index, CRTMOD);
        ko_decompose(ta, ell, base, bg, CRTMOD, dec);
        const uint64_t* key = giant + (size_t)(c - 1) * 2 * 2 * N;
        NTT_CRT(tb);
        vadd(result + N, result + N, tb, CRTMOD);
        for (int i = 0; i < ell; i++) {
            NTT_CRT(POLY(dec, i));
            vmul(tmp, POLY(dec, i), key + (size_t)(2 * i) * N, CRTMOD);
            vsub(result, result, tmp, CRTMOD);
            vmul(tmp, POLY(dec, i), key + (size_t)(2 * i + 1) * N, CRTMOD);
            vsub(result + N, result + N, tmp, CRTMOD);
        }
    }
    free(ta); free(tb); free(tmp); free(dec);
}

/* the giant steps of one sub-database on its scan output (output is INTT'd in place) */
int ko_giant_steps(uint64_t* result, uint64_t* output, int N1, const uint64_t* giant) {
    int N2 = N / 2 / N1;
    memcpy(result, output, 8 * 2 * N);
    eval_auto_rns_crt(result, output, N2, N1, giant);
    return 0;
}

/* matrix_vector_mul_bsgs_rns_crt_large, twosteps.cpp:1527-1579 */
int ko_matrix_vector_mul(const uint64_t* datacrt, int r, int N1, uint64_t* query_inout,
                         const uint64_t* baby, const uint64_t* giant, const int32_t* perms,
                         uint64_t* result, uint64_t* cipherbuf_out) {
    if (N1 < 2 || N1 > N / 2 || (N1 & (N1 - 1))) return -1;
    int N2 = N / 2 / N1, N1h = N1 / 2;
    uint64_t* rot = calloc((size_t)(N1 - 1) * 2 * N, sizeof(uint64_t));
    uint64_t* inter_crt = malloc(8 * 2 * N);
    uint64_t* inter_bs = malloc(8 * 2 * N);
    uint64_t* q_crt = query_inout;
    uint64_t* q_bs = query_inout + 2 * N;

    /* evalAutoSRNSSmallKeys, twosteps.cpp:1206-1214 */
    baby_half(1, N1h, q_crt, q_bs, baby, perms, rot, inter_crt, inter_bs);
    baby_half(0, N1h, inter_crt, inter_bs, baby, perms, rot, NULL, NULL);

    /* reorientCipher, twosteps.cpp:1386-1403 */
    uint64_t* cb = cipherbuf_out ? cipherbuf_out : malloc(8 * (size_t)N1 * N * 2);
    for (int i = 0; i < N; i++) {
        for (int j = 0; j < N1; j++) {
            uint64_t va = j == 0 ? q_crt[i] : rot[(size_t)(2 * (j - 1)) * N + i];
            uint64_t vb = j == 0 ? q_crt[N + i] : rot[(size_t)(2 * (j - 1) + 1) * N + i];
            cb[(size_t)i * 2 * N1 + 2 * j] = ko_barrett_coeff(va, 0) | ko_barrett_coeff(va, 1) << 32;
            cb[(size_t)i * 2 * N1 + 2 * j + 1] = ko_barrett_coeff(vb, 0) | ko_barrett_coeff(vb, 1) << 32;
        }
    }
    uint64_t* output = malloc(8 * (size_t)N2 * 2 * N);
    size_t num_words = (size_t)N * N / 2;
    for (int k = 0; k < r; k++) {
        ko_scan(datacrt + (size_t)k * num_words, cb, N1, output);
        memcpy(result + (size_t)k * 2 * N, output, 8 * 2 * N);
        eval_auto_rns_crt(result + (size_t)k * 2 * N, output, N2, N1, giant);
    }
    if (!cipherbuf_out) free(cb);
    free(output); free(rot); free(inter_crt); free(inter_bs);
    return 0;
}

/* ------------------------------------------------------------------ */
/* second dimension and packing                                         */

/* externalProduct, lwe.cpp:761-808 (RGSW ell=2, base 2^20, Bg 2^18: test-pir.cpp:71) */
int ko_external_product(uint64_t* ext, uint64_t* fd, const uint64_t* rgsw) {
    const int ell = 2;
    uint64_t* dec = malloc(8 * (size_t)2 * ell * N);
    uint64_t* tmp = malloc(8 * N);
    INTT_CRT(fd);
    INTT_CRT(fd + N);
    ko_decompose_rlwe(fd, fd + N, ell, 1u << 20, 1u << 18, CRTMOD, dec);
    for (int i = 0; i < 2 * ell; i++) {
        NTT_CRT(POLY(dec, i));
        vmul(tmp, POLY(dec, i), rgsw + (size_t)(2 * i) * N, CRTMOD);
        vadd(ext, ext, tmp, CRTMOD);
    }
    for (int i = 0; i < 2 * ell; i++) {
        vmul(tmp, POLY(dec, i), rgsw + (size_t)(2 * i + 1) * N, CRTMOD);
        vadd(ext + N, ext + N, tmp, CRTMOD);
    }
    INTT_CRT(ext);
    INTT_CRT(ext + N);
    free(dec); free(tmp);
    return 0;
}

/* RlweCiphertext::multConst, lwe.cpp:102-119 (negacyclic X^number; q left for zeros) */
static void mult_const(uint64_t* c, int number) {
    uint64_t* t = malloc(8 * 2 * N);
    memcpy(t, c, 8 * 2 * N);
    for (int p = 0; p < 2; p++) {
        uint64_t* x = c + (size_t)p * N;
        const uint64_t* tx = t + (size_t)p * N;
        for (int i = 0; i < N - number; i++) x[i + number] = tx[i];
        for (int i = N - number; i < N; i++) x[i + number - N] = CRTMOD - tx[i];
    }
    free(t);
}

/* evalAuto, answer.cpp:576-648, on a coefficient-form ciphertext */
static void eval_auto(uint64_t* res, int index, const uint64_t* key) {
    const int ell = 4;
    const uint64_t base = 0, bg = 1u << 14;   /* test-pir.cpp:88 */
    uint64_t* ta = malloc(8 * N);
    uint64_t* tb = malloc(8 * N);
    uint64_t* tmp = malloc(8 * N);
    uint64_t* dec = malloc(8 * (size_t)ell * N);
    automorphic_raw(ta, res, index, CRTMOD);
    automorphic_raw(tb, res + N, index, CRTMOD);
    memset(res, 0, 8 * N);
    ko_decompose(ta, ell, base, bg, CRTMOD, dec);
    memcpy(res + N, tb, 8 * N);
    NTT_CRT(res + N);
    for (int i = 0; i < ell; i++) {
        NTT_CRT(POLY(dec, i));
        vmul(tmp, POLY(dec, i), key + (size_t)(2 * i) * N, CRTMOD);
        vsub(res, res, tmp, CRTMOD);
        vmul(tmp, POLY(dec, i), key + (size_t)(2 * i + 1) * N, CRTMOD);
        vsub(res + N, res + N, tmp, CRTMOD);
    }
    INTT_CRT(res);
    INTT_CRT(res + N);
    free(ta); free(tb); free(tmp); free(dec);
}

/* packingRLWEs, answer.cpp:800-835, over convertTwoRLWEs, answer.cpp:720-739 */
int ko_packing(uint64_t* rl, int r, const uint64_t* packing, uint64_t* response) {
    if (r < 1 || (r & (r - 1))) return -1;
    uint64_t* temp = malloc(8 * 2 * N);
    for (int i = r / 2; i > 0; i >>= 1) {
        int level = 0;
        while ((1 << level) < i) level++;           /* key N/i + 1 is level log2(i) */
        const uint64_t* key = packing + (size_t)level * 4 * 2 * N;
        for (int j = 0; j < i; j++) {
            uint64_t* res = rl + (size_t)j * 2 * N;
            uint64_t* cip = rl + (size_t)(i + j) * 2 * N;
            int xn = r / (r / i);                   /* XNdiv2l = rlweNums / twol */
            mult_const(cip, xn);
            memcpy(temp, res, 8 * 2 * N);
            vsub(res, res, cip, CRTMOD);
            vsub(res + N, res + N, cip + N, CRTMOD);
            vadd(cip, cip, temp, CRTMOD);
            vadd(cip + N, cip + N, temp + N, CRTMOD);
            eval_auto(res, N / xn + 1, key);
            vadd(res, res, cip, CRTMOD);
            vadd(res + N, res + N, cip + N, CRTMOD);
        }
    }
    memcpy(response, rl, 8 * 2 * N);
    free(temp);
    return 0;
}

/* test-pir.cpp:110-116 */
int ko_answer(const uint64_t* datacrt, int r, int N1, const uint64_t* query,
              const uint64_t* baby, const uint64_t* giant, const uint64_t* packing,
              const uint64_t* rgsw, const int32_t* perms, uint64_t* response,
              uint64_t* bsgs_out, uint64_t* ext_out) {
    uint64_t* q = malloc(8 * 4 * N);
    uint64_t* res = malloc(8 * (size_t)r * 2 * N);
    uint64_t* ext = calloc((size_t)r * 2 * N, sizeof(uint64_t));
    memcpy(q, query, 8 * 4 * N);
    int rc = ko_matrix_vector_mul(datacrt, r, N1, q, baby, giant, perms, res, NULL);
    if (rc == 0) {
        if (bsgs_out) memcpy(bsgs_out, res, 8 * (size_t)r * 2 * N);
        for (int j = 0; j < r; j++)
            ko_external_product(ext + (size_t)j * 2 * N, res + (size_t)j * 2 * N, rgsw);
        if (ext_out) memcpy(ext_out, ext, 8 * (size_t)r * 2 * N);
        rc = ko_packing(ext, r, packing, response);
    }
    free(q); free(res); free(ext);
    return rc;
}
