/*
 * CPU oracle for the Toothpaste blind-rotation hot path (TEST INFRASTRUCTURE).
 * See tp_oracle.h for the contract. Plain C11 + unsigned __int128; scalar code
 * only, written for clarity rather than speed. Citations are file:line in the
 * reference project.
 */
#include "tp_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

#define P TPO_P
#define EPS 0xFFFFFFFFULL

/* ------------------------------------------------------------------------- */
/* sampler                                                                   */
/* ------------------------------------------------------------------------- */

void tpo_rng_seed(tpo_rng* r, uint64_t seed) { r->s = seed; }

uint64_t tpo_next64(tpo_rng* r) {
    uint64_t z = (r->s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

uint64_t tpo_uniform(tpo_rng* r, uint64_t q) {
    if (q == 0) return tpo_next64(r);
    uint64_t mask = q - 1;
    mask |= mask >> 1; mask |= mask >> 2; mask |= mask >> 4;
    mask |= mask >> 8; mask |= mask >> 16; mask |= mask >> 32;
    for (;;) {
        uint64_t x = tpo_next64(r) & mask;
        if (x < q) return x;
    }
}

uint64_t tpo_gaussian(tpo_rng* r, double std_dev, uint64_t q) {
    if (std_dev == 0.0) return 0;
    const double u1 = (double)((tpo_next64(r) >> 11) + 1) * 0x1.0p-53;  /* (0, 1] */
    const double u2 = (double)(tpo_next64(r) >> 11) * 0x1.0p-53;        /* [0, 1) */
    const double rad = sqrt(-2.0 * log(u1));
    const double ang = 6.283185307179586 * u2;
    const double z = rad * cos(ang);
    const long long k = llround(z * std_dev);
    if (k >= 0) return (uint64_t)k % q;
    const uint64_t m = (uint64_t)(-k) % q;
    return m == 0 ? 0 : q - m;
}

/* ------------------------------------------------------------------------- */
/* Goldilocks arithmetic: canonical in, canonical out                        */
/* ------------------------------------------------------------------------- */

uint64_t tpo_add(uint64_t a, uint64_t b) {
    u128 s = (u128)a + b;
    if (s >= P) s -= P;
    return (uint64_t)s;
}

uint64_t tpo_sub(uint64_t a, uint64_t b) { return a >= b ? a - b : a + (P - b); }

/* 128-bit value -> canonical, with 2^64 = 2^32 - 1 and 2^96 = -1 (mod p)
 * (elemops::reduce128, lib/include/backend/solinas_internal.h:62-73). */
static uint64_t reduce128(u128 x) {
    const uint64_t lo = (uint64_t)x, hi = (uint64_t)(x >> 64);
    const uint64_t hh = hi >> 32, hl = hi & EPS;
    uint64_t t = lo - hh;
    if (lo < hh) t -= EPS;
    const uint64_t u = (hl << 32) - hl;
    uint64_t r = t + u;
    if (r < u) r += EPS;
    return r >= P ? r - P : r;
}

uint64_t tpo_mul(uint64_t a, uint64_t b) { return reduce128((u128)a * b); }

uint64_t tpo_pow(uint64_t b, uint64_t e) {
    uint64_t r = 1;
    b %= P;
    while (e) {
        if (e & 1) r = tpo_mul(r, b);
        b = tpo_mul(b, b);
        e >>= 1;
    }
    return r;
}

uint64_t tpo_inv(uint64_t a) { return a % P == 0 ? 0 : tpo_pow(a, P - 2); }

/* generic modulus helpers (LWE arithmetic mod q) */
static uint64_t addq(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a + b) % q); }
static uint64_t subq(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : (uint64_t)((u128)a + q - b); }
static uint64_t mulq(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }

/* ceil(log2(x)); IntLog2 of lib/src/utils/math_utils.cpp:11-25 */
static uint64_t int_log2(uint64_t x) {
    if (x <= 1) return 0;
    uint64_t r = 0;
    x -= 1;
    while (x) { r++; x >>= 1; }
    return r;
}

/* ------------------------------------------------------------------------- */
/* NTT                                                                       */
/* ------------------------------------------------------------------------- */

static uint32_t brv(uint32_t x, unsigned bits) {
    uint32_t r = 0;
    for (unsigned i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

typedef struct {
    uint64_t N;
    unsigned logn;
    uint64_t* psi_rev;      /* psi^brv(k) */
    uint64_t* psi_inv_rev;  /* psi^-brv(k) */
    uint64_t n_inv;
} ntt_tables;

static pthread_mutex_t g_tab_lock = PTHREAD_MUTEX_INITIALIZER;
static ntt_tables* g_tabs[17];

uint64_t tpo_psi(uint64_t N) {
    unsigned logn = (unsigned)int_log2(N);
    return tpo_pow(7, (P - 1) >> (logn + 1));
}

/* Twiddle tables as in SolinasWorker's constructor (lib/src/backend/solinas.cpp:168-192). */
static const ntt_tables* get_tables(uint64_t N) {
    if (N < 2 || N > 65536 || (N & (N - 1))) return NULL;
    unsigned logn = (unsigned)int_log2(N);
    pthread_mutex_lock(&g_tab_lock);
    if (!g_tabs[logn]) {
        ntt_tables* t = (ntt_tables*)calloc(1, sizeof(ntt_tables));
        t->N = N;
        t->logn = logn;
        t->psi_rev = (uint64_t*)malloc(N * 8);
        t->psi_inv_rev = (uint64_t*)malloc(N * 8);
        const uint64_t psi = tpo_psi(N);
        const uint64_t psi_inv = tpo_inv(psi);
        uint64_t* pw = (uint64_t*)malloc(N * 8);
        uint64_t* pwi = (uint64_t*)malloc(N * 8);
        pw[0] = pwi[0] = 1;
        for (uint64_t i = 1; i < N; ++i) {
            pw[i] = tpo_mul(pw[i - 1], psi);
            pwi[i] = tpo_mul(pwi[i - 1], psi_inv);
        }
        for (uint64_t i = 0; i < N; ++i) {
            t->psi_rev[i] = pw[brv((uint32_t)i, logn)];
            t->psi_inv_rev[i] = pwi[brv((uint32_t)i, logn)];
        }
        free(pw);
        free(pwi);
        t->n_inv = tpo_inv(N);
        g_tabs[logn] = t;
    }
    const ntt_tables* res = g_tabs[logn];
    pthread_mutex_unlock(&g_tab_lock);
    return res;
}

/* Cooley-Tukey, natural order in, bit-reversed order out
 * (lib/src/backend/solinas.cpp:228-261: block i of the level with m blocks uses psi_rev[m+i]). */
int tpo_ntt_forward(uint64_t N, uint64_t* out, const uint64_t* in) {
    const ntt_tables* tb = get_tables(N);
    if (!tb) return -1;
    if (out != in) memmove(out, in, N * 8);
    for (uint64_t m = 1, t = N / 2; m < N; m <<= 1, t >>= 1) {
        for (uint64_t i = 0; i < m; ++i) {
            const uint64_t w = tb->psi_rev[m + i];
            uint64_t* a = out + 2 * i * t;
            for (uint64_t j = 0; j < t; ++j) {
                const uint64_t u = a[j];
                const uint64_t v = tpo_mul(a[j + t], w);
                a[j] = tpo_add(u, v);
                a[j + t] = tpo_sub(u, v);
            }
        }
    }
    return 0;
}

/* Gentleman-Sande, bit-reversed in, natural out, times 1/N
 * (lib/src/backend/solinas.cpp:263-313). */
int tpo_ntt_backward(uint64_t N, uint64_t* out, const uint64_t* in) {
    const ntt_tables* tb = get_tables(N);
    if (!tb) return -1;
    if (out != in) memmove(out, in, N * 8);
    for (uint64_t m = N / 2, t = 1; m >= 1; m >>= 1, t <<= 1) {
        for (uint64_t i = 0; i < m; ++i) {
            const uint64_t w = tb->psi_inv_rev[m + i];
            uint64_t* a = out + 2 * i * t;
            for (uint64_t j = 0; j < t; ++j) {
                const uint64_t u = a[j];
                const uint64_t v = a[j + t];
                a[j] = tpo_add(u, v);
                a[j + t] = tpo_mul(tpo_sub(u, v), w);
            }
        }
    }
    for (uint64_t j = 0; j < N; ++j) out[j] = tpo_mul(out[j], tb->n_inv);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* gadget decomposition                                                      */
/* ------------------------------------------------------------------------- */

/* GetCorrectorForSignedToUnsigned (lib/include/static/gadget_decomp.h:16-28). */
static void signed_corrector(uint64_t q, uint64_t modulus_bits, uint64_t basis_bits,
                             uint64_t* corr, uint64_t* least) {
    uint64_t c = 0;
    int64_t shift = (int64_t)modulus_bits - (int64_t)basis_bits;
    while (shift > 0) {
        c += 1ULL << (shift + (int64_t)basis_bits - 1);
        shift -= (int64_t)basis_bits;
    }
    const uint64_t l = 1ULL << (shift + (int64_t)basis_bits - 1);
    c += l;
    *corr = c % q;
    *least = l;
}

/* Signed digits of one canonical value, most significant first
 * (lib/include/static/gadget_decomp.h:156-205: x' = x + corr, digit j =
 * ((x' >> (64 - beta - j*beta)) & mask) - 2^(beta-1); at j == max_digits-1
 * shift 0 and the least-digit correction). Digits are returned mod q. */
static void signed_digits_scalar(uint64_t x, uint64_t q, uint64_t modulus_bits, uint64_t digits,
                                 uint64_t basis_log2, uint64_t* d) {
    uint64_t corr, least;
    signed_corrector(q, modulus_bits, basis_log2, &corr, &least);
    const uint64_t xc = addq(x, corr, q);
    uint64_t mask = (1ULL << basis_log2) - 1;
    int64_t shift = (int64_t)modulus_bits - (int64_t)basis_log2;
    const uint64_t max_digits = modulus_bits / basis_log2 + (modulus_bits % basis_log2 == 0 ? 0 : 1);
    for (uint64_t j = 0; j < digits; ++j) {
        uint64_t delta = 1ULL << (basis_log2 - 1);
        if (j == max_digits - 1) {
            delta = least;
            shift = 0;
            mask = (delta << 1) - 1;
        }
        const uint64_t raw = (xc >> shift) & mask;
        d[j] = subq(raw, delta, q);
        shift -= (int64_t)basis_log2;
    }
}

void tpo_signed_digits(uint64_t* out, const uint64_t* in, uint64_t N, uint64_t digits, uint64_t basis_log2) {
    uint64_t d[64];
    for (uint64_t i = 0; i < N; ++i) {
        signed_digits_scalar(in[i], P, 64, digits, basis_log2, d);
        for (uint64_t j = 0; j < digits; ++j) out[j * N + i] = d[j];
    }
}

/* MuxOperator first_shift = beta * (ceil(64/beta) - 1) (lib/src/operators/mux_operator.cpp:24-26). */
static uint64_t unsigned_first_shift(uint64_t basis_log2) {
    return basis_log2 * ((64 + basis_log2 - 1) / basis_log2 - 1);
}

void tpo_unsigned_digits(uint64_t* out, const uint64_t* in, uint64_t N, uint64_t digits, uint64_t basis_log2) {
    const uint64_t mask = (1ULL << basis_log2) - 1;
    const uint64_t first = unsigned_first_shift(basis_log2);
    for (uint64_t j = 0; j < digits; ++j) {
        const uint64_t shift = first - j * basis_log2;
        for (uint64_t i = 0; i < N; ++i) out[j * N + i] = (in[i] >> shift) & mask;
    }
}

/* ------------------------------------------------------------------------- */
/* encryption / keygen                                                       */
/* ------------------------------------------------------------------------- */

/* RLWEEncryptor::MakeRLWE (lib/src/base_crypto.cpp:27-58). */
void tpo_make_rlwe(tpo_rng* r, uint64_t N, double std_dev, uint64_t* out, const uint64_t* msg,
                   const uint64_t* sk_ntt, int msg_is_ntt) {
    uint64_t* e = (uint64_t*)malloc(N * 8);
    for (uint64_t i = 0; i < N; ++i) out[i] = tpo_uniform(r, P);
    for (uint64_t i = 0; i < N; ++i) e[i] = tpo_gaussian(r, std_dev, P);
    for (uint64_t i = 0; i < N; ++i) out[N + i] = tpo_mul(out[i], sk_ntt[i]);
    if (msg_is_ntt) {
        tpo_ntt_forward(N, e, e);
        for (uint64_t i = 0; i < N; ++i) e[i] = tpo_add(e[i], msg[i]);
    } else {
        for (uint64_t i = 0; i < N; ++i) e[i] = tpo_add(e[i], msg[i]);
        tpo_ntt_forward(N, e, e);
    }
    for (uint64_t i = 0; i < N; ++i) out[N + i] = tpo_add(out[N + i], e[i]);
    free(e);
}

/* Rows of an RGSW with explicit gadget factors: rows 0..l-1 encrypt -s*m*g[j],
 * rows l..2l-1 encrypt m*g[j], drawn in the order MakeRGSW draws them (smallest
 * factor first). */
static void make_rgsw_rows(tpo_rng* r, uint64_t N, double std_dev, uint64_t* out, const uint64_t* msg,
                           const uint64_t* sk_ntt, const uint64_t* g, uint64_t digits, int msg_is_ntt) {
    uint64_t* m = (uint64_t*)calloc(3 * N, 8);
    uint64_t* row = (uint64_t*)malloc(2 * N * 8);
    if (msg_is_ntt) {
        memcpy(m, msg, N * 8);
    } else {
        tpo_ntt_forward(N, m, msg);
    }
    for (uint64_t i = 0; i < N; ++i) m[2 * N + i] = tpo_mul(m[i], sk_ntt[i]);
    for (uint64_t i = 0; i < N; ++i) m[N + i] = tpo_sub(0, m[2 * N + i]);
    for (uint64_t d = 0; d < digits; ++d) {
        const uint64_t off = digits - d - 1;
        const uint64_t f = g[off] % P;
        for (uint64_t i = 0; i < 2 * N; ++i) row[i] = tpo_mul(m[i], f);
        tpo_make_rlwe(r, N, std_dev, out + off * 2 * N, row + N, sk_ntt, 1);
        tpo_make_rlwe(r, N, std_dev, out + off * 2 * N + 2 * N * digits, row, sk_ntt, 1);
    }
    free(m);
    free(row);
}

/* RLWEEncryptor::MakeRGSW (lib/src/base_crypto.cpp:60-97): row j carries
 * g_j = B^(max_digits-1-j), max_digits = ceil(log2(Q)/log2(B)) computed in long
 * double as the reference computes it. */
void tpo_make_rgsw(tpo_rng* r, uint64_t N, double std_dev, uint64_t* out, const uint64_t* msg,
                   const uint64_t* sk_ntt, uint64_t basis, uint64_t digits, int msg_is_ntt) {
    const uint64_t max_digits = (uint64_t)ceill(log2l((long double)P) / log2l((long double)basis));
    uint64_t g[64];
    for (uint64_t j = 0; j < digits; ++j) g[j] = tpo_pow(basis % P, max_digits - 1 - j);
    make_rgsw_rows(r, N, std_dev, out, msg, sk_ntt, g, digits, msg_is_ntt);
}

/* RLWEEncryptor::PhaseRLWE (lib/src/base_crypto.cpp:99-108). */
void tpo_phase_rlwe(uint64_t N, uint64_t* out, const uint64_t* rlwe, const uint64_t* sk_ntt) {
    for (uint64_t i = 0; i < N; ++i) out[i] = tpo_sub(rlwe[N + i], tpo_mul(rlwe[i], sk_ntt[i]));
    tpo_ntt_backward(N, out, out);
}

uint64_t tpo_brk_words(int variant, uint64_t N, uint64_t n, uint64_t digits) {
    switch (variant) {
        case TPO_CGGI_BINARY: return n * 4 * N * digits;
        case TPO_CGGI_TERNARY: return n * 8 * N * digits;
        case TPO_BMMP_BINARY: return 3 * (n / 2) * 4 * N * digits;
        default: return 0;
    }
}

static void br_keygen_rows(tpo_rng* r, int variant, uint64_t N, uint64_t n, const uint64_t* g, uint64_t digits,
                           double std_dev, const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t* brk) {
    uint64_t* sk = (uint64_t*)malloc(N * 8);
    uint64_t* data = (uint64_t*)calloc(2 * N, 8);
    const uint64_t rg = 4 * N * digits;
    tpo_ntt_forward(N, sk, rlwe_key);
    if (variant == TPO_CGGI_BINARY) {
        /* cggi_blind_rotation.cpp:264-280 */
        for (uint64_t i = 0; i < n; ++i) {
            data[0] = lwe_key[i];
            make_rgsw_rows(r, N, std_dev, brk + i * rg, data, sk, g, digits, 0);
        }
    } else if (variant == TPO_CGGI_TERNARY) {
        /* cggi_blind_rotation.cpp:282-311 */
        for (uint64_t i = 0; i < n; ++i) {
            data[0] = lwe_key[i] == 1;
            data[N] = lwe_key[i] != 0 && lwe_key[i] != 1;
            make_rgsw_rows(r, N, std_dev, brk + i * 2 * rg, data, sk, g, digits, 0);
            make_rgsw_rows(r, N, std_dev, brk + i * 2 * rg + rg, data + N, sk, g, digits, 0);
        }
    } else {
        /* bmmp_blind_rotation.cpp:229-262 */
        for (uint64_t i = 0; i < n; i += 2) {
            uint64_t* chunk = brk + 3 * (i >> 1) * rg;
            data[0] = lwe_key[i];
            make_rgsw_rows(r, N, std_dev, chunk, data, sk, g, digits, 0);
            data[0] = lwe_key[i + 1];
            make_rgsw_rows(r, N, std_dev, chunk + rg, data, sk, g, digits, 0);
            data[0] = lwe_key[i + 1] * lwe_key[i];
            make_rgsw_rows(r, N, std_dev, chunk + 2 * rg, data, sk, g, digits, 0);
        }
    }
    free(sk);
    free(data);
}

void tpo_br_keygen(tpo_rng* r, int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits,
                   double std_dev, const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t* brk) {
    const uint64_t L = 1ULL << basis_log2;
    const uint64_t max_digits = (uint64_t)ceill(log2l((long double)P) / log2l((long double)L));
    uint64_t g[64];
    for (uint64_t j = 0; j < digits; ++j) g[j] = tpo_pow(L, max_digits - 1 - j);
    br_keygen_rows(r, variant, N, n, g, digits, std_dev, lwe_key, rlwe_key, brk);
}

/* Blind-rotation key whose RGSW rows carry g_j = 2^(64 - beta(j+1)), the weights of
 * the signed decomposition's digits (gadget_decomp.h:176). Equal to the reference's
 * key when beta divides 64; for other bases it is the consistent-gadget variant used
 * only by the decryption tests. */
void tpo_br_keygen_aligned(tpo_rng* r, int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits,
                           double std_dev, const uint64_t* lwe_key, const uint64_t* rlwe_key, uint64_t* brk) {
    uint64_t g[64];
    for (uint64_t j = 0; j < digits; ++j) g[j] = 1ULL << (64 - basis_log2 * (j + 1));
    br_keygen_rows(r, variant, N, n, g, digits, std_dev, lwe_key, rlwe_key, brk);
}

/* ------------------------------------------------------------------------- */
/* blind rotation                                                            */
/* ------------------------------------------------------------------------- */

/* NTT(X^k) for 0 <= k < 2N (k >= N gives -NTT(X^(k-N))), the rows of the
 * reference's SetupMonomials table (cggi_blind_rotation.cpp:474-485). */
static void monomial_ntt(uint64_t N, uint64_t k, uint64_t* out) {
    memset(out, 0, N * 8);
    if (k < N) out[k] = 1;
    else out[k - N] = P - 1;
    tpo_ntt_forward(N, out, out);
}

typedef struct {
    uint64_t N, digits, basis_log2;
    uint64_t* tmp;     /* 2N */
    uint64_t* dig;     /* 2*digits*N: NTT-domain digit polys, A digits then B digits */
    uint64_t* ep;      /* 2N: external product output */
    uint64_t* mon;     /* 3N: monomial / weight polys */
} br_scratch;

static void scratch_init(br_scratch* s, uint64_t N, uint64_t digits, uint64_t basis_log2) {
    s->N = N; s->digits = digits; s->basis_log2 = basis_log2;
    s->tmp = (uint64_t*)malloc(2 * N * 8);
    s->dig = (uint64_t*)malloc(2 * digits * N * 8);
    s->ep = (uint64_t*)malloc(2 * N * 8);
    s->mon = (uint64_t*)malloc(3 * N * 8);
}

static void scratch_free(br_scratch* s) { free(s->tmp); free(s->dig); free(s->ep); free(s->mon); }

/* Digits of the coefficient-domain pair s->tmp = [A | B], each forward-NTT'd into s->dig. */
static void decompose_pair(br_scratch* s, int is_signed) {
    const uint64_t N = s->N, l = s->digits;
    for (int h = 0; h < 2; ++h) {
        if (is_signed) tpo_signed_digits(s->dig + h * l * N, s->tmp + h * N, N, l, s->basis_log2);
        else tpo_unsigned_digits(s->dig + h * l * N, s->tmp + h * N, N, l, s->basis_log2);
    }
    for (uint64_t j = 0; j < 2 * l; ++j) tpo_ntt_forward(N, s->dig + j * N, s->dig + j * N);
}

/* ep = sum_r dig_r * rgsw_row_r (both halves); the RGSW external product of
 * MuxOperator::ExternalProduct / the row sums of TernaryCMux and MultiMux
 * (mux_operator.cpp:30-84,114-121,182-187,276-282). */
static void ext_prod(br_scratch* s, const uint64_t* rgsw) {
    const uint64_t N = s->N, l = s->digits;
    memset(s->ep, 0, 2 * N * 8);
    for (uint64_t r = 0; r < 2 * l; ++r) {
        const uint64_t* d = s->dig + r * N;
        const uint64_t* row = rgsw + r * 2 * N;
        for (uint64_t k = 0; k < N; ++k) {
            s->ep[k] = tpo_add(s->ep[k], tpo_mul(d[k], row[k]));
            s->ep[N + k] = tpo_add(s->ep[N + k], tpo_mul(d[k], row[N + k]));
        }
    }
}

int tpo_blind_rotate(int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits,
                     const uint64_t* brk, uint64_t* result, const uint64_t* lwe, const uint64_t* acc,
                     int out_coef) {
    if (!get_tables(N) || digits == 0 || basis_log2 == 0 || basis_log2 > 32) return -1;
    if (variant == TPO_BMMP_BINARY && (n % 2)) return -1;
    br_scratch s;
    scratch_init(&s, N, digits, basis_log2);
    const uint64_t N2 = 2 * N;
    const uint64_t rg = 4 * N * digits;

    /* BlindRotate: result = copy of acc (cggi_blind_rotation.cpp:242) */
    if (result != acc) memmove(result, acc, N2 * 8);
    tpo_ntt_forward(N, result, result);
    tpo_ntt_forward(N, result + N, result + N);
    /* acc *= X^b (cggi_blind_rotation.cpp:336-355) */
    monomial_ntt(N, lwe[n] % N2, s.mon);
    for (uint64_t k = 0; k < N; ++k) {
        result[k] = tpo_mul(result[k], s.mon[k]);
        result[N + k] = tpo_mul(result[N + k], s.mon[k]);
    }

    if (variant == TPO_CGGI_BINARY) {
        /* BlindRotateBinary loop (cggi_blind_rotation.cpp:366-385) + BinaryCMux (mux_operator.cpp:136-152) */
        for (uint64_t i = 0; i < n; ++i) {
            const uint64_t a = lwe[i] % N2;   /* inputs are specified in [0, 2N) */
            if (a == 0) continue;
            monomial_ntt(N, N2 - a, s.mon);                              /* X^{-a} */
            for (uint64_t k = 0; k < N; ++k) s.mon[k] = tpo_sub(s.mon[k], 1);  /* - 1 */
            for (uint64_t k = 0; k < N; ++k) {
                s.tmp[k] = tpo_mul(result[k], s.mon[k]);
                s.tmp[N + k] = tpo_mul(result[N + k], s.mon[k]);
            }
            tpo_ntt_backward(N, s.tmp, s.tmp);
            tpo_ntt_backward(N, s.tmp + N, s.tmp + N);
            decompose_pair(&s, 0);
            ext_prod(&s, brk + i * rg);
            for (uint64_t k = 0; k < N2; ++k) result[k] = tpo_add(result[k], s.ep[k]);
        }
    } else if (variant == TPO_CGGI_TERNARY) {
        /* BlindRotateTernary loop (cggi_blind_rotation.cpp:440-471) + TernaryCMux (mux_operator.cpp:156-202) */
        for (uint64_t i = 0; i < n; ++i) {
            const uint64_t a = lwe[i] % N2;   /* inputs are specified in [0, 2N) */
            if (a == 0) continue;
            uint64_t* mpos = s.mon;       /* X^{-a} - 1 */
            uint64_t* mneg = s.mon + N;   /* X^{a} - 1 */
            monomial_ntt(N, N2 - a, mpos);
            monomial_ntt(N, a, mneg);
            for (uint64_t k = 0; k < N; ++k) {
                mpos[k] = tpo_sub(mpos[k], 1);
                mneg[k] = tpo_sub(mneg[k], 1);
            }
            tpo_ntt_backward(N, s.tmp, result);
            tpo_ntt_backward(N, s.tmp + N, result + N);
            decompose_pair(&s, 1);
            const uint64_t* lo = brk + i * 2 * rg;
            const uint64_t* hi = lo + rg;
            ext_prod(&s, lo);
            for (uint64_t k = 0; k < N; ++k) {
                result[k] = tpo_add(result[k], tpo_mul(s.ep[k], mpos[k]));
                result[N + k] = tpo_add(result[N + k], tpo_mul(s.ep[N + k], mpos[k]));
            }
            ext_prod(&s, hi);
            for (uint64_t k = 0; k < N; ++k) {
                result[k] = tpo_add(result[k], tpo_mul(s.ep[k], mneg[k]));
                result[N + k] = tpo_add(result[N + k], tpo_mul(s.ep[N + k], mneg[k]));
            }
        }
    } else if (variant == TPO_BMMP_BINARY) {
        /* BMMP BlindRotateBinary (bmmp_blind_rotation.cpp:398-416), BuildStepPolynomials
         * (:280-323), MultiMux with k = 3 (mux_operator.cpp:204-294) */
        uint64_t* w = (uint64_t*)malloc(3 * N * 8);
        for (uint64_t i = 0; i < n; i += 2) {
            const uint64_t a0 = (N2 - lwe[i]) & (N2 - 1);
            const uint64_t a1 = (N2 - lwe[i + 1]) & (N2 - 1);
            const uint64_t sum = (a0 + a1) & (N2 - 1);
            monomial_ntt(N, a0, w);
            monomial_ntt(N, a1, w + N);
            monomial_ntt(N, sum, w + 2 * N);
            for (uint64_t k = 0; k < N; ++k) {
                const uint64_t x0 = w[k], x1 = w[N + k];
                w[2 * N + k] = tpo_add(tpo_sub(tpo_sub(w[2 * N + k], x0), x1), 1);
                w[k] = tpo_sub(x0, 1);
                w[N + k] = tpo_sub(x1, 1);
            }
            tpo_ntt_backward(N, s.tmp, result);
            tpo_ntt_backward(N, s.tmp + N, result + N);
            decompose_pair(&s, 1);
            const uint64_t* keys = brk + 3 * (i >> 1) * rg;
            for (int c = 0; c < 3; ++c) {
                ext_prod(&s, keys + c * rg);
                for (uint64_t k = 0; k < N; ++k) {
                    result[k] = tpo_add(result[k], tpo_mul(s.ep[k], w[c * N + k]));
                    result[N + k] = tpo_add(result[N + k], tpo_mul(s.ep[N + k], w[c * N + k]));
                }
            }
        }
        free(w);
    } else {
        scratch_free(&s);
        return -1;
    }

    if (out_coef) {
        tpo_ntt_backward(N, result, result);
        tpo_ntt_backward(N, result + N, result + N);
    }
    scratch_free(&s);
    return 0;
}

typedef struct {
    int variant;
    uint64_t N, n, basis_log2, digits, count, out_coef;
    const uint64_t* brk;
    uint64_t* results;
    const uint64_t* lwes;
    const uint64_t* accs;
    int tid, threads;
    int rc;
} br_job;

static void* br_worker(void* arg) {
    br_job* j = (br_job*)arg;
    j->rc = 0;
    for (uint64_t b = (uint64_t)j->tid; b < j->count; b += (uint64_t)j->threads) {
        int rc = tpo_blind_rotate(j->variant, j->N, j->n, j->basis_log2, j->digits, j->brk,
                                  j->results + b * 2 * j->N, j->lwes + b * (j->n + 1),
                                  j->accs + b * 2 * j->N, (int)j->out_coef);
        if (rc) j->rc = rc;
    }
    return NULL;
}

int tpo_blind_rotate_many(int variant, uint64_t N, uint64_t n, uint64_t basis_log2, uint64_t digits,
                          const uint64_t* brk, uint64_t* results, const uint64_t* lwes,
                          const uint64_t* accs, uint64_t count, int out_coef, int threads) {
    if (threads < 1) threads = 1;
    if (!get_tables(N)) return -1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    br_job* jobs = (br_job*)malloc(sizeof(br_job) * (size_t)threads);
    for (int t = 0; t < threads; ++t) {
        br_job j = {variant, N, n, basis_log2, digits, count, (uint64_t)out_coef, brk, results, lwes, accs, t, threads, 0};
        jobs[t] = j;
        pthread_create(&th[t], NULL, br_worker, &jobs[t]);
    }
    int rc = 0;
    for (int t = 0; t < threads; ++t) {
        pthread_join(th[t], NULL);
        if (jobs[t].rc) rc = jobs[t].rc;
    }
    free(th);
    free(jobs);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* key switching                                                             */
/* ------------------------------------------------------------------------- */

/* RLWEtoRLWEConverter::KeyGen (lib/src/operators/rlwe_conversion.cpp:187-218). */
void tpo_rlwe_ks_keygen(tpo_rng* r, uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev,
                        const uint64_t* source_key, const uint64_t* target_key, uint64_t* ksk) {
    uint64_t* tk = (uint64_t*)malloc(N * 8);
    uint64_t* g = (uint64_t*)malloc(N * 8);
    tpo_ntt_forward(N, tk, target_key);
    uint64_t gij = 1ULL << (64 - basis_log2);
    for (uint64_t i = 0; i < digits; ++i) {
        for (uint64_t k = 0; k < N; ++k) g[k] = tpo_mul(source_key[k] % P, gij % P);
        tpo_make_rlwe(r, N, std_dev, ksk + i * 2 * N, g, tk, 0);
        gij >>= basis_log2;
        if (gij == 0) gij = 1;
    }
    free(tk);
    free(g);
}

/* RLWEtoRLWEConverter::Convert (lib/src/operators/rlwe_conversion.cpp:224-249). */
void tpo_rlwe_ks(uint64_t N, uint64_t basis_log2, uint64_t digits, const uint64_t* ksk,
                 uint64_t* out, const uint64_t* in) {
    uint64_t* d = (uint64_t*)malloc(digits * N * 8);
    tpo_signed_digits(d, in, N, digits, basis_log2);
    for (uint64_t j = 0; j < digits; ++j) tpo_ntt_forward(N, d + j * N, d + j * N);
    for (uint64_t k = 0; k < N; ++k) {
        uint64_t sa = 0, sb = 0;
        for (uint64_t j = 0; j < digits; ++j) {
            sa = tpo_add(sa, tpo_mul(d[j * N + k], ksk[j * 2 * N + k]));
            sb = tpo_add(sb, tpo_mul(d[j * N + k], ksk[j * 2 * N + N + k]));
        }
        out[k] = tpo_sub(out[k], sa);
        out[N + k] = tpo_sub(out[N + k], sb);
    }
    for (uint64_t k = 0; k < N; ++k) out[N + k] = tpo_add(out[N + k], in[N + k]);
    free(d);
}

/* LWEEncryptor::MakeLWE (lib/src/base_crypto.cpp:137-155). */
void tpo_make_lwe(tpo_rng* r, uint64_t q, uint64_t n, double std_dev, uint64_t* out, uint64_t msg,
                  const uint64_t* secret) {
    for (uint64_t i = 0; i < n; ++i) out[i] = tpo_uniform(r, q);
    uint64_t b = tpo_gaussian(r, std_dev, q);
    for (uint64_t i = 0; i < n; ++i) b = addq(b, mulq(out[i], secret[i] % q, q), q);
    out[n] = addq(b, msg % q, q);
}

/* LWEtoLWEConverter::KeyGen (lib/src/operators/lwe_conversion.cpp:174-203). */
void tpo_lwe_ks_keygen(tpo_rng* r, uint64_t q, uint64_t n_in, uint64_t n_out, uint64_t basis_log2,
                       uint64_t digits, double std_dev, const uint64_t* source_key,
                       const uint64_t* target_key, uint64_t* ksk) {
    const uint64_t mb = int_log2(q);
    for (uint64_t i = 0; i < n_in; ++i) {
        uint64_t* chunk = ksk + i * digits * (n_out + 1);
        uint64_t g = 1ULL << (mb - basis_log2);
        for (uint64_t j = 0; j < digits; ++j, chunk += n_out + 1) {
            const uint64_t entry = mulq(g % q, source_key[i] % q, q);
            tpo_make_lwe(r, q, n_out, std_dev, chunk, entry, target_key);
            g >>= basis_log2;
        }
    }
}

/* LWEtoLWEConverter::Convert (lib/src/operators/lwe_conversion.cpp:205-239). */
void tpo_lwe_ks(uint64_t q, uint64_t n_in, uint64_t n_out, uint64_t basis_log2, uint64_t digits,
                const uint64_t* ksk, uint64_t* out, const uint64_t* in) {
    const uint64_t mb = int_log2(q);
    uint64_t* acc = (uint64_t*)calloc(n_out + 1, 8);
    out[n_out] = in[n_in];
    uint64_t d[64];
    for (uint64_t i = 0; i < n_in; ++i) {
        signed_digits_scalar(in[i], q, mb, digits, basis_log2, d);
        const uint64_t* chunk = ksk + i * digits * (n_out + 1);
        for (uint64_t j = 0; j < digits; ++j, chunk += n_out + 1)
            for (uint64_t k = 0; k <= n_out; ++k) acc[k] = addq(acc[k], mulq(chunk[k], d[j], q), q);
    }
    for (uint64_t k = 0; k <= n_out; ++k) out[k] = subq(out[k], acc[k], q);
    free(acc);
}

/* ------------------------------------------------------------------------- */
/* automorphisms and packing                                                 */
/* ------------------------------------------------------------------------- */

/* EvalNegacyclicAutomorphism (lib/src/utils/math_utils.cpp:70-85) and
 * ApplyAutomorphism (lib/src/operators/automorphism_evaluation.cpp:183-206):
 * coefficient i moves to i*index mod 2N, negated when that lands in [N, 2N). */
void tpo_negacyclic_automorphism(uint64_t* out, const uint64_t* in, uint64_t index, uint64_t N) {
    for (uint64_t i = 0; i < N; ++i) {
        const uint64_t t = (i * index) & (2 * N - 1);
        const uint64_t v = in[i];
        out[t & (N - 1)] = t >= N ? (v == 0 ? 0 : P - v) : v;
    }
}

/* AutomorphismContext::ConstructOperator (automorphism_evaluation.cpp:43-63):
 * a key switch from s(X^index) to s(X). */
void tpo_auto_keygen(tpo_rng* r, uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev,
                     uint64_t index, const uint64_t* rlwe_key, uint64_t* ksk) {
    uint64_t* ka = (uint64_t*)malloc(N * 8);
    tpo_negacyclic_automorphism(ka, rlwe_key, index, N);
    tpo_rlwe_ks_keygen(r, N, basis_log2, digits, std_dev, ka, rlwe_key, ksk);
    free(ka);
}

/* AutomorphismEvaluator::Eval (automorphism_evaluation.cpp:150-159). */
void tpo_auto_eval(uint64_t N, uint64_t basis_log2, uint64_t digits, uint64_t index,
                   const uint64_t* ksk, uint64_t* out, const uint64_t* in) {
    uint64_t* buf = (uint64_t*)malloc(2 * N * 8);
    tpo_negacyclic_automorphism(buf, in, index, N);
    tpo_negacyclic_automorphism(buf + N, in + N, index, N);
    tpo_ntt_forward(N, buf + N, buf + N);
    tpo_rlwe_ks(N, basis_log2, digits, ksk, out, buf);
    free(buf);
}

/* LWEtoRLWEPackingContext::ConstructOperator (lwe_to_rlwe_packing.cpp:46-58):
 * one automorphism key per index 2^j + 1, j = 1..logN, in that order. */
void tpo_pack_keygen(tpo_rng* r, uint64_t N, uint64_t basis_log2, uint64_t digits, double std_dev,
                     const uint64_t* rlwe_key, uint64_t* keys) {
    const uint64_t logn = int_log2(N);
    for (uint64_t j = 1; j <= logn; ++j)
        tpo_auto_keygen(r, N, basis_log2, digits, std_dev, (1ULL << j) + 1, rlwe_key,
                        keys + (j - 1) * 2 * N * digits);
}

/* L0Setup (lwe_to_rlwe_packing.cpp:238-251): LWE (a, b) -> RLWE (A, B) with
 * const-coef phase b - <a,s>, scaled by N^-1; B has only its constant term. */
static void l0_setup(uint64_t N, uint64_t* out, const uint64_t* in) {
    const uint64_t ninv = tpo_inv(N);
    memset(out, 0, 2 * N * 8);
    out[0] = in[0];
    for (uint64_t i = 1; i < N / 2; ++i) {
        out[i] = tpo_sub(0, in[N - i]);
        out[N - i] = tpo_sub(0, in[i]);
    }
    out[N / 2] = tpo_sub(0, in[N / 2]);
    out[N] = in[N];
    for (uint64_t i = 0; i <= N; ++i) out[i] = tpo_mul(out[i], ninv);
}

/* One packing merge at output level L (lwe_to_rlwe_packing.cpp:180-214):
 * rot = X^(N>>L) * left; left' = right + rot; right' = right - rot;
 * left' += INTT(Auto_{2^L+1}(right')). Writes the merged RLWE to `left`. */
static void pack_merge(uint64_t N, uint64_t basis_log2, uint64_t digits, const uint64_t* keys,
                       uint64_t L, uint64_t* left, uint64_t* right, uint64_t* rot) {
    const uint64_t shift = N >> L;
    for (int h = 0; h < 2; ++h) {
        const uint64_t* src = left + h * N;
        uint64_t* dst = rot + h * N;
        for (uint64_t j = 0; j < shift; ++j) dst[j] = tpo_sub(0, src[N - shift + j]);
        for (uint64_t j = 0; j < N - shift; ++j) dst[shift + j] = src[j];
    }
    for (uint64_t k = 0; k < 2 * N; ++k) {
        const uint64_t l = tpo_add(rot[k], right[k]);
        right[k] = tpo_sub(right[k], rot[k]);
        left[k] = l;
    }
    memset(rot, 0, 2 * N * 8);
    tpo_auto_eval(N, basis_log2, digits, (1ULL << L) + 1, keys + (L - 1) * 2 * N * digits, rot, right);
    tpo_ntt_backward(N, rot, rot);
    tpo_ntt_backward(N, rot + N, rot + N);
    for (uint64_t k = 0; k < 2 * N; ++k) left[k] = tpo_add(left[k], rot[k]);
}

static uint64_t rev_bits(uint64_t x, unsigned bits) {
    uint64_t r = 0;
    for (unsigned i = 0; i < bits; ++i) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

/* LWEtoRLWEPacker::Pack (lwe_to_rlwe_packing.cpp:129-236), restated level by level:
 * the reference's stack walks the same balanced binary tree, element c being
 * input[(len-1) ^ brv_{log len}(c)], left child = earlier element. */
int tpo_pack(uint64_t N, uint64_t basis_log2, uint64_t digits, const uint64_t* keys,
             uint64_t* out, const uint64_t* in, uint64_t len) {
    const uint64_t logn = int_log2(N);
    const uint64_t logl = int_log2(len);
    if (!get_tables(N) || len < 2 || (1ULL << logl) != len || len > N) return -1;
    uint64_t* nodes = (uint64_t*)malloc(len * 2 * N * 8);
    uint64_t* rot = (uint64_t*)malloc(2 * N * 8);
    for (uint64_t c = 0; c < len; ++c) {
        const uint64_t src = (len - 1) ^ rev_bits(c, (unsigned)logl);
        l0_setup(N, nodes + c * 2 * N, in + src * (N + 1));
    }
    for (uint64_t L = 1; L <= logl; ++L) {
        const uint64_t stride = 1ULL << L;
        for (uint64_t c = 0; c < len; c += stride)
            pack_merge(N, basis_log2, digits, keys, L, nodes + c * 2 * N, nodes + (c + stride / 2) * 2 * N, rot);
    }
    /* trailing traces when len < N (lwe_to_rlwe_packing.cpp:228-234) */
    for (uint64_t i = 0; i < logn - logl; ++i) {
        const uint64_t j = logn - i;
        memset(rot, 0, 2 * N * 8);
        tpo_auto_eval(N, basis_log2, digits, (1ULL << j) + 1, keys + (j - 1) * 2 * N * digits, rot, nodes);
        tpo_ntt_backward(N, rot, rot);
        tpo_ntt_backward(N, rot + N, rot + N);
        for (uint64_t k = 0; k < 2 * N; ++k) nodes[k] = tpo_add(nodes[k], rot[k]);
    }
    memcpy(out, nodes, 2 * N * 8);
    free(nodes);
    free(rot);
    return 0;
}

int tpo_pack_consecutive(uint64_t N, uint64_t basis_log2, uint64_t digits, const uint64_t* keys,
                         uint64_t* out, const uint64_t* in, uint64_t len) {
    const uint64_t logn = int_log2(N);
    if (!get_tables(N) || len < 2 || len > N) return -1;
    uint64_t* slots = (uint64_t*)calloc((logn + 2) * 2 * N, 8);
    uint64_t* rot = (uint64_t*)malloc(2 * N * 8);
    uint64_t level[72], fake[72];
    uint64_t head = 0, elem = 0;
    /* element e is real when its input index (N-1) ^ brv(e) is below len (line 276) */
#define CONSEC_PUSH(slot)                                                      \
    do {                                                                       \
        const uint64_t src = (N - 1) ^ rev_bits(elem, (unsigned)logn);          \
        uint64_t* dst = slots + (slot) * 2 * N;                                 \
        memset(dst, 0, 2 * N * 8);                                              \
        if (src < len) l0_setup(N, dst, in + src * (N + 1));                    \
        level[slot] = 0;                                                        \
        fake[slot] = src >= len;                                                \
        ++elem;                                                                 \
    } while (0)
    CONSEC_PUSH(0);
    head = 1;
    CONSEC_PUSH(1);
    while (level[0] != logn) {
        const uint64_t hl = head > 0 ? level[head] : UINT64_MAX;
        const uint64_t nl = head > 0 ? level[head - 1] : 0;
        if (hl == nl) {
            if (fake[head] && fake[head - 1]) { /* two empty subtrees: no work (lines 327-331) */
                --head;
                level[head] = hl + 1;
                fake[head] = 1;
                continue;
            }
            pack_merge(N, basis_log2, digits, keys, hl + 1, slots + (head - 1) * 2 * N, slots + head * 2 * N, rot);
            --head;
            level[head] = hl + 1;
            fake[head] = 0;
        } else {
            ++head;
            CONSEC_PUSH(head);
        }
    }
#undef CONSEC_PUSH
    memcpy(out, slots, 2 * N * 8);
    free(slots);
    free(rot);
    return 0;
}

void tpo_sample_extract(uint64_t* out_lwe, const uint64_t* rlwe, uint64_t index, uint64_t N) {
    for (uint64_t i = 0; i <= index; ++i) out_lwe[i] = rlwe[index - i];
    for (uint64_t i = index + 1; i < N; ++i) {
        const uint64_t v = rlwe[N - i];
        if (v != 0) out_lwe[i] = P - v;
    }
    out_lwe[N] = rlwe[N + index];
}

/* ------------------------------------------------------------------------- */
/* modulus switching                                                         */
/* ------------------------------------------------------------------------- */

/* ModulusSwitch (lib/src/static/modulus_switching.cpp:36-93) for the FLOOR,
 * CEIL and ROUND types, in x86 80-bit long double exactly as the reference
 * computes it: (target * (long double)v) / source, then floorl / ceill /
 * roundl, then one conditional subtraction of the target. type: 0 ROUND,
 * 1 FLOOR, 2 CEIL (lib/include/static/modulus_switching.h:24-29). */
int tpo_modulus_switch(uint64_t* vec, uint64_t n, uint64_t source, uint64_t target, int type) {
    const long double sM = (long double)source, tM = (long double)target;
    for (uint64_t i = 0; i < n; ++i) {
        const long double v = (tM * (long double)vec[i]) / sM;
        uint64_t r;
        if (type == 0) r = (uint64_t)roundl(v);
        else if (type == 1) r = (uint64_t)floorl(v);
        else if (type == 2) r = (uint64_t)ceill(v);
        else return -1;
        if (r >= target) r -= target;
        vec[i] = r;
    }
    return 0;
}

/* ---- LWE -> RGSW scheme switching ------------------------------------------ */

/* LWEtoRGSWConverter's constructor (lwe_to_rgsw_conversion.cpp:120-160): block
 * size N/D; the first block holds +-scale centred on X^0, block b >= 1 holds
 * scale * 2^(b*basebits) starting at X^(b*bs - bs/2); then times 2^-1, and the
 * copy at [N, 2N) negated. max_digits = ceil(log2(p)/basebits) = ceil(64/basebits)
 * (log2(p) is within 2^-31 of 64). */
int tpo_ss_test_poly(uint64_t N, uint64_t D, uint64_t basebits, uint64_t* acc) {
    if (D == 0 || basebits == 0 || N % D || ((N / D) & 1)) return -1;
    const uint64_t max_digits = (64 + basebits - 1) / basebits;
    if (max_digits < D || basebits * (max_digits - D) >= 31) return -1;
    const uint64_t bs = N / D;
    uint64_t scale = 1ULL << (basebits * (max_digits - D));
    memset(acc, 0, 3 * N * 8);
    for (uint64_t i = 0; i < bs / 2; ++i) {
        acc[N + i] = scale;
        acc[2 * N - i - 1] = P - scale;
    }
    for (uint64_t b = 1; b < D; ++b) {
        scale <<= basebits;
        for (uint64_t j = 0; j < bs; ++j) acc[N + b * bs + j - bs / 2] = scale;
    }
    const uint64_t half = tpo_inv(2);
    for (uint64_t i = 0; i < N; ++i) {
        acc[2 * N + i] = tpo_mul(acc[N + i], half);
        acc[N + i] = tpo_sub(0, acc[2 * N + i]);
    }
    return 0;
}

/* TraceEvaluator::Eval (trace_evaluation.cpp:138-156), in place on [A | B]
 * coefficients: x *= N^-1; for index N+1 down to 3: x += INTT(Auto_index(x));
 * then both halves to the NTT domain. */
static void trace_eval(uint64_t N, uint64_t bl, uint64_t dg, const uint64_t* keys, uint64_t* x, uint64_t* tmp) {
    const uint64_t ninv = tpo_inv(N);
    const uint64_t logn = int_log2(N);
    for (uint64_t i = 0; i < 2 * N; ++i) x[i] = tpo_mul(x[i], ninv);
    for (uint64_t j = logn; j >= 1; --j) {
        memset(tmp, 0, 2 * N * 8);
        tpo_auto_eval(N, bl, dg, (1ULL << j) + 1, keys + (j - 1) * 2 * N * dg, tmp, x);
        tpo_ntt_backward(N, tmp, tmp);
        tpo_ntt_backward(N, tmp + N, tmp + N);
        for (uint64_t i = 0; i < 2 * N; ++i) x[i] = tpo_add(x[i], tmp[i]);
    }
    tpo_ntt_forward(N, x, x);
    tpo_ntt_forward(N, x + N, x + N);
}

void tpo_trace_eval(uint64_t N, uint64_t bl, uint64_t dg, const uint64_t* keys, uint64_t* out, const uint64_t* in) {
    uint64_t* tmp = (uint64_t*)malloc(2 * N * 8);
    memmove(out, in, 2 * N * 8);
    trace_eval(N, bl, dg, keys, out, tmp);
    free(tmp);
}

int tpo_lwe_to_rgsw(int variant, uint64_t N, uint64_t n, uint64_t br_bl, uint64_t br_dg, const uint64_t* brk,
                    uint64_t tr_bl, uint64_t tr_dg, const uint64_t* trace_keys, uint64_t sq_bl, uint64_t sq_dg,
                    const uint64_t* sq_key, uint64_t D, uint64_t out_bl, const uint64_t* lwe, uint64_t* out) {
    uint64_t* acc = (uint64_t*)malloc(3 * N * 8);
    uint64_t* buf = (uint64_t*)malloc(4 * N * 8);
    int rc = tpo_ss_test_poly(N, D, out_bl, acc);
    uint64_t* left = out;
    uint64_t* right = out + 2 * N * D;
    const uint64_t bs = N / D;
    if (rc == 0) rc = tpo_blind_rotate(variant, N, n, br_bl, br_dg, brk, right, lwe, acc, 1);
    if (rc == 0) {
        /* B += tp (line 180); [A, -A, B, -B] and the row rotations (lines 188-200) */
        for (uint64_t i = 0; i < N; ++i) right[N + i] = tpo_add(right[N + i], acc[2 * N + i]);
        for (uint64_t i = 0; i < N; ++i) {
            buf[i] = right[i];
            buf[N + i] = tpo_sub(0, right[i]);
            buf[2 * N + i] = right[N + i];
            buf[3 * N + i] = tpo_sub(0, right[N + i]);
        }
        for (uint64_t d = 1; d < D; ++d) {
            memcpy(right + d * 2 * N, buf + d * bs, N * 8);
            memcpy(right + d * 2 * N + N, buf + 2 * N + d * bs, N * 8);
        }
        for (uint64_t d = 0; d < D; ++d) trace_eval(N, tr_bl, tr_dg, trace_keys, right + d * 2 * N, buf);
        /* RLWE(-s m) from RLWE(m) per row (lines 208-224) */
        for (uint64_t d = 0; d < D; ++d) {
            uint64_t* m = right + d * 2 * N;
            uint64_t* sm = left + d * 2 * N;
            memset(buf, 0, 2 * N * 8);
            tpo_ntt_backward(N, buf, m);
            memset(sm, 0, 2 * N * 8);
            tpo_rlwe_ks(N, sq_bl, sq_dg, sq_key, sm, buf);
            for (uint64_t i = 0; i < 2 * N; ++i) sm[i] = tpo_sub(0, sm[i]);
            for (uint64_t i = 0; i < N; ++i) sm[i] = tpo_add(sm[i], m[N + i]);
        }
    }
    free(acc);
    free(buf);
    return rc;
}

void tpo_ss_keygen(tpo_rng* r, int variant, uint64_t N, uint64_t n, uint64_t br_bl, uint64_t br_dg, uint64_t tr_bl,
                   uint64_t tr_dg, uint64_t sq_bl, uint64_t sq_dg, double std_dev, const uint64_t* lwe_key,
                   const uint64_t* rlwe_key, uint64_t* brk, uint64_t* trace_keys, uint64_t* sq_key) {
    tpo_br_keygen(r, variant, N, n, br_bl, br_dg, std_dev, lwe_key, rlwe_key, brk);
    tpo_pack_keygen(r, N, tr_bl, tr_dg, std_dev, rlwe_key, trace_keys);
    uint64_t* sq = (uint64_t*)malloc(N * 8);
    tpo_ntt_forward(N, sq, rlwe_key);
    for (uint64_t i = 0; i < N; ++i) sq[i] = tpo_mul(sq[i], sq[i]);
    tpo_ntt_backward(N, sq, sq);
    tpo_rlwe_ks_keygen(r, N, sq_bl, sq_dg, std_dev, sq, rlwe_key, sq_key);
    free(sq);
}

/* ---- SAP digit decomposition ------------------------------------------------ */

uint64_t tpo_ref_int_log2(uint64_t x) { return int_log2(x); }

static void ntt_pair(uint64_t N, uint64_t* x, int forward) {
    if (forward) {
        tpo_ntt_forward(N, x, x);
        tpo_ntt_forward(N, x + N, x + N);
    } else {
        tpo_ntt_backward(N, x, x);
        tpo_ntt_backward(N, x + N, x + N);
    }
}

static void mul_pair(uint64_t N, uint64_t* x, const uint64_t* poly) {
    for (uint64_t i = 0; i < N; ++i) {
        x[i] = tpo_mul(x[i], poly[i]);
        x[N + i] = tpo_mul(x[N + i], poly[i]);
    }
}

static uint64_t brev_bits(uint64_t x, uint64_t bits) {
    uint64_t r = 0;
    for (uint64_t b = 0; b < bits; ++b) r |= ((x >> b) & 1) << (bits - 1 - b);
    return r;
}

/* One node of the truncation tree (lines 243-289), depth first like the reference:
 * a leaf adds x * X^brev(e) to out; an inner node at level l splits x into
 * x + Auto(x) (exponent 2e) and (x - Auto(x)) * X^-(N >> l) (exponent 2e + 1),
 * Auto = Auto_{2^l + 1} of INTT(x), all in the NTT domain. */
static void trunc_node(uint64_t N, uint64_t bl, uint64_t dg, const uint64_t* keys, uint64_t L, uint64_t level,
                       uint64_t e, uint64_t* x, uint64_t* out) {
    uint64_t* poly = (uint64_t*)calloc(N, 8);
    if (level == 0) {
        poly[brev_bits(e, L)] = 1;
        tpo_ntt_forward(N, poly, poly);
        mul_pair(N, x, poly);
        for (uint64_t i = 0; i < 2 * N; ++i) out[i] = tpo_add(out[i], x[i]);
        free(poly);
        return;
    }
    poly[N - (N >> level)] = P - 1;
    tpo_ntt_forward(N, poly, poly);
    uint64_t* c = (uint64_t*)malloc(2 * N * 8);
    uint64_t* a = (uint64_t*)calloc(2 * N, 8);
    uint64_t* t = (uint64_t*)malloc(2 * N * 8);
    memcpy(c, x, 2 * N * 8);
    ntt_pair(N, c, 0);
    const uint64_t j = level;                       /* index 2^level + 1 is key j - 1 */
    tpo_auto_eval(N, bl, dg, (1ULL << j) + 1, keys + (j - 1) * 2 * N * dg, a, c);
    for (uint64_t i = 0; i < 2 * N; ++i) {
        t[i] = tpo_sub(x[i], a[i]);
        x[i] = tpo_add(x[i], a[i]);
    }
    mul_pair(N, t, poly);
    trunc_node(N, bl, dg, keys, L, level - 1, 2 * e + 1, t, out);
    trunc_node(N, bl, dg, keys, L, level - 1, 2 * e, x, out);
    free(c);
    free(a);
    free(t);
    free(poly);
}

int tpo_sap_homtrunc(uint64_t N, uint64_t bl, uint64_t dg, const uint64_t* keys, uint64_t radix, uint64_t* out,
                     const uint64_t* in) {
    if (radix < 1 || (radix & (radix - 1)) || radix > N || !get_tables(N)) return -1;
    const uint64_t logn = int_log2(N), logr = tpo_ref_int_log2(radix);
    uint64_t* pad = (uint64_t*)calloc(N, 8);
    uint64_t* x = (uint64_t*)malloc(2 * N * 8);
    uint64_t* c = (uint64_t*)malloc(2 * N * 8);
    uint64_t* a = (uint64_t*)malloc(2 * N * 8);
    /* sum_{i < radix} X^(i - (radix - 1)) (lines 212-217) */
    for (uint64_t i = N - (radix - 1); i < N; ++i) pad[i] = P - 1;
    pad[0] = 1;
    tpo_ntt_forward(N, pad, pad);
    const uint64_t ninv = tpo_inv(N);
    for (uint64_t i = 0; i < 2 * N; ++i) x[i] = tpo_mul(in[i], ninv);
    mul_pair(N, x, pad);
    /* partial trace (lines 229-238) */
    for (uint64_t i = 0; i < logr; ++i) {
        const uint64_t j = logn - i;
        memcpy(c, x, 2 * N * 8);
        ntt_pair(N, c, 0);
        memset(a, 0, 2 * N * 8);
        tpo_auto_eval(N, bl, dg, (1ULL << j) + 1, keys + (j - 1) * 2 * N * dg, a, c);
        for (uint64_t k = 0; k < 2 * N; ++k) x[k] = tpo_add(x[k], a[k]);
    }
    memset(out, 0, 2 * N * 8);
    trunc_node(N, bl, dg, keys, logn - logr, logn - logr, 0, x, out);
    free(pad);
    free(x);
    free(c);
    free(a);
    return 0;
}

int tpo_sap_reset(int variant, uint64_t N, uint64_t n, uint64_t br_bl, uint64_t br_dg, const uint64_t* brk,
                  uint64_t ks_bl, uint64_t ks_dg, const uint64_t* ksk, uint64_t radix, uint64_t* acc) {
    if (!get_tables(N)) return -1;
    const uint64_t r = tpo_ref_int_log2(radix);
    uint64_t* poly = (uint64_t*)calloc(N, 8);
    uint64_t* ext = (uint64_t*)calloc(N + 1, 8);
    uint64_t* lwe = (uint64_t*)calloc(n + 1, 8);
    uint64_t* fresh = (uint64_t*)calloc(2 * N, 8);
    /* overflow extraction polynomial (lines 320-324) */
    for (uint64_t i = 1; i < N; ++i) poly[i] = tpo_sub(0, ((N - i) >> r) << r);
    tpo_ntt_forward(N, poly, poly);
    mul_pair(N, acc, poly);
    ntt_pair(N, acc, 0);
    tpo_sample_extract(ext, acc, 0, N);
    tpo_lwe_ks(P, N, n, ks_bl, ks_dg, ksk, lwe, ext);
    tpo_modulus_switch(lwe, n + 1, P, 2 * N, 1);
    fresh[N] = P / (2 * N);
    const int rc = tpo_blind_rotate(variant, N, n, br_bl, br_dg, brk, acc, lwe, fresh, 0);
    free(poly);
    free(ext);
    free(lwe);
    free(fresh);
    return rc;
}

int tpo_sap_decompose(int variant, uint64_t N, uint64_t n, uint64_t br_bl, uint64_t br_dg, const uint64_t* brk,
                      uint64_t tr_bl, uint64_t tr_dg, const uint64_t* keys, uint64_t ks_bl, uint64_t ks_dg,
                      const uint64_t* ksk, uint64_t radix, uint64_t beta, uint64_t restart, const uint64_t* in,
                      uint64_t* out, uint64_t out_digits) {
    if (radix < 2 || (radix & (radix - 1)) || radix > N || !get_tables(N) || restart == 0) return -1;
    const uint64_t r = tpo_ref_int_log2(radix), mask = radix - 1, q_in = 2 * N;
    uint64_t* acc = (uint64_t*)calloc(2 * N, 8);
    uint64_t* ext = (uint64_t*)malloc(2 * N * 8);
    uint64_t* xp = (uint64_t*)calloc(N, 8);
    uint64_t* copy = (uint64_t*)malloc((n + 1) * 8);
    uint64_t* sub = (uint64_t*)malloc((n + 1) * 8);
    int rc = 0;
    /* acc = (0, Q/2N), B in the NTT domain (lines 389-392) */
    acc[N] = P / (2 * N);
    tpo_ntt_forward(N, acc + N, acc + N);
    /* x -> x mod radix, reversed (lines 394-399) */
    for (uint64_t i = 1; i < N; ++i) xp[N - i] = tpo_sub(0, i & mask);
    tpo_ntt_forward(N, xp, xp);
    memcpy(copy, in, (n + 1) * 8);
    /* input modulus from the words themselves (lines 409-416) */
    uint64_t M = 1ULL << tpo_ref_int_log2(in[0]);
    for (uint64_t i = 1; i <= n; ++i)
        if (M <= in[i]) M <<= 1;
    uint64_t d = 0;
    while (M > 1) {
        for (uint64_t i = 0; i <= n; ++i) {
            sub[i] = copy[i] & mask;
            copy[i] >>= r;
        }
        M >>= r;
        sub[n] = (uint64_t)(((unsigned __int128)sub[n] + radix * beta) % q_in);
        copy[n] = copy[n] >= beta ? copy[n] - beta : copy[n] + M - beta;
        ntt_pair(N, acc, 0);
        rc = tpo_blind_rotate(variant, N, n, br_bl, br_dg, brk, acc, sub, acc, 0);
        if (rc) break;
        for (uint64_t i = 0; i < N; ++i) {
            ext[i] = tpo_mul(acc[i], xp[i]);
            ext[N + i] = tpo_mul(acc[N + i], xp[i]);
        }
        ntt_pair(N, ext, 0);
        if (d >= out_digits) {
            rc = -1;
            break;
        }
        tpo_sample_extract(out + d * (N + 1), ext, 0, N);
        if ((d + 1) % restart == 0 && M != 0) {
            rc = tpo_sap_reset(variant, N, n, br_bl, br_dg, brk, ks_bl, ks_dg, ksk, 0, acc);
            if (rc) break;
        }
        rc = tpo_sap_homtrunc(N, tr_bl, tr_dg, keys, radix, ext, acc);
        if (rc) break;
        memcpy(acc, ext, 2 * N * 8);
        ++d;
    }
    free(acc);
    free(ext);
    free(xp);
    free(copy);
    free(sub);
    return rc ? -1 : (int)d;
}

void tpo_sap_keygen(tpo_rng* r, int variant, uint64_t N, uint64_t n, uint64_t br_bl, uint64_t br_dg, uint64_t tr_bl,
                    uint64_t tr_dg, uint64_t ks_bl, uint64_t ks_dg, double std_dev, const uint64_t* lwe_key,
                    const uint64_t* rlwe_key, uint64_t* brk, uint64_t* trace_keys, uint64_t* lwe_ksk) {
    tpo_br_keygen(r, variant, N, n, br_bl, br_dg, std_dev, lwe_key, rlwe_key, brk);
    tpo_pack_keygen(r, N, tr_bl, tr_dg, std_dev, rlwe_key, trace_keys);
    tpo_lwe_ks_keygen(r, P, N, n, ks_bl, ks_dg, std_dev, rlwe_key, lwe_key, lwe_ksk);
}
