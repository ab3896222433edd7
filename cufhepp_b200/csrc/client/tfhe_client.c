/*
 * Client side of the gate API: seeded key generation, encryption and
 * decryption in the TFHEpp layouts the gate engine consumes.
 *
 * In the reference these come from TFHEpp (SecretKey, EvalKey::emplacebk /
 * emplaceiksk, tlweSymEncrypt / tlweSymDecrypt; used by
 * test/test_gate_gpu.cc:50-58 and test/test_util.h:20-27).  TFHEpp is an empty
 * submodule in the reference tree, so this file restates the published TFHE
 * key-generation and encryption procedures for the parameter sets of
 * params.h.  All randomness is derived from a 64-bit seed and a per-object
 * stream index, so key material is reproducible and independent of the
 * number of OpenMP threads.
 *
 * Torus elements are uint32_t (Torus32) or uint64_t (Torus64).  A binary key
 * is an int32_t array of 0/1.  Encrypting bit b uses message b ? +mu : -mu
 * (test/test_util.h:23-27).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../params.h"

/* ---------------------------------------------------------------- RNG ---- */
/* xoshiro256** (Blackman & Vigna, public domain algorithm), seeded through
 * splitmix64 from (seed, stream). */
typedef struct {
    uint64_t s[4];
} crng_t;

static uint64_t splitmix64(uint64_t* x)
{
    uint64_t z = (*x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

static inline uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

static void crng_seed(crng_t* r, uint64_t seed, uint64_t stream)
{
    uint64_t x = seed ^ (0xd1b54a32d192ed03ull * (stream + 1));
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}

static inline uint64_t crng_u64(crng_t* r)
{
    uint64_t* s = r->s;
    const uint64_t res = rotl64(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl64(s[3], 45);
    return res;
}

static inline uint32_t crng_u32(crng_t* r) { return (uint32_t)(crng_u64(r) >> 32); }

/* uniform double in (0, 1] with 53 random bits */
static inline double crng_unit(crng_t* r)
{
    return ((double)(crng_u64(r) >> 11) + 1.0) * (1.0 / 9007199254740992.0);
}

/* Box-Muller: one standard normal sample */
static inline double crng_normal(crng_t* r)
{
    const double u1 = crng_unit(r);
    const double u2 = crng_unit(r);
    return sqrt(-2.0 * log(u1)) * cos(6.283185307179586476925286766559 * u2);
}

/* Gaussian torus noise with standard deviation alpha (in torus units) */
static inline uint32_t noise32(crng_t* r, double alpha)
{
    double e = crng_normal(r) * alpha;
    e -= nearbyint(e);
    return (uint32_t)(int64_t)llrint(e * 4294967296.0);
}

static inline uint64_t noise64(crng_t* r, double alpha)
{
    double e = crng_normal(r) * alpha;
    e -= nearbyint(e);
    /* |e| <= 1/2, so e * 2^63 fits in int64 after halving the scale */
    return (uint64_t)(int64_t)llrint(e * 9223372036854775808.0) << 1;
}

/* ------------------------------------------------------------ keys ------ */
void tfhe_keygen_binary(uint64_t seed, uint64_t stream, uint32_t n, int32_t* key)
{
    crng_t r;
    crng_seed(&r, seed, stream);
    for (uint32_t i = 0; i < n; i++) key[i] = (int32_t)(crng_u64(&r) >> 63);
}

/* ------------------------------------------------------------- TLWE ------ */
static void tlwe32_encrypt_rng(crng_t* r, const int32_t* key, uint32_t n,
                               uint32_t msg, double alpha, uint32_t* out)
{
    uint32_t b = msg + noise32(r, alpha);
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t a = crng_u32(r);
        out[i] = a;
        b += a * (uint32_t)key[i];
    }
    out[n] = b;
}

void tfhe_tlwe32_encrypt(uint64_t seed, uint64_t stream, const int32_t* key,
                         uint32_t n, uint32_t msg, double alpha, uint32_t* out)
{
    crng_t r;
    crng_seed(&r, seed, stream);
    tlwe32_encrypt_rng(&r, key, n, msg, alpha, out);
}

/* Encrypt count bits; ciphertext i uses stream (stream0 + i). */
void tfhe_tlwe32_encrypt_bits(uint64_t seed, uint64_t stream0, const int32_t* key,
                              uint32_t n, const uint8_t* bits, uint64_t count,
                              uint32_t mu, double alpha, uint32_t* out)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; i++) {
        crng_t r;
        crng_seed(&r, seed, stream0 + (uint64_t)i);
        const uint32_t msg = bits[i] ? mu : (uint32_t)(0u - mu);
        tlwe32_encrypt_rng(&r, key, n, msg, alpha, out + (uint64_t)i * (n + 1));
    }
}

uint32_t tfhe_tlwe32_phase(const int32_t* key, uint32_t n, const uint32_t* c)
{
    uint32_t p = c[n];
    for (uint32_t i = 0; i < n; i++) p -= c[i] * (uint32_t)key[i];
    return p;
}

void tfhe_tlwe32_phase_batch(const int32_t* key, uint32_t n, const uint32_t* c,
                             uint64_t count, uint32_t* phase)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; i++)
        phase[i] = tfhe_tlwe32_phase(key, n, c + (uint64_t)i * (n + 1));
}

/* decrypted bit = (signed phase > 0), as TFHEpp::tlweSymDecrypt */
void tfhe_tlwe32_decrypt_bits(const int32_t* key, uint32_t n, const uint32_t* c,
                              uint64_t count, uint8_t* bits)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)count; i++)
        bits[i] = (int32_t)tfhe_tlwe32_phase(key, n, c + (uint64_t)i * (n + 1)) > 0;
}

/* ------------------------------------------------------------ TRLWE ------ */
/* out[n] += (a * s)[n] mod X^N+1 for a binary key s (exact, mod 2^32) */
static void negacyclic_addmul_binary32(uint32_t* out, const uint32_t* a,
                                       const int32_t* s, uint32_t N)
{
    for (uint32_t m = 0; m < N; m++) {
        if (!s[m]) continue;
        /* X^m * a: coefficient n gets a[n-m] for n>=m, -a[n-m+N] for n<m */
        for (uint32_t n = 0; n < m; n++) out[n] -= a[n + N - m];
        for (uint32_t n = m; n < N; n++) out[n] += a[n - m];
    }
}

static void negacyclic_addmul_binary64(uint64_t* out, const uint64_t* a,
                                       const int32_t* s, uint32_t N)
{
    for (uint32_t m = 0; m < N; m++) {
        if (!s[m]) continue;
        for (uint32_t n = 0; n < m; n++) out[n] -= a[n + N - m];
        for (uint32_t n = m; n < N; n++) out[n] += a[n - m];
    }
}

/* TRLWE (k = 1) of message polynomial msg (may be NULL = 0): out[2][N] */
static void trlwe32_encrypt_rng(crng_t* r, const int32_t* key, uint32_t N,
                                const uint32_t* msg, double alpha, uint32_t* out)
{
    uint32_t* a = out;
    uint32_t* b = out + N;
    for (uint32_t i = 0; i < N; i++) a[i] = crng_u32(r);
    for (uint32_t i = 0; i < N; i++) b[i] = (msg ? msg[i] : 0u) + noise32(r, alpha);
    negacyclic_addmul_binary32(b, a, key, N);
}

static void trlwe64_encrypt_rng(crng_t* r, const int32_t* key, uint32_t N,
                                double alpha, uint64_t* out)
{
    uint64_t* a = out;
    uint64_t* b = out + N;
    for (uint32_t i = 0; i < N; i++) a[i] = crng_u64(r);
    for (uint32_t i = 0; i < N; i++) b[i] = noise64(r, alpha);
    negacyclic_addmul_binary64(b, a, key, N);
}

void tfhe_trlwe32_encrypt(uint64_t seed, uint64_t stream, const int32_t* key,
                          uint32_t N, const uint32_t* msg, double alpha,
                          uint32_t* out)
{
    crng_t r;
    crng_seed(&r, seed, stream);
    trlwe32_encrypt_rng(&r, key, N, msg, alpha, out);
}

/* phase polynomial b - a*s of a k = 1 TRLWE */
void tfhe_trlwe32_phase(const int32_t* key, uint32_t N, const uint32_t* c,
                        uint32_t* phase)
{
    uint32_t* neg_a = (uint32_t*)malloc(sizeof(uint32_t) * N);
    for (uint32_t i = 0; i < N; i++) {
        neg_a[i] = 0u - c[i];
        phase[i] = c[N + i];
    }
    negacyclic_addmul_binary32(phase, neg_a, key, N);
    free(neg_a);
}

/* ------------------------------------------------------------ TRGSW ------ */
/* TRGSW(m) under a k = 1 key: rows r = j*l + d are TRLWE encryptions of 0
 * with m * 2^(w - (d+1) Bgbit) added to coefficient 0 of polynomial j. */
static void trgsw32_encrypt_rng(crng_t* r, const int32_t* key, uint32_t N,
                                uint32_t l, uint32_t bgbit, int32_t m,
                                double alpha, uint32_t* out)
{
    for (uint32_t j = 0; j < 2; j++)
        for (uint32_t d = 0; d < l; d++) {
            uint32_t* row = out + (uint64_t)(j * l + d) * 2 * N;
            trlwe32_encrypt_rng(r, key, N, NULL, alpha, row);
            row[j * N] += (uint32_t)m * (1u << (32 - (d + 1) * bgbit));
        }
}

static void trgsw64_encrypt_rng(crng_t* r, const int32_t* key, uint32_t N,
                                uint32_t l, uint32_t bgbit, int32_t m,
                                double alpha, uint64_t* out)
{
    for (uint32_t j = 0; j < 2; j++)
        for (uint32_t d = 0; d < l; d++) {
            uint64_t* row = out + (uint64_t)(j * l + d) * 2 * N;
            trlwe64_encrypt_rng(r, key, N, alpha, row);
            row[j * N] += (uint64_t)(int64_t)m * (1ull << (64 - (d + 1) * bgbit));
        }
}

void tfhe_trgsw32_encrypt(uint64_t seed, uint64_t stream, const int32_t* key,
                          uint32_t N, uint32_t l, uint32_t bgbit, int32_t m,
                          double alpha, uint32_t* out)
{
    crng_t r;
    crng_seed(&r, seed, stream);
    trgsw32_encrypt_rng(&r, key, N, l, bgbit, m, alpha, out);
}

/* ------------------------------------------------- bootstrapping key ------ */
/* lvl01 bootstrapping key.  kb = 0: TRGSW[n0] encrypting key0[i].
 * kb = 1 (KeyBundle, 2 addends): TRGSW[n0/2][3] encrypting, for the pair
 * (s0, s1) = (key0[2p], key0[2p+1]): s0*s1, s0*(1-s1), (1-s0)*s1
 * (consumed in that order by include/gatebootstrapping_gpu.cuh:966-994). */
void tfhe_bk32_gen(uint64_t seed, const int32_t* key0, uint32_t n0,
                   const int32_t* key1, uint32_t N, uint32_t l, uint32_t bgbit,
                   double alpha, int kb, uint32_t* out)
{
    const uint64_t trgsw_words = (uint64_t)2 * l * 2 * N;
    const int64_t count = kb ? (int64_t)(n0 / 2) * 3 : (int64_t)n0;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t e = 0; e < count; e++) {
        int32_t m;
        if (!kb)
            m = key0[e];
        else {
            const int64_t p = e / 3, which = e % 3;
            const int32_t s0 = key0[2 * p], s1 = key0[2 * p + 1];
            m = which == 0 ? s0 * s1 : which == 1 ? s0 * (1 - s1) : (1 - s0) * s1;
        }
        crng_t r;
        crng_seed(&r, seed, 0x100000000ull + (uint64_t)e);
        trgsw32_encrypt_rng(&r, key1, N, l, bgbit, m, alpha, out + (uint64_t)e * trgsw_words);
    }
}

void tfhe_bk64_gen(uint64_t seed, const int32_t* key0, uint32_t n0,
                   const int32_t* key2, uint32_t N, uint32_t l, uint32_t bgbit,
                   double alpha, int kb, uint64_t* out)
{
    const uint64_t trgsw_words = (uint64_t)2 * l * 2 * N;
    const int64_t count = kb ? (int64_t)(n0 / 2) * 3 : (int64_t)n0;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t e = 0; e < count; e++) {
        int32_t m;
        if (!kb)
            m = key0[e];
        else {
            const int64_t p = e / 3, which = e % 3;
            const int32_t s0 = key0[2 * p], s1 = key0[2 * p + 1];
            m = which == 0 ? s0 * s1 : which == 1 ? s0 * (1 - s1) : (1 - s0) * s1;
        }
        crng_t r;
        crng_seed(&r, seed, 0x200000000ull + (uint64_t)e);
        trgsw64_encrypt_rng(&r, key2, N, l, bgbit, m, alpha, out + (uint64_t)e * trgsw_words);
    }
}

/* ------------------------------------------------- key switching key ------ */
/* ksk[i][j][k] = TLWE<target>( (k+1) * key_src[i] / 2^((j+1) basebit) ) for
 * i < n_src, j < t, k < 2^(basebit-1); target is Torus32 (lvl0). */
void tfhe_ksk32_gen(uint64_t seed, const int32_t* key_src, uint32_t n_src,
                    const int32_t* key0, uint32_t n0, uint32_t basebit,
                    uint32_t t, double alpha, uint32_t* out)
{
    const uint32_t nb = 1u << (basebit - 1);
    const uint64_t row = n0 + 1;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n_src; i++) {
        crng_t r;
        crng_seed(&r, seed, 0x300000000ull + (uint64_t)i);
        for (uint32_t j = 0; j < t; j++)
            for (uint32_t k = 0; k < nb; k++) {
                const uint32_t msg =
                    (uint32_t)((k + 1) * (uint32_t)key_src[i]) << (32 - (j + 1) * basebit);
                tlwe32_encrypt_rng(&r, key0, n0, msg, alpha,
                                   out + (((uint64_t)i * t + j) * nb + k) * row);
            }
    }
}

/* ------------------------------------------------------------ Torus64 --- */
/* phase polynomial b - a*s of a k = 1 Torus64 TRLWE */
void tfhe_trlwe64_phase(const int32_t* key, uint32_t N, const uint64_t* c, uint64_t* phase)
{
    uint64_t* neg_a = (uint64_t*)malloc(sizeof(uint64_t) * N);
    for (uint32_t i = 0; i < N; i++) {
        neg_a[i] = 0ull - c[i];
        phase[i] = c[N + i];
    }
    negacyclic_addmul_binary64(phase, neg_a, key, N);
    free(neg_a);
}

uint64_t tfhe_tlwe64_phase(const int32_t* key, uint32_t n, const uint64_t* c)
{
    uint64_t p = c[n];
    for (uint32_t i = 0; i < n; i++) p -= c[i] * (uint64_t)(uint32_t)key[i];
    return p;
}

/* ------------------------------------------ private key switching key ---- */
/* Key of the private functional key switching TLWE<src> (Torus64, n_src
 * mask coefficients) -> TRLWE<lvl1> that circuit bootstrapping uses
 * (CGGI17, the privKS lvl2 -> lvl1 of the circuit-bootstrapping workload):
 *   out[i][j][u] = TRLWE_s1( f(c) ),  i in [0, n_src], j < t, u < 2^basebit - 1,
 *   c = k_i * v_{j,u},  k_i = key_src[i] (i < n_src), k_{n_src} = -1,
 *   v_{j,u} = (u + 1) 2^(64 - (j+1) basebit) rounded to Torus32,
 *   f(x) = -x * s1(X) for func 0 (the rows that carry the message in the
 *   mask polynomial) and f(x) = x for func 1 (rows carrying it in b).
 * Layout [n_src + 1][t][2^basebit - 1][2][N] uint32; row (i, j, u) uses RNG
 * stream 0x400000000 + ((func (n_src+1) + i) t + j) (2^basebit - 1) + u. */
void tfhe_privks_gen(uint64_t seed, const int32_t* key_src, uint32_t n_src, const int32_t* key1,
                     uint32_t N, uint32_t basebit, uint32_t t, double alpha, int func,
                     uint32_t* out)
{
    const uint32_t nu = (1u << basebit) - 1;
    const int64_t rows = (int64_t)(n_src + 1) * t * nu;
#pragma omp parallel
    {
        uint32_t* msg = (uint32_t*)malloc(sizeof(uint32_t) * N);
#pragma omp for schedule(static)
        for (int64_t q = 0; q < rows; q++) {
            const uint32_t u = (uint32_t)(q % nu);
            const uint32_t j = (uint32_t)((q / nu) % t);
            const uint32_t i = (uint32_t)(q / ((int64_t)nu * t));
            const int shift = 64 - (int)((j + 1) * basebit);
            const uint64_t v64 = (uint64_t)(u + 1) << shift;
            const uint32_t v = (uint32_t)((v64 + (1ull << 31)) >> 32);
            const uint32_t k = i < n_src ? (uint32_t)key_src[i] : 0xFFFFFFFFu;
            const uint32_t c = k * v;
            for (uint32_t m = 0; m < N; m++)
                msg[m] = func == 0 ? (uint32_t)(0u - c * (uint32_t)key1[m]) : (m == 0 ? c : 0u);
            crng_t r;
            crng_seed(&r, seed, 0x400000000ull + ((uint64_t)func * (n_src + 1) + i) * t * nu +
                                   (uint64_t)j * nu + u);
            trlwe32_encrypt_rng(&r, key1, N, msg, alpha, out + (uint64_t)q * 2 * N);
        }
        free(msg);
    }
}
