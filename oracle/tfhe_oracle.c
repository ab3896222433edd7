/*
 * ORACLE -- test infrastructure only.
 *
 * A CPU restatement of cuFHEpp's lvl1 TFHE gate-bootstrapping path, used as
 * the checker of the CUDA engine by tests/, by __graft_entry__.smoke() and as
 * the timed CPU baseline of bench.py.  The product path never links or calls
 * this code.
 *
 * The reference cannot be compiled here: every source includes TFHEpp
 * headers and thirdparties/TFHEpp is an empty, unpinned submodule
 * (.gitmodules:1-3).  Parity against TFHEpp itself is therefore unpinned; this
 * restatement follows the cuFHEpp device code cited on each function and is
 * pinned on the reference's own known-answer tests
 * (test/test_accumulate_diag.cu, test/test_fft_roundtrip.cu), which
 * tests/test_oracle_kat.py re-runs against it.
 *
 * Two arithmetic forms of the external product are provided:
 *   ORC_EXACT : schoolbook negacyclic products in Z_{2^32}[X]/(X^N+1) --
 *               the exact result every bit-exact claim is measured against;
 *   ORC_FP64  : the reference's FP64 negacyclic FFNT (fold, twist, N/2-point
 *               complex FFT, multiply-accumulate, inverse, untwist, llrint),
 *               with the tables of src/ntt_small_modulus.cu:207-244.
 *
 * Parameters (lvl1 path; TFHEpp lvl0param/lvl1param/lvl10param):
 *   n0 = 636, N = 1024, k = 1, l = 2, Bgbit = 8, IKS basebit = 2, t = 7,
 *   Torus32, mu = 2^29.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define O_N0 636
#define O_N 1024
#define O_NBIT 10
#define O_HALF 512
#define O_L 2
#define O_BGBIT 8
#define O_BG 256
#define O_ROWS 4             /* (k+1) * l */
#define O_TRLWE (2 * O_N)    /* words */
#define O_TRGSW (O_ROWS * O_TRLWE)
#define O_T 7
#define O_BASEBIT 2
#define O_TLWE0 (O_N0 + 1)
#define O_TLWE1 (O_N + 1)
#define O_MU (1u << 29)

enum { ORC_EXACT = 0, ORC_FP64 = 1 };

/* ------------------------------------------------ polynomial helpers ---- */

/* out = X^a * p mod X^N+1 for a in [0, 2N)
 * (index rotation with sign flip: include/gatebootstrapping_gpu.cuh:114-121) */
static void rotate_poly(uint32_t* out, const uint32_t* p, uint32_t a)
{
    const uint32_t am = a & (O_N - 1), neg = a >> O_NBIT;
    for (uint32_t n = 0; n < O_N; n++) {
        const uint32_t v = p[(n - a) & (O_N - 1)];
        out[n] = ((n < am) ^ neg) ? 0u - v : v;
    }
}

/* Gadget decomposition of one Torus32 polynomial into l signed digits in
 * [-Bg/2, Bg/2), digit 0 most significant.
 * include/gatebootstrapping_gpu.cuh:20-29 (offsetgen), :122-128 and
 * :931-948 (digit extraction). */
void orc_decompose(const uint32_t* poly, int32_t* digits /* [l][N] */)
{
    uint32_t off = 0;
    for (int i = 1; i <= O_L; i++) off += (uint32_t)(O_BG / 2) << (32 - i * O_BGBIT);
    const uint32_t round = 1u << (32 - O_L * O_BGBIT - 1);
    for (int n = 0; n < O_N; n++) {
        const uint32_t t = poly[n] + off + round;
        for (int d = 0; d < O_L; d++)
            digits[d * O_N + n] =
                (int32_t)((t >> (32 - (d + 1) * O_BGBIT)) & (O_BG - 1)) - O_BG / 2;
    }
}

/* out += d * key mod (X^N+1, 2^32): exact schoolbook negacyclic product of a
 * signed digit polynomial and a Torus32 polynomial. */
static void negacyclic_mac_exact(uint32_t* restrict out, const int32_t* restrict d,
                                 const uint32_t* restrict key)
{
    for (int m = 0; m < O_N; m++) {
        const uint32_t dm = (uint32_t)d[m];
        if (!dm) continue;
        const uint32_t* kw = key + O_N - m;
        for (int n = 0; n < m; n++) out[n] -= dm * kw[n];
        const uint32_t* kp = key - m;
        for (int n = m; n < O_N; n++) out[n] += dm * kp[n];
    }
}

/* Exact external product: out = sum_r dec_r(in) * C[r] with the digit rows
 * r = j*l + d taken from polynomial j of the TRLWE `in`
 * (include/gatebootstrapping_gpu.cuh:159-179, coefficient domain). */
void orc_extprod_exact(const uint32_t* trgsw, const uint32_t* in, uint32_t* out)
{
    int32_t dig[O_L * O_N];
    memset(out, 0, sizeof(uint32_t) * O_TRLWE);
    for (int j = 0; j < 2; j++) {
        orc_decompose(in + j * O_N, dig);
        for (int d = 0; d < O_L; d++) {
            const int r = j * O_L + d;
            for (int oj = 0; oj < 2; oj++)
                negacyclic_mac_exact(out + oj * O_N, dig + d * O_N,
                                     trgsw + (r * 2 + oj) * O_N);
        }
    }
}

/* ---------------------------------------------------------- FP64 FFNT ---- */
/* Tables of src/ntt_small_modulus.cu:207-244: twist[i] = e^{2 pi i i/2N},
 * untwist[i] = conj(twist[i]) / (N/2); the N/2-point transform uses roots
 * e^{+2 pi i k/(N/2)} forward and their conjugates inverse.  The transform
 * below is a plain iterative radix-2 FFT with natural-order output; the
 * reference's stage order (include/ntt_small_modulus.cuh:977-1182) differs
 * only in FP64 rounding. */
typedef struct {
    double complex twist[O_HALF];
    double complex untwist[O_HALF];
    double complex root[O_HALF];  /* e^{2 pi i k / 512} */
    uint16_t bitrev[O_HALF];
    double complex* xai;          /* [2N][N/2] = FFNT(X^a - 1) */
} orc_fft_t;

static void fft512(const orc_fft_t* c, double complex* x, int inverse)
{
    for (int i = 0; i < O_HALF; i++) {
        const int j = c->bitrev[i];
        if (i < j) {
            double complex t = x[i];
            x[i] = x[j];
            x[j] = t;
        }
    }
    for (int len = 2; len <= O_HALF; len <<= 1) {
        const int half = len >> 1, step = O_HALF / len;
        for (int s = 0; s < O_HALF; s += len)
            for (int k = 0; k < half; k++) {
                double complex w = c->root[k * step];
                if (inverse) w = conj(w);
                const double complex u = x[s + k], v = x[s + k + half] * w;
                x[s + k] = u + v;
                x[s + k + half] = u - v;
            }
    }
}

/* fold + twist + forward FFNT of a real polynomial given as doubles */
static void ffnt_forward(const orc_fft_t* c, const double* re, double complex* out)
{
    for (int i = 0; i < O_HALF; i++)
        out[i] = (re[i] + I * re[i + O_HALF]) * c->twist[i];
    fft512(c, out, 0);
}

orc_fft_t* orc_fft_create(void)
{
    orc_fft_t* c = (orc_fft_t*)calloc(1, sizeof(orc_fft_t));
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < O_HALF; i++) {
        const long double tw = pi * i / O_N; /* 2 pi i / 2N */
        c->twist[i] = (double)cosl(tw) + I * (double)sinl(tw);
        c->untwist[i] = ((double)cosl(tw) - I * (double)sinl(tw)) / O_HALF;
        const long double ro = 2 * pi * i / O_HALF;
        c->root[i] = (double)cosl(ro) + I * (double)sinl(ro);
        int r = 0;
        for (int b = 0; b < 9; b++) r |= ((i >> b) & 1) << (8 - b);
        c->bitrev[i] = (uint16_t)r;
    }
    /* xai[a] = FFNT(X^a - 1), a in [0, 2N)   (src/ntt_small_modulus.cu:560-607) */
    c->xai = (double complex*)malloc(sizeof(double complex) * 2 * O_N * O_HALF);
    double poly[O_N];
    for (int a = 0; a < 2 * O_N; a++) {
        memset(poly, 0, sizeof(poly));
        poly[0] = -1.0;
        poly[a & (O_N - 1)] += (a >= O_N) ? -1.0 : 1.0;
        ffnt_forward(c, poly, c->xai + (size_t)a * O_HALF);
    }
    return c;
}

void orc_fft_destroy(orc_fft_t* c)
{
    if (!c) return;
    free(c->xai);
    free(c);
}

/* Bootstrapping key to the Fourier domain: each polynomial read as signed
 * int32, scaled by 2^-32, folded, twisted, transformed
 * (src/bootstrap_gpu.cu:59-112).  ntrgsw TRGSWs of [4][2][N] words ->
 * [ntrgsw][4][2][N/2] complex. */
void orc_bk_to_fft(const orc_fft_t* c, const uint32_t* bk, int ntrgsw, double complex* out)
{
#pragma omp parallel for schedule(static)
    for (int p = 0; p < ntrgsw * O_ROWS * 2; p++) {
        double re[O_N];
        for (int i = 0; i < O_N; i++)
            re[i] = (double)(int32_t)bk[(size_t)p * O_N + i] * (1.0 / 4294967296.0);
        ffnt_forward(c, re, out + (size_t)p * O_HALF);
    }
}

/* inverse FFNT + untwist + llrint(x 2^32) -> Torus32
 * (include/gatebootstrapping_gpu.cuh:183-220) */
static void ffnt_inverse_round(const orc_fft_t* c, double complex* acc, uint32_t* out, int add)
{
    fft512(c, acc, 1);
    for (int i = 0; i < O_HALF; i++) {
        const double complex v = acc[i] * c->untwist[i];
        const uint32_t lo = (uint32_t)(int32_t)llrint(creal(v) * 4294967296.0);
        const uint32_t hi = (uint32_t)(int32_t)llrint(cimag(v) * 4294967296.0);
        if (add) {
            out[i] += lo;
            out[i + O_HALF] += hi;
        } else {
            out[i] = lo;
            out[i + O_HALF] = hi;
        }
    }
}

/* digits of row r of `in` -> Fourier domain */
static void digits_fft(const orc_fft_t* c, const uint32_t* in, double complex spec[O_ROWS][O_HALF])
{
    int32_t dig[O_L * O_N];
    double re[O_N];
    for (int j = 0; j < 2; j++) {
        orc_decompose(in + j * O_N, dig);
        for (int d = 0; d < O_L; d++) {
            for (int i = 0; i < O_N; i++) re[i] = (double)dig[d * O_N + i];
            ffnt_forward(c, re, spec[j * O_L + d]);
        }
    }
}

/* FP64 external product with a Fourier-domain TRGSW:
 * out (=|+=) round(IFFNT(sum_r FFNT(dec_r) * C_r)) */
void orc_extprod_fp64(const orc_fft_t* c, const double complex* trgsw_f,
                      const uint32_t* in, uint32_t* out, int add)
{
    double complex spec[O_ROWS][O_HALF], acc[2][O_HALF];
    digits_fft(c, in, spec);
    memset(acc, 0, sizeof(acc));
    for (int r = 0; r < O_ROWS; r++)
        for (int oj = 0; oj < 2; oj++)
            for (int f = 0; f < O_HALF; f++)
                acc[oj][f] += spec[r][f] * trgsw_f[(r * 2 + oj) * O_HALF + f];
    for (int oj = 0; oj < 2; oj++) ffnt_inverse_round(c, acc[oj], out + oj * O_N, add);
}

/* ------------------------------------------------------ blind rotation ---- */

/* acc.a = 0, acc.b = X^bar * vec(mu), with the bar == 2N special case
 * (include/gatebootstrapping_gpu.cuh:31-53) */
void orc_test_vector(uint32_t bar, uint32_t mu, uint32_t* acc)
{
    for (uint32_t i = 0; i < O_N; i++) {
        acc[i] = 0;
        if (bar == 2 * O_N)
            acc[O_N + i] = mu;
        else
            acc[O_N + i] = ((i < (bar & (O_N - 1))) ^ (bar >> O_NBIT)) ? 0u - mu : mu;
    }
}

/* one non-KB CMUX step: acc += ExtProd(BK_i, X^abar acc - acc)
 * (include/gatebootstrapping_gpu.cuh:69-221) */
void orc_cmux_step_exact(uint32_t* acc, const uint32_t* bk_i, uint32_t abar)
{
    uint32_t diff[O_TRLWE], prod[O_TRLWE];
    for (int j = 0; j < 2; j++) {
        rotate_poly(diff + j * O_N, acc + j * O_N, abar);
        for (int n = 0; n < O_N; n++) diff[j * O_N + n] -= acc[j * O_N + n];
    }
    orc_extprod_exact(bk_i, diff, prod);
    for (int i = 0; i < O_TRLWE; i++) acc[i] += prod[i];
}

void orc_cmux_step_fp64(const orc_fft_t* c, uint32_t* acc, const double complex* bkf_i,
                        uint32_t abar)
{
    uint32_t diff[O_TRLWE];
    for (int j = 0; j < 2; j++) {
        rotate_poly(diff + j * O_N, acc + j * O_N, abar);
        for (int n = 0; n < O_N; n++) diff[j * O_N + n] -= acc[j * O_N + n];
    }
    orc_extprod_fp64(c, bkf_i, diff, acc, 1);
}

/* KeyBundle (2 addends) step: acc = ExtProd(KB, acc) with
 *   KB = H + bk0 (X^{a0+a1} - 1) + bk1 (X^{a0} - 1) + bk2 (X^{a1} - 1)
 * (include/gatebootstrapping_gpu.cuh:895-1033, combine at :966-994; gadget
 * H from src/ntt_small_modulus.cu:679-700).  Exact: KB is formed in the
 * coefficient domain mod 2^32, then one exact external product. */
void orc_kb_step_exact(uint32_t* acc, const uint32_t* bk3, uint32_t a0, uint32_t a1)
{
    uint32_t* kb = (uint32_t*)malloc(sizeof(uint32_t) * O_TRGSW);
    uint32_t rot[O_N];
    const uint32_t a01 = (a0 + a1) & (2 * O_N - 1);
    const uint32_t av[3] = {a01, a0, a1};
    memset(kb, 0, sizeof(uint32_t) * O_TRGSW);
    for (int r = 0; r < O_ROWS; r++) {
        const int j = r / O_L, d = r % O_L;
        kb[(r * 2 + j) * O_N] += 1u << (32 - (d + 1) * O_BGBIT);
        for (int e = 0; e < 3; e++)
            for (int oj = 0; oj < 2; oj++) {
                const uint32_t* p = bk3 + (size_t)e * O_TRGSW + (r * 2 + oj) * O_N;
                uint32_t* q = kb + (r * 2 + oj) * O_N;
                rotate_poly(rot, p, av[e]);
                for (int n = 0; n < O_N; n++) q[n] += rot[n] - p[n];
            }
    }
    uint32_t out[O_TRLWE];
    orc_extprod_exact(kb, acc, out);
    memcpy(acc, out, sizeof(out));
    free(kb);
}

void orc_kb_step_fp64(const orc_fft_t* c, uint32_t* acc, const double complex* bkf3,
                      uint32_t a0, uint32_t a1)
{
    double complex spec[O_ROWS][O_HALF], accf[2][O_HALF];
    const uint32_t a01 = (a0 + a1) & (2 * O_N - 1);
    const double complex* x0 = c->xai + (size_t)a0 * O_HALF;
    const double complex* x1 = c->xai + (size_t)a1 * O_HALF;
    const double complex* x01 = c->xai + (size_t)a01 * O_HALF;
    const size_t trgsw_f = O_ROWS * 2 * O_HALF;
    digits_fft(c, acc, spec);
    memset(accf, 0, sizeof(accf));
    for (int r = 0; r < O_ROWS; r++) {
        const int j = r / O_L, d = r % O_L;
        const double h = ldexp(1.0, -(d + 1) * O_BGBIT); /* FFNT(H * 2^-32) */
        for (int oj = 0; oj < 2; oj++) {
            const double complex* b0 = bkf3 + 0 * trgsw_f + (r * 2 + oj) * O_HALF;
            const double complex* b1 = bkf3 + 1 * trgsw_f + (r * 2 + oj) * O_HALF;
            const double complex* b2 = bkf3 + 2 * trgsw_f + (r * 2 + oj) * O_HALF;
            for (int f = 0; f < O_HALF; f++) {
                double complex comb = (oj == j) ? h : 0.0;
                comb += b2[f] * x1[f];
                comb += b1[f] * x0[f];
                comb += b0[f] * x01[f];
                accf[oj][f] += spec[r][f] * comb;
            }
        }
    }
    for (int oj = 0; oj < 2; oj++) ffnt_inverse_round(c, accf[oj], acc + oj * O_N, 0);
}

static inline uint32_t modswitch(uint32_t phase) { return phase >> (32 - 1 - O_NBIT); }

/* Blind rotation of a lvl0 TLWE x (637 words) into acc (TRLWE).
 * bar = 2N - modswitch(b) without rounding; abar_i = modswitch(a_i + 2^20)
 * (include/gatebootstrapping_gpu.cuh:801-884, :1335-1380).
 * steps < 0 runs every step; otherwise only the first `steps` CMUX steps (or
 * KB pairs), which the tests use to compare intermediate accumulators.
 * bk: coefficient-domain key for ORC_EXACT, Fourier-domain (double complex)
 * key for ORC_FP64. */
void orc_blind_rotate(const uint32_t* x, uint32_t mu, const void* bk, int kb, int mode,
                      const orc_fft_t* c, int steps, uint32_t* acc)
{
    const uint32_t bar = 2 * O_N - modswitch(x[O_N0]);
    orc_test_vector(bar, mu, acc);
    const uint32_t ro = 1u << (32 - 2 - O_NBIT);
    if (!kb) {
        const int n = steps < 0 || steps > O_N0 ? O_N0 : steps;
        for (int i = 0; i < n; i++) {
            const uint32_t ab = modswitch(x[i] + ro);
            if (mode == ORC_EXACT)
                orc_cmux_step_exact(acc, (const uint32_t*)bk + (size_t)i * O_TRGSW, ab);
            else
                orc_cmux_step_fp64(c, acc,
                                   (const double complex*)bk + (size_t)i * O_ROWS * 2 * O_HALF,
                                   ab);
        }
    } else {
        const int n = steps < 0 || steps > O_N0 / 2 ? O_N0 / 2 : steps;
        for (int p = 0; p < n; p++) {
            const uint32_t a0 = modswitch(x[2 * p] + ro), a1 = modswitch(x[2 * p + 1] + ro);
            if (mode == ORC_EXACT)
                orc_kb_step_exact(acc, (const uint32_t*)bk + (size_t)p * 3 * O_TRGSW, a0, a1);
            else
                orc_kb_step_fp64(c, acc,
                                 (const double complex*)bk + (size_t)p * 3 * O_ROWS * 2 * O_HALF,
                                 a0, a1);
        }
    }
}

/* SampleExtract at index 0 (src/bootstrap_gpu.cu:1201-1221) */
void orc_sample_extract(const uint32_t* acc, uint32_t* tlwe1)
{
    tlwe1[0] = acc[0];
    for (int n = 1; n < O_N; n++) tlwe1[n] = 0u - acc[O_N - n];
    tlwe1[O_N] = acc[O_N];
}

/* --------------------------------------------------- key switching ---- */
/* Identity key switching lvl1 -> lvl0 of x = ca*in0 + cb*in1 (+off on b)
 * (include/keyswitch_gpu.cuh:13-23 offsets, :189-256 pre-add form; with
 * ca = 1, cb = 0, off = 0 it is KeySwitchFromTLWE, :128-187). */
void orc_iks_preadd(const uint32_t* in0, const uint32_t* in1, int32_t ca, int32_t cb,
                    uint32_t off, const uint32_t* ksk, uint32_t* out)
{
    uint32_t decomp = 0;
    for (int i = 1; i <= O_T; i++) decomp += 2u << (32 - i * O_BASEBIT);
    const uint32_t round = 1u << (32 - (1 + O_BASEBIT * O_T));
    uint32_t res[O_TLWE0];
    memset(res, 0, sizeof(res));
    res[O_N0] = (uint32_t)ca * in0[O_N] + (in1 ? (uint32_t)cb * in1[O_N] : 0u) + off;
    for (int i = 0; i < O_N; i++) {
        const uint32_t xi = (uint32_t)ca * in0[i] + (in1 ? (uint32_t)cb * in1[i] : 0u);
        const uint32_t t = xi + decomp + round;
        for (int j = 0; j < O_T; j++) {
            const int32_t v = (int32_t)((t >> (32 - (j + 1) * O_BASEBIT)) & 3u) - 2;
            if (v == 0) continue;
            const uint32_t* row = ksk + (((size_t)i * O_T + j) * 2 + (v > 0 ? v - 1 : -v - 1)) * O_TLWE0;
            if (v > 0)
                for (int o = 0; o < O_TLWE0; o++) res[o] -= row[o];
            else
                for (int o = 0; o < O_TLWE0; o++) res[o] += row[o];
        }
    }
    memcpy(out, res, sizeof(res));
}

/* ------------------------------------------------------------- gates ---- */
/* gate ids (same numbering as the engine's C-ABI) */
enum {
    G_NAND = 0, G_OR, G_ORYN, G_ORNY, G_AND, G_ANDYN, G_ANDNY, G_NOR, G_XOR,
    G_XNOR, G_NOT, G_COPY, G_MUX, G_NMUX
};

/* (casign, cbsign, offset) per binary gate: src/bootstrap_gpu.cu:1905-1914,
 * :1937-1946 */
static int gate_table(int g, int32_t* ca, int32_t* cb, uint32_t* off)
{
    const uint32_t mu = O_MU;
    switch (g) {
    case G_NAND: *ca = -1; *cb = -1; *off = mu; return 1;
    case G_NOR: *ca = -1; *cb = -1; *off = 0u - mu; return 1;
    case G_XNOR: *ca = -2; *cb = -2; *off = 0u - 2 * mu; return 1;
    case G_AND: *ca = 1; *cb = 1; *off = 0u - mu; return 1;
    case G_OR: *ca = 1; *cb = 1; *off = mu; return 1;
    case G_XOR: *ca = 2; *cb = 2; *off = 2 * mu; return 1;
    case G_ANDNY: *ca = -1; *cb = 1; *off = 0u - mu; return 1;
    case G_ANDYN: *ca = 1; *cb = -1; *off = 0u - mu; return 1;
    case G_ORNY: *ca = -1; *cb = 1; *off = mu; return 1;
    case G_ORYN: *ca = 1; *cb = -1; *off = mu; return 1;
    default: return 0;
    }
}

typedef struct {
    const void* bk;    /* exact: uint32 coefficient BK; fp64: Fourier BK */
    const uint32_t* ksk;
    int kb;
    int mode;
    const orc_fft_t* fft;
} orc_keys_t;

/* lvl0 pre-add for the BR->IKS order (folded into the modulus switch by
 * __BlindRotatePreAdd[KeyBundle]__, :1382-1429 and :1432-1521) */
static void preadd0(const uint32_t* a, const uint32_t* b, int32_t ca, int32_t cb, uint32_t off,
                    uint32_t* x)
{
    for (int i = 0; i < O_N0; i++) x[i] = (uint32_t)ca * a[i] + (uint32_t)cb * b[i];
    x[O_N0] = off + (uint32_t)ca * a[O_N0] + (uint32_t)cb * b[O_N0];
}

/* One gate.  level 1: Ctxt<lvl1> I/O, IKS -> BR order
 * (src/bootstrap_gpu.cu:1223-1246, :1277-1302); level 0: Ctxt<lvl0> I/O,
 * BR -> IKS order (:1248-1273, :1305-1331).  Mux/NMux: :1557-1672,
 * :1949-2197, :2224-2344.  Not/Copy: :2200-2222. */
void orc_gate(int gate, int level, const uint32_t* in0, const uint32_t* in1,
              const uint32_t* in2, uint32_t* out, const orc_keys_t* k)
{
    const uint32_t mu = O_MU;
    const int words = level == 1 ? O_TLWE1 : O_TLWE0;
    if (gate == G_NOT || gate == G_COPY) {
        for (int i = 0; i < words; i++) out[i] = gate == G_NOT ? 0u - in0[i] : in0[i];
        return;
    }
    uint32_t acc[O_TRLWE], t1[O_TLWE1], tmp1[O_TLWE1], x0[O_TLWE0];
    int32_t ca, cb;
    uint32_t off;
    const int mux = gate == G_MUX || gate == G_NMUX;
    /* lanes: binary gate -> 1 lane; mux -> (inc, in1, 1, 1, -mu) and
     * (inc, in0, -1, 1, -mu) */
    const int lanes = mux ? 2 : 1;
    uint32_t sum[O_TLWE1];
    memset(sum, 0, sizeof(sum));
    for (int ln = 0; ln < lanes; ln++) {
        const uint32_t *a, *b;
        if (mux) {
            a = in0;
            b = ln == 0 ? in1 : in2;
            ca = ln == 0 ? 1 : -1;
            cb = 1;
            off = 0u - mu;
        } else {
            a = in0;
            b = in1;
            gate_table(gate, &ca, &cb, &off);
        }
        if (level == 1)
            orc_iks_preadd(a, b, ca, cb, off, k->ksk, x0);
        else
            preadd0(a, b, ca, cb, off, x0);
        orc_blind_rotate(x0, mu, k->bk, k->kb, k->mode, k->fft, -1, acc);
        orc_sample_extract(acc, t1);
        for (int i = 0; i < O_TLWE1; i++) sum[i] += t1[i];
    }
    if (gate == G_MUX) sum[O_N] += mu;
    if (gate == G_NMUX) {
        for (int i = 0; i < O_TLWE1; i++) sum[i] = 0u - sum[i];
        sum[O_N] -= mu;
    }
    if (level == 1) {
        memcpy(out, sum, sizeof(sum));
    } else {
        memcpy(tmp1, sum, sizeof(sum));
        orc_iks_preadd(tmp1, NULL, 1, 0, 0, k->ksk, out);
    }
}

/* count gates, OpenMP over gates; inputs and out are [count][words]. */
void orc_gate_batch(const int32_t* gates, int level, const uint32_t* in0, const uint32_t* in1,
                    const uint32_t* in2, uint32_t* out, int64_t count, const void* bk,
                    const uint32_t* ksk, int kb, int mode, const orc_fft_t* fft)
{
    const orc_keys_t k = {bk, ksk, kb, mode, fft};
    const int words = level == 1 ? O_TLWE1 : O_TLWE0;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < count; g++)
        orc_gate(gates[g], level, in0 + g * words, in1 ? in1 + g * words : NULL,
                 in2 ? in2 + g * words : NULL, out + g * words, &k);
}

/* Blind rotation of count lvl0 TLWEs (OpenMP over inputs), first `steps`
 * steps only when steps >= 0: acc_out is [count][2][N]. */
void orc_blind_rotate_batch(const uint32_t* x, const uint32_t* mu, int64_t count, const void* bk,
                            int kb, int mode, const orc_fft_t* fft, int steps, uint32_t* acc_out)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < count; g++)
        orc_blind_rotate(x + g * O_TLWE0, mu[g], bk, kb, mode, fft, steps, acc_out + g * O_TRLWE);
}

void orc_iks_batch(const uint32_t* in0, const uint32_t* in1, const int32_t* ca, const int32_t* cb,
                   const uint32_t* off, const uint32_t* ksk, int64_t count, uint32_t* out)
{
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < count; g++)
        orc_iks_preadd(in0 + g * O_TLWE1, in1 ? in1 + g * O_TLWE1 : NULL, ca[g], cb[g], off[g],
                       ksk, out + g * O_TLWE0);
}

/* ---------------------------------------- FFNT known-answer helpers ---- */
/* test/test_fft_roundtrip.cu:19-124: fold+twist+FFT then IFFT+untwist (no
 * rounding); and the negacyclic square of a real polynomial. */
void orc_ffnt_roundtrip(const orc_fft_t* c, const double* in, double* out)
{
    double complex z[O_HALF];
    ffnt_forward(c, in, z);
    fft512(c, z, 1);
    for (int i = 0; i < O_HALF; i++) {
        const double complex v = z[i] * c->untwist[i];
        out[i] = creal(v);
        out[i + O_HALF] = cimag(v);
    }
}

void orc_ffnt_square(const orc_fft_t* c, const double* in, double* out)
{
    double complex z[O_HALF];
    ffnt_forward(c, in, z);
    for (int i = 0; i < O_HALF; i++) z[i] = z[i] * z[i];
    fft512(c, z, 1);
    for (int i = 0; i < O_HALF; i++) {
        const double complex v = z[i] * c->untwist[i];
        out[i] = creal(v);
        out[i + O_HALF] = cimag(v);
    }
}

/* exact negacyclic product of two double polynomials (schoolbook,
 * test/test_fft_roundtrip.cu:125-138) */
void orc_negacyclic_mul_f64(const double* a, const double* b, double* out)
{
    for (int i = 0; i < O_N; i++) out[i] = 0.0;
    for (int i = 0; i < O_N; i++)
        for (int j = 0; j < O_N; j++) {
            const int idx = i + j;
            if (idx < O_N)
                out[idx] += a[i] * b[j];
            else
                out[idx - O_N] -= a[i] * b[j];
        }
}

/* exact negacyclic product of a signed digit polynomial and a Torus32
 * polynomial (the INT8 path's contract) */
void orc_negacyclic_mul_exact(const int32_t* d, const uint32_t* key, uint32_t* out)
{
    memset(out, 0, sizeof(uint32_t) * O_N);
    negacyclic_mac_exact(out, d, key);
}

/* ===================================================================== */
/* lvl0 -> lvl2 gate bootstrapping (N = 2048, k = 1, l = 4, Bgbit = 10,   */
/* Torus64) and lvl2 -> lvl0 key switching (basebit 2, t 7): the          */
/* *_lvl02 gates (src/cufhe_gates_gpu.cu:826-979), same templates at      */
/* lvl02param / lvl20param.                                               */
/* ===================================================================== */
#define O2_N 2048
#define O2_NBIT 11
#define O2_HALF 1024
#define O2_L 4
#define O2_BGBIT 10
#define O2_ROWS 8
#define O2_TRLWE (2 * O2_N)
#define O2_TRGSW (O2_ROWS * O2_TRLWE)
#define O2_TLWE2 (O2_N + 1)

static void rotate_poly64(uint64_t* out, const uint64_t* p, uint32_t a)
{
    const uint32_t am = a & (O2_N - 1), neg = a >> O2_NBIT;
    for (uint32_t n = 0; n < O2_N; n++) {
        const uint64_t v = p[(n - a) & (O2_N - 1)];
        out[n] = ((n < am) ^ neg) ? 0ull - v : v;
    }
}

/* l = 4 signed digits of 10 bits (include/gatebootstrapping_gpu.cuh:20-29) */
void orc2_decompose(const uint64_t* poly, int32_t* digits)
{
    uint64_t off = 0;
    for (int i = 1; i <= O2_L; i++) off += (uint64_t)512 << (64 - i * O2_BGBIT);
    const uint64_t round = 1ull << (64 - O2_L * O2_BGBIT - 1);
    for (int n = 0; n < O2_N; n++) {
        const uint64_t t = poly[n] + off + round;
        for (int d = 0; d < O2_L; d++)
            digits[d * O2_N + n] = (int32_t)((t >> (64 - (d + 1) * O2_BGBIT)) & 1023u) - 512;
    }
}

static void negacyclic_mac_exact64(uint64_t* restrict out, const int32_t* restrict d,
                                   const uint64_t* restrict key)
{
    for (int m = 0; m < O2_N; m++) {
        const uint64_t dm = (uint64_t)(int64_t)d[m];
        if (!dm) continue;
        const uint64_t* kw = key + O2_N - m;
        for (int n = 0; n < m; n++) out[n] -= dm * kw[n];
        const uint64_t* kp = key - m;
        for (int n = m; n < O2_N; n++) out[n] += dm * kp[n];
    }
}

void orc2_extprod_exact(const uint64_t* trgsw, const uint64_t* in, uint64_t* out)
{
    int32_t* dig = (int32_t*)malloc(sizeof(int32_t) * O2_L * O2_N);
    memset(out, 0, sizeof(uint64_t) * O2_TRLWE);
    for (int j = 0; j < 2; j++) {
        orc2_decompose(in + j * O2_N, dig);
        for (int d = 0; d < O2_L; d++) {
            const int r = j * O2_L + d;
            for (int oj = 0; oj < 2; oj++)
                negacyclic_mac_exact64(out + oj * O2_N, dig + d * O2_N,
                                       trgsw + ((size_t)r * 2 + oj) * O2_N);
        }
    }
    free(dig);
}

void orc2_cmux_step_exact(uint64_t* acc, const uint64_t* bk_i, uint32_t abar)
{
    uint64_t* diff = (uint64_t*)malloc(sizeof(uint64_t) * 2 * O2_TRLWE);
    uint64_t* prod = diff + O2_TRLWE;
    for (int j = 0; j < 2; j++) {
        rotate_poly64(diff + j * O2_N, acc + j * O2_N, abar);
        for (int n = 0; n < O2_N; n++) diff[j * O2_N + n] -= acc[j * O2_N + n];
    }
    orc2_extprod_exact(bk_i, diff, prod);
    for (int i = 0; i < O2_TRLWE; i++) acc[i] += prod[i];
    free(diff);
}

void orc2_kb_step_exact(uint64_t* acc, const uint64_t* bk3, uint32_t a0, uint32_t a1)
{
    uint64_t* kb = (uint64_t*)calloc(O2_TRGSW, sizeof(uint64_t));
    uint64_t* rot = (uint64_t*)malloc(sizeof(uint64_t) * (O2_N + O2_TRLWE));
    uint64_t* out = rot + O2_N;
    const uint32_t a01 = (a0 + a1) & (2 * O2_N - 1);
    const uint32_t av[3] = {a01, a0, a1};
    for (int r = 0; r < O2_ROWS; r++) {
        const int j = r / O2_L, d = r % O2_L;
        kb[((size_t)r * 2 + j) * O2_N] += 1ull << (64 - (d + 1) * O2_BGBIT);
        for (int e = 0; e < 3; e++)
            for (int oj = 0; oj < 2; oj++) {
                const uint64_t* p = bk3 + (size_t)e * O2_TRGSW + ((size_t)r * 2 + oj) * O2_N;
                uint64_t* q = kb + ((size_t)r * 2 + oj) * O2_N;
                rotate_poly64(rot, p, av[e]);
                for (int n = 0; n < O2_N; n++) q[n] += rot[n] - p[n];
            }
    }
    orc2_extprod_exact(kb, acc, out);
    memcpy(acc, out, sizeof(uint64_t) * O2_TRLWE);
    free(rot);
    free(kb);
}

/* ---- FP64 FFNT for N = 2048 (1024-point transform) ---- */
typedef struct {
    double complex twist[O2_HALF];
    double complex untwist[O2_HALF];
    double complex root[O2_HALF];   /* e^{2 pi i k / 1024} */
    double complex psi[2 * O2_N];   /* e^{i pi t / 2048}: KeyBundle factors by evaluation */
    uint16_t bitrev[O2_HALF];
} orc_fft2_t;

orc_fft2_t* orc_fft2_create(void)
{
    orc_fft2_t* c = (orc_fft2_t*)calloc(1, sizeof(orc_fft2_t));
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int i = 0; i < O2_HALF; i++) {
        const long double tw = pi * i / O2_N;
        c->twist[i] = (double)cosl(tw) + I * (double)sinl(tw);
        c->untwist[i] = ((double)cosl(tw) - I * (double)sinl(tw)) / O2_HALF;
        const long double ro = 2 * pi * i / O2_HALF;
        c->root[i] = (double)cosl(ro) + I * (double)sinl(ro);
        int r = 0;
        for (int b = 0; b < 10; b++) r |= ((i >> b) & 1) << (9 - b);
        c->bitrev[i] = (uint16_t)r;
    }
    for (int t = 0; t < 2 * O2_N; t++) {
        const long double a = pi * t / O2_N;
        c->psi[t] = (double)cosl(a) + I * (double)sinl(a);
    }
    return c;
}

void orc_fft2_destroy(orc_fft2_t* c) { free(c); }

static void fft1024(const orc_fft2_t* c, double complex* x, int inverse)
{
    for (int i = 0; i < O2_HALF; i++) {
        const int j = c->bitrev[i];
        if (i < j) {
            double complex t = x[i];
            x[i] = x[j];
            x[j] = t;
        }
    }
    for (int len = 2; len <= O2_HALF; len <<= 1) {
        const int half = len >> 1, step = O2_HALF / len;
        for (int s = 0; s < O2_HALF; s += len)
            for (int k = 0; k < half; k++) {
                double complex w = c->root[k * step];
                if (inverse) w = conj(w);
                const double complex u = x[s + k], v = x[s + k + half] * w;
                x[s + k] = u + v;
                x[s + k + half] = u - v;
            }
    }
}

static void ffnt2_forward(const orc_fft2_t* c, const double* re, double complex* out)
{
    for (int i = 0; i < O2_HALF; i++) out[i] = (re[i] + I * re[i + O2_HALF]) * c->twist[i];
    fft1024(c, out, 0);
}

/* FP64 -> Torus64 as include/utils_gpu.cuh:48-65 (mantissa shift, wraps mod 2^64) */
uint64_t orc_double_to_torus64(double d)
{
    uint64_t i;
    memcpy(&i, &d, 8);
    const int expo = (int)(i >> 52) & 0x7FF;
    if (expo == 0) return 0;
    const uint64_t m = (i & 0x000FFFFFFFFFFFFFull) | 0x0010000000000000ull;
    const int shift = expo - 1075;
    uint64_t val;
    if (shift >= 64)
        val = 0;
    else if (shift >= 0)
        val = m << shift;
    else if (shift > -64)
        val = m >> (-shift);
    else
        val = 0;
    return (i >> 63) ? 0ull - val : val;
}

void orc2_bk_to_fft(const orc_fft2_t* c, const uint64_t* bk, int ntrgsw, double complex* out)
{
#pragma omp parallel for schedule(static)
    for (int p = 0; p < ntrgsw * O2_ROWS * 2; p++) {
        double* re = (double*)malloc(sizeof(double) * O2_N);
        for (int i = 0; i < O2_N; i++)
            re[i] = (double)(int64_t)bk[(size_t)p * O2_N + i] * (1.0 / 18446744073709551616.0);
        ffnt2_forward(c, re, out + (size_t)p * O2_HALF);
        free(re);
    }
}

static void ffnt2_inverse_round(const orc_fft2_t* c, double complex* acc, uint64_t* out, int add)
{
    fft1024(c, acc, 1);
    for (int i = 0; i < O2_HALF; i++) {
        const double complex v = acc[i] * c->untwist[i];
        const uint64_t lo = orc_double_to_torus64(creal(v) * 18446744073709551616.0);
        const uint64_t hi = orc_double_to_torus64(cimag(v) * 18446744073709551616.0);
        if (add) {
            out[i] += lo;
            out[i + O2_HALF] += hi;
        } else {
            out[i] = lo;
            out[i + O2_HALF] = hi;
        }
    }
}

static void digits2_fft(const orc_fft2_t* c, const uint64_t* in, double complex* spec /*[8][1024]*/)
{
    int32_t* dig = (int32_t*)malloc(sizeof(int32_t) * O2_L * O2_N);
    double* re = (double*)malloc(sizeof(double) * O2_N);
    for (int j = 0; j < 2; j++) {
        orc2_decompose(in + j * O2_N, dig);
        for (int d = 0; d < O2_L; d++) {
            for (int i = 0; i < O2_N; i++) re[i] = (double)dig[d * O2_N + i];
            ffnt2_forward(c, re, spec + (size_t)(j * O2_L + d) * O2_HALF);
        }
    }
    free(re);
    free(dig);
}

void orc2_cmux_step_fp64(const orc_fft2_t* c, uint64_t* acc, const double complex* bkf_i,
                         uint32_t abar)
{
    uint64_t* diff = (uint64_t*)malloc(sizeof(uint64_t) * O2_TRLWE);
    double complex* spec = (double complex*)malloc(sizeof(double complex) * (O2_ROWS + 2) * O2_HALF);
    double complex* accf = spec + O2_ROWS * O2_HALF;
    for (int j = 0; j < 2; j++) {
        rotate_poly64(diff + j * O2_N, acc + j * O2_N, abar);
        for (int n = 0; n < O2_N; n++) diff[j * O2_N + n] -= acc[j * O2_N + n];
    }
    digits2_fft(c, diff, spec);
    memset(accf, 0, sizeof(double complex) * 2 * O2_HALF);
    for (int r = 0; r < O2_ROWS; r++)
        for (int oj = 0; oj < 2; oj++)
            for (int f = 0; f < O2_HALF; f++)
                accf[oj * O2_HALF + f] +=
                    spec[r * O2_HALF + f] * bkf_i[((size_t)r * 2 + oj) * O2_HALF + f];
    for (int oj = 0; oj < 2; oj++) ffnt2_inverse_round(c, accf + oj * O2_HALF, acc + oj * O2_N, 1);
    free(spec);
    free(diff);
}

void orc2_kb_step_fp64(const orc_fft2_t* c, uint64_t* acc, const double complex* bkf3, uint32_t a0,
                       uint32_t a1)
{
    double complex* spec = (double complex*)malloc(sizeof(double complex) * (O2_ROWS + 2) * O2_HALF);
    double complex* accf = spec + O2_ROWS * O2_HALF;
    const uint32_t a01 = (a0 + a1) & (2 * O2_N - 1);
    const size_t trgsw_f = (size_t)O2_ROWS * 2 * O2_HALF;
    digits2_fft(c, acc, spec);
    memset(accf, 0, sizeof(double complex) * 2 * O2_HALF);
    for (int f = 0; f < O2_HALF; f++) {
        const uint32_t e = 1u + 4u * (uint32_t)f;
        const double complex x0 = c->psi[(e * a0) & (2 * O2_N - 1)] - 1.0;
        const double complex x1 = c->psi[(e * a1) & (2 * O2_N - 1)] - 1.0;
        const double complex x01 = c->psi[(e * a01) & (2 * O2_N - 1)] - 1.0;
        for (int r = 0; r < O2_ROWS; r++) {
            const int j = r / O2_L, d = r % O2_L;
            const double h = ldexp(1.0, -(d + 1) * O2_BGBIT);
            for (int oj = 0; oj < 2; oj++) {
                const size_t o = ((size_t)r * 2 + oj) * O2_HALF + f;
                double complex comb = (oj == j) ? h : 0.0;
                comb += bkf3[2 * trgsw_f + o] * x1;
                comb += bkf3[1 * trgsw_f + o] * x0;
                comb += bkf3[0 * trgsw_f + o] * x01;
                accf[oj * O2_HALF + f] += spec[r * O2_HALF + f] * comb;
            }
        }
    }
    for (int oj = 0; oj < 2; oj++) ffnt2_inverse_round(c, accf + oj * O2_HALF, acc + oj * O2_N, 0);
    free(spec);
}

void orc2_test_vector(uint32_t bar, uint64_t mu, uint64_t* acc)
{
    for (uint32_t i = 0; i < O2_N; i++) {
        acc[i] = 0;
        if (bar == 2 * O2_N)
            acc[O2_N + i] = mu;
        else
            acc[O2_N + i] = ((i < (bar & (O2_N - 1))) ^ (bar >> O2_NBIT)) ? 0ull - mu : mu;
    }
}

/* lvl0 TLWE -> lvl2 TRLWE: bar = 2N - (b >> 20), abar = (a + 2^19) >> 20 */
void orc2_blind_rotate(const uint32_t* x, uint64_t mu, const void* bk, int kb, int mode,
                       const orc_fft2_t* c, int steps, uint64_t* acc)
{
    const uint32_t bar = 2 * O2_N - (x[O_N0] >> (32 - 1 - O2_NBIT));
    orc2_test_vector(bar, mu, acc);
    const uint32_t ro = 1u << (32 - 2 - O2_NBIT);
    const size_t trgsw_f = (size_t)O2_ROWS * 2 * O2_HALF;
    if (!kb) {
        const int n = steps < 0 || steps > O_N0 ? O_N0 : steps;
        for (int i = 0; i < n; i++) {
            const uint32_t ab = (x[i] + ro) >> (32 - 1 - O2_NBIT);
            if (mode == ORC_EXACT)
                orc2_cmux_step_exact(acc, (const uint64_t*)bk + (size_t)i * O2_TRGSW, ab);
            else
                orc2_cmux_step_fp64(c, acc, (const double complex*)bk + (size_t)i * trgsw_f, ab);
        }
    } else {
        const int n = steps < 0 || steps > O_N0 / 2 ? O_N0 / 2 : steps;
        for (int p = 0; p < n; p++) {
            const uint32_t a0 = (x[2 * p] + ro) >> (32 - 1 - O2_NBIT);
            const uint32_t a1 = (x[2 * p + 1] + ro) >> (32 - 1 - O2_NBIT);
            if (mode == ORC_EXACT)
                orc2_kb_step_exact(acc, (const uint64_t*)bk + (size_t)p * 3 * O2_TRGSW, a0, a1);
            else
                orc2_kb_step_fp64(c, acc, (const double complex*)bk + (size_t)p * 3 * trgsw_f, a0, a1);
        }
    }
}

void orc2_sample_extract(const uint64_t* acc, uint64_t* tlwe2)
{
    tlwe2[0] = acc[0];
    for (int n = 1; n < O2_N; n++) tlwe2[n] = 0ull - acc[O2_N - n];
    tlwe2[O2_N] = acc[O2_N];
}

/* lvl2 -> lvl0 identity key switching (KeySwitchFromTLWE<lvl20param>,
 * include/keyswitch_gpu.cuh:128-187; Torus64 -> Torus32 conversion of b with
 * rounding, :33-50).  ksk: TLWE<lvl0>[2048][7][2]. */
void orc20_iks(const uint64_t* in, const uint32_t* ksk, uint32_t* out)
{
    uint64_t decomp = 0;
    for (int i = 1; i <= O_T; i++) decomp += 2ull << (64 - i * O_BASEBIT);
    const uint64_t round = 1ull << (64 - (1 + O_BASEBIT * O_T));
    uint32_t res[O_TLWE0];
    memset(res, 0, sizeof(res));
    res[O_N0] = (uint32_t)((in[O2_N] + (1ull << 31)) >> 32);
    for (int i = 0; i < O2_N; i++) {
        const uint64_t t = in[i] + decomp + round;
        for (int j = 0; j < O_T; j++) {
            const int32_t v = (int32_t)((t >> (64 - (j + 1) * O_BASEBIT)) & 3u) - 2;
            if (v == 0) continue;
            const uint32_t* row =
                ksk + (((size_t)i * O_T + j) * 2 + (v > 0 ? v - 1 : -v - 1)) * O_TLWE0;
            if (v > 0)
                for (int o = 0; o < O_TLWE0; o++) res[o] -= row[o];
            else
                for (int o = 0; o < O_TLWE0; o++) res[o] += row[o];
        }
    }
    memcpy(out, res, sizeof(res));
}

/* *_lvl02 gates: Ctxt<lvl0> I/O, lvl0 pre-add, blind rotation to lvl2, mux
 * combination on the TRLWE (+mu2), SampleExtract, key switch lvl2 -> lvl0. */
void orc2_gate(int gate, const uint32_t* in0, const uint32_t* in1, const uint32_t* in2,
               uint32_t* out, const void* bk, const uint32_t* ksk, int kb, int mode,
               const orc_fft2_t* c)
{
    const uint64_t mu2 = 1ull << 61;
    if (gate == G_NOT || gate == G_COPY) {
        for (int i = 0; i < O_TLWE0; i++) out[i] = gate == G_NOT ? 0u - in0[i] : in0[i];
        return;
    }
    uint64_t* acc = (uint64_t*)malloc(sizeof(uint64_t) * (O2_TRLWE + 2 * O2_TLWE2));
    uint64_t* t2 = acc + O2_TRLWE;
    uint64_t* sum = t2 + O2_TLWE2;
    uint32_t x0[O_TLWE0];
    int32_t ca, cb;
    uint32_t off;
    const int mux = gate == G_MUX || gate == G_NMUX;
    memset(sum, 0, sizeof(uint64_t) * O2_TLWE2);
    for (int ln = 0; ln < (mux ? 2 : 1); ln++) {
        const uint32_t* b;
        if (mux) {
            b = ln == 0 ? in1 : in2;
            ca = ln == 0 ? 1 : -1;
            cb = 1;
            off = 0u - O_MU;
        } else {
            b = in1;
            gate_table(gate, &ca, &cb, &off);
        }
        preadd0(in0, b, ca, cb, off, x0);
        orc2_blind_rotate(x0, mu2, bk, kb, mode, c, -1, acc);
        orc2_sample_extract(acc, t2);
        for (int i = 0; i < O2_TLWE2; i++) sum[i] += t2[i];
    }
    if (gate == G_MUX) sum[O2_N] += mu2;
    if (gate == G_NMUX) {
        for (int i = 0; i < O2_TLWE2; i++) sum[i] = 0ull - sum[i];
        sum[O2_N] -= mu2;
    }
    orc20_iks(sum, ksk, out);
    free(acc);
}

void orc2_gate_batch(const int32_t* gates, const uint32_t* in0, const uint32_t* in1,
                     const uint32_t* in2, uint32_t* out, int64_t count, const void* bk,
                     const uint32_t* ksk, int kb, int mode, const orc_fft2_t* c)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < count; g++)
        orc2_gate(gates[g], in0 + g * O_TLWE0, in1 ? in1 + g * O_TLWE0 : NULL,
                  in2 ? in2 + g * O_TLWE0 : NULL, out + g * O_TLWE0, bk, ksk, kb, mode, c);
}

void orc2_blind_rotate_batch(const uint32_t* x, uint64_t mu, int64_t count, const void* bk,
                             int kb, int mode, const orc_fft2_t* c, int steps, uint64_t* acc_out)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t g = 0; g < count; g++)
        orc2_blind_rotate(x + g * O_TLWE0, mu, bk, kb, mode, c, steps, acc_out + g * O2_TRLWE);
}

void orc20_iks_batch(const uint64_t* in, const uint32_t* ksk, int64_t count, uint32_t* out)
{
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < count; g++) orc20_iks(in + g * O2_TLWE2, ksk, out + g * O_TLWE0);
}

void orc2_ffnt_roundtrip(const orc_fft2_t* c, const double* in, double* out)
{
    double complex z[O2_HALF];
    ffnt2_forward(c, in, z);
    fft1024(c, z, 1);
    for (int i = 0; i < O2_HALF; i++) {
        const double complex v = z[i] * c->untwist[i];
        out[i] = creal(v);
        out[i + O2_HALF] = cimag(v);
    }
}

void orc2_ffnt_square(const orc_fft2_t* c, const double* in, double* out)
{
    double complex z[O2_HALF];
    ffnt2_forward(c, in, z);
    for (int i = 0; i < O2_HALF; i++) z[i] = z[i] * z[i];
    fft1024(c, z, 1);
    for (int i = 0; i < O2_HALF; i++) {
        const double complex v = z[i] * c->untwist[i];
        out[i] = creal(v);
        out[i + O2_HALF] = cimag(v);
    }
}

/* ===================================================================== */
/* Circuit bootstrapping (CGGI17 form) and CMUX lookup tables.           */
/*   lvl0 TLWE -> 3 blind rotations to lvl2 (test polynomial mu_i =      */
/*   2^(64 - 6(i+1) - 1), then b += mu_i: message m 2^(64 - 6(i+1)))     */
/*   -> private functional key switching lvl2 -> lvl1 (basebit 4, t 10) */
/*   with f(x) = -x s1 (rows j = 0) and f(x) = x (rows j = 1)            */
/*   -> TRGSW<lvl1> with l = 3, Bgbit = 6, row r = j l + i.              */
/* The reference's circuit bootstrapping is annihilation-based            */
/* (src/circuitbootstrapping_gpu.cu) and has no private key switching,   */
/* so these functions restate the published CGGI17 procedure; their      */
/* parity is unpinned against the reference.  The CMUX is the reference's */
/* CMUX (src/bootstrap_gpu.cu:704-813): d0 + ExtProd(C, d1 - d0).         */
/* ===================================================================== */
#define PKS_BASEBIT 4
#define PKS_T 10
#define PKS_NU 15

/* exact private key switching: out[2][N] = -sum_i sum_j key[i][j][d_ij - 1]
 * over the n_src + 1 words of the Torus64 input (TFHEpp PrivKeySwitch) */
void orc_privks(const uint64_t* tlwe, uint32_t n_src, const uint32_t* key, uint32_t* out)
{
    memset(out, 0, sizeof(uint32_t) * O_TRLWE);
    const uint64_t off = 1ull << (64 - (1 + PKS_BASEBIT * PKS_T));
    for (uint32_t i = 0; i <= n_src; i++) {
        const uint64_t abar = tlwe[i] + off;
        for (int j = 0; j < PKS_T; j++) {
            const uint32_t d = (uint32_t)(abar >> (64 - (j + 1) * PKS_BASEBIT)) & 15u;
            if (!d) continue;
            const uint32_t* row = key + (((size_t)i * PKS_T + j) * PKS_NU + d - 1) * O_TRLWE;
            for (int w = 0; w < O_TRLWE; w++) out[w] -= row[w];
        }
    }
}

void orc_privks_batch(const uint64_t* tlwe, int64_t count, uint32_t n_src, const uint32_t* key,
                      uint32_t* out)
{
#pragma omp parallel for schedule(static)
    for (int64_t u = 0; u < count; u++)
        orc_privks(tlwe + u * (n_src + 1), n_src, key, out + u * O_TRLWE);
}

/* signed gadget digits (L digits of bgbit bits, digit 0 most significant)
 * of a Torus32 polynomial, with the offset + rounding of
 * include/gatebootstrapping_gpu.cuh:20-29 */
static void decompose_g(const uint32_t* poly, int L, int bgbit, int32_t* digits)
{
    const uint32_t half = 1u << (bgbit - 1), mask = (1u << bgbit) - 1;
    uint32_t off = 0;
    for (int i = 1; i <= L; i++) off += half << (32 - i * bgbit);
    off += 1u << (32 - L * bgbit - 1);
    for (int n = 0; n < O_N; n++) {
        const uint32_t t = poly[n] + off;
        for (int d = 0; d < L; d++)
            digits[d * O_N + n] = (int32_t)((t >> (32 - (d + 1) * bgbit)) & mask) - (int32_t)half;
    }
}

/* exact external product with a TRGSW of 2L rows (row r = j L + d) */
void orc_extprod_exact_g(const uint32_t* trgsw, const uint32_t* in, int L, int bgbit, uint32_t* out)
{
    int32_t* dig = (int32_t*)malloc(sizeof(int32_t) * L * O_N);
    memset(out, 0, sizeof(uint32_t) * O_TRLWE);
    for (int j = 0; j < 2; j++) {
        decompose_g(in + j * O_N, L, bgbit, dig);
        for (int d = 0; d < L; d++)
            for (int oj = 0; oj < 2; oj++)
                negacyclic_mac_exact(out + oj * O_N, dig + d * O_N,
                                     trgsw + ((size_t)(j * L + d) * 2 + oj) * O_N);
    }
    free(dig);
}

/* FP64 form: trgsw_f = [2L][2][N/2] Fourier rows (orc_polys_to_fft) */
void orc_extprod_fp64_g(const orc_fft_t* c, const double complex* trgsw_f, const uint32_t* in,
                        int L, int bgbit, uint32_t* out)
{
    int32_t* dig = (int32_t*)malloc(sizeof(int32_t) * L * O_N);
    double complex* spec = (double complex*)malloc(sizeof(double complex) * (2 * L + 2) * O_HALF);
    double complex* acc = spec + 2 * L * O_HALF;
    double re[O_N];
    for (int j = 0; j < 2; j++) {
        decompose_g(in + j * O_N, L, bgbit, dig);
        for (int d = 0; d < L; d++) {
            for (int i = 0; i < O_N; i++) re[i] = (double)dig[d * O_N + i];
            ffnt_forward(c, re, spec + (size_t)(j * L + d) * O_HALF);
        }
    }
    memset(acc, 0, sizeof(double complex) * 2 * O_HALF);
    for (int r = 0; r < 2 * L; r++)
        for (int oj = 0; oj < 2; oj++)
            for (int f = 0; f < O_HALF; f++)
                acc[oj * O_HALF + f] += spec[r * O_HALF + f] * trgsw_f[(r * 2 + oj) * O_HALF + f];
    for (int oj = 0; oj < 2; oj++) ffnt_inverse_round(c, acc + oj * O_HALF, out + oj * O_N, 0);
    free(spec);
    free(dig);
}

/* Torus32 polynomials -> Fourier domain (src/bootstrap_gpu.cu:59-112) */
void orc_polys_to_fft(const orc_fft_t* c, const uint32_t* polys, int64_t npolys,
                      double complex* out)
{
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < npolys; p++) {
        double re[O_N];
        for (int i = 0; i < O_N; i++)
            re[i] = (double)(int32_t)polys[p * O_N + i] * (1.0 / 4294967296.0);
        ffnt_forward(c, re, out + p * O_HALF);
    }
}

/* CMUX: out = d0 + ExtProd(C, d1 - d0) */
void orc_cmux_g(const void* trgsw, const uint32_t* d1, const uint32_t* d0, int L, int bgbit,
                int mode, const orc_fft_t* c, uint32_t* out)
{
    uint32_t diff[O_TRLWE], prod[O_TRLWE];
    for (int w = 0; w < O_TRLWE; w++) diff[w] = d1[w] - d0[w];
    if (mode == ORC_EXACT)
        orc_extprod_exact_g((const uint32_t*)trgsw, diff, L, bgbit, prod);
    else
        orc_extprod_fp64_g(c, (const double complex*)trgsw, diff, L, bgbit, prod);
    for (int w = 0; w < O_TRLWE; w++) out[w] = d0[w] + prod[w];
}

void orc_cmux_batch_g(const void* trgsw, const uint32_t* d1, const uint32_t* d0, int64_t count,
                      int L, int bgbit, int mode, const orc_fft_t* c, uint32_t* out)
{
    const size_t tw = (size_t)2 * L * 2 * (mode == ORC_EXACT ? O_N : O_HALF);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < count; i++) {
        const void* t = mode == ORC_EXACT ? (const void*)((const uint32_t*)trgsw + i * tw)
                                          : (const void*)((const double complex*)trgsw + i * tw);
        orc_cmux_g(t, d1 + i * O_TRLWE, d0 + i * O_TRLWE, L, bgbit, mode, c, out + i * O_TRLWE);
    }
}

#define CB_L 3
#define CB_BGBIT 6

/* circuit bootstrapping of one lvl0 TLWE to TRGSW<lvl1> [6][2][N] */
void orc_circuit_bootstrap(const uint32_t* tlwe0, const void* bk2, int kb, int mode,
                           const orc_fft2_t* c2, const uint32_t* privks0, const uint32_t* privks1,
                           uint32_t* trgsw)
{
    uint64_t* acc = (uint64_t*)malloc(sizeof(uint64_t) * (O2_TRLWE + O2_TLWE2));
    uint64_t* t2 = acc + O2_TRLWE;
    for (int i = 0; i < CB_L; i++) {
        const uint64_t mu = 1ull << (64 - (i + 1) * CB_BGBIT - 1);
        orc2_blind_rotate(tlwe0, mu, bk2, kb, mode, c2, -1, acc);
        orc2_sample_extract(acc, t2);
        t2[O2_N] += mu;
        orc_privks(t2, O2_N, privks0, trgsw + (size_t)(0 * CB_L + i) * O_TRLWE);
        orc_privks(t2, O2_N, privks1, trgsw + (size_t)(1 * CB_L + i) * O_TRLWE);
    }
    free(acc);
}

void orc_circuit_bootstrap_batch(const uint32_t* tlwe0, int64_t count, const void* bk2, int kb,
                                 int mode, const orc_fft2_t* c2, const uint32_t* privks0,
                                 const uint32_t* privks1, uint32_t* trgsw)
{
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t u = 0; u < count; u++)
        orc_circuit_bootstrap(tlwe0 + u * O_TLWE0, bk2, kb, mode, c2, privks0, privks1,
                              trgsw + u * 2 * CB_L * O_TRLWE);
}

/* SampleExtract at coefficient k of a TRLWE<lvl1> */
static void sample_extract_k(const uint32_t* acc, int k, uint32_t* tlwe1)
{
    for (int n = 0; n < O_N; n++)
        tlwe1[n] = n <= k ? acc[k - n] : 0u - acc[O_N + k - n];
    tlwe1[O_N] = acc[O_N + k];
}

/* 8-bit -> 8-bit lookup table by a CMUX tree over 8 address TRGSWs
 * (trgsw[k] selects on address bit k, LSB first); the 8 output bits are
 * packed in coefficients 0..7 of the leaves (+mu for 1, -mu for 0), and
 * SampleExtract at coefficient b gives output bit b as a TLWE<lvl1>. */
void orc_lut_eval(const void* trgsw8, const uint8_t* lut, uint32_t mu, int L, int bgbit, int mode,
                  const orc_fft_t* c, uint32_t* out /* [8][N+1] */)
{
    uint32_t* nodes = (uint32_t*)calloc((size_t)256 * O_TRLWE, sizeof(uint32_t));
    for (int x = 0; x < 256; x++)
        for (int b = 0; b < 8; b++)
            nodes[(size_t)x * O_TRLWE + O_N + b] = ((lut[x] >> b) & 1) ? mu : 0u - mu;
    const size_t tw = (size_t)2 * L * 2 * (mode == ORC_EXACT ? O_N : O_HALF);
    for (int k = 0, w = 256; k < 8; k++, w >>= 1) {
        const void* t = mode == ORC_EXACT ? (const void*)((const uint32_t*)trgsw8 + k * tw)
                                          : (const void*)((const double complex*)trgsw8 + k * tw);
        for (int m = 0; m < w / 2; m++)
            orc_cmux_g(t, nodes + (size_t)(2 * m + 1) * O_TRLWE, nodes + (size_t)(2 * m) * O_TRLWE,
                       L, bgbit, mode, c, nodes + (size_t)m * O_TRLWE);
    }
    for (int b = 0; b < 8; b++) sample_extract_k(nodes, b, out + (size_t)b * O_TLWE1);
    free(nodes);
}

void orc_lut_eval_batch(const void* trgsw, const uint8_t* luts, int64_t count, uint32_t mu, int L,
                        int bgbit, int mode, const orc_fft_t* c, uint32_t* out)
{
    const size_t tw = (size_t)8 * 2 * L * 2 * (mode == ORC_EXACT ? O_N : O_HALF);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < count; q++) {
        const void* t = mode == ORC_EXACT ? (const void*)((const uint32_t*)trgsw + q * tw)
                                          : (const void*)((const double complex*)trgsw + q * tw);
        orc_lut_eval(t, luts + q * 256, mu, L, bgbit, mode, c, out + q * 8 * O_TLWE1);
    }
}
