/*
 * TFHE parameter sets of the lvl1 gate-bootstrapping path.
 *
 * The reference takes these from TFHEpp's params.hpp (an empty submodule in
 * the reference tree); the values below are the ones its kernels are
 * instantiated with for the 128-bit lvl1 path:
 *   lvl0  : LWE, n = 636, binary key, noise std 9.25e-5           (lvl0param)
 *   lvl1  : GLWE k = 1, N = 1024, l = 2, Bgbit = 8, std 2^-25      (lvl1param)
 *   lvl10 : identity key switching lvl1 -> lvl0, basebit = 2, t = 7 (lvl10param)
 *   mu    : 1/8 on both levels (lvl0param::mu, lvl1param::mu = 2^29)
 *   lvl2  : GLWE k = 1, N = 2048, l = 4, Bgbit = 10, Torus64, std 2^-44
 *   lvl20 : lvl2 -> lvl0 key switching, basebit = 2, t = 7 (TFHEpp constants
 *           are absent from the reference tree; this choice is recorded here)
 *
 * Layouts follow TFHEpp as the reference kernels read them:
 *   TLWE<P>    T[k*n + 1], b last          (include/keyswitch_gpu.cuh:82-83)
 *   TRLWE<P>   T[k+1][N], b = poly k       (include/gatebootstrapping_gpu.cuh:43-49)
 *   TRGSW<P>   TRLWE[(k+1)*l], row = j*l+d (include/gatebootstrapping_gpu.cuh:166-167)
 *   BK (no KB) TRGSW[n0]                   (src/bootstrap_gpu.cu:233-235)
 *   BK (KB=2)  TRGSW[n0/2][3]              (src/bootstrap_gpu.cu:284-290)
 *   KSK lvl10  TLWE<lvl0>[N][t][2^(basebit-1)] (include/keyswitch_gpu.cuh:106-113)
 */
#pragma once
#include <stdint.h>

#define CUFHE_LVL0_N 636u
#define CUFHE_LVL0_ALPHA 9.25e-5

#define CUFHE_LVL1_NBIT 10u
#define CUFHE_LVL1_N 1024u
#define CUFHE_LVL1_K 1u
#define CUFHE_LVL1_L 2u
#define CUFHE_LVL1_BGBIT 8u
#define CUFHE_LVL1_ALPHA 2.98023223876953125e-08 /* 2^-25 */

#define CUFHE_LVL10_BASEBIT 2u
#define CUFHE_LVL10_T 7u

#define CUFHE_MU32 (1u << 29) /* 1/8 in Torus32 */

#define CUFHE_LVL2_NBIT 11u
#define CUFHE_LVL2_N 2048u
#define CUFHE_LVL2_L 4u
#define CUFHE_LVL2_BGBIT 10u
#define CUFHE_LVL2_ALPHA 5.684341886080801486968994140625e-14 /* 2^-44 */
#define CUFHE_MU64 (1ull << 61)
#define CUFHE_LVL20_BASEBIT 2u
#define CUFHE_LVL20_T 7u

/* derived sizes (words) */
#define CUFHE_TLWE0_WORDS (CUFHE_LVL0_N + 1u)                 /* 637  */
#define CUFHE_TLWE1_WORDS (CUFHE_LVL1_K * CUFHE_LVL1_N + 1u)  /* 1025 */
#define CUFHE_TRLWE1_WORDS ((CUFHE_LVL1_K + 1u) * CUFHE_LVL1_N) /* 2048 */
#define CUFHE_TRGSW1_ROWS ((CUFHE_LVL1_K + 1u) * CUFHE_LVL1_L) /* 4 */
#define CUFHE_TRGSW1_WORDS (CUFHE_TRGSW1_ROWS * CUFHE_TRLWE1_WORDS) /* 8192 */
#define CUFHE_BK1_WORDS ((uint64_t)CUFHE_LVL0_N * CUFHE_TRGSW1_WORDS)
#define CUFHE_BKKB1_WORDS ((uint64_t)(CUFHE_LVL0_N / 2u) * 3u * CUFHE_TRGSW1_WORDS)
#define CUFHE_KSK10_WORDS                                                  \
    ((uint64_t)CUFHE_LVL1_N * CUFHE_LVL10_T * (1u << (CUFHE_LVL10_BASEBIT - 1u)) * \
     CUFHE_TLWE0_WORDS)

/* lvl0 -> lvl2 path (uint64 words for lvl2 objects) */
#define CUFHE_TLWE2_WORDS (CUFHE_LVL2_N + 1u)                  /* 2049 */
#define CUFHE_TRLWE2_WORDS (2u * CUFHE_LVL2_N)                  /* 4096 */
#define CUFHE_TRGSW2_ROWS (2u * CUFHE_LVL2_L)                   /* 8 */
#define CUFHE_TRGSW2_WORDS (CUFHE_TRGSW2_ROWS * CUFHE_TRLWE2_WORDS) /* 32768 */
#define CUFHE_BK2_WORDS ((uint64_t)CUFHE_LVL0_N * CUFHE_TRGSW2_WORDS)
#define CUFHE_BKKB2_WORDS ((uint64_t)(CUFHE_LVL0_N / 2u) * 3u * CUFHE_TRGSW2_WORDS)
#define CUFHE_KSK20_WORDS                                                  \
    ((uint64_t)CUFHE_LVL2_N * CUFHE_LVL20_T * (1u << (CUFHE_LVL20_BASEBIT - 1u)) * \
     CUFHE_TLWE0_WORDS)
