/*
 * tfhe_client.h -- CPU client library (libcufhe_client.so): seeded key
 * generation, encryption and decryption in the TFHEpp layouts the engine
 * consumes.  Stands in for the TFHEpp calls the reference's users make
 * (TFHEpp::SecretKey, EvalKey::emplacebk / emplaceiksk, tlweSymEncrypt,
 * tlweSymDecrypt; test/test_gate_gpu.cc:50-58, test/test_util.h:20-27).
 * Keys are int32 arrays of 0/1; randomness is derived from (seed, stream).
 */
#ifndef TFHE_CLIENT_H
#define TFHE_CLIENT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

void tfhe_keygen_binary(uint64_t seed, uint64_t stream, uint32_t n, int32_t* key);
void tfhe_tlwe32_encrypt(uint64_t seed, uint64_t stream, const int32_t* key, uint32_t n,
                         uint32_t msg, double alpha, uint32_t* out);
void tfhe_tlwe32_encrypt_bits(uint64_t seed, uint64_t stream0, const int32_t* key, uint32_t n,
                              const uint8_t* bits, uint64_t count, uint32_t mu, double alpha,
                              uint32_t* out);
uint32_t tfhe_tlwe32_phase(const int32_t* key, uint32_t n, const uint32_t* c);
void tfhe_tlwe32_phase_batch(const int32_t* key, uint32_t n, const uint32_t* c, uint64_t count,
                             uint32_t* phase);
void tfhe_tlwe32_decrypt_bits(const int32_t* key, uint32_t n, const uint32_t* c, uint64_t count,
                              uint8_t* bits);
void tfhe_trlwe32_encrypt(uint64_t seed, uint64_t stream, const int32_t* key, uint32_t N,
                          const uint32_t* msg, double alpha, uint32_t* out);
void tfhe_trlwe32_phase(const int32_t* key, uint32_t N, const uint32_t* c, uint32_t* phase);
void tfhe_trgsw32_encrypt(uint64_t seed, uint64_t stream, const int32_t* key, uint32_t N,
                          uint32_t l, uint32_t bgbit, int32_t m, double alpha, uint32_t* out);
/* bootstrapping key: kb = 0 -> TRGSW[n0], kb = 1 -> TRGSW[n0/2][3] */
void tfhe_bk32_gen(uint64_t seed, const int32_t* key0, uint32_t n0, const int32_t* key1,
                   uint32_t N, uint32_t l, uint32_t bgbit, double alpha, int kb, uint32_t* out);
/* key-switching key TLWE<lvl0>[n_src][t][2^(basebit-1)] */
void tfhe_ksk32_gen(uint64_t seed, const int32_t* key_src, uint32_t n_src, const int32_t* key0,
                    uint32_t n0, uint32_t basebit, uint32_t t, double alpha, uint32_t* out);
/* lvl0 -> lvl2 bootstrapping key (Torus64 TRGSW<lvl2>, N = 2048, l = 4,
 * Bgbit = 10): kb = 0 -> TRGSW[n0], kb = 1 -> TRGSW[n0/2][3]; the lvl2 -> lvl0
 * key-switching key is tfhe_ksk32_gen with the lvl2 key as key_src. */
void tfhe_bk64_gen(uint64_t seed, const int32_t* key0, uint32_t n0, const int32_t* key2,
                   uint32_t N, uint32_t l, uint32_t bgbit, double alpha, int kb, uint64_t* out);
void tfhe_trlwe64_phase(const int32_t* key, uint32_t N, const uint64_t* c, uint64_t* phase);
uint64_t tfhe_tlwe64_phase(const int32_t* key, uint32_t n, const uint64_t* c);

#ifdef __cplusplus
}
#endif

#endif /* TFHE_CLIENT_H */
