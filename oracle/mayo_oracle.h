/*
 * mayo_oracle.h -- CPU restatement of SysuCrypto/cuMAYO's batched MAYO path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker for the CUDA
 * engine in cumayo_b200/ and the timed CPU baseline ("port") in bench.py.
 * Nothing in the product path links, loads or calls it.
 *
 * Every routine restates the reference's algorithm (file:line cited at each
 * function) with plain byte/nibble loops.  Parity of this restatement with
 * the reference is pinned by golden vectors produced by the reference's own
 * CUDA build (tests/golden/), by hashlib (SHAKE) and by the `cryptography`
 * package (AES-128-CTR).
 */
#ifndef MAYO_ORACLE_H
#define MAYO_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Parameter set, mirrors include/params.h:10-92 of the reference. */
typedef struct {
    int id;            /* 1, 2, 3, 5 */
    int n, m, o, k;
    int v;             /* n - o; equals m in every set */
    int menc;          /* m / 2: bytes per m-vector */
    int sk_bytes, pk_bytes, p_bytes, o_bytes, p1_bytes, p2_bytes;
    int digest_bytes, pairs;
    uint8_t poly_c[4]; /* f(z) = z^m + c3 z^3 + c2 z^2 + c1 z + c0 */
    int sig_bytes;     /* k*n/2 + sk_bytes */
    int esk_bytes;     /* sk + o_bytes + p_bytes */
    int epk_bytes;     /* p_bytes + pk_bytes - 16 */
} mayo_oracle_params;

/* Returns NULL for an unknown set id. */
const mayo_oracle_params *mayo_oracle_get_params(int set_id);

/* ---- primitives ---- */
void mayo_oracle_shake128(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen);
void mayo_oracle_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen);
/* AES-128 in counter mode; 16-byte counter block = 0^8 || BE64(i), i = 0,1,.. */
void mayo_oracle_aes128_ctr(const uint8_t key[16], uint8_t *out, size_t outlen);
uint8_t mayo_oracle_gf16_mul(uint8_t a, uint8_t b);
uint8_t mayo_oracle_gf16_inv(uint8_t a);
/* SHA-256 of the AES S-box and of the GF(16) multiplication table as used by
 * the oracle (lets a test compare them to digests of the reference's tables). */
void mayo_oracle_table_digest(uint8_t sbox_sha[32], uint8_t gf16_sha[32]);

/* ---- MAYO operations (single instance) ---- */
/* Keypair of instance `index` in a call started at `rand_index`:
 * seed_sk = SHAKE128(LE64(rand_index + 2*index + 1)).  sk: sk_bytes; pk: pk_bytes. */
int mayo_oracle_keypair(int set_id, uint64_t rand_index, uint64_t index, uint8_t *sk, uint8_t *pk);
/* Keypair from a caller-provided seed_sk (sk_bytes). */
int mayo_oracle_keypair_from_seed(int set_id, const uint8_t *seed_sk, uint8_t *pk);
/* esk = seed_sk || O || P1 || L (esk_bytes). */
int mayo_oracle_expandsk(int set_id, const uint8_t *csk, uint8_t *esk);
/* epk = P1 || P2 || P3 (epk_bytes). */
int mayo_oracle_expandpk(int set_id, const uint8_t *cpk, uint8_t *epk);
/* Signature of msg under esk.  Returns the number of attempts used (1..255),
 * or 0 when every attempt was rejected (the reference then still emits the
 * last attempt's signature, and so does the oracle).
 * force_reject: the first `force_reject` attempts are treated as rejected
 * (test hook, 0 in normal use). */
int mayo_oracle_sign(int set_id, const uint8_t *esk, const uint8_t *msg, size_t mlen,
                     uint8_t *sig, int force_reject);
/* 0 = accept, 1 = reject (reference src/verify.cu:203-211). */
int mayo_oracle_verify(int set_id, const uint8_t *epk, const uint8_t *msg, size_t mlen,
                       const uint8_t *sig);

/* ---- batched helpers for the CPU baseline (OpenMP, one instance per thread) ---- */
int mayo_oracle_max_threads(void);
void mayo_oracle_set_threads(int nthreads);
void mayo_oracle_keypair_batch(int set_id, uint64_t rand_index, size_t batch,
                               uint8_t *sk, uint8_t *pk);
void mayo_oracle_keypair_from_seed_batch(int set_id, size_t batch, const uint8_t *seeds,
                                         uint8_t *pk);
void mayo_oracle_expandsk_batch(int set_id, size_t batch, const uint8_t *csk, uint8_t *esk);
void mayo_oracle_expandpk_batch(int set_id, size_t batch, const uint8_t *cpk, uint8_t *epk);
/* Messages: msg + msg_off[i], length msg_len[i].  esk_stride 0 = one shared key. */
void mayo_oracle_sign_batch(int set_id, size_t batch, const uint8_t *esk, size_t esk_stride,
                            const uint8_t *msg, const uint64_t *msg_off, const uint32_t *msg_len,
                            uint8_t *sig, int32_t *attempts);
void mayo_oracle_verify_batch(int set_id, size_t batch, const uint8_t *epk, size_t epk_stride,
                              const uint8_t *msg, const uint64_t *msg_off, const uint32_t *msg_len,
                              const uint8_t *sig, uint8_t *result);

#ifdef __cplusplus
}
#endif
#endif
