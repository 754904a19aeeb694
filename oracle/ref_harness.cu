// ref_harness.cu -- C-ABI shim around the UNMODIFIED reference (SysuCrypto/cuMAYO)
// compiled from its own sources for sm_100a (see oracle/Makefile, target `ref`).
//
// TEST INFRASTRUCTURE ONLY: used to generate golden vectors on a B200 and as the
// timed reference arm of bench.py.  Each wrapper forwards to the reference's own
// public entry point of the same name (include/api.cuh:9-47) unchanged.
#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>

#include "api.cuh"
#include "aes128_ctr.cuh"
#include "params.h"

#define S(x) reinterpret_cast<cudaStream_t>(x)

extern "C" {

int ref_version() { return MAYO_VERSION; }

// n, m, o, k, sk, pk, p, o_bytes, p1, p2, digest, pairs
void ref_params(long *p) {
    const long v[] = {MAYO_N, MAYO_M, MAYO_O, MAYO_K, MAYO_SK_BYTES, MAYO_PK_BYTES, MAYO_P_BYTES,
                      MAYO_O_BYTES, MAYO_P1_BYTES, MAYO_P2_BYTES, MAYO_DIGEST_BYTES, MAYO_Pair};
    for (int i = 0; i < 12; i++) p[i] = v[i];
}

// include/aes128_ctr.cuh:16 -- must run once per process before any launch.
void ref_init() { aes128_tables_init(); }

int ref_sync() { return (int)cudaDeviceSynchronize(); }
int ref_last_error() { return (int)cudaGetLastError(); }

void ref_keypair(uint8_t *pool, size_t pitch, size_t batch, void *st, size_t rand_index) {
    crypto_sign_keypair(pool, pitch, batch, S(st), rand_index);
}
void ref_keypair_DtH(uint8_t *pk, uint8_t *sk, uint8_t *pool, size_t pitch, size_t batch, void *st) {
    crypto_sign_keypair_DtH(pk, sk, pool, pitch, batch, S(st));
}
void ref_expandsk_HtD(uint8_t *csk, uint8_t *pool, size_t pitch, size_t batch, void *st) {
    crypto_sign_expandsk_HtD(csk, pool, pitch, batch, S(st));
}
void ref_expandsk(uint8_t *pool, size_t pitch, size_t batch, void *st) {
    crypto_sign_expandsk(pool, pitch, batch, S(st));
}
void ref_expandsk_DtH(uint8_t *esk, uint8_t *pool, size_t pitch, size_t batch, void *st) {
    crypto_sign_expandsk_DtH(esk, pool, pitch, batch, S(st));
}
void ref_expandpk_HtD(uint8_t *cpk, uint8_t *pool, size_t pitch, size_t batch, void *st) {
    crypto_sign_expandpk_HtD(cpk, pool, pitch, batch, S(st));
}
void ref_expandpk(uint8_t *pool, size_t pitch, size_t batch, void *st) {
    crypto_sign_expandpk(pool, pitch, batch, S(st));
}
void ref_expandpk_DtH(uint8_t *epk, uint8_t *pool, size_t pitch, size_t batch, void *st) {
    crypto_sign_expandpk_DtH(epk, pool, pitch, batch, S(st));
}
void ref_sign_HtD(uint8_t *esk, uint8_t *msg, size_t mlen, uint8_t *pool, size_t pitch, size_t batch,
                  void *st) {
    crypto_sign_sign_HtD(esk, msg, mlen, pool, pitch, batch, S(st));
}
void ref_sign(uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *st) {
    crypto_sign_sign(pool, mlen, pitch, batch, S(st));
}
void ref_sign_DtH(uint8_t *sig, uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *st) {
    crypto_sign_sign_DtH(sig, pool, mlen, pitch, batch, S(st));
}
void ref_signWithesk_HtD(uint8_t *csk, uint8_t *msg, size_t mlen, uint8_t *pool, size_t pitch,
                         size_t batch, void *st) {
    crypto_sign_signWithesk_HtD(csk, msg, mlen, pool, pitch, batch, S(st));
}
void ref_signWithesk(uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *st) {
    crypto_sign_signWithesk(pool, mlen, pitch, batch, S(st));
}
void ref_signWithesk_DtH(uint8_t *sig, uint8_t *pool, size_t mlen, size_t pitch, size_t batch,
                         void *st) {
    crypto_sign_signWithesk_DtH(sig, pool, mlen, pitch, batch, S(st));
}
void ref_verify_HtD(uint8_t *epk, uint8_t *msg, uint8_t *sig, size_t mlen, uint8_t *pool, size_t pitch,
                    size_t batch, void *st) {
    crypto_sign_verify_HtD(epk, msg, sig, mlen, pool, pitch, batch, S(st));
}
void ref_verify(uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *st) {
    crypto_sign_verify(pool, mlen, pitch, batch, S(st));
}
void ref_verify_DtH(uint8_t *res, size_t mlen, uint8_t *pool, size_t pitch, size_t batch, void *st) {
    crypto_sign_verify_DtH(res, mlen, pool, pitch, batch, S(st));
}
void ref_verifyWithepk_HtD(uint8_t *cpk, uint8_t *msg, uint8_t *sig, size_t mlen, uint8_t *pool,
                           size_t pitch, size_t batch, void *st) {
    crypto_sign_verifyWithepk_HtD(cpk, msg, sig, mlen, pool, pitch, batch, S(st));
}
void ref_verifyWithepk(uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *st) {
    crypto_sign_verifyWithepk(pool, mlen, pitch, batch, S(st));
}
void ref_verifyWithepk_DtH(uint8_t *res, size_t mlen, uint8_t *pool, size_t pitch, size_t batch,
                           void *st) {
    crypto_sign_verifyWithepk_DtH(res, mlen, pool, pitch, batch, S(st));
}

}  // extern "C"
