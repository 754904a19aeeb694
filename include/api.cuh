// api.cuh -- drop-in replacement for SysuCrypto/cuMAYO's include/api.cuh.
//
// Same names, signatures, default arguments and void returns as the reference's 20 entry
// points (include/api.cuh:9-47 of the reference), plus aes128_tables_init()
// (include/aes128_ctr.cuh:16).  The parameter set is chosen at compile time with
// -DMAYO_VERSION={1,2,3,5}, as in the reference; each wrapper forwards to the C-ABI of
// libmayo_b200.so (mayo_b200.h) with that set.  Link with -lmayo_b200.
//
// Unlike the reference, failures are not silent: the status of the last call made through
// these wrappers on the calling thread is available from mayo_api_last_status().
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "mayo_b200.h"

#ifndef MAYO_VERSION
#error "MAYO_VERSION =1,2,3,5"
#endif

namespace mayo_api_detail {
inline int &last_status() {
    static thread_local int s = MAYO_B200_OK;
    return s;
}
inline void note(int s) { last_status() = s; }
}  // namespace mayo_api_detail

inline int mayo_api_last_status() { return mayo_api_detail::last_status(); }

inline void aes128_tables_init() { mayo_api_detail::note(mayo_b200_init()); }

inline void crypto_sign_keypair(uint8_t *d_keypair_mem_pool, size_t keypair_mem_pool_pitch, size_t batch_size = 1,
                                cudaStream_t stream = nullptr, size_t rand_index = 0) {
    mayo_api_detail::note(
        mayo_b200_keypair(MAYO_VERSION, d_keypair_mem_pool, keypair_mem_pool_pitch, batch_size, stream, rand_index));
}
inline void crypto_sign_keypair_DtH(uint8_t *pk, uint8_t *sk, uint8_t *d_keypair_mem_pool, size_t pitch,
                                    size_t batch_size, cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_keypair_DtH(MAYO_VERSION, pk, sk, d_keypair_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_expandsk_HtD(uint8_t *csk, uint8_t *d_expandsk_mem_pool, size_t pitch, size_t batch_size,
                                     cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_expandsk_HtD(MAYO_VERSION, csk, d_expandsk_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_expandsk(uint8_t *d_expandsk_mem_pool, size_t pitch, size_t batch_size,
                                 cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_expandsk(MAYO_VERSION, d_expandsk_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_expandsk_DtH(uint8_t *esk, uint8_t *d_expandsk_mem_pool, size_t pitch, size_t batch_size,
                                     cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_expandsk_DtH(MAYO_VERSION, esk, d_expandsk_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_expandpk_HtD(uint8_t *cpk, uint8_t *d_expandpk_mem_pool, size_t pitch, size_t batch_size,
                                     cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_expandpk_HtD(MAYO_VERSION, cpk, d_expandpk_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_expandpk(uint8_t *d_expandpk_mem_pool, size_t pitch, size_t batch_size,
                                 cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_expandpk(MAYO_VERSION, d_expandpk_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_expandpk_DtH(uint8_t *epk, uint8_t *d_expandpk_mem_pool, size_t pitch, size_t batch_size,
                                     cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_expandpk_DtH(MAYO_VERSION, epk, d_expandpk_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_sign_HtD(uint8_t *cesk, uint8_t *cMess, size_t mlen, uint8_t *d_sign_mem_pool, size_t pitch,
                                 size_t batch_size, cudaStream_t stream = nullptr) {
    mayo_api_detail::note(
        mayo_b200_sign_HtD(MAYO_VERSION, cesk, cMess, mlen, d_sign_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_sign(uint8_t *d_sign_mem_pool, size_t Mlen, size_t pitch, size_t batch_size,
                             cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_sign(MAYO_VERSION, d_sign_mem_pool, Mlen, pitch, batch_size, stream));
}
inline void crypto_sign_sign_DtH(uint8_t *sig, uint8_t *d_sig_mem_pool, size_t Mlen, size_t pitch, size_t batch_size,
                                 cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_sign_DtH(MAYO_VERSION, sig, d_sig_mem_pool, Mlen, pitch, batch_size, stream));
}
inline void crypto_sign_signWithesk_HtD(uint8_t *cesk, uint8_t *cMess, size_t mlen, uint8_t *d_sign_mem_pool,
                                        size_t pitch, size_t batch_size, cudaStream_t stream = nullptr) {
    mayo_api_detail::note(
        mayo_b200_signWithesk_HtD(MAYO_VERSION, cesk, cMess, mlen, d_sign_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_signWithesk(uint8_t *d_sign_mem_pool, size_t Mlen, size_t pitch, size_t batch_size,
                                    cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_signWithesk(MAYO_VERSION, d_sign_mem_pool, Mlen, pitch, batch_size, stream));
}
inline void crypto_sign_signWithesk_DtH(uint8_t *sig, uint8_t *d_sig_mem_pool, size_t Mlen, size_t pitch,
                                        size_t batch_size, cudaStream_t stream = nullptr) {
    mayo_api_detail::note(
        mayo_b200_signWithesk_DtH(MAYO_VERSION, sig, d_sig_mem_pool, Mlen, pitch, batch_size, stream));
}
inline void crypto_sign_verify_HtD(uint8_t *epk, uint8_t *Mess, uint8_t *sig, size_t mlen,
                                   uint8_t *d_verify_mem_pool, size_t pitch, size_t batch_size,
                                   cudaStream_t stream = nullptr) {
    mayo_api_detail::note(
        mayo_b200_verify_HtD(MAYO_VERSION, epk, Mess, sig, mlen, d_verify_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_verify(uint8_t *d_verify_mem_pool, size_t Mlen, size_t pitch, size_t batch_size,
                               cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_verify(MAYO_VERSION, d_verify_mem_pool, Mlen, pitch, batch_size, stream));
}
inline void crypto_sign_verify_DtH(uint8_t *verify, size_t Mlen, uint8_t *d_verify_mem_pool, size_t pitch,
                                   size_t batch_size, cudaStream_t stream = nullptr) {
    mayo_api_detail::note(
        mayo_b200_verify_DtH(MAYO_VERSION, verify, Mlen, d_verify_mem_pool, pitch, batch_size, stream));
}
inline void crypto_sign_verifyWithepk_HtD(uint8_t *epk, uint8_t *Mess, uint8_t *sig, size_t mlen,
                                          uint8_t *d_verify_mem_pool, size_t pitch, size_t batch_size,
                                          cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_verifyWithepk_HtD(MAYO_VERSION, epk, Mess, sig, mlen, d_verify_mem_pool, pitch,
                                                      batch_size, stream));
}
inline void crypto_sign_verifyWithepk(uint8_t *d_verify_mem_pool, size_t Mlen, size_t pitch, size_t batch_size,
                                      cudaStream_t stream = nullptr) {
    mayo_api_detail::note(mayo_b200_verifyWithepk(MAYO_VERSION, d_verify_mem_pool, Mlen, pitch, batch_size, stream));
}
inline void crypto_sign_verifyWithepk_DtH(uint8_t *verify, size_t Mlen, uint8_t *d_verify_mem_pool, size_t pitch,
                                          size_t batch_size, cudaStream_t stream = nullptr) {
    mayo_api_detail::note(
        mayo_b200_verifyWithepk_DtH(MAYO_VERSION, verify, Mlen, d_verify_mem_pool, pitch, batch_size, stream));
}
