// capi.cu -- the C-ABI of libmayo_b200.so (declared in include/mayo_b200.h).
//
// Pool-offset arithmetic and host<->device copies mirror the reference's src/api.cu
// function by function (cited below); the kernels behind them are this project's.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/mayo_b200.h"
#include "common.cuh"
#include "ops.h"

namespace mayo {

thread_local int g_last_cuda_error = 0;

int api_cuda_rc(cudaError_t e) {
    if (e == cudaSuccess) return MAYO_B200_OK;
    g_last_cuda_error = (int)e;
    return MAYO_B200_ERR_CUDA;
}

int api_launch_rc(int rc) {
    // cudaGetLastError also clears the error a failed launch left, so the next call's
    // cudaPeekAtLastError reports only its own launches
    if (rc == ST_CUDA) g_last_cuda_error = (int)cudaGetLastError();
    return rc;
}

thread_local Inject tl_inject;
Inject &inject() { return tl_inject; }

}  // namespace mayo

namespace {

using namespace mayo;


struct Sz {
    size_t sk, pk, sig, esk, epk, p, o_bytes, scratch;
    int n, m, o, k, digest;
};

bool sizes_of(int set, Sz &z) {
    switch (set) {
#define FILL(ID)                                                                                        \
    case ID: {                                                                                          \
        using S = Set<ID>;                                                                              \
        z = Sz{S::sk, S::pk, S::sig, S::esk, S::epk, S::p, S::o_bytes, S::scratch, S::n, S::m, S::o, S::k, \
               S::digest};                                                                              \
        return true;                                                                                    \
    }
        FILL(1) FILL(2) FILL(3) FILL(5)
#undef FILL
        default: return false;
    }
}

inline size_t A(size_t x) { return align128z(x); }
inline cudaStream_t S_(void *s) { return reinterpret_cast<cudaStream_t>(s); }

int cuda_rc(cudaError_t e) { return mayo::api_cuda_rc(e); }
int kernel_rc(int rc) { return mayo::api_launch_rc(rc); }

// Row sizes of each reference entry point (tests/bench_stream.cu:25-31, 82, 133 of the reference).
size_t row_keypair(const Sz &z) { return A(z.sk) + A(z.pk) + A(z.p); }
size_t row_sign(const Sz &z, size_t mlen) { return z.esk + mlen + z.sig + z.scratch; }
size_t row_sign_wesk(const Sz &z, size_t mlen) { return A(z.esk) + A(mlen) + A(z.sig) + z.scratch; }
size_t row_verify(const Sz &z, size_t mlen) { return A(z.epk) + A(mlen) + A(z.sig) + 1; }

// Common argument checks: set known, pool present, pitch large enough to step rows.
int check(const void *pool, size_t pitch, size_t batch, size_t row, size_t mlen = 0) {
    if (batch == 0) return MAYO_B200_OK;
    if (!pool) return MAYO_B200_ERR_ARG;
    if (batch > 0x7fffffffu || mlen > 0x7fffffffu) return MAYO_B200_ERR_ARG;
    if (batch > 1 && pitch < row) return MAYO_B200_ERR_ARG;
    return MAYO_B200_OK;
}

int copy2d(void *dst, size_t dpitch, const void *src, size_t spitch, size_t width, size_t batch, cudaMemcpyKind kind,
           void *stream) {
    if (batch == 0 || width == 0) return MAYO_B200_OK;
    if (!dst || !src) return MAYO_B200_ERR_ARG;
    return cuda_rc(cudaMemcpy2DAsync(dst, dpitch, src, spitch, width, batch, kind, S_(stream)));
}

}  // namespace

extern "C" {

MAYO_B200_API int mayo_b200_abi_version(void) { return MAYO_B200_ABI_VERSION; }

MAYO_B200_API int mayo_b200_get_sizes(int set, size_t mlen_hint, mayo_b200_sizes *out) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    if (!out) return MAYO_B200_ERR_ARG;
    out->set = set;
    out->n = z.n;
    out->m = z.m;
    out->o = z.o;
    out->k = z.k;
    out->digest_bytes = z.digest;
    out->sk_bytes = z.sk;
    out->pk_bytes = z.pk;
    out->sig_bytes = z.sig;
    out->esk_bytes = z.esk;
    out->epk_bytes = z.epk;
    out->p_bytes = z.p;
    out->scratch_bytes = z.scratch;
    out->pitch_keypair = row_keypair(z);
    out->pitch_expandsk = z.esk;
    out->pitch_expandpk = z.epk;
    out->pitch_sign = row_sign(z, mlen_hint);
    out->pitch_sign_with_esk = row_sign_wesk(z, mlen_hint);
    out->pitch_verify = row_verify(z, mlen_hint);
    return MAYO_B200_OK;
}

MAYO_B200_API int mayo_b200_init(void) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return cuda_rc(cudaGetLastError());
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, dev);
    if (e != cudaSuccess) return cuda_rc(e);
    if (prop.major != 10) return MAYO_B200_ERR_CUDA;
    return MAYO_B200_OK;
}

MAYO_B200_API const char *mayo_b200_status_string(int status) {
    switch (status) {
        case MAYO_B200_OK: return "ok";
        case MAYO_B200_ERR_SET: return "unknown MAYO parameter set (expected 1, 2, 3 or 5)";
        case MAYO_B200_ERR_ARG: return "invalid argument (null pointer, pitch too small or size out of range)";
        case MAYO_B200_ERR_CUDA: return "CUDA error (see mayo_b200_last_cuda_error)";
        case MAYO_B200_ERR_TOO_LARGE: return "batch exceeds the fixed workspace of mayo_b200_sign_many_noalloc";
        default: return "unknown status";
    }
}

MAYO_B200_API int mayo_b200_last_cuda_error(void) { return mayo::g_last_cuda_error; }

MAYO_B200_API int mayo_b200_test_inject(int kind, uint32_t arg, uint32_t spin) {
    if (kind < MAYO_B200_INJECT_NONE || kind > MAYO_B200_INJECT_PRODUCT_STALL) return MAYO_B200_ERR_ARG;
    mayo::inject() = mayo::Inject{kind, arg, spin};
    return MAYO_B200_OK;
}

// ---- keypair (src/api.cu:17-38) ----
MAYO_B200_API int mayo_b200_keypair(int set, uint8_t *pool, size_t pitch, size_t batch, void *stream,
                                    size_t rand_index) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, row_keypair(z));
    if (rc || !batch) return rc;
    return kernel_rc(launch_keypair(set, pool, pitch, batch, S_(stream), rand_index));
}
MAYO_B200_API int mayo_b200_keypair_from_seed(int set, uint8_t *pool, size_t pitch, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, row_keypair(z));
    if (rc || !batch) return rc;
    return kernel_rc(launch_keypair_seeded(set, pool, pitch, batch, S_(stream)));
}
MAYO_B200_API int mayo_b200_keypair_DtH(int set, uint8_t *pk, uint8_t *sk, const uint8_t *pool, size_t pitch,
                                        size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, A(z.sk) + z.pk);
    if (rc || !batch) return rc;
    rc = copy2d(pk, z.pk, pool + A(z.sk), pitch, z.pk, batch, cudaMemcpyDeviceToHost, stream);
    if (rc) return rc;
    return copy2d(sk, z.sk, pool, pitch, z.sk, batch, cudaMemcpyDeviceToHost, stream);
}

// ---- expand-sk (src/api.cu:40-62) ----
MAYO_B200_API int mayo_b200_expandsk_HtD(int set, const uint8_t *csk, uint8_t *pool, size_t pitch, size_t batch,
                                         void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, z.sk);
    if (rc || !batch) return rc;
    return copy2d(pool, pitch, csk, z.sk, z.sk, batch, cudaMemcpyHostToDevice, stream);
}
MAYO_B200_API int mayo_b200_expandsk(int set, uint8_t *pool, size_t pitch, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, z.esk);
    if (rc || !batch) return rc;
    return kernel_rc(launch_expandsk(set, pool, pitch, batch, S_(stream)));
}
MAYO_B200_API int mayo_b200_expandsk_DtH(int set, uint8_t *esk, const uint8_t *pool, size_t pitch, size_t batch,
                                         void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, z.esk);
    if (rc || !batch) return rc;
    return copy2d(esk, z.esk, pool, pitch, z.esk, batch, cudaMemcpyDeviceToHost, stream);
}

// ---- expand-pk (src/api.cu:64-85) ----
MAYO_B200_API int mayo_b200_expandpk_HtD(int set, const uint8_t *cpk, uint8_t *pool, size_t pitch, size_t batch,
                                         void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, z.epk);
    if (rc || !batch) return rc;
    return copy2d(pool + z.p - 16, pitch, cpk, z.pk, z.pk, batch, cudaMemcpyHostToDevice, stream);
}
MAYO_B200_API int mayo_b200_expandpk(int set, uint8_t *pool, size_t pitch, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, z.epk);
    if (rc || !batch) return rc;
    return kernel_rc(launch_expandpk(set, pool, pitch, batch, S_(stream)));
}
MAYO_B200_API int mayo_b200_expandpk_DtH(int set, uint8_t *epk, const uint8_t *pool, size_t pitch, size_t batch,
                                         void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, z.epk);
    if (rc || !batch) return rc;
    return copy2d(epk, z.epk, pool, pitch, z.epk, batch, cudaMemcpyDeviceToHost, stream);
}

// ---- sign on an expanded key (src/api.cu:88-114) ----
MAYO_B200_API int mayo_b200_sign_HtD(int set, const uint8_t *esk, const uint8_t *msg, size_t mlen, uint8_t *pool,
                                     size_t pitch, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, z.esk + mlen, mlen);
    if (rc || !batch) return rc;
    rc = copy2d(pool, pitch, esk, z.esk, z.esk, batch, cudaMemcpyHostToDevice, stream);
    if (rc) return rc;
    return copy2d(pool + z.esk, pitch, msg, mlen, mlen, batch, cudaMemcpyHostToDevice, stream);
}
MAYO_B200_API int mayo_b200_sign(int set, uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, row_sign(z, mlen), mlen);
    if (rc || !batch) return rc;
    const size_t msg_off = z.esk, sig_off = msg_off + mlen, scratch_off = sig_off + z.sig;
    return kernel_rc(launch_sign(set, pool, pitch, batch, S_(stream), mlen, msg_off, sig_off, scratch_off));
}
MAYO_B200_API int mayo_b200_sign_DtH(int set, uint8_t *sig, const uint8_t *pool, size_t mlen, size_t pitch,
                                     size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, z.esk + mlen + z.sig, mlen);
    if (rc || !batch) return rc;
    return copy2d(sig, z.sig, pool + z.esk + mlen, pitch, z.sig, batch, cudaMemcpyDeviceToHost, stream);
}

// ---- sign from a compact key (src/api.cu:116-144) ----
MAYO_B200_API int mayo_b200_signWithesk_HtD(int set, const uint8_t *csk, const uint8_t *msg, size_t mlen,
                                            uint8_t *pool, size_t pitch, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, A(z.esk) + mlen, mlen);
    if (rc || !batch) return rc;
    rc = copy2d(pool, pitch, csk, z.sk, z.sk, batch, cudaMemcpyHostToDevice, stream);
    if (rc) return rc;
    return copy2d(pool + A(z.esk), pitch, msg, mlen, mlen, batch, cudaMemcpyHostToDevice, stream);
}
MAYO_B200_API int mayo_b200_signWithesk(int set, uint8_t *pool, size_t mlen, size_t pitch, size_t batch,
                                        void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, row_sign_wesk(z, mlen), mlen);
    if (rc || !batch) return rc;
    rc = kernel_rc(launch_expandsk(set, pool, pitch, batch, S_(stream)));
    if (rc) return rc;
    const size_t msg_off = A(z.esk), sig_off = msg_off + A(mlen), scratch_off = sig_off + A(z.sig);
    return kernel_rc(launch_sign(set, pool, pitch, batch, S_(stream), mlen, msg_off, sig_off, scratch_off));
}
MAYO_B200_API int mayo_b200_signWithesk_DtH(int set, uint8_t *sig, const uint8_t *pool, size_t mlen, size_t pitch,
                                            size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, A(z.esk) + A(mlen) + z.sig, mlen);
    if (rc || !batch) return rc;
    return copy2d(sig, z.sig, pool + A(z.esk) + A(mlen), pitch, z.sig, batch, cudaMemcpyDeviceToHost, stream);
}

// ---- verify on an expanded key (src/api.cu:146-178) ----
MAYO_B200_API int mayo_b200_verify_HtD(int set, const uint8_t *epk, const uint8_t *msg, const uint8_t *sig,
                                       size_t mlen, uint8_t *pool, size_t pitch, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, A(z.epk) + A(mlen) + A(z.sig), mlen);
    if (rc || !batch) return rc;
    const size_t epklen = A(z.epk), siglen = A(z.sig);
    rc = copy2d(pool, pitch, epk, epklen, epklen, batch, cudaMemcpyHostToDevice, stream);
    if (rc) return rc;
    rc = copy2d(pool + epklen, pitch, msg, mlen, mlen, batch, cudaMemcpyHostToDevice, stream);
    if (rc) return rc;
    return copy2d(pool + epklen + A(mlen), pitch, sig, siglen, siglen, batch, cudaMemcpyHostToDevice, stream);
}
MAYO_B200_API int mayo_b200_verify(int set, uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, row_verify(z, mlen), mlen);
    if (rc || !batch) return rc;
    const size_t msg_off = A(z.epk), sig_off = msg_off + A(mlen), res_off = sig_off + A(z.sig);
    return kernel_rc(launch_verify(set, pool, pitch, batch, S_(stream), mlen, msg_off, sig_off, res_off));
}
MAYO_B200_API int mayo_b200_verify_DtH(int set, uint8_t *result, size_t mlen, const uint8_t *pool, size_t pitch,
                                       size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, row_verify(z, mlen), mlen);
    if (rc || !batch) return rc;
    const size_t res_off = A(z.epk) + A(mlen) + A(z.sig);
    return copy2d(result, 1, pool + res_off, pitch, 1, batch, cudaMemcpyDeviceToHost, stream);
}

// ---- verify from a compact key (src/api.cu:180-218) ----
MAYO_B200_API int mayo_b200_verifyWithepk_HtD(int set, const uint8_t *cpk, const uint8_t *msg, const uint8_t *sig,
                                              size_t mlen, uint8_t *pool, size_t pitch, size_t batch,
                                              void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, A(z.epk) + A(mlen) + z.sig, mlen);
    if (rc || !batch) return rc;
    rc = copy2d(pool + z.p - 16, pitch, cpk, z.pk, z.pk, batch, cudaMemcpyHostToDevice, stream);
    if (rc) return rc;
    rc = copy2d(pool + A(z.epk), pitch, msg, mlen, mlen, batch, cudaMemcpyHostToDevice, stream);
    if (rc) return rc;
    return copy2d(pool + A(z.epk) + A(mlen), pitch, sig, z.sig, z.sig, batch, cudaMemcpyHostToDevice, stream);
}
MAYO_B200_API int mayo_b200_verifyWithepk(int set, uint8_t *pool, size_t mlen, size_t pitch, size_t batch,
                                          void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    int rc = check(pool, pitch, batch, row_verify(z, mlen), mlen);
    if (rc || !batch) return rc;
    rc = kernel_rc(launch_expandpk(set, pool, pitch, batch, S_(stream)));
    if (rc) return rc;
    const size_t msg_off = A(z.epk), sig_off = msg_off + A(mlen), res_off = sig_off + A(z.sig);
    return kernel_rc(launch_verify(set, pool, pitch, batch, S_(stream), mlen, msg_off, sig_off, res_off));
}
MAYO_B200_API int mayo_b200_verifyWithepk_DtH(int set, uint8_t *result, size_t mlen, const uint8_t *pool,
                                              size_t pitch, size_t batch, void *stream) {
    return mayo_b200_verify_DtH(set, result, mlen, pool, pitch, batch, stream);
}

// ---- extension: explicit operand arrays ----
MAYO_B200_API size_t mayo_b200_sign_ws_bytes(int set) { return sign_ws_bytes(set); }

MAYO_B200_API int mayo_b200_sign_many(int set, const uint8_t *esk, size_t esk_stride, const uint8_t *msgs,
                                      const uint64_t *msg_off, const uint32_t *msg_len, size_t msg_stride,
                                      size_t mlen, uint8_t *sig, size_t sig_stride, uint8_t *ws, size_t batch,
                                      void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    if (batch == 0) return MAYO_B200_OK;
    if (!esk || !sig || !ws || batch > 0x7fffffffu || mlen > 0x7fffffffu) return MAYO_B200_ERR_ARG;
    if ((msg_off == nullptr) != (msg_len == nullptr)) return MAYO_B200_ERR_ARG;
    if (!msgs && (msg_off || mlen)) return MAYO_B200_ERR_ARG;
    if (batch > 1 && sig_stride < z.sig) return MAYO_B200_ERR_ARG;
    SignIO io{esk, esk_stride, MsgIO{msgs, msg_stride, msg_off, msg_len, (uint32_t)mlen}, sig, sig_stride, ws,
              sign_ws_bytes(set)};
    return kernel_rc(launch_sign_io(set, io, batch, S_(stream)));
}

MAYO_B200_API int mayo_b200_verify_many(int set, const uint8_t *epk, size_t epk_stride, const uint8_t *msgs,
                                        const uint64_t *msg_off, const uint32_t *msg_len, size_t msg_stride,
                                        size_t mlen, const uint8_t *sig, size_t sig_stride, uint8_t *result,
                                        size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    if (batch == 0) return MAYO_B200_OK;
    if (!epk || !sig || !result || batch > 0x7fffffffu || mlen > 0x7fffffffu) return MAYO_B200_ERR_ARG;
    if ((msg_off == nullptr) != (msg_len == nullptr)) return MAYO_B200_ERR_ARG;
    if (!msgs && (msg_off || mlen)) return MAYO_B200_ERR_ARG;
    if (batch > 1 && sig_stride < z.sig) return MAYO_B200_ERR_ARG;
    VerifyIO io{epk, epk_stride, MsgIO{msgs, msg_stride, msg_off, msg_len, (uint32_t)mlen}, sig, sig_stride, result,
                1};
    return kernel_rc(launch_verify_io(set, io, batch, S_(stream)));
}

MAYO_B200_API size_t mayo_b200_sign_shared_ws_bytes(int set, size_t batch) {
    return mayo::shared_ws_bytes(set, false, batch);
}

MAYO_B200_API int mayo_b200_sign_shared(int set, const uint8_t *esk, const uint8_t *msgs, const uint64_t *msg_off,
                                        const uint32_t *msg_len, size_t msg_stride, size_t mlen, uint8_t *sig,
                                        size_t sig_stride, uint8_t *ws, size_t batch, void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    if (batch == 0) return MAYO_B200_OK;
    if (!esk || !sig || !ws || batch > 0x7fffffffu || mlen > 0x7fffffffu) return MAYO_B200_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(ws) & 15) return MAYO_B200_ERR_ARG;  // bulk copies need 16-byte alignment
    if ((msg_off == nullptr) != (msg_len == nullptr)) return MAYO_B200_ERR_ARG;
    if (!msgs && (msg_off || mlen)) return MAYO_B200_ERR_ARG;
    if (batch > 1 && sig_stride < z.sig) return MAYO_B200_ERR_ARG;
    SignIO io{esk, 0, MsgIO{msgs, msg_stride, msg_off, msg_len, (uint32_t)mlen}, sig, sig_stride, nullptr, 0};
    return kernel_rc(mayo::launch_sign_shared(set, io, ws, batch, S_(stream)));
}

MAYO_B200_API int mayo_b200_shared_timing(int enable) { return kernel_rc(mayo::shared_timing(enable)); }

MAYO_B200_API int mayo_b200_shared_set_shape(int set, const mayo_b200_shared_shape *shape) {
    return mayo::shared_set_shape(set, shape ? (int)shape->hash_threads : 0, shape ? (int)shape->tail_instances : 0,
                                  shape ? (int)shape->product_ctas : 0);
}

MAYO_B200_API int mayo_b200_shared_get_shape(int set, mayo_b200_shared_shape *shape) {
    if (!shape) return MAYO_B200_ERR_ARG;
    int h = 0, g = 0, pc = 0;
    const int rc = mayo::shared_get_shape(set, &h, &g, &pc);
    shape->hash_threads = (uint32_t)h;
    shape->tail_instances = (uint32_t)g;
    shape->product_ctas = (uint32_t)pc;
    return rc;
}

MAYO_B200_API int mayo_b200_shared_timing_read(float *ms) {
    if (!ms) return MAYO_B200_ERR_ARG;
    const int rc = mayo::shared_timing_read(ms);
    return rc == mayo::ST_OK ? MAYO_B200_OK : (rc == mayo::ST_BAD_ARG ? MAYO_B200_ERR_ARG : MAYO_B200_ERR_CUDA);
}

MAYO_B200_API size_t mayo_b200_verify_shared_ws_bytes(int set, size_t batch) {
    return mayo::shared_ws_bytes(set, true, batch);
}

MAYO_B200_API int mayo_b200_verify_shared(int set, const uint8_t *epk, const uint8_t *msgs, const uint64_t *msg_off,
                                          const uint32_t *msg_len, size_t msg_stride, size_t mlen, const uint8_t *sig,
                                          size_t sig_stride, uint8_t *result, uint8_t *ws, size_t batch,
                                          void *stream) {
    Sz z;
    if (!sizes_of(set, z)) return MAYO_B200_ERR_SET;
    if (batch == 0) return MAYO_B200_OK;
    if (!epk || !sig || !result || !ws || batch > 0x7fffffffu || mlen > 0x7fffffffu) return MAYO_B200_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(ws) & 15) return MAYO_B200_ERR_ARG;
    if ((msg_off == nullptr) != (msg_len == nullptr)) return MAYO_B200_ERR_ARG;
    if (!msgs && (msg_off || mlen)) return MAYO_B200_ERR_ARG;
    if (batch > 1 && sig_stride < z.sig) return MAYO_B200_ERR_ARG;
    VerifyIO io{epk, 0, MsgIO{msgs, msg_stride, msg_off, msg_len, (uint32_t)mlen}, sig, sig_stride, result, 1};
    return kernel_rc(mayo::launch_verify_shared(set, io, ws, batch, S_(stream)));
}

}  // extern "C"
