// ops.h -- internal launchers of the B200 MAYO engine (C++ linkage, not part of the C-ABI).
// Every launcher takes the reference's pitched pool (row b = instance b) and byte offsets
// inside a row; it launches asynchronously on `st` and returns a mayo_status code.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace mayo {

// Threads per CTA of the thread-per-instance hash kernels: their registers allow 8 such CTAs per
// SM, so small CTAs spread a batch evenly over the 148 SMs (whole waves).
constexpr int HASH_NT = 64;

// Status codes shared with include/mayo_b200.h.
enum : int {
    ST_OK = 0,
    ST_BAD_SET = 1,
    ST_BAD_ARG = 2,
    ST_CUDA = 3,
};

// Keypair of instances [0, batch): seed_sk = SHAKE128(LE64(rand_index + 2b + 1)).
// Row layout (reference src/api.cu:17-26): sk @0, pk @A(SK), P1||P2 scratch @A(SK)+A(PK).
int launch_keypair(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st, uint64_t rand_index);
// Keypair from caller seeds already stored at row offset 0 (sk_bytes each).
int launch_keypair_seeded(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st);
// esk = sk || O || P1 || L in place over a row that holds sk at offset 0 (src/api.cu:47-54).
int launch_expandsk(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st);
// epk = P1 || P2 || P3 in place over a row that holds cpk at offset P-16 (src/api.cu:64-77).
int launch_expandpk(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st);
// Verify with epk at row offset 0; message, signature and result byte at the given offsets.
int launch_verify(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st, size_t mlen, size_t msg_off,
                  size_t sig_off, size_t res_off);
// Sign with esk at row offset 0; message and signature at the given offsets; `scratch_off`
// points at the reference's per-row scratch (k*m*ceil(o/2) bytes) used as workspace.
int launch_sign(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st, size_t mlen, size_t msg_off,
                size_t sig_off, size_t scratch_off);

// Where instance i's operands live.  A stride of 0 on a key shares one key across the batch.
// Messages are either msg + i*msg_stride with length mlen, or (when msg_off is non-null, a
// device array) msg + msg_off[i] with length msg_len[i].
struct MsgIO {
    const uint8_t *msg;
    size_t msg_stride;
    const uint64_t *msg_off;
    const uint32_t *msg_len;
    uint32_t mlen;
#ifdef __CUDACC__
    __device__ __forceinline__ const uint8_t *ptr(size_t i) const { return msg_off ? msg + msg_off[i] : msg + i * msg_stride; }
    __device__ __forceinline__ uint32_t len(size_t i) const { return msg_len ? msg_len[i] : mlen; }
#endif
};
struct SignIO {
    const uint8_t *esk;  // seed_sk || O || P1 || L
    size_t esk_stride;
    MsgIO m;
    uint8_t *sig;
    size_t sig_stride;
    uint8_t *ws;  // per-instance workspace of sign_ws_bytes(set) bytes
    size_t ws_stride;
};
struct VerifyIO {
    const uint8_t *epk;  // P1 || P2 || P3
    size_t epk_stride;
    MsgIO m;
    const uint8_t *sig;
    size_t sig_stride;
    uint8_t *res;  // 0 = accept, 1 = reject
    size_t res_stride;
};
int launch_sign_io(int set, const SignIO &io, size_t batch, cudaStream_t st);
// Only the hash stage of sign (digest, salt, t, V || r for ctr 0 into io.ws).
// order (optional, batch entries): thread i hashes instance order[i]
int launch_sign_hash(int set, const SignIO &io, size_t batch, cudaStream_t st, const uint32_t *order = nullptr,
                     int nt = HASH_NT);
int launch_verify_io(int set, const VerifyIO &io, size_t batch, cudaStream_t st);
// Workspace bytes per instance used by sign (digest, salt, t, V || r).
size_t sign_ws_bytes(int set);
// One key for the whole batch, its products on the tensor cores (op_shared.cu).
size_t shared_ws_bytes(int set, bool verify, size_t batch);
int launch_sign_shared(int set, const SignIO &io, uint8_t *ws, size_t batch, cudaStream_t st);
int launch_verify_shared(int set, const VerifyIO &io, uint8_t *ws, size_t batch, cudaStream_t st);
int shared_timing(int enable);
int shared_timing_read(float *ms);
// Runtime shape of the shared-key path per set: hash-kernel CTA threads, sign-tail instances per
// CTA, CTAs per key-product tile (1, or a CTA pair).
int shared_set_shape(int set, int hash_nt, int tail_g, int product_ctas);
int shared_get_shape(int set, int *hash_nt, int *tail_g, int *product_ctas);

// Status plumbing of the C-ABI (capi.cu): a failed CUDA call or launch is recorded as the calling
// thread's last CUDA error (mayo_b200_last_cuda_error) and reported as ST_CUDA.  api_launch_rc
// takes a launcher's status and, for ST_CUDA, reads and clears the runtime's last error.
int api_cuda_rc(cudaError_t e);
int api_launch_rc(int rc);

// Failure injection for tests (mayo_b200_test_inject), per host thread; kind 0 = off.
struct Inject {
    int kind = 0;
    uint32_t arg = 0, spin = 0;
};
Inject &inject();

}  // namespace mayo
