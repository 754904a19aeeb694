// noalloc.cu -- mayo_b200_sign_many_noalloc: batched sign that needs no caller workspace.
//
// mayo_b200_sign_many needs a device workspace of mayo_b200_sign_ws_bytes(set) bytes per
// instance (digest, salt, t and V||r, written by the hashing kernel and read by the signing
// kernel).  Some callers cannot allocate device memory to hold it: a serving process whose
// device-memory budget is fixed when it starts, or a host program that owns the allocator and
// does not let a plug-in library call cudaMalloc.  This entry point keeps that workspace in a
// fixed-size array compiled into the library instead.
//
// Limits and behaviour:
//   * the array is kNoAllocWsBytes (4 MiB); every GPU that loads the library holds it until
//     the process exits;
//   * a batch needs batch * mayo_b200_sign_ws_bytes(set) bytes of it; larger batches are
//     rejected with MAYO_B200_ERR_TOO_LARGE (mayo_b200_sign_noalloc_max_batch gives the limit);
//   * the first call on each device looks up the array's device address on that device
//     (cudaGetSymbolAddress); make that first call before any stream capture;
//   * every call uses the same array and it keeps whatever the last call left in it; nothing
//     in it needs to start at zero (the hashing kernel writes every byte the signing kernel
//     reads), but calls whose work overlaps on the GPU (different streams, no ordering between
//     them) race on the array and must not be issued;
//   * no cudaMalloc, cudaFree or other allocating call is made.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/mayo_b200.h"
#include "common.cuh"
#include "ops.h"

namespace {

constexpr size_t kNoAllocWsBytes = size_t(4) << 20;

static __device__ __align__(256) uint8_t g_noalloc_ws[kNoAllocWsBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_ws_addr[kMaxDevices] = {};

// Device address of g_noalloc_ws on the current device (looked up once per device).
int noalloc_ws(void **out, int *cuda_err) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *cuda_err = (int)e;
        return MAYO_B200_ERR_CUDA;
    }
    if (dev < 0 || dev >= kMaxDevices) return MAYO_B200_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ws_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_ws);
        if (e != cudaSuccess || p == nullptr) {
            *cuda_err = (int)e;
            return MAYO_B200_ERR_CUDA;
        }
        g_ws_addr[dev] = p;
    }
    *out = g_ws_addr[dev];
    return MAYO_B200_OK;
}

int sig_bytes_of(int set) {
    switch (set) {
        case 1: return mayo::Set<1>::sig;
        case 2: return mayo::Set<2>::sig;
        case 3: return mayo::Set<3>::sig;
        case 5: return mayo::Set<5>::sig;
        default: return 0;
    }
}

}  // namespace

extern "C" {

MAYO_B200_API size_t mayo_b200_sign_noalloc_max_batch(int set) {
    const size_t ws = mayo::sign_ws_bytes(set);
    return ws ? kNoAllocWsBytes / ws : 0;
}

MAYO_B200_API int mayo_b200_sign_many_noalloc(int set, const uint8_t *esk, size_t esk_stride, const uint8_t *msgs,
                                              const uint64_t *msg_off, const uint32_t *msg_len, size_t msg_stride,
                                              size_t mlen, uint8_t *sig, size_t sig_stride, size_t batch,
                                              void *stream) {
    const size_t ws_bytes = mayo::sign_ws_bytes(set);
    if (ws_bytes == 0) return MAYO_B200_ERR_SET;
    if (batch == 0) return MAYO_B200_OK;
    if (batch > kNoAllocWsBytes / ws_bytes) return MAYO_B200_ERR_TOO_LARGE;
    if (!esk || !sig || mlen > 0x7fffffffu) return MAYO_B200_ERR_ARG;
    if ((msg_off == nullptr) != (msg_len == nullptr)) return MAYO_B200_ERR_ARG;
    if (!msgs && (msg_off || mlen)) return MAYO_B200_ERR_ARG;
    if (batch > 1 && sig_stride < (size_t)sig_bytes_of(set)) return MAYO_B200_ERR_ARG;
    void *ws = nullptr;
    int cuda_err = 0;
    int rc = noalloc_ws(&ws, &cuda_err);
    if (rc != MAYO_B200_OK) return rc;
    mayo::SignIO io{esk, esk_stride, mayo::MsgIO{msgs, msg_stride, msg_off, msg_len, (uint32_t)mlen},
                    sig, sig_stride, static_cast<uint8_t *>(ws), ws_bytes};
    rc = mayo::launch_sign_io(set, io, batch, reinterpret_cast<cudaStream_t>(stream));
    return rc == mayo::ST_OK ? MAYO_B200_OK : (rc == mayo::ST_BAD_SET ? MAYO_B200_ERR_SET : MAYO_B200_ERR_CUDA);
}

}  // extern "C"
