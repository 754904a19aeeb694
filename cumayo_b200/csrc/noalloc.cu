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
//     (cudaGetSymbolAddress) and keeps it for that device's current CUDA context; a call made
//     in a new context of the device (after cudaDeviceReset, say) looks it up again.  Make the
//     first call before any stream capture: the look-up is not a stream operation, and a first
//     call made while a stream is being captured may fail with MAYO_B200_ERR_CUDA;
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

// The device address of the array belongs to a CUDA context: after cudaDeviceReset the device's
// next primary context loads the module again, possibly elsewhere.  So the cache is keyed on the
// context's id (cuCtxGetId, unique for the life of the process), read through the runtime's
// driver entry points so that the library needs no link dependency on libcuda.
using CtxGetCurrentFn = int (*)(void **ctx);                      // cuCtxGetCurrent
using CtxGetIdFn = int (*)(void *ctx, unsigned long long *id);  // cuCtxGetId
struct WsEntry {
    unsigned long long ctx_id;
    void *addr;
};
std::mutex g_mu;
WsEntry g_ws[kMaxDevices] = {};
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;
bool g_entry_points = false;

// Id of the calling thread's current context, 0 when none is current yet.  Called with g_mu held.
cudaError_t current_ctx_id(unsigned long long *id) {
    *id = 0;
    if (!g_entry_points) {
        cudaDriverEntryPointQueryResult q1, q2;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", reinterpret_cast<void **>(&g_ctx_current),
                                                cudaEnableDefault, &q1);
        if (e == cudaSuccess)
            e = cudaGetDriverEntryPoint("cuCtxGetId", reinterpret_cast<void **>(&g_ctx_id), cudaEnableDefault, &q2);
        if (e != cudaSuccess) return e;
        if (q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !g_ctx_current || !g_ctx_id)
            return cudaErrorNotSupported;
        g_entry_points = true;
    }
    void *ctx = nullptr;
    if (g_ctx_current(&ctx) != 0) return cudaErrorContextIsDestroyed;
    if (ctx && g_ctx_id(ctx, id) != 0) return cudaErrorContextIsDestroyed;
    return cudaSuccess;
}

// Device address of g_noalloc_ws in the current device's current context.  Status as in
// mayo_b200_status; a failed CUDA call is recorded for mayo_b200_last_cuda_error.
int noalloc_ws(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mayo::api_cuda_rc(e);
    if (dev < 0 || dev >= kMaxDevices) return MAYO_B200_ERR_ARG;
    std::lock_guard<std::mutex> lock(g_mu);
    unsigned long long id = 0;
    if ((e = current_ctx_id(&id)) != cudaSuccess) return mayo::api_cuda_rc(e);
    if (id == 0 || g_ws[dev].addr == nullptr || g_ws[dev].ctx_id != id) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_ws);  // creates the primary context if none is current
        if (e != cudaSuccess) return mayo::api_cuda_rc(e);
        if (p == nullptr) return mayo::api_cuda_rc(cudaErrorInvalidSymbol);
        if ((e = current_ctx_id(&id)) != cudaSuccess) return mayo::api_cuda_rc(e);
        g_ws[dev] = WsEntry{id, p};
    }
    *out = g_ws[dev].addr;
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
    const int rc = noalloc_ws(&ws);
    if (rc != MAYO_B200_OK) return rc;
    mayo::SignIO io{esk, esk_stride, mayo::MsgIO{msgs, msg_stride, msg_off, msg_len, (uint32_t)mlen},
                    sig, sig_stride, static_cast<uint8_t *>(ws), ws_bytes};
    // the launcher's status codes are the C-ABI's; a failed launch is recorded and cleared
    return mayo::api_launch_rc(mayo::launch_sign_io(set, io, batch, reinterpret_cast<cudaStream_t>(stream)));
}

}  // extern "C"
