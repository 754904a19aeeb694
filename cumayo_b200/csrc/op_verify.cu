// op_verify.cu -- batched MAYO verify on B200 (reference src/verify.cu:9-212): one CTA per
// instance running verify_instance (verify_body.cuh).
#include "ops.h"
#include "verify_body.cuh"

namespace mayo {

template <int SET>
__device__ __forceinline__ void verify_cta(const VerifyIO &io) {
    extern __shared__ __align__(16) uint8_t smem[];
    const size_t inst = blockIdx.x;
    verify_instance<SET, VerifyCfg<SET>::NC>(smem, threadIdx.x, io.epk + inst * io.epk_stride, io.m.ptr(inst),
                                             io.m.len(inst), io.sig + inst * io.sig_stride,
                                             io.res + inst * io.res_stride);
}
template <int SET>
__global__ void __launch_bounds__(VerifyCfg<SET>::NT) verify_kernel(const VerifyIO io) {
    verify_cta<SET>(io);
}
// MAYO_3: its shared memory allows 6 CTAs per SM; registers capped to match
template <>
__global__ void __launch_bounds__(VerifyCfg<3>::NT, 6) verify_kernel<3>(const VerifyIO io) {
    verify_cta<3>(io);
}

template <int SET>
static int verify_t(const VerifyIO &io, size_t batch, cudaStream_t st) {
    using C = VerifyCfg<SET>;
    if (!set_smem_attr(verify_kernel<SET>, C::total)) return ST_CUDA;
    verify_kernel<SET><<<(unsigned)batch, C::NT, C::total, st>>>(io);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

int launch_verify_io(int set, const VerifyIO &io, size_t batch, cudaStream_t st) {
    if (batch == 0) return ST_OK;
    switch (set) {
        case 1: return verify_t<1>(io, batch, st);
        case 2: return verify_t<2>(io, batch, st);
        case 3: return verify_t<3>(io, batch, st);
        case 5: return verify_t<5>(io, batch, st);
        default: return ST_BAD_SET;
    }
}

int launch_verify(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st, size_t mlen, size_t msg_off,
                  size_t sig_off, size_t res_off) {
    VerifyIO io{pool, pitch, MsgIO{pool + msg_off, pitch, nullptr, nullptr, (uint32_t)mlen}, pool + sig_off, pitch,
                pool + res_off, pitch};
    return launch_verify_io(set, io, batch, st);
}

}  // namespace mayo
