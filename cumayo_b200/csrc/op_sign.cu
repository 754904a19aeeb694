// op_sign.cu -- batched MAYO sign on B200 (reference src/sign.cu:10-477).
//
// sign_hash_kernel (thread per instance, Keccak in registers) writes digest, salt, t and the
// first V||r into the per-instance workspace; sign_kernel (CTA per instance) runs the attempts of
// sign_body.cuh, retrying with ctr + 1 while the system is singular (at most 255 attempts,
// sign.cu:244-470), and writes s || salt.
#include "sign_body.cuh"

namespace mayo {

template <int SET>
__global__ void sign_hash_kernel(const SignIO io, uint32_t batch, const uint32_t *order) {
    using S = Set<SET>;
    using WS = SignWs<SET>;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    const uint32_t inst = order ? order[i] : i;  // order: instances grouped by message blocks
    const uint8_t *seed_sk = io.esk + (size_t)inst * io.esk_stride;
    uint8_t *ws = io.ws + (size_t)inst * io.ws_stride;
    alignas(8) uint8_t digest[S::digest];
    alignas(8) uint8_t salt[S::sk];
    {
        Sponge<136> sp;  // digest = SHAKE256(M) (sign.cu:225)
        sp.init();
        sp.absorb(io.m.ptr(inst), io.m.len(inst));
        sp.finalize();
        sp.squeeze(digest, S::digest);
    }
    {
        Sponge<136> sp;  // salt = SHAKE256(digest || 0^SK || seed_sk) (sign.cu:230-238)
        sp.init();
        sp.absorb(digest, S::digest);
        sp.absorb_zeros(S::sk);
        sp.absorb(seed_sk, S::sk);
        sp.finalize();
        sp.squeeze(salt, S::sk);
    }
    {
        Sponge<136> sp;  // t = SHAKE256(digest || salt) (sign.cu:240-243)
        sp.init();
        sp.absorb(digest, S::digest);
        sp.absorb(salt, S::sk);
        sp.finalize();
        sp.squeeze(ws + WS::t, S::menc);
    }
    {
        Sponge<136> sp;  // V || r for ctr = 0 (sign.cu:250-252)
        sp.init();
        sp.absorb(digest, S::digest);
        sp.absorb(salt, S::sk);
        sp.absorb(seed_sk, S::sk);
        sp.absorb_zeros(1);  // ctr = 0
        sp.finalize();
        sp.squeeze(ws + WS::vr, S::vr);
    }
    static_assert(WS::dig % 8 == 0 && WS::salt % 8 == 0 && S::digest % 8 == 0 && S::sk % 8 == 0, "word copies");
    if ((reinterpret_cast<uintptr_t>(ws) & 7) == 0) {  // the shared-key workspace; pool scratch may be unaligned
        for (int i = 0; i < S::digest / 8; i++)
            reinterpret_cast<uint64_t *>(ws + WS::dig)[i] = reinterpret_cast<const uint64_t *>(digest)[i];
        for (int i = 0; i < S::sk / 8; i++)
            reinterpret_cast<uint64_t *>(ws + WS::salt)[i] = reinterpret_cast<const uint64_t *>(salt)[i];
    } else {
        for (int i = 0; i < S::digest; i++) ws[WS::dig + i] = digest[i];
        for (int i = 0; i < S::sk; i++) ws[WS::salt + i] = salt[i];
    }
}

template <int SET>
__global__ void __launch_bounds__(SignCfg<SET>::NT) sign_kernel(const SignIO io) {
    extern __shared__ __align__(16) uint8_t smem[];
    constexpr int NT = SignCfg<SET>::NT;
    const int tid = threadIdx.x;
    const size_t inst = blockIdx.x;
    const uint8_t *esk = io.esk + inst * io.esk_stride;
    sign_load_ws<SET, NT>(smem, tid, esk, io.ws + inst * io.ws_stride);
#pragma unroll 1
    for (int ctr = 0; ctr < 255; ctr++) {
        if (ctr > 0) sign_next_vr<SET, NT>(smem, tid, ctr);
        if (sign_attempt<SET, NT>(smem, tid, esk)) break;
    }
    sign_write<SET, NT>(smem, tid, esk, io.sig + inst * io.sig_stride);
}

template <int SET>
static int sign_t(const SignIO &io, size_t batch, cudaStream_t st) {
    using C = SignCfg<SET>;
    sign_hash_kernel<SET><<<(unsigned)((batch + HASH_NT - 1) / HASH_NT), HASH_NT, 0, st>>>(io, (uint32_t)batch, nullptr);
    if (!set_smem_attr(sign_kernel<SET>, C::total)) return ST_CUDA;
    sign_kernel<SET><<<(unsigned)batch, C::NT, C::total, st>>>(io);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

int launch_sign_hash(int set, const SignIO &io, size_t batch, cudaStream_t st, const uint32_t *order, int nt) {
    if (batch == 0) return ST_OK;
    const unsigned g = (unsigned)((batch + nt - 1) / nt);
    const uint32_t b = (uint32_t)batch;
    switch (set) {
        case 1: sign_hash_kernel<1><<<g, nt, 0, st>>>(io, b, order); break;
        case 2: sign_hash_kernel<2><<<g, nt, 0, st>>>(io, b, order); break;
        case 3: sign_hash_kernel<3><<<g, nt, 0, st>>>(io, b, order); break;
        case 5: sign_hash_kernel<5><<<g, nt, 0, st>>>(io, b, order); break;
        default: return ST_BAD_SET;
    }
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

int launch_sign_io(int set, const SignIO &io, size_t batch, cudaStream_t st) {
    if (batch == 0) return ST_OK;
    switch (set) {
        case 1: return sign_t<1>(io, batch, st);
        case 2: return sign_t<2>(io, batch, st);
        case 3: return sign_t<3>(io, batch, st);
        case 5: return sign_t<5>(io, batch, st);
        default: return ST_BAD_SET;
    }
}

size_t sign_ws_bytes(int set) {
    switch (set) {
        case 1: return SignWs<1>::total;
        case 2: return SignWs<2>::total;
        case 3: return SignWs<3>::total;
        case 5: return SignWs<5>::total;
        default: return 0;
    }
}

int launch_sign(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st, size_t mlen, size_t msg_off,
                size_t sig_off, size_t scratch_off) {
    SignIO io{pool, pitch, MsgIO{pool + msg_off, pitch, nullptr, nullptr, (uint32_t)mlen},
              pool + sig_off, pitch, pool + scratch_off, pitch};
    return launch_sign_io(set, io, batch, st);
}

}  // namespace mayo
