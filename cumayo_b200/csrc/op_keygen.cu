// op_keygen.cu -- batched keypair, expand-sk and expand-pk on B200.
//
// keypair  (reference src/keypair.cu:10-121):  hash kernel (thread per instance: seed_sk,
//          seed_pk || O) -> AES-CTR kernel (P1 || P2 into the row's scratch) -> P3 engine kernel.
// expandsk (src/expandsk.cu:9-81): hash kernel (O, seed_pk) -> AES-CTR -> L engine kernel.
// expandpk (src/expandpk.cu:9-23): AES-CTR only.
#include "aes.cuh"
#include "keygen_body.cuh"
#include "ops.h"

namespace mayo {

// ---------------------------------------------------------------------------------------------
// Hash kernels: one thread per instance, Keccak state in registers.
// ---------------------------------------------------------------------------------------------
// keypair: seed_sk = SHAKE128(LE64(rand_index + 2*inst + 1), SK) (src/keypair.cu:35-45) unless
// `seeded`; then seed_pk || O = SHAKE256(seed_sk) (src/keypair.cu:47-50).  seed_pk goes to pk[0:16];
// O is parked in pk[16 : 16 + O_BYTES] until the P3 kernel overwrites that region.
template <int SET>
__global__ void keypair_hash_kernel(uint8_t *pool, size_t pitch, uint32_t batch, uint64_t rand_index, int seeded) {
    using S = Set<SET>;
    const uint32_t inst = blockIdx.x * blockDim.x + threadIdx.x;
    if (inst >= batch) return;
    uint8_t *row = pool + (size_t)inst * pitch;
    uint8_t *sk = row;
    uint8_t *pk = row + align128(S::sk);
    if (!seeded) {
        const uint64_t ctr = rand_index + (uint64_t)(uint32_t)(2u * inst) + 1;
        uint8_t cb[8];
#pragma unroll
        for (int i = 0; i < 8; i++) cb[i] = (uint8_t)(ctr >> (8 * i));
        Sponge<168> sp;
        sp.init();
        sp.absorb(cb, 8);
        sp.finalize();
        sp.squeeze(sk, S::sk);
    }
    Sponge<136> sp2;
    sp2.init();
    sp2.absorb(sk, S::sk);
    sp2.finalize();
    sp2.squeeze(pk, 16);
    sp2.squeeze(pk + 16, S::o_bytes);
}

// expandsk: seed_pk || O = SHAKE256(seed_sk) (src/expandsk.cu:28-35).  O goes to its esk slot;
// seed_pk is parked in the last 16 bytes of the P region, which the AES tail kernel writes last.
template <int SET>
__global__ void expandsk_hash_kernel(uint8_t *pool, size_t pitch, uint32_t batch) {
    using S = Set<SET>;
    const uint32_t inst = blockIdx.x * blockDim.x + threadIdx.x;
    if (inst >= batch) return;
    uint8_t *row = pool + (size_t)inst * pitch;
    Sponge<136> sp;
    sp.init();
    sp.absorb(row, S::sk);
    sp.finalize();
    sp.squeeze(row + S::sk + S::o_bytes + S::p - 16, 16);
    sp.squeeze(row + S::sk, S::o_bytes);
}

// ---------------------------------------------------------------------------------------------
// P3 (keypair) and L (expandsk) engine kernels: one CTA per instance.
// ---------------------------------------------------------------------------------------------
template <int SET>
__global__ void __launch_bounds__(KeyCfg<SET>::NT) p3_kernel(uint8_t *pool, size_t pitch) {
    using S = Set<SET>;
    using C = KeyCfg<SET>;
    extern __shared__ __align__(16) uint8_t smem[];
    const int tid = threadIdx.x;
    uint8_t *row = pool + (size_t)blockIdx.x * pitch;
    uint8_t *pk = row + align128(S::sk);
    const uint8_t *P1 = pk + align128(S::pk);
    // O is parked in pk[16:]: copy it to shared memory before P3 overwrites that region
    for (int i = tid; i < S::o_bytes; i += C::NT) smem[C::off_o + i] = pk[16 + i];
    __syncthreads();
    // batched row loads (CU = 4) measured faster for MAYO_2's P3 only (MAYO_1/3/5: 0.494 -> 0.502,
    // 1.18 -> 1.20, 2.89 -> 3.04 ms per 1,024 keypairs; MAYO_2 0.475 -> 0.462)
    p3_instance<SET, C::NT, true, SET == 2 ? 4 : 1>(smem, tid, P1, P1 + S::p1, pk + 16);
}

template <int SET>
__global__ void __launch_bounds__(KeyCfg<SET>::NT) l_kernel(uint8_t *pool, size_t pitch) {
    using S = Set<SET>;
    using C = KeyCfg<SET>;
    constexpr int J = C::J, R = C::R, NT = C::NT;
    extern __shared__ __align__(16) uint8_t smem[];
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *bs = reinterpret_cast<uint4 *>(smem + C::off_bs);
    uint8_t *s_O = smem + C::off_o;
    const int tid = threadIdx.x;
    uint8_t *row = pool + (size_t)blockIdx.x * pitch;
    const uint8_t *P1 = row + S::sk + S::o_bytes;
    uint8_t *P2 = row + S::sk + S::o_bytes + S::p1;

    for (int i = tid; i < S::o_bytes; i += NT) s_O[i] = row[S::sk + i];
    __syncthreads();
    build_o_masks<SET>(masks, s_O, tid, NT);
    __syncthreads();

    // four row groups' loads in flight per thread: L reads P1 twice (rows and columns) with
    // little else to hide the latency (MAYO_1 signWithesk 1.10 -> 1.07 ms per 1,024, MAYO_5
    // 7.13 -> 6.97)
    Engine<SET, J, R, true, 4> eng;
    eng.setup(masks, bs, tid);
    const LRows<SET> rows{P1, P2};
#pragma unroll 1
    for (int r0 = 0; r0 < S::v; r0 += R) {
        if (SET >= 3 && tid < 32) eng.prefetch(rows, r0 + R, S::v, tid);  // next pass into L2
        eng.convert(rows, r0, S::v, tid, NT);
        __syncthreads();
        const int r = r0 + eng.rs;
        if (eng.active && r < S::v) {
            const G4 T = eng.row_product(rows, r);  // L[r][j]
            store_group<SET>(P2 + (size_t)(r * S::o + eng.j) * S::menc, eng.w, T);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------------------------
static int aes_expand(uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st, size_t key_off, size_t out_off,
                      uint32_t nbytes, bool key_in_output) {
    // the main kernel writes whole blocks that neither run past nbytes nor touch the key
    uint32_t nblk_main = nbytes / 16;
    if (key_in_output) nblk_main = min(nblk_main, (uint32_t)((key_off - out_off) / 16));
    const uint32_t nblk = (nbytes + 15) / 16;
    if (nblk_main > 0) {
        if (!set_smem_attr(aes_ctr_kernel, AES_SMEM)) return ST_CUDA;
        // near-equal chunks of at most AES_BLOCKS_PER_CTA blocks per instance
        const uint32_t chunks = (nblk_main + AES_BLOCKS_PER_CTA - 1) / AES_BLOCKS_PER_CTA;
        const uint32_t bpc = (nblk_main + chunks - 1) / chunks;
        // instances on the grid's y dimension, at most 65,535 per launch
        for (size_t b0 = 0; b0 < batch; b0 += 65535) {
            const unsigned nb = (unsigned)(batch - b0 < 65535 ? batch - b0 : 65535);
            aes_ctr_kernel<<<dim3(chunks, nb), AES_THREADS, AES_SMEM, st>>>(pool + b0 * pitch, pitch, key_off, out_off,
                                                                             nblk_main, bpc, 128u);
        }
    }
    if (nblk_main < nblk)
        aes_ctr_tail_kernel<<<(unsigned)((batch + AES_TAIL_THREADS - 1) / AES_TAIL_THREADS), AES_TAIL_THREADS, 0, st>>>(
            pool, pitch, key_off, out_off, nblk_main, nbytes, (uint32_t)batch);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

template <int SET>
static int keypair_t(uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st, uint64_t rand_index, bool seeded) {
    using S = Set<SET>;
    using C = KeyCfg<SET>;
    keypair_hash_kernel<SET><<<(unsigned)((batch + 127) / 128), 128, 0, st>>>(pool, pitch, (uint32_t)batch, rand_index,
                                                                                 seeded ? 1 : 0);
    const size_t pk_off = align128(S::sk);
    int rc = aes_expand(pool, pitch, batch, st, pk_off, pk_off + align128(S::pk), S::p, false);
    if (rc) return rc;
    if (!set_smem_attr(p3_kernel<SET>, C::total)) return ST_CUDA;
    p3_kernel<SET><<<(unsigned)batch, C::NT, C::total, st>>>(pool, pitch);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

template <int SET>
static int expandsk_t(uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st) {
    using S = Set<SET>;
    using C = KeyCfg<SET>;
    expandsk_hash_kernel<SET><<<(unsigned)((batch + 127) / 128), 128, 0, st>>>(pool, pitch, (uint32_t)batch);
    const size_t out_off = S::sk + S::o_bytes;
    int rc = aes_expand(pool, pitch, batch, st, out_off + S::p - 16, out_off, S::p, true);
    if (rc) return rc;
    if (!set_smem_attr(l_kernel<SET>, C::total)) return ST_CUDA;
    l_kernel<SET><<<(unsigned)batch, C::NT, C::total, st>>>(pool, pitch);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

template <int SET>
static int expandpk_t(uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st) {
    using S = Set<SET>;
    return aes_expand(pool, pitch, batch, st, S::p - 16, 0, S::p, true);
}

#define MAYO_DISPATCH(set, call)             \
    switch (set) {                           \
        case 1: { constexpr int SET = 1; return call; } \
        case 2: { constexpr int SET = 2; return call; } \
        case 3: { constexpr int SET = 3; return call; } \
        case 5: { constexpr int SET = 5; return call; } \
        default: return ST_BAD_SET;          \
    }

int launch_keypair(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st, uint64_t rand_index) {
    if (batch == 0) return ST_OK;
    MAYO_DISPATCH(set, (keypair_t<SET>(pool, pitch, batch, st, rand_index, false)))
}
int launch_keypair_seeded(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st) {
    if (batch == 0) return ST_OK;
    MAYO_DISPATCH(set, (keypair_t<SET>(pool, pitch, batch, st, 0, true)))
}
int launch_expandsk(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st) {
    if (batch == 0) return ST_OK;
    MAYO_DISPATCH(set, (expandsk_t<SET>(pool, pitch, batch, st)))
}
int launch_expandpk(int set, uint8_t *pool, size_t pitch, size_t batch, cudaStream_t st) {
    if (batch == 0) return ST_OK;
    MAYO_DISPATCH(set, (expandpk_t<SET>(pool, pitch, batch, st)))
}

}  // namespace mayo
