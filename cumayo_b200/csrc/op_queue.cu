// op_queue.cu -- persistent work-queue kernel: keypair / sign / verify instances of all four
// parameter sets pulled by resident CTAs from one device queue.
//
// A work item is a 32-bit word: op (2 bits), parameter-set index (2 bits: MAYO_1, 2, 3, 5),
// sign attempt counter (8 bits) and instance index (20 bits).  Each CTA (160 threads) takes the
// next item with an atomic ticket, runs it with the same device functions as the batched
// kernels, and takes the next.  A sign attempt whose linear system is singular is not retried
// in place: the CTA pushes (sign, ctr + 1) to the tail of the queue and moves on, so one rare
// rejection never holds a CTA (or a whole launch) back.  The queue is drained when every
// published item is finished (done == tail; `done` is read before `tail`, so a push from an
// unfinished item can never be missed).  Waits are bounded: a ticket that stays unpublished past
// `spin_limit` sleeps sets an error code and ends the CTA instead of hanging.
#include <cuda_runtime.h>

#include "../../include/mayo_b200.h"
#include "aes.cuh"
#include "keygen_body.cuh"
#include "ops.h"
#include "sign_body.cuh"
#include "verify_body.cuh"

namespace mayo {

constexpr int Q_NT = 160;  // threads per queue CTA
constexpr int Q_NCV = 128; // verify compute threads (+ one hashing warp)
constexpr uint32_t Q_EMPTY = 0xFFFFFFFFu;
constexpr uint32_t Q_STOP = 0xFFFFFFFEu;

__host__ __device__ constexpr int set_of_index(int si) { return si == 0 ? 1 : si == 1 ? 2 : si == 2 ? 3 : 5; }

template <int SET>
struct QueueLayout {
    using KC = KeyCfg<SET, Q_NT>;
    static constexpr size_t aes_end = 256 * 32 * 4 + 44 * 4;  // replicated T0 + round keys
    static_assert(KC::off_o >= aes_end, "O must not overlap the AES tables");
    static constexpr size_t kp_seedpk = KC::off_o + pad16(Set<SET>::o_bytes);
    static constexpr size_t kp_total = kp_seedpk + 16;
    static constexpr size_t total_raw = kp_total > SignCfg<SET, Q_NT>::total
                                            ? (kp_total > VerifyCfg<SET, Q_NCV>::total ? kp_total
                                                                                       : VerifyCfg<SET, Q_NCV>::total)
                                            : (SignCfg<SET, Q_NT>::total > VerifyCfg<SET, Q_NCV>::total
                                                   ? SignCfg<SET, Q_NT>::total
                                                   : VerifyCfg<SET, Q_NCV>::total);
};
static_assert(VerifyCfg<1, Q_NCV>::NT == Q_NT && VerifyCfg<5, Q_NCV>::NT == Q_NT, "verify CTA shape");

using QueueOps = mayo_b200_queue_ops;

struct QueueArgs {
    QueueOps ops[4];
    uint32_t *items;
    uint32_t capacity;
    uint32_t *ctrl;  // [0] head ticket, [1] tail, [2] done, [3] error, [4] pushes
    uint8_t *scratch;
    size_t scratch_stride;
    uint32_t spin_limit;
};

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) { return *reinterpret_cast<const volatile uint32_t *>(p); }

__device__ uint32_t queue_pop(const QueueArgs &q) {
    const uint32_t idx = atomicAdd(&q.ctrl[0], 1u);
    for (uint32_t it = 0;; it++) {
        if (idx < q.capacity) {
            const uint32_t v = ld_volatile(&q.items[idx]);
            if (v != Q_EMPTY) {
                __threadfence();
                return v;
            }
        }
        const uint32_t done = ld_volatile(&q.ctrl[2]);
        __threadfence();
        const uint32_t tail = ld_volatile(&q.ctrl[1]);
        if (idx >= tail && done == tail) return Q_STOP;  // drained: no unfinished item can push
        // A ticket past the last slot can only end with the drain; a ticket inside the queue
        // waits for its item to be published.  Both waits are bounded.
        if (it >= q.spin_limit) {
            atomicCAS(&q.ctrl[3], 0u, (uint32_t)MAYO_B200_QUEUE_ERR_TIMEOUT);
            return Q_STOP;
        }
        __nanosleep(200);
    }
}

__device__ void queue_push(const QueueArgs &q, uint32_t item) {
    const uint32_t slot = atomicAdd(&q.ctrl[1], 1u);
    if (slot >= q.capacity) {
        atomicCAS(&q.ctrl[3], 0u, (uint32_t)MAYO_B200_QUEUE_ERR_FULL);
        // the slot never becomes visible; count the item as finished so the queue still drains
        atomicAdd(&q.ctrl[2], 1u);
        return;
    }
    atomicAdd(&q.ctrl[4], 1u);
    __threadfence();
    *reinterpret_cast<volatile uint32_t *>(&q.items[slot]) = item;
}

// ---- keypair from a caller seed on one CTA: hash (warp 0), AES-CTR (all), P3 (engine) ----
template <int SET>
__device__ void queue_keypair(uint8_t *smem, int tid, const QueueOps &ops, uint32_t inst, uint8_t *scratch) {
    using S = Set<SET>;
    using QL = QueueLayout<SET>;
    using KC = KeyCfg<SET, Q_NT>;
    const uint8_t *seed = ops.kp_seed + (size_t)inst * S::sk;
    uint8_t *pk = ops.kp_pk + (size_t)inst * S::pk;
    uint8_t *s_O = smem + KC::off_o;
    uint8_t *s_seedpk = smem + QL::kp_seedpk;
    if (tid < 32) {
        // seed_pk || O = SHAKE256(seed_sk) (src/keypair.cu:47), squeezed into the AES area, which is
        // free until the tables are built below
        WarpKeccak wk;
        wk.setup(tid);
        uint8_t *tmp = smem;
        warp_shake<136>(tmp, 16 + S::o_bytes, seed, S::sk, wk, tid);
        for (int i = tid; i < 16; i += 32) s_seedpk[i] = tmp[i];
        for (int i = tid; i < S::o_bytes; i += 32) s_O[i] = tmp[16 + i];
    }
    __syncthreads();
    // AES-CTR of P1 || P2 into this CTA's scratch (src/keypair.cu:52)
    uint32_t *T = reinterpret_cast<uint32_t *>(smem);
    uint32_t *rk_s = T + 256 * 32;
    for (int i = tid; i < 256 * 32; i += Q_NT) T[i] = c_aes.te0[i >> 5];
    if (tid == 0) aes128_key_schedule(s_seedpk, rk_s);
    __syncthreads();
    {
        uint32_t rk[44];
#pragma unroll
        for (int i = 0; i < 44; i++) rk[i] = rk_s[i];
        const uint32_t *Tl = T + (tid & 31);
        const uint32_t nblk = (S::p + 15) / 16;  // the scratch has room for the whole last block
        for (uint32_t blk = tid; blk < nblk; blk += Q_NT) {
            const AesOut o = aes128_ctr_block(Tl, rk, blk);
            st16(scratch + (size_t)blk * 16, bswap32(o.w0), bswap32(o.w1), bswap32(o.w2), bswap32(o.w3));
        }
    }
    __syncthreads();  // scratch writes visible to the whole CTA; AES tables no longer needed
    for (int i = tid; i < 16; i += Q_NT) pk[i] = s_seedpk[i];
    p3_instance<SET, Q_NT, false>(smem, tid, scratch, scratch + S::p1, pk + 16);
}

template <int SET>
__device__ void queue_sign(uint8_t *smem, int tid, const QueueArgs &q, const QueueOps &ops, uint32_t inst, int ctr,
                           uint32_t item) {
    using S = Set<SET>;
    const uint8_t *esk = ops.sg_esk + (size_t)(inst % ops.sg_nkeys) * S::esk;
    sign_hash_cta<SET, Q_NT>(smem, tid, esk, ops.sg_msg + (size_t)inst * ops.sg_mlen, ops.sg_mlen, ctr);
    const bool ok = sign_attempt<SET, Q_NT>(smem, tid, esk);
    if (ok || ctr >= 254) {
        // success, or the 255th rejection: the reference emits the last attempt (x = r)
        sign_write<SET, Q_NT>(smem, tid, esk, ops.sg_sig + (size_t)inst * S::sig);
    } else if (tid == 0) {
        queue_push(q, (item & ~(0xFFu << 20)) | ((uint32_t)(ctr + 1) << 20));
    }
}

template <int SET>
__device__ void queue_verify(uint8_t *smem, int tid, const QueueOps &ops, uint32_t inst) {
    using S = Set<SET>;
    const uint8_t *epk = ops.vf_epk + (size_t)(inst % ops.vf_nkeys) * S::epk;
    verify_instance<SET, Q_NCV>(smem, tid, epk, ops.vf_msg + (size_t)inst * ops.vf_mlen, ops.vf_mlen,
                                ops.vf_sig + (size_t)inst * S::sig, ops.vf_res + inst);
}

template <int SET>
__device__ __forceinline__ void queue_dispatch(uint8_t *smem, int tid, const QueueArgs &q, uint32_t op, uint32_t inst,
                                               int ctr, uint32_t item, uint8_t *scratch) {
    const QueueOps &ops = q.ops[SET == 1 ? 0 : SET == 2 ? 1 : SET == 3 ? 2 : 3];
    if (op == MAYO_B200_OP_KEYPAIR) queue_keypair<SET>(smem, tid, ops, inst, scratch);
    else if (op == MAYO_B200_OP_SIGN) queue_sign<SET>(smem, tid, q, ops, inst, ctr, item);
    else queue_verify<SET>(smem, tid, ops, inst);
}

__global__ void __launch_bounds__(Q_NT) queue_kernel(const QueueArgs q) {
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t s_item;
    const int tid = threadIdx.x;
    uint8_t *scratch = q.scratch + (size_t)blockIdx.x * q.scratch_stride;
    for (;;) {
        if (tid == 0) s_item = queue_pop(q);
        __syncthreads();
        const uint32_t item = s_item;
        __syncthreads();
        if (item == Q_STOP) break;
        const uint32_t op = item >> 30, si = (item >> 28) & 3, inst = item & 0xFFFFF;
        const int ctr = (int)((item >> 20) & 0xFF);
        switch (si) {
            case 0: queue_dispatch<1>(smem, tid, q, op, inst, ctr, item, scratch); break;
            case 1: queue_dispatch<2>(smem, tid, q, op, inst, ctr, item, scratch); break;
            case 2: queue_dispatch<3>(smem, tid, q, op, inst, ctr, item, scratch); break;
            default: queue_dispatch<5>(smem, tid, q, op, inst, ctr, item, scratch); break;
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicAdd(&q.ctrl[2], 1u);
        }
    }
}

// Queue reset: slots [0, n) <- items, [n, capacity) <- empty, counters <- (0, n, 0, 0, 0).
__global__ void queue_reset_kernel(uint32_t *slots, const uint32_t *items, uint32_t n, uint32_t capacity,
                                   uint32_t *ctrl) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < capacity) slots[i] = i < n ? items[i] : Q_EMPTY;
    if (i < 8) ctrl[i] = i == 1 ? n : 0u;
}

size_t queue_smem_bytes() {
    size_t m = 0;
    const size_t t[4] = {QueueLayout<1>::total_raw, QueueLayout<2>::total_raw, QueueLayout<3>::total_raw,
                         QueueLayout<5>::total_raw};
    for (size_t x : t) m = x > m ? x : m;
    return pad16(m);
}

size_t queue_scratch_stride() { return pad16((size_t)Set<5>::p + 16); }

int launch_queue(const QueueOps ops[4], const uint32_t *items, uint32_t n, uint32_t *slots, uint32_t capacity,
                 uint32_t *ctrl, uint8_t *scratch, uint32_t ctas, uint32_t spin_limit, cudaStream_t st) {
    if (n > capacity || ctas == 0) return ST_BAD_ARG;
    queue_reset_kernel<<<(capacity + 255) / 256, 256, 0, st>>>(slots, items, n, capacity, ctrl);
    const size_t smem = queue_smem_bytes();
    if (!set_smem_attr(queue_kernel, smem)) return ST_CUDA;
    QueueArgs q{};
    for (int i = 0; i < 4; i++) q.ops[i] = ops[i];
    q.items = slots;
    q.capacity = capacity;
    q.ctrl = ctrl;
    q.scratch = scratch;
    q.scratch_stride = queue_scratch_stride();
    q.spin_limit = spin_limit;
    queue_kernel<<<ctas, Q_NT, smem, st>>>(q);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

}  // namespace mayo

// ---- C-ABI ----
namespace {
constexpr size_t kCtrlBytes = 256;
size_t slots_bytes(uint32_t capacity) { return (((size_t)capacity * 4) + 255) / 256 * 256; }
}  // namespace

extern "C" {

MAYO_B200_API size_t mayo_b200_queue_mem_bytes(uint32_t capacity, uint32_t ctas) {
    return kCtrlBytes + slots_bytes(capacity) + (size_t)ctas * mayo::queue_scratch_stride();
}

MAYO_B200_API int mayo_b200_queue_ctas_per_sm(void) {
    int per_sm = 0;
    const size_t smem = mayo::queue_smem_bytes();
    if (!mayo::set_smem_attr(mayo::queue_kernel, smem)) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, mayo::queue_kernel, mayo::Q_NT, smem) != cudaSuccess)
        return 0;
    return per_sm;
}

MAYO_B200_API int mayo_b200_queue_run(const mayo_b200_queue_ops ops[4], const uint32_t *items, uint32_t n,
                                      void *queue_mem, uint32_t capacity, uint32_t ctas, uint32_t spin_limit,
                                      void *stream) {
    if (!ops || !queue_mem || (n && !items) || n > capacity || ctas == 0 || capacity > (1u << 28))
        return MAYO_B200_ERR_ARG;
    uint8_t *base = static_cast<uint8_t *>(queue_mem);
    uint32_t *ctrl = reinterpret_cast<uint32_t *>(base);
    uint32_t *slots = reinterpret_cast<uint32_t *>(base + kCtrlBytes);
    uint8_t *scratch = base + kCtrlBytes + slots_bytes(capacity);
    const int rc = mayo::launch_queue(ops, items, n, slots, capacity, ctrl, scratch, ctas,
                                      spin_limit ? spin_limit : (1u << 24), reinterpret_cast<cudaStream_t>(stream));
    return rc == mayo::ST_OK ? MAYO_B200_OK : (rc == mayo::ST_BAD_ARG ? MAYO_B200_ERR_ARG : MAYO_B200_ERR_CUDA);
}

}  // extern "C"
