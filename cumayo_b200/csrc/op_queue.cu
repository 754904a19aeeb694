// op_queue.cu -- persistent work queue: keypair / sign / verify items of all four parameter sets.
//
// A work item is a 32-bit word: op (2 bits), parameter-set index (2 bits: MAYO_1, 2, 3, 5),
// sign attempt counter (8 bits) and instance index (20 bits).  A run
//   1. fills every bucket's slots with "empty" and zeroes the control words,
//   2. partitions the caller's mixed item array into 12 buckets, one per (set, op), keeping the
//      order within a bucket,
//   3. forks streams and launches one persistent kernel per bucket whose operands are set.
// Each (set, op) has its own kernel because their CTAs need 35-81 KB of shared memory and 56-128
// registers per thread: one kernel shaped for the largest would run MAYO_1 at two CTAs per SM
// instead of five, and MAYO_5's keypair and verify at two instead of three.  Each kernel has the
// shape of the batched kernel for its (set, op).  On forked streams the kernels share the SMs,
// and the CTAs of a kernel launched later take the SMs of one whose bucket has drained, so one
// bucket's tail overlaps another's work.
//
// Inside a kernel each CTA takes the next item (see queue_pop), runs it with the same device
// functions as the batched kernels, and takes the next; a CTA that finds its bucket empty exits
// at once and frees its SM for the other buckets' kernels.  A sign attempt whose linear system is singular is not retried in place: the CTA
// pushes (sign, ctr + 1) to the tail of its bucket and goes on popping, so the item is served
// either by that CTA or by another one still running.  No CTA waits for another kernel, so the
// kernels need not be co-resident.  Every wait is bounded: past `spin_limit` it sets an error
// code and ends the CTA.
#include <cuda_runtime.h>

#include "../../include/mayo_b200.h"
#include "aes.cuh"
#include "keygen_body.cuh"
#include "ops.h"
#include "sign_body.cuh"
#include "verify_body.cuh"

namespace mayo {

constexpr uint32_t Q_EMPTY = 0xFFFFFFFFu;
constexpr uint32_t Q_STOP = 0xFFFFFFFEu;
constexpr int Q_BUCKETS = 12;             // (set index) * 3 + op
constexpr int Q_CTRL_WORDS = 16;          // control words per bucket; block 12 counts invalid ops
constexpr size_t Q_SM_SMEM = 228 * 1024;  // shared memory per SM (sm_100)
constexpr size_t Q_CTA_RESERVED = 1024;   // shared memory the runtime reserves per CTA

template <int SET, int OP>
struct QueueCfg;

template <int SET>
struct QueueCfg<SET, MAYO_B200_OP_KEYPAIR> {
    using S = Set<SET>;
    using KC = KeyCfg<SET>;
    static constexpr int NT = KC::NT;
    // replicated T0 (and ror16(T0) where the P3 engine's area below O holds both: MAYO_5) and the
    // round keys; the tables are dead once the keystream is written
    static constexpr int NTAB = KC::off_o >= 2 * 256 * 32 * 4 + 44 * 4 ? 2 : 1;
    static constexpr size_t aes_end = NTAB * 256 * 32 * 4 + 44 * 4;
    static_assert(KC::off_o >= aes_end, "O must not overlap the AES tables");
    static constexpr size_t seedpk = KC::off_o + pad16(S::o_bytes);
    static constexpr size_t smem = seedpk + 16;
    static constexpr size_t scratch = pad16((size_t)S::p + 16);  // P1 || P2 of one keypair
};

template <int SET>
struct QueueCfg<SET, MAYO_B200_OP_SIGN> {
    static constexpr int NT = SignCfg<SET>::NT;
    static constexpr size_t smem = SignCfg<SET>::total;
    static constexpr size_t scratch = 0;
};

template <int SET>
struct QueueCfg<SET, MAYO_B200_OP_VERIFY> {
    static constexpr int NT = VerifyCfg<SET>::NT;
    static constexpr size_t smem = VerifyCfg<SET>::total;
    static constexpr size_t scratch = 0;
};

// CTAs of a bucket's kernel that fit in one SM's shared memory: the register budget per thread
// is set so that registers do not lower the residency further.
template <int SET, int OP>
struct QueueFit {
    static constexpr int fit = (int)(Q_SM_SMEM / (QueueCfg<SET, OP>::smem + Q_CTA_RESERVED));
    static constexpr int MINB = fit > 8 ? 8 : (fit < 1 ? 1 : fit);
};

using QueueOps = mayo_b200_queue_ops;

struct QueueArgs {
    QueueOps ops;
    uint32_t *slots;
    uint32_t capacity;
    uint32_t *ctrl;  // [0] head, [1] tail, [2] done, [3] error, [4] pushes
    uint8_t *scratch;
    size_t scratch_stride;
    uint32_t spin_limit;
};

__device__ __forceinline__ uint32_t ld_volatile(const uint32_t *p) { return *reinterpret_cast<const volatile uint32_t *>(p); }

__device__ __forceinline__ void queue_error(uint32_t *ctrl, uint32_t code) { atomicCAS(&ctrl[3], 0u, code); }

// Take the next item.  Near the end of a bucket head moves by compare-and-swap and only while
// head < tail, so no ticket is handed out past the published items and a CTA that finds its
// bucket empty leaves at once, freeing its SM for the other buckets' kernels.  A sign re-enqueued
// later is still served: the CTA that pushed it keeps popping, and it either takes the item
// itself or finds it taken by another CTA.  While at least gridDim items remain, head moves by
// atomicAdd (no retries under contention); such a ticket can overshoot the tail only if other
// CTAs popped several times in between, and then it waits, as every ticket past the tail must,
// for a push into its slot or for the bucket to drain (done == tail: `done` is read first, so a
// push from an unfinished item cannot be missed).  Every wait is bounded by spin_limit.
__device__ uint32_t queue_wait_slot(const QueueArgs &q, uint32_t h, uint32_t &it) {
    for (;; it++) {
        const uint32_t v = ld_volatile(&q.slots[h]);
        if (v != Q_EMPTY) {
            __threadfence();
            return v;
        }
        const uint32_t done = ld_volatile(&q.ctrl[2]);
        __threadfence();
        const uint32_t tail = ld_volatile(&q.ctrl[1]);
        if (h >= tail && done == tail) return Q_STOP;  // drained: no unfinished item can push
        if (it >= q.spin_limit) {
            queue_error(q.ctrl, MAYO_B200_QUEUE_ERR_TIMEOUT);
            return Q_STOP;
        }
        __nanosleep(100);
    }
}

__device__ uint32_t queue_pop(const QueueArgs &q) {
    uint32_t it = 0;
    for (;;) {
        const uint32_t h = ld_volatile(&q.ctrl[0]);
        const uint32_t t = ld_volatile(&q.ctrl[1]);
        const uint32_t lim = t < q.capacity ? t : q.capacity;
        if (h >= lim) return Q_STOP;
        if (lim - h >= gridDim.x) {
            const uint32_t h2 = atomicAdd(&q.ctrl[0], 1u);
            return h2 < q.capacity ? queue_wait_slot(q, h2, it) : Q_STOP;
        }
        if (atomicCAS(&q.ctrl[0], h, h + 1) == h) return queue_wait_slot(q, h, it);
        if (++it >= q.spin_limit) {  // lost the race that many times
            queue_error(q.ctrl, MAYO_B200_QUEUE_ERR_TIMEOUT);
            return Q_STOP;
        }
    }
}

__device__ void queue_push(const QueueArgs &q, uint32_t item) {
    const uint32_t slot = atomicAdd(&q.ctrl[1], 1u);
    if (slot >= q.capacity) {
        queue_error(q.ctrl, MAYO_B200_QUEUE_ERR_FULL);
        atomicAdd(&q.ctrl[2], 1u);  // the item is dropped: count it as finished
        return;
    }
    atomicAdd(&q.ctrl[4], 1u);
    __threadfence();
    *reinterpret_cast<volatile uint32_t *>(&q.slots[slot]) = item;
}

// Operands of one instance, checked against the counts and key tables the caller declared.
struct ItemRefs {
    const uint8_t *key;
    const uint8_t *msg;
    uint32_t mlen;
    bool ok;
};

template <int SET, int OP>
__device__ ItemRefs queue_refs(const QueueOps &o, uint32_t inst) {
    using S = Set<SET>;
    ItemRefs r{nullptr, nullptr, 0, false};
    if (OP == MAYO_B200_OP_KEYPAIR) {
        r.ok = inst < o.kp_count && o.kp_seed && o.kp_pk;
        return r;
    }
    constexpr bool sg = OP == MAYO_B200_OP_SIGN;
    const uint8_t *keys = sg ? o.sg_esk : o.vf_epk;
    const uint32_t nkeys = sg ? o.sg_nkeys : o.vf_nkeys, count = sg ? o.sg_count : o.vf_count;
    const uint32_t *kidx = sg ? o.sg_key : o.vf_key;
    const uint8_t *msgs = sg ? o.sg_msg : o.vf_msg;
    const uint64_t *moff = sg ? o.sg_msg_off : o.vf_msg_off;
    const uint32_t *mlen = sg ? o.sg_msg_len : o.vf_msg_len;
    const uint32_t stride = sg ? o.sg_mlen : o.vf_mlen;
    const bool outs = sg ? o.sg_sig != nullptr : (o.vf_sig != nullptr && o.vf_res != nullptr);
    if (inst >= count || !keys || nkeys == 0 || !outs) return r;
    const uint32_t k = kidx ? kidx[inst] : inst % nkeys;
    if (k >= nkeys) return r;
    r.key = keys + (size_t)k * (sg ? S::esk : S::epk);
    r.mlen = mlen ? mlen[inst] : stride;
    r.msg = msgs ? msgs + (moff ? moff[inst] : (uint64_t)inst * stride) : nullptr;
    r.ok = r.msg != nullptr || r.mlen == 0;
    if (!r.msg) r.msg = keys;  // zero-length message: any readable address
    return r;
}

// ---- keypair from a caller seed on one CTA: hash (warp 0), AES-CTR (all), P3 (engine) ----
template <int SET>
__device__ void queue_keypair(uint8_t *smem, int tid, const QueueOps &ops, uint32_t inst, uint8_t *scratch) {
    using S = Set<SET>;
    using QC = QueueCfg<SET, MAYO_B200_OP_KEYPAIR>;
    constexpr int NT = QC::NT;
    const uint8_t *seed = ops.kp_seed + (size_t)inst * S::sk;
    uint8_t *pk = ops.kp_pk + (size_t)inst * S::pk;
    uint8_t *s_O = smem + QC::KC::off_o;
    uint8_t *s_seedpk = smem + QC::seedpk;
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
    constexpr int NTAB = QueueCfg<SET, MAYO_B200_OP_KEYPAIR>::NTAB;
    uint32_t *T = reinterpret_cast<uint32_t *>(smem);
    uint32_t *rk_s = T + NTAB * 256 * 32;
    // warp 0's lane 0 runs the (serial) key schedule while the other warps build the tables
    if (tid == 0) aes128_key_schedule(s_seedpk, rk_s);
    for (int i = tid - 32; i < 256 * 32; i += NT - 32) {
        if (i < 0) break;
        const uint32_t v = c_aes.te0[i >> 5];
        T[i] = v;
        if (NTAB == 2) T[256 * 32 + i] = ror16(v);
    }
    __syncthreads();
    {
        uint32_t rk[44];
#pragma unroll
        for (int i = 0; i < 44; i++) rk[i] = rk_s[i];
        const uint32_t base = (uint32_t)__cvta_generic_to_shared(T + (tid & 31));
        const uint32_t k128 = c_aes_stride;
        const uint32_t nblk = (S::p + 15) / 16;  // the scratch has room for the whole last block
        for (uint32_t blk = tid; blk < nblk; blk += NT) {
            const AesOut o = aes128_ctr_block_t<NTAB>(base, rk, blk, k128);
            st16(scratch + (size_t)blk * 16, bswap32(o.w0), bswap32(o.w1), bswap32(o.w2), bswap32(o.w3));
        }
    }
    __syncthreads();  // scratch writes visible to the whole CTA; AES tables no longer needed
    for (int i = tid; i < 16; i += NT) pk[i] = s_seedpk[i];
    p3_instance<SET, NT, false>(smem, tid, scratch, scratch + S::p1, pk + 16);
}

template <int SET>
__device__ void queue_sign(uint8_t *smem, int tid, const QueueArgs &q, const ItemRefs &r, uint32_t inst, int ctr,
                           uint32_t item) {
    using S = Set<SET>;
    constexpr int NT = QueueCfg<SET, MAYO_B200_OP_SIGN>::NT;
    sign_hash_cta<SET, NT>(smem, tid, r.key, r.msg, r.mlen, ctr);
    const bool ok = sign_attempt<SET, NT>(smem, tid, r.key);
    if (ok || ctr >= 254) {
        // success, or the 255th rejection: the reference emits the last attempt (x = r)
        sign_write<SET, NT>(smem, tid, r.key, q.ops.sg_sig + (size_t)inst * S::sig);
    } else if (tid == 0) {
        queue_push(q, (item & ~(0xFFu << 20)) | ((uint32_t)(ctr + 1) << 20));
    }
}

template <int SET, int OP>
__global__ void __launch_bounds__(QueueCfg<SET, OP>::NT, QueueFit<SET, OP>::MINB) queue_kernel(const QueueArgs q) {
    using S = Set<SET>;
    extern __shared__ __align__(16) uint8_t smem[];
    __shared__ uint32_t s_item;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = queue_pop(q);
        __syncthreads();
        const uint32_t item = s_item;
        __syncthreads();
        if (item == Q_STOP) break;
        const uint32_t inst = item & 0xFFFFF;
        const ItemRefs r = queue_refs<SET, OP>(q.ops, inst);
        if (!r.ok) {
            if (tid == 0) queue_error(q.ctrl, MAYO_B200_QUEUE_ERR_OPERAND);
        } else if constexpr (OP == MAYO_B200_OP_KEYPAIR) {
            queue_keypair<SET>(smem, tid, q.ops, inst, q.scratch + (size_t)blockIdx.x * q.scratch_stride);
        } else if constexpr (OP == MAYO_B200_OP_SIGN) {
            queue_sign<SET>(smem, tid, q, r, inst, (int)((item >> 20) & 0xFF), item);
        } else {
            verify_instance<SET, VerifyCfg<SET>::NC>(smem, tid, r.key, r.msg, r.mlen,
                                                     q.ops.vf_sig + (size_t)inst * S::sig, q.ops.vf_res + inst);
        }
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            atomicAdd(&q.ctrl[2], 1u);
        }
    }
}

// Every bucket's slots <- empty, control words <- 0.
constexpr int Q_CTRL_TOTAL = (Q_BUCKETS + 1) * Q_CTRL_WORDS;
__global__ void queue_fill_kernel(uint32_t *slots, size_t nslots, uint32_t *ctrl) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nslots) slots[i] = Q_EMPTY;
    if (i < Q_CTRL_TOTAL) ctrl[i] = 0u;
}

// Stable partition of items[0, n) into the 12 (set, op) buckets (one CTA: per 1024-item chunk,
// warp ballots give each item's rank within its warp and bucket, a scan over the warps gives the
// warp's offset).  Items of a bucket without a kernel (`active` bit clear) are dropped with an
// operand error in that bucket's control words, items with op 3 likewise in block 12.  n_dev,
// when given, lowers n.  `phantom` (failure injection for tests) raises the tail of every bucket
// with items by one slot that stays empty, as if a push had been lost.
constexpr int Q_PART_NT = 1024;
__global__ void __launch_bounds__(Q_PART_NT) queue_partition_kernel(const uint32_t *items, uint32_t n,
                                                                    const uint32_t *n_dev, uint32_t *slots,
                                                                    uint32_t capacity, uint32_t *ctrl,
                                                                    uint32_t active, uint32_t phantom) {
    __shared__ uint32_t s_warp[Q_PART_NT / 32][Q_BUCKETS + 1];
    __shared__ uint32_t s_base[Q_BUCKETS + 1];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (n_dev) {
        const uint32_t nd = *n_dev;
        n = nd < n ? nd : n;
    }
    if (tid <= Q_BUCKETS) s_base[tid] = 0;
    __syncthreads();
    for (uint32_t start = 0; start < n; start += Q_PART_NT) {
        const uint32_t i = start + tid;
        const uint32_t it = i < n ? items[i] : 0u;
        const uint32_t op = it >> 30;
        const int b = i >= n ? -1 : (op == 3 ? Q_BUCKETS : (int)(((it >> 28) & 3) * 3 + op));
        uint32_t rank = 0;
#pragma unroll
        for (int k = 0; k <= Q_BUCKETS; k++) {
            const uint32_t bal = __ballot_sync(0xFFFFFFFFu, b == k);
            if (b == k) rank = __popc(bal & ((1u << lane) - 1u));
            if (lane == 0) s_warp[warp][k] = __popc(bal);
        }
        __syncthreads();
        if (tid <= Q_BUCKETS) {
            uint32_t acc = s_base[tid];
            for (int w = 0; w < Q_PART_NT / 32; w++) {
                const uint32_t c = s_warp[w][tid];
                s_warp[w][tid] = acc;
                acc += c;
            }
            s_base[tid] = acc;
        }
        __syncthreads();
        if (b >= 0 && b < Q_BUCKETS && ((active >> b) & 1u)) {
            const uint32_t pos = s_warp[warp][b] + rank;
            if (pos < capacity) slots[(size_t)b * capacity + pos] = it;
        }
        __syncthreads();
    }
    if (tid <= Q_BUCKETS) {
        uint32_t *c = ctrl + tid * Q_CTRL_WORDS;
        const uint32_t cnt = s_base[tid];
        if (tid == Q_BUCKETS || !((active >> tid) & 1u)) {
            c[0] = cnt;  // dropped
            if (cnt) c[3] = MAYO_B200_QUEUE_ERR_OPERAND;
        } else {
            const uint32_t t = cnt + (cnt && phantom ? 1u : 0u);
            c[1] = t < capacity ? t : capacity;
            if (cnt > capacity) c[3] = MAYO_B200_QUEUE_ERR_FULL;
        }
    }
}

// ---- host side ----
template <int SET, int OP>
int bucket_ctas_per_sm() {
    using QC = QueueCfg<SET, OP>;
    if (!set_smem_attr(queue_kernel<SET, OP>, QC::smem)) return 0;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, queue_kernel<SET, OP>, QC::NT, QC::smem) != cudaSuccess)
        return 0;
    return per_sm;
}

template <int SET, int OP>
int bucket_launch(const QueueArgs &a, uint32_t ctas, cudaStream_t st) {
    using QC = QueueCfg<SET, OP>;
    if (!set_smem_attr(queue_kernel<SET, OP>, QC::smem)) return ST_CUDA;
    queue_kernel<SET, OP><<<ctas, QC::NT, QC::smem, st>>>(a);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

// Per bucket: residency (`launch` false) or launch.
template <int SET, int OP>
int bucket_call(bool launch, const QueueArgs *a, uint32_t ctas, cudaStream_t st) {
    return launch ? bucket_launch<SET, OP>(*a, ctas, st) : bucket_ctas_per_sm<SET, OP>();
}

template <int SET>
int bucket_call_op(int op, bool launch, const QueueArgs *a, uint32_t ctas, cudaStream_t st) {
    switch (op) {
        case MAYO_B200_OP_KEYPAIR: return bucket_call<SET, MAYO_B200_OP_KEYPAIR>(launch, a, ctas, st);
        case MAYO_B200_OP_SIGN: return bucket_call<SET, MAYO_B200_OP_SIGN>(launch, a, ctas, st);
        default: return bucket_call<SET, MAYO_B200_OP_VERIFY>(launch, a, ctas, st);
    }
}

int bucket_dispatch(int b, bool launch, const QueueArgs *a = nullptr, uint32_t ctas = 0, cudaStream_t st = nullptr) {
    const int si = b / 3, op = b % 3;
    switch (si) {
        case 0: return bucket_call_op<1>(op, launch, a, ctas, st);
        case 1: return bucket_call_op<2>(op, launch, a, ctas, st);
        case 2: return bucket_call_op<3>(op, launch, a, ctas, st);
        default: return bucket_call_op<5>(op, launch, a, ctas, st);
    }
}

size_t keypair_scratch(int si) {
    switch (si) {
        case 0: return QueueCfg<1, MAYO_B200_OP_KEYPAIR>::scratch;
        case 1: return QueueCfg<2, MAYO_B200_OP_KEYPAIR>::scratch;
        case 2: return QueueCfg<3, MAYO_B200_OP_KEYPAIR>::scratch;
        default: return QueueCfg<5, MAYO_B200_OP_KEYPAIR>::scratch;
    }
}

// Streams and events the kernels fork onto, per host thread, device and caller stream (created
// on the first call, outside any graph capture, and kept for the life of the thread), so that
// runs issued on different caller streams stay concurrent.  Past Q_FORK_SETS caller streams the
// last set is shared: still correct (its streams keep the runs in issue order), only serialised.
struct ForkSet {
    int dev = -1;
    cudaStream_t caller = nullptr;
    cudaStream_t s[Q_BUCKETS];
    cudaEvent_t fork, join[Q_BUCKETS];
};
constexpr int Q_FORK_SETS = 16;
thread_local ForkSet tl_fork[Q_FORK_SETS];
thread_local int tl_fork_used = 0;

ForkSet *fork_set(int dev, cudaStream_t caller) {
    for (int i = 0; i < tl_fork_used; i++)
        if (tl_fork[i].dev == dev && tl_fork[i].caller == caller) return &tl_fork[i];
    if (tl_fork_used == Q_FORK_SETS) {
        for (int i = Q_FORK_SETS - 1; i >= 0; i--)
            if (tl_fork[i].dev == dev) return &tl_fork[i];
        return nullptr;
    }
    ForkSet &f = tl_fork[tl_fork_used];
    for (int i = 0; i < Q_BUCKETS; i++)
        if (cudaStreamCreateWithFlags(&f.s[i], cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&f.join[i], cudaEventDisableTiming) != cudaSuccess)
            return nullptr;
    if (cudaEventCreateWithFlags(&f.fork, cudaEventDisableTiming) != cudaSuccess) return nullptr;
    f.dev = dev;
    f.caller = caller;
    tl_fork_used++;
    return &f;
}

}  // namespace mayo

// ---- C-ABI ----
namespace {
constexpr size_t kCtrlBytes = 1024;
static_assert(mayo::Q_CTRL_TOTAL * 4 <= kCtrlBytes, "control words");
// Default launch order: the buckets with the longest items first, so the short ones fill the
// tails (measured per-item times on B200, longest first).
constexpr uint8_t kDefaultOrder[mayo::Q_BUCKETS] = {9, 10, 11, 6, 7, 8, 0, 3, 1, 2, 4, 5};

size_t slots_bytes(uint32_t capacity) { return (((size_t)capacity * 4) + 255) / 256 * 256; }

int device_sms(int *dev) {
    if (cudaGetDevice(dev) != cudaSuccess) return 0;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, *dev) != cudaSuccess) return 0;
    return sms;
}

// Residency of every bucket's kernel and the byte offsets of the four keypair buckets' scratch
// (after the control words and all slots), each sized for sms x its maximal residency.
bool queue_layout(uint32_t capacity, uint32_t sms, int per_sm[mayo::Q_BUCKETS], size_t off[5]) {
    for (int b = 0; b < mayo::Q_BUCKETS; b++) {
        per_sm[b] = mayo::bucket_dispatch(b, false);
        if (per_sm[b] <= 0) return false;
    }
    off[0] = kCtrlBytes + mayo::Q_BUCKETS * slots_bytes(capacity);
    for (int si = 0; si < 4; si++)
        off[si + 1] = off[si] + (size_t)sms * per_sm[si * 3 + MAYO_B200_OP_KEYPAIR] * mayo::keypair_scratch(si);
    return true;
}

bool bucket_active(const mayo_b200_queue_ops &o, int op) {
    if (op == MAYO_B200_OP_KEYPAIR) return o.kp_seed && o.kp_pk;
    if (op == MAYO_B200_OP_SIGN) return o.sg_esk && o.sg_sig;
    return o.vf_epk && o.vf_sig && o.vf_res;
}
}  // namespace

extern "C" {

MAYO_B200_API size_t mayo_b200_queue_mem_bytes(uint32_t capacity, uint32_t sms) {
    int dev = 0;
    const int dsms = device_sms(&dev);
    if (!dsms) return 0;
    if (!sms) sms = (uint32_t)dsms;
    int per_sm[mayo::Q_BUCKETS];
    size_t off[5];
    if (!queue_layout(capacity, sms, per_sm, off)) return 0;
    return off[4];
}

MAYO_B200_API int mayo_b200_queue_ctas_per_sm(int set, int op) {
    const int si = set == 1 ? 0 : set == 2 ? 1 : set == 3 ? 2 : set == 5 ? 3 : -1;
    if (si < 0 || op < 0 || op > 2) return 0;
    return mayo::bucket_dispatch(si * 3 + op, false);
}

MAYO_B200_API int mayo_b200_queue_run(const mayo_b200_queue_ops ops[4], const uint32_t *items, uint32_t n,
                                      const uint32_t *n_device, void *queue_mem, uint32_t capacity,
                                      const mayo_b200_queue_shape *shape, uint32_t spin_limit, void *stream) {
    using mayo::Q_BUCKETS;
    if (!ops || !queue_mem || (n && !items) || n > capacity || capacity == 0 || capacity > (1u << 28))
        return MAYO_B200_ERR_ARG;
    int dev = 0;
    const int dsms = device_sms(&dev);
    if (!dsms) return MAYO_B200_ERR_CUDA;
    const uint32_t sms = shape && shape->sms ? shape->sms : (uint32_t)dsms;
    int per_sm[Q_BUCKETS];
    size_t off[5];
    if (!queue_layout(capacity, sms, per_sm, off)) return MAYO_B200_ERR_CUDA;
    uint8_t order[Q_BUCKETS];
    for (int k = 0; k < Q_BUCKETS; k++) order[k] = kDefaultOrder[k];
    if (shape) {
        bool seen[Q_BUCKETS] = {}, perm = true;
        for (int k = 0; k < Q_BUCKETS; k++) {
            const uint8_t v = shape->launch_order[k];
            if (v >= Q_BUCKETS || seen[v]) perm = false;
            else seen[v] = true;
        }
        if (perm)
            for (int k = 0; k < Q_BUCKETS; k++) order[k] = shape->launch_order[k];
        for (int b = 0; b < Q_BUCKETS; b++)
            if (shape->ctas_per_sm[b] > per_sm[b]) return MAYO_B200_ERR_ARG;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    mayo::ForkSet *fs = mayo::fork_set(dev, st);
    if (!fs) return MAYO_B200_ERR_CUDA;

    uint8_t *base = static_cast<uint8_t *>(queue_mem);
    uint32_t *ctrl = reinterpret_cast<uint32_t *>(base);
    uint32_t *slots = reinterpret_cast<uint32_t *>(base + kCtrlBytes);
    const uint32_t cap_words = (uint32_t)(slots_bytes(capacity) / 4);  // each bucket's slots (padded)
    const size_t nslots = (size_t)cap_words * Q_BUCKETS;
    uint32_t active = 0;
    for (int b = 0; b < Q_BUCKETS; b++)
        if (bucket_active(ops[b / 3], b % 3)) active |= 1u << b;

    const size_t fill_n = nslots > (size_t)mayo::Q_CTRL_TOTAL ? nslots : (size_t)mayo::Q_CTRL_TOTAL;
    mayo::queue_fill_kernel<<<(unsigned)((fill_n + 255) / 256), 256, 0, st>>>(slots, nslots, ctrl);
    const uint32_t phantom = mayo::inject().kind == MAYO_B200_INJECT_QUEUE_LOST_PUSH ? 1u : 0u;
    mayo::queue_partition_kernel<<<1, mayo::Q_PART_NT, 0, st>>>(items, n, n_device, slots, cap_words, ctrl, active,
                                                                phantom);
    if (cudaPeekAtLastError() != cudaSuccess || cudaEventRecord(fs->fork, st) != cudaSuccess) return MAYO_B200_ERR_CUDA;
    int k = 0;
    for (int j = 0; j < Q_BUCKETS; j++) {
        const int b = order[j];
        if (!(active & (1u << b))) continue;
        cudaStream_t s = fs->s[k];
        if (cudaStreamWaitEvent(s, fs->fork, 0) != cudaSuccess) return MAYO_B200_ERR_CUDA;
        const uint32_t per = shape && shape->ctas_per_sm[b] ? shape->ctas_per_sm[b] : (uint32_t)per_sm[b];
        mayo::QueueArgs a{};
        a.ops = ops[b / 3];
        a.slots = slots + (size_t)b * cap_words;
        a.capacity = cap_words;
        a.ctrl = ctrl + b * mayo::Q_CTRL_WORDS;
        a.scratch = b % 3 == MAYO_B200_OP_KEYPAIR ? base + off[b / 3] : nullptr;
        a.scratch_stride = mayo::keypair_scratch(b / 3);
        a.spin_limit = spin_limit ? spin_limit : (1u << 24);
        if (mayo::bucket_dispatch(b, true, &a, per * sms, s) != mayo::ST_OK) return MAYO_B200_ERR_CUDA;
        if (cudaEventRecord(fs->join[k], s) != cudaSuccess || cudaStreamWaitEvent(st, fs->join[k], 0) != cudaSuccess)
            return MAYO_B200_ERR_CUDA;
        k++;
    }
    return MAYO_B200_OK;
}

}  // extern "C"
