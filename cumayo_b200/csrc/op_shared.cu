// op_shared.cu -- sign / verify of a batch under ONE key, with the key's heavy products on the
// tensor cores (tcgen05.mma, kind::i8).
//
// The per-instance engine (engine.cuh) spends most of a signature on T_j[r] = sum_c P1[r][c] V_j[c]
// (U = V^T P1 V) and M_j[b] = sum_a V_j[a] L[a][b] (src/sign.cu:254-330, 396-437), and most of a
// verification on T_j[r] = sum_c P[r][c] s_j[c] (src/verify.cu:72-182).  When every instance of a
// batch uses the same key these are one matrix product over the whole batch: GF(16) is GF(2)^4,
// multiplication by a field element a is the 4x4 bit matrix Mul(a)[b][b'] = bit b of (a * x^b'),
// so with every entry expanded to its bit matrix
//     bit b of coordinate t of T_j[r]  =  sum over (c, b') of  Mul(P[r][c]_t)[b][b'] * bit b' of V_j[c]   (mod 2)
// -- a 0/1 matrix A (rows (r, t, b), columns (c, b')) times a 0/1 matrix B (rows (c, b'),
// columns (instance, j)).  A is stored as 0 / 128, so the tensor cores' exact s32 sums are
// 128 x the integer sums and the epilogue keeps bit 7 of each.
//
// Kernels:
//   shared_a_kernel     builds A from the key, tiled for the MMA (one 128-row tile = the four bit
//                       planes of one 32-coordinate group of one row r) in the K-major, no-swizzle
//                       shared-memory layout, so a run of k-steps of a tile moves to shared memory
//                       with one bulk copy; for sign also the key's O planes.
//   shared_gemm_kernel  one CTA per 256 instance vectors (B, built in shared memory from their
//                       nibbles, resident): a loader warp streams A through a ring of chunks, two
//                       issuer warps run the MMAs of alternate tiles into two TMEM accumulators,
//                       and eight warps read an accumulator back (tcgen05.ld, 16-bit halves),
//                       gather bit 7 of 32 sums into one word -- one 32-coordinate bit plane -- and
//                       store the planes.  Zero blocks of A (columns c < r of the triangular P1 / P)
//                       are skipped.  Waits are bounded: a timeout sets the status word and unwinds.
//   Messages of different lengths: hash_order_count/scatter_kernel first group the instances by
//   SHAKE256 block count, and the hash kernels take them in that order.
//   sign: sign_hash_kernel (thread per instance) -> product -> sign_shared_tail_kernel (first
//         attempt from the planes in a compact CTA) -> sign_shared_fix_kernel (retries of the
//         rare singular first attempts with the engine).
//   verify: verify_hash_kernel (thread per instance: digest, t) -> product ->
//         verify_shared_tail_kernel (U from the planes, Horner, compare; a small CTA).
//   If the status word shows a failed product, the tails do nothing and the fix-up kernels run
//   every instance through the per-instance engine, so results stay correct.
#include <cuda_runtime.h>

#include <atomic>

#include "../../include/mayo_b200.h"
#include "launch_util.cuh"
#include "ops.h"
#include "sign_body.cuh"
#include "tc.cuh"
#include "verify_body.cuh"

namespace mayo {

constexpr uint32_t SH_SPIN = 1u << 22;  // mbarrier polls before a wait gives up
constexpr size_t SH_SMEM_MAX = 226 * 1024;
constexpr int SH_EPI_NT = 256;              // 8 epilogue warps: warp w reads TMEM lanes 32 (w % 4).., half w / 4
constexpr int SH_ISSUE_WARP = SH_EPI_NT / 32;       // warps 8, 9: MMA issuers (even / odd tiles)
constexpr int SH_LOAD_WARP = SH_ISSUE_WARP + 2;     // warp 10: key loader
constexpr int SH_GEMM_NT = SH_EPI_NT + 96;
constexpr int SH_FIX_CTAS = 2 * 148;
constexpr int ORD_CTAS = 64, ORD_NT = 256, ORD_BINS = 8;  // hashing-order sort: grid cap, threads, bins

// The product for sign (rows: T_j[r] over P1 for r < v, then M_j[b] over L) or verify (rows
// T_j[r] over [[P1, P2], [0, P3]] for r < n).
template <int SET, bool VERIFY>
struct SharedProb {
    using S = Set<SET>;
    static constexpr int W = S::W;
    static constexpr int NVEC = VERIFY ? S::n : S::v;         // entries of one vector V_j / s_j
    static constexpr int NROWS = VERIFY ? S::n : S::v + S::o;  // m-vector rows of the result
    static constexpr int KPAD = (4 * NVEC + 31) / 32 * 32;    // bytes of one B column (K)
    static constexpr int KSTEPS = KPAD / 32;                   // MMAs of K = 32 per tile
    static constexpr int NGROUPS = NROWS * W;  // 128-row groups of the key matrix (row rr, group w)
    // One MMA: M = 128 vector columns, N = 128 key rows (one group), K = 32.  NB = 2 M-blocks of
    // vectors share every k-step of key rows, so each key byte brought into shared memory feeds
    // 256 vector columns (the key stream from L2 is what bounds this kernel); an accumulator takes
    // NB x 128 = 256 TMEM columns (two of them: double-buffered).  The key rows stream through a
    // ring of NCH chunks of up to CK k-steps of one tile (one bulk copy, one commit each: more
    // frequent commits stall the tensor pipe; a chunk never spans two tiles, so its MMAs take
    // compile-time descriptor offsets -- the single issuing thread cannot afford more than a few
    // instructions per MMA).
    static constexpr int G = 1;
    static constexpr int NINST = 256;
    static constexpr int KROWS = 128 * G;
    static constexpr size_t SLOT = (size_t)2 * KROWS * 16;  // one k-step of key rows: [2][KROWS][16 B]
    static constexpr size_t BAR_BYTES = 1024;               // mbarriers (2 NCH + 6) and flags
    static constexpr int nch_fit(int ck) { return (int)((SH_SMEM_MAX - (size_t)NINST * KPAD - BAR_BYTES) / (ck * SLOT)); }
    // k-steps per chunk: a tile's k-steps in near-equal chunks of at most 8 (MAYO_2 verify, 11
    // k-steps: 6 + 5 takes 0.96 ms where 8 + 3 takes 0.99), or 4 when fewer than three 8-step
    // chunks fit beside the vectors
    static constexpr int CK_EVEN = (KSTEPS + (KSTEPS + 7) / 8 - 1) / ((KSTEPS + 7) / 8);
    static constexpr int CK = nch_fit(8) >= 3 ? CK_EVEN : 4;
    static constexpr int NCH_FIT = nch_fit(CK);
    static constexpr int NCH = NCH_FIT < 16 ? NCH_FIT : 16;
    static_assert(NCH >= 2, "key ring");
    static_assert((2 * NCH + 6) * 8 + 12 <= (int)BAR_BYTES, "barrier area");
    static constexpr int NTILES = (NGROUPS + G - 1) / G;
    static constexpr size_t TILE = (size_t)KROWS * KPAD;
    static constexpr int NB = NINST / 128;  // MMA M-blocks of 128 vector columns
    static constexpr int NI = NINST / S::k; // instances per CTA
    static constexpr size_t SMEM = (size_t)NINST * KPAD + (size_t)NCH * CK * SLOT + BAR_BYTES;
    static_assert(NB * KROWS <= 256, "accumulator columns");
    static constexpr size_t PLANES = (size_t)S::k * NROWS * W;  // uint4 per instance
    // first column c that can be nonzero in row rr
    __host__ __device__ static constexpr int c_min(int rr) { return VERIFY ? rr : (rr < S::v ? rr : 0); }
    // coordinate t of entry (rr, c) of the key matrix, 0 where it is structurally zero
    __device__ static uint32_t entry(const uint8_t *key, int rr, int c, int t) {
        const uint8_t *e = nullptr;
        if (VERIFY) {  // key = epk = P1 || P2 || P3
            if (c >= rr) {
                if (rr < S::v)
                    e = c < S::v ? key + (size_t)tri(rr, c, S::v) * S::menc
                                 : key + S::p1 + (size_t)(rr * S::o + (c - S::v)) * S::menc;
                else
                    e = key + S::p1 + S::p2 + (size_t)tri(rr - S::v, c - S::v, S::o) * S::menc;
            }
        } else {  // key = esk = seed_sk || O || P1 || L
            const uint8_t *P1 = key + S::sk + S::o_bytes, *L = P1 + S::p1;
            if (rr < S::v) {
                if (c >= rr) e = P1 + (size_t)tri(rr, c, S::v) * S::menc;
            } else {
                e = L + (size_t)(c * S::o + (rr - S::v)) * S::menc;
            }
        }
        return e ? (e[t >> 1] >> ((t & 1) * 4)) & 0xFu : 0u;
    }
};

// The same product on a CTA pair (shared_gemm2_kernel, tcgen05 cta_group::2): each MMA has
// M = 256 vector columns (128 from each CTA) and N = 128 key rows of which each CTA holds 64, so
// each SM streams half of every key tile.  A tile is stored as two halves, [half][K / 16][64][16]
// (half 0 = bit planes 0-1, rows 0-63; half 1 = planes 2-3): a CTA's chunk of k-steps is one
// contiguous run of SLOT2-byte k-steps in its half.
template <int SET, bool VERIFY>
struct PairProb {
    using P = SharedProb<SET, VERIFY>;
    static constexpr int HROWS = 64;                                  // key rows per CTA and tile
    static constexpr size_t SLOT2 = (size_t)2 * HROWS * 16;           // one k-step of them
    static constexpr size_t HALF = P::TILE / 2;                       // bytes of a tile half
    static constexpr int nch_fit(int ck) {
        return (int)((SH_SMEM_MAX - (size_t)P::NINST * P::KPAD - P::BAR_BYTES) / (ck * SLOT2));
    }
    // k-steps per chunk: a whole tile where four such chunks fit beside the vectors (a CTA holds
    // half of each k-step, so they fit for MAYO_1/2/3), else the one-CTA kernel's split.  One chunk
    // per tile halves the issuers' chunk checks and commits: at 65,536 instances MAYO_2 verify
    // 0.746 -> 0.699 ms, MAYO_1 sign 2.98 -> 2.65 ms, MAYO_3 sign 6.54 -> 6.40 ms.
    static constexpr int CK = nch_fit(P::KSTEPS) >= 4 ? P::KSTEPS : P::CK_EVEN;
    static constexpr int NCH = nch_fit(CK) < 16 ? nch_fit(CK) : 16;
    static_assert(NCH >= 2, "key ring");
    static_assert((3 * NCH + 7) * 8 + 12 <= (int)P::BAR_BYTES, "barrier area");
    static constexpr size_t SMEM = (size_t)P::NINST * P::KPAD + (size_t)NCH * CK * SLOT2 + P::BAR_BYTES;
};

// Workspace: control words ([0] status: 0 = product ran, 1 = it gave up; [1] sign retries), A
// tiles, (sign) the O planes of the key, per-instance hash results (sign: digest, salt, t, V || r; verify: t), per-instance
// planes, (sign) the list of instances whose first attempt was singular.
template <int SET, bool VERIFY>
struct SharedWs {
    using P = SharedProb<SET, VERIFY>;
    static constexpr int NW = (Set<SET>::menc + 3) / 4;
    static constexpr size_t a = 256;
    static constexpr size_t a_bytes = (size_t)P::NTILES * P::TILE;
    static constexpr int OPL = VERIFY ? 0 : Set<SET>::o * Set<SET>::W;  // O planes (sign), uint4 items
    static constexpr size_t op_bytes = (size_t)OPL * 16;
    static constexpr size_t inst = VERIFY ? pad16((size_t)NW * 4) : pad16(SignWs<SET>::total);
    static constexpr size_t planes = P::PLANES * 16;
    static constexpr size_t retry = VERIFY ? 0 : 4;
    static constexpr size_t order = 4;  // hashing order (instances grouped by message blocks)
    static constexpr size_t hist_bytes = (size_t)ORD_CTAS * ORD_BINS * 4;
    static constexpr size_t head = a + a_bytes + op_bytes + hist_bytes;
    static size_t bytes(size_t batch) { return head + batch * (inst + planes + retry + order); }
    static size_t op_off() { return a + a_bytes; }
    static size_t hist_off() { return a + a_bytes + op_bytes; }
    static size_t inst_off() { return head; }
    static size_t planes_off(size_t batch) { return head + batch * inst; }
    static size_t retry_off(size_t batch) { return head + batch * (inst + planes); }
    static size_t order_off(size_t batch) { return head + batch * (inst + planes + retry); }
};

// ---- hashing order ----
// The hash kernels run one instance per thread, and a warp runs as many Keccak-f permutations as
// its longest message needs.  With lengths that differ per instance, a counting sort by the
// number of SHAKE256 blocks of the message (capped at ORD_BINS - 1 full blocks) lets each warp
// hash messages of one size class.  Each instance's outputs go to its own workspace row, so the
// order changes no byte.  Two launches: per-CTA bin counts over a contiguous chunk, then a
// scatter from each (bin, CTA) start.
__device__ __forceinline__ uint32_t msg_bin(const MsgIO &m, uint32_t i) {
    const uint32_t b = m.len(i) / 136;
    return b < (uint32_t)ORD_BINS - 1 ? b : (uint32_t)ORD_BINS - 1;
}
__device__ __forceinline__ void ord_chunk(uint32_t batch, uint32_t &b0, uint32_t &b1) {
    const uint32_t per = (batch + gridDim.x - 1) / gridDim.x;
    b0 = blockIdx.x * per;
    b1 = b0 + per < batch ? b0 + per : batch;
}
__global__ void __launch_bounds__(ORD_NT) hash_order_count_kernel(const MsgIO m, uint32_t batch, uint32_t *hist) {
    __shared__ uint32_t h[ORD_BINS];
    if (threadIdx.x < ORD_BINS) h[threadIdx.x] = 0;
    __syncthreads();
    uint32_t b0, b1;
    ord_chunk(batch, b0, b1);
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += ORD_NT) atomicAdd(&h[msg_bin(m, i)], 1u);
    __syncthreads();
    if (threadIdx.x < ORD_BINS) hist[blockIdx.x * ORD_BINS + threadIdx.x] = h[threadIdx.x];
}
__global__ void __launch_bounds__(ORD_NT)
    hash_order_scatter_kernel(const MsgIO m, uint32_t batch, const uint32_t *hist, uint32_t *order) {
    __shared__ uint32_t cur[ORD_BINS];
    if (threadIdx.x < 32) {  // start of (bin t, this CTA): every lower bin, then bin t of earlier CTAs
        uint32_t acc[ORD_BINS];
#pragma unroll
        for (int t = 0; t < ORD_BINS; t++) acc[t] = 0;
        for (uint32_t c = threadIdx.x; c < gridDim.x; c += 32)
#pragma unroll
            for (int b = 0; b < ORD_BINS; b++) {
                const uint32_t v = hist[c * ORD_BINS + b];
#pragma unroll
                for (int t = 0; t < ORD_BINS; t++) acc[t] += (b < t || (b == t && c < blockIdx.x)) ? v : 0u;
            }
#pragma unroll
        for (int t = 0; t < ORD_BINS; t++) {
            const uint32_t tot = __reduce_add_sync(0xffffffffu, acc[t]);
            if (threadIdx.x == 0) cur[t] = tot;
        }
    }
    __syncthreads();
    uint32_t b0, b1;
    ord_chunk(batch, b0, b1);
    for (uint32_t i = b0 + threadIdx.x; i < b1; i += ORD_NT) order[atomicAdd(&cur[msg_bin(m, i)], 1u)] = i;
}
// The order for a call, or nullptr when every message has the same length (nothing to group).
template <int SET, bool VERIFY>
static const uint32_t *launch_hash_order(const MsgIO &m, uint8_t *ws, size_t batch, cudaStream_t st) {
    using WSL = SharedWs<SET, VERIFY>;
    if (!m.msg_len || batch < 2 * (size_t)HASH_NT) return nullptr;
    const size_t want = (batch + ORD_NT - 1) / ORD_NT;
    const unsigned g = (unsigned)(want < (size_t)ORD_CTAS ? want : (size_t)ORD_CTAS);
    uint32_t *hist = reinterpret_cast<uint32_t *>(ws + WSL::hist_off());
    uint32_t *order = reinterpret_cast<uint32_t *>(ws + WSL::order_off(batch));
    hash_order_count_kernel<<<g, ORD_NT, 0, st>>>(m, (uint32_t)batch, hist);
    hash_order_scatter_kernel<<<g, ORD_NT, 0, st>>>(m, (uint32_t)batch, hist, order);
    return order;
}

// A, tiled: group gi = rr * W + w holds rows rho = 32 b + q (bit plane b; row q carries coordinate
// 32 w + cq(q), cq(q) = 8 ((q >> 2) & 3) + 2 (q & 3) + (q >> 4), the order in which the epilogue's
// packing of 32 sums lands each coordinate on its bit of a G4 plane) and K bytes 4 c + b'; a
// tile is G consecutive groups, layout [K / 16][G * 128 rows][16 bytes].  One thread per 16
// bytes (PAIR: the two halves of PairProb).  Also resets the control words and (sign) writes
// the key's O planes after the tiles, one thread per item.
template <int SET, bool VERIFY, bool PAIR>
__global__ void shared_a_kernel(const uint8_t *key, uint8_t *A, uint32_t *ctl, uint4 *opl) {
    using P = SharedProb<SET, VERIFY>;
    using S = Set<SET>;
    constexpr size_t per_group = (size_t)(P::KPAD / 16) * 128;
    constexpr size_t a_items = (size_t)P::NTILES * P::G * per_group;
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < 2) ctl[idx] = 0;
    if (idx >= a_items) {
        if constexpr (!VERIFY) {  // key = esk = seed_sk || O || P1 || L
            if (idx < a_items + (size_t)SharedWs<SET, false>::OPL)
                g4_st(opl + (idx - a_items), o_plane_item<SET>(key + S::sk, (int)(idx - a_items)));
        }
        return;
    }
    const int gi = (int)(idx / per_group);  // group (the last tile's second group may be padding)
    const int rem = (int)(idx - (size_t)gi * per_group);
    const int ch = rem / 128, rho = rem - ch * 128;
    const int rr = gi / P::W, w = gi - rr * P::W, b = rho >> 5, tp = rho & 31;
    const int t = 32 * w + 8 * ((tp >> 2) & 3) + 2 * (tp & 3) + (tp >> 4);
    uint32_t wd[4] = {0u, 0u, 0u, 0u};
    if (gi < P::NGROUPS && t < S::m) {
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int c = 4 * ch + q;
            if (c >= P::NVEC) continue;
            const uint32_t a = P::entry(key, rr, c, t);
            uint32_t v = 0;
#pragma unroll
            for (int bp = 0; bp < 4; bp++) v |= ((gf16_mul_ct(a, 1u << bp) >> b) & 1u) << (8 * bp + 7);
            wd[q] = v;
        }
    }
    const int tile = gi / P::G, g = gi - tile * P::G;
    if constexpr (PAIR) {
        static_assert(P::G == 1, "pair tiles hold one group");
        constexpr int H = PairProb<SET, VERIFY>::HROWS;
        *reinterpret_cast<uint4 *>(A + (size_t)tile * P::TILE + (size_t)(rho / H) * PairProb<SET, VERIFY>::HALF +
                                   (size_t)ch * H * 16 + (size_t)(rho % H) * 16) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
    } else {
        *reinterpret_cast<uint4 *>(A + (size_t)tile * P::TILE + (size_t)ch * P::KROWS * 16 +
                                   (size_t)(g * 128 + rho) * 16) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
    }
}

// The key tiles hold 0 / 128, so every sum is 128 x (the GF(2) sum): bit 7 of its low byte is the
// result.  The sums come from TMEM as pairs of low 16-bit halves (tcgen05.ld .pack::16b: register
// i = sums 2i, 2i + 1 in bits 0-15, 16-31).  One permute per four sums replicates those four bit
// 7s over bytes 0-3 (byte j <- sum 4 k + j), one LOP3 keeps bit k of each byte: bit 8 j + k <-
// sum 4 k + j (the A tile's row order makes this a G4 plane).
__device__ __forceinline__ uint32_t pack_bit7x32(const uint32_t (&r)[16]) {
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) x |= tc::prmt(r[2 * k], r[2 * k + 1], 0xECA8u) & (0x01010101u << k);
    return x;
}

// Bounded wait on an mbarrier phase that also gives up as soon as another warp of the CTA has
// recorded a failure in *fail (checked every 64 polls).
__device__ __forceinline__ bool wait_or_fail(uint64_t *bar, uint32_t parity, uint32_t limit, const uint32_t *fail) {
    for (uint32_t i = 0; i < limit; i += 64) {
        if (tc::mbar_wait(bar, parity, 64)) return true;
        if (*reinterpret_cast<const volatile uint32_t *>(fail)) return false;
    }
    return false;
}

// Whole-warp forms for the MMA issuers, whose loop every lane runs so that the values the MMAs
// take stay warp-uniform; each result is the same in every lane.
constexpr uint32_t WARP_ALL = 0xFFFFFFFFu;
__device__ __forceinline__ bool warp_wait_or_fail(uint64_t *bar, uint32_t parity, uint32_t limit, const uint32_t *fail) {
    return __all_sync(WARP_ALL, wait_or_fail(bar, parity, limit, fail));
}
// The same for an mbarrier that the other CTA of a pair arrives on (acquire at cluster scope).
__device__ __forceinline__ bool warp_wait_cluster_or_fail(uint64_t *bar, uint32_t parity, uint32_t limit,
                                                          const uint32_t *fail) {
    bool seen = false;
    for (uint32_t i = 0; i < limit && !seen; i += 64) {
        seen = tc::mbar_wait_cluster(bar, parity, 64);
        if (!seen && *reinterpret_cast<const volatile uint32_t *>(fail)) break;
    }
    return __all_sync(WARP_ALL, seen);
}
__device__ __forceinline__ bool warp_flag(const uint32_t *f) {
    return __any_sync(WARP_ALL, *reinterpret_cast<const volatile uint32_t *>(f) != 0);
}
// Bounded wait until the loader has started chunk c's copy (armed the slot's barrier for it).
__device__ __forceinline__ bool warp_wait_armed(const uint32_t *loaded, uint32_t c, uint32_t limit) {
    for (uint32_t polls = 0; __any_sync(WARP_ALL, *reinterpret_cast<const volatile uint32_t *>(loaded) <= c);)
        if (++polls >= limit) return false;
    __threadfence_block();
    return true;
}

// The CTA's vector columns in shared memory, [KPAD/16][NINST][16]: column n = (instance n / k,
// vector j = n % k), K byte 4 c + b' = bit b' of entry c (0 past the vectors or the batch).
// Threads 0 .. NTH-1.  Each thread issues the loads of up to 24 items before it stores any, so
// they are in flight together (MAYO_1/2/3: all of a thread's items, one round of memory latency):
// the build is on the path before the first MMA (3.6 / 5.0 us of a MAYO_2 sign / verify pair
// CTA's 87 / 98 us with eight in flight; 0.616 -> 0.611 ms and 0.695 -> 0.684 ms with 24).
template <int SET, bool VERIFY, int NTH>
__device__ __forceinline__ void build_vector_columns(uint8_t *sB, const uint8_t *__restrict__ vec, size_t vec_stride,
                                                     uint32_t inst0, uint32_t batch, int tid) {
    using P = SharedProb<SET, VERIFY>;
    using S = Set<SET>;
    constexpr int NIN = P::NINST, ITEMS = (P::KPAD / 16) * NIN, ITER = (ITEMS + NTH - 1) / NTH, B = ITER < 24 ? ITER : 24;
#pragma unroll 1
    for (int q0 = 0; q0 < ITER; q0 += B) {
        uint32_t lo[B], hi[B], sh[B];
#pragma unroll
        for (int u = 0; u < B; u++) {
            const int idx = tid + (q0 + u) * NTH;
            const int ch = idx / NIN, n = idx - ch * NIN;
            const uint32_t inst = inst0 + (uint32_t)(n / S::k);
            const int j = n % S::k;
            lo[u] = hi[u] = sh[u] = 0;
            if (q0 + u < ITER && idx < ITEMS && n < P::NI * S::k && inst < batch && 4 * ch < P::NVEC) {
                // the item's four nibbles from one little-endian word (the bytes after a vector
                // are the next vector's, r's or the salt's, so all four exist); aligned word
                // loads only, the second one only where the word is split
                const int nib0 = j * P::NVEC + 4 * ch;
                const uintptr_t a = reinterpret_cast<uintptr_t>(vec + (size_t)inst * vec_stride + (nib0 >> 1));
                const uint32_t *w = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
                sh[u] = (uint32_t)(a & 3) * 8 + (uint32_t)(nib0 & 1) * 4;
                lo[u] = __ldg(w);
                hi[u] = (a & 3) ? __ldg(w + 1) : 0u;
            }
        }
#pragma unroll
        for (int u = 0; u < B; u++) {
            const int idx = tid + (q0 + u) * NTH;
            if (q0 + u >= ITER || idx >= ITEMS) continue;
            const int ch = idx / NIN, n = idx - ch * NIN;
            const uint32_t x4 = __funnelshift_r(lo[u], hi[u], sh[u]);  // sh <= 3 * 8 + 4
            uint32_t wd[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const uint32_t x = 4 * ch + q < P::NVEC ? (x4 >> (4 * q)) & 0xFu : 0u;
                wd[q] = (x * 0x00204081u) & 0x01010101u;  // bit b' -> byte b'
            }
            *reinterpret_cast<uint4 *>(sB + ((size_t)ch * NIN + n) * 16) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
        }
    }
}

// vec: instance i's vectors start at vec + i * vec_stride, entry c of vector j is nibble
// j * NVEC + c.  planes: instance i at planes + i * PLANES, [j][row][w].
//
// The MMA puts the vector columns on M (TMEM lanes) and the 128 rows of a key tile on N, so each
// epilogue thread owns one vector column and reads the 32 sums of one bit plane of its tile
// from its own TMEM lane: packing them into the plane's word is thread-local.
//
// Warp-specialized: one thread of warp 10 streams the key rows (a k-step = all 128 rows of a
// group, K = 32) through a ring of NCH chunks of up to CK k-steps of one tile, one bulk copy per
// chunk, refilling a chunk once the MMAs that read it completed; one thread each of warps 8 and 9
// issues the MMAs of the even / odd tiles into TMEM accumulator 0 / 1 once that accumulator has
// been read out; warps 0-7 are the epilogue -- they wait for a tile's MMAs, read their sums
// (tcgen05.ld), hand the accumulator back (acc_free), pack and store.  Barriers: full[chunk]
// (copy landed), empty[chunk] (commit: its MMAs completed), mma_done[acc] (commit), acc_free[acc]
// (8 arrivals), drain[issuer] (an issuer's last commit).  The loader starts as soon as the
// barriers exist; the others first build the vector columns.
//
// `spin` bounds the waits of the steady state (polls); the unwind waits keep SH_SPIN.
// `stall_after` is failure injection for tests: the loader silently stops after that many
// chunks, so the issuers' waits for the next chunk run out (0xFFFFFFFF: never).
template <int SET, bool VERIFY>
__global__ void __launch_bounds__(SH_GEMM_NT, 1)
    shared_gemm_kernel(const uint8_t *__restrict__ A, const uint8_t *__restrict__ vec, size_t vec_stride,
                       uint4 *__restrict__ planes, uint32_t batch, uint32_t *ctl, uint32_t spin,
                       uint32_t stall_after) {
    using P = SharedProb<SET, VERIFY>;
    using S = Set<SET>;
    constexpr int NIN = P::NINST, KPAD = P::KPAD, NT = P::NTILES, NB = P::NB, G = P::G;
    constexpr int KR = P::KROWS;
    constexpr uint32_t NCH = (uint32_t)P::NCH, CK = (uint32_t)P::CK, SLOT = (uint32_t)P::SLOT;
    constexpr uint32_t IDESC = tc::idesc_u8(128, KR);
    constexpr uint32_t ACC = KR * NB;  // TMEM columns of one accumulator
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sB = smem;                                            // [KPAD/16][NIN][16] vector columns
    uint8_t *ring = smem + (size_t)NIN * KPAD;                      // NCH x CK x [2][KR][16] key rows
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + (size_t)NCH * CK * SLOT);  // [NCH]
    uint64_t *empty = full + NCH;                                   // [NCH]
    uint64_t *mma_done = empty + NCH;                               // [2]
    uint64_t *acc_free = mma_done + 2;                              // [2]
    uint64_t *drain = acc_free + 2;                                 // [2]
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(drain + 2);
    uint32_t *s_fail = s_tmem + 1;
    uint32_t *s_loaded = s_tmem + 2;  // chunks whose copy the loader has started (armed full[])
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t inst0 = blockIdx.x * (uint32_t)P::NI;

    if (tid == 0) {
        for (uint32_t i = 0; i < NCH; i++) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            tc::mbar_init(&mma_done[i], 1);
            tc::mbar_init(&acc_free[i], SH_EPI_NT / 32);
        }
        tc::mbar_init(&drain[0], 1);
        tc::mbar_init(&drain[1], 1);
        tc::fence_mbar_init();
        *s_fail = 0;
        *s_loaded = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(s_tmem, 2 * ACC);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tbase = *s_tmem;
    // K bytes 32 s .. 32 s + 31 hold columns 8 s .. 8 s + 7; a tile's first group has the smallest
    // row, so the smallest first nonzero column: k-steps below s0 are zero for every row of the
    // tile and are neither copied nor multiplied
    auto first_step = [](int tile) { return P::c_min((tile * G) / P::W) / 8; };
    // Every CTA walks all tiles, starting at its own offset: CTAs that run at the same time then
    // read different key rows, spread over the L2 slices.  The i-th tile of this CTA is tile_of(i).
    const int t_off = (int)((blockIdx.x % 128u) * (uint32_t)NT / 128u);
    auto tile_of = [&](int i) { return i + t_off < NT ? i + t_off : i + t_off - NT; };
    if (warp == SH_LOAD_WARP) {
        // ---------------- loader: chunk c (k-steps a .. a + n - 1 of one tile) -> slot c % NCH ----------------
        if (lane == 0) {
            uint32_t c = 0;
            bool ok = true, stalled = false;
#pragma unroll 1
            for (int i = 0; i < NT && ok && !stalled; i++) {
                const int t = tile_of(i);
                const uint8_t *src = A + (size_t)t * P::TILE;
#pragma unroll 1
                for (int a = first_step(t); a < P::KSTEPS; a += (int)CK, c++) {
                    const uint32_t cs = c % NCH;
                    if (c >= stall_after) {  // failure injection: stop without telling the other warps
                        stalled = true;
                        break;
                    }
                    if (*reinterpret_cast<volatile uint32_t *>(s_fail) ||
                        (c >= NCH && !wait_or_fail(&empty[cs], (c / NCH - 1) & 1u, spin, s_fail))) {
                        ok = false;
                        break;
                    }
                    const uint32_t n = P::KSTEPS - a < (int)CK ? (uint32_t)(P::KSTEPS - a) : CK;
                    tc::mbar_arrive_expect_tx(&full[cs], n * SLOT);
                    tc::bulk_g2s(ring + (size_t)cs * CK * SLOT, src + (size_t)a * SLOT, n * SLOT, &full[cs]);
                    __threadfence_block();
                    *reinterpret_cast<volatile uint32_t *>(s_loaded) = c + 1;
                }
            }
            if (!ok) atomicOr(s_fail, 1u);
            // unwind: no copy of this CTA may be in flight when it exits (the last chunk loaded
            // into each slot is the latest phase of its barrier)
            for (uint32_t ch = c > NCH ? c - NCH : 0; ch < c; ch++)
                tc::mbar_wait(&full[ch % NCH], (ch / NCH) & 1u, SH_SPIN);
        }
    } else {
        build_vector_columns<SET, VERIFY, SH_LOAD_WARP * 32>(sB, vec, vec_stride, inst0, batch, tid);
        tc::fence_async_smem();
        bar_sync(1, SH_LOAD_WARP * 32);  // warps 0-9: the vector columns are in place
    }
    if (warp == SH_ISSUE_WARP || warp == SH_ISSUE_WARP + 1) {
        // ---------------- MMA issuers: warp 8 the even tiles, warp 9 the odd ones ----------------
        // Two issuers, so one issues while the other waits and does its bookkeeping (tiles are
        // only 1-20 k-steps).  The whole warp runs the loop and the waits, so every value the
        // MMAs take is warp-uniform; one lane (the same throughout: a commit tracks the MMAs of
        // the thread that issues it) issues the MMAs and commits.  Run by one lane alone, every
        // step of this loop took 100-300 cycles and the tensor pipe waited for the issuers.
        const int me = warp - SH_ISSUE_WARP;
        const bool leader = tc::elect_one();
        const uint64_t kd0 = tc::desc_kmajor(tc::smem_u32(ring), (uint32_t)KR * 16u, 128u);
        const uint64_t vd0 = tc::desc_kmajor(tc::smem_u32(sB), (uint32_t)NIN * 16u, 128u);
        // descriptor start addresses are in 16-byte units (bits 0-13; every address here is
        // below 2^18 bytes, so adding to the descriptor never carries out of the field)
        constexpr uint64_t KD_STEP = SLOT >> 4, VD_STEP = (2u * NIN * 16u) >> 4, VD_BLOCK = 2048u >> 4;
        uint32_t c = 0;  // global chunk number (the loader's order)
        bool ok = true;
#pragma unroll 1
        for (int i = 0; i < NT && ok; i++) {
            const int s0 = first_step(tile_of(i));
            if ((i & 1) != me) {  // the other issuer's tile: skip its chunks
                c += (uint32_t)((P::KSTEPS - s0 + (int)CK - 1) / (int)CK);
                continue;
            }
            const int b = i & 1;
            const uint32_t dacc = tbase + (uint32_t)b * ACC;
#pragma unroll 1
            for (int a = s0; a < P::KSTEPS; a += (int)CK, c++) {
                const uint32_t cs = c % NCH;
                // The other issuer's tile may hold unloaded chunks older than c, so slot cs can
                // still be a phase behind chunk c: a parity wait is only meaningful once the
                // loader has armed chunk c's phase.
                if (!warp_wait_armed(s_loaded, c, spin) ||
                    !__all_sync(WARP_ALL, tc::mbar_wait(&full[cs], (c / NCH) & 1u, spin))) {
                    ok = false;
                    break;
                }
                // Only now wait for accumulator b (the epilogue of tile i - 2): the checks above
                // and the loop's bookkeeping then overlap that epilogue, and the MMAs follow the
                // accumulator's release at once.
                if (a == s0) {
                    if (i >= 2 && !warp_wait_or_fail(&acc_free[b], (uint32_t)((i - 2) >> 1) & 1u, spin, s_fail)) {
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                }
                const int n = P::KSTEPS - a;  // k-steps of this chunk: min(n, CK)
                const uint64_t kdc = kd0 + (uint64_t)cs * (CK * KD_STEP);
                const uint64_t vdc = vd0 + (uint64_t)a * VD_STEP;
                const uint32_t acc0 = a > s0 ? 1u : 0u;
                if (leader) {
#pragma unroll
                    for (int u = 0; u < (int)CK; u++) {
                        if (u < n) {
#pragma unroll
                            for (int h = 0; h < NB; h++)
                                tc::mma_i8(dacc + (uint32_t)h * KR, vdc + (uint64_t)u * VD_STEP + (uint64_t)h * VD_BLOCK,
                                           kdc + (uint64_t)u * KD_STEP, IDESC, u > 0 ? 1u : acc0);
                        }
                    }
                    tc::mma_commit(&empty[cs]);  // the chunk may be refilled once these MMAs completed
                }
                __syncwarp();
            }
            if (!ok) break;
            if (leader) tc::mma_commit(&mma_done[b]);  // the accumulator may be read
            __syncwarp();
            if ((i & 15) == me && warp_flag(s_fail)) ok = false;
        }
        if (!ok && leader) atomicOr(s_fail, 1u);
        // unwind: every MMA of this warp (and so every commit arrival it issued before) lands
        // before TMEM is freed
        if (leader) tc::mma_commit(&drain[me]);
        __syncwarp();
        tc::mbar_wait(&drain[me], 0u, SH_SPIN);
    } else if (warp < SH_ISSUE_WARP) {
        // ---------------- epilogue ----------------
        // warp: TMEM lanes 32 (warp % 4).. = vector columns.  Warps 0-3 / 4-7 split the work:
        // two M-blocks -> block 0 / 1, all four planes; two groups per tile -> group 0 / 1;
        // otherwise planes 0-1 / 2-3.
        constexpr int PL = (NB == 2 || G == 2) ? 4 : 2;
        const int grp = warp & 3, half = warp >> 2;
        const int h = NB == 2 ? half : 0;
        const int g = G == 2 ? half : 0;
        const int pl0 = PL == 4 ? 0 : 2 * half;
        const int n = h * 128 + grp * 32 + lane;  // this thread's vector column
        const uint32_t inst = inst0 + (uint32_t)(n / S::k);
        const int j = n % S::k;
        const bool live = n < P::NI * S::k && inst < batch;
        uint4 *dst = planes + (size_t)inst * P::PLANES + (size_t)j * P::NROWS * P::W;
        const uint32_t taddr =
            tbase + ((uint32_t)(grp * 32) << 16) + (uint32_t)(h * KR + g * 128) + (uint32_t)pl0 * 32u;
#pragma unroll 1
        for (int i = 0; i < NT; i++) {
            const int b = i & 1;
            if (!wait_or_fail(&mma_done[b], (uint32_t)(i >> 1) & 1u, spin, s_fail)) {
                atomicOr(s_fail, 1u);
                break;
            }
            tc::fence_after_sync();
            uint32_t r[PL][16];
#pragma unroll
            for (int p = 0; p < PL; p++) tc::tmem_ld32_pack16(taddr + (uint32_t)b * ACC + (uint32_t)p * 32u, r[p]);
            tc::tmem_wait_ld();
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&acc_free[b]);  // the accumulator may be overwritten now
            uint32_t wd[PL];
#pragma unroll
            for (int p = 0; p < PL; p++) wd[p] = pack_bit7x32(r[p]);
            const int gi = tile_of(i) * G + g;  // group = (row gi / W, coordinate group gi % W)
            if (live && gi < P::NGROUPS) {
                uint32_t *o = reinterpret_cast<uint32_t *>(dst + gi);
                if (PL == 4)
                    *reinterpret_cast<uint4 *>(o) = make_uint4(wd[0], wd[PL > 1 ? 1 : 0], wd[PL > 2 ? 2 : 0], wd[PL > 3 ? 3 : 0]);
                else
                    *reinterpret_cast<uint2 *>(o + pl0) = make_uint2(wd[0], wd[PL > 1 ? 1 : 0]);
            }
            if (*reinterpret_cast<volatile uint32_t *>(s_fail)) break;
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0 && *s_fail) atomicOr(ctl, 1u);
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tbase, 2 * ACC);
    }
}

// ---- the same product on a CTA pair (cluster of two CTAs, tcgen05 cta_group::2) ----
// Roles as in shared_gemm_kernel, with the key rows of every tile split between the two CTAs:
//   * each CTA's loader streams its half of the key rows (PairProb layout) into its own ring and
//     its full[] barrier tracks its own copies;
//   * in the odd CTA, warp 8 forwards each landed chunk to the even CTA's fwd[] barrier (in chunk
//     order, so every parity wait is on the current phase);
//   * the even CTA's issuers wait for both halves (full[], fwd[]) and issue the pair MMAs
//     (M = 256: 128 vector columns from each CTA; N = 128 key rows, 64 from each CTA); their
//     commits arrive on both CTAs' empty[] and mma_done[] barriers (multicast to the pair);
//   * both CTAs' epilogues read their own TMEM (128 vector columns x 128 key rows per M-block),
//     exactly as in the one-CTA kernel, and hand each accumulator back on the even CTA's
//     acc_free[] (16 warps).
// Every wait is bounded; a CTA that gives up sets its failure word, unwinds as the one-CTA
// kernel does (its own copies, the even CTA's own MMAs), and both CTAs meet at the cluster
// barrier before TMEM is freed, so no MMA reads a CTA's shared memory after it has left.
template <int SET, bool VERIFY>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(SH_GEMM_NT, 1)
    shared_gemm2_kernel(const uint8_t *__restrict__ A, const uint8_t *__restrict__ vec, size_t vec_stride,
                        uint4 *__restrict__ planes, uint32_t batch, uint32_t *ctl, uint32_t spin,
                        uint32_t stall_after) {
    using P = SharedProb<SET, VERIFY>;
    using Q = PairProb<SET, VERIFY>;
    using S = Set<SET>;
    constexpr int NIN = P::NINST, KPAD = P::KPAD, NT = P::NTILES, NB = P::NB;
    constexpr int KR = P::KROWS;
    constexpr uint32_t NCH = (uint32_t)Q::NCH, CK = (uint32_t)Q::CK, SLOT = (uint32_t)Q::SLOT2;
    constexpr uint32_t IDESC = tc::idesc_u8(256, KR);
    constexpr uint32_t ACC = KR * NB;  // TMEM columns of one accumulator
    static_assert(P::G == 1, "one key group per tile");
    extern __shared__ __align__(1024) uint8_t smem[];
    uint8_t *sB = smem;                                            // [KPAD/16][NIN][16] vector columns
    uint8_t *ring = smem + (size_t)NIN * KPAD;                      // NCH x CK x [2][64][16] key rows
    uint64_t *full = reinterpret_cast<uint64_t *>(ring + (size_t)NCH * CK * SLOT);  // [NCH] own copies
    uint64_t *fwd = full + NCH;                                     // [NCH] even CTA: odd CTA's copies
    uint64_t *empty = fwd + NCH;                                    // [NCH]
    uint64_t *mma_done = empty + NCH;                               // [2]
    uint64_t *acc_free = mma_done + 2;                              // [2] even CTA: 16 epilogue warps
    uint64_t *drain = acc_free + 2;                                 // [2]
    uint64_t *vec_ready = drain + 2;                                // even CTA: odd CTA's vectors built
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(vec_ready + 1);
    uint32_t *s_fail = s_tmem + 1;
    uint32_t *s_loaded = s_tmem + 2;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t rank = tc::cluster_ctarank();
    const bool lead = rank == 0;
    const uint32_t inst0 = blockIdx.x * (uint32_t)P::NI;

    if (tid == 0) {
        for (uint32_t i = 0; i < NCH; i++) {
            tc::mbar_init(&full[i], 1);
            tc::mbar_init(&fwd[i], 1);
            tc::mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < 2; i++) {
            tc::mbar_init(&mma_done[i], 1);
            tc::mbar_init(&acc_free[i], 2 * SH_EPI_NT / 32);
        }
        tc::mbar_init(&drain[0], 1);
        tc::mbar_init(&drain[1], 1);
        tc::mbar_init(vec_ready, 1);
        tc::fence_mbar_init();
        *s_fail = 0;
        *s_loaded = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc2(s_tmem, 2 * ACC);
        tc::tmem_relinquish2();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::cluster_sync();  // both CTAs' barriers and TMEM exist before any arrive or MMA crosses CTAs
    tc::fence_after_sync();
    const uint32_t tbase = *s_tmem;
    auto first_step = [](int tile) { return P::c_min(tile / P::W) / 8; };
    // both CTAs of a pair walk the tiles in the same order, from the pair's own offset
    const int t_off = (int)(((blockIdx.x >> 1) % 128u) * (uint32_t)NT / 128u);
    auto tile_of = [&](int i) { return i + t_off < NT ? i + t_off : i + t_off - NT; };
    if (warp == SH_LOAD_WARP) {
        // ---------------- loader (both CTAs): chunk c -> slot c % NCH of this CTA's ring ----------------
        if (lane == 0) {
            uint32_t c = 0;
            bool ok = true, stalled = false;
#pragma unroll 1
            for (int i = 0; i < NT && ok && !stalled; i++) {
                const int t = tile_of(i);
                const uint8_t *src = A + (size_t)t * P::TILE + (size_t)rank * Q::HALF;
#pragma unroll 1
                for (int a = first_step(t); a < P::KSTEPS; a += (int)CK, c++) {
                    const uint32_t cs = c % NCH;
                    if (c >= stall_after) {  // failure injection: stop without telling the other warps
                        stalled = true;
                        break;
                    }
                    if (*reinterpret_cast<volatile uint32_t *>(s_fail) ||
                        (c >= NCH && !wait_or_fail(&empty[cs], (c / NCH - 1) & 1u, spin, s_fail))) {
                        ok = false;
                        break;
                    }
                    const uint32_t n = P::KSTEPS - a < (int)CK ? (uint32_t)(P::KSTEPS - a) : CK;
                    tc::mbar_arrive_expect_tx(&full[cs], n * SLOT);
                    tc::bulk_g2s(ring + (size_t)cs * CK * SLOT, src + (size_t)a * SLOT, n * SLOT, &full[cs]);
                    __threadfence_block();
                    *reinterpret_cast<volatile uint32_t *>(s_loaded) = c + 1;
                }
            }
            if (!ok) atomicOr(s_fail, 1u);
            // unwind: no copy of this CTA in flight when it leaves
            for (uint32_t ch = c > NCH ? c - NCH : 0; ch < c; ch++)
                tc::mbar_wait(&full[ch % NCH], (ch / NCH) & 1u, SH_SPIN);
            // and, on a normal end, the even CTA's last commits have arrived on this CTA's empty[]
            if (ok && !stalled)
                for (uint32_t ch = c > NCH ? c - NCH : 0; ch < c; ch++)
                    wait_or_fail(&empty[ch % NCH], (ch / NCH) & 1u, spin, s_fail);
        }
    } else {
        build_vector_columns<SET, VERIFY, SH_LOAD_WARP * 32>(sB, vec, vec_stride, inst0, batch, tid);
        tc::fence_async_smem();
        bar_sync(1, SH_LOAD_WARP * 32);  // warps 0-9: the vector columns are in place
        // the even CTA's MMAs read the odd CTA's vector columns too: tell it they are in place
        if (!lead && tid == 0) tc::mbar_arrive_remote(vec_ready, 0);
    }
    if (!lead && warp == SH_ISSUE_WARP) {
        // ---------------- odd CTA, warp 8: forward each landed chunk to the even CTA ----------------
        // In chunk order: chunk c - NCH was forwarded before, so slot c % NCH's barrier is in chunk
        // c's phase and the parity wait cannot pass on an older phase.  The whole warp waits (as
        // the issuers do); one lane arrives.
        const bool leader = tc::elect_one();
        uint32_t c = 0;
        bool ok = true;
#pragma unroll 1
        for (int i = 0; i < NT && ok; i++) {
            const int t = tile_of(i);
#pragma unroll 1
            for (int a = first_step(t); a < P::KSTEPS; a += (int)CK, c++) {
                const uint32_t cs = c % NCH;
                if (!warp_wait_or_fail(&full[cs], (c / NCH) & 1u, spin, s_fail)) {
                    ok = false;
                    break;
                }
                if (leader) tc::mbar_arrive_remote_relaxed(&fwd[cs], 0);  // the chunk's bytes have landed
                __syncwarp();
            }
        }
        if (!ok && leader) atomicOr(s_fail, 1u);
    } else if (lead && (warp == SH_ISSUE_WARP || warp == SH_ISSUE_WARP + 1)) {
        // ---------------- even CTA: MMA issuers, warp 8 the even tiles, warp 9 the odd ones ----------------
        // As in shared_gemm_kernel: the whole warp runs the loop, one lane issues and commits.
        const int me = warp - SH_ISSUE_WARP;
        const bool leader = tc::elect_one();
        // B: this CTA's half of a k-step, [2][64 rows][16 B] (the odd CTA's half at the same address)
        const uint64_t kd0 = tc::desc_kmajor(tc::smem_u32(ring), (uint32_t)Q::HROWS * 16u, 128u);
        const uint64_t vd0 = tc::desc_kmajor(tc::smem_u32(sB), (uint32_t)NIN * 16u, 128u);
        constexpr uint64_t KD_STEP = SLOT >> 4, VD_STEP = (2u * NIN * 16u) >> 4, VD_BLOCK = 2048u >> 4;
        uint32_t c = 0;
        bool ok = warp_wait_cluster_or_fail(vec_ready, 0u, spin, s_fail);  // the odd CTA's vector columns
#pragma unroll 1
        for (int i = 0; i < NT && ok; i++) {
            const int s0 = first_step(tile_of(i));
            if ((i & 1) != me) {
                c += (uint32_t)((P::KSTEPS - s0 + (int)CK - 1) / (int)CK);
                continue;
            }
            const int b = i & 1;
            const uint32_t dacc = tbase + (uint32_t)b * ACC;
#pragma unroll 1
            for (int a = s0; a < P::KSTEPS; a += (int)CK, c++) {
                const uint32_t cs = c % NCH;
                // chunk c armed by this CTA's loader: the slot's barriers are in chunk c's phase
                if (!warp_wait_armed(s_loaded, c, spin) ||
                    !__all_sync(WARP_ALL, tc::mbar_wait(&full[cs], (c / NCH) & 1u, spin)) ||
                    !__all_sync(WARP_ALL, tc::mbar_wait_cluster(&fwd[cs], (c / NCH) & 1u, spin))) {
                    ok = false;
                    break;
                }
                // then accumulator b: both CTAs' epilogues (16 warps, half of them remote) have
                // read tile i - 2 from it
                if (a == s0) {
                    if (i >= 2 && !warp_wait_cluster_or_fail(&acc_free[b], (uint32_t)((i - 2) >> 1) & 1u, spin, s_fail)) {
                        ok = false;
                        break;
                    }
                    tc::fence_after_sync();
                }
                const int n = P::KSTEPS - a;
                const uint64_t kdc = kd0 + (uint64_t)cs * (CK * KD_STEP);
                const uint64_t vdc = vd0 + (uint64_t)a * VD_STEP;
                const uint32_t acc0 = a > s0 ? 1u : 0u;
                if (leader) {
#pragma unroll
                    for (int u = 0; u < (int)CK; u++) {
                        if (u < n) {
#pragma unroll
                            for (int h = 0; h < NB; h++)
                                tc::mma2_i8(dacc + (uint32_t)h * KR, vdc + (uint64_t)u * VD_STEP + (uint64_t)h * VD_BLOCK,
                                            kdc + (uint64_t)u * KD_STEP, IDESC, u > 0 ? 1u : acc0);
                        }
                    }
                    tc::mma2_commit_mc(&empty[cs], 0x3);  // both CTAs may refill the chunk's slot
                }
                __syncwarp();
            }
            if (!ok) break;
            if (leader) tc::mma2_commit_mc(&mma_done[b], 0x3);  // both CTAs' epilogues may read accumulator b
            __syncwarp();
            if ((i & 15) == me && warp_flag(s_fail)) ok = false;
        }
        if (!ok && leader) atomicOr(s_fail, 1u);
        // unwind: every MMA this warp issued (reading both CTAs' shared memory) has completed
        if (leader) tc::mma2_commit_mc(&drain[me], 0x1);
        __syncwarp();
        tc::mbar_wait(&drain[me], 0u, SH_SPIN);
    } else if (warp < SH_ISSUE_WARP) {
        // ---------------- epilogue (both CTAs), as in shared_gemm_kernel ----------------
        constexpr int PL = 4;
        static_assert(NB == 2, "two M-blocks: warps 0-3 block 0, warps 4-7 block 1");
        const int grp = warp & 3, h = warp >> 2;
        const int n = h * 128 + grp * 32 + lane;
        const uint32_t inst = inst0 + (uint32_t)(n / S::k);
        const int j = n % S::k;
        const bool live = n < P::NI * S::k && inst < batch;
        uint4 *dst = planes + (size_t)inst * P::PLANES + (size_t)j * P::NROWS * P::W;
        const uint32_t taddr = tbase + ((uint32_t)(grp * 32) << 16) + (uint32_t)(h * KR);
#pragma unroll 1
        for (int i = 0; i < NT; i++) {
            const int b = i & 1;
            if (!wait_or_fail(&mma_done[b], (uint32_t)(i >> 1) & 1u, spin, s_fail)) {
                atomicOr(s_fail, 1u);
                break;
            }
            tc::fence_after_sync();
            uint32_t r[PL][16];
#pragma unroll
            for (int p = 0; p < PL; p++) tc::tmem_ld32_pack16(taddr + (uint32_t)b * ACC + (uint32_t)p * 32u, r[p]);
            tc::tmem_wait_ld();
            tc::fence_before_sync();
            __syncwarp();
            if (lane == 0) {  // accumulator b may be overwritten now (as far as this warp goes)
                // relaxed: the loads above have completed (wait::ld), and a release would first
                // wait for this warp's plane stores of the previous tile
                if (lead) tc::mbar_arrive(&acc_free[b]);
                else tc::mbar_arrive_remote_relaxed(&acc_free[b], 0);
            }
            uint32_t wd[PL];
#pragma unroll
            for (int p = 0; p < PL; p++) wd[p] = pack_bit7x32(r[p]);
            const int gi = tile_of(i);
            if (live && gi < P::NGROUPS)
                *reinterpret_cast<uint4 *>(dst + gi) = make_uint4(wd[0], wd[1], wd[2], wd[3]);
            if (*reinterpret_cast<volatile uint32_t *>(s_fail)) break;
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    // the pair meets here: the even CTA's MMAs and every arrive that crosses CTAs are complete,
    // so neither CTA's shared memory is read or written after it leaves
    tc::cluster_sync();
    if (tid == 0 && *s_fail) atomicOr(ctl, 1u);
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc2(tbase, 2 * ACC);
    }
}

// ---- sign ----
// First attempt from the planes, in a CTA without engine staging (more CTAs per SM).  A singular
// first attempt goes to the retry list; the fix-up kernel finishes it with the engine.
// SH_TAIL_G instances per CTA (sign_attempt's interleaved elimination: the G pivot owners of a
// step share one publish and the live columns fill whole warps); a CTA's last instances past the
// batch repeat the batch's last instance and write nothing.
// G (instances per CTA) is a runtime choice of the shared-key shape (mayo_b200_shared_set_shape):
// 1, 2 or 4, the autotuner's candidates (4 only where the CTA fits in shared memory).
template <int SET, int G>
struct TailShape {
    // threads per signature: three warps where the elimination's ko + 1 columns fit (MAYO_1: 81,
    // MAYO_2: 69); the engine's row slots shrink with them (R = 3 / 12).  More signatures per SM
    // at the same registers: MAYO_2 G = 4, 4 CTAs of 384 threads at 40 registers (16 signatures
    // per SM against 12 with 128 threads), 1.643 -> 1.494 ms at 65,536.
    static constexpr int TNT = (SET == 1 || SET == 2) ? 96 : SignCfg<SET>::NT;
    static constexpr int NT = TNT * G;
    // MAYO_5: 5 CTAs of 160 threads per SM held to a register budget (72 registers)
    // MAYO_2: the elimination's per-step chain needs signatures in flight more than registers.
    // With 128 threads per signature at 65,536: G = 1, 9 CTAs per SM (56 registers) 1.866 ms;
    // G = 2 with 5 CTAs (48 registers) 1.739 ms (4 CTAs: 1.889, 6: 1.777); G = 4 with 3 CTAs
    // (40 registers, 12 signatures per SM) 1.661 ms (2 CTAs: 2.055).  With 96 threads: G = 2 at 7
    // CTAs and G = 4 at 4 CTAs per SM (the same registers).
    static constexpr int MINB = SET == 5 ? (G == 1 ? 5 : 2) : (SET == 2 ? (G == 1 ? 1 : G == 2 ? 7 : 4) : 1);
    static constexpr size_t SMEM = (size_t)G * SignCfg<SET, TNT, true>::total;
};
template <int SET, int G>
__global__ void __launch_bounds__(TailShape<SET, G>::NT, TailShape<SET, G>::MINB)
    sign_shared_tail_kernel(const uint8_t *esk, uint8_t *sig, size_t sig_stride, const uint8_t *wsi, size_t wsi_stride,
                            const uint4 *planes, const uint4 *opl, uint32_t *ctl, uint32_t *retry, uint32_t batch) {
    using P = SharedProb<SET, false>;
    using C = SignCfg<SET, TailShape<SET, G>::TNT, true>;
    constexpr int NT = C::NT;
    extern __shared__ __align__(16) uint8_t smem0[];
    if (ctl[0]) return;  // the product gave up: the fix-up kernel signs everything
    const int T = threadIdx.x, g = T / NT, tid = T % NT;
    const uint32_t inst = blockIdx.x * G + (uint32_t)g;
    const bool live = inst < batch;
    const uint32_t src = live ? inst : batch - 1;
    uint8_t *smem = smem0 + (size_t)g * C::total;
    sign_load_ws<SET, NT, true>(smem, tid, esk, wsi + (size_t)src * wsi_stride);
    const bool ok = sign_attempt<SET, NT, true, G>(smem0, T, esk, planes + (size_t)src * P::PLANES);
    sign_write<SET, NT, true>(smem, tid, esk, ok && live ? sig + (size_t)inst * sig_stride : nullptr, opl);
    if (!ok && live && tid == 0) retry[atomicAdd(&ctl[1], 1u)] = inst;
}

// Retries (attempts ctr >= 1 of the listed instances) with the engine, or every instance from
// ctr = 0 if the product gave up.  A grid-stride loop over a count read on the device.
template <int SET>
__global__ void __launch_bounds__(SignCfg<SET>::NT)
    sign_shared_fix_kernel(const uint8_t *esk, uint8_t *sig, size_t sig_stride, const uint8_t *wsi, size_t wsi_stride,
                           const uint4 *opl, const uint32_t *ctl, const uint32_t *retry, uint32_t batch) {
    extern __shared__ __align__(16) uint8_t smem[];
    constexpr int NT = SignCfg<SET>::NT;
    const int tid = threadIdx.x;
    const bool all = ctl[0] != 0;
    const uint32_t count = all ? batch : ctl[1];
#pragma unroll 1
    for (uint32_t idx = blockIdx.x; idx < count; idx += gridDim.x) {
        const uint32_t inst = all ? idx : retry[idx];
        sign_load_ws<SET, NT>(smem, tid, esk, wsi + (size_t)inst * wsi_stride);
#pragma unroll 1
        for (int ctr = all ? 0 : 1; ctr < 255; ctr++) {
            if (ctr > 0) sign_next_vr<SET, NT>(smem, tid, ctr);
            if (sign_attempt<SET, NT>(smem, tid, esk)) break;
        }
        sign_write<SET, NT>(smem, tid, esk, sig + (size_t)inst * sig_stride, opl);
        __syncthreads();
    }
}

// ---- verify ----
// Thread per instance: digest = SHAKE256(M), t = SHAKE256(digest || salt) (src/verify.cu:37-48).
template <int SET>
__global__ void verify_hash_kernel(const VerifyIO io, uint8_t *tws, size_t tws_stride, uint32_t batch,
                                   const uint32_t *order) {
    using S = Set<SET>;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= batch) return;
    const uint32_t inst = order ? order[i] : i;  // order: instances grouped by message blocks
    alignas(8) uint8_t digest[S::digest];
    Sponge<136> sp;
    sp.init();
    sp.absorb(io.m.ptr(inst), io.m.len(inst));
    sp.finalize();
    sp.squeeze(digest, S::digest);
    Sponge<136> sp2;
    sp2.init();
    sp2.absorb(digest, S::digest);
    sp2.absorb(io.sig + (size_t)inst * io.sig_stride + S::k * S::n / 2, S::sk);  // salt
    sp2.finalize();
    uint8_t *t = tws + (size_t)inst * tws_stride;
    sp2.squeeze(t, S::menc);
    for (int i = S::menc; i < (S::menc + 3) / 4 * 4; i++) t[i] = 0;
}

// U_ij = s_i^T T_j from the planes, y = Horner over the pairs, compare with t.  No engine
// staging, no hashing: a small CTA.
template <int SET>
struct VTailCfg {
    using S = Set<SET>;
    // threads per verification, measured at 65,536: MAYO_1 96 (2.18 ms against 2.26 with 128, 3.25
    // with 256), MAYO_2 96 (0.279 against 0.291, 0.309 with 64), MAYO_3 128 (5.14 against 5.23 with
    // 96, 5.35 with 256), MAYO_5 256 (8.90 against 9.62 with 128, 15.5 with 64)
    static constexpr int J = S::k, W = S::W, NW = (S::menc + 3) / 4,
                         NT = SET == 5 ? 256 : SET == 3 ? 128 : 96;
    static constexpr int R = NT / (J * W);
    static_assert(R >= 1, "verify tail threads");
    static constexpr size_t off_masks = 0;
    static constexpr size_t off_x = off_masks + (size_t)S::n * J * 16;
    static constexpr size_t off_upk = off_x + (size_t)J * J * W * 16;
    static constexpr size_t off_t = off_upk + pad16((size_t)S::pairs * NW * 4);
    static constexpr size_t total = off_t + pad16((size_t)NW * 4);
};

template <int SET>
__global__ void __launch_bounds__(VTailCfg<SET>::NT)
    verify_shared_tail_kernel(const VerifyIO io, const uint8_t *tws, size_t tws_stride, const uint4 *planes,
                              const uint32_t *ctl) {
    using S = Set<SET>;
    using C = VTailCfg<SET>;
    using P = SharedProb<SET, true>;
    constexpr int J = C::J, W = C::W, NW = C::NW, R = C::R;
    extern __shared__ __align__(16) uint8_t smem[];
    if (ctl[0]) return;  // the product gave up: the fix-up kernel verifies everything
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *xacc = reinterpret_cast<uint4 *>(smem + C::off_x);
    uint32_t *upk = reinterpret_cast<uint32_t *>(smem + C::off_upk);
    uint32_t *s_t = reinterpret_cast<uint32_t *>(smem + C::off_t);
    const int tid = threadIdx.x;
    const size_t inst = blockIdx.x;
    const uint8_t *sig = io.sig + inst * io.sig_stride;
    for (int idx = tid; idx < S::n * J; idx += C::NT) {  // column c of s_j (src/verify.cu:62-70)
        const int c = idx / J, jj = idx - c * J;
        const int q = jj * S::n + c;
        masks[idx] = scalar_masks((sig[q >> 1] >> ((q & 1) * 4)) & 0xFu);
    }
    for (int i = tid; i < J * J * W * 4; i += C::NT) reinterpret_cast<uint32_t *>(xacc)[i] = 0;
    for (int i = tid; i < NW; i += C::NT) s_t[i] = reinterpret_cast<const uint32_t *>(tws + inst * tws_stride)[i];
    __syncthreads();
    if (tid < J * W * R) {
        const int j = tid % J, w = (tid / J) % W, rs = tid / (J * W);
        const uint4 *pl = planes + inst * P::PLANES + (size_t)j * S::n * W + w;
        G4 X[J];
#pragma unroll
        for (int i = 0; i < J; i++) X[i] = g4_zero();
        // unrolled so that several rows' plane loads are in flight at once
#pragma unroll 2
        for (int r = rs; r < S::n; r += R) {
            const G4 T = g4_ld(pl + (size_t)r * W);
            const uint4 *mr = masks + (size_t)r * J;
#pragma unroll
            for (int i = 0; i < J; i++) g4_madd(X[i], T, mr[i]);
        }
#pragma unroll
        for (int i = 0; i < J; i++) g4_atomic_xor(xacc + ((size_t)i * J + j) * W + w, X[i]);
    }
    __syncthreads();
    for (int idx = tid; idx < S::pairs * W; idx += C::NT) {  // U_ij (i <= j) to packed words
        const int pid = idx / W, ww = idx - pid * W;
        int i = 0, rem = pid;
        while (rem >= J - i) {
            rem -= J - i;
            i++;
        }
        const int j = i + rem;
        G4 u = g4_ld(xacc + ((size_t)i * J + j) * W + ww);
        if (i != j) u = g4_xor(u, g4_ld(xacc + ((size_t)j * J + i) * W + ww));
        const uint4 pk = g4_to_packed(u);
        const uint32_t wd[4] = {pk.x, pk.y, pk.z, pk.w};
#pragma unroll
        for (int q = 0; q < 4; q++)
            if (4 * ww + q < NW) upk[pid * NW + 4 * ww + q] = wd[q];
    }
    __syncthreads();
    if (tid < 32) {  // y = Horner over the pairs (i = k-1..0, j = i..k-1), compare (src/verify.cu:185-211)
        const int lane = tid;
        uint32_t y = 0;
#pragma unroll 1
        for (int i = S::k - 1; i >= 0; i--)
#pragma unroll 1
            for (int j = i; j < S::k; j++) {
                y = times_z_lane<SET>(y, lane);
                if (lane < NW) y ^= upk[pair_index(i, j, S::k) * NW + lane];
            }
        const uint32_t tw = lane < NW ? s_t[lane] : 0u;
        const bool eq = __all_sync(0xffffffffu, y == tw);
        if (lane == 0) io.res[inst * io.res_stride] = eq ? 0 : 1;
    }
}

// Every instance with the engine, only if the product gave up.
template <int SET>
__global__ void __launch_bounds__(VerifyCfg<SET>::NT)
    verify_shared_fix_kernel(const VerifyIO io, const uint32_t *ctl, uint32_t batch) {
    extern __shared__ __align__(16) uint8_t smem[];
    if (!ctl[0]) return;
#pragma unroll 1
    for (uint32_t inst = blockIdx.x; inst < batch; inst += gridDim.x) {
        verify_instance<SET, VerifyCfg<SET>::NC>(smem, threadIdx.x, io.epk, io.m.ptr(inst), io.m.len(inst),
                                                 io.sig + (size_t)inst * io.sig_stride, io.res + inst * io.res_stride);
        __syncthreads();
    }
}

// ---- optional per-kernel timing (profiling aid, off by default; per host thread) ----
struct ShTiming {
    bool on = false, ready = false;
    cudaEvent_t ev[6];
    int n = 0;
};
thread_local ShTiming tl_tm;
static void tmark(cudaStream_t st) {
    if (tl_tm.on && tl_tm.ready && tl_tm.n < 6) cudaEventRecord(tl_tm.ev[tl_tm.n++], st);
}

// ---- runtime shape of the shared-key path, per parameter set (mayo_b200_shared_set_shape) ----
struct SharedShape {
    std::atomic<int> hash_nt;  // threads per CTA of the thread-per-instance hash kernels
    std::atomic<int> tail_g;   // instances per sign-tail CTA
    std::atomic<int> pair;     // the key product on CTA pairs (shared_gemm2_kernel)
};
// Defaults (MAYO_1, 2, 3, 5), measured at 65,536 instances: the pair product is the faster one
// for every set (MAYO_5 sign 14.0 against 18.5 ms: one CTA's key ring holds only four chunks
// beside its vectors); signatures per sign-tail CTA: four for MAYO_2 (1.494 ms against 1.631 with
// two, 1.840 with one), two for MAYO_1 (5.12 ms against 7.11 with one, 8.22 with four), one for
// MAYO_3 and MAYO_5 (13.49 / 29.73 ms against 14.62 / 36.03 with two).
constexpr int default_tail_g(int si) { return si == 1 ? 4 : si == 0 ? 2 : 1; }
SharedShape g_shape[4] = {{HASH_NT, default_tail_g(0), 1}, {HASH_NT, default_tail_g(1), 1},
                          {HASH_NT, default_tail_g(2), 1}, {HASH_NT, default_tail_g(3), 1}};
static int shape_index(int set) { return set == 1 ? 0 : set == 2 ? 1 : set == 3 ? 2 : set == 5 ? 3 : -1; }

// ---- launchers ----
template <int SET, bool VERIFY>
static int launch_product(const uint8_t *key, const uint8_t *vec, size_t vec_stride, uint8_t *ws, size_t batch,
                          cudaStream_t st) {
    using P = SharedProb<SET, VERIFY>;
    using WSL = SharedWs<SET, VERIFY>;
    uint32_t *ctl = reinterpret_cast<uint32_t *>(ws);
    uint8_t *A = ws + WSL::a;
    const bool pair = g_shape[shape_index(SET)].pair.load(std::memory_order_relaxed) != 0;
    const size_t a_threads = (size_t)P::NTILES * P::G * (P::KPAD / 16) * 128 + WSL::OPL;
    if (pair)
        shared_a_kernel<SET, VERIFY, true><<<(unsigned)((a_threads + 255) / 256), 256, 0, st>>>(
            key, A, ctl, reinterpret_cast<uint4 *>(ws + WSL::op_off()));
    else
        shared_a_kernel<SET, VERIFY, false><<<(unsigned)((a_threads + 255) / 256), 256, 0, st>>>(
            key, A, ctl, reinterpret_cast<uint4 *>(ws + WSL::op_off()));
    tmark(st);
    uint4 *planes = reinterpret_cast<uint4 *>(ws + WSL::planes_off(batch));
    const Inject &inj = inject();
    const bool stall = inj.kind == MAYO_B200_INJECT_PRODUCT_STALL;
    const uint32_t spin = stall && inj.spin ? inj.spin : SH_SPIN;
    const unsigned ctas = (unsigned)((batch + P::NI - 1) / P::NI);
    if (pair) {
        using Q = PairProb<SET, VERIFY>;
        if (!set_smem_attr(shared_gemm2_kernel<SET, VERIFY>, Q::SMEM)) return ST_CUDA;
        // clusters of two: an even number of CTAs (a last CTA without instances still takes part)
        shared_gemm2_kernel<SET, VERIFY><<<(ctas + 1) / 2 * 2, SH_GEMM_NT, Q::SMEM, st>>>(
            A, vec, vec_stride, planes, (uint32_t)batch, ctl, spin, stall ? inj.arg : 0xFFFFFFFFu);
    } else {
        if (!set_smem_attr(shared_gemm_kernel<SET, VERIFY>, P::SMEM)) return ST_CUDA;
        shared_gemm_kernel<SET, VERIFY><<<ctas, SH_GEMM_NT, P::SMEM, st>>>(
            A, vec, vec_stride, planes, (uint32_t)batch, ctl, spin, stall ? inj.arg : 0xFFFFFFFFu);
    }
    tmark(st);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

static unsigned fix_grid(size_t batch) { return (unsigned)(batch < SH_FIX_CTAS ? batch : SH_FIX_CTAS); }

// The sign tail with G instances per CTA (ST_BAD_ARG where such a CTA does not fit).
template <int SET, int G>
static int launch_sign_tail(const SignIO &io, const uint4 *planes, const uint4 *opl, uint32_t *ctl, uint32_t *retry,
                            size_t batch, cudaStream_t st) {
    using TS = TailShape<SET, G>;
    if constexpr (TS::SMEM > SH_SMEM_MAX) {
        return ST_BAD_ARG;
    } else {
        if (!set_smem_attr(sign_shared_tail_kernel<SET, G>, TS::SMEM)) return ST_CUDA;
        sign_shared_tail_kernel<SET, G><<<(unsigned)((batch + G - 1) / G), TS::NT, TS::SMEM, st>>>(
            io.esk, io.sig, io.sig_stride, io.ws, io.ws_stride, planes, opl, ctl, retry, (uint32_t)batch);
        return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
    }
}

template <int SET>
static int sign_shared_t(const SignIO &io0, uint8_t *ws, size_t batch, cudaStream_t st) {
    using WSL = SharedWs<SET, false>;
    using CF = SignCfg<SET>;
    SignIO io = io0;
    io.esk_stride = 0;
    io.ws = ws + WSL::inst_off();
    io.ws_stride = WSL::inst;
    tl_tm.n = 0;
    tmark(st);
    const SharedShape &shp = g_shape[shape_index(SET)];
    const int hnt = shp.hash_nt.load(std::memory_order_relaxed), tg = shp.tail_g.load(std::memory_order_relaxed);
    const uint32_t *order = launch_hash_order<SET, false>(io.m, ws, batch, st);
    int rc = launch_sign_hash(SET, io, batch, st, order, hnt);
    tmark(st);
    if (rc != ST_OK) return rc;
    rc = launch_product<SET, false>(io.esk, io.ws + SignWs<SET>::vr, io.ws_stride, ws, batch, st);
    if (rc != ST_OK) return rc;
    uint32_t *ctl = reinterpret_cast<uint32_t *>(ws);
    uint32_t *retry = reinterpret_cast<uint32_t *>(ws + WSL::retry_off(batch));
    const uint4 *planes = reinterpret_cast<const uint4 *>(ws + WSL::planes_off(batch));
    const uint4 *opl = reinterpret_cast<const uint4 *>(ws + WSL::op_off());
    rc = tg == 4 ? launch_sign_tail<SET, 4>(io, planes, opl, ctl, retry, batch, st)
         : tg == 2 ? launch_sign_tail<SET, 2>(io, planes, opl, ctl, retry, batch, st)
                   : launch_sign_tail<SET, 1>(io, planes, opl, ctl, retry, batch, st);
    if (rc != ST_OK) return rc;
    tmark(st);
    if (!set_smem_attr(sign_shared_fix_kernel<SET>, CF::total)) return ST_CUDA;
    sign_shared_fix_kernel<SET><<<fix_grid(batch), CF::NT, CF::total, st>>>(
        io.esk, io.sig, io.sig_stride, io.ws, io.ws_stride, reinterpret_cast<const uint4 *>(ws + WSL::op_off()), ctl,
        retry, (uint32_t)batch);
    tmark(st);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

template <int SET>
static int verify_shared_t(const VerifyIO &io0, uint8_t *ws, size_t batch, cudaStream_t st) {
    using WSL = SharedWs<SET, true>;
    using CT = VTailCfg<SET>;
    using CF = VerifyCfg<SET>;
    VerifyIO io = io0;
    io.epk_stride = 0;
    uint8_t *tws = ws + WSL::inst_off();
    tl_tm.n = 0;
    tmark(st);
    const uint32_t *order = launch_hash_order<SET, true>(io.m, ws, batch, st);
    const int hnt = g_shape[shape_index(SET)].hash_nt.load(std::memory_order_relaxed);
    verify_hash_kernel<SET><<<(unsigned)((batch + hnt - 1) / hnt), hnt, 0, st>>>(io, tws, WSL::inst, (uint32_t)batch,
                                                                             order);
    tmark(st);
    int rc = launch_product<SET, true>(io.epk, io.sig, io.sig_stride, ws, batch, st);
    if (rc != ST_OK) return rc;
    const uint32_t *ctl = reinterpret_cast<const uint32_t *>(ws);
    if (!set_smem_attr(verify_shared_tail_kernel<SET>, CT::total)) return ST_CUDA;
    verify_shared_tail_kernel<SET><<<(unsigned)batch, CT::NT, CT::total, st>>>(
        io, tws, WSL::inst, reinterpret_cast<const uint4 *>(ws + WSL::planes_off(batch)), ctl);
    tmark(st);
    if (!set_smem_attr(verify_shared_fix_kernel<SET>, CF::total)) return ST_CUDA;
    verify_shared_fix_kernel<SET><<<fix_grid(batch), CF::NT, CF::total, st>>>(io, ctl, (uint32_t)batch);
    tmark(st);
    return cudaPeekAtLastError() == cudaSuccess ? ST_OK : ST_CUDA;
}

size_t shared_ws_bytes(int set, bool verify, size_t batch) {
    switch (set) {
        case 1: return verify ? SharedWs<1, true>::bytes(batch) : SharedWs<1, false>::bytes(batch);
        case 2: return verify ? SharedWs<2, true>::bytes(batch) : SharedWs<2, false>::bytes(batch);
        case 3: return verify ? SharedWs<3, true>::bytes(batch) : SharedWs<3, false>::bytes(batch);
        case 5: return verify ? SharedWs<5, true>::bytes(batch) : SharedWs<5, false>::bytes(batch);
        default: return 0;
    }
}

int shared_timing(int enable) {
    if (enable && !tl_tm.ready) {
        for (int i = 0; i < 6; i++)
            if (cudaEventCreate(&tl_tm.ev[i]) != cudaSuccess) return ST_CUDA;
        tl_tm.ready = true;
    }
    tl_tm.on = enable != 0;
    tl_tm.n = 0;
    return ST_OK;
}

int shared_timing_read(float *ms) {
    if (!tl_tm.ready || tl_tm.n != 6) return ST_BAD_ARG;
    if (cudaEventSynchronize(tl_tm.ev[5]) != cudaSuccess) return ST_CUDA;
    for (int i = 0; i < 5; i++)
        if (cudaEventElapsedTime(&ms[i], tl_tm.ev[i], tl_tm.ev[i + 1]) != cudaSuccess) return ST_CUDA;
    return ST_OK;
}

// Shared memory a sign-tail CTA of g instances needs (0 for a bad set).
static size_t tail_smem(int set, int g) {
    switch (set) {
        case 1: return (size_t)g * SignCfg<1, TailShape<1, 1>::TNT, true>::total;
        case 2: return (size_t)g * SignCfg<2, TailShape<2, 1>::TNT, true>::total;
        case 3: return (size_t)g * SignCfg<3, 0, true>::total;
        case 5: return (size_t)g * SignCfg<5, 0, true>::total;
        default: return 0;
    }
}

int shared_set_shape(int set, int hash_nt, int tail_g, int product_ctas) {
    const int si = shape_index(set);
    if (si < 0) return ST_BAD_SET;
    if (hash_nt == 0) hash_nt = HASH_NT;
    if (tail_g == 0) tail_g = default_tail_g(si);
    if (hash_nt < 32 || hash_nt > 1024 || hash_nt % 32 || (tail_g != 1 && tail_g != 2 && tail_g != 4)) return ST_BAD_ARG;
    if (tail_smem(set, tail_g) > SH_SMEM_MAX) return ST_BAD_ARG;
    if (product_ctas == 0) product_ctas = 2;
    if (product_ctas != 1 && product_ctas != 2) return ST_BAD_ARG;
    g_shape[si].hash_nt.store(hash_nt);
    g_shape[si].tail_g.store(tail_g);
    g_shape[si].pair.store(product_ctas == 2 ? 1 : 0);
    return ST_OK;
}

int shared_get_shape(int set, int *hash_nt, int *tail_g, int *product_ctas) {
    const int si = shape_index(set);
    if (si < 0) return ST_BAD_SET;
    *hash_nt = g_shape[si].hash_nt.load();
    *tail_g = g_shape[si].tail_g.load();
    *product_ctas = g_shape[si].pair.load() ? 2 : 1;
    return ST_OK;
}

int launch_sign_shared(int set, const SignIO &io, uint8_t *ws, size_t batch, cudaStream_t st) {
    if (batch == 0) return ST_OK;
    switch (set) {
        case 1: return sign_shared_t<1>(io, ws, batch, st);
        case 2: return sign_shared_t<2>(io, ws, batch, st);
        case 3: return sign_shared_t<3>(io, ws, batch, st);
        case 5: return sign_shared_t<5>(io, ws, batch, st);
        default: return ST_BAD_SET;
    }
}

int launch_verify_shared(int set, const VerifyIO &io, uint8_t *ws, size_t batch, cudaStream_t st) {
    if (batch == 0) return ST_OK;
    switch (set) {
        case 1: return verify_shared_t<1>(io, ws, batch, st);
        case 2: return verify_shared_t<2>(io, ws, batch, st);
        case 3: return verify_shared_t<3>(io, ws, batch, st);
        case 5: return verify_shared_t<5>(io, ws, batch, st);
        default: return ST_BAD_SET;
    }
}

}  // namespace mayo
