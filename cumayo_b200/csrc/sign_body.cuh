// sign_body.cuh -- one MAYO signature on one CTA (reference src/sign.cu:10-477), shared by the
// batched sign kernel and the persistent work-queue kernel.
//
//   U = V^T P1 V and y = sum z^l U_l + t        engine over P1 rows          (sign.cu:396-460)
//   M_i = V_i L                                  engine over the columns of L (sign.cu:256-330)
//   A = sum z^l M                                packed z-shifts, one thread per column (sign.cu:333-393)
//   x = solve(A, y, r)                           Gauss-Jordan over bit-planes, no data branches (sign.cu:10-145)
// No branch and no memory address depends on a value derived from the secret key; only the
// attempt count is data dependent, as in MAYO.  In the elimination the pivot's inverse comes
// from a shift of a 64-bit register constant and each column's factor from mask arithmetic
// (sign_eliminate), where the reference's elimination (sign.cu:48-100) branches on the entries
// and indexes its multiplication and inverse tables with them.
//
// Why the elimination may differ from the reference's and still give identical bytes: when
// rank A = m, the reference's pivot columns are the lexicographically first column basis of A
// (a property of A alone), and x = r + z with z the unique vector supported on those columns
// solving A z = y - A r.  Gauss-Jordan with any pivot-row choice finds the same columns and the
// same z.  Rank < m is detected by both (the reference: last echelon row zero).
#pragma once

#include "engine.cuh"
#include "launch_util.cuh"
#include "ops.h"

namespace mayo {

// Workspace layout inside the row's scratch region (k*m*ceil(o/2) bytes, at least 2304).
template <int SET>
struct SignWs {
    using S = Set<SET>;
    static constexpr int dig = 0, salt = S::digest, t = S::digest + S::sk, vr = S::digest + S::sk + S::menc;
    static constexpr int total = vr + S::vr;
    static_assert(total <= S::scratch, "workspace fits the reference scratch region");
};

// COMPACT: no engine staging (the first attempt from precomputed products only); the bit-plane
// columns of A then get a region of their own.
template <int SET, int NT_ = 0, bool COMPACT = false>
struct SignCfg {
    using S = Set<SET>;
    static constexpr int J = S::k, W = S::W;
    static constexpr int NT = NT_ ? NT_ : (SET == 5 ? 160 : 128);
    // engine row slots: J * W * R threads run the engine, so fewer threads get fewer slots
    static constexpr int R0 = SET == 2 ? 16 : (SET == 1 ? 4 : 2);
    static constexpr int R = NT / (J * W) < R0 ? NT / (J * W) : R0;
    static constexpr int NCOL = S::ko + 1;  // columns of [A | y]
    static constexpr int CPT = (NCOL + NT - 1) / NT;
    static constexpr int NW = (S::menc + 3) / 4;
    static_assert(J * W * R <= NT, "engine threads");
    // shared memory (bytes); the bit-plane columns of A reuse the engine staging area
    static constexpr size_t off_masks = 0;
    static constexpr size_t off_bs = off_masks + (size_t)S::v * J * 16;
    static constexpr size_t sz_bs = COMPACT ? 0 : (size_t)R * S::n * W * 16;
    static constexpr size_t sz_acol = (size_t)NCOL * W * 16;
    static constexpr size_t sz_x = (size_t)J * J * W * 16;
    // With engine staging, the U accumulators reuse it: they are written after the U loop's last
    // read of the staging area and consumed before the M loop's first write.
    static constexpr bool X_IN_BS = !COMPACT && sz_bs >= sz_x;
    static constexpr size_t off_x = X_IN_BS ? off_bs : off_bs + (sz_bs > sz_acol ? sz_bs : sz_acol);
    static constexpr size_t off_upk = X_IN_BS ? off_bs + (sz_bs > sz_acol ? sz_bs : sz_acol) : off_x + sz_x;
    static constexpr size_t off_mpk = off_upk + pad16((size_t)S::pairs * NW * 4);
    static constexpr size_t off_piv = off_mpk + pad16((size_t)S::k * S::o * NW * 4);
    // pivot buffer (uint4 items, two of them: step parity): the published pivot column ([w]), the
    // pivot row's one-hot words (2 items), the basis multiples of a_p^-1 (1 item; see sign_eliminate)
    static constexpr int PIVQ = W + 3;
    static_assert(W <= 8, "one-hot words fit in two items");
    static constexpr size_t off_rhs = off_piv + (size_t)2 * PIVQ * 16;
    static constexpr size_t off_y = off_rhs + (size_t)W * 16;
    static constexpr size_t off_key = off_y + pad16(NW * 4);
    static constexpr size_t off_t = off_key + pad16(S::digest + 2 * S::sk + 1);
    static constexpr size_t off_vr = off_t + pad16(NW * 4);
    static constexpr size_t off_xs = off_vr + pad16(S::vr);
    static constexpr size_t off_flag = off_xs + pad16(S::ko);
    static constexpr size_t total = off_flag + 16;
};

template <int SET>
struct P1Rows {  // rows r < v of the upper-triangular P1 (sign.cu:402-418)
    using S = Set<SET>;
    const uint8_t *P1;
    __device__ __forceinline__ int count(int r) const { return S::v - r; }
    __device__ __forceinline__ const uint8_t *entry(int r, int e) const {
        return P1 + (size_t)tri(r, r + e, S::v) * S::menc;
    }
    __device__ __forceinline__ int col(int r, int e) const { return r + e; }
};

template <int SET>
struct LColRows {  // "row" b = column b of L: entries L[a][b], a < v (sign.cu:274-319)
    using S = Set<SET>;
    const uint8_t *L;
    __device__ __forceinline__ int count(int) const { return S::v; }
    __device__ __forceinline__ const uint8_t *entry(int b, int a) const {
        return L + (size_t)(a * S::o + b) * S::menc;
    }
    __device__ __forceinline__ int col(int, int a) const { return a; }
};

__device__ __forceinline__ int pair_index_s(int i, int j, int k) { return i * k - (i * (i - 1)) / 2 + (j - i); }
// Position of pair (a <= b) in the A-assembly order (sign.cu:333-392): i = 0..k-1, j = k-1..i.
__device__ __forceinline__ int ell_of(int a, int b, int k) { return a * k - (a * (a - 1)) / 2 + (k - 1 - b); }

// Packed word q (8 coordinates) of z^ell * u for a packed m-vector u (NW words in shared memory),
// without the fold: coordinates >= m are dropped.
template <int SET>
__device__ __forceinline__ uint32_t zshift_word(const uint32_t *u, int q, int ell) {
    using S = Set<SET>;
    constexpr int NW = (S::menc + 3) / 4;
    const int Q = ell >> 3, sh = (ell & 7) * 4;
    const int qa = q - Q, qb = q - Q - 1;
    const uint32_t a = (qa >= 0 && qa < NW) ? u[qa] : 0u;
    const uint32_t b = (qb >= 0 && qb < NW) ? u[qb] : 0u;
    uint32_t w = sh ? ((a << sh) | (b >> (32 - sh))) : a;
    if (q == S::m / 8 && (S::m % 8)) w &= (1u << (4 * (S::m % 8))) - 1;
    if (q >= (S::m + 7) / 8) w = 0;
    return w;
}
// Packed word q of u >> (4 * shift) coordinates (shift > 0): coordinates shift.. move to 0..
template <int SET>
__device__ __forceinline__ uint32_t zdown_word(const uint32_t *u, int q, int shift) {
    using S = Set<SET>;
    constexpr int NW = (S::menc + 3) / 4;
    const int Q = shift >> 3, sh = (shift & 7) * 4;
    const int qa = q + Q, qb = q + Q + 1;
    const uint32_t a = (qa < NW) ? u[qa] : 0u;
    const uint32_t b = (qb < NW) ? u[qb] : 0u;
    return sh ? ((a >> sh) | (b << (32 - sh))) : a;
}

// Shared-memory views of one signing CTA.
#define MAYO_SIGN_VIEWS                                                                       \
    using S = Set<SET>;                                                                       \
    using C = SignCfg<SET, NT_, CP_>;                                                         \
    constexpr int J = C::J, W = C::W, R = C::R, NT = C::NT, NW = C::NW, KO = S::ko, CPT = C::CPT; \
    (void)J; (void)R; (void)KO; (void)CPT; (void)NW;

// Plain path: digest, salt, t and V||r(ctr = 0) from the workspace written by sign_hash_kernel.
template <int SET, int NT_, bool CP_ = false>
__device__ __forceinline__ void sign_load_ws(uint8_t *smem, int tid, const uint8_t *esk, const uint8_t *ws) {
    MAYO_SIGN_VIEWS
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *bs = reinterpret_cast<uint4 *>(smem + C::off_bs);
    uint4 *acol = reinterpret_cast<uint4 *>(smem + C::off_bs);  // [NCOL][W], after the engine phases
    uint4 *xacc = reinterpret_cast<uint4 *>(smem + C::off_x);
    uint32_t *upk = reinterpret_cast<uint32_t *>(smem + C::off_upk);
    uint32_t *mpk = reinterpret_cast<uint32_t *>(smem + C::off_mpk);  // [k][o][NW]
    uint4 *pivbuf = reinterpret_cast<uint4 *>(smem + C::off_piv);     // [2][PIVQ]
    uint4 *rhsacc = reinterpret_cast<uint4 *>(smem + C::off_rhs);     // [W]
    uint32_t *ypk = reinterpret_cast<uint32_t *>(smem + C::off_y);
    uint8_t *s_key = smem + C::off_key;  // digest || salt || seed_sk || ctr
    uint8_t *s_t = smem + C::off_t;
    uint8_t *s_vr = smem + C::off_vr;
    uint8_t *s_x = smem + C::off_xs;
    int *s_flag = reinterpret_cast<int *>(smem + C::off_flag);
    (void)masks; (void)bs; (void)acol; (void)xacc; (void)upk; (void)mpk; (void)pivbuf; (void)rhsacc; (void)ypk; (void)s_key; (void)s_t; (void)s_vr; (void)s_x; (void)s_flag;
    using WS = SignWs<SET>;
    if (CP_) {
        // compact tail: the workspace row is 16-byte aligned and padded to 16 bytes, so it comes
        // in with one 16-byte load per thread (into the V-mask area, free until the attempt)
        constexpr int NV = (WS::total + 15) / 16;
        static_assert((size_t)NV <= (size_t)S::v * J, "workspace staging fits the mask area");
#pragma unroll 1
        for (int i = tid; i < NV; i += NT) masks[i] = reinterpret_cast<const uint4 *>(ws)[i];
#pragma unroll 1
        for (int i = tid; i < S::sk; i += NT) s_key[S::digest + S::sk + i] = esk[i];
        __syncthreads();
        const uint8_t *st = reinterpret_cast<const uint8_t *>(masks);
#pragma unroll 1
        for (int i = tid; i < S::digest + S::sk; i += NT) s_key[i] = st[WS::dig + i];
#pragma unroll 1
        for (int i = tid; i < NW * 4; i += NT) s_t[i] = i < S::menc ? st[WS::t + i] : 0;
#pragma unroll 1
        for (int i = tid; i < S::vr; i += NT) s_vr[i] = st[WS::vr + i];
    } else {
        for (int i = tid; i < S::digest + S::sk; i += NT) s_key[i] = ws[WS::dig + i];
        for (int i = tid; i < S::sk; i += NT) s_key[S::digest + S::sk + i] = esk[i];
        for (int i = tid; i < NW * 4; i += NT) s_t[i] = i < S::menc ? ws[WS::t + i] : 0;
        for (int i = tid; i < S::vr; i += NT) s_vr[i] = ws[WS::vr + i];
    }
    __syncthreads();
}

// Queue path: the CTA hashes itself (warp 0, warp-cooperative Keccak): digest = SHAKE256(M),
// salt = SHAKE256(digest || 0^SK || seed_sk), t = SHAKE256(digest || salt), V || r for `ctr`
// (sign.cu:225-252).  All threads must call it.
template <int SET, int NT_, bool CP_ = false>
__device__ __forceinline__ void sign_hash_cta(uint8_t *smem, int tid, const uint8_t *esk, const uint8_t *msg,
                                              uint32_t mlen, int ctr) {
    MAYO_SIGN_VIEWS
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *bs = reinterpret_cast<uint4 *>(smem + C::off_bs);
    uint4 *acol = reinterpret_cast<uint4 *>(smem + C::off_bs);  // [NCOL][W], after the engine phases
    uint4 *xacc = reinterpret_cast<uint4 *>(smem + C::off_x);
    uint32_t *upk = reinterpret_cast<uint32_t *>(smem + C::off_upk);
    uint32_t *mpk = reinterpret_cast<uint32_t *>(smem + C::off_mpk);  // [k][o][NW]
    uint4 *pivbuf = reinterpret_cast<uint4 *>(smem + C::off_piv);     // [2][PIVQ]
    uint4 *rhsacc = reinterpret_cast<uint4 *>(smem + C::off_rhs);     // [W]
    uint32_t *ypk = reinterpret_cast<uint32_t *>(smem + C::off_y);
    uint8_t *s_key = smem + C::off_key;  // digest || salt || seed_sk || ctr
    uint8_t *s_t = smem + C::off_t;
    uint8_t *s_vr = smem + C::off_vr;
    uint8_t *s_x = smem + C::off_xs;
    int *s_flag = reinterpret_cast<int *>(smem + C::off_flag);
    (void)masks; (void)bs; (void)acol; (void)xacc; (void)upk; (void)mpk; (void)pivbuf; (void)rhsacc; (void)ypk; (void)s_key; (void)s_t; (void)s_vr; (void)s_x; (void)s_flag;
    uint8_t *s_salt = s_x;  // s_x is free until the attempt writes x
    if (tid < 32) {
        const int lane = tid;
        WarpKeccak wk;
        wk.setup(lane);
        warp_shake<136>(s_key, S::digest, msg, (int)mlen, wk, lane);
        for (int i = lane; i < S::sk; i += 32) {
            s_key[S::digest + i] = 0;
            s_key[S::digest + S::sk + i] = esk[i];
        }
        if (lane == 0) s_key[S::digest + 2 * S::sk] = (uint8_t)ctr;
        __syncwarp();
        warp_shake<136>(s_salt, S::sk, s_key, S::digest + 2 * S::sk, wk, lane);
        for (int i = lane; i < S::sk; i += 32) s_key[S::digest + i] = s_salt[i];
        for (int i = lane; i < NW * 4; i += 32) s_t[i] = 0;
        __syncwarp();
        warp_shake<136>(s_t, S::menc, s_key, S::digest + S::sk, wk, lane);
        warp_shake<136>(s_vr, S::vr, s_key, S::digest + 2 * S::sk + 1, wk, lane);
    }
    __syncthreads();
}

// V || r for attempt `ctr` from the digest, salt and seed already in shared memory.
template <int SET, int NT_, bool CP_ = false>
__device__ __forceinline__ void sign_next_vr(uint8_t *smem, int tid, int ctr) {
    MAYO_SIGN_VIEWS
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *bs = reinterpret_cast<uint4 *>(smem + C::off_bs);
    uint4 *acol = reinterpret_cast<uint4 *>(smem + C::off_bs);  // [NCOL][W], after the engine phases
    uint4 *xacc = reinterpret_cast<uint4 *>(smem + C::off_x);
    uint32_t *upk = reinterpret_cast<uint32_t *>(smem + C::off_upk);
    uint32_t *mpk = reinterpret_cast<uint32_t *>(smem + C::off_mpk);  // [k][o][NW]
    uint4 *pivbuf = reinterpret_cast<uint4 *>(smem + C::off_piv);     // [2][PIVQ]
    uint4 *rhsacc = reinterpret_cast<uint4 *>(smem + C::off_rhs);     // [W]
    uint32_t *ypk = reinterpret_cast<uint32_t *>(smem + C::off_y);
    uint8_t *s_key = smem + C::off_key;  // digest || salt || seed_sk || ctr
    uint8_t *s_t = smem + C::off_t;
    uint8_t *s_vr = smem + C::off_vr;
    uint8_t *s_x = smem + C::off_xs;
    int *s_flag = reinterpret_cast<int *>(smem + C::off_flag);
    (void)masks; (void)bs; (void)acol; (void)xacc; (void)upk; (void)mpk; (void)pivbuf; (void)rhsacc; (void)ypk; (void)s_key; (void)s_t; (void)s_vr; (void)s_x; (void)s_flag;
    if (tid < 32) {
        const int lane = tid;
        WarpKeccak wk;
        wk.setup(lane);
        if (lane == 0) s_key[S::digest + 2 * S::sk] = (uint8_t)ctr;
        __syncwarp();
        warp_shake<136>(s_vr, S::vr, s_key, S::digest + 2 * S::sk + 1, wk, lane);
    }
    __syncthreads();
}

template <int SET, int NT_, bool CP_, int G>
__device__ __forceinline__ bool sign_eliminate(uint8_t *smem0, int T);

// One attempt on the V || r in shared memory: x on success, x = r on a singular system.
// Returns whether the system had full rank.  All threads of the CTA must call it.
// `pre`, when given, holds this attempt's T_j[r] = P1[r] V_j (rows r < v) and M_j[b] = V_j L[:, b]
// (rows v + b) as bit-plane groups [j][row][w], computed for a whole batch on the tensor cores
// (op_shared.cu); the two engine passes over P1 and L are then skipped.
//
// G instances per CTA (G * NT threads; instance g's shared memory at smem0 + g * C::total): thread
// T works on instance T / NT as thread T % NT everywhere except in the elimination, where the
// instances' columns are interleaved -- thread T owns column KO - T / G of instance T % G -- so
// the G pivot owners of a step sit in one warp (one publish for G instances) and the live
// columns of a step fill whole warps.  All control flow and barriers are the same for every
// instance (nothing depends on the data), so the instances run one shared barrier sequence.
// With G = 1 smem0 / T are the instance's shared memory / thread index.  `esk` and `pre` are the
// thread's own instance's (T / NT).  The result is that instance's.
template <int SET, int NT_, bool CP_ = false, int G = 1>
__device__ __forceinline__ bool sign_attempt(uint8_t *smem0, int T, const uint8_t *esk, const uint4 *pre = nullptr) {
    static_assert(G == 1 || G == 2 || G == 4, "instances per CTA");
    const int tid = G == 1 ? T : T % SignCfg<SET, NT_, CP_>::NT;
    uint8_t *smem = smem0 + (G == 1 ? 0 : (size_t)(T / SignCfg<SET, NT_, CP_>::NT) * SignCfg<SET, NT_, CP_>::total);
    MAYO_SIGN_VIEWS
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *bs = reinterpret_cast<uint4 *>(smem + C::off_bs);
    uint4 *acol = reinterpret_cast<uint4 *>(smem + C::off_bs);  // [NCOL][W], after the engine phases
    uint4 *xacc = reinterpret_cast<uint4 *>(smem + C::off_x);
    uint32_t *upk = reinterpret_cast<uint32_t *>(smem + C::off_upk);
    uint32_t *mpk = reinterpret_cast<uint32_t *>(smem + C::off_mpk);  // [k][o][NW]
    uint4 *pivbuf = reinterpret_cast<uint4 *>(smem + C::off_piv);     // [2][PIVQ]
    uint4 *rhsacc = reinterpret_cast<uint4 *>(smem + C::off_rhs);     // [W]
    uint32_t *ypk = reinterpret_cast<uint32_t *>(smem + C::off_y);
    uint8_t *s_key = smem + C::off_key;  // digest || salt || seed_sk || ctr
    uint8_t *s_t = smem + C::off_t;
    uint8_t *s_vr = smem + C::off_vr;
    uint8_t *s_x = smem + C::off_xs;
    int *s_flag = reinterpret_cast<int *>(smem + C::off_flag);
    (void)masks; (void)bs; (void)acol; (void)xacc; (void)upk; (void)mpk; (void)pivbuf; (void)rhsacc; (void)ypk; (void)s_key; (void)s_t; (void)s_vr; (void)s_x; (void)s_flag;
    const int lane = tid & 31;
    (void)lane;
    const uint8_t *P1 = esk + S::sk + S::o_bytes;
    const uint8_t *L = P1 + S::p1;
    Engine<SET, J, R> eng;
    eng.setup(masks, bs, tid);
    // ---- masks of V: masks[c][i] = V_i[c] ----
    for (int idx = tid; idx < S::v * J; idx += NT) {
        const int c = idx / J, i = idx - c * J;
        const int q = i * S::m + c;
        masks[idx] = scalar_masks((s_vr[q >> 1] >> ((q & 1) * 4)) & 0xF);
    }
    __syncthreads();

    // ---- U = V^T P1 V: X[i][j] = sum_r V_i[r] T_j[r]; thread (j, w, rs) takes rows rs, rs + R, ... ----
    G4 X[J];
#pragma unroll
    for (int i = 0; i < J; i++) X[i] = g4_zero();
    if (CP_ || pre) {  // a compact CTA has no engine staging: precomputed products only
        constexpr int NROWS = S::v + S::o;
        if (eng.active) {
#pragma unroll 1
            for (int r = eng.rs; r < S::v; r += R) {
                const G4 T = g4_ld(pre + ((size_t)eng.j * NROWS + r) * W + eng.w);
                const uint4 *mr = masks + (size_t)r * J;
#pragma unroll
                for (int i = 0; i < J; i++) g4_madd(X[i], T, mr[i]);
            }
        }
    } else {
        const P1Rows<SET> rows{P1};
#pragma unroll 1
        for (int r0 = 0; r0 < S::v; r0 += R) {
            // the next pass's rows of P1, or after the last the first columns of L, into L2:
            // MAYO_3/5 (MAYO_5 signWithesk 6.96 -> 6.63 ms per 1,024; MAYO_1/2 measured slower)
            if (SET >= 3 && tid < 32) {
                if (r0 + R < S::v)
                    eng.prefetch(rows, r0 + R, S::v, tid);
                else
                    eng.prefetch(LColRows<SET>{L}, 0, S::o, tid);
            }
            eng.convert(rows, r0, S::v, tid, NT);
            __syncthreads();
            const int r = r0 + eng.rs;
            if (eng.active && r < S::v) {
                const G4 T = eng.row_product(rows, r);
                const uint4 *mr = masks + (size_t)r * J;
#pragma unroll
                for (int i = 0; i < J; i++) g4_madd(X[i], T, mr[i]);
            }
            __syncthreads();
        }
    }
    // the accumulators may share the engine staging area, whose last read is behind the loop's
    // final barrier: zero them, then combine the threads' partial sums
    for (int i = tid; i < J * J * W * 4; i += NT) reinterpret_cast<uint32_t *>(xacc)[i] = 0;
    __syncthreads();
    if (eng.active) {
#pragma unroll
        for (int i = 0; i < J; i++) g4_atomic_xor(xacc + ((size_t)i * J + eng.j) * W + eng.w, X[i]);
    }
    __syncthreads();
    for (int idx = tid; idx < S::pairs * W; idx += NT) {
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

    // ---- y = sum z^l U_l + t (warp 0) while the others compute M = V L ----
    if (tid < 32) {
        uint32_t y = 0;
#pragma unroll 1
        for (int i = S::k - 1; i >= 0; i--)
#pragma unroll 1
            for (int j = i; j < S::k; j++) {
                y = times_z_lane<SET>(y, lane);
                if (lane < NW) y ^= upk[pair_index_s(i, j, S::k) * NW + lane];
            }
        if (lane < NW) ypk[lane] = y ^ reinterpret_cast<const uint32_t *>(s_t)[lane];
    }
    if (CP_ || pre) {  // a compact CTA has no engine staging: precomputed products only
        constexpr int NROWS = S::v + S::o;
        for (int idx = tid; idx < J * S::o * W; idx += NT) {
            const int w = idx % W, jb = idx / W, b = jb % S::o, j = jb / S::o;
            const uint4 pk = g4_to_packed(g4_ld(pre + ((size_t)j * NROWS + S::v + b) * W + w));
            const uint32_t wd[4] = {pk.x, pk.y, pk.z, pk.w};
            uint32_t *dst = mpk + ((size_t)j * S::o + b) * NW;
#pragma unroll
            for (int q = 0; q < 4; q++)
                if (4 * w + q < NW) dst[4 * w + q] = wd[q];
        }
        __syncthreads();
    } else {
        const LColRows<SET> rows{L};
#pragma unroll 1
        for (int b0 = 0; b0 < S::o; b0 += R) {
            if (SET >= 3 && tid < 32) eng.prefetch(rows, b0 + R, S::o, tid);
            eng.convert(rows, b0, S::o, tid, NT);
            __syncthreads();
            const int b = b0 + eng.rs;
            if (eng.active && b < S::o) {
                const G4 T = eng.row_product(rows, b);  // M_j[b], j = eng.j
                const uint4 pk = g4_to_packed(T);
                const uint32_t wd[4] = {pk.x, pk.y, pk.z, pk.w};
                uint32_t *dst = mpk + ((size_t)eng.j * S::o + b) * NW;
#pragma unroll
                for (int q = 0; q < 4; q++)
                    if (4 * eng.w + q < NW) dst[4 * eng.w + q] = wd[q];
            }
            __syncthreads();
        }
    }

    // ---- A columns (i, b) = sum_j z^{l(i,j)} M_j[b] with one fold by f(z); RHS column = y ----
    for (int c = tid; c < C::NCOL; c += NT) {
        uint32_t acc[NW];
#pragma unroll
        for (int q = 0; q < NW; q++) acc[q] = 0;
        if (c < KO) {
            const int i = c / S::o, b = c - i * S::o;
            // The overflow of each z^ell M_j (coordinates m-ell..m-1, moved to 0..ell-1) is
            // summed over j and folded by f(z) once: the fold is linear.  ell < k(k+1)/2, so only
            // the first OVW packed words can hold overflow, and the fold (shifts by n < 4
            // coordinates) touches only the first FW words.
            constexpr int ELL_MAX = S::k * (S::k + 1) / 2 - 1;
            constexpr int OVW = (ELL_MAX + 7) / 8 < NW ? (ELL_MAX + 7) / 8 : NW;
            constexpr int FW = OVW + 1 < NW ? OVW + 1 : NW;
            uint32_t ovs[OVW];
#pragma unroll
            for (int q = 0; q < OVW; q++) ovs[q] = 0;
#pragma unroll 1
            for (int j = 0; j < S::k; j++) {
                const int ell = i <= j ? ell_of(i, j, S::k) : ell_of(j, i, S::k);
                const uint32_t *u = mpk + ((size_t)j * S::o + b) * NW;
                if constexpr (NW <= 10) {
                    // z^ell u without the fold: the packed words shifted up by 4 ell bits -- a
                    // funnel shift by the sub-word part, then a barrel shift by whole words (ell
                    // is below k(k+1)/2, so at most QMAX words) -- coordinates >= m dropped.
                    // (Larger sets keep the per-word form: fewer live registers.)
                    constexpr int QMAX = (S::k * (S::k + 1) / 2 - 1) >> 3;
                    const uint32_t sh = (uint32_t)(ell & 7) * 4u;
                    const int Q = ell >> 3;
                    uint32_t v[NW];
#pragma unroll
                    for (int q = 0; q < NW; q++) v[q] = u[q];
#pragma unroll
                    for (int q = NW - 1; q >= 0; q--) v[q] = __funnelshift_l(q > 0 ? v[q - 1] : 0u, v[q], sh);
#pragma unroll
                    for (int st = 1; st <= QMAX; st <<= 1) {
                        const bool take = (Q & st) != 0;
#pragma unroll
                        for (int q = NW - 1; q >= 0; q--) v[q] = take ? (q >= st ? v[q - st] : 0u) : v[q];
                    }
                    if (S::m % 8) v[S::m / 8] &= (1u << (4 * (S::m % 8))) - 1u;
#pragma unroll
                    for (int q = 0; q < NW; q++)
                        if (q < (S::m + 7) / 8) acc[q] ^= v[q];
                } else {
#pragma unroll
                    for (int q = 0; q < NW; q++) acc[q] ^= zshift_word<SET>(u, q, ell);
                }
                if (ell > 0) {
                    // overflow coordinates m-ell..m-1 -> 0..ell-1 (coordinates >= ell masked)
#pragma unroll
                    for (int q = 0; q < OVW; q++) {
                        uint32_t ov = zdown_word<SET>(u, q, S::m - ell);
                        const int lo = 8 * q;
                        if (lo >= ell) ov = 0;
                        else if (lo + 8 > ell) ov &= (1u << (4 * (ell - lo))) - 1;
                        ovs[q] ^= ov;
                    }
                }
            }
            // + sum_n c_n z^n (overflow): the reduction by f(z) = z^m + sum_n c_n z^n
#pragma unroll
            for (int n = 0; n < 4; n++) {
                if (S::cf(n) == 0) continue;
                uint32_t prev = 0;
#pragma unroll
                for (int q = 0; q < FW; q++) {
                    const uint32_t mc = q < OVW ? nib8_mul_const(ovs[q], S::cf(n)) : 0u;
                    acc[q] ^= n ? ((mc << (4 * n)) | (prev >> (32 - 4 * n))) : mc;
                    prev = mc;
                }
            }
        } else {
#pragma unroll
            for (int q = 0; q < NW; q++) acc[q] = ypk[q];
        }
        // packed -> bit-planes
#pragma unroll
        for (int w = 0; w < W; w++) {
            const uint32_t a0 = 4 * w + 0 < NW ? acc[4 * w + 0] : 0u;
            const uint32_t a1 = 4 * w + 1 < NW ? acc[4 * w + 1] : 0u;
            const uint32_t a2 = 4 * w + 2 < NW ? acc[4 * w + 2] : 0u;
            const uint32_t a3 = 4 * w + 3 < NW ? acc[4 * w + 3] : 0u;
            g4_st(acol + (size_t)c * W + w, g4_from_packed(a0, a1, a2, a3));
        }
    }
    for (int i = tid; i < W * 4; i += NT) reinterpret_cast<uint32_t *>(rhsacc)[i] = 0;
    __syncthreads();
    const bool ok_mine = sign_eliminate<SET, NT_, CP_, G>(smem0, T);
    (void)ok_mine;
    return reinterpret_cast<const int *>(smem + C::off_flag)[0] != 0;
}

// The elimination of sign_attempt (sample_solution, src/sign.cu:10-145) for the G instances of a
// CTA: [A | y] (bit-plane columns in each instance's acol area), r from V || r; writes x and the
// rank flag of every instance.  Returns the flag of the instance whose column this thread owns.
template <int SET, int NT_, bool CP_, int G>
__device__ __forceinline__ bool sign_eliminate(uint8_t *smem0, int T) {
    using S = Set<SET>;
    using C = SignCfg<SET, NT_, CP_>;
    constexpr int W = C::W, NT = C::NT, KO = S::ko, CPT = C::CPT;
    // interleaved columns: thread T takes column rank u = T / G of instance T % G
    const int tid = G == 1 ? T : T / G;
    uint8_t *smem = smem0 + (G == 1 ? 0 : (size_t)(T % G) * C::total);
    uint4 *acol = reinterpret_cast<uint4 *>(smem + C::off_bs);    // [NCOL][W]
    uint4 *pivbuf = reinterpret_cast<uint4 *>(smem + C::off_piv);  // [2][PIVQ]
    uint4 *rhsacc = reinterpret_cast<uint4 *>(smem + C::off_rhs);  // [W]
    const uint8_t *s_vr = smem + C::off_vr;
    uint8_t *s_x = smem + C::off_xs;
    int *s_flag = reinterpret_cast<int *>(smem + C::off_flag);

    // ---- Gauss-Jordan without data branches.  Thread owns columns c = KO - (tid + NT q): the RHS on
    // thread 0 and the columns still to update (c > pc) on the lowest threads, so the work of a
    // step stays in as few warps as possible. ----
    G4 col[CPT][W];
    uint32_t rr[CPT];
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int c = KO - (tid + NT * q);
#pragma unroll
        for (int w = 0; w < W; w++) col[q][w] = c >= 0 ? g4_ld(acol + (size_t)c * W + w) : g4_zero();
        const int rn = S::k * S::m;  // r starts after the k V-vectors (sign.cu:250)
        rr[q] = (c >= 0 && c < KO) ? (s_vr[(rn + c) >> 1] >> (((rn + c) & 1) * 4)) & 0xF : 0u;
    }
    // y <- y - A r  (sample_solution, sign.cu:36-45)
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int c = KO - (tid + NT * q);
        if (c >= 0 && c < KO) {
            const uint4 mk = scalar_masks(rr[q]);
#pragma unroll
            for (int w = 0; w < W; w++) {
                G4 pr = g4_zero();
                g4_madd(pr, col[q][w], mk);
                g4_atomic_xor(rhsacc + w, pr);
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < CPT; q++)
        if (tid + NT * q == 0)  // the RHS column
#pragma unroll
            for (int w = 0; w < W; w++) col[q][w] = g4_xor(col[q][w], g4_ld(rhsacc + w));

    uint32_t pivoted[W];
    uint32_t my_oh[CPT][W], my_has[CPT];
#pragma unroll
    for (int w = 0; w < W; w++) pivoted[w] = 0;
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        my_has[q] = 0;
#pragma unroll
        for (int w = 0; w < W; w++) my_oh[q][w] = 0;
    }
    // The owner of a column computes its pivot (lowest unpivoted row with a nonzero entry) a_p; a
    // column with entry e in row p then takes col ^= (e / a_p)(a + e_p) (eliminates row p,
    // normalises the pivot row).  Two forms of what the owner publishes in buffer pcx & 1 (the
    // row's one-hot words at [W, W + 2) in both):
    //   * PREDIV (the shared-key tail, several signatures per CTA and many per SM, bound by the
    //     ALU): D' = a_p^-1 (a + e_p) at [0, W); a column applies the masks of its own entry's
    //     bits to the x-multiples of D' (col ^= e D'), forming no quotient.  MAYO_2 at 65,536:
    //     1.662 -> 1.633 ms.
    //   * otherwise (one signature per CTA, where the owner's chain sets each step's pace):
    //     D = a + e_p at [0, W) and the basis multiples B_s = a_p^-1 x^s at [W + 2]; a column forms
    //     e / a_p = sum_s e_s B_s by masks.  The owner's extra scalar product of the first form made
    //     these paths ~1 % slower.
    constexpr bool PREDIV = CP_;
    auto publish = [&](int q, int pcx) {
        uint4 *buf = pivbuf + (pcx & 1) * C::PIVQ;
        uint32_t *ohw = reinterpret_cast<uint32_t *>(buf + W);  // oh[0..W)
        uint32_t oh[W], found = 0;
#pragma unroll
        for (int w = 0; w < W; w++) {
            const G4 &a = col[q][w];
            const uint32_t nz = (a.p0 | a.p1 | a.p2 | a.p3) & ~pivoted[w];
            const uint32_t low = nz & (0u - nz);
            oh[w] = low & ~found;
            found |= 0u - (uint32_t)(nz != 0u);
        }
        uint32_t o0 = 0, o1 = 0, o2 = 0, o3 = 0;
#pragma unroll
        for (int w = 0; w < W; w++) {
            o0 |= col[q][w].p0 & oh[w];
            o1 |= col[q][w].p1 & oh[w];
            o2 |= col[q][w].p2 & oh[w];
            o3 |= col[q][w].p3 & oh[w];
        }
        // a_p (0 when the column has no unpivoted nonzero entry: then oh = 0 and no column changes)
        const uint32_t piv = (uint32_t)(o0 != 0) | ((uint32_t)(o1 != 0) << 1) | ((uint32_t)(o2 != 0) << 2) |
                             ((uint32_t)(o3 != 0) << 3);
        const uint32_t b0 = gf16_inv_reg(piv);  // a_p^-1 by a shift of a register constant
#pragma unroll
        for (int w = 0; w < W; w++) {
            G4 ap = col[q][w];
            ap.p0 ^= oh[w];
            if constexpr (PREDIV) {
                G4 d = g4_zero();
                g4_madd(d, ap, scalar_masks(b0));
                g4_st(buf + w, d);
            } else {
                g4_st(buf + w, ap);
            }
            ohw[w] = oh[w];
            my_oh[q][w] = oh[w];
        }
        if constexpr (!PREDIV) {  // x a_p^-1, x^2 a_p^-1, x^3 a_p^-1
            const uint32_t b1 = gf16_xtime(b0), b2 = gf16_xtime(b1), b3 = gf16_xtime(b2);
            buf[W + 2] = make_uint4(b0, b1, b2, b3);
        }
        my_has[q] = found;
    };
#pragma unroll
    for (int q = 0; q < CPT; q++)
        if (KO - (tid + NT * q) == 0) publish(q, 0);
    __syncthreads();
    // Warp w owns column ranks >= 32 w / G, i.e. columns <= KO - 32 w / G, so after step
    // KO - 32 w / G - 1 it has nothing left to update or publish: it leaves the loop, and the
    // steps' barrier counts only the warps still in it (the lowest ones; a public function of the
    // step).
    const int last_step = KO - 32 * (T >> 5) / G - 1;
#pragma unroll 1
    for (int pc = 0; pc <= last_step; pc++) {
        // Every column right of pc: col ^= col[p] * F'  (eliminates row p elsewhere, normalises
        // row p).  A column left of pc is already a unit vector e_p' (or has no entry in an
        // unpivoted row), so col[p] = 0 there for every later pivot row p and the update would
        // be a no-op; skipping it depends only on the public loop index.  Lookahead: the owner
        // of column pc + 1 publishes its pivot right after its own update, while the other
        // columns update, so each step needs one barrier and the owner's chain overlaps them.
        const uint4 *buf = pivbuf + (pc & 1) * C::PIVQ;
        const uint32_t *ohw = reinterpret_cast<const uint32_t *>(buf + W);
        G4 D[W];
        uint32_t oh[W];
#pragma unroll
        for (int w = 0; w < W; w++) {
            D[w] = g4_ld(buf + w);
            oh[w] = ohw[w];
            pivoted[w] |= oh[w];
        }
#pragma unroll
        for (int q = 0; q < CPT; q++) {
            const int c = KO - (tid + NT * q);
            if (c <= pc) continue;
            uint32_t e0 = 0, e1 = 0, e2 = 0, e3 = 0;
#pragma unroll
            for (int w = 0; w < W; w++) {
                e0 |= col[q][w].p0 & oh[w];
                e1 |= col[q][w].p1 & oh[w];
                e2 |= col[q][w].p2 & oh[w];
                e3 |= col[q][w].p3 & oh[w];
            }
            uint4 fm;
            if constexpr (PREDIV) {  // masks of e's bits (each e_s is 0 or the pivot row's one bit)
                fm = make_uint4(0u - (uint32_t)(e0 != 0u), 0u - (uint32_t)(e1 != 0u), 0u - (uint32_t)(e2 != 0u),
                                0u - (uint32_t)(e3 != 0u));
            } else {  // masks of e / a_p
                fm = scalar_masks(gf16_div_from_basis(e0, e1, e2, e3, buf[W + 2]));
            }
#pragma unroll
            for (int w = 0; w < W; w++) g4_madd(col[q][w], D[w], fm);
            if (c == pc + 1 && c < KO) publish(q, c);
        }
        const int nw = G * (KO - 1 - pc) / 32 + 1;  // warps with a column > pc (or column pc + 1)
        bar_sync(1, 32 * (nw < G * NT / 32 ? nw : G * NT / 32));
    }
    // rank test (sign.cu:107-115 rejects when the last echelon row is zero, i.e. rank < m): thread
    // 0 took part in every step, so its record of the pivot rows is complete
    if (tid == 0) {
        int rank = 0;
#pragma unroll
        for (int w = 0; w < W; w++) rank += __popc(pivoted[w]);
        s_flag[0] = rank == S::m ? 1 : 0;
    }
    // publish the reduced RHS; x = r + z (z_c = rhs[p(c)] on pivot columns)
#pragma unroll
    for (int q = 0; q < CPT; q++)
        if (tid + NT * q == 0)  // the RHS column
#pragma unroll
            for (int w = 0; w < W; w++) g4_st(rhsacc + w, col[q][w]);  // not a buffer still being read
    __syncthreads();
    const bool ok = s_flag[0] != 0;  // this column's instance
#pragma unroll
    for (int q = 0; q < CPT; q++) {
        const int c = KO - (tid + NT * q);
        if (c >= 0 && c < KO) {
            uint32_t z0 = 0, z1 = 0, z2 = 0, z3 = 0;
#pragma unroll
            for (int w = 0; w < W; w++) {
                const G4 h = g4_ld(rhsacc + w);
                z0 |= h.p0 & my_oh[q][w];
                z1 |= h.p1 & my_oh[q][w];
                z2 |= h.p2 & my_oh[q][w];
                z3 |= h.p3 & my_oh[q][w];
            }
            const uint32_t z = ((uint32_t)(z0 != 0) | ((uint32_t)(z1 != 0) << 1) | ((uint32_t)(z2 != 0) << 2) |
                                ((uint32_t)(z3 != 0) << 3)) & my_has[q];
            // a rejected attempt leaves x = r (sign.cu:31-33, 115)
            s_x[c] = (uint8_t)(rr[q] ^ (ok ? z : 0u));
        }
    }
    __syncthreads();
    return ok;
}

// Column q of O as bit planes, coordinate group w (item q * W + w): O is row-major v x o nibbles
// (O[t][q] at nibble t * o + q of the O block of esk).  A property of the key alone, so the
// shared-key path computes it once per call.
template <int SET>
__device__ __forceinline__ G4 o_plane_item(const uint8_t *O_g, int idx) {
    using S = Set<SET>;
    constexpr int W = S::W;
    const int q = idx / W, w = idx - q * W;
    uint32_t pk[4] = {0u, 0u, 0u, 0u};
#pragma unroll 4
    for (int e = 0; e < 32; e++) {
        const int t = 32 * w + e;
        if (t < S::m) {
            const int oi = t * S::o + q;
            pk[e >> 3] |= (uint32_t)((O_g[oi >> 1] >> ((oi & 1) * 4)) & 0xF) << (4 * (e & 7));
        }
    }
    return g4_from_packed(pk[0], pk[1], pk[2], pk[3]);
}

// s = V + O x, then salt (sign.cu:147-191, 474-477).  `opl`, when given, holds the O planes
// (o x W items of o_plane_item) precomputed for the key.
template <int SET, int NT_, bool CP_ = false>
__device__ __forceinline__ void sign_write(uint8_t *smem, int tid, const uint8_t *esk, uint8_t *sig,
                                           const uint4 *opl = nullptr) {
    MAYO_SIGN_VIEWS
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *bs = reinterpret_cast<uint4 *>(smem + C::off_bs);
    uint4 *acol = reinterpret_cast<uint4 *>(smem + C::off_bs);  // [NCOL][W], after the engine phases
    uint4 *xacc = reinterpret_cast<uint4 *>(smem + C::off_x);
    uint32_t *upk = reinterpret_cast<uint32_t *>(smem + C::off_upk);
    uint32_t *mpk = reinterpret_cast<uint32_t *>(smem + C::off_mpk);  // [k][o][NW]
    uint4 *pivbuf = reinterpret_cast<uint4 *>(smem + C::off_piv);     // [2][PIVQ]
    uint4 *rhsacc = reinterpret_cast<uint4 *>(smem + C::off_rhs);     // [W]
    uint32_t *ypk = reinterpret_cast<uint32_t *>(smem + C::off_y);
    uint8_t *s_key = smem + C::off_key;  // digest || salt || seed_sk || ctr
    uint8_t *s_t = smem + C::off_t;
    uint8_t *s_vr = smem + C::off_vr;
    uint8_t *s_x = smem + C::off_xs;
    int *s_flag = reinterpret_cast<int *>(smem + C::off_flag);
    (void)masks; (void)bs; (void)acol; (void)xacc; (void)upk; (void)mpk; (void)pivbuf; (void)rhsacc; (void)ypk; (void)s_key; (void)s_t; (void)s_vr; (void)s_x; (void)s_flag;
    // s_i = V_i + O x_i on bit planes: the columns of O as planes and the k x W accumulators in
    // the engine staging area (free after the attempt); each accumulator (i, w) takes its o
    // multiply-accumulates from SPL threads (shared-memory XOR to combine); nibbles are staged
    // one per byte (the mask area, also free) because s_i starts mid-byte when n is odd.
    constexpr int SPL = 4;
    uint4 *ocol = reinterpret_cast<uint4 *>(smem + C::off_bs);  // [o][W]
    uint4 *sacc = ocol + S::o * W;                                 // [k][W]
    uint8_t *snib = smem + C::off_masks;                           // [k * n]
    static_assert((size_t)(S::o + S::k) * W * 16 <= (C::sz_bs > C::sz_acol ? C::sz_bs : C::sz_acol),
                  "O planes and s accumulators fit");
    static_assert((size_t)S::k * S::n <= (size_t)S::v * J * 16, "nibble staging fits");
    if (opl) {
        for (int idx = tid; idx < S::o * W; idx += NT) ocol[idx] = opl[idx];
    } else {
        for (int idx = tid; idx < S::o * W; idx += NT) g4_st(ocol + idx, o_plane_item<SET>(esk + S::sk, idx));
    }
    for (int idx = tid; idx < S::k * S::o; idx += NT) {  // x_i: the last o nibbles of s_i
        const int i = idx / S::o, q = idx - i * S::o;
        snib[i * S::n + S::m + q] = s_x[idx];
    }
    for (int idx = tid; idx < S::k * W; idx += NT) {  // accumulator (i, w) starts as V_i group w
        const int i = idx / W, w = idx - i * W;
        // V_i group w: packed nibbles i * m + 32 w .. (m even, so byte aligned)
        const uint8_t *vb = s_vr + (i * S::m + 32 * w) / 2;
        const int nb = min(16, (S::m - 32 * w + 1) / 2);
        uint32_t pk[4] = {0u, 0u, 0u, 0u};
        for (int bb = 0; bb < nb; bb++) pk[bb >> 2] |= (uint32_t)vb[bb] << (8 * (bb & 3));
        if (S::m - 32 * w < 32 && ((S::m - 32 * w) & 1)) {  // odd tail: drop the extra nibble
            const int last = S::m - 32 * w;
            pk[last >> 3] &= ~(0xFu << (4 * (last & 7)));
        }
        g4_st(sacc + idx, g4_from_packed(pk[0], pk[1], pk[2], pk[3]));
    }
    __syncthreads();
    for (int idx = tid; idx < S::k * W * SPL; idx += NT) {
        const int g = idx / SPL, part = idx - g * SPL;
        const int i = g / W, w = g - i * W;
        G4 acc = g4_zero();
#pragma unroll 1
        for (int q = part; q < S::o; q += SPL) g4_madd(acc, g4_ld(ocol + q * W + w), scalar_masks(s_x[i * S::o + q]));
        g4_atomic_xor(sacc + g, acc);
    }
    __syncthreads();
    for (int idx = tid; idx < S::k * W * 4; idx += NT) {  // packed word qw of accumulator (i, w) -> 8 nibbles
        const int g = idx >> 2, qw = idx & 3;
        const int i = g / W, w = g - i * W;
        const uint4 u = g4_to_packed(g4_ld(sacc + g));
        const uint32_t wd = qw == 0 ? u.x : (qw == 1 ? u.y : (qw == 2 ? u.z : u.w));
#pragma unroll
        for (int e = 0; e < 8; e++) {
            const int c = 32 * w + 8 * qw + e;
            if (c < S::m) snib[i * S::n + c] = (uint8_t)((wd >> (4 * e)) & 0xF);
        }
    }
    __syncthreads();
    uint8_t *sigp = sig;  // nullptr: compute only (an instance of a multi-instance CTA that writes nothing)
    if (sigp) {
        for (int bidx = tid; bidx < S::k * S::n / 2; bidx += NT)
            sigp[bidx] = (uint8_t)(snib[2 * bidx] | (snib[2 * bidx + 1] << 4));
        for (int i = tid; i < S::sk; i += NT) sigp[S::k * S::n / 2 + i] = s_key[S::digest + i];
    }
}

}  // namespace mayo
