// verify_body.cuh -- one MAYO verify on one CTA (reference src/verify.cu:9-212), shared by the
// batched verify kernel and the persistent work-queue kernel.
//
// Threads 0..NC-1 evaluate U_ij = s_i^T P s_j (+ symmetric term) over the expanded public key
// P = [[P1, P2], [0, P3]] with the bit-sliced engine; threads NC..NC+31 (one warp) hash
// digest = SHAKE256(M) and t = SHAKE256(digest || salt) with the warp-cooperative Keccak at the
// same time.  Warp 0 then runs the Horner sum y = sum z^l U_l and compares it with t.
#pragma once

#include "engine.cuh"
#include "launch_util.cuh"

namespace mayo {

// NC = compute threads (a multiple of 32); the CTA has NC + 32 threads.
template <int SET, int NC_ = 0>
struct VerifyCfg {
    using S = Set<SET>;
    static constexpr int J = S::k, W = S::W;
    static constexpr int R_DEF = SET == 2 ? 16 : (SET == 1 ? 4 : 2);
    static constexpr int NC = NC_ ? NC_ : (J * W * R_DEF + 31) / 32 * 32;
    static constexpr int R = NC / (J * W) < R_DEF ? NC / (J * W) : R_DEF;  // row slots that fit
    static constexpr int NT = NC + 32;
    static constexpr int NW = (S::menc + 3) / 4;  // packed words per m-vector
    static_assert(R >= 1 && J * W * R <= NC, "engine threads");
    static constexpr size_t off_masks = 0;
    static constexpr size_t off_bs = off_masks + (size_t)S::n * J * 16;
    // the U accumulators, then U's packed words, reuse the key-row staging area once the row
    // loop is done (in place after it when they do not fit)
    static constexpr size_t off_x = off_bs;
    static constexpr size_t sz_bs = (size_t)R * S::n * W * 16, sz_x = (size_t)J * J * W * 16;
    static constexpr size_t sz_upk = pad16((size_t)S::pairs * NW * 4);
    static constexpr bool UPK_IN_BS = sz_x + sz_upk <= sz_bs;
    static constexpr size_t off_upk = UPK_IN_BS ? off_bs + sz_x : off_bs + (sz_bs > sz_x ? sz_bs : sz_x);
    static constexpr size_t off_sig = UPK_IN_BS ? off_bs + sz_bs : off_upk + sz_upk;
    static constexpr size_t off_key = off_sig + pad16(S::sig);
    static constexpr size_t off_t = off_key + pad16(S::digest + S::sk);
    static constexpr size_t total = off_t + pad16(NW * 4);
};

template <int SET>
struct VerifyRows {
    using S = Set<SET>;
    const uint8_t *P1, *P2, *P3;
    __device__ __forceinline__ int count(int r) const { return r < S::v ? (S::v - r) + S::o : S::n - r; }
    __device__ __forceinline__ const uint8_t *entry(int r, int e) const {
        if (r < S::v) {
            const int n1 = S::v - r;
            return e < n1 ? P1 + (size_t)tri(r, r + e, S::v) * S::menc : P2 + (size_t)(r * S::o + (e - n1)) * S::menc;
        }
        const int rr = r - S::v;
        return P3 + (size_t)tri(rr, rr + e, S::o) * S::menc;
    }
    __device__ __forceinline__ int col(int r, int e) const { return r + e; }
    // Ask L2 for row r's entries, one warp issuing (lane = 0..31): rows of P1 || P2 and of P3 are
    // contiguous runs of m-vectors, so one prefetch per 128-byte line of each run.
    __device__ __forceinline__ void prefetch(int r, int lane) const {
        if (r < S::v) {
            prefetch_lines(P1 + (size_t)tri(r, r, S::v) * S::menc, (S::v - r) * S::menc, lane);
            prefetch_lines(P2 + (size_t)r * S::o * S::menc, S::o * S::menc, lane);
        } else if (r < S::n) {
            const int rr = r - S::v;
            prefetch_lines(P3 + (size_t)tri(rr, rr, S::o) * S::menc, (S::o - rr) * S::menc, lane);
        }
    }
    // every address issued lies in [p, p + n): the first is p, the others start 128-byte lines
    __device__ __forceinline__ static void prefetch_lines(const uint8_t *p, int n, int lane) {
        const uintptr_t a = reinterpret_cast<uintptr_t>(p), end = a + (uintptr_t)n;
        for (uintptr_t l = (a & ~uintptr_t(127)) + 128u * (uintptr_t)lane; l < end; l += 128u * 32u) {
            const uintptr_t q = l < a ? a : l;
            asm volatile("prefetch.L2 [%0];" ::"l"(q));
        }
    }
};

__device__ __forceinline__ int pair_index(int i, int j, int k) { return i * k - (i * (i - 1)) / 2 + (j - i); }

// Verify one instance; every thread of the CTA (NC + 32 of them) must call it.  Writes 0
// (accept) or 1 (reject) to *res.  `smem` holds VerifyCfg<SET, NC>::total bytes.
// `pre`, when given, holds T_j[r] = P[r] s_j for every row r < n as bit-plane groups [j][r][w],
// computed for a whole batch on the tensor cores (op_shared.cu); the engine pass over the public
// key is then skipped.
template <int SET, int NC_>
__device__ __forceinline__ void verify_instance(uint8_t *smem, int tid, const uint8_t *epk, const uint8_t *msg,
                                                uint32_t mlen, const uint8_t *sig, uint8_t *res,
                                                const uint4 *pre = nullptr) {
    using S = Set<SET>;
    using C = VerifyCfg<SET, NC_>;
    constexpr int J = C::J, W = C::W, R = C::R, NC = C::NC, NW = C::NW;
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *bs = reinterpret_cast<uint4 *>(smem + C::off_bs);
    uint4 *xacc = reinterpret_cast<uint4 *>(smem + C::off_x);
    uint32_t *upk = reinterpret_cast<uint32_t *>(smem + C::off_upk);
    uint8_t *s_sig = smem + C::off_sig;
    uint8_t *s_key = smem + C::off_key;
    uint8_t *s_t = smem + C::off_t;

    for (int i = tid; i < S::sig; i += C::NT) s_sig[i] = sig[i];
    for (int i = tid; i < NW * 4; i += C::NT) s_t[i] = 0;
    __syncthreads();

    if (tid >= NC) {
        // ---- hashing warp: digest and target t (src/verify.cu:37-48) ----
        const int lane = tid - NC;
        WarpKeccak wk;
        wk.setup(lane);
        warp_shake<136>(s_key, S::digest, msg, (int)mlen, wk, lane);
        for (int i = lane; i < S::sk; i += 32) s_key[S::digest + i] = s_sig[S::k * S::n / 2 + i];
        __syncwarp();
        warp_shake<136>(s_t, S::menc, s_key, S::digest + S::sk, wk, lane);
    } else {
        // ---- masks of the signature scalars: column c of s_j (src/verify.cu:62-70) ----
        for (int idx = tid; idx < S::n * J; idx += NC) {
            const int c = idx / J, jj = idx - c * J;
            const int q = jj * S::n + c;
            const uint32_t nib = (s_sig[q >> 1] >> ((q & 1) * 4)) & 0xF;
            masks[idx] = scalar_masks(nib);
        }
        bar_sync(1, NC);

        // MAYO_3's verify is held to 80 registers for 6 CTAs per SM: the four-partial-sum row
        // product spills there (1.48 M against 1.51 M distinct-key verify/s), so it keeps g4_madd
        Engine<SET, J, R, SET != 3> eng;
        eng.setup(masks, bs, tid);
        const VerifyRows<SET> rows{epk, epk + S::p1, epk + S::p};
        G4 X[J];
#pragma unroll
        for (int i = 0; i < J; i++) X[i] = g4_zero();
        if (pre) {
            if (eng.active) {
#pragma unroll 1
                for (int r = eng.rs; r < S::n; r += R) {
                    const G4 T = g4_ld(pre + ((size_t)eng.j * S::n + r) * W + eng.w);
                    const uint4 *mr = masks + (size_t)r * J;
#pragma unroll
                    for (int i = 0; i < J; i++) g4_madd(X[i], T, mr[i]);
                }
            }
        } else {
#pragma unroll 1
            for (int r0 = 0; r0 < S::n; r0 += R) {
                // the next pass's key rows into L2, per entry (MAYO_1/5: distinct-key verify of
                // MAYO_5 0.745 -> 0.780 M/s, MAYO_1 verifyWithepk 1 % faster) or per 128-byte line of
                // each row's runs (MAYO_3, whose kernel is held to 80 registers: verifyWithepk 3 %
                // faster); MAYO_2's measured 3 % slower with either
                if (tid < 32) {
                    if constexpr (SET == 1 || SET == 5) eng.prefetch(rows, r0 + R, S::n, tid);
                    if constexpr (SET == 3)
#pragma unroll 1
                        for (int q = 0; q < R; q++) rows.prefetch(r0 + R + q, tid);
                }
                eng.convert(rows, r0, S::n, tid, NC);
                bar_sync(1, NC);
                const int r = r0 + eng.rs;
                if (eng.active && r < S::n) {
                    const G4 T = eng.row_product(rows, r);
                    const uint4 *mr = masks + (size_t)r * J;
#pragma unroll
                    for (int i = 0; i < J; i++) g4_madd(X[i], T, mr[i]);
                }
                bar_sync(1, NC);
            }
        }
        // the staging area is free now (the last row pass ended with a barrier): zero the
        // accumulators there, then combine the threads' partial sums
        for (int i = tid; i < J * J * W * 4; i += NC) reinterpret_cast<uint32_t *>(xacc)[i] = 0;
        bar_sync(1, NC);
        if (eng.active) {
#pragma unroll
            for (int i = 0; i < J; i++) g4_atomic_xor(xacc + ((size_t)i * J + eng.j) * W + eng.w, X[i]);
        }
        bar_sync(1, NC);
        // ---- U_ij (i <= j) to packed words ----
        for (int idx = tid; idx < S::pairs * W; idx += NC) {
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
    }
    __syncthreads();

    // ---- y = Horner over the pairs (i = k-1..0, j = i..k-1), compare with t (src/verify.cu:185-211) ----
    if (tid < 32) {
        const int lane = tid;
        uint32_t y = 0;
#pragma unroll 1
        for (int i = S::k - 1; i >= 0; i--)
#pragma unroll 1
            for (int j = i; j < S::k; j++) {
                y = times_z_lane<SET>(y, lane);
                if (lane < NW) y ^= upk[pair_index(i, j, S::k) * NW + lane];
            }
        const uint32_t tw = lane < NW ? reinterpret_cast<const uint32_t *>(s_t)[lane] : 0u;
        const bool eq = __all_sync(0xffffffffu, y == tw);
        if (lane == 0) *res = eq ? 0 : 1;
    }
}

}  // namespace mayo
