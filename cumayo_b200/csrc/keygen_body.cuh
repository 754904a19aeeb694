// keygen_body.cuh -- P3 of a keypair (reference src/keypair.cu:55-120) and L of an expanded
// secret key (src/expandsk.cu:37-80) on one CTA, shared by the batched kernels and the
// persistent work-queue kernel.
#pragma once

#include "engine.cuh"
#include "launch_util.cuh"

namespace mayo {

template <int SET, int NT_ = 0>
struct KeyCfg {
    using S = Set<SET>;
    static constexpr int J = S::o, W = S::W;
    static constexpr int R_DEF = SET == 1 ? 5 : (SET == 2 ? 3 : (SET == 3 ? 3 : 2));
    static constexpr int NT = NT_ ? NT_ : (J * W * R_DEF + 31) / 32 * 32;
    static constexpr int R = NT / (J * W) < R_DEF ? NT / (J * W) : R_DEF;
    static_assert(R >= 1 && J * W * R <= NT, "engine threads");
    static constexpr size_t off_masks = 0;
    static constexpr size_t off_bs = off_masks + (size_t)S::n * J * 16;
    static constexpr size_t off_x = off_bs + (size_t)R * S::n * W * 16;
    static constexpr size_t off_o = off_x + (size_t)J * J * W * 16;
    static constexpr size_t total = off_o + pad16(S::o_bytes);
};

// masks[c][b]: c < v -> O[c][b]; c >= v -> identity (adds P2 entries unscaled)
template <int SET>
__device__ __forceinline__ void build_o_masks(uint4 *masks, const uint8_t *s_O, int tid, int nthreads) {
    using S = Set<SET>;
    for (int idx = tid; idx < S::n * S::o; idx += nthreads) {
        const int c = idx / S::o, b = idx - c * S::o;
        uint32_t s;
        if (c < S::v) {
            const int q = c * S::o + b;
            s = (s_O[q >> 1] >> ((q & 1) * 4)) & 0xF;
        } else {
            s = (c - S::v == b) ? 1u : 0u;
        }
        masks[idx] = scalar_masks(s);
    }
}

template <int SET, bool RO = true>
struct P3Rows {  // rows r < v of [P1 | P2] (src/keypair.cu:67-92)
    using S = Set<SET>;
    static constexpr bool read_only = RO;
    const uint8_t *P1, *P2;
    __device__ __forceinline__ int count(int r) const { return (S::v - r) + S::o; }
    __device__ __forceinline__ const uint8_t *entry(int r, int e) const {
        const int n1 = S::v - r;
        return e < n1 ? P1 + (size_t)tri(r, r + e, S::v) * S::menc : P2 + (size_t)(r * S::o + (e - n1)) * S::menc;
    }
    __device__ __forceinline__ int col(int r, int e) const { return r + e; }
};

template <int SET>
struct LRows {  // row r of P1 + P1^T without the diagonal, then P2 row r (src/expandsk.cu:162-199)
    using S = Set<SET>;
    static constexpr bool read_only = false;  // L overwrites P2 in the same kernel
    const uint8_t *P1, *P2;
    __device__ __forceinline__ int count(int) const { return S::n; }
    __device__ __forceinline__ const uint8_t *entry(int r, int e) const {
        if (e < S::v) {
            if (e == r) return nullptr;
            return P1 + (size_t)(e > r ? tri(r, e, S::v) : tri(e, r, S::v)) * S::menc;
        }
        return P2 + (size_t)(r * S::o + (e - S::v)) * S::menc;
    }
    __device__ __forceinline__ int col(int, int e) const { return e; }
};

// P3 = Upper(O^T (P1 O + P2)) for one instance: O (o_bytes) already in smem at off_o; writes the
// packed upper triangle to P3out.  All NT threads must call it.  RO: P1/P2 read-only in this kernel.
template <int SET, int NT_, bool RO, int CU = 1>
__device__ __forceinline__ void p3_instance(uint8_t *smem, int tid, const uint8_t *P1, const uint8_t *P2,
                                            uint8_t *P3out) {
    using S = Set<SET>;
    using C = KeyCfg<SET, NT_>;
    constexpr int J = C::J, W = C::W, R = C::R, NT = C::NT;
    uint4 *masks = reinterpret_cast<uint4 *>(smem + C::off_masks);
    uint4 *bs = reinterpret_cast<uint4 *>(smem + C::off_bs);
    uint4 *xacc = reinterpret_cast<uint4 *>(smem + C::off_x);
    const uint8_t *s_O = smem + C::off_o;
    for (int i = tid; i < J * J * W * 4; i += NT) reinterpret_cast<uint32_t *>(xacc)[i] = 0;
    build_o_masks<SET>(masks, s_O, tid, NT);
    __syncthreads();

    Engine<SET, J, R, true, CU> eng;
    eng.setup(masks, bs, tid);
    const P3Rows<SET, RO> rows{P1, P2};
    G4 X[J];
#pragma unroll
    for (int i = 0; i < J; i++) X[i] = g4_zero();
#pragma unroll 1
    for (int r0 = 0; r0 < S::v; r0 += R) {
        // the next pass's rows into L2 (MAYO_1/3/5 keypairs 1-5 % faster, MAYO_2's 4 % slower)
        if (SET != 2 && tid < 32) eng.prefetch(rows, r0 + R, S::v, tid);
        eng.convert(rows, r0, S::v, tid, NT);
        __syncthreads();
        const int r = r0 + eng.rs;
        if (eng.active && r < S::v) {
            const G4 T = eng.row_product(rows, r);  // B[r][j] = (P1 O + P2)[r][j]
            const uint4 *mr = masks + (size_t)r * J;  // O[r][a]
#pragma unroll
            for (int a = 0; a < J; a++) g4_madd(X[a], T, mr[a]);
        }
        __syncthreads();
    }
    if (eng.active) {
#pragma unroll
        for (int a = 0; a < J; a++) g4_atomic_xor(xacc + ((size_t)a * J + eng.j) * W + eng.w, X[a]);
    }
    __syncthreads();
    // P3[a][b] = X_ab + X_ba (a < b), X_aa; upper triangle row-major
    for (int idx = tid; idx < S::o * (S::o + 1) / 2 * W; idx += NT) {
        const int pid = idx / W, ww = idx - pid * W;
        int a = 0, rem = pid;
        while (rem >= J - a) {
            rem -= J - a;
            a++;
        }
        const int b = a + rem;
        G4 u = g4_ld(xacc + ((size_t)a * J + b) * W + ww);
        if (a != b) u = g4_xor(u, g4_ld(xacc + ((size_t)b * J + a) * W + ww));
        store_group<SET>(P3out + (size_t)tri(a, b, S::o) * S::menc, ww, u);
    }
}

}  // namespace mayo
