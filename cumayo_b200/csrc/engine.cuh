// engine.cuh -- the m-vector multiply-accumulate engine used by every MAYO operation.
//
// All heavy arithmetic of MAYO has one shape: for a "row" r, a list of m-vector entries
// P[r][e] (each Menc packed bytes in HBM) and a scalar matrix S, compute for each output j
//     T_j[r] = sum_e S[col(r, e)][j] * P[r][e]
// and, for the public-map evaluations, also X[i][j] += S[r][i] * T_j[r].
//   keypair  P3 = Upper(O^T (P1 O + P2))      rows of P1|P2, S = [O; I]   (src/keypair.cu:55-120)
//   expandsk L  = (P1 + P1^T) O + P2           rows of P1 (both halves), S = [O; I] (src/expandsk.cu:37-80)
//   sign     M_i = V_i L                        "rows" are columns of L, S = V  (src/sign.cu:256-330)
//   sign     U_ij = V_i^T P1 V_j (+ sym)        rows of P1, S = V           (src/sign.cu:396-437)
//   verify   U_ij = s_i^T P s_j (+ sym)         rows of P1|P2 and P3, S = s (src/verify.cu:72-182)
//
// B200 mapping: one CTA per instance.  Threads are (j, w, rs): output j, 32-coordinate group w of
// the m-vector, row slot rs.  A batch of R rows is converted cooperatively from packed nibbles
// (5 aligned 32-bit loads, funnel shifts, a 4x4 bit transpose per nibble position) into
// bit-planes in shared memory; then each thread walks its row with two 128-bit shared loads
// (entry planes, broadcast across j; the scalar's four masks) and 16 LOP3 per entry-group.
// Scalars enter only through masks, so the arithmetic is constant time whatever the data.
#pragma once

#include "common.cuh"

namespace mayo {

// Packed bytes [p, p + n) (n <= 16) of an m-vector group as four LE words, touching only
// aligned 32-bit words that contain at least one requested byte.  RO selects the read-only
// (non-coherent) load path, valid only for data no thread writes during the kernel.
template <bool RO = true, bool GLOBAL = false>
__device__ __forceinline__ void load_group_words(const uint8_t *p, int n, uint32_t &w0, uint32_t &w1, uint32_t &w2,
                                                 uint32_t &w3) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t *q = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
    const uint32_t sh = (uint32_t)(a & 3) * 8;
    // number of aligned words covering [p, p + n)
    const int nw = (int)(((a & 3) + n + 3) >> 2);
    uint32_t x[5];
    // GLOBAL: the entry is known to be in global memory; the explicit global load (L1-cached,
    // coherent) lets the compiler issue it ahead of earlier shared-memory stores
#pragma unroll
    for (int i = 0; i < 5; i++) x[i] = i < nw ? (RO ? __ldg(q + i) : GLOBAL ? __ldca(q + i) : q[i]) : 0u;
    w0 = __funnelshift_r(x[0], x[1], sh);
    w1 = __funnelshift_r(x[1], x[2], sh);
    w2 = __funnelshift_r(x[2], x[3], sh);
    w3 = __funnelshift_r(x[3], x[4], sh);
    if (n < 16) {
        // clear bytes n..15
        const uint32_t keep[4] = {n >= 4 ? 0xffffffffu : (1u << (8 * n)) - 1,
                                  n >= 8 ? 0xffffffffu : (n <= 4 ? 0u : (1u << (8 * (n - 4))) - 1),
                                  n >= 12 ? 0xffffffffu : (n <= 8 ? 0u : (1u << (8 * (n - 8))) - 1),
                                  n <= 12 ? 0u : (1u << (8 * (n - 12))) - 1};
        w0 &= keep[0];
        w1 &= keep[1];
        w2 &= keep[2];
        w3 &= keep[3];
    }
}

// Bytes valid in group w of an m-vector of Menc bytes.
template <int MENC>
__device__ __forceinline__ int group_bytes(int w) {
    return min(16, MENC - 16 * w);
}

template <int SET, bool RO = true>
__device__ __forceinline__ G4 load_group(const uint8_t *entry, int w) {
    uint32_t w0, w1, w2, w3;
    load_group_words<RO>(entry + 16 * w, group_bytes<Set<SET>::menc>(w), w0, w1, w2, w3);
    return g4_from_packed(w0, w1, w2, w3);
}

// Rows functors may declare `static constexpr bool read_only = false;` when their entries are
// written during the same kernel; the default is the read-only load path.
template <class Rows, class = void>
struct RowsReadOnly {
    static constexpr bool value = true;
};
template <class Rows>
struct RowsReadOnly<Rows, decltype((void)Rows::read_only)> {
    static constexpr bool value = Rows::read_only;
};

// Write bit-plane group g (group w of an m-vector) as packed bytes to any address.
template <int SET>
__device__ __forceinline__ void store_group(uint8_t *entry, int w, G4 g) {
    const uint4 u = g4_to_packed(g);
    const int n = group_bytes<Set<SET>::menc>(w);
    uint8_t *p = entry + 16 * w;
    const uint32_t wd[4] = {u.x, u.y, u.z, u.w};
    if (n == 16 && (reinterpret_cast<uintptr_t>(p) & 3) == 0) {
        uint32_t *q = reinterpret_cast<uint32_t *>(p);
        q[0] = wd[0];
        q[1] = wd[1];
        q[2] = wd[2];
        q[3] = wd[3];
    } else {
#pragma unroll
        for (int i = 0; i < 16; i++)
            if (i < n) p[i] = (uint8_t)(wd[i >> 2] >> (8 * (i & 3)));
    }
}

// Shared-memory layout used by the engine.
template <int SET, int J, int R>
struct EngineSmem {
    using S = Set<SET>;
    static constexpr int W = S::W;
    static constexpr int MAXE = S::n;  // longest row: v + o entries
};

// Engine state of one thread.  Rows are described by a functor with
//   __device__ int count(int r) const;                  entries in row r
//   __device__ const uint8_t *entry(int r, int e) const; packed entry (nullptr -> zero vector)
//   __device__ int col(int r, int e) const;             scalar column of entry e
// X4: row products with four partial sums (row_product_x4, measured 3-4 % faster keypair, sign
// and verify at 1,024 instances, 4 % on the mixed queue); off where a kernel's register budget
// leaves no room for the twelve extra live registers.
// CU: groups whose loads a thread issues together in convert (1: one group at a time).
template <int SET, int J, int R, bool X4 = true, int CU = 1>
struct Engine {
    using S = Set<SET>;
    static constexpr int W = S::W;
    static constexpr int MAXE = S::n;
    static constexpr int ACTIVE = J * W * R;

    const uint4 *masks;  // [ncols][J]   masks of S[c][j]
    uint4 *bs;           // [R][MAXE][W] bit-plane staging of the current rows
    int j, w, rs;
    bool active;

    __device__ __forceinline__ void setup(const uint4 *masks_, uint4 *bs_, int tid) {
        masks = masks_;
        bs = bs_;
        active = tid < ACTIVE;
        const int t = active ? tid : 0;
        j = t % J;
        w = (t / J) % W;
        rs = t / (J * W);
    }

    // Convert rows [r0, r0 + R) (those < nrows) into bs; all `nthreads` threads take part.  With
    // CU > 1 a thread issues the loads of CU groups (entries in global memory only) before it
    // converts and stores any of them, so that CU round trips to L2 / HBM overlap.
    template <class Rows>
    __device__ __forceinline__ void convert(const Rows &rows, int r0, int nrows, int tid, int nthreads) {
        constexpr bool RO = RowsReadOnly<Rows>::value;
#pragma unroll 1
        for (int slot = 0; slot < R; slot++) {
            const int r = r0 + slot;
            if (r >= nrows) break;
            const int n = rows.count(r) * W;
            uint4 *dst = bs + (size_t)slot * MAXE * W;
            if constexpr (CU == 1) {
                for (int idx = tid; idx < n; idx += nthreads) {
                    const int e = idx / W, ww = idx - e * W;
                    const uint8_t *src = rows.entry(r, e);
                    G4 g = src ? load_group<SET, RO>(src, ww) : g4_zero();
                    g4_st(dst + idx, g);
                }
            } else {
#pragma unroll 1
                for (int i0 = tid; i0 < n; i0 += CU * nthreads) {
                    uint32_t x[CU][4];
#pragma unroll
                    for (int u = 0; u < CU; u++) {
                        const int idx = i0 + u * nthreads;
                        x[u][0] = x[u][1] = x[u][2] = x[u][3] = 0u;
                        if (idx < n) {
                            const int e = idx / W, ww = idx - e * W;
                            const uint8_t *src = rows.entry(r, e);
                            if (src)
                                load_group_words<RO, true>(src + 16 * ww, group_bytes<S::menc>(ww), x[u][0], x[u][1],
                                                           x[u][2], x[u][3]);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < CU; u++) {
                        const int idx = i0 + u * nthreads;
                        if (idx < n) g4_st(dst + idx, g4_from_packed(x[u][0], x[u][1], x[u][2], x[u][3]));
                    }
                }
            }
        }
    }

    // Ask L2 for the entries of rows [r0, r0 + R) (those < nrows), both 128-byte lines an entry
    // can touch, one warp issuing (lane = 0..31); no completion to wait for.  Called one pass
    // ahead of convert, so that the next rows' loads hit L2 instead of HBM.
    template <class Rows>
    __device__ __forceinline__ void prefetch(const Rows &rows, int r0, int nrows, int lane) const {
#pragma unroll 1
        for (int slot = 0; slot < R; slot++) {
            const int r = r0 + slot;
            if (r >= nrows) break;
            const int cnt = rows.count(r);
            for (int e = lane; e < cnt; e += 32) {
                const uint8_t *p = rows.entry(r, e);
                if (p) {
                    asm volatile("prefetch.L2 [%0];" ::"l"(p));
                    asm volatile("prefetch.L2 [%0];" ::"l"(p + S::menc - 1));
                }
            }
        }
    }

    // T_j[r] for this thread's (j, w) over row r = r0 + rs (call only when active and r < nrows).
    template <class Rows>
    __device__ __forceinline__ G4 row_product(const Rows &rows, int r) const {
        if constexpr (X4) return row_product_x4(rows, r);
        G4 acc = g4_zero();
        const int cnt = rows.count(r);
        const uint4 *bp = bs + (size_t)rs * MAXE * W + w;
        const int c0 = rows.col(r, 0);
        const uint4 *mp = masks + (size_t)c0 * J + j;
#pragma unroll 4
        for (int e = 0; e < cnt; e++) {
            const G4 v = g4_ld(bp + e * W);
            const uint4 m = mp[e * J];
            g4_madd(acc, v, m);
        }
        return acc;
    }
    // The same with four partial sums, one per power of x, folded once at the end of the row
    // (g4x4_madd): three XORs fewer per entry, twelve more live registers.
    template <class Rows>
    __device__ __forceinline__ G4 row_product_x4(const Rows &rows, int r) const {
        G4x4 acc = g4x4_zero();
        const int cnt = rows.count(r);
        const uint4 *bp = bs + (size_t)rs * MAXE * W + w;
        const int c0 = rows.col(r, 0);
        const uint4 *mp = masks + (size_t)c0 * J + j;
#pragma unroll 4
        for (int e = 0; e < cnt; e++) {
            const G4 v = g4_ld(bp + e * W);
            const uint4 m = mp[e * J];
            g4x4_madd(acc, v, m);
        }
        return g4x4_fold(acc);
    }
};

// XOR-accumulate a G4 into shared memory (atomic, so row slots can share one accumulator).
__device__ __forceinline__ void g4_atomic_xor(uint4 *dst, const G4 &g) {
    uint32_t *d = reinterpret_cast<uint32_t *>(dst);
    atomicXor(d + 0, g.p0);
    atomicXor(d + 1, g.p1);
    atomicXor(d + 2, g.p2);
    atomicXor(d + 3, g.p3);
}

// Named barrier over the first `n` threads (n a multiple of 32).
__device__ __forceinline__ void bar_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
// Named barrier that also returns the OR of `pred` over the participating threads (uniform).
__device__ __forceinline__ bool bar_red_or(int id, int n, bool pred) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)pred), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

// ---------------------------------------------------------------------------------------------
// z * y mod f(z) on a packed m-vector held one 32-bit word (8 coordinates) per lane, lanes
// 0..NW-1 (others hold zero).  Constant time.  Reference: include/poly.cuh:11-69.
// ---------------------------------------------------------------------------------------------
template <int SET>
__device__ __forceinline__ uint32_t times_z_lane(uint32_t y, int lane) {
    using S = Set<SET>;
    constexpr int m = S::m;
    constexpr int NW = (S::menc + 3) / 4;
    constexpr int top_lane = (m - 1) / 8, top_nib = (m - 1) % 8;
    const uint32_t prev = __shfl_up_sync(0xffffffffu, y, 1);
    const uint32_t topw = __shfl_sync(0xffffffffu, y, top_lane);
    const uint32_t top = (topw >> (4 * top_nib)) & 0xF;
    uint32_t r = (y << 4) | (lane > 0 ? (prev >> 28) : 0u);
    // drop what moved to coordinate m (and beyond)
    if (lane == m / 8 && (m % 8) != 0) r &= (1u << (4 * (m % 8))) - 1;
    if (lane >= NW || (lane == m / 8 && (m % 8) == 0)) r = 0;
    if (lane == 0) {
        const uint32_t f = gf16_mul_ct(top, S::cf(0)) | (gf16_mul_ct(top, S::cf(1)) << 4) |
                           (gf16_mul_ct(top, S::cf(2)) << 8) | (gf16_mul_ct(top, S::cf(3)) << 12);
        r ^= f;
    }
    return r;
}

}  // namespace mayo
