// common.cuh -- parameter sets, Keccak, bitsliced GF(16) and small utilities shared by
// every kernel of the B200 MAYO engine.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace mayo {

// ---------------------------------------------------------------------------------------------
// Parameter sets.  Values are the reference's include/params.h:10-92; the derived sizes are
// asserted below.  One template instance per set, so all four sets live in one library
// (the reference selects one set per binary at compile time).
// ---------------------------------------------------------------------------------------------
template <int SET>
struct Set;

#define MAYO_SET(ID, N, M, O, K, SKB, PKB, PB, OB, P1B, P2B, DIG, PAIRS, C0, C1, C2, C3)                 \
    template <>                                                                                         \
    struct Set<ID> {                                                                                    \
        static constexpr int id = ID, n = N, m = M, o = O, k = K;                                       \
        static constexpr int sk = SKB, pk = PKB, p = PB, o_bytes = OB, p1 = P1B, p2 = P2B;              \
        static constexpr int digest = DIG, pairs = PAIRS;                                               \
        /* tail of f(z) = z^m + c3 z^3 + c2 z^2 + c1 z + c0 */                                          \
        __host__ __device__ static constexpr uint32_t cf(int i) {                                       \
            return i == 0 ? C0 : i == 1 ? C1 : i == 2 ? C2 : C3;                                        \
        }                                                                                               \
        static constexpr int v = n - o, menc = m / 2, W = (m + 31) / 32;                                \
        static constexpr int sig = k * n / 2 + sk, esk = sk + o_bytes + p, epk = p + pk - 16;           \
        static constexpr int ko = k * o, vr = n * k / 2, e1 = v * (v + 1) / 2;                          \
        static constexpr int scratch = k * m * ((o + 1) / 2);                                           \
        static_assert(v == m, "every MAYO set has v == m");                                             \
        static_assert(p1 == menc * v * (v + 1) / 2, "P1 size");                                         \
        static_assert(p2 == menc * v * o, "P2 size");                                                   \
        static_assert(p == p1 + p2, "P size");                                                          \
        static_assert(pk == 16 + menc * o * (o + 1) / 2, "PK size");                                    \
        static_assert(o_bytes == v * o / 2, "O size");                                                  \
        static_assert(pairs == k * (k + 1) / 2, "pairs");                                               \
        static_assert(ko >= m, "system must be wide");                                                  \
        static_assert(pairs + 3 < m, "a single fold by f(z) suffices");                                 \
    };

MAYO_SET(1, 86, 78, 8, 10, 24, 1420, 144495, 312, 120159, 24336, 32, 55, 0x8, 0x1, 0x1, 0x0)
MAYO_SET(2, 81, 64, 17, 4, 24, 4912, 101376, 544, 66560, 34816, 32, 10, 0x8, 0x0, 0x2, 0x8)
MAYO_SET(3, 118, 108, 10, 11, 32, 2986, 376164, 540, 317844, 58320, 48, 66, 0x8, 0x0, 0x1, 0x7)
MAYO_SET(5, 154, 142, 12, 12, 40, 5554, 841847, 852, 720863, 120984, 64, 78, 0x4, 0x0, 0x8, 0x1)
#undef MAYO_SET

__host__ __device__ constexpr int align128(int x) { return (x + 127) / 128 * 128; }
__host__ __device__ constexpr size_t align128z(size_t x) { return (x + 127) / 128 * 128; }
// upper-triangular dim x dim (r <= c) entry index, row-major (reference include/code.h:14-20)
__host__ __device__ constexpr int tri(int r, int c, int dim) { return c - r + dim * r - (r * (r - 1)) / 2; }

// ---------------------------------------------------------------------------------------------
// Small device utilities
// ---------------------------------------------------------------------------------------------
// LOP3 truth tables are functions of a = 0xF0, b = 0xCC, c = 0xAA.
__host__ __device__ __forceinline__ uint32_t lop_xor3(uint32_t a, uint32_t b, uint32_t c) {
#ifdef __CUDA_ARCH__
    uint32_t r;
    asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(a), "r"(b), "r"(c));  // a ^ b ^ c
    return r;
#else
    return a ^ b ^ c;
#endif
}
// a ^ (b & c): 0xF0 ^ (0xCC & 0xAA) = 0x78
__host__ __device__ __forceinline__ uint32_t lop_xand(uint32_t a, uint32_t b, uint32_t c) {
#ifdef __CUDA_ARCH__
    uint32_t r;
    asm("lop3.b32 %0, %1, %2, %3, 0x78;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
#else
    return a ^ (b & c);
#endif
}

// 4-byte little-endian load from an arbitrary byte address; bytes p..p+3 must be valid.
// Uses aligned word loads only, so it never touches a word without a valid byte.
__device__ __forceinline__ uint32_t ld_le32(const uint8_t *p) {
    uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t *q = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
    uint32_t sh = (uint32_t)(a & 3) * 8;
    uint32_t lo = __ldg(q);
    if (sh == 0) return lo;
    uint32_t hi = __ldg(q + 1);
    return __funnelshift_r(lo, hi, sh);
}

// Little-endian load of n (0..8) bytes at p, zero-filled above.
__device__ __forceinline__ uint64_t ld_le64_part(const uint8_t *p, int n) {
    if (n >= 8 && (reinterpret_cast<uintptr_t>(p) & 7) == 0) return *reinterpret_cast<const uint64_t *>(p);
    uint64_t w = 0;
#pragma unroll
    for (int b = 0; b < 8; b++)
        if (b < n) w |= (uint64_t)p[b] << (8 * b);
    return w;
}

// ---------------------------------------------------------------------------------------------
// Keccak-f[1600] (FIPS 202).  Constants derived at compile time from the definitions: rho
// offsets from the (x, y) -> (y, 2x + 3y) walk, iota constants from the rc() LFSR.
// ---------------------------------------------------------------------------------------------
struct KeccakTables {
    uint64_t rc[24];
    int rho[25];
};
__host__ __device__ constexpr KeccakTables make_keccak_tables() {
    KeccakTables t{};
    int x = 1, y = 0;
    t.rho[0] = 0;
    for (int i = 0; i < 24; i++) {
        t.rho[x + 5 * y] = ((i + 1) * (i + 2) / 2) % 64;
        int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    for (int ir = 0; ir < 24; ir++) {
        uint64_t rcv = 0;
        for (int j = 0; j <= 6; j++) {
            int tt = (j + 7 * ir) % 255;
            unsigned r = 1;
            for (int s = 1; s <= tt; s++) {
                r <<= 1;
                if (r & 0x100) r ^= 0x171;
                r &= 0xFF;
            }
            if (r & 1) rcv |= (uint64_t)1 << ((1 << j) - 1);
        }
        t.rc[ir] = rcv;
    }
    return t;
}
constexpr KeccakTables kKeccak = make_keccak_tables();
__constant__ uint64_t c_keccak_rc[24] = {
    kKeccak.rc[0],  kKeccak.rc[1],  kKeccak.rc[2],  kKeccak.rc[3],  kKeccak.rc[4],  kKeccak.rc[5],
    kKeccak.rc[6],  kKeccak.rc[7],  kKeccak.rc[8],  kKeccak.rc[9],  kKeccak.rc[10], kKeccak.rc[11],
    kKeccak.rc[12], kKeccak.rc[13], kKeccak.rc[14], kKeccak.rc[15], kKeccak.rc[16], kKeccak.rc[17],
    kKeccak.rc[18], kKeccak.rc[19], kKeccak.rc[20], kKeccak.rc[21], kKeccak.rc[22], kKeccak.rc[23]};
__constant__ int c_keccak_rho[25] = {
    kKeccak.rho[0],  kKeccak.rho[1],  kKeccak.rho[2],  kKeccak.rho[3],  kKeccak.rho[4],
    kKeccak.rho[5],  kKeccak.rho[6],  kKeccak.rho[7],  kKeccak.rho[8],  kKeccak.rho[9],
    kKeccak.rho[10], kKeccak.rho[11], kKeccak.rho[12], kKeccak.rho[13], kKeccak.rho[14],
    kKeccak.rho[15], kKeccak.rho[16], kKeccak.rho[17], kKeccak.rho[18], kKeccak.rho[19],
    kKeccak.rho[20], kKeccak.rho[21], kKeccak.rho[22], kKeccak.rho[23], kKeccak.rho[24]};

// 64-bit rotate by a constant as two 32-bit funnel shifts of the halves (fewer instructions
// than the compiler's generic 64-bit rotate: measured 20 % fewer per Keccak-f on sm_100a).
template <int R>
__device__ __forceinline__ uint64_t rotl64c(uint64_t a) {
    if constexpr (R == 0) {
        return a;
    } else {
        const uint32_t lo = (uint32_t)a, hi = (uint32_t)(a >> 32);
        uint32_t nlo, nhi;
        if constexpr (R < 32) {
            nhi = __funnelshift_l(lo, hi, R);
            nlo = __funnelshift_l(hi, lo, R);
        } else if constexpr (R == 32) {
            nhi = lo;
            nlo = hi;
        } else {
            nhi = __funnelshift_l(hi, lo, R - 32);
            nlo = __funnelshift_l(lo, hi, R - 32);
        }
        return ((uint64_t)nhi << 32) | nlo;
    }
}

// One thread, whole state in registers.
__device__ __forceinline__ void keccak_f1600(uint64_t (&A)[25]) {
#pragma unroll 1
    for (int round = 0; round < 24; ++round) {
        uint64_t C[5], D[5], B[25];
#pragma unroll
        for (int x = 0; x < 5; x++) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
#pragma unroll
        for (int x = 0; x < 5; x++) D[x] = C[(x + 4) % 5] ^ rotl64c<1>(C[(x + 1) % 5]);
#define KRP(X, Y)                                                                            \
    B[(Y) + 5 * ((2 * (X) + 3 * (Y)) % 5)] = rotl64c<kKeccak.rho[(X) + 5 * (Y)]>(A[(X) + 5 * (Y)] ^ D[X]);
        KRP(0, 0) KRP(1, 0) KRP(2, 0) KRP(3, 0) KRP(4, 0)
        KRP(0, 1) KRP(1, 1) KRP(2, 1) KRP(3, 1) KRP(4, 1)
        KRP(0, 2) KRP(1, 2) KRP(2, 2) KRP(3, 2) KRP(4, 2)
        KRP(0, 3) KRP(1, 3) KRP(2, 3) KRP(3, 3) KRP(4, 3)
        KRP(0, 4) KRP(1, 4) KRP(2, 4) KRP(3, 4) KRP(4, 4)
#undef KRP
#pragma unroll
        for (int y = 0; y < 5; y++)
#pragma unroll
            for (int x = 0; x < 5; x++)
                A[x + 5 * y] = B[x + 5 * y] ^ ((~B[(x + 1) % 5 + 5 * y]) & B[(x + 2) % 5 + 5 * y]);
        A[0] ^= c_keccak_rc[round];
    }
}

// Per-thread SHAKE sponge (rate in bytes: 168 for SHAKE128, 136 for SHAKE256).
template <int RATE>
struct Sponge {
    static constexpr int RW = RATE / 8;
    uint64_t s[25];
    int pos;  // bytes absorbed in the current block

    __device__ __forceinline__ void init() {
#pragma unroll
        for (int i = 0; i < 25; i++) s[i] = 0;
        pos = 0;
    }
    // Absorb `len` bytes from any generic address (global, shared or local).  The state stays
    // in registers: every state word is addressed with a compile-time index.
    __device__ void absorb(const uint8_t *p, uint32_t len) {
        // Global memory from the start of a block: aligned 8-byte loads, each word of the block
        // funnel-shifted out of two of them (one new load per word), instead of one load per byte
        // of an unaligned message.  Every aligned word read holds at least one input byte, so no
        // read leaves the pages the input lies in; bytes outside the input are masked off.
        const bool aligned_path = __isGlobal(p) != 0;
        while (aligned_path && pos == 0 && len >= (uint32_t)RATE) {
            const uint32_t off = (uint32_t)(reinterpret_cast<uintptr_t>(p) & 7u);
            const uint64_t *q = reinterpret_cast<const uint64_t *>(p - off);
            if (off == 0) {
#pragma unroll
                for (int i = 0; i < RW; i++) s[i] ^= q[i];
            } else {
                const uint32_t sh = 8u * off;
                uint64_t w0 = q[0];
#pragma unroll
                for (int i = 0; i < RW; i++) {
                    const uint64_t w1 = q[i + 1];
                    s[i] ^= (w0 >> sh) | (w1 << (64u - sh));
                    w0 = w1;
                }
            }
            keccak_f1600(s);
            p += RATE;
            len -= RATE;
        }
        if (aligned_path && pos == 0 && len > 0) {  // a last partial block (len < RATE)
            const uint32_t off = (uint32_t)(reinterpret_cast<uintptr_t>(p) & 7u);
            const uint64_t *q = reinterpret_cast<const uint64_t *>(p - off);
            const int n = (int)len;
            const uint32_t sh = 8u * off;
            uint64_t w0 = q[0];
#pragma unroll
            for (int i = 0; i < RW; i++) {
                if (8 * i < n) {
                    uint64_t v;
                    if (off == 0) {
                        v = i ? q[i] : w0;
                    } else {
                        // the word's last input byte lies in the next aligned word, or the input
                        // ends inside this one (and no later word has input bytes)
                        const int last = min(8 * i + 7, n - 1);
                        const uint64_t w1 = (int)off + last >= 8 * (i + 1) ? q[i + 1] : 0ull;
                        v = (w0 >> sh) | (w1 << (64u - sh));
                        w0 = w1;
                    }
                    if (8 * i + 8 > n) v &= ~0ull >> (64 - 8 * (n - 8 * i));
                    s[i] ^= v;
                }
            }
            pos = n;
            return;
        }
        if ((reinterpret_cast<uintptr_t>(p) & 7) == 0 && ((pos | (int)len) & 7) == 0) {
            // whole aligned words at a word position (any memory space: exactly the input's words)
            const uint64_t *q = reinterpret_cast<const uint64_t *>(p);
            while (len > 0) {
                const int take = min((int)len, RATE - pos);
#pragma unroll
                for (int i = 0; i < RW; i++)
                    if (8 * i >= pos && 8 * i < pos + take) s[i] ^= q[i - (pos >> 3)];
                q += take >> 3;
                pos += take;
                len -= take;
                if (pos == RATE) {
                    keccak_f1600(s);
                    pos = 0;
                }
            }
            return;
        }
        while (len > 0) {
            const int take = min((int)len, RATE - pos);
#pragma unroll
            for (int i = 0; i < RW; i++) {
                const int lo = max(8 * i, pos), hi = min(8 * i + 8, pos + take);
                if (lo < hi) s[i] ^= ld_le64_part(p + (lo - pos), hi - lo) << (8 * (lo - 8 * i));
            }
            pos += take;
            p += take;
            len -= take;
            if (pos == RATE) {
                keccak_f1600(s);
                pos = 0;
            }
        }
    }
    // Absorb n zero bytes: XOR with zero leaves the state; only the position moves.
    __device__ __forceinline__ void absorb_zeros(int n) {
        while (n > 0) {
            const int take = min(n, RATE - pos);
            pos += take;
            n -= take;
            if (pos == RATE) {
                keccak_f1600(s);
                pos = 0;
            }
        }
    }
    __device__ __forceinline__ void absorb_byte(uint8_t b) {
#pragma unroll
        for (int i = 0; i < RW; i++)
            if (i == (pos >> 3)) s[i] ^= (uint64_t)b << (8 * (pos & 7));
        if (++pos == RATE) {
            keccak_f1600(s);
            pos = 0;
        }
    }
    __device__ __forceinline__ void finalize() {
#pragma unroll
        for (int i = 0; i < RW; i++)
            if (i == (pos >> 3)) s[i] ^= (uint64_t)0x1F << (8 * (pos & 7));
        s[RW - 1] ^= 0x8000000000000000ull;
        pos = RATE;  // squeeze position: forces a permutation before the first output byte
    }
    // Squeeze `len` bytes into any generic address.
    __device__ void squeeze(uint8_t *out, uint32_t len) {
        while (len > 0) {
            if (pos == RATE) {
                keccak_f1600(s);
                pos = 0;
            }
            const int take = min((int)len, RATE - pos);
            const int lo = pos, hi = pos + take;
            if ((pos & 7) == 0 && (reinterpret_cast<uintptr_t>(out) & 7) == 0) {
                // aligned output: whole state words as 8-byte stores, then the last bytes
                uint64_t *o64 = reinterpret_cast<uint64_t *>(out);
#pragma unroll
                for (int i = 0; i < RW; i++) {
                    if (8 * i >= lo && 8 * i + 8 <= hi) {
                        o64[i - (lo >> 3)] = s[i];
                    } else if (8 * i >= lo && 8 * i < hi) {
#pragma unroll
                        for (int b = 0; b < 8; b++)
                            if (8 * i + b < hi) out[8 * i + b - lo] = (uint8_t)(s[i] >> (8 * b));
                    }
                }
            } else {
#pragma unroll
                for (int i = 0; i < RW; i++)
#pragma unroll
                    for (int b = 0; b < 8; b++) {
                        const int bp = 8 * i + b;
                        if (bp >= lo && bp < hi) out[bp - lo] = (uint8_t)(s[i] >> (8 * b));
                    }
            }
            out += take;
            len -= take;
            pos += take;
        }
    }
};

// Warp-cooperative Keccak-f[1600]: lane L < 25 holds lane word A[x + 5y] (x = L % 5, y = L / 5).
// All 32 lanes must call it (lanes 25..31 carry junk and are ignored).
struct WarpKeccak {
    int x, src_c0, src_c1, src_pi, src_chi1, src_chi2, rho;
    __device__ __forceinline__ void setup(int lane) {
        int L = lane < 25 ? lane : 0;
        x = L % 5;
        int y = L / 5;
        src_c0 = (x + 4) % 5;  // D[x] = C[x-1] ^ rot(C[x+1], 1)
        src_c1 = (x + 1) % 5;
        // pi: destination (X, Y) = (y, 2x + 3y) pulls from source lane ((X + 3Y) % 5) + 5X
        src_pi = ((x + 3 * y) % 5) + 5 * x;
        src_chi1 = (x + 1) % 5 + 5 * y;
        src_chi2 = (x + 2) % 5 + 5 * y;
        rho = c_keccak_rho[L];
    }
    __device__ __forceinline__ uint64_t rotl_var(uint64_t a, int r) const {
        return r == 0 ? a : ((a << r) | (a >> (64 - r)));
    }
    __device__ uint64_t permute(uint64_t a, int lane) const {
        const unsigned FULL = 0xffffffffu;
#pragma unroll 1
        for (int round = 0; round < 24; round++) {
            uint64_t c = __shfl_sync(FULL, a, x) ^ __shfl_sync(FULL, a, x + 5) ^ __shfl_sync(FULL, a, x + 10) ^
                         __shfl_sync(FULL, a, x + 15) ^ __shfl_sync(FULL, a, x + 20);
            uint64_t d = __shfl_sync(FULL, c, src_c0) ^ rotl64c<1>(__shfl_sync(FULL, c, src_c1));
            a ^= d;
            uint64_t b = __shfl_sync(FULL, rotl_var(a, rho), src_pi);
            a = b ^ (~__shfl_sync(FULL, b, src_chi1) & __shfl_sync(FULL, b, src_chi2));
            if (lane == 0) a ^= c_keccak_rc[round];
        }
        return a;
    }
};

// SHAKE over a shared-memory input with the warp-cooperative permutation; output to shared.
// in_len/out_len in bytes; `in` and `out` must not overlap.
template <int RATE>
__device__ void warp_shake(uint8_t *out, int out_len, const uint8_t *in, int in_len, const WarpKeccak &wk,
                           int lane) {
    uint64_t a = 0;
    int off = 0;
    for (;;) {
        int blk = min(in_len - off, RATE);
        bool last = (in_len - off) < RATE;
        uint64_t w = 0;
        if (lane < RATE / 8) {
#pragma unroll
            for (int b = 0; b < 8; b++) {
                int pos = lane * 8 + b;
                uint8_t byte = pos < blk ? in[off + pos] : 0;
                if (last && pos == blk) byte ^= 0x1F;
                if (last && pos == RATE - 1) byte ^= 0x80;
                w |= (uint64_t)byte << (8 * b);
            }
        }
        a ^= w;
        if (last) break;
        a = wk.permute(a, lane);
        off += RATE;
    }
    for (int o = 0; o < out_len; o += RATE) {
        a = wk.permute(a, lane);
        __syncwarp();
        if (lane < RATE / 8) {
#pragma unroll
            for (int b = 0; b < 8; b++) {
                int pos = o + lane * 8 + b;
                if (pos < out_len) out[pos] = (uint8_t)(a >> (8 * b));
            }
        }
    }
    __syncwarp();
}

// ---------------------------------------------------------------------------------------------
// Bitsliced GF(16) = GF(2)[x]/(x^4 + x + 1) (the reference's field, src/gf16.cu:10-58).
//
// A group is 32 coordinates of an m-vector held as four bit-planes.  Conversion from the
// packed nibble layout (16 bytes, coordinate 2j = low nibble of byte j) is a 4x4 bit transpose
// at each nibble position of the four little-endian words, so plane bit b holds coordinate
// 8*(b & 3) + (b >> 2) of the group.  The transform is its own inverse.  Every coordinate-wise
// operation is indifferent to this order; the few operations that mix coordinates (z-shifts)
// run on the packed layout.
// ---------------------------------------------------------------------------------------------
struct G4 {
    uint32_t p0, p1, p2, p3;
};

__host__ __device__ __forceinline__ void transpose4(uint32_t &w0, uint32_t &w1, uint32_t &w2, uint32_t &w3) {
    uint32_t t;
    t = ((w0 >> 2) ^ w2) & 0x33333333u;
    w2 ^= t;
    w0 ^= t << 2;
    t = ((w1 >> 2) ^ w3) & 0x33333333u;
    w3 ^= t;
    w1 ^= t << 2;
    t = ((w0 >> 1) ^ w1) & 0x55555555u;
    w1 ^= t;
    w0 ^= t << 1;
    t = ((w2 >> 1) ^ w3) & 0x55555555u;
    w3 ^= t;
    w2 ^= t << 1;
}

__host__ __device__ __forceinline__ G4 g4_from_packed(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3) {
    transpose4(w0, w1, w2, w3);
    return G4{w0, w1, w2, w3};
}
__host__ __device__ __forceinline__ uint4 g4_to_packed(G4 g) {
    transpose4(g.p0, g.p1, g.p2, g.p3);
    return make_uint4(g.p0, g.p1, g.p2, g.p3);
}
__host__ __device__ __forceinline__ G4 g4_xor(G4 a, G4 b) { return G4{a.p0 ^ b.p0, a.p1 ^ b.p1, a.p2 ^ b.p2, a.p3 ^ b.p3}; }
__host__ __device__ __forceinline__ G4 g4_zero() { return G4{0, 0, 0, 0}; }
__host__ __device__ __forceinline__ G4 g4_ld(const uint4 *p) {
    uint4 u = *p;
    return G4{u.x, u.y, u.z, u.w};
}
__host__ __device__ __forceinline__ void g4_st(uint4 *p, G4 g) { *p = make_uint4(g.p0, g.p1, g.p2, g.p3); }

// Scalar s as four all-ones/all-zero masks (bit t of s -> mask t).
__host__ __device__ __forceinline__ uint4 scalar_masks(uint32_t s) {
    return make_uint4(0u - (s & 1), 0u - ((s >> 1) & 1), 0u - ((s >> 2) & 1), 0u - ((s >> 3) & 1));
}

// acc += s * v with s given as masks; constant time (no data-dependent branch or address).
// s*v = sum_t s_t * (x^t v), x*(v0,v1,v2,v3) = (v3, v0^v3, v1, v2).
__host__ __device__ __forceinline__ void g4_madd(G4 &acc, const G4 &v, const uint4 &m) {
    const uint32_t s03 = v.p0 ^ v.p3, s23 = v.p2 ^ v.p3, s12 = v.p1 ^ v.p2;
    acc.p0 = lop_xand(lop_xand(lop_xand(lop_xand(acc.p0, m.x, v.p0), m.y, v.p3), m.z, v.p2), m.w, v.p1);
    acc.p1 = lop_xand(lop_xand(lop_xand(lop_xand(acc.p1, m.x, v.p1), m.y, s03), m.z, s23), m.w, s12);
    acc.p2 = lop_xand(lop_xand(lop_xand(lop_xand(acc.p2, m.x, v.p2), m.y, v.p1), m.z, s03), m.w, s23);
    acc.p3 = lop_xand(lop_xand(lop_xand(lop_xand(acc.p3, m.x, v.p3), m.y, v.p2), m.z, v.p1), m.w, s03);
}

// The same product accumulated as four partial sums, one per power of x: A_t += s_t v (16 LOP3
// and no x-multiples of v per call), folded once into A_0 + x A_1 + x^2 A_2 + x^3 A_3 by
// g4x4_fold.  For a sum of many products this saves the three XORs g4_madd spends per call on
// x v, x^2 v, x^3 v.  Constant time.
struct G4x4 {
    G4 a0, a1, a2, a3;
};
__host__ __device__ __forceinline__ G4x4 g4x4_zero() { return G4x4{g4_zero(), g4_zero(), g4_zero(), g4_zero()}; }
__host__ __device__ __forceinline__ void g4x4_madd(G4x4 &A, const G4 &v, const uint4 &m) {
    A.a0.p0 = lop_xand(A.a0.p0, m.x, v.p0);
    A.a0.p1 = lop_xand(A.a0.p1, m.x, v.p1);
    A.a0.p2 = lop_xand(A.a0.p2, m.x, v.p2);
    A.a0.p3 = lop_xand(A.a0.p3, m.x, v.p3);
    A.a1.p0 = lop_xand(A.a1.p0, m.y, v.p0);
    A.a1.p1 = lop_xand(A.a1.p1, m.y, v.p1);
    A.a1.p2 = lop_xand(A.a1.p2, m.y, v.p2);
    A.a1.p3 = lop_xand(A.a1.p3, m.y, v.p3);
    A.a2.p0 = lop_xand(A.a2.p0, m.z, v.p0);
    A.a2.p1 = lop_xand(A.a2.p1, m.z, v.p1);
    A.a2.p2 = lop_xand(A.a2.p2, m.z, v.p2);
    A.a2.p3 = lop_xand(A.a2.p3, m.z, v.p3);
    A.a3.p0 = lop_xand(A.a3.p0, m.w, v.p0);
    A.a3.p1 = lop_xand(A.a3.p1, m.w, v.p1);
    A.a3.p2 = lop_xand(A.a3.p2, m.w, v.p2);
    A.a3.p3 = lop_xand(A.a3.p3, m.w, v.p3);
}
// x v for a group of coordinates: x (v0, v1, v2, v3) = (v3, v0 + v3, v1, v2) since x^4 = x + 1.
__host__ __device__ __forceinline__ G4 g4_times_x(const G4 &v) { return G4{v.p3, v.p0 ^ v.p3, v.p1, v.p2}; }
__host__ __device__ __forceinline__ G4 g4x4_fold(const G4x4 &A) {
    G4 t = g4_xor(g4_times_x(A.a3), A.a2);
    t = g4_xor(g4_times_x(t), A.a1);
    return g4_xor(g4_times_x(t), A.a0);
}

// Scalar GF(16) product without tables or branches (constant time).
__host__ __device__ __forceinline__ uint32_t gf16_mul_ct(uint32_t a, uint32_t b) {
    uint32_t r = (0u - (b & 1)) & a;
    r ^= (0u - ((b >> 1) & 1)) & (a << 1);
    r ^= (0u - ((b >> 2) & 1)) & (a << 2);
    r ^= (0u - ((b >> 3) & 1)) & (a << 3);
    // reduce degrees 6..4 with x^4 = x + 1
    uint32_t h = r >> 4;  // bits of x^4, x^5, x^6
    r = (r & 0xF) ^ h ^ (h << 1);
    uint32_t h2 = r >> 4;  // x^6 -> x^3 + x^2 may leave one more carry from (h << 1)
    r = (r & 0xF) ^ h2 ^ (h2 << 1);
    return r & 0xF;
}
// Inverse as a^14 (constant time; 0 -> 0).
__host__ __device__ __forceinline__ uint32_t gf16_inv_ct(uint32_t a) {
    uint32_t a2 = gf16_mul_ct(a, a), a4 = gf16_mul_ct(a2, a2), a8 = gf16_mul_ct(a4, a4);
    return gf16_mul_ct(gf16_mul_ct(a2, a4), a8);
}

// Inverses of 0..15 as one 64-bit constant (nibble a = a^-1, 0^-1 := 0).  Read with a shift by
// 4a: no memory access and no branch, so constant time in a.
__host__ __device__ constexpr uint32_t gf16_mul_cx(uint32_t a, uint32_t b) {
    uint32_t r = 0;
    for (int i = 0; i < 4; i++)
        if (b & (1u << i)) r ^= a << i;
    for (int d = 6; d >= 4; d--)
        if (r & (1u << d)) r ^= 0x13u << (d - 4);  // x^4 = x + 1
    return r;
}
__host__ __device__ constexpr uint64_t gf16_inv_table() {
    uint64_t t = 0;
    for (uint32_t a = 1; a < 16; a++)
        for (uint32_t b = 1; b < 16; b++)
            if (gf16_mul_cx(a, b) == 1) t |= (uint64_t)b << (4 * a);
    return t;
}
constexpr uint64_t kGf16InvTable = gf16_inv_table();
__host__ __device__ __forceinline__ uint32_t gf16_inv_reg(uint32_t a) {
    return (uint32_t)(kGf16InvTable >> (4 * (a & 0xF))) & 0xFu;
}
// x * b in GF(16) (x^4 = x + 1), without branches.
__host__ __device__ __forceinline__ uint32_t gf16_xtime(uint32_t b) {
    return ((b << 1) & 0xFu) ^ ((0u - (b >> 3)) & 0x3u);
}
// Quotient e / a from the basis multiples B_s = a^-1 x^s (s = 0..3) and the bits e_s of e:
// e / a = sum_s e_s B_s.  The bits come as words that are zero or not; masks select the B_s, so
// the quotient costs no memory access and no branch on e or a.
__host__ __device__ __forceinline__ uint32_t gf16_div_from_basis(uint32_t e0, uint32_t e1, uint32_t e2, uint32_t e3,
                                                                const uint4 &B) {
    return ((0u - (uint32_t)(e0 != 0u)) & B.x) ^ ((0u - (uint32_t)(e1 != 0u)) & B.y) ^
           ((0u - (uint32_t)(e2 != 0u)) & B.z) ^ ((0u - (uint32_t)(e3 != 0u)) & B.w);
}

// Multiply the eight packed nibbles of a word by a public constant c (0..15).
__host__ __device__ __forceinline__ uint32_t nib8_mul_const(uint32_t w, uint32_t c) {
    uint32_t r = 0, t = w;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (c & (1u << i)) r ^= t;
        uint32_t hi = (t >> 3) & 0x11111111u;
        t = ((t & 0x77777777u) << 1) ^ hi ^ (hi << 1);
    }
    return r;
}

}  // namespace mayo
