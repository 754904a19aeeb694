// aes.cuh -- AES-128 in the counter mode the reference uses for P1||P2 expansion
// (reference src/aes128_ctr.cu:124-283): key = seed_pk, block i encrypts the 16-byte counter
// 0^8 || BE64(i), output bytes in standard AES order, a final partial block keeps its leading
// bytes.
//
// B200 layout: the round table T0 (Te0 of FIPS-197 in big-endian words) replicated 32 times in
// shared memory, entry x of copy c at word 32*x + c, so lane c always hits bank c and the 16
// data-dependent lookups of a round never conflict.  The other three round tables are byte
// rotations of T0.  The expansion kernel keeps T0, ror8(T0) and ror16(T0) (96 KB, two CTAs of 384
// threads per SM) and rotates only for the fourth; the work-queue kernel's keypair keeps T0 (and
// ror16(T0) for MAYO_5) in the area its P3 engine uses next and rotates with PRMT.  The S-box for
// the last round is byte 1 of T0[x].  Tables are computed at compile time from GF(2^8) arithmetic.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace mayo {

struct AesTables {
    uint32_t te0[256];
    uint8_t sbox[256];
};

__host__ __device__ constexpr uint8_t gf256_mulc(uint8_t a, uint8_t b) {
    uint8_t r = 0;
    for (int i = 0; i < 8; i++) {
        if (b & 1) r ^= a;
        uint8_t hi = a & 0x80;
        a = (uint8_t)(a << 1);
        if (hi) a ^= 0x1B;
        b >>= 1;
    }
    return r;
}

__host__ __device__ constexpr AesTables make_aes_tables() {
    AesTables t{};
    // exp/log over the generator 0x03
    uint8_t ex[256] = {}, lg[256] = {};
    uint8_t g = 1;
    for (int i = 0; i < 255; i++) {
        ex[i] = g;
        lg[g] = (uint8_t)i;
        g = gf256_mulc(g, 3);
    }
    for (int x = 0; x < 256; x++) {
        uint8_t inv = x ? ex[(255 - lg[x]) % 255] : 0;
        uint8_t s = inv, r = inv;
        for (int i = 0; i < 4; i++) {
            r = (uint8_t)((r << 1) | (r >> 7));
            s ^= r;
        }
        s ^= 0x63;
        t.sbox[x] = s;
        t.te0[x] = ((uint32_t)gf256_mulc(s, 2) << 24) | ((uint32_t)s << 16) | ((uint32_t)s << 8) |
                   (uint32_t)gf256_mulc(s, 3);
    }
    return t;
}

__constant__ AesTables c_aes = make_aes_tables();

__device__ __forceinline__ uint32_t ror8(uint32_t x) { return __byte_perm(x, x, 0x0321); }
__device__ __forceinline__ uint32_t ror16(uint32_t x) { return __byte_perm(x, x, 0x1032); }
__device__ __forceinline__ uint32_t ror24(uint32_t x) { return __byte_perm(x, x, 0x2103); }
__device__ __forceinline__ uint32_t byte_of(uint32_t x, int b) { return __byte_perm(x, 0, 0x4440 | b); }

// AES-128 key schedule (FIPS-197 5.2) from 16 key bytes at any address; `sb` is the S-box (the
// constant-memory copy by default, a shared-memory copy where threads look up different bytes).
__device__ inline void aes128_key_schedule(const uint8_t *key, uint32_t *rk, const uint8_t *sb = nullptr) {
    if (!sb) sb = c_aes.sbox;
#pragma unroll
    for (int i = 0; i < 4; i++)
        rk[i] = ((uint32_t)key[4 * i] << 24) | ((uint32_t)key[4 * i + 1] << 16) | ((uint32_t)key[4 * i + 2] << 8) |
                key[4 * i + 3];
    uint32_t rcon = 1;
#pragma unroll
    for (int i = 4; i < 44; i++) {
        uint32_t t = rk[i - 1];
        if (i % 4 == 0) {
            t = (t << 8) | (t >> 24);
            t = ((uint32_t)sb[t >> 24] << 24) | ((uint32_t)sb[(t >> 16) & 0xFF] << 16) |
                ((uint32_t)sb[(t >> 8) & 0xFF] << 8) | sb[t & 0xFF];
            t ^= rcon << 24;
            rcon = gf256_mulc((uint8_t)rcon, 2);
        }
        rk[i] = rk[i - 4] ^ t;
    }
}

// The four big-endian state words of an encrypted counter block.
struct AesOut {
    uint32_t w0, w1, w2, w3;
};

// The table stride (128 bytes) as a value the compiler cannot fold, for kernels without a
// launch argument for it: a constant-bank operand keeps the address arithmetic an IMAD.
__constant__ uint32_t c_aes_stride = 128;

// Encrypt counter block `blk` with NTAB replicated round tables in shared memory, 32 KB apart
// from `base` (the shared-memory address of T0 with this lane's column added):
//   NTAB = 3: T0, ror8(T0), ror16(T0)   (the expansion kernel, 96 KB)
//   NTAB = 2: T0, ror16(T0)             (the work queue's keypair where its P3 area holds both)
//   NTAB = 1: T0                        (the work queue's keypair otherwise)
// the other round tables by PRMT rotations.  A lookup is a byte extraction, one IMAD for the
// address (the multiplier `k128` = 128 is a kernel argument or a constant-bank value, so the
// address arithmetic stays on the IMAD pipe instead of joining the extractions, rotations and
// XORs on the logic pipe, which with the table reads sets the pace) and the read.  Measured at
// MAYO_1's 1,024 x 9,031 blocks: one table with PRMT rotations and shifted-index addresses
// 0.250 ms, IMAD addresses 0.234, two tables 0.222, three tables in two CTAs of 384 threads per
// SM 0.203 (byte-exact).
template <int NTAB, class RK>
__device__ __forceinline__ AesOut aes128_ctr_block_t(uint32_t base, const RK &rk, uint32_t blk, uint32_t k128) {
    static_assert(NTAB >= 1 && NTAB <= 3, "one to three tables");
    auto ld = [&](uint32_t x, auto tab) {
        constexpr int T = decltype(tab)::value;
        uint32_t v;
        if constexpr (T == 0)
            asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(x * k128 + base));
        else if constexpr (T == 1)
            asm volatile("ld.shared.u32 %0, [%1+32768];" : "=r"(v) : "r"(x * k128 + base));
        else
            asm volatile("ld.shared.u32 %0, [%1+65536];" : "=r"(v) : "r"(x * k128 + base));
        return v;
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    auto r0 = [&](uint32_t x) { return ld(x, I0{}); };  // T0[x]
    auto r8 = [&](uint32_t x) {                          // ror8(T0[x])
        if constexpr (NTAB == 3) return ld(x, I1{});
        else return ror8(ld(x, I0{}));
    };
    auto r16 = [&](uint32_t x) {  // ror16(T0[x])
        if constexpr (NTAB == 3) return ld(x, I2{});
        else if constexpr (NTAB == 2) return ld(x, I1{});
        else return ror16(ld(x, I0{}));
    };
    auto r24 = [&](uint32_t x) {  // ror24(T0[x])
        if constexpr (NTAB == 1) return ror24(ld(x, I0{}));
        else return ror8(r16(x));
    };
    uint32_t s0 = rk[0], s1 = rk[1], s2 = rk[2], s3 = blk ^ rk[3];
#pragma unroll
    for (int r = 1; r < 10; r++) {
        const uint32_t a = r0(s0 >> 24) ^ r8(byte_of(s1, 2)) ^ r16(byte_of(s2, 1)) ^ r24(byte_of(s3, 0)) ^ rk[4 * r];
        const uint32_t b = r0(s1 >> 24) ^ r8(byte_of(s2, 2)) ^ r16(byte_of(s3, 1)) ^ r24(byte_of(s0, 0)) ^ rk[4 * r + 1];
        const uint32_t c = r0(s2 >> 24) ^ r8(byte_of(s3, 2)) ^ r16(byte_of(s0, 1)) ^ r24(byte_of(s1, 0)) ^ rk[4 * r + 2];
        const uint32_t d = r0(s3 >> 24) ^ r8(byte_of(s0, 2)) ^ r16(byte_of(s1, 1)) ^ r24(byte_of(s2, 0)) ^ rk[4 * r + 3];
        s0 = a;
        s1 = b;
        s2 = c;
        s3 = d;
    }
    // last round: S-box = byte 1 of T0[x]
#define LASTW(a, b, c, d, k)                                                                   \
    (__byte_perm(__byte_perm(r0((a) >> 24), r0(byte_of(b, 2)), 0x1500),                         \
                 __byte_perm(r0(byte_of(c, 1)), r0(byte_of(d, 0)), 0x0015), 0x3254) ^            \
     rk[k])
    AesOut o;
    o.w0 = LASTW(s0, s1, s2, s3, 40);
    o.w1 = LASTW(s1, s2, s3, s0, 41);
    o.w2 = LASTW(s2, s3, s0, s1, 42);
    o.w3 = LASTW(s3, s0, s1, s2, 43);
#undef LASTW
    return o;
}

// Big-endian words -> little-endian words of the byte stream.
__device__ __forceinline__ uint32_t bswap32(uint32_t x) { return __byte_perm(x, 0, 0x0123); }

// Store 16 stream bytes (as 4 LE words) at any address, widest aligned stores possible.
__device__ __forceinline__ void st16(uint8_t *p, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    uintptr_t ad = reinterpret_cast<uintptr_t>(p);
    if ((ad & 15) == 0) {
        *reinterpret_cast<uint4 *>(p) = make_uint4(a, b, c, d);
    } else if ((ad & 7) == 0) {
        reinterpret_cast<uint2 *>(p)[0] = make_uint2(a, b);
        reinterpret_cast<uint2 *>(p)[1] = make_uint2(c, d);
    } else if ((ad & 3) == 0) {
        uint32_t *q = reinterpret_cast<uint32_t *>(p);
        q[0] = a;
        q[1] = b;
        q[2] = c;
        q[3] = d;
    } else {
        const uint32_t w[4] = {a, b, c, d};
#pragma unroll
        for (int i = 0; i < 16; i++) p[i] = (uint8_t)(w[i >> 2] >> (8 * (i & 3)));
    }
}

// ---------------------------------------------------------------------------------------------
// Kernel: AES-CTR keystream into a pitched pool.  grid = (chunks, batch); chunk x of instance
// blockIdx.y takes blocks [x * bpc, min((x + 1) * bpc, nblk_main)) to row + out_off, keyed by 16
// bytes at row + key_off.  The launcher splits an instance's blocks into near-equal chunks of at
// most AES_BLOCKS_PER_CTA.  When the key overlaps the output (expand-pk, expand-sk keep seed_pk
// in the last 16 output bytes until expansion), nblk_main excludes the blocks that overlap the
// key and aes_ctr_tail_kernel finishes them afterwards, one thread per instance.
// ---------------------------------------------------------------------------------------------
constexpr int AES_THREADS = 384;
constexpr int AES_BLOCKS_PER_CTA = 3072;
constexpr size_t AES_SMEM = 3 * 256 * 32 * 4;  // T0, ror8(T0), ror16(T0), each replicated 32 times

static __global__ void __launch_bounds__(AES_THREADS, 2)
    aes_ctr_kernel(uint8_t *pool, size_t pitch, size_t key_off, size_t out_off, uint32_t nblk_main, uint32_t bpc,
                   uint32_t k128) {
    extern __shared__ uint32_t aes_smem[];  // [3][256 * 32] words
    __shared__ uint32_t rk_s[44];
    uint8_t *row = pool + (size_t)blockIdx.y * pitch;
    // warp 0's lane 0 runs the (serial) key schedule while the other warps build the tables
    if (threadIdx.x == 0) aes128_key_schedule(row + key_off, rk_s);
    for (int i = (int)threadIdx.x - 32; i < 256 * 32; i += AES_THREADS - 32) {
        if (i < 0) break;
        const uint32_t v = c_aes.te0[i >> 5];
        aes_smem[i] = v;
        aes_smem[256 * 32 + i] = ror8(v);
        aes_smem[2 * 256 * 32 + i] = ror16(v);
    }
    __syncthreads();
    uint32_t rk[44];
#pragma unroll
    for (int i = 0; i < 44; i++) rk[i] = rk_s[i];
    const uint32_t base = (uint32_t)__cvta_generic_to_shared(aes_smem + (threadIdx.x & 31));
    uint8_t *out = row + out_off;
    const uint32_t b0 = blockIdx.x * bpc;
    const uint32_t b1 = min(b0 + bpc, nblk_main);
    for (uint32_t blk = b0 + threadIdx.x; blk < b1; blk += AES_THREADS) {
        AesOut o = aes128_ctr_block_t<3>(base, rk, blk, k128);
        st16(out + (size_t)blk * 16, bswap32(o.w0), bswap32(o.w1), bswap32(o.w2), bswap32(o.w3));
    }
}

// Blocks [nblk_main, ceil(nbytes/16)) for each instance (key read before any byte is written).
// One thread per instance, at most two blocks each; the threads of a warp look up different
// bytes, so the tables are copied to shared memory first (constant memory would serialise them).
constexpr int AES_TAIL_THREADS = 128;
static __global__ void __launch_bounds__(AES_TAIL_THREADS)
    aes_ctr_tail_kernel(uint8_t *pool, size_t pitch, size_t key_off, size_t out_off, uint32_t nblk_main,
                        uint32_t nbytes, uint32_t batch) {
    __shared__ uint32_t te[256];
    __shared__ uint8_t sb[256];
    for (int i = threadIdx.x; i < 256; i += AES_TAIL_THREADS) {
        te[i] = c_aes.te0[i];
        sb[i] = c_aes.sbox[i];
    }
    __syncthreads();
    const uint32_t inst = blockIdx.x * blockDim.x + threadIdx.x;
    if (inst >= batch) return;
    uint8_t *row = pool + (size_t)inst * pitch;
    uint32_t rk[44];
    aes128_key_schedule(row + key_off, rk, sb);
    const uint32_t nblk = (nbytes + 15) / 16;
    uint8_t buf[32];
    for (uint32_t blk = nblk_main; blk < nblk; blk++) {
        uint32_t s0 = rk[0], s1 = rk[1], s2 = rk[2], s3 = blk ^ rk[3];
        for (int r = 1; r < 10; r++) {
            const uint32_t t0 = te[s0 >> 24] ^ ror8(te[(s1 >> 16) & 255]) ^ ror16(te[(s2 >> 8) & 255]) ^
                                ror24(te[s3 & 255]) ^ rk[4 * r];
            const uint32_t t1 = te[s1 >> 24] ^ ror8(te[(s2 >> 16) & 255]) ^ ror16(te[(s3 >> 8) & 255]) ^
                                ror24(te[s0 & 255]) ^ rk[4 * r + 1];
            const uint32_t t2 = te[s2 >> 24] ^ ror8(te[(s3 >> 16) & 255]) ^ ror16(te[(s0 >> 8) & 255]) ^
                                ror24(te[s1 & 255]) ^ rk[4 * r + 2];
            const uint32_t t3 = te[s3 >> 24] ^ ror8(te[(s0 >> 16) & 255]) ^ ror16(te[(s1 >> 8) & 255]) ^
                                ror24(te[s2 & 255]) ^ rk[4 * r + 3];
            s0 = t0;
            s1 = t1;
            s2 = t2;
            s3 = t3;
        }
        uint32_t o[4];
        o[0] = ((uint32_t)sb[s0 >> 24] << 24 | (uint32_t)sb[(s1 >> 16) & 255] << 16 | (uint32_t)sb[(s2 >> 8) & 255] << 8 |
                sb[s3 & 255]) ^ rk[40];
        o[1] = ((uint32_t)sb[s1 >> 24] << 24 | (uint32_t)sb[(s2 >> 16) & 255] << 16 | (uint32_t)sb[(s3 >> 8) & 255] << 8 |
                sb[s0 & 255]) ^ rk[41];
        o[2] = ((uint32_t)sb[s2 >> 24] << 24 | (uint32_t)sb[(s3 >> 16) & 255] << 16 | (uint32_t)sb[(s0 >> 8) & 255] << 8 |
                sb[s1 & 255]) ^ rk[42];
        o[3] = ((uint32_t)sb[s3 >> 24] << 24 | (uint32_t)sb[(s0 >> 16) & 255] << 16 | (uint32_t)sb[(s1 >> 8) & 255] << 8 |
                sb[s2 & 255]) ^ rk[43];
        for (int i = 0; i < 16; i++) buf[(blk - nblk_main) * 16 + i] = (uint8_t)(o[i >> 2] >> (24 - 8 * (i & 3)));
    }
    // write only after every tail block is computed (the key may sit in these bytes)
    uint8_t *out = row + out_off + (size_t)nblk_main * 16;
    const uint32_t nb = nbytes - nblk_main * 16;
    for (uint32_t i = 0; i < nb; i++) out[i] = buf[i];
}

}  // namespace mayo
