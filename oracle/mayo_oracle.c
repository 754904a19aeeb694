/*
 * mayo_oracle.c -- CPU restatement of SysuCrypto/cuMAYO (see mayo_oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker and the CPU baseline.  The
 * product (cumayo_b200/) never links or calls this file.
 *
 * Citations are file:line within the reference project.
 */
#include "mayo_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Parameter sets: include/params.h:10-92                                    */
/* ------------------------------------------------------------------------ */
#define MK(ID, N, M, O, K, SK, PK, P, OB, P1, P2, DIG, PAIR, C0, C1, C2, C3)                 \
    {ID, N, M, O, K, (N) - (O), (M) / 2, SK, PK, P, OB, P1, P2, DIG, PAIR, {C0, C1, C2, C3}, \
     (K) * (N) / 2 + (SK), (SK) + (OB) + (P), (P) + (PK)-16}

static const mayo_oracle_params PARAMS[4] = {
    MK(1, 86, 78, 8, 10, 24, 1420, 144495, 312, 120159, 24336, 32, 55, 0x8, 0x1, 0x1, 0x0),
    MK(2, 81, 64, 17, 4, 24, 4912, 101376, 544, 66560, 34816, 32, 10, 0x8, 0x0, 0x2, 0x8),
    MK(3, 118, 108, 10, 11, 32, 2986, 376164, 540, 317844, 58320, 48, 66, 0x8, 0x0, 0x1, 0x7),
    MK(5, 154, 142, 12, 12, 40, 5554, 841847, 852, 720863, 120984, 64, 78, 0x4, 0x0, 0x8, 0x1),
};

const mayo_oracle_params *mayo_oracle_get_params(int set_id) {
    for (int i = 0; i < 4; i++)
        if (PARAMS[i].id == set_id) return &PARAMS[i];
    return NULL;
}

/* ------------------------------------------------------------------------ */
/* Keccak-f[1600] and SHAKE (FIPS 202).  The reference's warp-cooperative    */
/* version is src/fips202.cu:49-158; it computes the standard permutation    */
/* and standard SHAKE padding (domain byte 0x1F, final bit 0x80 at rate-1,   */
/* src/fips202.cu:124-130).  Constants are derived here from the FIPS 202    */
/* definitions (rho offsets by the (x,y) walk, iota by the rc LFSR).          */
/* ------------------------------------------------------------------------ */
static uint64_t keccak_rc[24];
static unsigned keccak_rho[25];
static int keccak_ready = 0;

static int rc_bit(int t) {
    /* FIPS 202 Algorithm 5.  Bit i of `r` holds R[i]; R starts as 10000000. */
    if (t % 255 == 0) return 1;
    unsigned r = 1;
    for (int i = 1; i <= t % 255; i++) {
        r <<= 1;                 /* R = 0 || R (9 bits) */
        if (r & 0x100) r ^= 0x171; /* R[0],R[4],R[5],R[6] ^= R[8]; drop R[8] */
        r &= 0xFF;
    }
    return (int)(r & 1);
}

static void keccak_init_tables(void) {
    if (keccak_ready) return;
    /* rho offsets */
    memset(keccak_rho, 0, sizeof(keccak_rho));
    int x = 1, y = 0;
    for (int t = 0; t < 24; t++) {
        keccak_rho[x + 5 * y] = (unsigned)(((t + 1) * (t + 2) / 2) % 64);
        int nx = y, ny = (2 * x + 3 * y) % 5;
        x = nx;
        y = ny;
    }
    /* iota constants */
    for (int ir = 0; ir < 24; ir++) {
        uint64_t rc = 0;
        for (int j = 0; j <= 6; j++)
            if (rc_bit(j + 7 * ir)) rc |= (uint64_t)1 << ((1u << j) - 1);
        keccak_rc[ir] = rc;
    }
    keccak_ready = 1;
}

static inline uint64_t rotl64(uint64_t a, unsigned r) { return r ? (a << r) | (a >> (64 - r)) : a; }

static void keccak_f1600(uint64_t A[25]) {
    for (int ir = 0; ir < 24; ir++) {
        uint64_t C[5], D[5], B[25];
        for (int x = 0; x < 5; x++) C[x] = A[x] ^ A[x + 5] ^ A[x + 10] ^ A[x + 15] ^ A[x + 20];
        for (int x = 0; x < 5; x++) D[x] = C[(x + 4) % 5] ^ rotl64(C[(x + 1) % 5], 1);
        for (int i = 0; i < 25; i++) A[i] ^= D[i % 5];
        /* rho and pi: B[y, 2x+3y] = rot(A[x,y], r[x,y]) */
        for (int x = 0; x < 5; x++)
            for (int y = 0; y < 5; y++)
                B[y + 5 * ((2 * x + 3 * y) % 5)] = rotl64(A[x + 5 * y], keccak_rho[x + 5 * y]);
        /* chi */
        for (int y = 0; y < 5; y++)
            for (int x = 0; x < 5; x++)
                A[x + 5 * y] = B[x + 5 * y] ^ ((~B[(x + 1) % 5 + 5 * y]) & B[(x + 2) % 5 + 5 * y]);
        A[0] ^= keccak_rc[ir];
    }
}

static void shake(unsigned rate, uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) {
    keccak_init_tables();
    uint64_t A[25];
    memset(A, 0, sizeof(A));
    uint8_t block[200];
    while (inlen >= rate) {
        for (unsigned i = 0; i < rate / 8; i++) {
            uint64_t w = 0;
            for (int b = 0; b < 8; b++) w |= (uint64_t)in[8 * i + b] << (8 * b);
            A[i] ^= w;
        }
        keccak_f1600(A);
        in += rate;
        inlen -= rate;
    }
    memset(block, 0, sizeof(block));
    memcpy(block, in, inlen);
    block[inlen] ^= 0x1F;
    block[rate - 1] ^= 0x80;
    for (unsigned i = 0; i < rate / 8; i++) {
        uint64_t w = 0;
        for (int b = 0; b < 8; b++) w |= (uint64_t)block[8 * i + b] << (8 * b);
        A[i] ^= w;
    }
    while (outlen > 0) {
        keccak_f1600(A);
        size_t take = outlen < rate ? outlen : rate;
        for (size_t i = 0; i < take; i++) out[i] = (uint8_t)(A[i / 8] >> (8 * (i % 8)));
        out += take;
        outlen -= take;
    }
}

void mayo_oracle_shake128(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) {
    shake(168, out, outlen, in, inlen);
}
void mayo_oracle_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) {
    shake(136, out, outlen, in, inlen);
}

/* ------------------------------------------------------------------------ */
/* AES-128 (FIPS 197), counter mode as the reference uses it:                */
/* src/aes128_ctr.cu:124-283 -- one 16-byte block per counter value blk,     */
/* counter block = 0x00 x 8 || BE64(blk), blk = 0,1,2,..; output stored big- */
/* endian word by word, i.e. the standard AES output byte order.  The last   */
/* partial block keeps its leading bytes (src/aes128_ctr.cu:114-122).        */
/* Tables are computed from the field definition, not copied.                */
/* ------------------------------------------------------------------------ */
static uint8_t aes_sbox[256];
static uint32_t aes_te[4][256];
static int aes_ready = 0;

static uint8_t gf256_mul(uint8_t a, uint8_t b) {
    uint8_t r = 0;
    while (b) {
        if (b & 1) r ^= a;
        a = (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1B : 0));
        b >>= 1;
    }
    return r;
}

static void aes_init_tables(void) {
    if (aes_ready) return;
    for (int x = 0; x < 256; x++) {
        uint8_t inv = 0;
        if (x) {
            for (int y = 1; y < 256; y++)
                if (gf256_mul((uint8_t)x, (uint8_t)y) == 1) {
                    inv = (uint8_t)y;
                    break;
                }
        }
        uint8_t s = inv;
        uint8_t r = inv;
        for (int i = 0; i < 4; i++) {
            r = (uint8_t)((r << 1) | (r >> 7));
            s ^= r;
        }
        aes_sbox[x] = (uint8_t)(s ^ 0x63);
    }
    for (int x = 0; x < 256; x++) {
        uint8_t s = aes_sbox[x];
        uint32_t w = ((uint32_t)gf256_mul(s, 2) << 24) | ((uint32_t)s << 16) | ((uint32_t)s << 8) |
                     (uint32_t)gf256_mul(s, 3);
        for (int t = 0; t < 4; t++) {
            aes_te[t][x] = w;
            w = (w >> 8) | (w << 24);
        }
    }
    aes_ready = 1;
}

static void aes128_key_schedule(const uint8_t key[16], uint32_t rk[44]) {
    for (int i = 0; i < 4; i++)
        rk[i] = ((uint32_t)key[4 * i] << 24) | ((uint32_t)key[4 * i + 1] << 16) |
                ((uint32_t)key[4 * i + 2] << 8) | key[4 * i + 3];
    uint8_t rcon = 1;
    for (int i = 4; i < 44; i++) {
        uint32_t t = rk[i - 1];
        if (i % 4 == 0) {
            t = (t << 8) | (t >> 24);
            t = ((uint32_t)aes_sbox[t >> 24] << 24) | ((uint32_t)aes_sbox[(t >> 16) & 0xFF] << 16) |
                ((uint32_t)aes_sbox[(t >> 8) & 0xFF] << 8) | aes_sbox[t & 0xFF];
            t ^= (uint32_t)rcon << 24;
            rcon = gf256_mul(rcon, 2);
        }
        rk[i] = rk[i - 4] ^ t;
    }
}

static void aes128_encrypt_words(const uint32_t rk[44], uint32_t s[4]) {
    uint32_t s0 = s[0] ^ rk[0], s1 = s[1] ^ rk[1], s2 = s[2] ^ rk[2], s3 = s[3] ^ rk[3];
    for (int r = 1; r < 10; r++) {
        uint32_t t0 = aes_te[0][s0 >> 24] ^ aes_te[1][(s1 >> 16) & 0xFF] ^ aes_te[2][(s2 >> 8) & 0xFF] ^
                      aes_te[3][s3 & 0xFF] ^ rk[4 * r];
        uint32_t t1 = aes_te[0][s1 >> 24] ^ aes_te[1][(s2 >> 16) & 0xFF] ^ aes_te[2][(s3 >> 8) & 0xFF] ^
                      aes_te[3][s0 & 0xFF] ^ rk[4 * r + 1];
        uint32_t t2 = aes_te[0][s2 >> 24] ^ aes_te[1][(s3 >> 16) & 0xFF] ^ aes_te[2][(s0 >> 8) & 0xFF] ^
                      aes_te[3][s1 & 0xFF] ^ rk[4 * r + 2];
        uint32_t t3 = aes_te[0][s3 >> 24] ^ aes_te[1][(s0 >> 16) & 0xFF] ^ aes_te[2][(s1 >> 8) & 0xFF] ^
                      aes_te[3][s2 & 0xFF] ^ rk[4 * r + 3];
        s0 = t0;
        s1 = t1;
        s2 = t2;
        s3 = t3;
    }
#define SB(x) ((uint32_t)aes_sbox[(x)&0xFF])
    s[0] = (SB(s0 >> 24) << 24 | SB(s1 >> 16) << 16 | SB(s2 >> 8) << 8 | SB(s3)) ^ rk[40];
    s[1] = (SB(s1 >> 24) << 24 | SB(s2 >> 16) << 16 | SB(s3 >> 8) << 8 | SB(s0)) ^ rk[41];
    s[2] = (SB(s2 >> 24) << 24 | SB(s3 >> 16) << 16 | SB(s0 >> 8) << 8 | SB(s1)) ^ rk[42];
    s[3] = (SB(s3 >> 24) << 24 | SB(s0 >> 16) << 16 | SB(s1 >> 8) << 8 | SB(s2)) ^ rk[43];
#undef SB
}

void mayo_oracle_aes128_ctr(const uint8_t key[16], uint8_t *out, size_t outlen) {
    aes_init_tables();
    uint32_t rk[44];
    aes128_key_schedule(key, rk);
    uint64_t blk = 0;
    while (outlen > 0) {
        uint32_t s[4] = {0, 0, (uint32_t)(blk >> 32), (uint32_t)blk};
        aes128_encrypt_words(rk, s);
        uint8_t b[16];
        for (int i = 0; i < 16; i++) b[i] = (uint8_t)(s[i / 4] >> (24 - 8 * (i % 4)));
        size_t take = outlen < 16 ? outlen : 16;
        memcpy(out, b, take);
        out += take;
        outlen -= take;
        blk++;
    }
}

/* ------------------------------------------------------------------------ */
/* GF(16) = GF(2)[x]/(x^4 + x + 1): src/gf16.cu:10-58 (product table) and    */
/* src/gf16.cu:3-8 (inverse table) describe this field.                      */
/* ------------------------------------------------------------------------ */
uint8_t mayo_oracle_gf16_mul(uint8_t a, uint8_t b) {
    a &= 0xF;
    b &= 0xF;
    unsigned r = 0;
    for (int i = 0; i < 4; i++)
        if (b & (1 << i)) r ^= (unsigned)a << i;
    for (int d = 6; d >= 4; d--)
        if (r & (1u << d)) r ^= 0x13u << (d - 4);
    return (uint8_t)r;
}

uint8_t mayo_oracle_gf16_inv(uint8_t a) {
    a &= 0xF;
    if (!a) return 0;
    for (uint8_t b = 1; b < 16; b++)
        if (mayo_oracle_gf16_mul(a, b) == 1) return b;
    return 0;
}

static uint8_t MUL[16][16];
static int mul_ready = 0;
static void mul_init(void) {
    if (mul_ready) return;
    for (int a = 0; a < 16; a++)
        for (int b = 0; b < 16; b++) MUL[a][b] = mayo_oracle_gf16_mul((uint8_t)a, (uint8_t)b);
    mul_ready = 1;
}

/* Multiply both nibbles of byte x by scalar s: include/gf16.cuh:30-40. */
static inline uint8_t mul2(uint8_t x, uint8_t s) {
    return (uint8_t)((MUL[x >> 4][s & 0xF] << 4) | MUL[x & 0xF][s & 0xF]);
}

/* ---------------- SHA-256 (for table digests only) ---------------------- */
static void sha256(const uint8_t *msg, size_t len, uint8_t out[32]) {
    static const uint32_t K0[64] = {
        0x428a2f98, 0x71374491, 0xb5c0fbcf, 0xe9b5dba5, 0x3956c25b, 0x59f111f1, 0x923f82a4, 0xab1c5ed5,
        0xd807aa98, 0x12835b01, 0x243185be, 0x550c7dc3, 0x72be5d74, 0x80deb1fe, 0x9bdc06a7, 0xc19bf174,
        0xe49b69c1, 0xefbe4786, 0x0fc19dc6, 0x240ca1cc, 0x2de92c6f, 0x4a7484aa, 0x5cb0a9dc, 0x76f988da,
        0x983e5152, 0xa831c66d, 0xb00327c8, 0xbf597fc7, 0xc6e00bf3, 0xd5a79147, 0x06ca6351, 0x14292967,
        0x27b70a85, 0x2e1b2138, 0x4d2c6dfc, 0x53380d13, 0x650a7354, 0x766a0abb, 0x81c2c92e, 0x92722c85,
        0xa2bfe8a1, 0xa81a664b, 0xc24b8b70, 0xc76c51a3, 0xd192e819, 0xd6990624, 0xf40e3585, 0x106aa070,
        0x19a4c116, 0x1e376c08, 0x2748774c, 0x34b0bcb5, 0x391c0cb3, 0x4ed8aa4a, 0x5b9cca4f, 0x682e6ff3,
        0x748f82ee, 0x78a5636f, 0x84c87814, 0x8cc70208, 0x90befffa, 0xa4506ceb, 0xbef9a3f7, 0xc67178f2};
    uint32_t h[8] = {0x6a09e667, 0xbb67ae85, 0x3c6ef372, 0xa54ff53a,
                     0x510e527f, 0x9b05688c, 0x1f83d9ab, 0x5be0cd19};
    size_t total = ((len + 9 + 63) / 64) * 64;
    uint8_t *buf = (uint8_t *)calloc(total, 1);
    memcpy(buf, msg, len);
    buf[len] = 0x80;
    uint64_t bits = (uint64_t)len * 8;
    for (int i = 0; i < 8; i++) buf[total - 1 - i] = (uint8_t)(bits >> (8 * i));
#define ROR(x, n) (((x) >> (n)) | ((x) << (32 - (n))))
    for (size_t off = 0; off < total; off += 64) {
        uint32_t w[64];
        for (int i = 0; i < 16; i++)
            w[i] = (uint32_t)buf[off + 4 * i] << 24 | (uint32_t)buf[off + 4 * i + 1] << 16 |
                   (uint32_t)buf[off + 4 * i + 2] << 8 | buf[off + 4 * i + 3];
        for (int i = 16; i < 64; i++) {
            uint32_t s0 = ROR(w[i - 15], 7) ^ ROR(w[i - 15], 18) ^ (w[i - 15] >> 3);
            uint32_t s1 = ROR(w[i - 2], 17) ^ ROR(w[i - 2], 19) ^ (w[i - 2] >> 10);
            w[i] = w[i - 16] + s0 + w[i - 7] + s1;
        }
        uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
        for (int i = 0; i < 64; i++) {
            uint32_t S1 = ROR(e, 6) ^ ROR(e, 11) ^ ROR(e, 25);
            uint32_t ch = (e & f) ^ (~e & g);
            uint32_t t1 = hh + S1 + ch + K0[i] + w[i];
            uint32_t S0 = ROR(a, 2) ^ ROR(a, 13) ^ ROR(a, 22);
            uint32_t mj = (a & b) ^ (a & c) ^ (b & c);
            uint32_t t2 = S0 + mj;
            hh = g;
            g = f;
            f = e;
            e = d + t1;
            d = c;
            c = b;
            b = a;
            a = t1 + t2;
        }
        h[0] += a; h[1] += b; h[2] += c; h[3] += d;
        h[4] += e; h[5] += f; h[6] += g; h[7] += hh;
    }
#undef ROR
    free(buf);
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 4; j++) out[4 * i + j] = (uint8_t)(h[i] >> (24 - 8 * j));
}

void mayo_oracle_table_digest(uint8_t sbox_sha[32], uint8_t gf16_sha[32]) {
    aes_init_tables();
    mul_init();
    sha256(aes_sbox, 256, sbox_sha);
    uint8_t t[256];
    for (int a = 0; a < 16; a++)
        for (int b = 0; b < 16; b++) t[16 * a + b] = MUL[a][b];
    sha256(t, 256, gf16_sha);
}

/* ------------------------------------------------------------------------ */
/* Index maps: include/code.h:6-38                                           */
/*   nibble k of a packed stream = low nibble of byte k/2 if k even, high    */
/*   nibble otherwise (GET_matrix, code.h:6-11);                              */
/*   upper-triangular dim x dim m-vector (r <= c) at entry                   */
/*   c - r + dim*r - r(r-1)/2 (idx_mattri, code.h:14-20);                    */
/*   rectangular rows x cols m-vector at entry cols*r + c (idx_mat).         */
/* ------------------------------------------------------------------------ */
static inline uint8_t nib(const uint8_t *p, int k) { return (uint8_t)((p[k >> 1] >> ((k & 1) * 4)) & 0xF); }
static inline void set_nib(uint8_t *p, int k, uint8_t v) {
    int sh = (k & 1) * 4;
    p[k >> 1] = (uint8_t)((p[k >> 1] & ~(0xF << sh)) | ((v & 0xF) << sh));
}
static inline int tri(int r, int c, int dim) { return c - r + dim * r - (r * (r - 1)) / 2; }

/* ------------------------------------------------------------------------ */
/* Keypair: src/keypair.cu:32-120                                            */
/* ------------------------------------------------------------------------ */
static void p3_from(const mayo_oracle_params *P, const uint8_t *Obytes, const uint8_t *P1,
                    const uint8_t *P2, uint8_t *P3) {
    /* keypair.cu:55-120: per byte i of the m-vectors, B = P1*O + P2 row by
     * row, then acc[a<=b] ^= O[r][a]*B[b] (+ O[r][b]*B[a] for a != b). */
    const int m = P->m, o = P->o, menc = P->menc;
    const int OT = o * (o + 1) / 2;
    uint8_t *acc = (uint8_t *)malloc((size_t)OT);
    uint8_t *B = (uint8_t *)malloc((size_t)o);
    for (int i = 0; i < menc; i++) {
        memset(acc, 0, (size_t)OT);
        for (int r = 0; r < m; r++) {
            memset(B, 0, (size_t)o);
            for (int k = r; k < m; k++) {
                uint8_t p = P1[(size_t)tri(r, k, m) * menc + i];
                for (int b = 0; b < o; b++) B[b] ^= mul2(p, nib(Obytes, k * o + b));
            }
            for (int b = 0; b < o; b++) B[b] ^= P2[(size_t)(r * o + b) * menc + i];
            for (int a = 0; a < o; a++) {
                uint8_t oa = nib(Obytes, r * o + a);
                for (int b = a; b < o; b++) {
                    uint8_t t = mul2(B[b], oa);
                    if (a != b) t ^= mul2(B[a], nib(Obytes, r * o + b));
                    acc[tri(a, b, o)] ^= t;
                }
            }
        }
        for (int a = 0; a < o; a++)
            for (int b = a; b < o; b++) P3[(size_t)tri(a, b, o) * menc + i] = acc[tri(a, b, o)];
    }
    free(acc);
    free(B);
}

int mayo_oracle_keypair_from_seed(int set_id, const uint8_t *seed_sk, uint8_t *pk) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return -1;
    mul_init();
    size_t slen = 16 + (size_t)P->o_bytes;
    uint8_t *S = (uint8_t *)malloc(slen);
    mayo_oracle_shake256(S, slen, seed_sk, (size_t)P->sk_bytes);          /* keypair.cu:47 */
    uint8_t *Pm = (uint8_t *)malloc((size_t)P->p_bytes);
    mayo_oracle_aes128_ctr(S, Pm, (size_t)P->p_bytes);                    /* keypair.cu:52 */
    memcpy(pk, S, 16);                                                    /* keypair.cu:49-50 */
    p3_from(P, S + 16, Pm, Pm + P->p1_bytes, pk + 16);
    free(S);
    free(Pm);
    return 0;
}

int mayo_oracle_keypair(int set_id, uint64_t rand_index, uint64_t index, uint8_t *sk, uint8_t *pk) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return -1;
    /* keypair.cu:35-40: counter rand_index + 2*blockIdx + 1, 8 bytes LE, SHAKE128 */
    uint64_t ctr = rand_index + (uint64_t)(uint32_t)(2u * (uint32_t)index) + 1;
    uint8_t cb[8];
    for (int i = 0; i < 8; i++) cb[i] = (uint8_t)(ctr >> (8 * i));
    mayo_oracle_shake128(sk, (size_t)P->sk_bytes, cb, 8);
    return mayo_oracle_keypair_from_seed(set_id, sk, pk);
}

/* ------------------------------------------------------------------------ */
/* Expand-sk: src/expandsk.cu:28-80; layout src/api.cu:47-54                 */
/* ------------------------------------------------------------------------ */
int mayo_oracle_expandsk(int set_id, const uint8_t *csk, uint8_t *esk) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return -1;
    mul_init();
    const int m = P->m, o = P->o, menc = P->menc;
    size_t slen = 16 + (size_t)P->o_bytes;
    uint8_t *S = (uint8_t *)malloc(slen);
    mayo_oracle_shake256(S, slen, csk, (size_t)P->sk_bytes);
    uint8_t *dsk = esk, *dO = esk + P->sk_bytes, *dP1 = dO + P->o_bytes, *dP2 = dP1 + P->p1_bytes;
    memmove(dsk, csk, (size_t)P->sk_bytes);
    memcpy(dO, S + 16, (size_t)P->o_bytes);
    mayo_oracle_aes128_ctr(S, dP1, (size_t)P->p_bytes);
    const uint8_t *Ob = S + 16;
    uint8_t *tmp = (uint8_t *)malloc((size_t)o);
    for (int i = 0; i < menc; i++) {
        for (int r = 0; r < m; r++) {
            memset(tmp, 0, (size_t)o);
            for (int k = r + 1; k < m; k++) {
                uint8_t p = dP1[(size_t)tri(r, k, m) * menc + i];
                for (int b = 0; b < o; b++) tmp[b] ^= mul2(p, nib(Ob, k * o + b));
            }
            for (int k = 0; k < r; k++) {
                uint8_t p = dP1[(size_t)tri(k, r, m) * menc + i];
                for (int b = 0; b < o; b++) tmp[b] ^= mul2(p, nib(Ob, k * o + b));
            }
            for (int b = 0; b < o; b++) dP2[(size_t)(r * o + b) * menc + i] ^= tmp[b];
        }
    }
    free(tmp);
    free(S);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Expand-pk: src/expandpk.cu:9-23 with the src/api.cu:64-77 layout: AES      */
/* writes P1||P2 over [0, P), cpk's P3 follows at P.                         */
/* ------------------------------------------------------------------------ */
int mayo_oracle_expandpk(int set_id, const uint8_t *cpk, uint8_t *epk) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return -1;
    uint8_t seed[16];
    memcpy(seed, cpk, 16);
    memmove(epk + P->p_bytes, cpk + 16, (size_t)P->pk_bytes - 16);
    mayo_oracle_aes128_ctr(seed, epk, (size_t)P->p_bytes);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* z * y mod f(z) on a packed m-vector: include/poly.cuh:11-69               */
/* ------------------------------------------------------------------------ */
static void times_z(const mayo_oracle_params *P, uint8_t *y) {
    const int m = P->m;
    uint8_t top = nib(y, m - 1);
    for (int c = m - 1; c >= 1; c--) set_nib(y, c, nib(y, c - 1));
    set_nib(y, 0, 0);
    for (int n = 0; n < 4; n++) set_nib(y, n, (uint8_t)(nib(y, n) ^ MUL[top][P->poly_c[n]]));
}

/* ------------------------------------------------------------------------ */
/* U_ij = s_i^T P s_j + s_j^T P s_i (i < j), s_i^T P s_i (i == j), for a      */
/* block upper-triangular P = [[P1, P2], [0, P3]] and y = Horner over the    */
/* pairs (i = k-1..0, j = i..k-1) of y <- z*y + U_ij.                         */
/* sign: src/sign.cu:396-460 (P1 only); verify: src/verify.cu:72-200.         */
/* s: k vectors of `len` nibbles (s_i at nibble offset i*stride).             */
/* ------------------------------------------------------------------------ */
static void eval_public_map(const mayo_oracle_params *P, const uint8_t *P1, const uint8_t *P2,
                            const uint8_t *P3, const uint8_t *s, int stride, int kk, uint8_t *y) {
    const int m = P->m, o = P->o, menc = P->menc, v = P->v;
    const int npairs = kk * (kk + 1) / 2;
    uint8_t *U = (uint8_t *)calloc((size_t)npairs * menc, 1);
    uint8_t *T = (uint8_t *)malloc((size_t)kk);
#define PID(i, j) ((i) * kk - ((i) * ((i)-1)) / 2 + ((j) - (i)))
#define SV(i, c) nib(s, (i) * stride + (c))
    for (int l = 0; l < menc; l++) {
        /* P1 block: rows r < v, columns c in [r, v) with s_i[c] */
        for (int r = 0; r < v; r++) {
            memset(T, 0, (size_t)kk);
            for (int c = r; c < v; c++) {
                uint8_t p = P1[(size_t)tri(r, c, m) * menc + l];
                for (int i = 0; i < kk; i++) T[i] ^= mul2(p, SV(i, c));
            }
            for (int i = 0; i < kk; i++)
                for (int j = i; j < kk; j++) {
                    uint8_t t = mul2(T[j], SV(i, r));
                    if (i != j) t ^= mul2(T[i], SV(j, r));
                    U[(size_t)PID(i, j) * menc + l] ^= t;
                }
        }
        if (P2) {
            for (int r = 0; r < v; r++) {
                memset(T, 0, (size_t)kk);
                for (int c = 0; c < o; c++) {
                    uint8_t p = P2[(size_t)(r * o + c) * menc + l];
                    for (int i = 0; i < kk; i++) T[i] ^= mul2(p, SV(i, v + c));
                }
                for (int i = 0; i < kk; i++)
                    for (int j = i; j < kk; j++) {
                        uint8_t t = mul2(T[j], SV(i, r));
                        if (i != j) t ^= mul2(T[i], SV(j, r));
                        U[(size_t)PID(i, j) * menc + l] ^= t;
                    }
            }
        }
        if (P3) {
            for (int r = 0; r < o; r++) {
                memset(T, 0, (size_t)kk);
                for (int c = r; c < o; c++) {
                    uint8_t p = P3[(size_t)tri(r, c, o) * menc + l];
                    for (int i = 0; i < kk; i++) T[i] ^= mul2(p, SV(i, v + c));
                }
                for (int i = 0; i < kk; i++)
                    for (int j = i; j < kk; j++) {
                        uint8_t t = mul2(T[j], SV(i, v + r));
                        if (i != j) t ^= mul2(T[i], SV(j, v + r));
                        U[(size_t)PID(i, j) * menc + l] ^= t;
                    }
            }
        }
    }
    memset(y, 0, (size_t)menc);
    for (int i = kk - 1; i >= 0; i--)
        for (int j = i; j < kk; j++) {
            times_z(P, y);
            for (int l = 0; l < menc; l++) y[l] ^= U[(size_t)PID(i, j) * menc + l];
        }
#undef PID
#undef SV
    free(U);
    free(T);
}

/* ------------------------------------------------------------------------ */
/* sample_solution: src/sign.cu:10-145, restated step by step (pivot search  */
/* from the current pivot row, swap, normalise, eliminate below; reject when */
/* the last row is zero; back-substitution bottom-up).                       */
/* A: m x ko nibbles (one per byte here), y: m nibbles, r/x: ko nibbles.     */
/* ------------------------------------------------------------------------ */
static int sample_solution(int m, int ko, uint8_t *A, uint8_t *y, const uint8_t *rv, uint8_t *x) {
    for (int c = 0; c < ko; c++) x[c] = rv[c];
    for (int r = 0; r < m; r++) {
        uint8_t acc = 0;
        for (int c = 0; c < ko; c++) acc ^= MUL[A[r * ko + c]][rv[c]];
        y[r] ^= acc;
    }
    int piv_row = 0;
    for (int piv_col = 0; piv_col < ko && piv_row < m; piv_col++) {
        int p = -1;
        for (int rr = piv_row; rr < m; rr++)
            if (A[rr * ko + piv_col]) {
                p = rr;
                break;
            }
        if (p < 0) continue;
        if (p != piv_row) {
            uint8_t t = y[piv_row];
            y[piv_row] = y[p];
            y[p] = t;
            for (int c = 0; c < ko; c++) {
                uint8_t u = A[piv_row * ko + c];
                A[piv_row * ko + c] = A[p * ko + c];
                A[p * ko + c] = u;
            }
        }
        uint8_t inv = mayo_oracle_gf16_inv(A[piv_row * ko + piv_col]);
        y[piv_row] = MUL[y[piv_row]][inv];
        for (int c = 0; c < ko; c++) A[piv_row * ko + c] = MUL[A[piv_row * ko + c]][inv];
        for (int rr = piv_row + 1; rr < m; rr++) {
            uint8_t f = A[rr * ko + piv_col];
            if (!f) continue;
            y[rr] ^= MUL[y[piv_row]][f];
            for (int c = 0; c < ko; c++) A[rr * ko + c] ^= MUL[A[piv_row * ko + c]][f];
        }
        piv_row++;
    }
    int last_zero = 1;
    for (int c = 0; c < ko; c++)
        if (A[(m - 1) * ko + c]) {
            last_zero = 0;
            break;
        }
    if (last_zero) return 0;
    for (int rr = m - 1; rr >= 0; rr--) {
        int c = -1;
        for (int cc = 0; cc < ko; cc++)
            if (A[rr * ko + cc]) {
                c = cc;
                break;
            }
        if (c < 0) continue;
        uint8_t alpha = y[rr];
        if (alpha) {
            x[c] ^= alpha;
            for (int r = 0; r < m; r++) y[r] ^= MUL[alpha][A[r * ko + c]];
        }
    }
    return 1;
}

/* ------------------------------------------------------------------------ */
/* Sign: src/sign.cu:194-477                                                 */
/* ------------------------------------------------------------------------ */
int mayo_oracle_sign(int set_id, const uint8_t *esk, const uint8_t *msg, size_t mlen, uint8_t *sig,
                     int force_reject) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return -1;
    mul_init();
    const int m = P->m, o = P->o, k = P->k, n = P->n, v = P->v, menc = P->menc;
    const int sk = P->sk_bytes, dig = P->digest_bytes;
    const int ko = k * o;
    const uint8_t *seed_sk = esk;
    const uint8_t *Ob = esk + sk;
    const uint8_t *P1 = Ob + P->o_bytes;
    const uint8_t *L = P1 + P->p1_bytes;

    /* s_key = digest || R (=0, then salt) || seed_sk || ctr (sign.cu:195-243) */
    const int keylen = dig + 2 * sk;
    uint8_t *key = (uint8_t *)calloc((size_t)keylen + 1, 1);
    mayo_oracle_shake256(key, (size_t)dig, msg, mlen);
    memcpy(key + dig + sk, seed_sk, (size_t)sk);
    uint8_t *salt = (uint8_t *)malloc((size_t)sk);
    mayo_oracle_shake256(salt, (size_t)sk, key, (size_t)keylen);
    memcpy(key + dig, salt, (size_t)sk);
    uint8_t *t = (uint8_t *)malloc((size_t)menc);
    mayo_oracle_shake256(t, (size_t)menc, key, (size_t)(dig + sk));

    const int vr_bytes = n * k / 2;
    uint8_t *Vr = (uint8_t *)malloc((size_t)vr_bytes);
    uint8_t *Mm = (uint8_t *)malloc((size_t)k * m * o);    /* M_i[row][b] nibbles */
    uint8_t *A = (uint8_t *)malloc((size_t)m * ko);
    uint8_t *y = (uint8_t *)malloc((size_t)menc);
    uint8_t *y4 = (uint8_t *)malloc((size_t)m);
    uint8_t *rv = (uint8_t *)malloc((size_t)ko);
    uint8_t *x = (uint8_t *)calloc((size_t)ko, 1);
    int attempts_used = 0;

    for (int ctr = 0; ctr < 255; ctr++) {
        key[keylen] = (uint8_t)ctr;
        mayo_oracle_shake256(Vr, (size_t)vr_bytes, key, (size_t)keylen + 1);   /* sign.cu:250-252 */
        const uint8_t *V = Vr;                       /* V_i = nibbles [i*m, i*m + v) */
        const uint8_t *rp = Vr + k * menc;           /* r: ko nibbles */
        for (int c = 0; c < ko; c++) rv[c] = nib(rp, c);

        /* M_i = V_i * L: M_i[row][b] = sum_a V_i[a] * L[a][b][row] (sign.cu:256-330) */
        for (int i = 0; i < k; i++)
            for (int row = 0; row < m; row++)
                for (int b = 0; b < o; b++) {
                    uint8_t acc = 0;
                    for (int a = 0; a < v; a++)
                        acc ^= MUL[nib(V, i * m + a)][nib(L + (size_t)(a * o + b) * menc, row)];
                    Mm[((size_t)i * m + row) * o + b] = acc;
                }

        /* A assembly with z^ell shifts and one fold by f(z) (sign.cu:333-393) */
        memset(A, 0, (size_t)m * ko);
        int ell = 0;
        for (int i = 0; i < k; i++)
            for (int j = k - 1; j >= i; j--) {
                for (int row = 0; row < m; row++) {
                    int tr = row + ell;
                    for (int b = 0; b < o; b++) {
                        uint8_t mj = Mm[((size_t)j * m + row) * o + b];
                        uint8_t mi = Mm[((size_t)i * m + row) * o + b];
                        if (tr < m) {
                            A[tr * ko + i * o + b] ^= mj;
                            if (i != j) A[tr * ko + j * o + b] ^= mi;
                        } else {
                            for (int q = 0; q < 4; q++) {
                                int rr = tr - m + q;
                                A[rr * ko + i * o + b] ^= MUL[mj][P->poly_c[q]];
                                if (i != j) A[rr * ko + j * o + b] ^= MUL[mi][P->poly_c[q]];
                            }
                        }
                    }
                }
                ell++;
            }

        /* y = sum z^ell U_ell + t (sign.cu:396-460) */
        eval_public_map(P, P1, NULL, NULL, V, m, k, y);
        for (int l = 0; l < menc; l++) y[l] ^= t[l];
        for (int r = 0; r < m; r++) y4[r] = nib(y, r);

        int ok = sample_solution(m, ko, A, y4, rv, x);
        if (ctr < force_reject) {
            /* a rejected attempt leaves x = r (sign.cu:31-33, returns before back-substitution) */
            ok = 0;
            for (int c = 0; c < ko; c++) x[c] = rv[c];
        }
        if (ok) {
            attempts_used = ctr + 1;
            break;
        }
    }

    /* s_packed (sign.cu:147-191) and the salt (sign.cu:475-477) */
    const uint8_t *V = Vr;
    int total = k * n;
    for (int e = 0; e < total; e += 2) {
        uint8_t nb[2];
        for (int h = 0; h < 2; h++) {
            int ee = e + h, i = ee / n, tt = ee - i * n;
            uint8_t val;
            if (tt < m) {
                uint8_t acc = 0;
                for (int q = 0; q < o; q++) acc ^= MUL[nib(Ob, tt * o + q)][x[i * o + q]];
                val = (uint8_t)(nib(V, i * m + tt) ^ acc);
            } else {
                val = x[i * o + (tt - m)];
            }
            nb[h] = val;
        }
        sig[e / 2] = (uint8_t)(nb[0] | (nb[1] << 4));
    }
    memcpy(sig + total / 2, salt, (size_t)sk);

    free(key); free(salt); free(t); free(Vr); free(Mm); free(A); free(y); free(y4); free(rv); free(x);
    return attempts_used;
}

/* ------------------------------------------------------------------------ */
/* Verify: src/verify.cu:9-212                                               */
/* ------------------------------------------------------------------------ */
int mayo_oracle_verify(int set_id, const uint8_t *epk, const uint8_t *msg, size_t mlen,
                       const uint8_t *sig) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return -1;
    mul_init();
    const int menc = P->menc, dig = P->digest_bytes, sk = P->sk_bytes;
    uint8_t *key = (uint8_t *)malloc((size_t)(dig + sk));
    mayo_oracle_shake256(key, (size_t)dig, msg, mlen);
    memcpy(key + dig, sig + P->k * P->n / 2, (size_t)sk);
    uint8_t *t = (uint8_t *)malloc((size_t)menc);
    mayo_oracle_shake256(t, (size_t)menc, key, (size_t)(dig + sk));
    const uint8_t *P1 = epk, *P2 = epk + P->p1_bytes, *P3 = P2 + P->p2_bytes;
    uint8_t *y = (uint8_t *)malloc((size_t)menc);
    eval_public_map(P, P1, P2, P3, sig, P->n, P->k, y);
    int eq = memcmp(y, t, (size_t)menc) == 0;
    free(key);
    free(t);
    free(y);
    return eq ? 0 : 1;
}

/* ------------------------------------------------------------------------ */
/* Batched CPU baseline helpers                                               */
/* ------------------------------------------------------------------------ */
int mayo_oracle_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void mayo_oracle_set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

static void warm_tables(void) {
    keccak_init_tables();
    aes_init_tables();
    mul_init();
}

void mayo_oracle_keypair_batch(int set_id, uint64_t rand_index, size_t batch, uint8_t *sk, uint8_t *pk) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return;
    warm_tables();
#pragma omp parallel for schedule(dynamic, 1)
    for (long b = 0; b < (long)batch; b++)
        mayo_oracle_keypair(set_id, rand_index, (uint64_t)b, sk + (size_t)b * P->sk_bytes,
                            pk + (size_t)b * P->pk_bytes);
}

void mayo_oracle_keypair_from_seed_batch(int set_id, size_t batch, const uint8_t *seeds, uint8_t *pk) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return;
    warm_tables();
#pragma omp parallel for schedule(dynamic, 1)
    for (long b = 0; b < (long)batch; b++)
        mayo_oracle_keypair_from_seed(set_id, seeds + (size_t)b * P->sk_bytes, pk + (size_t)b * P->pk_bytes);
}

void mayo_oracle_expandsk_batch(int set_id, size_t batch, const uint8_t *csk, uint8_t *esk) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return;
    warm_tables();
#pragma omp parallel for schedule(dynamic, 1)
    for (long b = 0; b < (long)batch; b++)
        mayo_oracle_expandsk(set_id, csk + (size_t)b * P->sk_bytes, esk + (size_t)b * P->esk_bytes);
}

void mayo_oracle_expandpk_batch(int set_id, size_t batch, const uint8_t *cpk, uint8_t *epk) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return;
    warm_tables();
#pragma omp parallel for schedule(dynamic, 1)
    for (long b = 0; b < (long)batch; b++)
        mayo_oracle_expandpk(set_id, cpk + (size_t)b * P->pk_bytes, epk + (size_t)b * P->epk_bytes);
}

void mayo_oracle_sign_batch(int set_id, size_t batch, const uint8_t *esk, size_t esk_stride,
                            const uint8_t *msg, const uint64_t *msg_off, const uint32_t *msg_len,
                            uint8_t *sig, int32_t *attempts) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return;
    warm_tables();
#pragma omp parallel for schedule(dynamic, 1)
    for (long b = 0; b < (long)batch; b++) {
        int a = mayo_oracle_sign(set_id, esk + (size_t)b * esk_stride, msg + msg_off[b], msg_len[b],
                                 sig + (size_t)b * P->sig_bytes, 0);
        if (attempts) attempts[b] = a;
    }
}

void mayo_oracle_verify_batch(int set_id, size_t batch, const uint8_t *epk, size_t epk_stride,
                              const uint8_t *msg, const uint64_t *msg_off, const uint32_t *msg_len,
                              const uint8_t *sig, uint8_t *result) {
    const mayo_oracle_params *P = mayo_oracle_get_params(set_id);
    if (!P) return;
    warm_tables();
#pragma omp parallel for schedule(dynamic, 1)
    for (long b = 0; b < (long)batch; b++)
        result[b] = (uint8_t)mayo_oracle_verify(set_id, epk + (size_t)b * epk_stride, msg + msg_off[b],
                                                msg_len[b], sig + (size_t)b * P->sig_bytes);
}
