// Host-side checks of the bitsliced GF(16) helpers in cumayo_b200/csrc/common.cuh (the
// functions are __host__ __device__, so they run here on the CPU).  Built and run by
// tests/test_host_arith.py; prints "OK" or the first failing case.
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include "common.cuh"

using namespace mayo;

static uint32_t ref_mul(uint32_t a, uint32_t b) {  // carry-less product mod x^4 + x + 1
    uint32_t r = 0;
    for (int i = 0; i < 4; i++) if (b >> i & 1) r ^= a << i;
    for (int d = 6; d >= 4; d--) if (r >> d & 1) r ^= 0x13u << (d - 4);
    return r & 0xF;
}
static uint64_t rng_state = 88172645463325252ull;
static uint32_t rnd() { rng_state ^= rng_state << 13; rng_state ^= rng_state >> 7; rng_state ^= rng_state << 17; return (uint32_t)rng_state; }
static uint32_t nib(const uint32_t *w, int c) { return (w[c / 8] >> (4 * (c % 8))) & 0xF; }
#define FAIL(...) do { printf(__VA_ARGS__); printf("\n"); return 1; } while (0)

int main() {
    for (uint32_t a = 0; a < 16; a++) {
        for (uint32_t b = 0; b < 16; b++)
            if (gf16_mul_ct(a, b) != ref_mul(a, b)) FAIL("gf16_mul_ct %u %u", a, b);
        if (a && ref_mul(a, gf16_inv_ct(a)) != 1) FAIL("gf16_inv_ct %u", a);
        if (gf16_inv_reg(a) != gf16_inv_ct(a)) FAIL("gf16_inv_reg %u", a);
    }
    if (gf16_inv_ct(0) != 0) FAIL("inv(0)");
    for (uint32_t p = 0; p < 16; p++) {  // the elimination's quotient e / p from the basis multiples
        const uint32_t b0 = gf16_inv_reg(p), b1 = gf16_xtime(b0), b2 = gf16_xtime(b1), b3 = gf16_xtime(b2);
        const uint4 B = make_uint4(b0, b1, b2, b3);
        for (uint32_t e = 0; e < 16; e++) {
            // entry bits as words that are zero or not (any set bit counts), as the columns hold them
            const uint32_t sh = rnd() & 31;
            const uint32_t d = gf16_div_from_basis((e & 1) << sh, ((e >> 1) & 1) << sh, ((e >> 2) & 1) << sh,
                                                   ((e >> 3) & 1) << sh, B);
            if (p == 0 ? d != 0 : ref_mul(d, p) != e) FAIL("gf16 div %u / %u", e, p);
        }
    }
    for (int it = 0; it < 2000; it++) {
        uint32_t w[4] = {rnd(), rnd(), rnd(), rnd()}, s = rnd() & 0xF;
        // packed -> planes: plane bit b holds coordinate 8*(b&3) + (b>>2)
        G4 g = g4_from_packed(w[0], w[1], w[2], w[3]);
        const uint32_t pl[4] = {g.p0, g.p1, g.p2, g.p3};
        for (int b = 0; b < 32; b++) {
            uint32_t v = 0;
            for (int t = 0; t < 4; t++) v |= ((pl[t] >> b) & 1) << t;
            if (v != nib(w, 8 * (b & 3) + (b >> 2))) FAIL("transpose layout it=%d b=%d", it, b);
        }
        uint4 back = g4_to_packed(g);
        if (back.x != w[0] || back.y != w[1] || back.z != w[2] || back.w != w[3]) FAIL("transpose involution");
        // acc += s * v, coordinate-wise
        uint32_t a0[4] = {rnd(), rnd(), rnd(), rnd()};
        G4 acc = g4_from_packed(a0[0], a0[1], a0[2], a0[3]);
        g4_madd(acc, g, scalar_masks(s));
        uint4 r = g4_to_packed(acc);
        const uint32_t rw[4] = {r.x, r.y, r.z, r.w};
        for (int c = 0; c < 32; c++)
            if (nib(rw, c) != (nib(a0, c) ^ ref_mul(nib(w, c), s))) FAIL("g4_madd it=%d c=%d", it, c);
        // the four-partial-sum form of a sum of products equals the g4_madd sum
        {
            G4 ref = g4_zero();
            G4x4 A = g4x4_zero();
            for (int q = 0; q < 5; q++) {
                const G4 v = g4_from_packed(rnd(), rnd(), rnd(), rnd());
                const uint4 mk = scalar_masks(rnd() & 0xF);
                g4_madd(ref, v, mk);
                g4x4_madd(A, v, mk);
            }
            const G4 f = g4x4_fold(A);
            if (f.p0 != ref.p0 || f.p1 != ref.p1 || f.p2 != ref.p2 || f.p3 != ref.p3) FAIL("g4x4_madd it=%d", it);
        }
        // eight packed nibbles times a public constant
        uint32_t m = nib8_mul_const(w[0], s);
        for (int c = 0; c < 8; c++)
            if (((m >> (4 * c)) & 0xF) != ref_mul((w[0] >> (4 * c)) & 0xF, s)) FAIL("nib8_mul_const");
    }
    printf("OK\n");
    return 0;
}
