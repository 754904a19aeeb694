// A small C++ caller of the reference's batched API, compiled against this repository's drop-in
// header include/api.cuh (-DMAYO_VERSION=N) and linked with libmayo_b200.so: the code a user of
// the reference's include/api.cuh writes (its names, default arguments and pool layouts, as in
// the reference's tests/bench_stream.cu), with nothing from this library's own API.
//
//   dropin_driver <out_file> [batch] [mlen]
//
// keypair (rand_index 0) -> keypair_DtH -> signWithesk (HtD, kernel, DtH) -> verifyWithepk (HtD,
// kernel, DtH) on the good signatures and again with one nibble of every other signature flipped.
// Writes sk || pk || sig || result(good) || result(corrupted) for the whole batch to out_file;
// tests/test_dropin.py compares them with the oracle.  Exit status 0, or 1 with a message.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "api.cuh"

#define CHECK(x)                                                                             \
    do {                                                                                     \
        if ((x) != cudaSuccess) {                                                            \
            std::fprintf(stderr, "%s failed: %s\n", #x, cudaGetErrorString(cudaGetLastError())); \
            return 1;                                                                        \
        }                                                                                    \
    } while (0)
#define CHECK_API(what)                                                                         \
    do {                                                                                        \
        if (mayo_api_last_status() != MAYO_B200_OK) {                                          \
            std::fprintf(stderr, "%s: %s\n", what, mayo_b200_status_string(mayo_api_last_status())); \
            return 1;                                                                           \
        }                                                                                       \
    } while (0)

static size_t a128(size_t x) { return (x + 127) / 128 * 128; }

int main(int argc, char **argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s out_file [batch] [mlen]\n", argv[0]);
        return 1;
    }
    const size_t batch = argc > 2 ? std::strtoul(argv[2], nullptr, 10) : 8;
    const size_t mlen = argc > 3 ? std::strtoul(argv[3], nullptr, 10) : 32;
    mayo_b200_sizes z;
    if (mayo_b200_get_sizes(MAYO_VERSION, mlen, &z) != MAYO_B200_OK) return 1;
    aes128_tables_init();
    CHECK_API("aes128_tables_init");
    cudaStream_t st;
    CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));

    // host buffers, pinned as in the reference benchmark
    uint8_t *h_pk, *h_sk, *h_msg, *h_sig, *h_res;
    CHECK(cudaMallocHost(&h_pk, batch * z.pk_bytes));
    CHECK(cudaMallocHost(&h_sk, batch * z.sk_bytes));
    CHECK(cudaMallocHost(&h_msg, batch * (mlen ? mlen : 1)));
    CHECK(cudaMallocHost(&h_sig, batch * z.sig_bytes));
    CHECK(cudaMallocHost(&h_res, 2 * batch));
    for (size_t i = 0; i < batch * mlen; i++) h_msg[i] = (uint8_t)(i * 131 + 7);

    // keypair pool: sk @0, pk @A(SK), P1||P2 scratch after
    uint8_t *kp;
    size_t kp_pitch;
    CHECK(cudaMallocPitch(&kp, &kp_pitch, a128(z.sk_bytes) + a128(z.pk_bytes) + a128(z.p_bytes), batch));
    crypto_sign_keypair(kp, kp_pitch, batch, st);  // rand_index defaults to 0
    CHECK_API("crypto_sign_keypair");
    crypto_sign_keypair_DtH(h_pk, h_sk, kp, kp_pitch, batch, st);
    CHECK_API("crypto_sign_keypair_DtH");

    // signWithesk pool: csk @0 (expanded in place), message @A(ESK), signature @A(ESK)+A(mlen)
    uint8_t *sp;
    size_t sp_pitch;
    const size_t scratch = (size_t)z.k * z.m * ((z.o + 1) / 2);
    CHECK(cudaMallocPitch(&sp, &sp_pitch, a128(z.esk_bytes) + a128(mlen) + a128(z.sig_bytes) + a128(scratch), batch));
    crypto_sign_signWithesk_HtD(h_sk, h_msg, mlen, sp, sp_pitch, batch, st);
    CHECK_API("crypto_sign_signWithesk_HtD");
    crypto_sign_signWithesk(sp, mlen, sp_pitch, batch, st);
    CHECK_API("crypto_sign_signWithesk");
    crypto_sign_signWithesk_DtH(h_sig, sp, mlen, sp_pitch, batch, st);
    CHECK_API("crypto_sign_signWithesk_DtH");
    CHECK(cudaStreamSynchronize(st));

    // verifyWithepk pool: cpk @P-16 (expanded in place), message @A(EPK), sig, result byte
    uint8_t *vp;
    size_t vp_pitch;
    CHECK(cudaMallocPitch(&vp, &vp_pitch, a128(z.epk_bytes) + a128(mlen) + a128(z.sig_bytes) + 1, batch));
    std::vector<uint8_t> bad(h_sig, h_sig + batch * z.sig_bytes);
    for (size_t i = 1; i < batch; i += 2) bad[i * z.sig_bytes + (i * 7) % z.sig_bytes] ^= 0x10;
    for (int pass = 0; pass < 2; pass++) {
        uint8_t *sigs = pass == 0 ? h_sig : bad.data();
        crypto_sign_verifyWithepk_HtD(h_pk, h_msg, sigs, mlen, vp, vp_pitch, batch, st);
        CHECK_API("crypto_sign_verifyWithepk_HtD");
        crypto_sign_verifyWithepk(vp, mlen, vp_pitch, batch, st);
        CHECK_API("crypto_sign_verifyWithepk");
        crypto_sign_verifyWithepk_DtH(h_res + pass * batch, mlen, vp, vp_pitch, batch, st);
        CHECK_API("crypto_sign_verifyWithepk_DtH");
        CHECK(cudaStreamSynchronize(st));
    }

    FILE *f = std::fopen(argv[1], "wb");
    if (!f) return 1;
    std::fwrite(h_sk, 1, batch * z.sk_bytes, f);
    std::fwrite(h_pk, 1, batch * z.pk_bytes, f);
    std::fwrite(h_sig, 1, batch * z.sig_bytes, f);
    std::fwrite(h_res, 1, 2 * batch, f);
    std::fclose(f);
    cudaFree(kp);
    cudaFree(sp);
    cudaFree(vp);
    cudaFreeHost(h_pk);
    cudaFreeHost(h_sk);
    cudaFreeHost(h_msg);
    cudaFreeHost(h_sig);
    cudaFreeHost(h_res);
    cudaStreamDestroy(st);
    return 0;
}
