// serve_stage.cu -- host-side staging of serving batches for the work queue (no device code).
//
// A serving batch arrives as request records that point into the caller's host memory.  Packing
// copies them, in one pass, into the input staging layout the queue's operands describe; the
// caller copies that buffer to the device in one transfer.  Unpacking scatters the output
// staging buffer (signatures, verify results) back to each request's `out`.
#include <cstring>

#include "../../include/mayo_b200.h"
#include "common.cuh"

namespace {

constexpr int kGroups = 8;  // 2 * set index + (op == verify)

int set_index(int set) { return set == 1 ? 0 : set == 2 ? 1 : set == 3 ? 2 : set == 5 ? 3 : -1; }

constexpr uint32_t kSig[4] = {mayo::Set<1>::sig, mayo::Set<2>::sig, mayo::Set<3>::sig, mayo::Set<5>::sig};
constexpr uint32_t kMaxSig = kSig[3] > kSig[2] ? (kSig[3] > kSig[0] ? kSig[3] : kSig[0]) : kSig[2];
static_assert(kMaxSig >= kSig[0] && kMaxSig >= kSig[1] && kMaxSig >= kSig[2] && kMaxSig >= kSig[3], "max signature");

constexpr size_t al16(size_t x) { return (x + 15) & ~size_t(15); }

// Group of a request, or -1 if the request is malformed.
int group_of(const mayo_b200_serve_req &r, uint32_t max_msg) {
    const int si = set_index(r.set);
    if (si < 0 || (r.op != MAYO_B200_OP_SIGN && r.op != MAYO_B200_OP_VERIFY)) return -1;
    if (r.mlen > max_msg || (r.mlen && !r.msg) || !r.out) return -1;
    if (r.op == MAYO_B200_OP_VERIFY && !r.sig) return -1;
    return 2 * si + (r.op == MAYO_B200_OP_VERIFY ? 1 : 0);
}

}  // namespace

extern "C" {

MAYO_B200_API size_t mayo_b200_serve_in_bytes(uint32_t n, uint32_t max_msg) {
    return al16(4 * (size_t)n) + (size_t)kGroups * 4 * 16 + (size_t)n * (8 + (size_t)max_msg + kMaxSig);
}

MAYO_B200_API size_t mayo_b200_serve_out_bytes(uint32_t n) { return (size_t)n * kMaxSig + kGroups * 16; }

MAYO_B200_API int mayo_b200_serve_pack(const mayo_b200_serve_req *req, uint32_t n, uint32_t max_msg,
                                       uint8_t *stage_in, size_t in_capacity, size_t out_capacity,
                                       mayo_b200_serve_layout *layout) {
    if (!layout || (n && (!req || !stage_in)) || n > (1u << 20)) return MAYO_B200_ERR_ARG;
    std::memset(layout, 0, sizeof(*layout));
    layout->n = n;
    layout->max_msg = max_msg;
    uint32_t cnt[kGroups] = {};
    for (uint32_t i = 0; i < n; i++) {
        const int g = group_of(req[i], max_msg);
        if (g < 0) return MAYO_B200_ERR_ARG;
        cnt[g]++;
    }
    size_t off = al16(4 * (size_t)n), out = 0;
    for (int g = 0; g < kGroups; g++) {
        if (!cnt[g]) continue;
        mayo_b200_serve_group &G = layout->group[g];
        const bool vf = g & 1;
        const size_t c = cnt[g], sb = kSig[g >> 1];
        G.count = cnt[g];
        G.set = (uint32_t)(g >> 1 == 0 ? 1 : g >> 1 == 1 ? 2 : g >> 1 == 2 ? 3 : 5);
        G.op = vf ? MAYO_B200_OP_VERIFY : MAYO_B200_OP_SIGN;
        G.key_off = off;
        off = al16(off + 4 * c);
        G.len_off = off;
        off = al16(off + 4 * c);
        G.msg_off = off;
        off = al16(off + c * max_msg);
        if (vf) {
            G.sig_off = off;
            off = al16(off + c * sb);
        }
        G.out_off = out;
        out = al16(out + (vf ? c : c * sb));
    }
    if (off > in_capacity || out > out_capacity) return MAYO_B200_ERR_ARG;
    layout->in_bytes = off;
    layout->out_bytes = out;
    uint32_t cur[kGroups] = {};
    for (uint32_t i = 0; i < n; i++) {
        const mayo_b200_serve_req &r = req[i];
        const int g = group_of(r, max_msg);
        const mayo_b200_serve_group &G = layout->group[g];
        const uint32_t rank = cur[g]++;
        const uint32_t item = ((uint32_t)r.op << 30) | ((uint32_t)(g >> 1) << 28) | rank;
        std::memcpy(stage_in + 4 * (size_t)i, &item, 4);
        std::memcpy(stage_in + G.key_off + 4 * (size_t)rank, &r.key_slot, 4);
        std::memcpy(stage_in + G.len_off + 4 * (size_t)rank, &r.mlen, 4);
        if (r.mlen) std::memcpy(stage_in + G.msg_off + (size_t)rank * max_msg, r.msg, r.mlen);
        if (g & 1) std::memcpy(stage_in + G.sig_off + (size_t)rank * kSig[g >> 1], r.sig, kSig[g >> 1]);
    }
    return MAYO_B200_OK;
}

MAYO_B200_API int mayo_b200_serve_unpack(const mayo_b200_serve_req *req, uint32_t n,
                                         const mayo_b200_serve_layout *layout, const uint8_t *stage_out) {
    if (!layout || (n && (!req || !stage_out)) || n != layout->n) return MAYO_B200_ERR_ARG;
    uint32_t cur[kGroups] = {};
    for (uint32_t i = 0; i < n; i++) {
        const mayo_b200_serve_req &r = req[i];
        const int g = group_of(r, layout->max_msg);
        if (g < 0 || cur[g] >= layout->group[g].count) return MAYO_B200_ERR_ARG;
        const uint32_t rank = cur[g]++;
        const mayo_b200_serve_group &G = layout->group[g];
        if (g & 1) r.out[0] = stage_out[G.out_off + rank];
        else std::memcpy(r.out, stage_out + G.out_off + (size_t)rank * kSig[g >> 1], kSig[g >> 1]);
    }
    return MAYO_B200_OK;
}

}  // extern "C"
