// serve_loop.cu -- the serving loop in C++ behind the C-ABI (no device code of its own).
//
// Continuous batching of MAYO sign / verify requests over the persistent work queue, with the
// expanded keys resident in HBM:
//   * requests (mayo_b200_serve_req records pointing into the caller's host memory) join a
//     waiting line;
//   * whenever one of the `inflight` batch slots is free and requests wait, the longest prefix of
//     the line (at most max_batch) whose keys fit in the key tables beside the keys that batches
//     in flight hold is admitted: keys that are not resident are expanded into free table rows
//     (seed -> keypair -> esk, epk), the batch is packed into the slot's pinned staging buffer,
//     copied to the device in one transfer, run by the work queue on the slot's stream, and its
//     results copied back in one transfer;
//   * a finished batch (its event complete) is unpacked into each request's `out` and its
//     requests are reported by tag; its key rows are released.
// Key tables: per parameter set `key_slots` rows of esk and of epk, least-recently-used eviction
// of rows no batch in flight uses (MayoKeyTable).  The caller supplies all device and pinned host
// memory; the server creates only CUDA streams and events.
//
// No counterpart in the reference, which offers only its synchronous batched pool API
// (include/api.cuh); this is the continuous-batching path of the benchmark's serving workload.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <new>
#include <vector>

#include "../../include/mayo_b200.h"
#include "common.cuh"
#include "ops.h"

// ---------------------------------------------------------------------------------------------
// key table: key id -> row of a set's key table, least-recently-used eviction, pinning
// ---------------------------------------------------------------------------------------------
struct mayo_b200_key_table {
    uint32_t cap = 0, nkeys = 0;
    std::vector<int32_t> slot_of, key_of, pins;
    std::vector<uint64_t> last;
    uint64_t tick = 0, misses = 0, evictions = 0;
    std::vector<uint8_t> mark;  // scratch: slots used by the batch being acquired
    std::vector<int32_t> used, cand;

    bool init(uint32_t capacity, uint32_t n_keys) {
        if (capacity == 0 || n_keys == 0) return false;
        cap = capacity;
        nkeys = n_keys;
        slot_of.assign(n_keys, -1);
        key_of.assign(capacity, -1);
        pins.assign(capacity, 0);
        last.assign(capacity, 0);
        mark.assign(capacity, 0);
        return true;
    }

    // Distinct resident slots of ids[0, n) into `used` (marks set); number of distinct missing ids
    // (their slot_of entries temporarily set to -2 to count them once, restored before return).
    uint32_t scan(const uint32_t *ids, uint32_t n) {
        used.clear();
        uint32_t nmiss = 0;
        for (uint32_t i = 0; i < n; i++) {
            const int32_t s = slot_of[ids[i]];
            if (s >= 0) {
                if (!mark[s]) {
                    mark[s] = 1;
                    used.push_back(s);
                }
            } else if (s == -1) {
                slot_of[ids[i]] = -2;
                nmiss++;
            }
        }
        for (uint32_t i = 0; i < n; i++)
            if (slot_of[ids[i]] == -2) slot_of[ids[i]] = -1;
        return nmiss;
    }
    void unmark() {
        for (int32_t s : used) mark[s] = 0;
    }

    bool valid(const uint32_t *ids, uint32_t n) const {
        for (uint32_t i = 0; i < n; i++)
            if (ids[i] >= nkeys) return false;
        return true;
    }

    // Whether acquire(ids) would find rows for its missing keys (no state change).
    bool can_load(const uint32_t *ids, uint32_t n) {
        const uint32_t nmiss = scan(ids, n);
        bool ok = true;
        if (nmiss) {
            uint32_t free = 0;
            for (uint32_t s = 0; s < cap; s++) free += (pins[s] == 0 && !mark[s]) ? 1u : 0u;
            ok = free >= nmiss;
        }
        unmark();
        return ok;
    }

    // Rows for ids[0, n) (slots[i]), loading the missing keys into unpinned rows not used by this
    // batch (empty rows first, then the least recently used); every distinct row the batch uses
    // is pinned once.  miss_ids / miss_slots receive the distinct missing ids and their new rows.
    int acquire(const uint32_t *ids, uint32_t n, int32_t *slots, std::vector<uint32_t> &miss_ids,
                std::vector<int32_t> &miss_slots) {
        miss_ids.clear();
        miss_slots.clear();
        if (!valid(ids, n)) return MAYO_B200_ERR_ARG;
        tick++;
        const uint32_t nmiss = scan(ids, n);
        if (nmiss) {
            cand.clear();
            for (uint32_t s = 0; s < cap; s++)
                if (pins[s] == 0 && !mark[s]) cand.push_back((int32_t)s);
            if (cand.size() < nmiss) {
                unmark();
                return MAYO_B200_ERR_FULL;
            }
            // empty rows first (priority -1), then the least recently used
            auto pri = [&](int32_t s) { return key_of[s] < 0 ? -1.0 : (double)last[s]; };
            std::nth_element(cand.begin(), cand.begin() + (nmiss - 1), cand.end(),
                             [&](int32_t a, int32_t b) { return pri(a) < pri(b) || (pri(a) == pri(b) && a < b); });
            uint32_t k = 0;
            for (uint32_t i = 0; i < n; i++) {
                const uint32_t id = ids[i];
                if (slot_of[id] >= 0) continue;
                const int32_t s = cand[k++];
                if (key_of[s] >= 0) {
                    slot_of[key_of[s]] = -1;
                    evictions++;
                }
                key_of[s] = (int32_t)id;
                slot_of[id] = s;
                miss_ids.push_back(id);
                miss_slots.push_back(s);
                mark[s] = 1;
                used.push_back(s);
            }
            misses += nmiss;
        }
        for (uint32_t i = 0; i < n; i++) slots[i] = slot_of[ids[i]];
        for (int32_t s : used) {
            last[s] = tick;
            pins[s]++;
        }
        unmark();
        return MAYO_B200_OK;
    }

    // Unpins every distinct row among slots[0, n) once (the rows one acquire returned).
    int release(const int32_t *slots, uint32_t n) {
        used.clear();
        for (uint32_t i = 0; i < n; i++) {
            const int32_t s = slots[i];
            if (s < 0 || (uint32_t)s >= cap) {
                unmark();
                return MAYO_B200_ERR_ARG;
            }
            if (!mark[s]) {
                mark[s] = 1;
                used.push_back(s);
            }
        }
        for (int32_t s : used)
            if (pins[s] <= 0) {
                unmark();
                return MAYO_B200_ERR_ARG;
            }
        for (int32_t s : used) pins[s]--;
        unmark();
        return MAYO_B200_OK;
    }
};

namespace {

using mayo::api_cuda_rc;
using mayo::api_launch_rc;

constexpr int kSets[4] = {1, 2, 3, 5};
constexpr size_t kAlign = 256;
inline size_t al(size_t x, size_t a = kAlign) { return (x + a - 1) / a * a; }
inline size_t a128(size_t x) { return (x + 127) / 128 * 128; }

struct SetSz {
    size_t sk, pk, esk, epk, p, sig;
};
SetSz set_sizes(int si) {
    switch (si) {
#define SZ(ID) \
    case ID: return SetSz{mayo::Set<kSets[ID]>::sk, mayo::Set<kSets[ID]>::pk, mayo::Set<kSets[ID]>::esk, \
                          mayo::Set<kSets[ID]>::epk, mayo::Set<kSets[ID]>::p, mayo::Set<kSets[ID]>::sig};
        SZ(0) SZ(1) SZ(2) SZ(3)
#undef SZ
        default: return SetSz{};
    }
}
// keypair pool row of set index si, rounded to 512 like cudaMallocPitch
size_t kp_pitch(int si) {
    const SetSz z = set_sizes(si);
    return (a128(z.sk) + a128(z.pk) + a128(z.p) + 511) / 512 * 512;
}

uint32_t expand_chunk(const mayo_b200_server_config &c) { return c.expand_chunk ? c.expand_chunk : 256; }
uint32_t key_rows(const mayo_b200_server_config &c, int si) {
    const uint32_t n = c.n_keys[si];
    return c.key_slots[si] && c.key_slots[si] < n ? c.key_slots[si] : n;
}
uint32_t queue_capacity(const mayo_b200_server_config &c) { return c.max_batch + c.max_batch / 8 + 64; }

// Device arena layout: per set the esk and epk tables, the expansion scratch (a keypair pool, an
// esk and an epk pool of expand_chunk rows, sized for the largest set), then per batch slot the
// queue memory, the input and the output staging.  Host (pinned) arena: per slot the input and
// output staging, then the seed staging of one expansion chunk.
struct Layout {
    size_t esk[4], epk[4], x_kp, x_esk, x_epk, dev_slot0, dev_slot, q_off, din_off, dout_off, dev_total;
    size_t host_slot, hin_off, hout_off, h_seed, host_total, qmem, in_bytes, out_bytes;
};
int layout_of(const mayo_b200_server_config &c, Layout &L) {
    if (c.max_batch == 0 || c.max_batch > (1u << 20) || c.inflight == 0 || c.inflight > 64 || c.max_msg > (1u << 20))
        return MAYO_B200_ERR_ARG;
    size_t off = 0;
    size_t max_kp = 0, max_esk = 0, max_epk = 0, max_sk = 0;
    for (int si = 0; si < 4; si++) {
        const SetSz z = set_sizes(si);
        const size_t rows = key_rows(c, si);
        L.esk[si] = off;
        off = al(off + rows * z.esk);
        L.epk[si] = off;
        off = al(off + rows * z.epk);
        if (c.n_keys[si]) {
            max_kp = std::max(max_kp, kp_pitch(si));
            max_esk = std::max(max_esk, z.esk);
            max_epk = std::max(max_epk, z.epk);
            max_sk = std::max(max_sk, z.sk);
        }
    }
    const size_t ch = expand_chunk(c);
    L.x_kp = off;
    off = al(off + ch * max_kp);
    L.x_esk = off;
    off = al(off + ch * max_esk);
    L.x_epk = off;
    off = al(off + ch * max_epk);
    L.qmem = mayo_b200_queue_mem_bytes(queue_capacity(c), 0);
    if (L.qmem == 0) return MAYO_B200_ERR_CUDA;
    L.in_bytes = mayo_b200_serve_in_bytes(c.max_batch, c.max_msg);
    L.out_bytes = mayo_b200_serve_out_bytes(c.max_batch);
    L.q_off = 0;
    L.din_off = al(L.qmem);
    L.dout_off = L.din_off + al(L.in_bytes);
    L.dev_slot = L.dout_off + al(L.out_bytes);
    L.dev_slot0 = off;
    L.dev_total = off + (size_t)c.inflight * L.dev_slot;
    L.hin_off = 0;
    L.hout_off = al(L.in_bytes);
    L.host_slot = L.hout_off + al(L.out_bytes);
    L.h_seed = (size_t)c.inflight * L.host_slot;
    L.host_total = L.h_seed + al(ch * max_sk);
    return MAYO_B200_OK;
}

struct Waiting {
    mayo_b200_serve_req req;
    uint64_t tag;
};

struct Slot {
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;
    uint8_t *qmem = nullptr, *d_in = nullptr, *d_out = nullptr, *h_in = nullptr, *h_out = nullptr;
    bool busy = false;
    std::vector<mayo_b200_serve_req> reqs;
    std::vector<uint64_t> tags;
    mayo_b200_serve_layout lay{};
    std::vector<int32_t> pinned[4];  // rows acquired per set
};

int set_index(int set) { return set == 1 ? 0 : set == 2 ? 1 : set == 3 ? 2 : set == 5 ? 3 : -1; }

}  // namespace

struct mayo_b200_server {
    mayo_b200_server_config cfg{};
    Layout L{};
    int dev = 0;
    const uint8_t *seeds[4] = {};
    mayo_b200_key_table tab[4];
    uint8_t *dmem = nullptr, *hmem = nullptr;
    cudaEvent_t x_ready = nullptr, x_copied = nullptr;
    bool x_any = false;
    std::vector<Slot> slots;
    std::deque<Waiting> waiting;
    std::deque<uint64_t> done;
    mayo_b200_server_stats st{};
    // scratch
    std::vector<uint32_t> ids[4];
    std::vector<int32_t> rows[4];
    std::vector<uint32_t> miss_ids;
    std::vector<int32_t> miss_slots;

    ~mayo_b200_server() {
        for (Slot &s : slots) {
            if (s.st) cudaStreamDestroy(s.st);
            if (s.ev) cudaEventDestroy(s.ev);
        }
        if (x_ready) cudaEventDestroy(x_ready);
        if (x_copied) cudaEventDestroy(x_copied);
    }

    // Whether the first k waiting requests' keys can all be resident at once now.
    bool fits(uint32_t k) {
        for (int si = 0; si < 4; si++) ids[si].clear();
        for (uint32_t i = 0; i < k; i++) {
            const Waiting &w = waiting[i];
            ids[set_index(w.req.set)].push_back(w.req.key_id);
        }
        for (int si = 0; si < 4; si++)
            if (!ids[si].empty() && !tab[si].can_load(ids[si].data(), (uint32_t)ids[si].size())) return false;
        return true;
    }
    uint32_t admit_len() {
        const uint32_t k = (uint32_t)std::min<size_t>(waiting.size(), cfg.max_batch);
        if (k == 0 || fits(k)) return k;
        uint32_t lo = 0, hi = k;  // fits(lo) holds, fits(hi) does not
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (fits(mid)) lo = mid;
            else hi = mid;
        }
        return lo;
    }

    // Expands keys miss_ids of set index si (seed -> pk -> esk, epk) into table rows miss_slots,
    // on stream s, through the scratch pools in chunks.
    int expand(int si, cudaStream_t s) {
        const SetSz z = set_sizes(si);
        const int set = kSets[si];
        const size_t kpp = kp_pitch(si), ch = expand_chunk(cfg);
        uint8_t *kp = dmem + L.x_kp, *xe = dmem + L.x_esk, *xp = dmem + L.x_epk, *hs = hmem + L.h_seed;
        for (size_t c0 = 0; c0 < miss_ids.size(); c0 += ch) {
            const size_t n = std::min(ch, miss_ids.size() - c0);
            // the seed staging and the scratch pools are shared: wait for their previous users
            if (x_any) {
                cudaError_t e = cudaEventSynchronize(x_copied);
                if (e != cudaSuccess) return api_cuda_rc(e);
                if ((e = cudaStreamWaitEvent(s, x_ready, 0)) != cudaSuccess) return api_cuda_rc(e);
            }
            for (size_t i = 0; i < n; i++) std::memcpy(hs + i * z.sk, seeds[si] + (size_t)miss_ids[c0 + i] * z.sk, z.sk);
            cudaError_t e = cudaMemcpy2DAsync(kp, kpp, hs, z.sk, z.sk, n, cudaMemcpyHostToDevice, s);
            if (e == cudaSuccess) e = cudaEventRecord(x_copied, s);
            if (e != cudaSuccess) return api_cuda_rc(e);
            int rc = api_launch_rc(mayo::launch_keypair_seeded(set, kp, kpp, n, s));
            if (rc != MAYO_B200_OK) return rc;
            // esk rows: seed_sk at offset 0, expanded in place; epk rows: cpk at P - 16
            e = cudaMemcpy2DAsync(xe, z.esk, kp, kpp, z.sk, n, cudaMemcpyDeviceToDevice, s);
            if (e == cudaSuccess)
                e = cudaMemcpy2DAsync(xp + z.p - 16, z.epk, kp + a128(z.sk), kpp, z.pk, n, cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return api_cuda_rc(e);
            if ((rc = api_launch_rc(mayo::launch_expandsk(set, xe, z.esk, n, s))) != MAYO_B200_OK) return rc;
            if ((rc = api_launch_rc(mayo::launch_expandpk(set, xp, z.epk, n, s))) != MAYO_B200_OK) return rc;
            for (size_t i = 0; i < n; i++) {
                const size_t row = (size_t)miss_slots[c0 + i];
                e = cudaMemcpyAsync(dmem + L.esk[si] + row * z.esk, xe + i * z.esk, z.esk, cudaMemcpyDeviceToDevice, s);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(dmem + L.epk[si] + row * z.epk, xp + i * z.epk, z.epk, cudaMemcpyDeviceToDevice,
                                        s);
                if (e != cudaSuccess) return api_cuda_rc(e);
            }
            if ((e = cudaEventRecord(x_ready, s)) != cudaSuccess) return api_cuda_rc(e);
            x_any = true;
            st.keys_expanded += n;
        }
        return MAYO_B200_OK;
    }

    void release(Slot &sl) {
        for (int si = 0; si < 4; si++) {
            if (!sl.pinned[si].empty()) tab[si].release(sl.pinned[si].data(), (uint32_t)sl.pinned[si].size());
            sl.pinned[si].clear();
        }
    }

    // Admits the longest fitting prefix of the waiting line into slot sl and launches it.
    int launch(Slot &sl, uint32_t k) {
        sl.reqs.resize(k);
        sl.tags.resize(k);
        for (uint32_t i = 0; i < k; i++) {
            sl.reqs[i] = waiting[i].req;
            sl.tags[i] = waiting[i].tag;
        }
        // key rows per set (and expansions of the missing keys, on this batch's stream)
        for (int si = 0; si < 4; si++) {
            ids[si].clear();
            rows[si].clear();
        }
        for (uint32_t i = 0; i < k; i++) ids[set_index(sl.reqs[i].set)].push_back(sl.reqs[i].key_id);
        int rc = MAYO_B200_OK;
        int si = 0;
        for (; si < 4 && rc == MAYO_B200_OK; si++) {
            if (ids[si].empty()) continue;
            rows[si].resize(ids[si].size());
            rc = tab[si].acquire(ids[si].data(), (uint32_t)ids[si].size(), rows[si].data(), miss_ids, miss_slots);
            if (rc != MAYO_B200_OK) break;
            sl.pinned[si] = rows[si];
            if (!miss_ids.empty()) rc = expand(si, sl.st);
        }
        if (rc != MAYO_B200_OK) {
            release(sl);
            return rc;
        }
        uint32_t cur[4] = {};
        for (uint32_t i = 0; i < k; i++) {
            const int s = set_index(sl.reqs[i].set);
            sl.reqs[i].key_slot = (uint32_t)rows[s][cur[s]++];
        }
        rc = mayo_b200_serve_pack(sl.reqs.data(), k, cfg.max_msg, sl.h_in, L.in_bytes, L.out_bytes, &sl.lay);
        if (rc != MAYO_B200_OK) {
            release(sl);
            return rc;
        }
        mayo_b200_queue_ops ops[4];
        std::memset(ops, 0, sizeof(ops));
        uint32_t groups = 0;
        for (const mayo_b200_serve_group &g : sl.lay.group) {
            if (!g.count) continue;
            groups++;
            const int gi = set_index((int)g.set);
            mayo_b200_queue_ops &o = ops[gi];
            const uint32_t nk = key_rows(cfg, gi);
            if (g.op == MAYO_B200_OP_SIGN) {
                o.sg_esk = dmem + L.esk[gi];
                o.sg_nkeys = nk;
                o.sg_key = reinterpret_cast<const uint32_t *>(sl.d_in + g.key_off);
                o.sg_msg = sl.d_in + g.msg_off;
                o.sg_msg_len = reinterpret_cast<const uint32_t *>(sl.d_in + g.len_off);
                o.sg_mlen = cfg.max_msg;
                o.sg_sig = sl.d_out + g.out_off;
                o.sg_count = g.count;
            } else {
                o.vf_epk = dmem + L.epk[gi];
                o.vf_nkeys = nk;
                o.vf_key = reinterpret_cast<const uint32_t *>(sl.d_in + g.key_off);
                o.vf_msg = sl.d_in + g.msg_off;
                o.vf_msg_len = reinterpret_cast<const uint32_t *>(sl.d_in + g.len_off);
                o.vf_mlen = cfg.max_msg;
                o.vf_sig = sl.d_in + g.sig_off;
                o.vf_res = sl.d_out + g.out_off;
                o.vf_count = g.count;
            }
        }
        cudaError_t e = x_any ? cudaStreamWaitEvent(sl.st, x_ready, 0) : cudaSuccess;
        if (e == cudaSuccess) e = cudaMemcpyAsync(sl.d_in, sl.h_in, sl.lay.in_bytes, cudaMemcpyHostToDevice, sl.st);
        if (e != cudaSuccess) {
            release(sl);
            return api_cuda_rc(e);
        }
        rc = mayo_b200_queue_run(ops, reinterpret_cast<const uint32_t *>(sl.d_in), k, nullptr, sl.qmem,
                                 queue_capacity(cfg), nullptr, 0, sl.st);
        if (rc != MAYO_B200_OK) {
            release(sl);
            return rc;
        }
        e = cudaMemcpyAsync(sl.h_out, sl.d_out, sl.lay.out_bytes, cudaMemcpyDeviceToHost, sl.st);
        if (e == cudaSuccess) e = cudaEventRecord(sl.ev, sl.st);
        if (e != cudaSuccess) {
            release(sl);
            return api_cuda_rc(e);
        }
        waiting.erase(waiting.begin(), waiting.begin() + k);
        sl.busy = true;
        st.batches++;
        st.requests_admitted += k;
        st.max_batch_seen = std::max<uint64_t>(st.max_batch_seen, k);
        st.kernel_launches += 2 + groups;  // queue fill + partition + one persistent kernel per (set, op)
        return MAYO_B200_OK;
    }

    // Finished batches -> results unpacked, rows released, tags to `done`.
    int collect() {
        for (Slot &sl : slots) {
            if (!sl.busy) continue;
            const cudaError_t q = cudaEventQuery(sl.ev);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess) return api_cuda_rc(q);
            const int rc = mayo_b200_serve_unpack(sl.reqs.data(), (uint32_t)sl.reqs.size(), &sl.lay, sl.h_out);
            release(sl);
            sl.busy = false;
            if (rc != MAYO_B200_OK) return rc;
            for (uint64_t t : sl.tags) done.push_back(t);
            st.requests_done += sl.tags.size();
        }
        return MAYO_B200_OK;
    }

    int admit() {
        for (Slot &sl : slots) {
            if (sl.busy || waiting.empty()) continue;
            const uint32_t k = admit_len();
            if (k == 0) break;  // wait for a batch in flight to release key rows
            const int rc = launch(sl, k);
            if (rc != MAYO_B200_OK) return rc;
        }
        return MAYO_B200_OK;
    }
};

extern "C" {

MAYO_B200_API mayo_b200_key_table *mayo_b200_key_table_create(uint32_t capacity, uint32_t n_keys) {
    mayo_b200_key_table *t = new (std::nothrow) mayo_b200_key_table();
    if (t && !t->init(capacity, n_keys)) {
        delete t;
        t = nullptr;
    }
    return t;
}
MAYO_B200_API void mayo_b200_key_table_destroy(mayo_b200_key_table *t) { delete t; }
MAYO_B200_API int mayo_b200_key_table_acquire(mayo_b200_key_table *t, const uint32_t *key_ids, uint32_t n,
                                              int32_t *slots, uint32_t *miss_ids, int32_t *miss_slots,
                                              uint32_t *n_miss) {
    if (!t || (n && (!key_ids || !slots))) return MAYO_B200_ERR_ARG;
    std::vector<uint32_t> mi;
    std::vector<int32_t> ms;
    const int rc = t->acquire(key_ids, n, slots, mi, ms);
    if (n_miss) *n_miss = (uint32_t)mi.size();
    for (size_t i = 0; i < mi.size(); i++) {
        if (miss_ids) miss_ids[i] = mi[i];
        if (miss_slots) miss_slots[i] = ms[i];
    }
    return rc;
}
MAYO_B200_API int mayo_b200_key_table_release(mayo_b200_key_table *t, const int32_t *slots, uint32_t n) {
    if (!t || (n && !slots)) return MAYO_B200_ERR_ARG;
    return t->release(slots, n);
}
MAYO_B200_API int mayo_b200_key_table_can_load(mayo_b200_key_table *t, const uint32_t *key_ids, uint32_t n) {
    if (!t || (n && !key_ids) || !t->valid(key_ids, n)) return -1;
    return t->can_load(key_ids, n) ? 1 : 0;
}
MAYO_B200_API int mayo_b200_key_table_info(const mayo_b200_key_table *t, mayo_b200_key_table_stats *out) {
    if (!t || !out) return MAYO_B200_ERR_ARG;
    out->capacity = t->cap;
    out->n_keys = t->nkeys;
    out->misses = t->misses;
    out->evictions = t->evictions;
    uint32_t pinned = 0, resident = 0;
    for (uint32_t s = 0; s < t->cap; s++) {
        pinned += t->pins[s] > 0;
        resident += t->key_of[s] >= 0;
    }
    out->pinned_slots = pinned;
    out->resident_keys = resident;
    return MAYO_B200_OK;
}
MAYO_B200_API int32_t mayo_b200_key_table_slot_of(const mayo_b200_key_table *t, uint32_t key_id) {
    return t && key_id < t->nkeys ? t->slot_of[key_id] : -1;
}
MAYO_B200_API int32_t mayo_b200_key_table_pins(const mayo_b200_key_table *t, uint32_t slot) {
    return t && slot < t->cap ? t->pins[slot] : -1;
}

MAYO_B200_API size_t mayo_b200_server_device_bytes(const mayo_b200_server_config *cfg) {
    Layout L;
    return cfg && layout_of(*cfg, L) == MAYO_B200_OK ? L.dev_total : 0;
}
MAYO_B200_API size_t mayo_b200_server_host_bytes(const mayo_b200_server_config *cfg) {
    Layout L;
    return cfg && layout_of(*cfg, L) == MAYO_B200_OK ? L.host_total : 0;
}

MAYO_B200_API int mayo_b200_server_create(const mayo_b200_server_config *cfg, const uint8_t *const seeds[4],
                                          void *device_mem, size_t device_bytes, void *host_pinned,
                                          size_t host_bytes, mayo_b200_server **out) {
    if (!cfg || !seeds || !out) return MAYO_B200_ERR_ARG;
    *out = nullptr;
    Layout L;
    int rc = layout_of(*cfg, L);
    if (rc != MAYO_B200_OK) return rc;
    if (!device_mem || !host_pinned || device_bytes < L.dev_total || host_bytes < L.host_total) return MAYO_B200_ERR_ARG;
    if ((reinterpret_cast<uintptr_t>(device_mem) | reinterpret_cast<uintptr_t>(host_pinned)) & (kAlign - 1))
        return MAYO_B200_ERR_ARG;
    uint32_t total_keys = 0;
    for (int si = 0; si < 4; si++) {
        if (cfg->n_keys[si] && !seeds[si]) return MAYO_B200_ERR_ARG;
        total_keys += cfg->n_keys[si];
    }
    if (total_keys == 0) return MAYO_B200_ERR_ARG;
    mayo_b200_server *s = new (std::nothrow) mayo_b200_server();
    if (!s) return MAYO_B200_ERR_ARG;
    s->cfg = *cfg;
    s->L = L;
    s->dmem = static_cast<uint8_t *>(device_mem);
    s->hmem = static_cast<uint8_t *>(host_pinned);
    cudaError_t e = cudaGetDevice(&s->dev);
    for (int si = 0; si < 4 && e == cudaSuccess; si++) {
        s->seeds[si] = seeds[si];
        if (cfg->n_keys[si]) s->tab[si].init(key_rows(*cfg, si), cfg->n_keys[si]);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->x_ready, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->x_copied, cudaEventDisableTiming);
    s->slots.resize(cfg->inflight);
    for (uint32_t i = 0; i < cfg->inflight && e == cudaSuccess; i++) {
        Slot &sl = s->slots[i];
        e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ev, cudaEventDisableTiming);
        uint8_t *d = s->dmem + L.dev_slot0 + (size_t)i * L.dev_slot;
        uint8_t *h = s->hmem + (size_t)i * L.host_slot;
        sl.qmem = d + L.q_off;
        sl.d_in = d + L.din_off;
        sl.d_out = d + L.dout_off;
        sl.h_in = h + L.hin_off;
        sl.h_out = h + L.hout_off;
    }
    if (e != cudaSuccess) {
        delete s;
        return api_cuda_rc(e);
    }
    *out = s;
    return MAYO_B200_OK;
}

MAYO_B200_API int mayo_b200_server_destroy(mayo_b200_server *srv) {
    if (!srv) return MAYO_B200_ERR_ARG;
    int rc = MAYO_B200_OK;
    for (Slot &sl : srv->slots)
        if (sl.busy) {
            const cudaError_t e = cudaEventSynchronize(sl.ev);
            if (e != cudaSuccess) rc = api_cuda_rc(e);
        }
    delete srv;
    return rc;
}

MAYO_B200_API int mayo_b200_server_submit(mayo_b200_server *srv, const mayo_b200_serve_req *req, uint32_t n,
                                          uint64_t first_tag) {
    if (!srv || (n && !req)) return MAYO_B200_ERR_ARG;
    for (uint32_t i = 0; i < n; i++) {  // check everything before taking anything
        const mayo_b200_serve_req &r = req[i];
        const int si = set_index(r.set);
        if (si < 0 || srv->cfg.n_keys[si] == 0 || r.key_id >= srv->cfg.n_keys[si]) return MAYO_B200_ERR_ARG;
        if ((r.op != MAYO_B200_OP_SIGN && r.op != MAYO_B200_OP_VERIFY) || r.mlen > srv->cfg.max_msg) return MAYO_B200_ERR_ARG;
        if ((r.mlen && !r.msg) || !r.out || (r.op == MAYO_B200_OP_VERIFY && !r.sig)) return MAYO_B200_ERR_ARG;
    }
    for (uint32_t i = 0; i < n; i++) srv->waiting.push_back(Waiting{req[i], first_tag + i});
    return MAYO_B200_OK;
}

MAYO_B200_API int mayo_b200_server_progress(mayo_b200_server *srv, uint64_t *done_tags, uint32_t cap,
                                            uint32_t *n_done) {
    if (!srv || (cap && !done_tags)) return MAYO_B200_ERR_ARG;
    int rc = srv->collect();
    if (rc == MAYO_B200_OK) rc = srv->admit();
    uint32_t k = 0;
    while (k < cap && !srv->done.empty()) {
        done_tags[k++] = srv->done.front();
        srv->done.pop_front();
    }
    if (n_done) *n_done = k;
    return rc;
}

MAYO_B200_API int mayo_b200_server_drain(mayo_b200_server *srv) {
    if (!srv) return MAYO_B200_ERR_ARG;
    for (;;) {
        int rc = srv->collect();
        if (rc == MAYO_B200_OK) rc = srv->admit();
        if (rc != MAYO_B200_OK) return rc;
        bool busy = false;
        for (Slot &sl : srv->slots) busy |= sl.busy;
        if (!busy && srv->waiting.empty()) return MAYO_B200_OK;
        if (!busy) return MAYO_B200_ERR_FULL;  // requests wait but none can be admitted
        for (Slot &sl : srv->slots)
            if (sl.busy) {
                const cudaError_t e = cudaEventSynchronize(sl.ev);
                if (e != cudaSuccess) return api_cuda_rc(e);
                break;
            }
    }
}

MAYO_B200_API int mayo_b200_server_get_stats(const mayo_b200_server *srv, mayo_b200_server_stats *out) {
    if (!srv || !out) return MAYO_B200_ERR_ARG;
    *out = srv->st;
    out->waiting = srv->waiting.size();
    uint32_t busy = 0;
    for (const Slot &sl : srv->slots) busy += sl.busy;
    out->batches_in_flight = busy;
    out->key_misses = out->key_evictions = 0;
    for (int si = 0; si < 4; si++) {
        out->key_misses += srv->tab[si].misses;
        out->key_evictions += srv->tab[si].evictions;
    }
    return MAYO_B200_OK;
}

MAYO_B200_API int mayo_b200_server_preload(mayo_b200_server *srv, int set, const uint32_t *key_ids, uint32_t n) {
    const int si = set_index(set);
    if (!srv || si < 0 || srv->cfg.n_keys[si] == 0 || (n && !key_ids)) return MAYO_B200_ERR_ARG;
    for (const Slot &sl : srv->slots)
        if (sl.busy) return MAYO_B200_ERR_ARG;
    mayo_b200_key_table &t = srv->tab[si];
    if (!t.valid(key_ids, n)) return MAYO_B200_ERR_ARG;
    cudaStream_t s = srv->slots[0].st;
    std::vector<int32_t> rows;
    for (uint32_t c0 = 0; c0 < n; c0 += t.cap) {
        const uint32_t c = std::min(t.cap, n - c0);
        rows.resize(c);
        int rc = t.acquire(key_ids + c0, c, rows.data(), srv->miss_ids, srv->miss_slots);
        if (rc != MAYO_B200_OK) return rc;
        if (!srv->miss_ids.empty()) rc = srv->expand(si, s);
        t.release(rows.data(), c);
        if (rc != MAYO_B200_OK) return rc;
    }
    return api_cuda_rc(cudaStreamSynchronize(s));
}

MAYO_B200_API int mayo_b200_server_queue_error(mayo_b200_server *srv) {
    if (!srv) return -1;
    int err = MAYO_B200_QUEUE_OK;
    uint32_t ctrl[13 * 16];
    for (Slot &sl : srv->slots) {
        if (sl.busy && cudaEventSynchronize(sl.ev) != cudaSuccess) return -1;
        if (cudaMemcpy(ctrl, sl.qmem, sizeof(ctrl), cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
        for (int b = 0; b < 13 && !err; b++) err = (int)ctrl[b * 16 + 3];
    }
    return err;
}

MAYO_B200_API int mayo_b200_server_run_open_loop(mayo_b200_server *srv, const mayo_b200_serve_req *req,
                                                 const double *arrival_s, uint32_t n, double time_limit_s,
                                                 double *latency_s, double *wall_s) {
    if (!srv || (n && (!req || !arrival_s || !latency_s))) return MAYO_B200_ERR_ARG;
    for (uint32_t i = 1; i < n; i++)
        if (!(arrival_s[i] >= arrival_s[i - 1])) return MAYO_B200_ERR_ARG;
    if (!srv->waiting.empty() || !srv->done.empty()) return MAYO_B200_ERR_ARG;
    for (Slot &sl : srv->slots)
        if (sl.busy) return MAYO_B200_ERR_ARG;
    for (uint32_t i = 0; i < n; i++) latency_s[i] = NAN;
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    auto now_s = [&] { return std::chrono::duration<double>(clk::now() - t0).count(); };
    uint32_t next = 0, finished = 0;
    int rc = MAYO_B200_OK;
    while (finished < n && rc == MAYO_B200_OK) {
        const double now = now_s();
        // requests that have arrived join the waiting line (tag = index)
        uint32_t hi = next;
        while (hi < n && arrival_s[hi] <= now) hi++;
        if (hi > next) {
            rc = mayo_b200_server_submit(srv, req + next, hi - next, next);
            next = hi;
            if (rc != MAYO_B200_OK) break;
        }
        rc = srv->collect();
        if (rc == MAYO_B200_OK) rc = srv->admit();
        if (!srv->done.empty()) {
            const double t = now_s();
            while (!srv->done.empty()) {
                const uint64_t tag = srv->done.front();
                srv->done.pop_front();
                latency_s[tag] = t - arrival_s[tag];
                finished++;
            }
        }
        if (time_limit_s > 0 && now > time_limit_s) {
            // stop admitting: finish what is in flight, drop what waits
            srv->waiting.clear();
            for (Slot &sl : srv->slots)
                if (sl.busy && cudaEventSynchronize(sl.ev) != cudaSuccess) rc = MAYO_B200_ERR_CUDA;
            if (rc == MAYO_B200_OK) rc = srv->collect();
            const double t = now_s();
            while (!srv->done.empty()) {
                const uint64_t tag = srv->done.front();
                srv->done.pop_front();
                latency_s[tag] = t - arrival_s[tag];
            }
            break;
        }
    }
    if (wall_s) *wall_s = now_s();
    return rc;
}

}  // extern "C"
