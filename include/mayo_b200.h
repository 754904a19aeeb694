/*
 * mayo_b200.h -- C-ABI of the B200 batched MAYO engine (libmayo_b200.so).
 *
 * Drop-in boundary for SysuCrypto/cuMAYO's batched API.  Each mayo_b200_<name> below
 * replaces the reference host function crypto_sign_<name> declared in include/api.cuh and
 * implemented in src/api.cu of the reference project (line numbers cited per function),
 * with the same pool layout, the same copies, the same argument order and asynchronous,
 * stream-ordered semantics.  Differences, all additive:
 *   - the MAYO parameter set (1, 2, 3 or 5) is the first argument instead of the
 *     compile-time MAYO_VERSION, so all four sets live in one library;
 *   - every function returns a mayo_b200_status instead of void;
 *   - streams are passed as void* (a cudaStream_t; NULL = legacy default stream).
 * include/api.cuh in this repository restores the reference's exact C++ signatures on top.
 *
 * Pools are caller-allocated, pitched device buffers: row b belongs to instance b.  Host
 * buffers passed to the _HtD/_DtH helpers are tightly packed per instance, except where a
 * function says otherwise (as in the reference).  The library never allocates memory.
 */
#ifndef MAYO_B200_H
#define MAYO_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define MAYO_B200_API __attribute__((visibility("default")))
#else
#define MAYO_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define MAYO_B200_ABI_VERSION 1

typedef enum mayo_b200_status {
    MAYO_B200_OK = 0,
    MAYO_B200_ERR_SET = 1,  /* parameter set is not 1, 2, 3 or 5 */
    MAYO_B200_ERR_ARG = 2,  /* null pointer, pitch too small, message too long, ... */
    MAYO_B200_ERR_CUDA = 3, /* a CUDA call failed; see mayo_b200_last_cuda_error() */
    MAYO_B200_ERR_TOO_LARGE = 4, /* batch exceeds mayo_b200_sign_noalloc_max_batch(set) */
    MAYO_B200_ERR_FULL = 5, /* key table: not enough rows free of batches in flight */
} mayo_b200_status;

/* Byte sizes of one parameter set (reference include/params.h:10-92 and derived sizes). */
typedef struct mayo_b200_sizes {
    int32_t set, n, m, o, k, digest_bytes;
    uint64_t sk_bytes;      /* compact secret key (seed_sk) */
    uint64_t pk_bytes;      /* compact public key (seed_pk || P3) */
    uint64_t sig_bytes;     /* k*n/2 + sk_bytes */
    uint64_t esk_bytes;     /* seed_sk || O || P1 || L */
    uint64_t epk_bytes;     /* P1 || P2 || P3 */
    uint64_t p_bytes;       /* P1 || P2 */
    uint64_t scratch_bytes; /* per-row sign scratch: k*m*ceil(o/2) */
    /* minimum pool pitches for each reference entry point, for a message of mlen_hint */
    uint64_t pitch_keypair, pitch_expandsk, pitch_expandpk;
    uint64_t pitch_sign, pitch_sign_with_esk, pitch_verify;
} mayo_b200_sizes;

MAYO_B200_API int mayo_b200_abi_version(void);
/* Sizes of `set`; pitches are computed for messages of `mlen_hint` bytes. */
MAYO_B200_API int mayo_b200_get_sizes(int set, size_t mlen_hint, mayo_b200_sizes *out);
/* Replaces aes128_tables_init() (reference include/aes128_ctr.cuh:16, src/aes128_ctr.cu:69-72).
 * All tables are compile-time constants here; this only checks that the current device can
 * run sm_100a code.  Calling it is optional. */
MAYO_B200_API int mayo_b200_init(void);
MAYO_B200_API const char *mayo_b200_status_string(int status);
/* Last cudaError_t seen by this library on the calling thread (0 = none). */
MAYO_B200_API int mayo_b200_last_cuda_error(void);

/* ---- Failure injection for tests (no counterpart in the reference: its kernels have no
 * waits and no error path, src/sign.cu:244-474) ----
 * Makes one of the library's bounded device waits run out on purpose, so a test can check that
 * the error is reported, that nothing hangs or faults and that the results stay right.  The
 * setting belongs to the calling host thread and applies to its later calls until it is
 * changed; MAYO_B200_INJECT_NONE (the default) turns it off.
 *   MAYO_B200_INJECT_QUEUE_LOST_PUSH: in mayo_b200_queue_run every bucket with items gets one
 *     slot past its items that nothing publishes (as if a push were lost).  The CTA that takes
 *     that slot waits `spin_limit` sleeps, records MAYO_B200_QUEUE_ERR_TIMEOUT in the bucket's
 *     control words and ends; every real item is still processed.  (arg, spin unused.)
 *   MAYO_B200_INJECT_PRODUCT_STALL: in mayo_b200_sign_shared / _verify_shared the key loader of
 *     each tensor-core product CTA stops after `arg` chunks without telling the other warps,
 *     and the product's waits give up after `spin` polls (0 = the default bound).  The product
 *     then sets its status word to 1 and the per-instance engine computes every result.
 * MAYO_B200_ERR_ARG for an unknown kind. */
enum {
    MAYO_B200_INJECT_NONE = 0,
    MAYO_B200_INJECT_QUEUE_LOST_PUSH = 1,
    MAYO_B200_INJECT_PRODUCT_STALL = 2
};
MAYO_B200_API int mayo_b200_test_inject(int kind, uint32_t arg, uint32_t spin);

/* ---- keypair: reference src/api.cu:17-38 ---- */
/* Instance b uses seed_sk = SHAKE128(LE64(rand_index + 2b + 1)).  Row: sk @0, pk @A128(SK),
 * P1||P2 scratch @A128(SK)+A128(PK). */
MAYO_B200_API int mayo_b200_keypair(int set, uint8_t *pool, size_t pitch, size_t batch, void *stream,
                                    size_t rand_index);
MAYO_B200_API int mayo_b200_keypair_DtH(int set, uint8_t *pk, uint8_t *sk, const uint8_t *pool, size_t pitch,
                                        size_t batch, void *stream);
/* Extension: keypair from caller seeds already placed at row offset 0 (sk_bytes each),
 * same row layout as mayo_b200_keypair. */
MAYO_B200_API int mayo_b200_keypair_from_seed(int set, uint8_t *pool, size_t pitch, size_t batch, void *stream);

/* ---- expand-sk: src/api.cu:40-62 (row: sk @0 -> esk in place) ---- */
MAYO_B200_API int mayo_b200_expandsk_HtD(int set, const uint8_t *csk, uint8_t *pool, size_t pitch, size_t batch,
                                         void *stream);
MAYO_B200_API int mayo_b200_expandsk(int set, uint8_t *pool, size_t pitch, size_t batch, void *stream);
MAYO_B200_API int mayo_b200_expandsk_DtH(int set, uint8_t *esk, const uint8_t *pool, size_t pitch, size_t batch,
                                         void *stream);

/* ---- expand-pk: src/api.cu:64-85 (row: cpk @P-16 -> epk = P1||P2||P3 @0) ---- */
MAYO_B200_API int mayo_b200_expandpk_HtD(int set, const uint8_t *cpk, uint8_t *pool, size_t pitch, size_t batch,
                                         void *stream);
MAYO_B200_API int mayo_b200_expandpk(int set, uint8_t *pool, size_t pitch, size_t batch, void *stream);
MAYO_B200_API int mayo_b200_expandpk_DtH(int set, uint8_t *epk, const uint8_t *pool, size_t pitch, size_t batch,
                                         void *stream);

/* ---- sign on an expanded key: src/api.cu:88-114 ----
 * Row: esk @0, message @ESK, signature @ESK+mlen, scratch (k*m*ceil(o/2)) after it. */
MAYO_B200_API int mayo_b200_sign_HtD(int set, const uint8_t *esk, const uint8_t *msg, size_t mlen, uint8_t *pool,
                                     size_t pitch, size_t batch, void *stream);
MAYO_B200_API int mayo_b200_sign(int set, uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *stream);
MAYO_B200_API int mayo_b200_sign_DtH(int set, uint8_t *sig, const uint8_t *pool, size_t mlen, size_t pitch,
                                     size_t batch, void *stream);

/* ---- sign from a compact key: src/api.cu:116-144 ----
 * Row: sk @0 (expanded in place), message @A(ESK), signature @A(ESK)+A(mlen), scratch after
 * A(SIG).  A(x) = x rounded up to 128. */
MAYO_B200_API int mayo_b200_signWithesk_HtD(int set, const uint8_t *csk, const uint8_t *msg, size_t mlen,
                                            uint8_t *pool, size_t pitch, size_t batch, void *stream);
MAYO_B200_API int mayo_b200_signWithesk(int set, uint8_t *pool, size_t mlen, size_t pitch, size_t batch,
                                        void *stream);
MAYO_B200_API int mayo_b200_signWithesk_DtH(int set, uint8_t *sig, const uint8_t *pool, size_t mlen, size_t pitch,
                                            size_t batch, void *stream);

/* ---- verify on an expanded key: src/api.cu:146-178 ----
 * Row: epk @0, message @A(EPK), signature @A(EPK)+A(mlen), result byte @+A(SIG)
 * (0 = accept, 1 = reject).  _HtD reads epk and sig with 128-byte-aligned host strides. */
MAYO_B200_API int mayo_b200_verify_HtD(int set, const uint8_t *epk, const uint8_t *msg, const uint8_t *sig,
                                       size_t mlen, uint8_t *pool, size_t pitch, size_t batch, void *stream);
MAYO_B200_API int mayo_b200_verify(int set, uint8_t *pool, size_t mlen, size_t pitch, size_t batch, void *stream);
MAYO_B200_API int mayo_b200_verify_DtH(int set, uint8_t *result, size_t mlen, const uint8_t *pool, size_t pitch,
                                       size_t batch, void *stream);

/* ---- verify from a compact key: src/api.cu:180-218 (cpk lands @P-16, then expanded) ---- */
MAYO_B200_API int mayo_b200_verifyWithepk_HtD(int set, const uint8_t *cpk, const uint8_t *msg, const uint8_t *sig,
                                              size_t mlen, uint8_t *pool, size_t pitch, size_t batch,
                                              void *stream);
MAYO_B200_API int mayo_b200_verifyWithepk(int set, uint8_t *pool, size_t mlen, size_t pitch, size_t batch,
                                          void *stream);
MAYO_B200_API int mayo_b200_verifyWithepk_DtH(int set, uint8_t *result, size_t mlen, const uint8_t *pool,
                                              size_t pitch, size_t batch, void *stream);

/* ---- Extension (no counterpart in the reference API): batched sign/verify over explicit
 * operand arrays instead of a pool.  Keys may be shared by the whole batch (stride 0, e.g. a
 * resident expanded key) and messages may have per-instance lengths (the reference takes one
 * Mlen per call, include/api.cuh:25-47).  All pointers are device pointers.
 *   message i = msgs + msg_off[i], msg_len[i] bytes    when msg_off != NULL (device arrays)
 *             = msgs + i * msg_stride, mlen bytes      otherwise
 * Results are byte-identical to the pool API on the same inputs. */
/* Per-instance workspace bytes of mayo_b200_sign_many (digest, salt, t, V||r); 0 for a bad set. */
MAYO_B200_API size_t mayo_b200_sign_ws_bytes(int set);
MAYO_B200_API int mayo_b200_sign_many(int set, const uint8_t *esk, size_t esk_stride, const uint8_t *msgs,
                                      const uint64_t *msg_off, const uint32_t *msg_len, size_t msg_stride,
                                      size_t mlen, uint8_t *sig, size_t sig_stride, uint8_t *ws, size_t batch,
                                      void *stream);
MAYO_B200_API int mayo_b200_verify_many(int set, const uint8_t *epk, size_t epk_stride, const uint8_t *msgs,
                                        const uint64_t *msg_off, const uint32_t *msg_len, size_t msg_stride,
                                        size_t mlen, const uint8_t *sig, size_t sig_stride, uint8_t *result,
                                        size_t batch, void *stream);

/* ---- Extension (no counterpart in the reference): one key for the whole batch ----
 * Same results as mayo_b200_sign_many / _verify_many with esk_stride / epk_stride 0, for batches
 * signed or verified under a single expanded key.  The key's products with every instance's
 * vectors (T = P1 V and M = V L for sign, T = P s for verify) run as one binary matrix product
 * over the batch on the tensor cores (each GF(16) entry as its 4x4 bit matrix, sums mod 2);
 * the rest of each operation runs per instance as in _many.  `ws` is device memory of
 * mayo_b200_*_shared_ws_bytes(set, batch) bytes, 16-byte aligned; its first 4 bytes hold a
 * status word after the call (0 = the tensor-core product ran; 1 = a bounded wait in it ran
 * out and the per-instance engine produced the results instead). */
MAYO_B200_API size_t mayo_b200_sign_shared_ws_bytes(int set, size_t batch);
MAYO_B200_API int mayo_b200_sign_shared(int set, const uint8_t *esk, const uint8_t *msgs, const uint64_t *msg_off,
                                        const uint32_t *msg_len, size_t msg_stride, size_t mlen, uint8_t *sig,
                                        size_t sig_stride, uint8_t *ws, size_t batch, void *stream);
MAYO_B200_API size_t mayo_b200_verify_shared_ws_bytes(int set, size_t batch);
/* Profiling aid: while enabled (nonzero), each mayo_b200_sign_shared / _verify_shared call made
 * from this host thread records CUDA events between its kernels on its stream (enable before any
 * stream capture; it creates the events); mayo_b200_shared_timing_read waits for the last such
 * call and gives the milliseconds of its kernels: [0] hash, [1] key tiles, [2] tensor-core
 * product, [3] per-instance tail, [4] fix-up.  MAYO_B200_ERR_ARG if no call was recorded. */
MAYO_B200_API int mayo_b200_shared_timing(int enable);
/* Launch shape of the shared-key calls of one parameter set, process-wide (set it before the
 * calls it should apply to; calls already issued keep theirs).  hash_threads: threads per CTA
 * of the thread-per-instance hash kernels (a multiple of 32, 32..1024; 0 = 64); tail_instances:
 * signatures per CTA of the sign tail (1, 2 or 4; 0 = 4 for MAYO_2, 2 for MAYO_1, else 1; with
 * more than one the instances' elimination columns are interleaved over the CTA's warps);
 * product_ctas: CTAs per tile of the tensor-core key product (1, or 2: a cluster of two CTAs on
 * two SMs running cta_group::2 MMAs, each SM streaming half of every key tile; 0 = 2).  The
 * defaults hold until a shape is set.  Results do not depend on the shape;
 * cumayo_b200.autotune times the candidates.  MAYO_B200_ERR_ARG for a shape out of range or
 * one whose CTA would not fit in shared memory; shape NULL = the defaults. */
typedef struct mayo_b200_shared_shape {
    uint32_t hash_threads, tail_instances, product_ctas;
} mayo_b200_shared_shape;
MAYO_B200_API int mayo_b200_shared_set_shape(int set, const mayo_b200_shared_shape *shape);
MAYO_B200_API int mayo_b200_shared_get_shape(int set, mayo_b200_shared_shape *shape);
MAYO_B200_API int mayo_b200_shared_timing_read(float *ms);
MAYO_B200_API int mayo_b200_verify_shared(int set, const uint8_t *epk, const uint8_t *msgs, const uint64_t *msg_off,
                                          const uint32_t *msg_len, size_t msg_stride, size_t mlen, const uint8_t *sig,
                                          size_t sig_stride, uint8_t *result, uint8_t *ws, size_t batch,
                                          void *stream);

/* ---- Extension (no counterpart in the reference): persistent work queue ----
 * A device queue of keypair / sign / verify items of all four parameter sets.  The mixed item
 * array is partitioned on the device (stably) into 12 buckets, one per (set, op), each drained by
 * its own persistent kernel shaped like the batched kernel for that (set, op) (their CTAs need
 * 35-81 KB of shared memory, so one kernel for all would hold every set to the residency of the
 * largest).  The kernels are launched on forked streams, so they share the SMs and fill each
 * other's tails.  A sign attempt with a singular system is re-enqueued with the next attempt
 * counter instead of being retried in place.  Every wait inside the kernels is bounded; an
 * overflowing bucket, a wait that runs out or an item with a missing operand ends with an error
 * code in the queue's control words instead of hanging or touching memory out of range.
 * Results are byte-identical to the batched calls.
 *
 * Operands per parameter set (device pointers; an op's pointers may be NULL if no item uses it):
 *   keypair  instance i < kp_count: seed kp_seed + i*sk_bytes -> pk at kp_pk + i*pk_bytes
 *   sign     instance i < sg_count: key sg_esk + K*esk_bytes with K = sg_key[i] (or i % sg_nkeys
 *            when sg_key is NULL); message sg_msg + sg_msg_off[i] of sg_msg_len[i] bytes (or
 *            sg_msg + i*sg_mlen of sg_mlen bytes when they are NULL) -> signature sg_sig + i*sig_bytes
 *   verify   instance i < vf_count: key vf_epk + K*epk_bytes likewise; message likewise;
 *            signature vf_sig + i*sig_bytes -> result byte vf_res[i] (0 accept, 1 reject)
 * Bucket b = 3 * (set index: MAYO_1, 2, 3, 5 -> 0..3) + op.  Queue memory
 * (mayo_b200_queue_mem_bytes bytes, device, caller-allocated): control words at offset 0, 16
 * uint32 per bucket (bucket b at word 16*b): [0] items taken, [1] items published, [2] items
 * finished, [3] error, [4] re-enqueued signs; block 12 counts items with an invalid op in [0]; a
 * bucket whose op has no operands counts its dropped items in [0].  Then the slots (capacity per
 * bucket), then the keypair buckets' per-CTA scratch. */
enum { MAYO_B200_OP_KEYPAIR = 0, MAYO_B200_OP_SIGN = 1, MAYO_B200_OP_VERIFY = 2 };
enum {
    MAYO_B200_QUEUE_OK = 0,
    MAYO_B200_QUEUE_ERR_FULL = 1,    /* more re-enqueued signs than slots */
    MAYO_B200_QUEUE_ERR_TIMEOUT = 2, /* a wait ran past spin_limit */
    MAYO_B200_QUEUE_ERR_OPERAND = 3  /* an item's instance, key index or operand is missing (item skipped) */
};
typedef struct mayo_b200_queue_ops {
    const uint8_t *kp_seed;
    uint8_t *kp_pk;
    uint32_t kp_count;
    const uint8_t *sg_esk;
    uint32_t sg_nkeys;
    const uint32_t *sg_key;
    const uint8_t *sg_msg;
    const uint64_t *sg_msg_off;
    const uint32_t *sg_msg_len;
    uint32_t sg_mlen;
    uint8_t *sg_sig;
    uint32_t sg_count;
    const uint8_t *vf_epk;
    uint32_t vf_nkeys;
    const uint32_t *vf_key;
    const uint8_t *vf_msg;
    const uint64_t *vf_msg_off;
    const uint32_t *vf_msg_len;
    uint32_t vf_mlen;
    const uint8_t *vf_sig;
    uint8_t *vf_res;
    uint32_t vf_count;
} mayo_b200_queue_ops;
/* Launch shape.  sms: SMs the queue memory was sized for (0 = all SMs of the device); per
 * bucket, ctas_per_sm (0 = the most that fit, at most mayo_b200_queue_ctas_per_sm) and the order
 * in which the bucket kernels are launched (launch_order must be a permutation of 0..11, else the
 * default: the buckets with the longest items first). */
typedef struct mayo_b200_queue_shape {
    uint32_t sms;
    uint8_t ctas_per_sm[12];
    uint8_t launch_order[12];
} mayo_b200_queue_shape;
/* Work item: op (MAYO_B200_OP_*), parameter set (1, 2, 3, 5), instance index < 2^20. */
static inline uint32_t mayo_b200_queue_item(int op, int set, uint32_t instance) {
    const uint32_t si = set == 1 ? 0u : set == 2 ? 1u : set == 3 ? 2u : 3u;
    return ((uint32_t)op << 30) | (si << 28) | (instance & 0xFFFFFu);
}
/* Device bytes of queue memory for `capacity` slots per bucket on `sms` SMs (0 = all); 0 on error. */
MAYO_B200_API size_t mayo_b200_queue_mem_bytes(uint32_t capacity, uint32_t sms);
/* Resident CTAs per SM of the queue kernel for (set, op) on the current device (0 on error). */
MAYO_B200_API int mayo_b200_queue_ctas_per_sm(int set, int op);
/* Reset the queue to items[0..n) (device array; when n_device is not NULL the count is
 * min(*n_device, n), read on the device, so a captured graph can be replayed with a varying
 * count) and run it to completion on `stream`.  capacity >= n; room beyond a bucket's items
 * holds its re-enqueued signs (n + n/8 + 64 is ample).  shape NULL = defaults.  Asynchronous;
 * runs on different streams (with their own queue memory) overlap.  The first call from a host
 * thread for a given stream creates the streams the bucket kernels fork onto; after that the
 * call is graph-capturable (no allocation, no host synchronisation).  spin_limit 0 = default. */
MAYO_B200_API int mayo_b200_queue_run(const mayo_b200_queue_ops ops[4], const uint32_t *items, uint32_t n,
                                      const uint32_t *n_device, void *queue_mem, uint32_t capacity,
                                      const mayo_b200_queue_shape *shape, uint32_t spin_limit, void *stream);

/* ---- Extension (no counterpart in the reference): serving-batch staging (host code) ----
 * A serving loop admits sign / verify requests whose messages, signatures and result buffers
 * live in the caller's host memory.  mayo_b200_serve_pack copies one batch of them, in one pass,
 * into a staging buffer laid out for the work queue (items, then per (set, op) group its key
 * slots, message lengths, messages at a max_msg stride and, for verifies, signatures at the
 * set's stride, every section 16-byte aligned); after the queue has run on the device copy of
 * that buffer, mayo_b200_serve_unpack copies each request's signature (sig_bytes of its set) or
 * verify result byte (0 accept, 1 reject) from the output staging buffer to its `out`.  The
 * layout gives each group's offsets, from which the caller fills mayo_b200_queue_ops.  Both
 * are plain host code (no CUDA calls). */
typedef struct mayo_b200_serve_req {
    const uint8_t *msg; /* mlen bytes */
    const uint8_t *sig; /* verify: sig_bytes of the set; unused for sign */
    uint8_t *out;       /* sign: sig_bytes of the set; verify: 1 byte */
    uint32_t mlen;
    uint32_t key_id;    /* the caller's key id (not read here) */
    uint32_t key_slot;  /* row of the set's key table (esk for sign, epk for verify) */
    uint8_t op;         /* MAYO_B200_OP_SIGN or MAYO_B200_OP_VERIFY */
    uint8_t set;        /* 1, 2, 3, 5 */
    uint8_t pad[2];
} mayo_b200_serve_req;
typedef struct mayo_b200_serve_group {
    uint32_t count; /* 0: the group is absent */
    uint32_t set, op, pad;
    uint64_t key_off, len_off, msg_off, sig_off; /* input staging offsets */
    uint64_t out_off;                            /* output staging offset */
} mayo_b200_serve_group;
typedef struct mayo_b200_serve_layout {
    uint32_t n, max_msg;
    uint64_t in_bytes, out_bytes;
    mayo_b200_serve_group group[8]; /* group 2*(set index) + (op == VERIFY) */
} mayo_b200_serve_layout;
/* Bytes of input / output staging a batch of n requests needs at most. */
MAYO_B200_API size_t mayo_b200_serve_in_bytes(uint32_t n, uint32_t max_msg);
MAYO_B200_API size_t mayo_b200_serve_out_bytes(uint32_t n);
/* MAYO_B200_ERR_ARG for an op other than sign / verify, an unknown set, mlen > max_msg, a NULL
 * message with mlen > 0, a NULL signature or output, or staging smaller than the layout. */
MAYO_B200_API int mayo_b200_serve_pack(const mayo_b200_serve_req *req, uint32_t n, uint32_t max_msg,
                                       uint8_t *stage_in, size_t in_capacity, size_t out_capacity,
                                       mayo_b200_serve_layout *layout);
MAYO_B200_API int mayo_b200_serve_unpack(const mayo_b200_serve_req *req, uint32_t n,
                                         const mayo_b200_serve_layout *layout, const uint8_t *stage_out);

/* ---- Extension (no counterpart in the reference): the serving loop (host code, C++) ----
 * Continuous batching of sign / verify requests (mayo_b200_serve_req) over the work queue, with
 * the expanded keys resident on the GPU.  Keys are registered per parameter set as their
 * sk_bytes seeds (key id = row of the seed array; the caller keeps the seeds alive for the
 * server's life) and expanded (keypair -> esk, epk) on first use into that set's key table of
 * `key_slots` rows; a full table evicts its least recently used rows that no batch in flight
 * uses.  Up to `inflight` batches are on the GPU at once, each with its own stream, queue memory
 * and staging.  The caller provides all memory: mayo_b200_server_device_bytes of device memory
 * and mayo_b200_server_host_bytes of pinned host memory (both 256-byte aligned); the server
 * creates CUDA streams and events only.  One host thread at a time may call a server.
 *
 * Key table (host only, usable on its own): key id -> row, least-recently-used eviction,
 * pinning.  acquire maps a batch's key ids to rows (slots[i] for key_ids[i]), loads the missing
 * ids into unpinned rows the batch does not use (empty rows first, then the least recently used)
 * and reports them (distinct ids and their rows), and pins every distinct row the batch uses
 * once; MAYO_B200_ERR_FULL (and no change) when too few rows are free; MAYO_B200_ERR_ARG for an
 * unknown id.  release unpins every distinct row among the given slots once (the slots one
 * acquire returned).  can_load: 1 if acquire would succeed, 0 if not, -1 on bad arguments. */
typedef struct mayo_b200_key_table mayo_b200_key_table;
typedef struct mayo_b200_key_table_stats {
    uint32_t capacity, n_keys, pinned_slots, resident_keys;
    uint64_t misses, evictions;
} mayo_b200_key_table_stats;
MAYO_B200_API mayo_b200_key_table *mayo_b200_key_table_create(uint32_t capacity, uint32_t n_keys);
MAYO_B200_API void mayo_b200_key_table_destroy(mayo_b200_key_table *t);
MAYO_B200_API int mayo_b200_key_table_acquire(mayo_b200_key_table *t, const uint32_t *key_ids, uint32_t n,
                                              int32_t *slots, uint32_t *miss_ids, int32_t *miss_slots,
                                              uint32_t *n_miss);
MAYO_B200_API int mayo_b200_key_table_release(mayo_b200_key_table *t, const int32_t *slots, uint32_t n);
MAYO_B200_API int mayo_b200_key_table_can_load(mayo_b200_key_table *t, const uint32_t *key_ids, uint32_t n);
MAYO_B200_API int mayo_b200_key_table_info(const mayo_b200_key_table *t, mayo_b200_key_table_stats *out);
MAYO_B200_API int32_t mayo_b200_key_table_slot_of(const mayo_b200_key_table *t, uint32_t key_id); /* -1: not resident */
MAYO_B200_API int32_t mayo_b200_key_table_pins(const mayo_b200_key_table *t, uint32_t slot);

typedef struct mayo_b200_server mayo_b200_server;
typedef struct mayo_b200_server_config {
    uint32_t max_batch;    /* requests per batch (<= 2^20) */
    uint32_t inflight;     /* batches on the GPU at once */
    uint32_t max_msg;      /* longest message, bytes */
    uint32_t expand_chunk; /* keys per expansion launch (scratch rows); 0 = 256 */
    uint32_t n_keys[4];    /* registered keys of MAYO_1, 2, 3, 5 */
    uint32_t key_slots[4]; /* resident rows per set (0 or >= n_keys: every key) */
} mayo_b200_server_config;
typedef struct mayo_b200_server_stats {
    uint64_t batches, requests_admitted, requests_done, max_batch_seen, kernel_launches, keys_expanded;
    uint64_t key_misses, key_evictions, waiting;
    uint32_t batches_in_flight, pad;
} mayo_b200_server_stats;
/* Memory the caller provides for `cfg` on the current device (0 on a bad configuration). */
MAYO_B200_API size_t mayo_b200_server_device_bytes(const mayo_b200_server_config *cfg);
MAYO_B200_API size_t mayo_b200_server_host_bytes(const mayo_b200_server_config *cfg);
/* seeds[i]: n_keys[i] * sk_bytes of set i (NULL where n_keys[i] is 0), host memory. */
MAYO_B200_API int mayo_b200_server_create(const mayo_b200_server_config *cfg, const uint8_t *const seeds[4],
                                          void *device_mem, size_t device_bytes, void *host_pinned,
                                          size_t host_bytes, mayo_b200_server **out);
/* Waits for the batches in flight, then frees the server (not the caller's memory). */
MAYO_B200_API int mayo_b200_server_destroy(mayo_b200_server *srv);
/* Appends n requests to the waiting line; request i gets tag first_tag + i.  The records are
 * copied; the memory they point to (message, signature, out) must stay valid until the request
 * is reported done.  Checks every request first (MAYO_B200_ERR_ARG: unknown set or key id, op
 * other than sign / verify, mlen > max_msg, missing pointer) and takes none on error. */
MAYO_B200_API int mayo_b200_server_submit(mayo_b200_server *srv, const mayo_b200_serve_req *req, uint32_t n,
                                          uint64_t first_tag);
/* One non-blocking pass: batches that finished are unpacked into their requests' `out` and their
 * rows released; free batch slots admit the longest prefix of the waiting line (<= max_batch)
 * whose keys fit; up to `cap` tags of finished requests go to done_tags (*n_done of them; the
 * rest wait for the next call). */
MAYO_B200_API int mayo_b200_server_progress(mayo_b200_server *srv, uint64_t *done_tags, uint32_t cap,
                                            uint32_t *n_done);
/* Runs progress until nothing waits and nothing is in flight (tags stay for progress to
 * report); MAYO_B200_ERR_FULL if requests wait whose keys can never fit the tables. */
MAYO_B200_API int mayo_b200_server_drain(mayo_b200_server *srv);
MAYO_B200_API int mayo_b200_server_get_stats(const mayo_b200_server *srv, mayo_b200_server_stats *out);
/* Makes keys resident ahead of their requests (expands the missing ones; waits until done).
 * Only on an idle server (no batch in flight); MAYO_B200_ERR_ARG for an unknown set or key id. */
MAYO_B200_API int mayo_b200_server_preload(mayo_b200_server *srv, int set, const uint32_t *key_ids, uint32_t n);
/* First queue error code (MAYO_B200_QUEUE_*) in the slots' last runs; waits for them; -1 on a
 * CUDA error. */
MAYO_B200_API int mayo_b200_server_queue_error(mayo_b200_server *srv);
/* Open-loop run on an idle server: request i joins the waiting line once arrival_s[i] seconds
 * (sorted) have passed since the call began, and latency_s[i] = the time its result was unpacked
 * minus arrival_s[i] (NaN if not served).  With time_limit_s > 0, no request is admitted after
 * that time (the batches in flight finish).  *wall_s = the run's duration. */
MAYO_B200_API int mayo_b200_server_run_open_loop(mayo_b200_server *srv, const mayo_b200_serve_req *req,
                                                 const double *arrival_s, uint32_t n, double time_limit_s,
                                                 double *latency_s, double *wall_s);

/* ---- Sign without caller workspace.  No counterpart in the reference API. ----
 * For callers that cannot allocate device memory (a service whose device-memory budget is
 * fixed at start-up, or a host program that owns the allocator and forbids a plug-in library
 * to call cudaMalloc) and so cannot provide the workspace mayo_b200_sign_many needs.  Same
 * arguments and results as mayo_b200_sign_many minus `ws`: the workspace is a 4 MiB array
 * compiled into the library, held by every GPU that loads the library until exit.  Batches
 * above mayo_b200_sign_noalloc_max_batch(set) return MAYO_B200_ERR_TOO_LARGE.  The first call
 * on a device looks up the array's address on that device and keeps it for the device's
 * current CUDA context; a call in a new context of the device (after cudaDeviceReset, for
 * instance) looks it up again.  Make the first call before any stream capture: the look-up is
 * not a stream operation, and a first call made while a stream is being captured may fail with
 * MAYO_B200_ERR_CUDA.  All calls share the array, so calls whose GPU work may overlap
 * (different streams without ordering) race and must not be issued.  Allocates nothing. */
MAYO_B200_API size_t mayo_b200_sign_noalloc_max_batch(int set);
MAYO_B200_API int mayo_b200_sign_many_noalloc(int set, const uint8_t *esk, size_t esk_stride, const uint8_t *msgs,
                                              const uint64_t *msg_off, const uint32_t *msg_len, size_t msg_stride,
                                              size_t mlen, uint8_t *sig, size_t sig_stride, size_t batch,
                                              void *stream);

#ifdef __cplusplus
}
#endif
#endif /* MAYO_B200_H */
