#!/usr/bin/env python3
"""Throughput benchmark of the B200 MAYO engine (and of the reference, --impl reference).

Default workload (one GPU): MAYO_2 shared-key sign and verify, batch 65,536.  One seeded
keypair is expanded once and stays resident in HBM; every instance signs its own message
(length uniform in [32, 1024] bytes, bytes from a seeded ChaCha20 stream) and the batch of
signatures is then verified.  A step = sign the batch + verify the batch; `value` counts
both operations.  Other workloads (--workload): c1 = MAYO_1 keypair -> sign -> verify, batch
1,024, distinct keys; c3-3 / c3-5 = MAYO_3 / MAYO_5 distinct-key verify, batch 16,384, 10%
corrupted signatures.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2]

Prints one JSON line (rank 0).  Under torchrun each rank runs the same per-GPU workload on
its own GPU (weak scaling, no collective on the data path); the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "sign/s and verify/s per B200 (MAYO_1/2/3/5), byte-exact; serving p50/p99 vs plain"
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def _hbm_peak() -> tuple[float, str]:
    """Measured copy bandwidth of this GPU pool (MEASURED_PEAKS.json), else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


HBM_PEAK_GBS, HBM_PEAK_SRC = _hbm_peak()


def _bf16_peak() -> tuple[float, str]:
    """Measured dense bf16 GEMM throughput (burst), TFLOP/s, else the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except (OSError, ValueError, KeyError):
        return 1590.0, "fallback"


BF16_PEAK_TFLOPS, BF16_PEAK_SRC = _bf16_peak()
LOP3_LANE_OPS_PER_CLK_SM = 64  # measured on this pool's B200 (profiles/int_pipes_b200.md)
A128 = lambda x: (x + 127) // 128 * 128  # noqa: E731
KERNEL_ROOF_DEF = {
    "alu": "algorithmic ops = 0.5 x the GF(16) MACs the kernel owns (16 LOP3 per 32 MACs) / kernel time; "
           "peak = measured LOP3 issue rate 64 lane-ops/clk/SM x 148 SMs x median SM clock",
    "tensor": "algorithmic ops = 2 x 16 binary MACs per GF(16) MAC of the key products / kernel time; "
              "peak = 2 x measured dense bf16 GEMM (int8 rate of the tensor cores)",
    "hbm": "algorithmic bytes read + written / kernel time; peak = measured copy bandwidth",
}
# DRAM bytes per instance (dram__bytes_read.sum + dram__bytes_write.sum of one launch / its
# instances) from ncu captures of the MAYO_2 shared-key kernels at 16,384 instances (the sign
# tail with four signatures per CTA: profiles/sign_tail_mayo2_shared_b16384.md; the products on
# CTA pairs: profiles/product_gemm_mayo2_shared_b16384.md; the verify tail from an earlier
# capture of the same command); the traffic grows in proportion to the instances, so a launch's
# traffic is this x its batch.
KERNEL_TRAFFIC_PER_INST = {2: {"sign.tail": (174.092544e6 + 4.883456e6) / 16384, "verify.tail": 177.242624e6 / 16384,
                               "sign.product": (11.437568e6 + 118.18368e6) / 16384,
                               "verify.product": (10.445568e6 + 119.318528e6) / 16384}}
# The same for verify_kernel<SET> on distinct keys (one capture of 4,096 instances per set,
# profiles/verify_distinct_mayo3_mayo5_b4096.md): the instance's EPK is read once.
VERIFY_TRAFFIC_PER_INST = {3: (1.557413e9 + 4.978176e6) / 4096, 5: (3.478466e9 + 4.699392e6) / 4096}

# ---------------------------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------------------------
WORKLOADS = {
    "c2": dict(set=2, batch=65536, kind="shared_sign_verify", mlen=(32, 1024)),
    "c1": dict(set=1, batch=1024, kind="keypair_sign_verify", mlen=(32, 32)),
    # the same keypair -> sign -> verify batch for the other sets (per-set figures)
    "c1-2": dict(set=2, batch=1024, kind="keypair_sign_verify", mlen=(32, 32)),
    "c1-3": dict(set=3, batch=1024, kind="keypair_sign_verify", mlen=(32, 32)),
    "c1-5": dict(set=5, batch=1024, kind="keypair_sign_verify", mlen=(32, 32)),
    "c3-3": dict(set=3, batch=16384, kind="distinct_verify", mlen=(32, 32)),
    "c3-5": dict(set=5, batch=16384, kind="distinct_verify", mlen=(32, 32)),
    "c4": dict(set=0, batch=262144, kind="mixed_queue", mlen=(32, 32)),
    "c5": dict(set=0, batch=16384, kind="serving", mlen=(32, 256)),
}

PARAMS = {1: (86, 78, 8, 10), 2: (81, 64, 17, 4), 3: (118, 108, 10, 11), 5: (154, 142, 12, 12)}


def mac_counts(s: int) -> dict:
    """Algorithmic GF(16) multiply-accumulates per operation (coordinate x scalar)."""
    n, m, o, k = PARAMS[s]
    v = n - o
    e1, e2, e3 = v * (v + 1) // 2, v * o, o * (o + 1) // 2
    sign = k * m * e1 + m * k * k * v + k * m * v * o + m * m * (k * o + 1)
    verify = k * m * (e1 + e2 + e3) + m * k * k * n
    keypair = o * m * (e1 + e2) + m * o * o * v
    return dict(sign=sign, verify=verify, keypair=keypair)


def chacha(key: bytes, n: int) -> np.ndarray:
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms
    enc = Cipher(algorithms.ChaCha20(key, b"\0" * 16), mode=None).encryptor()
    return np.frombuffer(enc.update(b"\0" * n), dtype=np.uint8)


def make_messages(seed: int, batch: int, lo: int, hi: int):
    """Seeded ChaCha20 stream: lengths uniform in [lo, hi], then message bytes."""
    key = (b"mayo-b200-bench-%d" % seed).ljust(32, b"\0")[:32]
    raw = chacha(key, 4 * batch)
    lens = (lo + (raw.view(np.uint32) % np.uint32(hi - lo + 1))).astype(np.uint32)
    offs = np.zeros(batch, np.uint64)
    offs[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
    total = int(lens.sum())
    body = chacha(key[::-1], total + 16)[16:16 + total].copy()
    return body, offs, lens


def seeds_for(seed: int, batch: int, skb: int) -> np.ndarray:
    key = (b"mayo-b200-keys-%d" % seed).ljust(32, b"\0")[:32]
    return chacha(key, batch * skb).reshape(batch, skb).copy()


# ---------------------------------------------------------------------------------------------
# distributed plumbing (one process per GPU)
# ---------------------------------------------------------------------------------------------
class Dist:
    """One process per GPU (torchrun's env); NCCL, or `gloo` (MAYO_BENCH_DIST_BACKEND) for the
    CPU tests of the multi-rank plumbing.  No collective touches the data path: ranks meet only
    at the barriers around the timed region and for the max of their times."""

    def __init__(self):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = os.environ.get("MAYO_BENCH_DIST_BACKEND", "nccl")
        self.pg = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist
            dist.init_process_group(self.backend, timeout=datetime.timedelta(seconds=120))
            self.pg = dist

    def barrier(self):
        if self.pg:
            if self.backend == "nccl":
                import torch
                self.pg.barrier(device_ids=[self.local])
                torch.cuda.synchronize()
            else:
                self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device="cuda" if self.backend == "nccl" else "cpu")
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


def weak_value(ops_per_rank_step: float, world: int, ms_per_step_max: float) -> float:
    """Whole-job throughput under weak scaling: every rank processes its own batch, so the job
    did world x the per-rank operations in the slowest rank's time."""
    return ops_per_rank_step * world / (ms_per_step_max / 1e3)


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.path = os.path.join("/tmp", f"mayo_clocks_{os.getpid()}.csv")

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------------------------------------
# our engine
# ---------------------------------------------------------------------------------------------
def run_ours(args, dist: Dist):
    import torch

    import cumayo_b200 as M

    wl = WORKLOADS[args.workload]
    s, batch = wl["set"], args.batch or wl["batch"]
    m = M.Mayo(s if s else 1)
    z = m.sizes
    dev = torch.device("cuda", dist.local)
    torch.cuda.set_device(dev)
    st = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device=dev)
    launches_per_step = 0
    seed = 1 + dist.rank
    plain_fn = None
    kernel_profile = None
    e2e_run = None
    device_streamed_step = None
    plain_api = "per-(set, op) batched launches: keypair_from_seed, sign_many, verify_many"
    plain_check = None
    gpu_outputs = None  # host copies of the last end-to-end step's outputs, for the oracle check

    if wl["kind"] == "shared_sign_verify":
        # one resident expanded key (esk, epk), messages of per-instance length
        sk_seed = seeds_for(seed, 1, z.sk_bytes)
        kp, kpitch = m.alloc_pool("keypair", 1)
        kp[: z.sk_bytes].copy_(torch.from_numpy(sk_seed[0]))
        m.crypto_sign_keypair_from_seed(kp, kpitch, 1, st)
        esk = torch.zeros(z.esk_bytes, dtype=torch.uint8, device=dev)
        esk[: z.sk_bytes].copy_(kp[: z.sk_bytes])
        m.crypto_sign_expandsk(esk, z.esk_bytes, 1, st)
        epk = torch.zeros(z.epk_bytes, dtype=torch.uint8, device=dev)
        pk_off = A128(z.sk_bytes)
        epk[z.p_bytes - 16: z.p_bytes - 16 + z.pk_bytes].copy_(kp[pk_off: pk_off + z.pk_bytes])
        m.crypto_sign_expandpk(epk, z.epk_bytes, 1, st)
        body, offs, lens = make_messages(seed, batch, *wl["mlen"])
        h_msgs = torch.from_numpy(body).pin_memory()
        h_offs = torch.from_numpy(offs.view(np.int64)).pin_memory()
        h_lens = torch.from_numpy(lens.view(np.int32)).pin_memory()
        d_msgs = h_msgs.to(dev)
        d_offs = h_offs.to(dev)
        d_lens = h_lens.to(dev)
        sig = torch.zeros(batch * z.sig_bytes, dtype=torch.uint8, device=dev)
        # one workspace serves both calls (verify runs after sign on the same stream)
        ws = torch.zeros(max(m.sign_shared_ws_bytes(batch), m.verify_shared_ws_bytes(batch)), dtype=torch.uint8,
                         device=dev)
        res = torch.zeros(batch, dtype=torch.uint8, device=dev)
        h_sig = torch.zeros(batch * z.sig_bytes, dtype=torch.uint8).pin_memory()
        h_res = torch.zeros(batch, dtype=torch.uint8).pin_memory()
        # per call: hashing order (count, scatter), hash, key tiles, tensor-core product, tail, fix-up
        launches_per_step = 14

        def sign_op():
            m.sign_shared(esk, d_msgs, sig, ws, batch, msg_off=d_offs, msg_len=d_lens, stream=st)

        def verify_op():
            m.verify_shared(epk, d_msgs, sig, res, ws, batch, msg_off=d_offs, msg_len=d_lens, stream=st)

        # the per-instance engine path (sign_many / verify_many with a shared key), same work
        ws_many = torch.zeros(batch * m.sign_ws_bytes(), dtype=torch.uint8, device=dev)
        sig_many = torch.zeros_like(sig)
        res_many = torch.zeros_like(res)

        def plain_fn():
            m.sign_many(esk, d_msgs, sig_many, ws_many, batch, msg_off=d_offs, msg_len=d_lens, stream=st)
            m.verify_many(epk, d_msgs, sig_many, res_many, batch, msg_off=d_offs, msg_len=d_lens, stream=st)

        plain_api = "per-instance engine: mayo_b200_sign_many / verify_many with esk/epk stride 0"

        def plain_check():  # the two paths must agree byte for byte
            return int((sig_many != sig).sum().item()) + int((res_many != res).sum().item())

        def h2d():
            d_msgs.copy_(h_msgs, non_blocking=True)
            d_offs.copy_(h_offs, non_blocking=True)
            d_lens.copy_(h_lens, non_blocking=True)

        def d2h():
            h_sig.copy_(sig, non_blocking=True)
            h_res.copy_(res, non_blocking=True)

        def gpu_outputs():
            return {"sig": h_sig.numpy().reshape(batch, z.sig_bytes), "res": h_res.numpy()}

        # End to end: the batch in `e2e_chunks` sub-batches on as many streams (the reference
        # benchmark's pattern), so one sub-batch's copies overlap another's kernels.  Each
        # sub-batch: H2D of its messages, offsets and lengths -> sign_shared -> verify_shared ->
        # D2H of its signatures and results.
        nch = max(1, min(args.e2e_chunks, batch))
        bounds = [batch * c // nch for c in range(nch + 1)]
        e2e_streams = [torch.cuda.Stream(dev) for _ in range(nch)]
        ws_c = [torch.zeros(max(m.sign_shared_ws_bytes(b1 - b0), m.verify_shared_ws_bytes(b1 - b0)),
                            dtype=torch.uint8, device=dev) for b0, b1 in zip(bounds, bounds[1:])]
        sb = z.sig_bytes

        def streamed_step(copies):
            start = torch.cuda.Event()
            start.record(st)
            for c, cs in enumerate(e2e_streams):
                b0, b1 = bounds[c], bounds[c + 1]
                m0, m1 = int(offs[b0]), int(offs[b1 - 1]) + int(lens[b1 - 1])
                cs.wait_event(start)
                with torch.cuda.stream(cs):
                    if copies:
                        d_msgs[m0:m1].copy_(h_msgs[m0:m1], non_blocking=True)
                        d_offs[b0:b1].copy_(h_offs[b0:b1], non_blocking=True)
                        d_lens[b0:b1].copy_(h_lens[b0:b1], non_blocking=True)
                    m.sign_shared(esk, d_msgs, sig[b0 * sb:b1 * sb], ws_c[c], b1 - b0, msg_off=d_offs[b0:b1],
                                  msg_len=d_lens[b0:b1], stream=cs)
                    m.verify_shared(epk, d_msgs, sig[b0 * sb:b1 * sb], res[b0:b1], ws_c[c], b1 - b0,
                                    msg_off=d_offs[b0:b1], msg_len=d_lens[b0:b1], stream=cs)
                    if copies:
                        h_sig[b0 * sb:b1 * sb].copy_(sig[b0 * sb:b1 * sb], non_blocking=True)
                        h_res[b0:b1].copy_(res[b0:b1], non_blocking=True)
                done = torch.cuda.Event()
                done.record(cs)
                st.wait_event(done)

        def device_streamed_step():  # the batch in sub-batches on streams, inputs already in HBM
            streamed_step(False)

        # End to end, pipelined over the steps as a serving host would run them: step k + 1's
        # messages, offsets and lengths go up (pinned host -> the other of two device input
        # buffers, on an upload stream) while step k's kernels run, and step k's signatures and
        # results come back (download stream) while step k + 1's run, from the other of two
        # device output buffers (a step's kernels never write a buffer still being read back).
        # Every step's copies are inside the timed region; only the first upload and the last
        # read-back are not overlapped.  The L2 flush stays between steps, after the next step's
        # upload.
        d_in = [(d_msgs, d_offs, d_lens),
                (torch.empty_like(d_msgs), torch.empty_like(d_offs), torch.empty_like(d_lens))]
        d_out = [(sig, res), (torch.empty_like(sig), torch.empty_like(res))]  # also double-buffered
        up_st, down_st = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

        def e2e_run(steps):
            done = [None, None]  # the kernels of the last step that used buffers p
            uploaded = [None, None]
            read = [None, None]  # the read-back of the last step that wrote output buffers p

            def upload(k):
                p = k & 1
                if done[p] is not None:
                    up_st.wait_event(done[p])
                with torch.cuda.stream(up_st):
                    for d, h in zip(d_in[p], (h_msgs, h_offs, h_lens)):
                        d.copy_(h, non_blocking=True)
                uploaded[p] = torch.cuda.Event()
                uploaded[p].record(up_st)

            upload(0)
            for k in range(steps):
                p = k & 1
                if k + 1 < steps:
                    upload(k + 1)
                st.wait_event(uploaded[p])
                if read[p] is not None:
                    st.wait_event(read[p])
                flush.fill_(1)
                dm, do, dl = d_in[p]
                so, ro = d_out[p]
                m.sign_shared(esk, dm, so, ws, batch, msg_off=do, msg_len=dl, stream=st)
                m.verify_shared(epk, dm, so, ro, ws, batch, msg_off=do, msg_len=dl, stream=st)
                done[p] = torch.cuda.Event()
                done[p].record(st)
                down_st.wait_event(done[p])
                with torch.cuda.stream(down_st):
                    h_sig.copy_(so, non_blocking=True)
                    h_res.copy_(ro, non_blocking=True)
                read[p] = torch.cuda.Event()
                read[p].record(down_st)
            fin = torch.cuda.Event()
            fin.record(down_st)
            st.wait_event(fin)

        h2d_bytes = body.nbytes + offs.nbytes + lens.nbytes
        d2h_bytes = batch * z.sig_bytes + batch
        phases = [("sign", sign_op), ("verify", verify_op)]
        ops_per_step = 2 * batch
        macs = mac_counts(s)
        work = {"sign": macs["sign"] * batch, "verify": macs["verify"] * batch}
        hbm_bytes = {"sign": z.esk_bytes + body.nbytes + batch * z.sig_bytes,
                     "verify": z.epk_bytes + body.nbytes + batch * (z.sig_bytes + 1)}
        cfg = {"workload": "MAYO_2 shared-key sign+verify", "set": "MAYO_2", "batch": batch,
               "msg_len": "uniform 32..1024 B", "key": "one expanded key resident in HBM",
               "l2": "flushed between steps (256 MiB write)",
               "api": "mayo_b200_sign_shared / verify_shared (key products on the tensor cores)",
               "e2e": "pipelined over steps: step k+1's inputs uploaded into a second device buffer while step "
                      "k's kernels run, step k's outputs read back while step k+1's run (all copies timed)",
               "value_streams": f"{nch} sub-batches, one stream each, inputs in HBM"}
        expected = np.zeros(batch, np.uint8)
        res_dev = lambda: res  # noqa: E731
        # Per-kernel algorithmic work (per call of `batch` instances) for the rooflines:
        #   product: GF(16) MACs of the key products done as binary MACs on the tensor cores
        #            (16 bit-products per GF(16) MAC, 2 ops each, int8 peak = 2 x bf16);
        #   tail:    the per-instance GF(16) MACs left to the integer pipes (0.5 lane-op each);
        #   hash:    bytes read and written in HBM.
        n_, m_, o_, k_ = PARAMS[s]
        v_ = n_ - o_
        e1_, e2_, e3_ = v_ * (v_ + 1) // 2, v_ * o_, o_ * (o_ + 1) // 2
        prod_macs = {"sign": k_ * m_ * e1_ + k_ * m_ * v_ * o_, "verify": k_ * m_ * (e1_ + e2_ + e3_)}
        tail_macs = {"sign": m_ * k_ * k_ * v_ + m_ * m_ * (k_ * o_ + 1), "verify": m_ * k_ * k_ * n_}
        kernel_model = {}
        for ph in ("sign", "verify"):
            kernel_model[(ph, "product")] = ("tensor", 32.0 * prod_macs[ph] * batch)
            kernel_model[(ph, "tail")] = ("alu", 0.5 * tail_macs[ph] * batch)
            kernel_model[(ph, "hash")] = ("hbm", float(body.nbytes + offs.nbytes + lens.nbytes +
                                                      batch * (z.sig_bytes if ph == "verify" else 0) + 64 * batch))

        def kernel_profile(steps):
            """Per-kernel times inside the shared-key calls (CUDA events between the kernels)."""
            acc = {}
            M.Mayo.shared_timing(True)
            try:
                for _ in range(steps):
                    flush.fill_(1)
                    for ph, fn in phases:
                        fn()
                        for kname, ms in M.Mayo.shared_timing_read().items():
                            acc[(ph, kname)] = acc.get((ph, kname), 0.0) + ms
            finally:
                M.Mayo.shared_timing(False)
            return {key: v / steps for key, v in acc.items()}
    elif wl["kind"] == "keypair_sign_verify":
        # every instance: seeded keypair -> sign (compact sk, expanded inside) -> verify (compact pk)
        mlen = wl["mlen"][0]
        seeds = seeds_for(seed, batch, z.sk_bytes)
        msgs = chacha((b"mayo-b200-msgs-%d" % seed).ljust(32, b"\0")[:32], batch * mlen).reshape(batch, mlen)
        kpool, kp = m.alloc_pool("keypair", batch)
        spool, sp = m.alloc_pool("signWithesk", batch, mlen)
        vpool, vp = m.alloc_pool("verifyWithepk", batch, mlen)
        K2, S2, V2 = kpool.view(batch, kp), spool.view(batch, sp), vpool.view(batch, vp)
        h_seeds = torch.from_numpy(seeds).pin_memory()
        h_msgs = torch.from_numpy(msgs.copy()).pin_memory()
        h_pk = torch.zeros((batch, z.pk_bytes), dtype=torch.uint8).pin_memory()
        h_sig = torch.zeros((batch, z.sig_bytes), dtype=torch.uint8).pin_memory()
        h_res = torch.zeros(batch, dtype=torch.uint8).pin_memory()
        pk_off, msg_s, msg_v = A128(z.sk_bytes), A128(z.esk_bytes), A128(z.epk_bytes)
        sig_s, sig_v = msg_s + A128(mlen), msg_v + A128(mlen)
        res_off = sig_v + A128(z.sig_bytes)
        K2[:, : z.sk_bytes].copy_(h_seeds)
        S2[:, msg_s: msg_s + mlen].copy_(h_msgs)
        V2[:, msg_v: msg_v + mlen].copy_(h_msgs)
        launches_per_step = 13  # keypair 4 (hash, AES, tail, P3), signWithesk 6, verifyWithepk 3

        def keypair_op():
            m.crypto_sign_keypair_from_seed(kpool, kp, batch, st)

        def sign_op():
            S2[:, : z.sk_bytes].copy_(K2[:, : z.sk_bytes])
            m.crypto_sign_signWithesk(spool, mlen, sp, batch, st)

        def verify_op():
            V2[:, z.p_bytes - 16: z.p_bytes - 16 + z.pk_bytes].copy_(K2[:, pk_off: pk_off + z.pk_bytes])
            V2[:, sig_v: sig_v + z.sig_bytes].copy_(S2[:, sig_s: sig_s + z.sig_bytes])
            m.crypto_sign_verifyWithepk(vpool, mlen, vp, batch, st)

        def h2d():
            K2[:, : z.sk_bytes].copy_(h_seeds, non_blocking=True)
            S2[:, msg_s: msg_s + mlen].copy_(h_msgs, non_blocking=True)
            V2[:, msg_v: msg_v + mlen].copy_(h_msgs, non_blocking=True)

        def d2h():
            h_pk.copy_(K2[:, pk_off: pk_off + z.pk_bytes], non_blocking=True)
            h_sig.copy_(S2[:, sig_s: sig_s + z.sig_bytes], non_blocking=True)
            h_res.copy_(V2[:, res_off], non_blocking=True)

        def gpu_outputs():
            return {"pk": h_pk.numpy(), "sig": h_sig.numpy(), "res": h_res.numpy()}

        h2d_bytes = seeds.nbytes + 2 * msgs.nbytes
        d2h_bytes = batch * (z.pk_bytes + z.sig_bytes + 1)
        phases = [("keypair", keypair_op), ("sign", sign_op), ("verify", verify_op)]
        ops_per_step = 3 * batch
        macs = mac_counts(s)
        expand_l = z.m * z.o * z.m * (z.m - 1)  # L = (P1 + P1^T) O + P2 inside signWithesk (v == m)
        work = {"keypair": macs["keypair"] * batch, "sign": (macs["sign"] + expand_l) * batch,
                "verify": macs["verify"] * batch}
        hbm_bytes = {"keypair": 2 * batch * z.p_bytes, "sign": 3 * batch * z.esk_bytes,
                     "verify": 2 * batch * z.epk_bytes}
        cfg = {"workload": f"MAYO_{s} keypair -> sign -> verify, distinct keys", "set": f"MAYO_{s}", "batch": batch,
               "msg_len": f"{mlen} B", "key": "per-instance seeded keypairs (ChaCha20)",
               "l2": "flushed between steps (256 MiB write)",
               "api": "crypto_sign_keypair_from_seed / signWithesk / verifyWithepk (pool API)"}
        expected = np.zeros(batch, np.uint8)
        res_dev = lambda: V2[:, res_off]  # noqa: E731
    elif wl["kind"] == "distinct_verify":
        # every instance has its own keypair; epk resident in the verify pool, 10% corrupted sigs
        mlen = wl["mlen"][0]
        dv = build_distinct_verify(m, batch, seed, mlen, st)
        vpool, vp, V2, msgs, sigs, bad_idx = dv["vpool"], dv["pitch"], dv["rows"], dv["msgs"], dv["sigs"], dv["bad"]
        msg_v, sig_v, res_off = dv["msg_off"], dv["sig_off"], dv["res_off"]
        h_sig = torch.from_numpy(sigs).pin_memory()
        h_msgs = torch.from_numpy(msgs.copy()).pin_memory()
        h_res = torch.zeros(batch, dtype=torch.uint8).pin_memory()
        launches_per_step = 1

        def verify_op():
            m.crypto_sign_verify(vpool, mlen, vp, batch, st)

        def h2d():
            V2[:, msg_v: msg_v + mlen].copy_(h_msgs, non_blocking=True)
            V2[:, sig_v: sig_v + z.sig_bytes].copy_(h_sig, non_blocking=True)

        def d2h():
            h_res.copy_(V2[:, res_off], non_blocking=True)

        def gpu_outputs():
            return {"pk": dv["pks"], "good_sig": dv["good_sigs"], "sig_in": sigs, "res": h_res.numpy()}

        h2d_bytes = msgs.nbytes + sigs.nbytes
        d2h_bytes = batch
        phases = [("verify", verify_op)]
        ops_per_step = batch
        work = {"verify": mac_counts(s)["verify"] * batch}
        hbm_bytes = {"verify": batch * (z.epk_bytes + z.sig_bytes + mlen)}
        cfg = {"workload": f"MAYO_{s} distinct-key verify", "set": f"MAYO_{s}", "batch": batch,
               "msg_len": f"{mlen} B", "key": "per-instance expanded public keys resident in HBM (pool rows)",
               "corrupted": "10% (one random nibble flipped), must return 1",
               "l2": "inputs larger than L2 (EPKs) and flushed between steps",
               "api": "crypto_sign_verify (pool API)"}
        expected = np.zeros(batch, np.uint8)
        expected[bad_idx] = 1
        res_dev = lambda: V2[:, res_off]  # noqa: E731
    elif wl["kind"] == "mixed_queue":
        phases, h2d, d2h, h2d_bytes, d2h_bytes, ops_per_step, work, hbm_bytes, cfg, expected, res_dev, h_res, \
            plain_fn, launches_per_step = setup_mixed_queue(args, dist, batch, seed, st)
    else:
        raise SystemExit(f"unknown workload {args.workload}")

    tuned = None
    if wl["kind"] == "shared_sign_verify" and args.shape:
        parts = [int(x) for x in args.shape.lower().split("x")]
        h_, g_, p_ = (parts + [1, 1, 1])[:3]
        m.set_shared_shape(h_, g_, p_)
        cfg["shape"] = {"hash_threads": h_, "tail_instances": g_, "product_ctas": p_, "chosen_by": "--shape"}
    elif wl["kind"] == "shared_sign_verify":
        # block shapes of the shared-key calls (hash CTA threads, sign-tail instances per CTA),
        # timed on this GPU by the autotuner (cached per GPU, library build, set and batch)
        from cumayo_b200 import autotune as AT
        tuned = AT.tune_shared(m, lambda: [fn() for _, fn in phases], batch, flush=lambda: flush.fill_(1))
        cfg["shape"] = {"hash_threads": tuned["hash_threads"], "tail_instances": tuned["tail_instances"],
                        "product_ctas": tuned.get("product_ctas", 1),
                        "chosen_by": "cumayo_b200.autotune.tune_shared",
                        "trials_ms": {f"{t['hash_threads']}x{t['tail_instances']}x{t.get('product_ctas', 1)}":
                                      round(t["ms"], 4) for t in tuned.get("trials", [])}}

    def step():
        flush.fill_(1)
        for _, fn in phases:
            fn()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    bad = int((res_dev().cpu().numpy() != expected).sum())

    # ---- device-resident timing ----
    ev = {name: [] for name, _ in phases}
    clocks = Clocks(dist.local)
    dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(st)
    for _ in range(args.steps):
        flush.fill_(1)
        for name, fn in phases:
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            fn()
            b.record(st)
            ev[name].append((a, b))
    t1.record(st)
    torch.cuda.synchronize()
    dist.barrier()
    total_ms = dist.max(t0.elapsed_time(t1))
    phase_ms = {name: sum(a.elapsed_time(b) for a, b in lst) / len(lst) for name, lst in ev.items()}

    # ---- device-resident, the batch in sub-batches on several streams (kernels of different
    # sub-batches overlap: e.g. one's hashing with another's tensor-core product) ----
    streamed_ms = None
    if device_streamed_step is not None:
        for _ in range(2):
            flush.fill_(1)
            device_streamed_step()
        torch.cuda.synchronize()
        dist.barrier()
        q0 = torch.cuda.Event(enable_timing=True)
        q1 = torch.cuda.Event(enable_timing=True)
        q0.record(st)
        for _ in range(args.steps):
            flush.fill_(1)
            device_streamed_step()
        q1.record(st)
        torch.cuda.synchronize()
        dist.barrier()
        streamed_ms = dist.max(q0.elapsed_time(q1))
        bad += int((res_dev().cpu().numpy() != expected).sum())

    # ---- end to end through the public API with host buffers (clocks keep sampling) ----
    if e2e_run is not None:  # warm the upload / download streams
        e2e_run(2)
        torch.cuda.synchronize()
    dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    if e2e_run is not None:
        e2e_run(args.steps)
    for _ in range(args.steps if e2e_run is None else 0):
        flush.fill_(1)
        h2d()
        for _, fn in phases:
            fn()
        d2h()
    e1.record(st)
    torch.cuda.synchronize()
    clk = clocks.stop()
    e2e_ms = dist.max(e0.elapsed_time(e1))
    bad_e2e = int((h_res.numpy() != expected).sum())

    ms_per_step = total_ms / args.steps
    value = weak_value(ops_per_step, dist.world, ms_per_step)
    sm_mhz = clk.get("sm_mhz") or 1965.0
    peak_ops = LOP3_LANE_OPS_PER_CLK_SM * 148 * sm_mhz * 1e6 / 1e9  # G lane-ops/s
    dom = max(phase_ms, key=phase_ms.get)
    ach_ops = 0.5 * work[dom] / (phase_ms[dom] / 1e3) / 1e9  # 16 LOP3 per 32 GF(16) MACs
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "ops/s", "n_gpus": dist.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (GF(16) bit-planes)", "data": "synthetic (seeded ChaCha20)",
        "config": cfg,
        "sign_per_s": round(batch * dist.world / (phase_ms["sign"] / 1e3), 1) if "sign" in phase_ms else None,
        "verify_per_s": round(batch * dist.world / (phase_ms["verify"] / 1e3), 1) if "verify" in phase_ms else None,
        "phase_ms": {k: round(v, 4) for k, v in phase_ms.items()},
        "value_streams": (round(ops_per_step * dist.world / (streamed_ms / args.steps / 1e3), 1)
                          if streamed_ms else None),
        "roofline_alu": {"bound": "alu", "kernel": f"{dom} ({args.workload})", "achieved": round(ach_ops, 1),
                         "peak": round(peak_ops, 1), "unit": "G int-ops/s", "frac": round(ach_ops / peak_ops, 4),
                         "traffic": None,
                         "definition": "algorithmic ops = 0.5 x GF(16) MACs (16 LOP3 per 32 MACs); peak = measured "
                                       "LOP3 issue rate 64 lane-ops/clk/SM x 148 SMs x median SM clock"},
        "roofline_hbm": {"bound": "hbm", "kernel": f"{dom} ({args.workload})",
                         "achieved": round(hbm_bytes[dom] / (phase_ms[dom] / 1e3) / 1e9, 2),
                         "peak": HBM_PEAK_GBS, "unit": "GB/s",
                         "frac": round(hbm_bytes[dom] / (phase_ms[dom] / 1e3) / 1e9 / HBM_PEAK_GBS, 5),
                         "traffic": (int(VERIFY_TRAFFIC_PER_INST[s] * batch)
                                     if wl["kind"] == "distinct_verify" and s in VERIFY_TRAFFIC_PER_INST else None),
                         "definition": "algorithmic bytes the kernel must move from HBM per launch / kernel time; "
                                       f"peak = copy bandwidth ({HBM_PEAK_SRC})"},
        "e2e": {"value": round(ops_per_step * dist.world / (e2e_ms / args.steps / 1e3), 1), "unit": "ops/s",
                "h2d_bytes_per_step": int(h2d_bytes), "d2h_bytes_per_step": int(d2h_bytes)},
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clk,
        "result_mismatches": bad + bad_e2e,
    }
    # The binding roof: distinct-key verify streams every EPK from HBM (bound hbm); the other
    # workloads keep keys L2-resident and are integer-ALU bound (bound alu).
    out["roofline"] = dict(out["roofline_hbm"] if wl["kind"] == "distinct_verify" else out["roofline_alu"])
    if kernel_profile is not None:
        kt = kernel_profile(args.steps)
        int8_peak = 2.0 * BF16_PEAK_TFLOPS

        def traffic(name):
            per = KERNEL_TRAFFIC_PER_INST.get(s, {}).get(name)
            return None if per is None else int(per * batch)
        kern = {}
        for key, ms in sorted(kt.items()):
            ent = {"ms": round(ms, 4), "share": round(ms / sum(kt.values()), 4)}
            if key in kernel_model and ms > 0:
                bound, amount = kernel_model[key]
                if bound == "tensor":
                    a_ = amount / (ms / 1e3) / 1e12
                    ent.update(bound="tensor", achieved=round(a_, 1), peak=round(int8_peak, 1), unit="Tops/s",
                               frac=round(a_ / int8_peak, 4))
                elif bound == "alu":
                    a_ = amount / (ms / 1e3) / 1e9
                    ent.update(bound="alu", achieved=round(a_, 1), peak=round(peak_ops, 1), unit="G int-ops/s",
                               frac=round(a_ / peak_ops, 4))
                else:
                    a_ = amount / (ms / 1e3) / 1e9
                    ent.update(bound="hbm", achieved=round(a_, 1), peak=HBM_PEAK_GBS, unit="GB/s",
                               frac=round(a_ / HBM_PEAK_GBS, 4))
            kern[f"{key[0]}.{key[1]}"] = ent
        out["kernels"] = kern
        top = max(kt, key=kt.get)
        t = kern[f"{top[0]}.{top[1]}"]
        out["roofline"] = {"bound": t.get("bound"), "kernel": f"{top[0]} {top[1]} kernel ({args.workload})",
                           "achieved": t.get("achieved"), "peak": t.get("peak"), "unit": t.get("unit"),
                           "frac": t.get("frac"), "traffic": traffic(f"{top[0]}.{top[1]}"),
                           "definition": KERNEL_ROOF_DEF[t.get("bound")]}
        pr = kern.get("sign.product", {})
        out["roofline_tensor"] = {"bound": "tensor", "kernel": f"sign product kernel ({args.workload})",
                                  "achieved": pr.get("achieved"), "peak": pr.get("peak"), "unit": "Tops/s",
                                  "frac": pr.get("frac"), "traffic": traffic("sign.product"),
                                  "definition": KERNEL_ROOF_DEF["tensor"]}
    if plain_fn is not None:
        # the same work as per-(set, op) batched launches on the same GPU
        for _ in range(args.warmup):
            plain_fn()
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(st)
        for _ in range(args.steps):
            flush.fill_(1)
            plain_fn()
        p1.record(st)
        torch.cuda.synchronize()
        plain_ms = dist.max(p0.elapsed_time(p1)) / args.steps
        out["plain"] = {"value": round(ops_per_step * dist.world / (plain_ms / 1e3), 1), "ms_per_step": round(plain_ms, 4),
                        "api": plain_api}
        if plain_check is not None:
            out["result_mismatches"] += plain_check()
    if wl["kind"] == "shared_sign_verify" and dist.world == 1 and getattr(args, "per_set", False):
        per = per_set_measure(args, dist, run_ours)
        m2 = per.setdefault(f"MAYO_{s}", {"mismatches": 0})
        m2["shared_key_batch"] = batch
        m2["shared_sign_per_s"] = out["sign_per_s"]
        m2["shared_verify_per_s"] = out["verify_per_s"]
        # the reference arm of this bench, when it ran on this GPU shortly before, leaves its
        # per-set figures in REF_PER_SET_FILE: add them and the ratios
        ref = None
        try:
            with open(REF_PER_SET_FILE) as f:
                ref = json.load(f)
            if ref.get("gpu") != gpu_identity(dist.local) or time.time() - float(ref.get("time", 0)) > 6 * 3600:
                ref = None
        except (OSError, ValueError):
            ref = None
        for key, ent in per.items():
            out["result_mismatches"] += ent["mismatches"]
            r = (ref or {}).get("per_set", {}).get(key)
            if r:
                ent["reference"] = {k: v for k, v in r.items() if k.endswith("_per_s")}
                ent["vs_reference"] = {k: round(ent[k] / v, 2) for k, v in ent["reference"].items()
                                       if k in ent and v}
        out["per_set"] = per
        out["per_set_note"] = ("ops/s, device-timed (CUDA events), L2 flushed between steps: keypair/sign/verify = "
                               "keypair_from_seed / signWithesk / verifyWithepk at batch 1,024 with distinct keys and "
                               "32-byte messages (the reference benchmark's operations); distinct_verify = "
                               "crypto_sign_verify at 16,384 (C3); shared = this line's MAYO_2 shared-key run. "
                               "'reference' = the reference's own build on this GPU, from this bench's reference arm "
                               + ("run at " + time.strftime("%Y-%m-%d %H:%M:%S", time.gmtime(float(ref["time"])))
                                  + " UTC" if ref else "(not run on this GPU: no ratio)"))
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(args, gpu_outputs() if gpu_outputs is not None else None)
        out["cpu_baseline"] = cb
        if cb is not None and cb.get("oracle_check") is not None:
            out["result_mismatches"] += cb["oracle_check"]["mismatches"]
    return out


def corrupt_tenth(sigs: np.ndarray, seed: int):
    """A seeded tenth of the signatures get one uniformly random nibble flipped (nonzero XOR)."""
    batch, sb = sigs.shape
    rng = np.random.default_rng(seed)
    bad_idx = np.sort(rng.choice(batch, batch // 10, replace=False))
    out = sigs.copy()
    for i in bad_idx:
        pos = int(rng.integers(0, 2 * sb))
        out[i, pos // 2] ^= np.uint8(int(rng.integers(1, 16)) << (4 * (pos % 2)))
    return out, bad_idx


def build_distinct_verify(m, batch: int, seed: int, mlen: int, st):
    """C3 inputs on the device: `batch` ChaCha20-seeded keypairs, each signing its own `mlen`-byte
    message (pool API), expanded public keys resident in a verify pool (the reference's verify
    layout), then a seeded tenth of the signatures corrupted.  Returns the pool and host copies."""
    import torch
    z = m.sizes
    seeds = seeds_for(seed, batch, z.sk_bytes)
    msgs = chacha((b"mayo-b200-msgs-%d" % seed).ljust(32, b"\0")[:32], batch * mlen).reshape(batch, mlen)
    vpool, vp = m.alloc_pool("verify", batch, mlen)
    V2 = vpool.view(batch, vp)
    msg_v = A128(z.epk_bytes)
    sig_v = msg_v + A128(mlen)
    res_off = sig_v + A128(z.sig_bytes)
    pks = np.zeros((batch, z.pk_bytes), np.uint8)
    chunk = 2048  # set-up in chunks: keypair pools are large for MAYO_5
    for c0 in range(0, batch, chunk):
        nb = min(chunk, batch - c0)
        kpool, kp = m.alloc_pool("keypair", nb)
        K2 = kpool.view(nb, kp)
        K2[:, : z.sk_bytes].copy_(torch.from_numpy(seeds[c0:c0 + nb]))
        m.crypto_sign_keypair_from_seed(kpool, kp, nb, st)
        pk_off = A128(z.sk_bytes)
        V2[c0:c0 + nb, z.p_bytes - 16: z.p_bytes - 16 + z.pk_bytes].copy_(K2[:, pk_off: pk_off + z.pk_bytes])
        pks[c0:c0 + nb] = K2[:, pk_off: pk_off + z.pk_bytes].cpu().numpy()
        spool, spch = m.alloc_pool("signWithesk", nb, mlen)
        S2 = spool.view(nb, spch)
        S2[:, : z.sk_bytes].copy_(K2[:, : z.sk_bytes])
        ms_ = A128(z.esk_bytes)
        S2[:, ms_: ms_ + mlen].copy_(torch.from_numpy(msgs[c0:c0 + nb]))
        m.crypto_sign_signWithesk(spool, mlen, spch, nb, st)
        ss_ = ms_ + A128(mlen)
        V2[c0:c0 + nb, sig_v: sig_v + z.sig_bytes].copy_(S2[:, ss_: ss_ + z.sig_bytes])
        del kpool, spool
    m.crypto_sign_expandpk(vpool, vp, batch, st)
    V2[:, msg_v: msg_v + mlen].copy_(torch.from_numpy(msgs))
    torch.cuda.synchronize()
    good_sigs = V2[:, sig_v: sig_v + z.sig_bytes].cpu().numpy()
    sigs, bad_idx = corrupt_tenth(good_sigs, seed)
    V2[:, sig_v: sig_v + z.sig_bytes].copy_(torch.from_numpy(sigs))
    return dict(vpool=vpool, pitch=vp, rows=V2, seeds=seeds, msgs=msgs, pks=pks, good_sigs=good_sigs, sigs=sigs,
                bad=bad_idx, msg_off=msg_v, sig_off=sig_v, res_off=res_off)


def expand_shared_key(m, key_seed: np.ndarray, dev, st):
    """(esk, epk) device tensors for one caller-seeded keypair, through the pool API."""
    import torch
    z = m.sizes
    kp, kpitch = m.alloc_pool("keypair", 1)
    kp[: z.sk_bytes].copy_(torch.from_numpy(key_seed))
    m.crypto_sign_keypair_from_seed(kp, kpitch, 1, st)
    esk = torch.zeros(z.esk_bytes, dtype=torch.uint8, device=dev)
    esk[: z.sk_bytes].copy_(kp[: z.sk_bytes])
    m.crypto_sign_expandsk(esk, z.esk_bytes, 1, st)
    epk = torch.zeros(z.epk_bytes, dtype=torch.uint8, device=dev)
    pk_off = A128(z.sk_bytes)
    epk[z.p_bytes - 16: z.p_bytes - 16 + z.pk_bytes].copy_(kp[pk_off: pk_off + z.pk_bytes])
    m.crypto_sign_expandpk(epk, z.epk_bytes, 1, st)
    return esk, epk


def setup_mixed_queue(args, dist, batch, seed, st):
    """C4: `batch` operations uniform over {MAYO_1,2,3,5} x {keypair, sign, verify}, shuffled, in
    one persistent queue launch replayed from a CUDA graph; shape chosen by the autotuner.  The
    same work as per-(set, op) batched launches is the comparison (`plain`)."""
    import torch

    import cumayo_b200 as M
    from cumayo_b200 import autotune as AT
    from cumayo_b200 import queue as Q
    dev = torch.cuda.current_device()
    sets, mlen = [1, 2, 3, 5], 32
    per = [batch // 12 + (1 if i < batch % 12 else 0) for i in range(12)]
    operands, entries, plain_parts = {}, [], []
    h2d_list, d2h_list, h_res_parts = [], [], []
    work_macs = 0.0
    for si, s in enumerate(sets):
        m = M.Mayo(s)
        z = m.sizes
        n_kp, n_sg, n_vf = per[3 * si], per[3 * si + 1], per[3 * si + 2]
        seeds = seeds_for(seed * 10 + s, n_kp, z.sk_bytes)
        esk, epk = expand_shared_key(m, seeds_for(seed * 10 + s + 5, 1, z.sk_bytes)[0], dev, st)
        msg_sg = chacha((b"c4-sign-%d-%d" % (seed, s)).ljust(32, b"\0"), n_sg * mlen).reshape(n_sg, mlen)
        msg_vf = chacha((b"c4-verify-%d-%d" % (seed, s)).ljust(32, b"\0"), n_vf * mlen).reshape(n_vf, mlen)
        d_seeds = torch.from_numpy(seeds).to(dev)
        d_pk = torch.zeros(n_kp * z.pk_bytes, dtype=torch.uint8, device=dev)
        d_msg_sg = torch.from_numpy(msg_sg.copy()).to(dev)
        d_sig_sg = torch.zeros(n_sg * z.sig_bytes, dtype=torch.uint8, device=dev)
        d_msg_vf = torch.from_numpy(msg_vf.copy()).to(dev)
        d_sig_vf = torch.zeros(n_vf * z.sig_bytes, dtype=torch.uint8, device=dev)
        d_res = torch.full((n_vf,), 0xEE, dtype=torch.uint8, device=dev)
        ws = torch.zeros(max(n_sg, n_vf) * m.sign_ws_bytes(), dtype=torch.uint8, device=dev)
        m.sign_many(esk, d_msg_vf, d_sig_vf, ws, n_vf, msg_stride=mlen, mlen=mlen, stream=st)  # valid signatures
        operands[s] = Q.SetOperands(kp_seed=d_seeds, kp_pk=d_pk, sg_esk=esk, sg_nkeys=1, sg_msg=d_msg_sg,
                                    sg_mlen=mlen, sg_sig=d_sig_sg, vf_epk=epk, vf_nkeys=1, vf_msg=d_msg_vf,
                                    vf_mlen=mlen, vf_sig=d_sig_vf, vf_res=d_res)
        entries += [(Q.OP_KEYPAIR, s, i) for i in range(n_kp)] + [(Q.OP_SIGN, s, i) for i in range(n_sg)] + \
                   [(Q.OP_VERIFY, s, i) for i in range(n_vf)]
        mc = mac_counts(s)
        work_macs += n_kp * mc["keypair"] + n_sg * mc["sign"] + n_vf * mc["verify"]
        # plain per-(set, op) launches doing the same work
        kpool, kpch = m.alloc_pool("keypair", n_kp)
        kpool.view(n_kp, kpch)[:, : z.sk_bytes].copy_(d_seeds)
        plain_parts.append((m, kpool, kpch, n_kp, esk, epk, d_msg_sg, d_sig_sg, n_sg, d_msg_vf, d_sig_vf,
                            d_res, n_vf, ws))
        h_seeds = torch.from_numpy(seeds).pin_memory()
        h_msgs = torch.from_numpy(msg_sg.copy()).pin_memory()
        h_msgv = torch.from_numpy(msg_vf.copy()).pin_memory()
        h_sigv = torch.empty(n_vf * z.sig_bytes, dtype=torch.uint8).pin_memory()
        torch.cuda.synchronize()
        h_sigv.copy_(d_sig_vf)
        h2d_list += [(d_seeds, h_seeds), (d_msg_sg, h_msgs), (d_msg_vf, h_msgv), (d_sig_vf, h_sigv)]
        h_res_s = torch.empty(n_vf, dtype=torch.uint8).pin_memory()
        h_res_parts.append(h_res_s)
        d2h_list += [(torch.empty(n_kp * z.pk_bytes, dtype=torch.uint8).pin_memory(), d_pk),
                     (torch.empty(n_sg * z.sig_bytes, dtype=torch.uint8).pin_memory(), d_sig_sg),
                     (h_res_s, d_res)]
    rng = np.random.default_rng(seed)
    items = Q.items_array([entries[i] for i in rng.permutation(len(entries))])
    q = Q.Queue(capacity=batch + batch // 8 + 64)
    for s, ops in operands.items():
        q.set_operands(s, ops)
    tuned = AT.tune_queue(q, items)
    q.capture()

    def queue_op():
        q.replay()

    def plain():
        for (m, kpool, kpch, n_kp, esk, epk, d_msg_sg, d_sig_sg, n_sg, d_msg_vf, d_sig_vf, d_res, n_vf,
             ws) in plain_parts:
            m.crypto_sign_keypair_from_seed(kpool, kpch, n_kp, st)
            m.sign_many(esk, d_msg_sg, d_sig_sg, ws, n_sg, msg_stride=mlen, mlen=mlen, stream=st)
            m.verify_many(epk, d_msg_vf, d_sig_vf, d_res, n_vf, msg_stride=mlen, mlen=mlen, stream=st)

    def h2d():
        for d, h in h2d_list:
            d.copy_(h, non_blocking=True)

    def d2h():
        for h, d in d2h_list:
            h.copy_(d, non_blocking=True)

    all_res = [ops.vf_res for ops in operands.values()]
    n_vf_total = sum(int(r.numel()) for r in all_res)
    expected = np.zeros(n_vf_total, np.uint8)
    res_dev = lambda: torch.cat(all_res)  # noqa: E731
    class _HostRes:  # host copies of every set's verify results, concatenated like res_dev()
        def numpy(self):
            return torch.cat(h_res_parts).numpy()

    h_res = _HostRes()
    h2d_bytes = sum(int(h.numel()) for _, h in h2d_list)
    d2h_bytes = sum(int(d.numel()) for _, d in d2h_list)
    cfg = {"workload": "mixed MAYO_1/2/3/5 x {keypair, sign, verify} in one persistent work queue "
                       "(device partition by (set, op), one persistent kernel each on forked streams)",
           "batch": batch, "msg_len": f"{mlen} B", "keys": "caller-seeded keypairs; one resident key per set "
                                                          "for sign/verify",
           "queue": {"sms": q.shape.sms, "ctas_per_sm": tuned["ctas_per_sm"], "launch_order": tuned["launch_order"],
                     "capacity": q.capacity, "autotune_trials": tuned.get("trials")},
           "graph": "CUDA graph (queue reset, partition, 12 persistent (set, op) kernels) replayed per step",
           "l2": "flushed between steps (256 MiB write)"}
    return ([("queue", queue_op)], h2d, d2h, h2d_bytes, d2h_bytes, batch, {"queue": work_macs},
            {"queue": 0}, cfg, expected, res_dev, h_res, plain, 14)


# ---------------------------------------------------------------------------------------------
# per-set figures: keypair / sign / verify of every parameter set (the reference benchmark's three
# operations, tests/bench_stream.cu:47-176 of the reference) and the distinct-key verifies
# ---------------------------------------------------------------------------------------------
PER_SET_RUNS = ("c1", "c1-2", "c1-3", "c1-5", "c3-3", "c3-5")
REF_PER_SET_FILE = os.path.join(tempfile.gettempdir(), "mayo_b200_reference_per_set.json")


def per_set_measure(args, dist, runner) -> dict:
    """Runs the per-set workloads with `runner` (run_ours or run_reference) and collects ops/s per
    set: keypair/sign/verify at batch 1,024 (distinct keys, 32-byte messages) and, for MAYO_3/5,
    the distinct-key verify at 16,384."""
    per = {}
    for name in PER_SET_RUNS:
        sub = argparse.Namespace(**vars(args))
        sub.workload, sub.batch, sub.no_cpu_baseline, sub.per_set = name, 0, True, False
        sub.steps, sub.warmup = min(args.steps, 10), max(3, min(args.warmup, 3))
        r = runner(sub, dist)
        wl = WORKLOADS[name]
        ent = per.setdefault(f"MAYO_{wl['set']}", {"mismatches": 0})
        ph = r.get("phase_ms", {})
        if wl["kind"] == "keypair_sign_verify":
            ent["batch"] = wl["batch"]
            for op in ("keypair", "sign", "verify"):
                if op in ph and ph[op] > 0:
                    ent[f"{op}_per_s"] = round(wl["batch"] / (ph[op] / 1e3), 1)
        else:
            ent["distinct_verify_batch"] = wl["batch"]
            if ph.get("verify", 0) > 0:
                ent["distinct_verify_per_s"] = round(wl["batch"] / (ph["verify"] / 1e3), 1)
        ent["mismatches"] += int(r.get("result_mismatches", 0))
    return per


def gpu_identity(dev_index: int) -> str:
    import torch
    p = torch.cuda.get_device_properties(dev_index)
    return f"{p.name}/{getattr(p, 'uuid', '')}"


# ---------------------------------------------------------------------------------------------
# CPU baseline: the oracle (a restatement of the reference's algorithm) on the host cores
# ---------------------------------------------------------------------------------------------
def cpu_baseline(args, gpu: dict | None = None, sample: int | None = None):
    """The oracle timed on the host cores on a bounded sample of the workload: the first `sample`
    instances of rank 0's own inputs (the ChaCha20 generators give the same prefix).  Its outputs
    for those instances are also compared byte for byte with the GPU's (`gpu`: host copies of the
    last end-to-end step), reported as `oracle_check`."""
    from oracle import oracle as O
    wl = WORKLOADS[args.workload]
    if wl["kind"] not in ("shared_sign_verify", "keypair_sign_verify", "distinct_verify"):
        return None  # mixed queue / serving: no single-set CPU leg
    s = wl["set"]
    P = O.params(s)
    threads = O.max_threads()

    def check(pairs, n):
        if gpu is None:
            return None
        bad = 0
        for name, want, got in pairs:
            bad += int((np.asarray(want) != np.asarray(got)).reshape(n, -1).any(axis=1).sum())
        return {"instances": n, "compared": [p[0] for p in pairs], "mismatches": bad}

    if wl["kind"] == "shared_sign_verify":
        sample = sample or 4096
        seed = seeds_for(1, 1, P.sk_bytes)[0].tobytes()
        pk = O.keypair_from_seed(s, seed)
        esk = np.frombuffer(O.expandsk(s, seed), np.uint8)[None, :]
        epk = np.frombuffer(O.expandpk(s, pk), np.uint8)[None, :]
        body, offs, lens = make_messages(1, sample, *wl["mlen"])
        msgs = [body[int(o):int(o) + int(n)].tobytes() for o, n in zip(offs, lens)]
        t = time.perf_counter()
        sig, _ = O.sign_batch(s, esk, msgs, shared_key=True)
        t_sign = time.perf_counter() - t
        t = time.perf_counter()
        res = O.verify_batch(s, epk, msgs, sig, shared_key=True)
        t_ver = time.perf_counter() - t
        assert int(res.sum()) == 0
        n = min(sample, gpu["sig"].shape[0]) if gpu else 0
        return {"value": round(2 * sample / (t_sign + t_ver), 1), "unit": "ops/s", "cores": threads, "kind": "port",
                "sample": f"{sample} signs + {sample} verifies of the same workload (shared MAYO_2 key, "
                          f"32..1024 B messages), OpenMP one instance per thread",
                "sign_per_s": round(sample / t_sign, 1), "verify_per_s": round(sample / t_ver, 1),
                "oracle_check": check([("signature", sig[:n], gpu["sig"][:n]), ("verify byte", res[:n], gpu["res"][:n])],
                                      n) if gpu else None}
    if wl["kind"] == "keypair_sign_verify":
        sample = sample or 4 * wl["batch"]
        seeds = seeds_for(1, sample, P.sk_bytes)
        msgs = chacha(b"mayo-b200-msgs-1".ljust(32, b"\0"), sample * 32).reshape(sample, 32)
        t = time.perf_counter()
        pk = O.keypair_from_seed_batch(s, seeds)
        t_kp = time.perf_counter() - t
        t = time.perf_counter()
        sig, _ = O.sign_batch(s, O.expandsk_batch(s, seeds), [bytes(x) for x in msgs])
        t_sign = time.perf_counter() - t
        t = time.perf_counter()
        res = O.verify_batch(s, O.expandpk_batch(s, pk), [bytes(x) for x in msgs], sig)
        t_ver = time.perf_counter() - t
        assert int(res.sum()) == 0
        n = min(sample, gpu["sig"].shape[0]) if gpu else 0
        return {"value": round(3 * sample / (t_kp + t_sign + t_ver), 1), "unit": "ops/s", "cores": threads,
                "kind": "port", "sample": f"{sample} instances of keypair -> sign (expand-sk inside) -> verify "
                                          f"(expand-pk inside), MAYO_{s}, OpenMP one instance per thread",
                "keypair_per_s": round(sample / t_kp, 1), "sign_per_s": round(sample / t_sign, 1),
                "verify_per_s": round(sample / t_ver, 1),
                "oracle_check": check([("public key", pk[:n], gpu["pk"][:n]), ("signature", sig[:n], gpu["sig"][:n]),
                                       ("verify byte", res[:n], gpu["res"][:n])], n) if gpu else None}
    if wl["kind"] == "distinct_verify":
        sample = sample or (512 if s == 5 else 1024)
        seeds = seeds_for(1, sample, P.sk_bytes)
        msgs = [bytes(x) for x in chacha(b"mayo-b200-msgs-1".ljust(32, b"\0"), sample * 32).reshape(sample, 32)]
        pk = O.keypair_from_seed_batch(s, seeds)
        sig, _ = O.sign_batch(s, O.expandsk_batch(s, seeds), msgs)
        epk = O.expandpk_batch(s, pk)
        # the GPU's own verify inputs (a tenth corrupted) when given, else the clean signatures
        vin = gpu["sig_in"][:sample] if gpu else sig
        t = time.perf_counter()
        res = O.verify_batch(s, epk, msgs, vin)
        t_ver = time.perf_counter() - t
        if gpu is None:
            assert int(res.sum()) == 0
        return {"value": round(sample / t_ver, 1), "unit": "ops/s", "cores": threads, "kind": "port",
                "sample": f"{sample} distinct-key verifies (expanded keys precomputed), MAYO_{s}, OpenMP one "
                          f"instance per thread",
                "oracle_check": check([("public key", pk, gpu["pk"][:sample]),
                                       ("signature", sig, gpu["good_sig"][:sample]),
                                       ("verify byte", res, gpu["res"][:sample])], sample) if gpu else None}
    return None


# ---------------------------------------------------------------------------------------------
# reference arm: the reference's own CUDA build (oracle/_ref) through its own API
# ---------------------------------------------------------------------------------------------
def run_reference(args, dist: Dist):
    import ctypes

    import torch
    wl = WORKLOADS[args.workload]
    s, batch = wl["set"], args.batch or wl["batch"]
    path = os.path.join(ROOT, "oracle", "_ref", f"libref_mayo{s}.so")
    if not os.path.exists(path):
        return {"impl": "reference", "unavailable": f"{path} not built (make -C oracle ref needs the reference sources)"}
    if wl["kind"] != "shared_sign_verify":
        return run_reference_pool(args, dist, path)
    L = ctypes.CDLL(path)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    for f in ("ref_sign", "ref_verify"):
        getattr(L, f).argtypes = [vp, sz, sz, sz, vp]
    L.ref_keypair.argtypes = [vp, sz, sz, vp, sz]
    L.ref_expandsk.argtypes = [vp, sz, sz, vp]
    L.ref_expandpk.argtypes = [vp, sz, sz, vp]
    L.ref_init()
    torch.cuda.set_device(dist.local)
    dev = torch.device("cuda", dist.local)
    from oracle import oracle as O
    P = O.params(s)
    # the shared key, expanded by the reference itself, then replicated into every pool row
    seed = seeds_for(1 + dist.rank, 1, P.sk_bytes)[0]
    pk = np.frombuffer(O.keypair_from_seed(s, seed.tobytes()), np.uint8)
    kp = torch.zeros(P.esk_bytes + 64, dtype=torch.uint8, device=dev)
    kp[: P.sk_bytes].copy_(torch.from_numpy(seed))
    L.ref_expandsk(kp.data_ptr(), P.esk_bytes, 1, None)
    esk = kp[: P.esk_bytes].clone()
    kq = torch.zeros(P.epk_bytes + 64, dtype=torch.uint8, device=dev)
    kq[P.p_bytes - 16: P.p_bytes - 16 + P.pk_bytes].copy_(torch.from_numpy(pk))
    L.ref_expandpk(kq.data_ptr(), P.epk_bytes, 1, None)
    epk = kq[: P.epk_bytes].clone()
    body, offs, lens = make_messages(1 + dist.rank, batch, *wl["mlen"])
    order = np.argsort(lens, kind="stable")
    maxlen = int(lens.max())
    sp = (P.esk_bytes + maxlen + P.sig_bytes + P.k * P.m * ((P.o + 1) // 2) + 511) // 512 * 512
    vpch = (A128(P.epk_bytes) + A128(maxlen) + A128(P.sig_bytes) + 1 + 511) // 512 * 512
    spool = torch.zeros((batch, sp), dtype=torch.uint8, device=dev)
    vpool = torch.zeros((batch, vpch), dtype=torch.uint8, device=dev)
    spool[:, : P.esk_bytes].copy_(esk.expand(batch, -1))
    vpool[:, : P.epk_bytes].copy_(epk.expand(batch, -1))
    groups = []
    i = 0
    slens = lens[order]
    while i < batch:
        j = i
        while j < batch and slens[j] == slens[i]:
            j += 1
        groups.append((i, j - i, int(slens[i])))
        i = j
    # messages into the rows (sorted by length), the reference's sign layout: msg @ESK
    for r, src in enumerate(order):
        o, n = int(offs[src]), int(lens[src])
        spool[r, P.esk_bytes: P.esk_bytes + n] = torch.from_numpy(body[o:o + n])
        vpool[r, A128(P.epk_bytes): A128(P.epk_bytes) + n] = torch.from_numpy(body[o:o + n])
    streams = [torch.cuda.Stream(device=dev) for _ in range(10)]

    def sign_all():
        for g, (r0, cnt, L_) in enumerate(groups):
            L.ref_sign(spool[r0].data_ptr(), L_, sp, cnt, streams[g % 10].cuda_stream)

    def copy_sigs():
        # reference verify layout: sig @A(EPK) + A(Mlen) (per-group offset)
        for r0, cnt, L_ in groups:
            so = P.esk_bytes + L_
            vo = A128(P.epk_bytes) + A128(L_)
            vpool[r0:r0 + cnt, vo: vo + P.sig_bytes].copy_(spool[r0:r0 + cnt, so: so + P.sig_bytes])

    def verify_all():
        for g, (r0, cnt, L_) in enumerate(groups):
            L.ref_verify(vpool[r0].data_ptr(), L_, vpch, cnt, streams[g % 10].cuda_stream)

    def timed(fn) -> float:
        cur = torch.cuda.current_stream()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cur)
        for sx in streams:
            sx.wait_event(a)
        fn()
        for sx in streams:
            e = torch.cuda.Event()
            e.record(sx)
            cur.wait_event(e)
        b.record(cur)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    for _ in range(args.warmup):
        timed(sign_all)
        copy_sigs()
        torch.cuda.synchronize()
        timed(verify_all)
    dist.barrier()
    ts, tv = [], []
    for _ in range(args.steps):
        ts.append(timed(sign_all))
        copy_sigs()
        torch.cuda.synchronize()
        tv.append(timed(verify_all))
    dist.barrier()
    res_off = [A128(P.epk_bytes) + A128(L_) + A128(P.sig_bytes) for _, _, L_ in groups]
    bad = 0
    for (r0, cnt, _), ro in zip(groups, res_off):
        bad += int(vpool[r0:r0 + cnt, ro].sum().item())
    ms = dist.max((sum(ts) + sum(tv)) / args.steps)
    value = 2 * batch * dist.world / (ms / 1e3)
    per = None
    if dist.world == 1 and getattr(args, "per_set", False):
        del spool, vpool
        torch.cuda.empty_cache()
        per = per_set_measure(args, dist, run_reference)
        m2 = per.setdefault(f"MAYO_{s}", {"mismatches": 0})
        m2["shared_key_batch"] = batch
        m2["shared_sign_per_s"] = round(batch / (sum(ts) / len(ts) / 1e3), 1)
        m2["shared_verify_per_s"] = round(batch / (sum(tv) / len(tv) / 1e3), 1)
        try:
            with open(REF_PER_SET_FILE, "w") as f:
                json.dump({"time": time.time(), "gpu": gpu_identity(dist.local), "per_set": per}, f)
        except OSError:
            pass
    return {"metric": METRIC, "value": round(value, 1), "unit": "ops/s", "impl": "reference", "n_gpus": dist.world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded ChaCha20)",
            "config": {"workload": "MAYO_2 shared-key sign+verify", "set": "MAYO_2", "batch": batch,
                       "msg_len": "uniform 32..1024 B",
                       "key": "expanded key replicated in every pool row (the reference API has no shared key)",
                       "api": "crypto_sign_sign / crypto_sign_verify, one launch per message length, "
                              "round-robin over 10 streams (the reference benchmark's stream pattern)"},
            "sign_per_s": round(batch * dist.world / (sum(ts) / len(ts) / 1e3), 1),
            "verify_per_s": round(batch * dist.world / (sum(tv) / len(tv) / 1e3), 1),
            "launches_per_step": 2 * len(groups), "rejected_valid_signatures": bad, "per_set": per,
            "cpu_baseline": {"value": round(value, 1), "unit": "ops/s", "cores": 0, "kind": "reference",
                             "sample": "not a CPU run: the reference has no CPU implementation; this arm times "
                                       "its own CUDA build on the same B200"},
            "e2e": {"value": round(value, 1), "unit": "ops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def _ref_lib(path):
    import ctypes
    L = ctypes.CDLL(path)
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    L.ref_keypair.argtypes = [vp, sz, sz, vp, sz]
    for f in ("ref_expandsk", "ref_expandpk"):
        getattr(L, f).argtypes = [vp, sz, sz, vp]
    for f in ("ref_sign", "ref_signWithesk", "ref_verify", "ref_verifyWithepk"):
        getattr(L, f).argtypes = [vp, sz, sz, sz, vp]
    L.ref_init()
    return L


def run_reference_pool(args, dist: Dist, path: str):
    """c1 and c3 on the reference's own build, pool API only (the reference generates its keys
    with its counter seeds, since its API takes no caller seed; the work is the same)."""
    import torch
    wl = WORKLOADS[args.workload]
    s, batch = wl["set"], args.batch or wl["batch"]
    from oracle import oracle as O
    P = O.params(s)
    L = _ref_lib(path)
    torch.cuda.set_device(dist.local)
    dev = torch.device("cuda", dist.local)
    cur = torch.cuda.current_stream()
    sptr = cur.cuda_stream
    mlen = wl["mlen"][0]
    rup = lambda x: (x + 511) // 512 * 512  # noqa: E731
    kp = rup(A128(P.sk_bytes) + A128(P.pk_bytes) + A128(P.p_bytes))
    sp = rup(A128(P.esk_bytes) + A128(mlen) + A128(P.sig_bytes) + A128(P.k * P.m * ((P.o + 1) // 2)))
    vp = rup(A128(P.epk_bytes) + A128(mlen) + A128(P.sig_bytes) + 1)
    pk_off, msg_s, msg_v = A128(P.sk_bytes), A128(P.esk_bytes), A128(P.epk_bytes)
    sig_s, sig_v = msg_s + A128(mlen), msg_v + A128(mlen)
    res_off = sig_v + A128(P.sig_bytes)
    msgs = torch.from_numpy(chacha(b"mayo-b200-msgs-1".ljust(32, b"\0"), batch * mlen).reshape(batch, mlen).copy())

    def ev_time(fn) -> float:
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cur)
        fn()
        b.record(cur)
        torch.cuda.synchronize()
        return a.elapsed_time(b)

    if wl["kind"] == "keypair_sign_verify":
        K = torch.zeros((batch, kp), dtype=torch.uint8, device=dev)
        S = torch.zeros((batch, sp), dtype=torch.uint8, device=dev)
        V = torch.zeros((batch, vp), dtype=torch.uint8, device=dev)
        S[:, msg_s: msg_s + mlen].copy_(msgs)
        V[:, msg_v: msg_v + mlen].copy_(msgs)

        def kp_op():
            L.ref_keypair(K.data_ptr(), kp, batch, sptr, 0)

        def sign_op():
            S[:, : P.sk_bytes].copy_(K[:, : P.sk_bytes])
            L.ref_signWithesk(S.data_ptr(), mlen, sp, batch, sptr)

        def verify_op():
            V[:, P.p_bytes - 16: P.p_bytes - 16 + P.pk_bytes].copy_(K[:, pk_off: pk_off + P.pk_bytes])
            V[:, sig_v: sig_v + P.sig_bytes].copy_(S[:, sig_s: sig_s + P.sig_bytes])
            L.ref_verifyWithepk(V.data_ptr(), mlen, vp, batch, sptr)

        phases = [("keypair", kp_op), ("sign", sign_op), ("verify", verify_op)]
        ops = 3 * batch
        expected = np.zeros(batch, np.uint8)
        cfg = {"workload": f"MAYO_{s} keypair -> sign -> verify, distinct keys", "set": f"MAYO_{s}",
               "batch": batch, "msg_len": f"{mlen} B",
               "api": "crypto_sign_keypair / signWithesk / verifyWithepk (counter-seeded keys)"}
    else:
        V = torch.zeros((batch, vp), dtype=torch.uint8, device=dev)
        chunk = 2048
        for c0 in range(0, batch, chunk):
            nb = min(chunk, batch - c0)
            K = torch.zeros((nb, kp), dtype=torch.uint8, device=dev)
            L.ref_keypair(K.data_ptr(), kp, nb, sptr, 2 * c0)
            S = torch.zeros((nb, sp), dtype=torch.uint8, device=dev)
            S[:, : P.sk_bytes].copy_(K[:, : P.sk_bytes])
            S[:, msg_s: msg_s + mlen].copy_(msgs[c0:c0 + nb])
            L.ref_signWithesk(S.data_ptr(), mlen, sp, nb, sptr)
            V[c0:c0 + nb, P.p_bytes - 16: P.p_bytes - 16 + P.pk_bytes].copy_(K[:, pk_off: pk_off + P.pk_bytes])
            V[c0:c0 + nb, sig_v: sig_v + P.sig_bytes].copy_(S[:, sig_s: sig_s + P.sig_bytes])
            del K, S
        L.ref_expandpk(V.data_ptr(), vp, batch, sptr)
        V[:, msg_v: msg_v + mlen].copy_(msgs)
        torch.cuda.synchronize()
        sig = V[:, sig_v: sig_v + P.sig_bytes].cpu().numpy()
        rng = np.random.default_rng(1)
        bad_idx = np.sort(rng.choice(batch, batch // 10, replace=False))
        for i in bad_idx:
            pos = int(rng.integers(0, 2 * P.sig_bytes))
            sig[i, pos // 2] ^= np.uint8(int(rng.integers(1, 16)) << (4 * (pos % 2)))
        V[:, sig_v: sig_v + P.sig_bytes].copy_(torch.from_numpy(sig))
        expected = np.zeros(batch, np.uint8)
        expected[bad_idx] = 1

        def verify_op():
            L.ref_verify(V.data_ptr(), mlen, vp, batch, sptr)

        phases = [("verify", verify_op)]
        ops = batch
        cfg = {"workload": f"MAYO_{s} distinct-key verify", "set": f"MAYO_{s}", "batch": batch,
               "msg_len": f"{mlen} B", "corrupted": "10%", "api": "crypto_sign_verify (epk resident in the pool)"}
    for _ in range(args.warmup):
        for _, fn in phases:
            fn()
    torch.cuda.synchronize()
    dist.barrier()
    per = {name: 0.0 for name, _ in phases}
    for _ in range(args.steps):
        for name, fn in phases:
            per[name] += ev_time(fn)
    dist.barrier()
    mism = int((V[:, res_off].cpu().numpy() != expected).sum())
    ms = dist.max(sum(per.values()) / args.steps)
    value = ops * dist.world / (ms / 1e3)
    out = {"metric": METRIC, "value": round(value, 1), "unit": "ops/s", "impl": "reference", "n_gpus": dist.world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded ChaCha20 messages)",
           "config": cfg, "phase_ms": {k: round(v / args.steps, 3) for k, v in per.items()},
           "result_mismatches": mism,
           "cpu_baseline": {"value": round(value, 1), "unit": "ops/s", "cores": 0, "kind": "reference",
                            "sample": "not a CPU run: the reference has no CPU implementation; this arm times its "
                                      "own CUDA build on the same B200"},
           "e2e": {"value": round(value, 1), "unit": "ops/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    for name in per:
        out[f"{name}_per_s"] = round(batch * dist.world / (per[name] / args.steps / 1e3), 1)
    return out


# ---------------------------------------------------------------------------------------------
# C5: serving (open-loop Poisson arrivals, continuous batching, resident key cache)
# ---------------------------------------------------------------------------------------------
SERVE_MIX = {1: 0.4, 2: 0.3, 3: 0.2, 5: 0.1}
SERVE_KEYS = {1: 1638, 2: 1229, 3: 819, 5: 410}  # 4096 resident keys at the set mix


def serving_stream(seed: int, rate: float, n: int, n_tmpl: dict, tmpl_base: dict):
    """n requests at `rate`/s: ChaCha20-driven exponential gaps; 70 % verify / 30 % sign; sets
    40/30/20/10; a uniform request template of the set; 1 % of verifies carry a corrupted
    signature.  Returns (arrivals, op, template index, corrupted)."""
    from cumayo_b200 import queue as Q
    from cumayo_b200 import serving as SV
    arr = SV.poisson_arrivals(rate, n, (b"c5-arrivals-%d-%d" % (seed, int(rate))).ljust(32, b"\0")[:32])
    u = chacha((b"c5-requests-%d-%d" % (seed, int(rate))).ljust(32, b"\0")[:32], 16 * n).view(np.uint32).reshape(n, 4)
    f = (u.astype(np.float64) + 0.5) / 2.0 ** 32
    op = np.where(f[:, 0] < 0.7, Q.OP_VERIFY, Q.OP_SIGN).astype(np.uint8)
    cum = np.cumsum([SERVE_MIX[s] for s in (1, 2, 3, 5)])
    set_id = np.array([1, 2, 3, 5])[np.searchsorted(cum, f[:, 1] * cum[-1], side="right").clip(0, 3)]
    base = np.array([tmpl_base[s] for s in set_id])
    cnt = np.array([n_tmpl[s] for s in set_id])
    tidx = base + (u[:, 2] % cnt.astype(np.uint32)).astype(np.int64)
    bad = (op == Q.OP_VERIFY) & (f[:, 3] < 0.01)
    return arr, op, tidx, bad


def run_serving(args, dist: Dist):
    import torch

    import cumayo_b200 as M
    from cumayo_b200 import queue as Q
    from cumayo_b200 import serving as SV
    dev = torch.device("cuda", dist.local)
    torch.cuda.set_device(dev)
    st = torch.cuda.current_stream()
    seed = 1 + dist.rank
    max_msg, budget = 256, 60 << 30
    max_batch = args.batch or WORKLOADS["c5"]["batch"]
    sets = (1, 2, 3, 5)

    # keys (all resident: 4096 keys ~ 2 GB of esk + epk, far inside the budget)
    seeds = {s: seeds_for(seed * 100 + s, SERVE_KEYS[s], M.sizes(s).sk_bytes) for s in sets}
    key_slots = SV.capacity_for_budget(budget // 2, SERVE_KEYS)
    server = SV.Server(seeds, key_slots=key_slots, max_batch=max_batch, inflight=args.inflight, max_msg=max_msg,
                       budget_bytes=budget, device=dev)
    for s in sets:  # load every key once, outside the timed runs
        server.preload(s, np.arange(SERVE_KEYS[s]))
    key_cache_bytes = sum(key_slots[s] * (M.sizes(s).esk_bytes + M.sizes(s).epk_bytes) for s in sets)

    # request templates: per set 4096 (key, message) pairs and their signatures, computed by the
    # server itself; a sample is checked against the plain batched sign_many below
    n_tmpl = {s: 4096 for s in sets}
    tmpl_base, tset, tkey, tmlen, tmsg = {}, [], [], [], []
    b = 0
    for s in sets:
        tmpl_base[s] = b
        b += n_tmpl[s]
        raw = chacha((b"c5-templates-%d-%d" % (seed, s)).ljust(32, b"\0")[:32], 8 * n_tmpl[s]).view(np.uint32)
        tset.append(np.full(n_tmpl[s], s, np.int64))
        tkey.append((raw[0::2] % SERVE_KEYS[s]).astype(np.int64))
        tmlen.append((32 + raw[1::2] % (max_msg - 31)).astype(np.uint32))
        tmsg.append(chacha((b"c5-msgs-%d-%d" % (seed, s)).ljust(32, b"\0")[:32], n_tmpl[s] * max_msg)
                    .reshape(n_tmpl[s], max_msg))
    tset, tkey, tmlen, tmsg = (np.concatenate(x) for x in (tset, tkey, tmlen, tmsg))
    T = tset.size
    tset = tset.astype(np.uint8)
    tsig = np.zeros((T, SV.MAX_SIG), np.uint8)
    ROW_MSG, ROW_SIG = np.uint64(max_msg), np.uint64(SV.MAX_SIG)

    # template signatures, written by the server straight into tsig
    for lo in range(0, T, max_batch):
        rows = np.arange(lo, min(T, lo + max_batch), dtype=np.uint64)
        r = SV.make_requests(np.full(rows.size, Q.OP_SIGN, np.uint8), tset[rows], tkey[rows], tmlen[rows],
                             tmsg.ctypes.data + rows * ROW_MSG, 0, tsig.ctypes.data + rows * ROW_SIG)
        server.submit(r, lo)
        server.drain()
    server.check_queue()
    tbad = tsig.copy()
    tbad[:, 7] ^= 0x40  # every template's signature, corrupted
    # cross-check: 64 templates per set through the plain batched path (keys expanded by the pool API)
    plain_bad = 0
    for s in sets:
        z = M.sizes(s)
        m_ = M.Mayo(s)
        rows = tmpl_base[s] + np.arange(64)
        kp, kpitch = m_.alloc_pool("keypair", 64)
        kp.view(64, kpitch)[:, : z.sk_bytes].copy_(torch.from_numpy(seeds[s][tkey[rows]]))
        m_.crypto_sign_keypair_from_seed(kp, kpitch, 64, st)
        esk = torch.zeros(64 * z.esk_bytes, dtype=torch.uint8, device=dev)
        esk.view(64, z.esk_bytes)[:, : z.sk_bytes].copy_(kp.view(64, kpitch)[:, : z.sk_bytes])
        m_.crypto_sign_expandsk(esk, z.esk_bytes, 64, st)
        msgs = torch.from_numpy(tmsg[rows].copy()).to(dev)
        lens = torch.from_numpy(tmlen[rows].astype(np.int32)).to(dev)
        offs = torch.arange(64, dtype=torch.int64, device=dev) * max_msg
        sig = torch.zeros(64 * z.sig_bytes, dtype=torch.uint8, device=dev)
        ws = torch.zeros(64 * m_.sign_ws_bytes(), dtype=torch.uint8, device=dev)
        m_.sign_many(esk, msgs.reshape(-1), sig, ws, 64, esk_stride=z.esk_bytes, msg_off=offs, msg_len=lens, stream=st)
        plain_bad += int((sig.cpu().numpy().reshape(64, z.sig_bytes) != tsig[rows, : z.sig_bytes]).any(1).sum())

    mismatches = [plain_bad]
    sig_len = np.array([M.sizes(int(x)).sig_bytes if x in sets else 0 for x in range(6)], np.int64)

    def runner(arr, op, tidx, bad):
        """The open-loop run of the native server over these requests; every result checked."""
        n = arr.size
        t = tidx.astype(np.uint64)
        sg = op == Q.OP_SIGN
        out_len = np.where(sg, sig_len[tset[tidx]], 1)
        out_off = np.zeros(n, np.int64)
        out_off[1:] = np.cumsum(out_len[:-1])
        out = np.zeros(int(out_len.sum()) + 1, np.uint8)
        sig_base = np.where(bad, np.uint64(tbad.ctypes.data), np.uint64(tsig.ctypes.data))
        r = SV.make_requests(op, tset[t], tkey[t], tmlen[t], tmsg.ctypes.data + t * ROW_MSG, sig_base + t * ROW_SIG,
                             np.uint64(out.ctypes.data) + out_off.astype(np.uint64))
        s0 = server.stats()
        lat, _ = server.run_open_loop(r, arr)
        s1 = server.stats()
        nb = 0
        for s_ in sets:
            rows = np.flatnonzero(sg & (tset[tidx] == s_))
            sb = int(sig_len[s_])
            got = out[out_off[rows][:, None] + np.arange(sb)]
            nb += int((got != tsig[tidx[rows], :sb]).any(1).sum())
        nb += int((out[out_off[~sg]] != bad[~sg].astype(np.uint8)).sum())
        nb += int(np.isnan(lat).sum())
        mismatches[0] += nb
        batches = s1["batches"] - s0["batches"]
        admitted = s1["requests_admitted"] - s0["requests_admitted"]
        return lat, float(np.nanmax(lat + arr)), (batches, admitted, s1["max_batch_seen"]), batches

    # closed-loop batched peak through the same path (every request waiting from t = 0)
    n_peak = max_batch * 12
    arr, op, tidx, bad = serving_stream(seed, 1e12, n_peak, n_tmpl, tmpl_base)
    arr[:] = 0.0
    runner(arr, op, tidx, bad)  # warm-up
    lat, span, bs, _ = runner(arr, op, tidx, bad)
    peak = n_peak / span

    # plain per-(set, op) batched launches of the same mix (one shared key per set, device inputs)
    counts = {(s, o): int(((tset[tidx] == s) & (op == o)).sum()) for s in sets for o in (Q.OP_SIGN, Q.OP_VERIFY)}
    plain_parts = []
    for s in sets:
        z = M.sizes(s)
        esk, epk = expand_shared_key(M.Mayo(s), seeds[s][0], dev, st)
        nmax = max(counts[(s, Q.OP_SIGN)], counts[(s, Q.OP_VERIFY)], 1)
        msgs = torch.from_numpy(np.resize(tmsg[tmpl_base[s]: tmpl_base[s] + n_tmpl[s]], (nmax, max_msg))).to(dev)
        lens = torch.from_numpy(np.resize(tmlen[tmpl_base[s]: tmpl_base[s] + n_tmpl[s]], nmax).astype(np.int32)).to(dev)
        offs = torch.arange(nmax, dtype=torch.int64, device=dev) * max_msg
        sig = torch.zeros(nmax * z.sig_bytes, dtype=torch.uint8, device=dev)
        ws = torch.zeros(nmax * M.Mayo(s).sign_ws_bytes(), dtype=torch.uint8, device=dev)
        res = torch.zeros(nmax, dtype=torch.uint8, device=dev)
        plain_parts.append((M.Mayo(s), esk, epk, msgs, offs, lens, sig, ws, res, counts[(s, Q.OP_SIGN)],
                            counts[(s, Q.OP_VERIFY)]))

    def plain():
        for m, esk, epk, msgs, offs, lens, sig, ws, res, ns, nv in plain_parts:
            if ns:
                m.sign_many(esk, msgs.reshape(-1), sig, ws, ns, msg_off=offs, msg_len=lens, stream=st)
            if nv:
                m.verify_many(epk, msgs.reshape(-1), sig, res, nv, msg_off=offs, msg_len=lens, stream=st)

    plain()
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(st)
    for _ in range(3):
        plain()
    p1.record(st)
    torch.cuda.synchronize()
    plain_peak = n_peak * 3 / (p0.elapsed_time(p1) / 1e3)

    # open-loop sweep
    target = 0.8 * peak
    rates = sorted({5e4, 2e5, 5e5, 1e6, round(target, -3), round(0.9 * peak, -3), 2e6})
    sweep, head = [], None
    clocks = Clocks(dist.local)
    clocks.start()
    l0 = server.stats()["kernel_launches"]
    for rate in rates:
        n = int(min(rate * 0.5, 1.2e6))
        arr, op, tidx, bad = serving_stream(seed, rate, n, n_tmpl, tmpl_base)
        lat, span, bs, nb = runner(arr, op, tidx, bad)
        row = dict(SV.latency_stats(lat), offered_per_s=rate, served_per_s=round(n / span, 1),
                   batches=int(nb), mean_batch=round(bs[1] / max(bs[0], 1), 1), max_batch=int(bs[2]))
        sweep.append(row)
        if rate == round(target, -3):
            head = row
    clk = clocks.stop()
    mean_sig = sum(SERVE_MIX[s] * M.sizes(s).sig_bytes for s in sets)
    bytes_in = 4 + 4 + 4 + float(tmlen.mean()) + 0.7 * mean_sig  # item, key slot, length, message, signature
    bytes_out = 0.3 * mean_sig + 0.7
    out = {
        "metric": METRIC, "value": head["served_per_s"], "unit": "req/s", "n_gpus": dist.world,
        "steps": len(rates), "warmup": 1, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (GF(16) bit-planes)", "data": "synthetic (seeded ChaCha20)",
        "config": {"workload": "serving: open-loop Poisson arrivals, 70 % verify / 30 % sign, sets 40/30/20/10, "
                               "4096 resident keys, continuous batching over the persistent queue",
                   "max_batch": max_batch, "inflight_batches": args.inflight, "msg_len": f"32..{max_msg} B",
                   "key_cache_bytes": key_cache_bytes, "device_bytes": server.device_bytes, "budget_bytes": budget,
                   "loop": "native (mayo_b200_server_run_open_loop, C++)",
                   "value": "requests/s served at an offered load of 0.8 x the closed-loop batched peak"},
        "p50_ms": head["p50_ms"], "p99_ms": head["p99_ms"], "p999_ms": head["p999_ms"],
        "offered_per_s": head["offered_per_s"],
        "batched_peak_per_s": round(peak, 1), "plain_batched_peak_per_s": round(plain_peak, 1),
        "sweep": sweep,
        "e2e": {"value": head["served_per_s"], "unit": "req/s",
                "h2d_bytes_per_step": int(bytes_in * head["n"] / max(head.get("batches", 1), 1)),
                "d2h_bytes_per_step": int(bytes_out * head["n"] / max(head.get("batches", 1), 1)),
                "note": "every number here is end to end (host request buffers in, host results out); "
                        "a step is one admitted batch"},
        "roofline": None,
        "gpu_launches": server.stats()["kernel_launches"] - l0,
        "clocks": clk,
        "result_mismatches": mismatches[0],
    }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--inflight", type=int, default=6, help="c5: batches on the GPU at once")
    ap.add_argument("--e2e-chunks", type=int, default=8,
                    help="c2: sub-batches (one stream each) of the value_streams measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--shape", default="",
                    help="c2: shared-key block shape HASHxTAIL[xPAIR] (hash CTA threads x signatures per tail CTA "
                         "x CTAs per product tile) instead of the autotuner's choice, e.g. 64x4x2")
    ap.add_argument("--no-per-set", dest="per_set", action="store_false",
                    help="skip the per-set keypair/sign/verify and distinct-key verify figures (default run)")
    ap.add_argument("--int-peak", action="store_true",
                    help="build and run bench_int_pipes.cu (integer-pipe rates) and exit")
    args = ap.parse_args()
    if args.int_peak:
        from cumayo_b200.build import ARCH, BUILD, nvcc
        os.makedirs(BUILD, exist_ok=True)
        exe = os.path.join(BUILD, "int_pipes")
        subprocess.run([nvcc()] + ARCH + ["-O3", "-o", exe, os.path.join(ROOT, "bench_int_pipes.cu")],
                       check=True)
        subprocess.run([exe], check=True)
        return
    dist = Dist()
    try:
        if args.impl == "reference":
            out = run_reference(args, dist)
        elif WORKLOADS[args.workload]["kind"] == "serving":
            out = run_serving(args, dist)
        else:
            out = run_ours(args, dist)
    finally:
        dist.close()
    if dist.rank == 0:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
