"""Serving loop for MAYO sign / verify requests on one GPU: continuous batching over the
persistent work queue, with the expanded keys resident in HBM under a byte budget.

Requests arrive one by one (an open-loop Poisson stream in the benchmark).  The server keeps up
to `inflight` batches on the GPU, each on its own stream with its own queue memory and staging
buffers.  Whenever a batch slot is free and requests are waiting, the waiting requests (up to
`max_batch`, oldest first) are admitted as one batch: their inputs are packed into one pinned
host buffer and copied to the device in one transfer, the queue partitions the batch by
(set, op) on the device and drains it with the per-(set, op) persistent kernels, and one
transfer brings the signatures and verify results back.  A request's latency is the time from
its arrival to the host seeing its batch's results.

Keys are registered per parameter set by id (their seeds) and expanded (esk for signing, epk for
verifying) on first use into a per-set table in HBM.  A full table evicts its least recently used
keys that no in-flight batch references.  Admission is bounded by the tables too: a batch takes
the longest prefix of the waiting requests whose keys fit beside the keys in-flight batches hold
(launch() itself raises CacheFull for a batch that does not fit).

This module has no counterpart in the reference, which offers only the synchronous batched pool
API (include/api.cuh).
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import queue as Q
from .api import A128, Mayo, MayoError, _check, lib, sizes

SETS = (1, 2, 3, 5)
MAX_SIG = max(sizes(s).sig_bytes for s in SETS)


class CacheFull(MayoError):
    pass


def _align(x: int, a: int = 16) -> int:
    return (x + a - 1) // a * a


# ---------------------------------------------------------------------------------------------
# key table bookkeeping (host only)
# ---------------------------------------------------------------------------------------------
class SlotTable:
    """Key id -> slot map of one parameter set's key table, least-recently-used eviction.

    `acquire` maps a batch's key ids to slots, choosing slots for the keys that are not resident
    (empty slots first, then the least recently used unpinned ones, never one this batch uses)
    and pins every slot the batch uses until `release`."""

    def __init__(self, capacity: int, n_keys: int):
        if capacity <= 0:
            raise MayoError("key table needs at least one slot")
        self.capacity = capacity
        self.slot_of = np.full(n_keys, -1, np.int64)
        self.key_of = np.full(capacity, -1, np.int64)
        self.last = np.zeros(capacity, np.int64)
        self.pins = np.zeros(capacity, np.int64)
        self.tick = 0
        self.misses = 0
        self.evictions = 0

    def acquire(self, key_ids: np.ndarray):
        """Returns (slot per key id, missing key ids, their new slots, slots to release).  The
        release handle may repeat slots: `pins[idx] += 1` with repeated indices adds once per
        distinct slot, which is the one pin per batch wanted."""
        key_ids = np.asarray(key_ids, np.int64)
        if key_ids.size and (key_ids.min() < 0 or key_ids.max() >= self.slot_of.size):
            raise MayoError("unknown key id")
        self.tick += 1
        slots = self.slot_of[key_ids]
        miss = np.zeros(0, np.int64)
        new_slots = np.zeros(0, np.int64)
        if (slots < 0).any():
            miss = np.unique(key_ids[slots < 0])
            cand_mask = self.pins == 0
            cand_mask[slots[slots >= 0]] = False
            cand = np.flatnonzero(cand_mask)
            if cand.size < miss.size:
                raise CacheFull(f"{miss.size} keys to load, {cand.size} slots free of in-flight batches")
            pri = np.where(self.key_of[cand] < 0, -1, self.last[cand])
            pick = cand if cand.size == miss.size else cand[np.argpartition(pri, miss.size - 1)[:miss.size]]
            old = self.key_of[pick]
            self.evictions += int((old >= 0).sum())
            self.slot_of[old[old >= 0]] = -1
            self.key_of[pick] = miss
            self.slot_of[miss] = pick
            self.misses += int(miss.size)
            new_slots = pick
            slots = self.slot_of[key_ids]
        self.last[slots] = self.tick
        self.pins[slots] += 1
        return slots, miss, new_slots, slots

    def release(self, su: np.ndarray) -> None:
        self.pins[su] -= 1

    def can_load(self, key_ids: np.ndarray) -> bool:
        """Whether acquire(key_ids) would find slots for its missing keys (no state change)."""
        key_ids = np.asarray(key_ids, np.int64)
        slots = self.slot_of[key_ids]
        if (slots >= 0).all():
            return True
        nmiss = int(np.unique(key_ids[slots < 0]).size)
        used = np.unique(slots[slots >= 0])
        free = int((self.pins == 0).sum()) - int((self.pins[used] == 0).sum())
        return free >= nmiss


class KeyCache:
    """Expanded keys resident in HBM: per parameter set, a table of `capacity[set]` esk rows and
    as many epk rows, filled on first use from the registered seeds.  Expansion runs on the
    stream of the batch that needs the keys; every later batch waits for it."""

    def __init__(self, seeds: dict, capacity: dict, device=None):
        import torch
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.seeds = {s: np.ascontiguousarray(v, np.uint8) for s, v in seeds.items()}
        self.tables, self.esk, self.epk, self.mayo = {}, {}, {}, {}
        for s, sd in self.seeds.items():
            z = sizes(s)
            cap = int(min(capacity[s], len(sd)))
            self.tables[s] = SlotTable(cap, len(sd))
            self.esk[s] = torch.zeros(cap * z.esk_bytes, dtype=torch.uint8, device=self.dev)
            self.epk[s] = torch.zeros(cap * z.epk_bytes, dtype=torch.uint8, device=self.dev)
            self.mayo[s] = Mayo(s)
        self.ready = None  # event after the last expansion

    @staticmethod
    def capacity_for_budget(budget_bytes: int, n_keys: dict) -> dict:
        """Slots per set: all keys if they fit, else the budget split by each set's key bytes."""
        need = {s: n * (sizes(s).esk_bytes + sizes(s).epk_bytes) for s, n in n_keys.items()}
        total = sum(need.values())
        if total <= budget_bytes:
            return dict(n_keys)
        return {s: max(1, int(n_keys[s] * budget_bytes / total)) for s in n_keys}

    def nbytes(self) -> int:
        return sum(int(t.numel()) for t in self.esk.values()) + sum(int(t.numel()) for t in self.epk.values())

    def acquire(self, set_id: int, key_ids: np.ndarray, stream):
        slots, miss, new_slots, su = self.tables[set_id].acquire(key_ids)
        if miss.size:
            self._expand(set_id, miss, new_slots, stream)
        return slots, su

    def release(self, set_id: int, su: np.ndarray) -> None:
        self.tables[set_id].release(su)

    def wait(self, stream) -> None:
        if self.ready is not None:
            stream.wait_event(self.ready)

    def _expand(self, s: int, key_ids: np.ndarray, slots: np.ndarray, stream) -> None:
        """seed -> (pk via keypair_from_seed) -> esk, epk, written into the given slots."""
        import torch
        m, z = self.mayo[s], sizes(s)
        n = int(key_ids.size)
        with torch.cuda.stream(stream):
            seeds = torch.from_numpy(self.seeds[s][key_ids]).to(self.dev, non_blocking=False)
            kp, kpitch = m.alloc_pool("keypair", n, device=self.dev)
            kp.view(n, kpitch)[:, : z.sk_bytes].copy_(seeds)
            m.crypto_sign_keypair_from_seed(kp, kpitch, n, stream)
            esk = torch.zeros(n * z.esk_bytes, dtype=torch.uint8, device=self.dev)
            esk.view(n, z.esk_bytes)[:, : z.sk_bytes].copy_(seeds)
            m.crypto_sign_expandsk(esk, z.esk_bytes, n, stream)
            epk = torch.zeros(n * z.epk_bytes, dtype=torch.uint8, device=self.dev)
            pk_off = A128(z.sk_bytes)
            epk.view(n, z.epk_bytes)[:, z.p_bytes - 16: z.p_bytes - 16 + z.pk_bytes].copy_(
                kp.view(n, kpitch)[:, pk_off: pk_off + z.pk_bytes])
            m.crypto_sign_expandpk(epk, z.epk_bytes, n, stream)
            idx = torch.from_numpy(slots).to(self.dev)
            self.esk[s].view(-1, z.esk_bytes).index_copy_(0, idx, esk.view(n, z.esk_bytes))
            self.epk[s].view(-1, z.epk_bytes).index_copy_(0, idx, epk.view(n, z.epk_bytes))
            ev = torch.cuda.Event()
            ev.record(stream)
        self.ready = ev


# ---------------------------------------------------------------------------------------------
# batch staging (host only; native: mayo_b200_serve_pack / _unpack)
# ---------------------------------------------------------------------------------------------
# mayo_b200_serve_req: one request, pointing into the caller's host memory
REQ_DTYPE = np.dtype([("msg", "<u8"), ("sig", "<u8"), ("out", "<u8"), ("mlen", "<u4"), ("key_id", "<u4"),
                      ("key_slot", "<u4"), ("op", "u1"), ("set", "u1"), ("pad", "u1", (2,))])
assert REQ_DTYPE.itemsize == 40


class _Group(ctypes.Structure):
    _fields_ = [("count", ctypes.c_uint32), ("set", ctypes.c_uint32), ("op", ctypes.c_uint32), ("pad", ctypes.c_uint32),
                ("key_off", ctypes.c_uint64), ("len_off", ctypes.c_uint64), ("msg_off", ctypes.c_uint64),
                ("sig_off", ctypes.c_uint64), ("out_off", ctypes.c_uint64)]


class Layout(ctypes.Structure):
    """mayo_b200_serve_layout: where pack() put each (set, op) group."""
    _fields_ = [("n", ctypes.c_uint32), ("max_msg", ctypes.c_uint32), ("in_bytes", ctypes.c_uint64),
                ("out_bytes", ctypes.c_uint64), ("group", _Group * 8)]


def _bind():
    L = lib()
    if not getattr(L, "_serve_bound", False):
        L.mayo_b200_serve_in_bytes.restype = ctypes.c_size_t
        L.mayo_b200_serve_in_bytes.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.mayo_b200_serve_out_bytes.restype = ctypes.c_size_t
        L.mayo_b200_serve_out_bytes.argtypes = [ctypes.c_uint32]
        L.mayo_b200_serve_pack.restype = ctypes.c_int
        L.mayo_b200_serve_pack.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p,
                                           ctypes.c_size_t, ctypes.c_size_t, ctypes.POINTER(Layout)]
        L.mayo_b200_serve_unpack.restype = ctypes.c_int
        L.mayo_b200_serve_unpack.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(Layout), ctypes.c_void_p]
        L._serve_bound = True
    return L


def make_requests(op, set_id, key_id, mlen, msg_ptr, sig_ptr, out_ptr) -> np.ndarray:
    """Request records from per-request columns (pointers as integers)."""
    n = int(np.asarray(op).shape[0])
    r = np.zeros(n, REQ_DTYPE)
    r["op"], r["set"], r["key_id"], r["mlen"] = op, set_id, key_id, mlen
    r["msg"], r["sig"], r["out"] = msg_ptr, sig_ptr, out_ptr
    return r


def requests_from_rows(op, set_id, key_id, mlen, msg: np.ndarray, sig: np.ndarray, out: np.ndarray) -> np.ndarray:
    """Request records whose message, signature and output are row i of C-contiguous 2-D uint8
    arrays (the caller keeps the arrays alive until the batch is unpacked)."""
    n = int(np.asarray(op).shape[0])
    for a in (msg, sig, out):
        if not a.flags["C_CONTIGUOUS"] or a.dtype != np.uint8 or a.ndim != 2 or a.shape[0] < n:
            raise MayoError("rows must be C-contiguous 2-D uint8 arrays")
    i = np.arange(n, dtype=np.uint64)
    return make_requests(op, set_id, key_id, mlen, msg.ctypes.data + i * np.uint64(msg.shape[1]),
                         sig.ctypes.data + i * np.uint64(sig.shape[1]), out.ctypes.data + i * np.uint64(out.shape[1]))


def in_bytes(n: int, max_msg: int) -> int:
    return int(_bind().mayo_b200_serve_in_bytes(n, max_msg))


def out_bytes(n: int) -> int:
    return int(_bind().mayo_b200_serve_out_bytes(n))


def pack(reqs: np.ndarray, max_msg: int, stage_in: np.ndarray, out_capacity: int) -> Layout:
    """Packs request records (key_slot filled) into stage_in (uint8, host); returns the layout."""
    lay = Layout()
    _check(_bind().mayo_b200_serve_pack(reqs.ctypes.data, reqs.size, max_msg, stage_in.ctypes.data, stage_in.size,
                                        out_capacity, ctypes.byref(lay)), "serve_pack")
    return lay


def unpack(reqs: np.ndarray, lay: Layout, stage_out: np.ndarray) -> None:
    """Copies each request's signature / verify result from stage_out to its `out`."""
    _check(_bind().mayo_b200_serve_unpack(reqs.ctypes.data, reqs.size, ctypes.byref(lay), stage_out.ctypes.data),
           "serve_unpack")


def poisson_arrivals(rate: float, n: int, key: bytes) -> np.ndarray:
    """Arrival times (seconds) of n requests at `rate` per second: exponential gaps driven by a
    ChaCha20 keystream (32-byte key)."""
    from cryptography.hazmat.primitives.ciphers import Cipher, algorithms
    enc = Cipher(algorithms.ChaCha20(key, b"\0" * 16), mode=None).encryptor()
    u = np.frombuffer(enc.update(b"\0" * (8 * n)), np.uint64)
    x = ((u >> np.uint64(11)).astype(np.float64) + 0.5) * (1.0 / (1 << 53))  # (0, 1)
    return np.cumsum(-np.log(x) / rate)


def latency_stats(lat: np.ndarray) -> dict:
    lat = lat[np.isfinite(lat)] * 1e3
    if lat.size == 0:
        return {"n": 0}
    return {"n": int(lat.size), "p50_ms": float(np.percentile(lat, 50)), "p90_ms": float(np.percentile(lat, 90)),
            "p99_ms": float(np.percentile(lat, 99)), "p999_ms": float(np.percentile(lat, 99.9)),
            "max_ms": float(lat.max()), "mean_ms": float(lat.mean())}


# ---------------------------------------------------------------------------------------------
# the server
# ---------------------------------------------------------------------------------------------
class _Slot:
    def __init__(self, server, idx):
        import torch
        self.idx = idx
        self.stream = torch.cuda.Stream(device=server.dev)
        self.queue = Q.Queue(capacity=server.max_batch + server.max_batch // 8 + 64, device=server.dev)
        self.h_in = torch.empty(server.in_bytes, dtype=torch.uint8).pin_memory()
        self.h_out = torch.empty(server.out_bytes, dtype=torch.uint8).pin_memory()
        self.d_in = torch.empty(server.in_bytes, dtype=torch.uint8, device=server.dev)
        self.d_out = torch.empty(server.out_bytes, dtype=torch.uint8, device=server.dev)
        self.in_np = self.h_in.numpy()
        self.out_np = self.h_out.numpy()
        self.event = torch.cuda.Event()
        self.busy = False
        self.tag = self.keep = self.reqs = self.layout = None
        self.pins = []


class Server:
    """Continuous-batching MAYO sign / verify server on one GPU.

    max_batch requests per batch, `inflight` batches on the GPU at once, messages up to
    max_msg bytes.  Device memory: the key cache plus, per in-flight batch, the queue memory and
    the staging buffers; `budget_bytes` bounds the total (MayoError if it does not fit)."""

    def __init__(self, cache: KeyCache, max_batch: int = 4096, inflight: int = 2, max_msg: int = 256,
                 budget_bytes: int = 60 << 30):
        self.cache = cache
        self.dev = cache.dev
        self.max_batch = max_batch
        self.max_msg = max_msg
        self.in_bytes = in_bytes(max_batch, max_msg)
        self.out_bytes = out_bytes(max_batch)
        self.slots = [_Slot(self, i) for i in range(inflight)]
        self.device_bytes = cache.nbytes() + sum(int(s.queue.mem.numel()) + int(s.queue.items.numel()) * 4 +
                                                 self.in_bytes + self.out_bytes for s in self.slots)
        if self.device_bytes > budget_bytes:
            raise MayoError(f"server needs {self.device_bytes} device bytes, budget {budget_bytes}")
        self.batches = 0
        self.kernel_launches = 0

    def free_slot(self):
        for s in self.slots:
            if not s.busy:
                return s
        return None

    def fits(self, reqs: np.ndarray, k: int) -> bool:
        """Whether the first k requests' keys can all be made resident now."""
        for s in SETS:
            rows = reqs["set"][:k] == s
            if rows.any() and not self.cache.tables[s].can_load(reqs["key_id"][:k][rows]):
                return False
        return True

    def admit_len(self, reqs: np.ndarray) -> int:
        """The longest prefix of reqs (at most max_batch) whose keys fit in the key tables beside
        the keys in-flight batches hold; 0 = wait for a batch to finish."""
        k = min(int(reqs.size), self.max_batch)
        if self.fits(reqs, k):
            return k
        lo, hi = 0, k  # fits(lo) holds, fits(hi) does not
        while hi - lo > 1:
            mid = (lo + hi) // 2
            if self.fits(reqs, mid):
                lo = mid
            else:
                hi = mid
        return lo

    def launch(self, reqs: np.ndarray, tag=None, keep=None) -> _Slot:
        """Admit one batch of request records (REQ_DTYPE; asynchronous).  The records and the
        memory they point to (`keep` holds whatever must stay alive) belong to the server until
        poll() returns the batch.  Raises if no slot is free or the keys do not fit."""
        import torch
        slot = self.free_slot()
        if slot is None:
            raise MayoError("no free batch slot")
        n = int(reqs.size)
        if n == 0 or n > self.max_batch:
            raise MayoError(f"batch of {n} requests (max {self.max_batch})")
        st = slot.stream
        pins = []
        try:
            for s in SETS:
                rows = np.flatnonzero(reqs["set"] == s)
                if rows.size:
                    ks, su = self.cache.acquire(s, reqs["key_id"][rows], st)
                    pins.append((s, su))
                    reqs["key_slot"][rows] = ks
            lay = pack(reqs, self.max_msg, slot.in_np, slot.out_np.size)
        except Exception:
            for s, su in pins:
                self.cache.release(s, su)
            raise
        q = slot.queue
        base_in, base_out = slot.d_in.data_ptr(), slot.d_out.data_ptr()
        ops = {s: Q.SetOperands(kp_count=0, sg_count=0, vf_count=0) for s in SETS}
        groups = 0
        for g in lay.group:
            if not g.count:
                continue
            groups += 1
            o, tab = ops[g.set], self.cache.tables[g.set]
            if g.op == Q.OP_SIGN:
                o.sg_esk, o.sg_nkeys, o.sg_key = self.cache.esk[g.set], tab.capacity, base_in + g.key_off
                o.sg_msg, o.sg_msg_len, o.sg_mlen = base_in + g.msg_off, base_in + g.len_off, self.max_msg
                o.sg_sig, o.sg_count = base_out + g.out_off, g.count
            else:
                o.vf_epk, o.vf_nkeys, o.vf_key = self.cache.epk[g.set], tab.capacity, base_in + g.key_off
                o.vf_msg, o.vf_msg_len, o.vf_mlen = base_in + g.msg_off, base_in + g.len_off, self.max_msg
                o.vf_sig, o.vf_res, o.vf_count = base_in + g.sig_off, base_out + g.out_off, g.count
        for s, o in ops.items():
            q.set_operands(s, o)
        with torch.cuda.stream(st):
            self.cache.wait(st)
            slot.d_in[: lay.in_bytes].copy_(slot.h_in[: lay.in_bytes], non_blocking=True)
            q.run_items(base_in, n, stream=st)
            slot.h_out[: lay.out_bytes].copy_(slot.d_out[: lay.out_bytes], non_blocking=True)
            slot.event.record(st)
        slot.busy, slot.tag, slot.keep, slot.reqs, slot.layout, slot.pins = True, tag, keep, reqs, lay, pins
        self.batches += 1
        self.kernel_launches += 2 + groups  # queue fill + partition + one persistent kernel per group
        return slot

    def poll(self):
        """Finished batches, their results unpacked into the requests' `out`: [(tag, keep)]."""
        done = []
        for slot in self.slots:
            if slot.busy and slot.event.query():
                unpack(slot.reqs, slot.layout, slot.out_np)
                done.append((slot.tag, slot.keep))
                for s, su in slot.pins:
                    self.cache.release(s, su)
                slot.busy, slot.pins, slot.reqs, slot.keep = False, [], None, None
        return done

    def drain(self):
        out = []
        while any(s.busy for s in self.slots):
            out += self.poll()
        return out

    def check_queue(self) -> None:
        """Raise if any slot's last run reported a queue error (synchronises)."""
        for s in self.slots:
            st = s.queue.stats()
            if st["error"] != Q.QUEUE_OK:
                raise MayoError(f"queue error {st['error']}")


def run_open_loop(server: Server, arrivals: np.ndarray, fetch, on_done=None, time_limit: float = None):
    """Serve requests arriving at `arrivals` (seconds from the start, sorted).  fetch(lo, hi)
    returns (request records for rows lo..hi-1, an object keeping their memory alive);
    on_done(lo, hi, keep) sees each finished batch.  Returns (latency per request in seconds,
    NaN if not served; wall seconds; batch sizes)."""
    n = int(arrivals.size)
    done_t = np.full(n, np.nan)
    nxt, finished = 0, 0
    sizes_ = []
    t0 = time.perf_counter()
    while finished < n:
        now = time.perf_counter() - t0
        for (lo, hi), keep in server.poll():
            done_t[lo:hi] = time.perf_counter() - t0
            finished += hi - lo
            if on_done is not None:
                on_done(lo, hi, keep)
        if nxt < n and server.free_slot() is not None:
            ready = int(np.searchsorted(arrivals, now, side="right"))
            if ready > nxt:
                reqs, keep = fetch(nxt, min(ready, nxt + server.max_batch))
                k = server.admit_len(reqs)  # bounded by the key tables
                if k:
                    server.launch(reqs[:k], tag=(nxt, nxt + k), keep=keep)
                    sizes_.append(k)
                    nxt += k
        if time_limit is not None and now > time_limit:
            for (lo, hi), keep in server.drain():
                done_t[lo:hi] = time.perf_counter() - t0
                if on_done is not None:
                    on_done(lo, hi, keep)
            break
    wall = time.perf_counter() - t0
    return done_t - arrivals, wall, np.array(sizes_, np.int64)
