"""Serving loop for MAYO sign / verify requests on one GPU: a thin mirror of the native server
(mayo_b200_server_* in libmayo_b200.so, C++: cumayo_b200/csrc/serve_loop.cu).

Requests (40-byte records pointing into the caller's host memory) join a waiting line.  The
server keeps up to `inflight` batches on the GPU, each on its own stream with its own queue
memory and staging buffers.  Whenever a batch slot is free and requests wait, the longest prefix
of the line (up to `max_batch`) whose keys fit in the key tables is admitted as one batch: keys
not resident are expanded into free table rows, the inputs are packed into one pinned buffer and
copied to the device in one transfer, the work queue partitions the batch by (set, op) on the
device and drains it with the per-(set, op) persistent kernels, and one transfer brings the
signatures and verify results back.  A request's latency is the time from its arrival to the
server unpacking its result.

Keys are registered per parameter set by id (their seeds) and expanded (esk for signing, epk for
verifying) on first use into a per-set table in HBM; a full table evicts its least recently used
rows that no batch in flight uses.

This module has no counterpart in the reference, which offers only the synchronous batched pool
API (include/api.cuh).
"""
from __future__ import annotations

import ctypes

import numpy as np

from .api import MayoError, _check, lib, sizes

SETS = (1, 2, 3, 5)
MAX_SIG = max(sizes(s).sig_bytes for s in SETS)
ERR_FULL = 5  # MAYO_B200_ERR_FULL


class CacheFull(MayoError):
    pass


def capacity_for_budget(budget_bytes: int, n_keys: dict) -> dict:
    """Key-table rows per set: all keys if they fit, else the budget split by each set's key bytes."""
    need = {s: n * (sizes(s).esk_bytes + sizes(s).epk_bytes) for s, n in n_keys.items()}
    total = sum(need.values())
    if total <= budget_bytes:
        return dict(n_keys)
    return {s: max(1, int(n_keys[s] * budget_bytes / total)) for s in n_keys}


# ---------------------------------------------------------------------------------------------
# key table (host only; native: mayo_b200_key_table_*)
# ---------------------------------------------------------------------------------------------
class _KeyTableStats(ctypes.Structure):
    _fields_ = [("capacity", ctypes.c_uint32), ("n_keys", ctypes.c_uint32), ("pinned_slots", ctypes.c_uint32),
                ("resident_keys", ctypes.c_uint32), ("misses", ctypes.c_uint64), ("evictions", ctypes.c_uint64)]


class SlotTable:
    """Key id -> row map of one parameter set's key table with least-recently-used eviction (the
    native table the server uses).  `acquire` maps a batch's key ids to rows, choosing rows for
    the keys that are not resident (empty rows first, then the least recently used unpinned
    ones, never one this batch uses) and pins every row the batch uses until `release`."""

    def __init__(self, capacity: int, n_keys: int):
        L = _bind()
        self._h = L.mayo_b200_key_table_create(capacity, n_keys) if capacity > 0 and n_keys > 0 else None
        if not self._h:
            raise MayoError("key table needs at least one row and one key")
        self.capacity, self.n_keys = capacity, n_keys

    def __del__(self):
        if getattr(self, "_h", None):
            _bind().mayo_b200_key_table_destroy(self._h)
            self._h = None

    @staticmethod
    def _ids(key_ids) -> np.ndarray:
        k = np.asarray(key_ids, np.int64)
        if k.size and (k.min() < 0 or k.max() >= 1 << 32):
            raise MayoError("unknown key id")
        return np.ascontiguousarray(k.astype(np.uint32))

    def acquire(self, key_ids):
        """Returns (row per key id, missing key ids, their new rows, rows to release)."""
        ids = self._ids(key_ids)
        n = ids.size
        slots = np.zeros(n, np.int32)
        miss = np.zeros(max(n, 1), np.uint32)
        new = np.zeros(max(n, 1), np.int32)
        nm = ctypes.c_uint32(0)
        rc = _bind().mayo_b200_key_table_acquire(self._h, ids.ctypes.data, n, slots.ctypes.data, miss.ctypes.data,
                                                 new.ctypes.data, ctypes.byref(nm))
        if rc == ERR_FULL:
            raise CacheFull("not enough key-table rows free of batches in flight")
        _check(rc, "key_table_acquire")
        k = nm.value
        return slots.astype(np.int64), miss[:k].astype(np.int64), new[:k].astype(np.int64), slots

    def release(self, su) -> None:
        su = np.ascontiguousarray(su, np.int32)
        _check(_bind().mayo_b200_key_table_release(self._h, su.ctypes.data, su.size), "key_table_release")

    def can_load(self, key_ids) -> bool:
        ids = self._ids(key_ids)
        r = _bind().mayo_b200_key_table_can_load(self._h, ids.ctypes.data, ids.size)
        if r < 0:
            raise MayoError("unknown key id")
        return r == 1

    def _info(self) -> _KeyTableStats:
        st = _KeyTableStats()
        _check(_bind().mayo_b200_key_table_info(self._h, ctypes.byref(st)), "key_table_info")
        return st

    @property
    def evictions(self) -> int:
        return int(self._info().evictions)

    @property
    def misses(self) -> int:
        return int(self._info().misses)

    @property
    def slot_of(self) -> np.ndarray:
        L = _bind()
        return np.array([L.mayo_b200_key_table_slot_of(self._h, i) for i in range(self.n_keys)], np.int64)

    @property
    def pins(self) -> np.ndarray:
        L = _bind()
        return np.array([L.mayo_b200_key_table_pins(self._h, i) for i in range(self.capacity)], np.int64)


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
        vp, u32, u64 = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64
        L.mayo_b200_key_table_create.restype = vp
        L.mayo_b200_key_table_create.argtypes = [u32, u32]
        L.mayo_b200_key_table_destroy.restype = None
        L.mayo_b200_key_table_destroy.argtypes = [vp]
        L.mayo_b200_key_table_acquire.restype = ctypes.c_int
        L.mayo_b200_key_table_acquire.argtypes = [vp, vp, u32, vp, vp, vp, ctypes.POINTER(u32)]
        L.mayo_b200_key_table_release.restype = ctypes.c_int
        L.mayo_b200_key_table_release.argtypes = [vp, vp, u32]
        L.mayo_b200_key_table_can_load.restype = ctypes.c_int
        L.mayo_b200_key_table_can_load.argtypes = [vp, vp, u32]
        L.mayo_b200_key_table_info.restype = ctypes.c_int
        L.mayo_b200_key_table_info.argtypes = [vp, ctypes.POINTER(_KeyTableStats)]
        L.mayo_b200_key_table_slot_of.restype = ctypes.c_int32
        L.mayo_b200_key_table_slot_of.argtypes = [vp, u32]
        L.mayo_b200_key_table_pins.restype = ctypes.c_int32
        L.mayo_b200_key_table_pins.argtypes = [vp, u32]
        for f in ("device_bytes", "host_bytes"):
            getattr(L, "mayo_b200_server_" + f).restype = ctypes.c_size_t
            getattr(L, "mayo_b200_server_" + f).argtypes = [ctypes.POINTER(_ServerConfig)]
        L.mayo_b200_server_create.restype = ctypes.c_int
        L.mayo_b200_server_create.argtypes = [ctypes.POINTER(_ServerConfig), ctypes.POINTER(vp), vp, ctypes.c_size_t,
                                              vp, ctypes.c_size_t, ctypes.POINTER(vp)]
        L.mayo_b200_server_destroy.restype = ctypes.c_int
        L.mayo_b200_server_destroy.argtypes = [vp]
        L.mayo_b200_server_submit.restype = ctypes.c_int
        L.mayo_b200_server_submit.argtypes = [vp, vp, u32, u64]
        L.mayo_b200_server_progress.restype = ctypes.c_int
        L.mayo_b200_server_progress.argtypes = [vp, vp, u32, ctypes.POINTER(u32)]
        L.mayo_b200_server_drain.restype = ctypes.c_int
        L.mayo_b200_server_drain.argtypes = [vp]
        L.mayo_b200_server_get_stats.restype = ctypes.c_int
        L.mayo_b200_server_get_stats.argtypes = [vp, ctypes.POINTER(_ServerStats)]
        L.mayo_b200_server_preload.restype = ctypes.c_int
        L.mayo_b200_server_preload.argtypes = [vp, ctypes.c_int, vp, u32]
        L.mayo_b200_server_queue_error.restype = ctypes.c_int
        L.mayo_b200_server_queue_error.argtypes = [vp]
        L.mayo_b200_server_run_open_loop.restype = ctypes.c_int
        L.mayo_b200_server_run_open_loop.argtypes = [vp, vp, vp, u32, ctypes.c_double, vp, ctypes.POINTER(ctypes.c_double)]
        L._serve_bound = True
    return L


class _ServerConfig(ctypes.Structure):
    _fields_ = [("max_batch", ctypes.c_uint32), ("inflight", ctypes.c_uint32), ("max_msg", ctypes.c_uint32),
                ("expand_chunk", ctypes.c_uint32), ("n_keys", ctypes.c_uint32 * 4), ("key_slots", ctypes.c_uint32 * 4)]


class _ServerStats(ctypes.Structure):
    _fields_ = [(f, ctypes.c_uint64) for f in ("batches", "requests_admitted", "requests_done", "max_batch_seen",
                                               "kernel_launches", "keys_expanded", "key_misses", "key_evictions",
                                               "waiting")] + [("batches_in_flight", ctypes.c_uint32),
                                                              ("pad", ctypes.c_uint32)]


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
# the server (native: mayo_b200_server_*)
# ---------------------------------------------------------------------------------------------
class Server:
    """Continuous-batching MAYO sign / verify server on one GPU (the native server).

    seeds: {set: (n_keys, sk_bytes) uint8 array} -- key id = row; key_slots: {set: resident rows}
    (default: every key).  max_batch requests per batch, `inflight` batches on the GPU at once,
    messages up to max_msg bytes.  The device and pinned host memory the server needs are
    allocated here (torch) and handed to it; `budget_bytes` bounds the device bytes."""

    def __init__(self, seeds: dict, key_slots: dict | None = None, max_batch: int = 4096, inflight: int = 2,
                 max_msg: int = 256, budget_bytes: int = 60 << 30, device=None, expand_chunk: int = 0):
        import torch
        L = _bind()
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.max_batch, self.max_msg = max_batch, max_msg
        cfg = _ServerConfig(max_batch, inflight, max_msg, expand_chunk)
        self._seeds = []
        ptrs = (ctypes.c_void_p * 4)()
        for i, s in enumerate(SETS):
            if s in seeds:
                a = np.ascontiguousarray(seeds[s], np.uint8)
                if a.ndim != 2 or a.shape[1] != sizes(s).sk_bytes:
                    raise MayoError(f"MAYO_{s} seeds must be (n, {sizes(s).sk_bytes}) uint8")
                self._seeds.append(a)
                cfg.n_keys[i] = a.shape[0]
                cfg.key_slots[i] = int((key_slots or {}).get(s, 0))
                ptrs[i] = a.ctypes.data
        with torch.cuda.device(self.dev):
            dbytes = L.mayo_b200_server_device_bytes(ctypes.byref(cfg))
            hbytes = L.mayo_b200_server_host_bytes(ctypes.byref(cfg))
        if dbytes == 0 or hbytes == 0:
            raise MayoError("invalid server configuration")
        if dbytes > budget_bytes:
            raise MayoError(f"server needs {dbytes} device bytes, budget {budget_bytes}")
        self.device_bytes, self.host_bytes = int(dbytes), int(hbytes)
        self._dmem = torch.empty(dbytes + 256, dtype=torch.uint8, device=self.dev)
        self._hmem = torch.empty(hbytes + 256, dtype=torch.uint8).pin_memory()
        dp = (self._dmem.data_ptr() + 255) // 256 * 256
        hp = (self._hmem.data_ptr() + 255) // 256 * 256
        h = ctypes.c_void_p()
        with torch.cuda.device(self.dev):
            _check(L.mayo_b200_server_create(ctypes.byref(cfg), ptrs, dp, dbytes, hp, hbytes, ctypes.byref(h)),
                   "server_create")
        self._h = h
        self._keep = {}  # tag -> objects whose memory requests point into, until done

    def close(self) -> None:
        if getattr(self, "_h", None):
            _check(_bind().mayo_b200_server_destroy(self._h), "server_destroy")
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def preload(self, set_id: int, key_ids) -> None:
        """Makes the keys resident now (only while no batch is in flight)."""
        ids = np.ascontiguousarray(np.asarray(key_ids, np.int64).astype(np.uint32))
        _check(_bind().mayo_b200_server_preload(self._h, set_id, ids.ctypes.data, ids.size), "server_preload")

    def submit(self, reqs: np.ndarray, first_tag: int = 0, keep=None) -> None:
        """Requests join the waiting line; request i gets tag first_tag + i.  The memory the
        records point into must stay alive until they are done (`keep` holds it until then)."""
        reqs = np.ascontiguousarray(reqs, REQ_DTYPE)
        _check(_bind().mayo_b200_server_submit(self._h, reqs.ctypes.data, reqs.size, first_tag), "server_submit")
        if keep is not None:
            self._keep[first_tag] = keep

    def progress(self, cap: int = 1 << 16) -> np.ndarray:
        """One non-blocking pass; returns the tags of requests finished since the last call."""
        buf = np.zeros(cap, np.uint64)
        n = ctypes.c_uint32(0)
        _check(_bind().mayo_b200_server_progress(self._h, buf.ctypes.data, cap, ctypes.byref(n)), "server_progress")
        return buf[: n.value]

    def drain(self) -> np.ndarray:
        """Serves everything submitted; returns the tags finished since the last progress()."""
        rc = _bind().mayo_b200_server_drain(self._h)
        if rc == ERR_FULL:
            raise CacheFull("waiting requests need more key-table rows than exist")
        _check(rc, "server_drain")
        out = []
        while True:
            t = self.progress()
            if t.size == 0:
                break
            out.append(t)
        self._keep.clear()
        return np.concatenate(out) if out else np.zeros(0, np.uint64)

    def run_open_loop(self, reqs: np.ndarray, arrivals: np.ndarray, time_limit: float = 0.0):
        """Open-loop run (native): request i arrives arrivals[i] seconds after the start.
        Returns (latency per request in seconds, NaN if not served; wall seconds)."""
        reqs = np.ascontiguousarray(reqs, REQ_DTYPE)
        arr = np.ascontiguousarray(arrivals, np.float64)
        lat = np.full(reqs.size, np.nan)
        wall = ctypes.c_double(0.0)
        _check(_bind().mayo_b200_server_run_open_loop(self._h, reqs.ctypes.data, arr.ctypes.data, reqs.size,
                                                      float(time_limit), lat.ctypes.data, ctypes.byref(wall)),
               "server_run_open_loop")
        return lat, wall.value

    def stats(self) -> dict:
        st = _ServerStats()
        _check(_bind().mayo_b200_server_get_stats(self._h, ctypes.byref(st)), "server_get_stats")
        return {f: int(getattr(st, f)) for f, _ in _ServerStats._fields_ if f != "pad"}

    def check_queue(self) -> None:
        """Raise if any batch slot's last queue run reported an error (synchronises)."""
        err = _bind().mayo_b200_server_queue_error(self._h)
        if err != 0:
            raise MayoError(f"queue error {err}")
