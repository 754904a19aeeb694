"""Persistent work queue (C-ABI ``mayo_b200_queue_*``): keypair / sign / verify items of all four
parameter sets, partitioned by set on the device and drained by one persistent kernel per set on
forked streams; rejected sign attempts re-enqueued on the device; optionally replayed from a
captured CUDA graph.

The caller owns all device memory (the queue memory here is a torch tensor); the library never
allocates.  Operand layout per parameter set is documented in include/mayo_b200.h.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from .api import MayoError, _check, _ptr, _stream, lib

OP_KEYPAIR, OP_SIGN, OP_VERIFY = 0, 1, 2
QUEUE_OK, QUEUE_ERR_FULL, QUEUE_ERR_TIMEOUT, QUEUE_ERR_OPERAND = 0, 1, 2, 3
SET_INDEX = {1: 0, 2: 1, 3: 2, 5: 3}
OPS = (OP_KEYPAIR, OP_SIGN, OP_VERIFY)
# bucket index b = 3 * set index + op; one persistent kernel per bucket
BUCKETS = [(s, op) for s in SET_INDEX for op in OPS]
# default launch order (the C library's): buckets with the longest items first
DEFAULT_ORDER = [(5, 0), (5, 1), (5, 2), (3, 0), (3, 1), (3, 2), (1, 0), (2, 0), (1, 1), (1, 2), (2, 1), (2, 2)]


def bucket(set_id: int, op: int) -> int:
    return 3 * SET_INDEX[set_id] + op


class _QueueOps(ctypes.Structure):
    _fields_ = [("kp_seed", ctypes.c_void_p), ("kp_pk", ctypes.c_void_p), ("kp_count", ctypes.c_uint32),
                ("sg_esk", ctypes.c_void_p), ("sg_nkeys", ctypes.c_uint32), ("sg_key", ctypes.c_void_p),
                ("sg_msg", ctypes.c_void_p), ("sg_msg_off", ctypes.c_void_p), ("sg_msg_len", ctypes.c_void_p),
                ("sg_mlen", ctypes.c_uint32), ("sg_sig", ctypes.c_void_p), ("sg_count", ctypes.c_uint32),
                ("vf_epk", ctypes.c_void_p), ("vf_nkeys", ctypes.c_uint32), ("vf_key", ctypes.c_void_p),
                ("vf_msg", ctypes.c_void_p), ("vf_msg_off", ctypes.c_void_p), ("vf_msg_len", ctypes.c_void_p),
                ("vf_mlen", ctypes.c_uint32), ("vf_sig", ctypes.c_void_p), ("vf_res", ctypes.c_void_p),
                ("vf_count", ctypes.c_uint32)]


class _QueueShape(ctypes.Structure):
    _fields_ = [("sms", ctypes.c_uint32), ("ctas_per_sm", ctypes.c_uint8 * 12), ("launch_order", ctypes.c_uint8 * 12)]


def _bind():
    L = lib()
    if not getattr(L, "_queue_bound", False):
        L.mayo_b200_queue_mem_bytes.restype = ctypes.c_size_t
        L.mayo_b200_queue_mem_bytes.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.mayo_b200_queue_ctas_per_sm.restype = ctypes.c_int
        L.mayo_b200_queue_ctas_per_sm.argtypes = [ctypes.c_int, ctypes.c_int]
        L.mayo_b200_queue_run.restype = ctypes.c_int
        L.mayo_b200_queue_run.argtypes = [ctypes.POINTER(_QueueOps), ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(_QueueShape),
                                          ctypes.c_uint32, ctypes.c_void_p]
        L._queue_bound = True
    return L


def ctas_per_sm(set_id: int, op: int) -> int:
    """Most CTAs of the (set, op) queue kernel resident on one SM of the current device."""
    return int(_bind().mayo_b200_queue_ctas_per_sm(set_id, op))


def item(op: int, set_id: int, instance: int) -> int:
    """Encoding of include/mayo_b200.h's mayo_b200_queue_item."""
    return (op << 30) | (SET_INDEX[set_id] << 28) | (instance & 0xFFFFF)


def items_array(entries) -> np.ndarray:
    """[(op, set, instance), ...] -> uint32 item array."""
    return np.array([item(o, s, i) for o, s, i in entries], dtype=np.uint32)


@dataclass
class SetOperands:
    """Device tensors for one parameter set (any may be None if its op is unused).  Counts left
    at None are taken from the output tensors; sg_key / vf_key (uint32 per instance) pick a key
    per instance, sg_msg_off (int64) / sg_msg_len (uint32 or int32) give per-instance messages."""
    kp_seed: object = None
    kp_pk: object = None
    kp_count: int = None
    sg_esk: object = None
    sg_nkeys: int = 1
    sg_key: object = None
    sg_msg: object = None
    sg_msg_off: object = None
    sg_msg_len: object = None
    sg_mlen: int = 0
    sg_sig: object = None
    sg_count: int = None
    vf_epk: object = None
    vf_nkeys: int = 1
    vf_key: object = None
    vf_msg: object = None
    vf_msg_off: object = None
    vf_msg_len: object = None
    vf_mlen: int = 0
    vf_sig: object = None
    vf_res: object = None
    vf_count: int = None


@dataclass
class Shape:
    """Launch shape: SMs the memory is sized for (0 = all), CTAs per SM per (set, op) bucket (0 or
    absent = the most that fit), the order the bucket kernels are launched in ((set, op) pairs;
    None = the library default, longest items first)."""
    sms: int = 0
    ctas_per_sm: dict = field(default_factory=dict)  # (set id, op) -> CTAs per SM
    launch_order: list = None

    def to_c(self) -> _QueueShape:
        c = _QueueShape()
        c.sms = self.sms
        for (s, op), v in self.ctas_per_sm.items():
            c.ctas_per_sm[bucket(s, op)] = int(v)
        order = self.launch_order or DEFAULT_ORDER
        for k, (s, op) in enumerate(order):
            c.launch_order[k] = bucket(s, op)
        return c


@dataclass
class Queue:
    """A device work queue with `capacity` slots per set, drained by one persistent kernel per
    parameter set on `shape.sms` SMs."""
    capacity: int
    shape: Shape = field(default_factory=Shape)
    device: object = None
    operands: dict = field(default_factory=dict)  # set id -> SetOperands

    def __post_init__(self):
        import torch
        L = _bind()
        dev = torch.device(self.device) if self.device is not None else \
            torch.device("cuda", torch.cuda.current_device())
        if self.shape.sms <= 0:
            self.shape.sms = torch.cuda.get_device_properties(dev).multi_processor_count
        nbytes = L.mayo_b200_queue_mem_bytes(self.capacity, self.shape.sms)
        if nbytes == 0:
            raise MayoError("queue memory size unavailable (no device, or a kernel cannot be resident)")
        self.mem = torch.zeros(nbytes, dtype=torch.uint8, device=dev)
        self.items = torch.zeros(self.capacity, dtype=torch.int32, device=dev)
        self.count = torch.zeros(1, dtype=torch.int32, device=dev)  # device-side item count (replays)
        self._ops = (_QueueOps * 4)()
        self.graph = None
        self.n = 0

    def set_operands(self, set_id: int, ops: SetOperands) -> None:
        from .api import sizes
        z = sizes(set_id)
        self.operands[set_id] = ops
        o = self._ops[SET_INDEX[set_id]]
        for f, _ in _QueueOps._fields_:
            v = getattr(ops, f)
            if f.endswith("count"):
                if v is None:
                    out = {"kp_count": (ops.kp_pk, z.pk_bytes), "sg_count": (ops.sg_sig, z.sig_bytes),
                           "vf_count": (ops.vf_res, 1)}[f]
                    v = out[0].numel() // out[1] if out[0] is not None else 0
                setattr(o, f, int(v))
            elif f.endswith(("nkeys", "mlen")):
                setattr(o, f, int(v))
            else:
                setattr(o, f, _ptr(v) or 0)

    def load(self, items: np.ndarray) -> int:
        """Copy work items into the queue's item buffer; returns their count."""
        import torch
        n = int(items.shape[0])
        if n > self.capacity:
            raise MayoError(f"{n} items exceed the queue capacity {self.capacity}")
        self.items[:n].copy_(torch.from_numpy(np.ascontiguousarray(items).view(np.int32)))
        self.count.fill_(n)
        self.n = n
        return n

    def run(self, stream=None, spin_limit: int = 0, n_max: int = None, device_count: bool = False) -> None:
        """Reset the queue to the loaded items and drain it (asynchronous on `stream`).  With
        device_count the item count is read on the device from `self.count` (at most n_max)."""
        L = _bind()
        shp = self.shape.to_c()
        n = self.n if n_max is None else n_max
        _check(L.mayo_b200_queue_run(self._ops, _ptr(self.items), n, _ptr(self.count) if device_count else None,
                                     _ptr(self.mem), self.capacity, ctypes.byref(shp), spin_limit, _stream(stream)),
               "queue_run")

    def run_items(self, items_ptr: int, n: int, stream=None, spin_limit: int = 0) -> None:
        """Run n items already on the device at `items_ptr` (e.g. inside a staged input buffer)."""
        if n > self.capacity:
            raise MayoError(f"{n} items exceed the queue capacity {self.capacity}")
        L = _bind()
        shp = self.shape.to_c()
        _check(L.mayo_b200_queue_run(self._ops, items_ptr, n, None, _ptr(self.mem), self.capacity, ctypes.byref(shp),
                                     spin_limit, _stream(stream)), "queue_run")

    def capture(self, device_count: bool = False) -> None:
        """Capture run() into a CUDA graph (replay with replay()).  With device_count the graph
        reads the item count from the device at each replay, up to the capacity."""
        import torch
        n_max = self.capacity if device_count else None
        s = torch.cuda.Stream(device=self.mem.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.run(s, n_max=n_max, device_count=device_count)  # warm-up outside capture
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=s):
            self.run(s, n_max=n_max, device_count=device_count)

    def replay(self) -> None:
        if self.graph is None:
            raise MayoError("capture() first")
        self.graph.replay()

    def stats(self) -> dict:
        """Control words after a run (synchronises): totals over the buckets, the first error code,
        per (set, op) bucket the same words ("taken" counts the items a bucket without operands
        dropped), and the items dropped for an invalid op."""
        c = self.mem[:13 * 64].cpu().numpy().view(np.uint32).reshape(13, 16)
        per = {(s, op): {"taken": int(c[b, 0]), "published": int(c[b, 1]), "finished": int(c[b, 2]),
                         "error": int(c[b, 3]), "requeued_signs": int(c[b, 4])}
               for b, (s, op) in enumerate(BUCKETS)}
        err = next((p["error"] for p in per.values() if p["error"]), int(c[12, 3]))
        tot = {k: sum(p[k] for p in per.values()) for k in ("published", "finished", "requeued_signs")}
        return dict(tot, error=err, per_bucket=per, invalid_op_items=int(c[12, 0]))
