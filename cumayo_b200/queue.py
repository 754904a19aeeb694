"""Persistent work queue (C-ABI ``mayo_b200_queue_*``): keypair / sign / verify items of all four
parameter sets drained by one launch of resident CTAs, rejected sign attempts re-enqueued on the
device, optionally replayed from a captured CUDA graph.

The caller owns all device memory (the queue memory here is a torch tensor); the library never
allocates.  Operand layout per parameter set is documented in include/mayo_b200.h.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from .api import MayoError, _check, _ptr, _stream, lib

OP_KEYPAIR, OP_SIGN, OP_VERIFY = 0, 1, 2
QUEUE_OK, QUEUE_ERR_FULL, QUEUE_ERR_TIMEOUT = 0, 1, 2
SET_INDEX = {1: 0, 2: 1, 3: 2, 5: 3}


class _QueueOps(ctypes.Structure):
    _fields_ = [("kp_seed", ctypes.c_void_p), ("kp_pk", ctypes.c_void_p),
                ("sg_esk", ctypes.c_void_p), ("sg_nkeys", ctypes.c_uint32), ("sg_msg", ctypes.c_void_p),
                ("sg_mlen", ctypes.c_uint32), ("sg_sig", ctypes.c_void_p),
                ("vf_epk", ctypes.c_void_p), ("vf_nkeys", ctypes.c_uint32), ("vf_msg", ctypes.c_void_p),
                ("vf_mlen", ctypes.c_uint32), ("vf_sig", ctypes.c_void_p), ("vf_res", ctypes.c_void_p)]


def _bind():
    L = lib()
    if not getattr(L, "_queue_bound", False):
        L.mayo_b200_queue_mem_bytes.restype = ctypes.c_size_t
        L.mayo_b200_queue_mem_bytes.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.mayo_b200_queue_ctas_per_sm.restype = ctypes.c_int
        L.mayo_b200_queue_run.restype = ctypes.c_int
        L.mayo_b200_queue_run.argtypes = [ctypes.POINTER(_QueueOps), ctypes.c_void_p, ctypes.c_uint32,
                                          ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                          ctypes.c_void_p]
        L._queue_bound = True
    return L


def item(op: int, set_id: int, instance: int) -> int:
    """Encoding of include/mayo_b200.h's mayo_b200_queue_item."""
    return (op << 30) | (SET_INDEX[set_id] << 28) | (instance & 0xFFFFF)


def items_array(entries) -> np.ndarray:
    """[(op, set, instance), ...] -> uint32 item array."""
    return np.array([item(o, s, i) for o, s, i in entries], dtype=np.uint32)


@dataclass
class SetOperands:
    """Device tensors for one parameter set (any may be None if its op is unused)."""
    kp_seed: object = None
    kp_pk: object = None
    sg_esk: object = None
    sg_nkeys: int = 1
    sg_msg: object = None
    sg_mlen: int = 0
    sg_sig: object = None
    vf_epk: object = None
    vf_nkeys: int = 1
    vf_msg: object = None
    vf_mlen: int = 0
    vf_sig: object = None
    vf_res: object = None


@dataclass
class Queue:
    """A device work queue with `capacity` slots drained by `ctas` resident CTAs."""
    capacity: int
    ctas: int = 0
    device: object = None
    operands: dict = field(default_factory=dict)  # set id -> SetOperands

    def __post_init__(self):
        import torch
        L = _bind()
        if self.ctas <= 0:
            per_sm = L.mayo_b200_queue_ctas_per_sm()
            if per_sm <= 0:
                raise MayoError("queue kernel cannot be resident on this device")
            sms = torch.cuda.get_device_properties(self.device or torch.cuda.current_device()).multi_processor_count
            self.ctas = per_sm * sms
        nbytes = L.mayo_b200_queue_mem_bytes(self.capacity, self.ctas)
        self.mem = torch.zeros(nbytes, dtype=torch.uint8, device=self.device or "cuda")
        self.items = torch.zeros(self.capacity, dtype=torch.int32, device=self.mem.device)
        self._ops = (_QueueOps * 4)()
        self.graph = None

    def set_operands(self, set_id: int, ops: SetOperands) -> None:
        self.operands[set_id] = ops
        o = self._ops[SET_INDEX[set_id]]
        for f, _ in _QueueOps._fields_:
            v = getattr(ops, f)
            if f.endswith(("nkeys", "mlen")):
                setattr(o, f, int(v))
            else:
                setattr(o, f, _ptr(v) or 0)

    def load(self, items: np.ndarray) -> int:
        """Copy work items into the queue's item buffer; returns their count."""
        import torch
        n = int(items.shape[0])
        if n > self.capacity:
            raise MayoError(f"{n} items exceed the queue capacity {self.capacity}")
        self.items[:n].copy_(torch.from_numpy(items.view(np.int32)))
        self.n = n
        return n

    def run(self, stream=None, spin_limit: int = 0) -> None:
        """Reset the queue to the loaded items and drain it (asynchronous on `stream`)."""
        L = _bind()
        _check(L.mayo_b200_queue_run(self._ops, _ptr(self.items), self.n, _ptr(self.mem), self.capacity, self.ctas,
                                     spin_limit, _stream(stream)), "queue_run")

    def capture(self) -> None:
        """Capture run() into a CUDA graph (replay with replay())."""
        import torch
        s = torch.cuda.Stream(device=self.mem.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.run(s)  # warm-up outside capture: sets the kernel's shared-memory attribute
        torch.cuda.current_stream().wait_stream(s)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=s):
            self.run(s)

    def replay(self) -> None:
        if self.graph is None:
            raise MayoError("capture() first")
        self.graph.replay()

    def stats(self) -> dict:
        """Control words after a run (synchronises)."""
        c = self.mem[:32].cpu().numpy().view(np.uint32)
        return {"tickets": int(c[0]), "published": int(c[1]), "finished": int(c[2]), "error": int(c[3]),
                "requeued_signs": int(c[4])}
