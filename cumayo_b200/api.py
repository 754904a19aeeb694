"""Host-side mirror of SysuCrypto/cuMAYO's batched API over libmayo_b200.so.

``Mayo(set_id)`` exposes the reference's 20 entry points under their reference names
(include/api.cuh:9-47), with the reference's argument order and pool layouts, plus
``aes128_tables_init``.  Device pools are CUDA ``torch.uint8`` tensors (or raw device
pointers); host buffers are numpy arrays or CPU tensors (pinned memory recommended, as in
the reference benchmark).  Streams are ``torch.cuda.Stream`` objects, raw ``cudaStream_t``
integers, or ``None`` for the legacy default stream (the reference's ``nullptr`` default).

Unlike the reference, which returns ``void`` and reports nothing, every call raises
``MayoError`` when the C-ABI returns a non-zero status.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libmayo_b200.so")

SETS = (1, 2, 3, 5)

_FUNCS = {
    # name: argument types after the leading `int set`
    "keypair": ("p", "z", "z", "p", "z"),
    "keypair_DtH": ("p", "p", "p", "z", "z", "p"),
    "keypair_from_seed": ("p", "z", "z", "p"),
    "expandsk_HtD": ("p", "p", "z", "z", "p"),
    "expandsk": ("p", "z", "z", "p"),
    "expandsk_DtH": ("p", "p", "z", "z", "p"),
    "expandpk_HtD": ("p", "p", "z", "z", "p"),
    "expandpk": ("p", "z", "z", "p"),
    "expandpk_DtH": ("p", "p", "z", "z", "p"),
    "sign_HtD": ("p", "p", "z", "p", "z", "z", "p"),
    "sign": ("p", "z", "z", "z", "p"),
    "sign_DtH": ("p", "p", "z", "z", "z", "p"),
    "signWithesk_HtD": ("p", "p", "z", "p", "z", "z", "p"),
    "signWithesk": ("p", "z", "z", "z", "p"),
    "signWithesk_DtH": ("p", "p", "z", "z", "z", "p"),
    "verify_HtD": ("p", "p", "p", "z", "p", "z", "z", "p"),
    "verify": ("p", "z", "z", "z", "p"),
    "verify_DtH": ("p", "z", "p", "z", "z", "p"),
    "verifyWithepk_HtD": ("p", "p", "p", "z", "p", "z", "z", "p"),
    "verifyWithepk": ("p", "z", "z", "z", "p"),
    "verifyWithepk_DtH": ("p", "z", "p", "z", "z", "p"),
}


class MayoError(RuntimeError):
    pass


class _Sizes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("set", "n", "m", "o", "k", "digest_bytes")] + [
        (n, ctypes.c_uint64) for n in ("sk_bytes", "pk_bytes", "sig_bytes", "esk_bytes", "epk_bytes", "p_bytes",
                                       "scratch_bytes", "pitch_keypair", "pitch_expandsk", "pitch_expandpk",
                                       "pitch_sign", "pitch_sign_with_esk", "pitch_verify")]


_lib = None


def lib() -> ctypes.CDLL:
    """Load libmayo_b200.so (built in-tree by ``python -m cumayo_b200.build``).  There is no
    fallback: without the library nothing in this package can run."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise MayoError(f"{LIB_PATH} is missing; build it with `python -m cumayo_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        T = {"p": ctypes.c_void_p, "z": ctypes.c_size_t}
        for name, args in _FUNCS.items():
            fn = getattr(L, "mayo_b200_" + name)
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_int] + [T[a] for a in args]
        L.mayo_b200_get_sizes.restype = ctypes.c_int
        L.mayo_b200_get_sizes.argtypes = [ctypes.c_int, ctypes.c_size_t, ctypes.POINTER(_Sizes)]
        L.mayo_b200_status_string.restype = ctypes.c_char_p
        L.mayo_b200_status_string.argtypes = [ctypes.c_int]
        L.mayo_b200_abi_version.restype = ctypes.c_int
        L.mayo_b200_init.restype = ctypes.c_int
        L.mayo_b200_last_cuda_error.restype = ctypes.c_int
        L.mayo_b200_sign_ws_bytes.restype = ctypes.c_size_t
        L.mayo_b200_sign_ws_bytes.argtypes = [ctypes.c_int]
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        L.mayo_b200_sign_many.restype = ctypes.c_int
        L.mayo_b200_sign_many.argtypes = [ctypes.c_int, vp, sz, vp, vp, vp, sz, sz, vp, sz, vp, sz, vp]
        L.mayo_b200_verify_many.restype = ctypes.c_int
        L.mayo_b200_verify_many.argtypes = [ctypes.c_int, vp, sz, vp, vp, vp, sz, sz, vp, sz, vp, sz, vp]
        L.mayo_b200_sign_noalloc_max_batch.restype = ctypes.c_size_t
        L.mayo_b200_sign_noalloc_max_batch.argtypes = [ctypes.c_int]
        L.mayo_b200_sign_many_noalloc.restype = ctypes.c_int
        L.mayo_b200_sign_many_noalloc.argtypes = [ctypes.c_int, vp, sz, vp, vp, vp, sz, sz, vp, sz, sz, vp]
        for nm in ("sign_shared_ws_bytes", "verify_shared_ws_bytes"):
            getattr(L, "mayo_b200_" + nm).restype = ctypes.c_size_t
            getattr(L, "mayo_b200_" + nm).argtypes = [ctypes.c_int, sz]
        L.mayo_b200_sign_shared.restype = ctypes.c_int
        L.mayo_b200_sign_shared.argtypes = [ctypes.c_int, vp, vp, vp, vp, sz, sz, vp, sz, vp, sz, vp]
        L.mayo_b200_verify_shared.restype = ctypes.c_int
        L.mayo_b200_verify_shared.argtypes = [ctypes.c_int, vp, vp, vp, vp, sz, sz, vp, sz, vp, vp, sz, vp]
        L.mayo_b200_shared_timing.restype = ctypes.c_int
        L.mayo_b200_shared_timing.argtypes = [ctypes.c_int]
        L.mayo_b200_shared_timing_read.restype = ctypes.c_int
        L.mayo_b200_shared_timing_read.argtypes = [ctypes.POINTER(ctypes.c_float)]
        L.mayo_b200_shared_set_shape.restype = ctypes.c_int
        L.mayo_b200_shared_set_shape.argtypes = [ctypes.c_int, ctypes.POINTER(SharedShape)]
        L.mayo_b200_shared_get_shape.restype = ctypes.c_int
        L.mayo_b200_shared_get_shape.argtypes = [ctypes.c_int, ctypes.POINTER(SharedShape)]
        L.mayo_b200_test_inject.restype = ctypes.c_int
        L.mayo_b200_test_inject.argtypes = [ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32]
        _lib = L
    return _lib


class SharedShape(ctypes.Structure):
    """mayo_b200_shared_shape: launch shape of a set's shared-key calls."""
    _fields_ = [("hash_threads", ctypes.c_uint32), ("tail_instances", ctypes.c_uint32),
                ("product_ctas", ctypes.c_uint32)]


INJECT_NONE, INJECT_QUEUE_LOST_PUSH, INJECT_PRODUCT_STALL = 0, 1, 2


def test_inject(kind: int, arg: int = 0, spin: int = 0) -> None:
    """Failure injection for tests (mayo_b200_test_inject), for calls from this thread:
    INJECT_QUEUE_LOST_PUSH gives every queue bucket a slot nothing publishes, so its bounded
    wait runs out (MAYO_B200_QUEUE_ERR_TIMEOUT); INJECT_PRODUCT_STALL stops the tensor-core
    product's key loader after `arg` chunks with waits of `spin` polls (the status word becomes
    1 and the per-instance engine computes the results); INJECT_NONE turns it off."""
    _check(lib().mayo_b200_test_inject(kind, arg, spin), "test_inject")


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().mayo_b200_status_string(rc).decode()
        cuda = lib().mayo_b200_last_cuda_error()
        raise MayoError(f"{what}: {msg} (status {rc}, cuda error {cuda})")


@dataclass(frozen=True)
class Sizes:
    set: int
    n: int
    m: int
    o: int
    k: int
    digest_bytes: int
    sk_bytes: int
    pk_bytes: int
    sig_bytes: int
    esk_bytes: int
    epk_bytes: int
    p_bytes: int
    scratch_bytes: int
    pitch_keypair: int
    pitch_expandsk: int
    pitch_expandpk: int
    pitch_sign: int
    pitch_sign_with_esk: int
    pitch_verify: int


def sizes(set_id: int, mlen: int = 0) -> Sizes:
    s = _Sizes()
    _check(lib().mayo_b200_get_sizes(int(set_id), int(mlen), ctypes.byref(s)), "get_sizes")
    return Sizes(**{f: getattr(s, f) for f, _ in _Sizes._fields_})


def A128(x: int) -> int:
    return (x + 127) // 128 * 128


def _ptr(x) -> int | None:
    """Address of a device tensor, host array/tensor or raw integer pointer."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise MayoError("host arrays must be C-contiguous")
        return x.ctypes.data
    if hasattr(x, "data_ptr"):
        if hasattr(x, "is_contiguous") and not x.is_contiguous():
            raise MayoError("tensors must be contiguous")
        return x.data_ptr()
    raise TypeError(f"cannot take the address of {type(x).__name__}")


def _stream(s) -> int | None:
    if s is None:
        return None
    if isinstance(s, int):
        return s
    if hasattr(s, "cuda_stream"):
        return s.cuda_stream
    raise TypeError(f"not a stream: {type(s).__name__}")


def aes128_tables_init() -> None:
    """Counterpart of the reference's aes128_tables_init() (include/aes128_ctr.cuh:16).  The
    B200 engine's tables are compile-time constants, so this only checks the device."""
    _check(lib().mayo_b200_init(), "init")


class Mayo:
    """One MAYO parameter set; methods carry the reference's names and argument order."""

    def __init__(self, set_id: int):
        if set_id not in SETS:
            raise MayoError(f"unknown MAYO parameter set {set_id}")
        self.set = set_id
        self.sizes = sizes(set_id)

    # keypair ------------------------------------------------------------------------------
    def crypto_sign_keypair(self, pool, pitch, batch_size=1, stream=None, rand_index=0):
        _check(lib().mayo_b200_keypair(self.set, _ptr(pool), pitch, batch_size, _stream(stream), rand_index),
               "crypto_sign_keypair")

    def crypto_sign_keypair_DtH(self, pk, sk, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_keypair_DtH(self.set, _ptr(pk), _ptr(sk), _ptr(pool), pitch, batch_size,
                                           _stream(stream)), "crypto_sign_keypair_DtH")

    def crypto_sign_keypair_from_seed(self, pool, pitch, batch_size=1, stream=None):
        """Extension: keypairs from seeds the caller placed at each row's offset 0."""
        _check(lib().mayo_b200_keypair_from_seed(self.set, _ptr(pool), pitch, batch_size, _stream(stream)),
               "crypto_sign_keypair_from_seed")

    # expand-sk ----------------------------------------------------------------------------
    def crypto_sign_expandsk_HtD(self, csk, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_expandsk_HtD(self.set, _ptr(csk), _ptr(pool), pitch, batch_size, _stream(stream)),
               "crypto_sign_expandsk_HtD")

    def crypto_sign_expandsk(self, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_expandsk(self.set, _ptr(pool), pitch, batch_size, _stream(stream)),
               "crypto_sign_expandsk")

    def crypto_sign_expandsk_DtH(self, esk, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_expandsk_DtH(self.set, _ptr(esk), _ptr(pool), pitch, batch_size, _stream(stream)),
               "crypto_sign_expandsk_DtH")

    # expand-pk ----------------------------------------------------------------------------
    def crypto_sign_expandpk_HtD(self, cpk, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_expandpk_HtD(self.set, _ptr(cpk), _ptr(pool), pitch, batch_size, _stream(stream)),
               "crypto_sign_expandpk_HtD")

    def crypto_sign_expandpk(self, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_expandpk(self.set, _ptr(pool), pitch, batch_size, _stream(stream)),
               "crypto_sign_expandpk")

    def crypto_sign_expandpk_DtH(self, epk, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_expandpk_DtH(self.set, _ptr(epk), _ptr(pool), pitch, batch_size, _stream(stream)),
               "crypto_sign_expandpk_DtH")

    # sign -----------------------------------------------------------------------------------
    def crypto_sign_sign_HtD(self, cesk, cMess, mlen, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_sign_HtD(self.set, _ptr(cesk), _ptr(cMess), mlen, _ptr(pool), pitch, batch_size,
                                        _stream(stream)), "crypto_sign_sign_HtD")

    def crypto_sign_sign(self, pool, Mlen, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_sign(self.set, _ptr(pool), Mlen, pitch, batch_size, _stream(stream)),
               "crypto_sign_sign")

    def crypto_sign_sign_DtH(self, sig, pool, Mlen, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_sign_DtH(self.set, _ptr(sig), _ptr(pool), Mlen, pitch, batch_size, _stream(stream)),
               "crypto_sign_sign_DtH")

    def crypto_sign_signWithesk_HtD(self, csk, cMess, mlen, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_signWithesk_HtD(self.set, _ptr(csk), _ptr(cMess), mlen, _ptr(pool), pitch,
                                               batch_size, _stream(stream)), "crypto_sign_signWithesk_HtD")

    def crypto_sign_signWithesk(self, pool, Mlen, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_signWithesk(self.set, _ptr(pool), Mlen, pitch, batch_size, _stream(stream)),
               "crypto_sign_signWithesk")

    def crypto_sign_signWithesk_DtH(self, sig, pool, Mlen, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_signWithesk_DtH(self.set, _ptr(sig), _ptr(pool), Mlen, pitch, batch_size,
                                               _stream(stream)), "crypto_sign_signWithesk_DtH")

    # verify ---------------------------------------------------------------------------------
    def crypto_sign_verify_HtD(self, epk, Mess, sig, mlen, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_verify_HtD(self.set, _ptr(epk), _ptr(Mess), _ptr(sig), mlen, _ptr(pool), pitch,
                                          batch_size, _stream(stream)), "crypto_sign_verify_HtD")

    def crypto_sign_verify(self, pool, Mlen, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_verify(self.set, _ptr(pool), Mlen, pitch, batch_size, _stream(stream)),
               "crypto_sign_verify")

    def crypto_sign_verify_DtH(self, verify, Mlen, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_verify_DtH(self.set, _ptr(verify), Mlen, _ptr(pool), pitch, batch_size,
                                          _stream(stream)), "crypto_sign_verify_DtH")

    def crypto_sign_verifyWithepk_HtD(self, cpk, Mess, sig, mlen, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_verifyWithepk_HtD(self.set, _ptr(cpk), _ptr(Mess), _ptr(sig), mlen, _ptr(pool),
                                                 pitch, batch_size, _stream(stream)),
               "crypto_sign_verifyWithepk_HtD")

    def crypto_sign_verifyWithepk(self, pool, Mlen, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_verifyWithepk(self.set, _ptr(pool), Mlen, pitch, batch_size, _stream(stream)),
               "crypto_sign_verifyWithepk")

    def crypto_sign_verifyWithepk_DtH(self, verify, Mlen, pool, pitch, batch_size, stream=None):
        _check(lib().mayo_b200_verifyWithepk_DtH(self.set, _ptr(verify), Mlen, _ptr(pool), pitch, batch_size,
                                                 _stream(stream)), "crypto_sign_verifyWithepk_DtH")

    # extension: explicit operand arrays (shared keys, per-instance message lengths) --------
    def sign_ws_bytes(self) -> int:
        return int(lib().mayo_b200_sign_ws_bytes(self.set))

    def sign_many(self, esk, msgs, sig, ws, batch, *, msg_off=None, msg_len=None, msg_stride=0, mlen=0,
                  esk_stride=0, sig_stride=None, stream=None):
        """Sign `batch` messages (device operands).  esk_stride=0 shares one expanded key."""
        z = self.sizes
        _check(lib().mayo_b200_sign_many(self.set, _ptr(esk), esk_stride, _ptr(msgs), _ptr(msg_off), _ptr(msg_len),
                                         msg_stride, mlen, _ptr(sig), z.sig_bytes if sig_stride is None else sig_stride,
                                         _ptr(ws), batch, _stream(stream)), "sign_many")

    def verify_many(self, epk, msgs, sig, result, batch, *, msg_off=None, msg_len=None, msg_stride=0, mlen=0,
                    epk_stride=0, sig_stride=None, stream=None):
        """Verify `batch` signatures (device operands); result[i] = 0 accept, 1 reject."""
        z = self.sizes
        _check(lib().mayo_b200_verify_many(self.set, _ptr(epk), epk_stride, _ptr(msgs), _ptr(msg_off),
                                           _ptr(msg_len), msg_stride, mlen, _ptr(sig),
                                           z.sig_bytes if sig_stride is None else sig_stride, _ptr(result), batch,
                                           _stream(stream)), "verify_many")

    def sign_shared_ws_bytes(self, batch: int) -> int:
        return int(lib().mayo_b200_sign_shared_ws_bytes(self.set, batch))

    def verify_shared_ws_bytes(self, batch: int) -> int:
        return int(lib().mayo_b200_verify_shared_ws_bytes(self.set, batch))

    def sign_shared(self, esk, msgs, sig, ws, batch, *, msg_off=None, msg_len=None, msg_stride=0, mlen=0,
                    sig_stride=None, stream=None):
        """sign_many under one expanded key for the whole batch, the key's products on the tensor
        cores.  ws: device memory of sign_shared_ws_bytes(batch) bytes, 16-byte aligned."""
        z = self.sizes
        _check(lib().mayo_b200_sign_shared(self.set, _ptr(esk), _ptr(msgs), _ptr(msg_off), _ptr(msg_len), msg_stride,
                                           mlen, _ptr(sig), z.sig_bytes if sig_stride is None else sig_stride,
                                           _ptr(ws), batch, _stream(stream)), "sign_shared")

    def verify_shared(self, epk, msgs, sig, result, ws, batch, *, msg_off=None, msg_len=None, msg_stride=0, mlen=0,
                      sig_stride=None, stream=None):
        """verify_many under one expanded public key for the whole batch, the key's products on
        the tensor cores.  ws: device memory of verify_shared_ws_bytes(batch) bytes."""
        z = self.sizes
        _check(lib().mayo_b200_verify_shared(self.set, _ptr(epk), _ptr(msgs), _ptr(msg_off), _ptr(msg_len),
                                             msg_stride, mlen, _ptr(sig),
                                             z.sig_bytes if sig_stride is None else sig_stride, _ptr(result),
                                             _ptr(ws), batch, _stream(stream)), "verify_shared")

    SHARED_KERNELS = ("hash", "key_tiles", "product", "tail", "fixup")

    def set_shared_shape(self, hash_threads: int = 0, tail_instances: int = 0, product_ctas: int = 0) -> None:
        """Launch shape of this set's sign_shared / verify_shared calls (process-wide): threads
        per CTA of the hash kernels, signatures per sign-tail CTA, CTAs per key-product tile
        (1 or a CTA pair); 0 = default."""
        sh = SharedShape(hash_threads, tail_instances, product_ctas)
        _check(lib().mayo_b200_shared_set_shape(self.set, ctypes.byref(sh)), "shared_set_shape")

    def shared_shape(self) -> dict:
        sh = SharedShape()
        _check(lib().mayo_b200_shared_get_shape(self.set, ctypes.byref(sh)), "shared_get_shape")
        return {"hash_threads": int(sh.hash_threads), "tail_instances": int(sh.tail_instances),
                "product_ctas": int(sh.product_ctas)}

    @staticmethod
    def shared_timing(enable: bool) -> None:
        """Profiling aid: record per-kernel CUDA events inside sign_shared / verify_shared calls
        made from this thread while enabled."""
        _check(lib().mayo_b200_shared_timing(1 if enable else 0), "shared_timing")

    @staticmethod
    def shared_timing_read() -> dict:
        """Milliseconds of each kernel of the last recorded sign_shared / verify_shared call."""
        buf = (ctypes.c_float * 5)()
        _check(lib().mayo_b200_shared_timing_read(buf), "shared_timing_read")
        return dict(zip(Mayo.SHARED_KERNELS, (float(x) for x in buf)))

    def sign_noalloc_max_batch(self) -> int:
        return int(lib().mayo_b200_sign_noalloc_max_batch(self.set))

    def sign_many_noalloc(self, esk, msgs, sig, batch, *, msg_off=None, msg_len=None, msg_stride=0, mlen=0,
                          esk_stride=0, sig_stride=None, stream=None):
        """sign_many without a caller workspace, for callers that cannot allocate device memory:
        the workspace is a fixed array inside the library (batch <= sign_noalloc_max_batch()).
        Calls must not overlap on the GPU.  The first call on a device (and the first after the
        device's context is replaced, e.g. by a device reset) looks up the array's address; make
        it outside stream capture: made during a capture it may fail with MayoError (status
        MAYO_B200_ERR_CUDA)."""
        z = self.sizes
        rc = lib().mayo_b200_sign_many_noalloc(self.set, _ptr(esk), esk_stride, _ptr(msgs), _ptr(msg_off),
                                               _ptr(msg_len), msg_stride, mlen, _ptr(sig),
                                               z.sig_bytes if sig_stride is None else sig_stride, batch,
                                               _stream(stream))
        if rc == 4:
            raise MayoError(f"sign_many_noalloc: batch {batch} exceeds the fixed workspace "
                            f"(at most {self.sign_noalloc_max_batch()} for MAYO_{self.set})")
        _check(rc, "sign_many_noalloc")

    # pools (the reference benchmark's sizes, tests/bench_stream.cu:25-31, 82, 133) ----------
    def pool_bytes(self, kind: str, mlen: int = 0) -> int:
        z = sizes(self.set, mlen)
        return {"keypair": z.pitch_keypair, "expandsk": z.pitch_expandsk, "expandpk": z.pitch_expandpk,
                "sign": z.pitch_sign, "signWithesk": z.pitch_sign_with_esk, "verify": z.pitch_verify,
                "verifyWithepk": z.pitch_verify}[kind]

    def alloc_pool(self, kind: str, batch: int, mlen: int = 0, device=None):
        """A zeroed device pool for `batch` instances, pitch rounded up to 512 bytes like
        cudaMallocPitch.  Returns (tensor, pitch)."""
        import torch
        pitch = (self.pool_bytes(kind, mlen) + 511) // 512 * 512
        t = torch.zeros(batch * pitch, dtype=torch.uint8, device=device or "cuda")
        return t, pitch
