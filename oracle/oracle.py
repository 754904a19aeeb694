"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the parity checker used by tests/, by
``__graft_entry__.smoke()`` and by bench.py's CPU-baseline leg.  The product
(the ``cumayo_b200`` package) never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    """Compile liboracle.so (gcc, OpenMP) if it is missing or stale."""
    src = os.path.join(_HERE, "mayo_oracle.c")
    hdr = os.path.join(_HERE, "mayo_oracle.h")
    stale = (not os.path.exists(_LIB_PATH) or
             os.path.getmtime(_LIB_PATH) < max(os.path.getmtime(src), os.path.getmtime(hdr)))
    if stale:
        subprocess.run(["make", "-C", _HERE, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return _LIB_PATH


class _Params(ctypes.Structure):
    _fields_ = [(name, ctypes.c_int) for name in (
        "id", "n", "m", "o", "k", "v", "menc", "sk_bytes", "pk_bytes", "p_bytes", "o_bytes",
        "p1_bytes", "p2_bytes", "digest_bytes", "pairs")] + [
        ("poly_c", ctypes.c_uint8 * 4)] + [(name, ctypes.c_int) for name in (
            "sig_bytes", "esk_bytes", "epk_bytes")]


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        L.mayo_oracle_get_params.restype = ctypes.POINTER(_Params)
        L.mayo_oracle_get_params.argtypes = [ctypes.c_int]
        for fn in ("mayo_oracle_shake128", "mayo_oracle_shake256"):
            getattr(L, fn).argtypes = [u8p, ctypes.c_size_t, u8p, ctypes.c_size_t]
        L.mayo_oracle_aes128_ctr.argtypes = [u8p, u8p, ctypes.c_size_t]
        L.mayo_oracle_gf16_mul.restype = ctypes.c_uint8
        L.mayo_oracle_gf16_mul.argtypes = [ctypes.c_uint8, ctypes.c_uint8]
        L.mayo_oracle_gf16_inv.restype = ctypes.c_uint8
        L.mayo_oracle_gf16_inv.argtypes = [ctypes.c_uint8]
        L.mayo_oracle_table_digest.argtypes = [u8p, u8p]
        L.mayo_oracle_keypair.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64, u8p, u8p]
        L.mayo_oracle_keypair_from_seed.argtypes = [ctypes.c_int, u8p, u8p]
        L.mayo_oracle_expandsk.argtypes = [ctypes.c_int, u8p, u8p]
        L.mayo_oracle_expandpk.argtypes = [ctypes.c_int, u8p, u8p]
        L.mayo_oracle_sign.argtypes = [ctypes.c_int, u8p, u8p, ctypes.c_size_t, u8p, ctypes.c_int]
        L.mayo_oracle_verify.argtypes = [ctypes.c_int, u8p, u8p, ctypes.c_size_t, u8p]
        L.mayo_oracle_max_threads.restype = ctypes.c_int
        L.mayo_oracle_set_threads.argtypes = [ctypes.c_int]
        L.mayo_oracle_keypair_batch.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.c_size_t, u8p, u8p]
        L.mayo_oracle_keypair_from_seed_batch.argtypes = [ctypes.c_int, ctypes.c_size_t, u8p, u8p]
        L.mayo_oracle_expandsk_batch.argtypes = [ctypes.c_int, ctypes.c_size_t, u8p, u8p]
        L.mayo_oracle_expandpk_batch.argtypes = [ctypes.c_int, ctypes.c_size_t, u8p, u8p]
        L.mayo_oracle_sign_batch.argtypes = [ctypes.c_int, ctypes.c_size_t, u8p, ctypes.c_size_t, u8p,
                                             ctypes.POINTER(ctypes.c_uint64),
                                             ctypes.POINTER(ctypes.c_uint32), u8p,
                                             ctypes.POINTER(ctypes.c_int32)]
        L.mayo_oracle_verify_batch.argtypes = [ctypes.c_int, ctypes.c_size_t, u8p, ctypes.c_size_t, u8p,
                                               ctypes.POINTER(ctypes.c_uint64),
                                               ctypes.POINTER(ctypes.c_uint32), u8p, u8p]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def _buf(data) -> np.ndarray:
    return np.ascontiguousarray(np.frombuffer(bytes(data), dtype=np.uint8))


@dataclass(frozen=True)
class Params:
    id: int
    n: int
    m: int
    o: int
    k: int
    v: int
    menc: int
    sk_bytes: int
    pk_bytes: int
    p_bytes: int
    o_bytes: int
    p1_bytes: int
    p2_bytes: int
    digest_bytes: int
    pairs: int
    poly_c: tuple
    sig_bytes: int
    esk_bytes: int
    epk_bytes: int


def params(set_id: int) -> Params:
    p = lib().mayo_oracle_get_params(set_id)
    if not p:
        raise ValueError(f"unknown MAYO set {set_id}")
    c = p.contents
    return Params(c.id, c.n, c.m, c.o, c.k, c.v, c.menc, c.sk_bytes, c.pk_bytes, c.p_bytes, c.o_bytes,
                  c.p1_bytes, c.p2_bytes, c.digest_bytes, c.pairs, tuple(c.poly_c), c.sig_bytes,
                  c.esk_bytes, c.epk_bytes)


def shake128(data: bytes, outlen: int) -> bytes:
    src = _buf(data) if len(data) else np.zeros(1, np.uint8)
    out = np.zeros(max(outlen, 1), np.uint8)
    lib().mayo_oracle_shake128(_p(out), outlen, _p(src), len(data))
    return out[:outlen].tobytes()


def shake256(data: bytes, outlen: int) -> bytes:
    src = _buf(data) if len(data) else np.zeros(1, np.uint8)
    out = np.zeros(max(outlen, 1), np.uint8)
    lib().mayo_oracle_shake256(_p(out), outlen, _p(src), len(data))
    return out[:outlen].tobytes()


def aes128_ctr(key: bytes, outlen: int) -> bytes:
    k = _buf(key)
    out = np.zeros(max(outlen, 1), np.uint8)
    lib().mayo_oracle_aes128_ctr(_p(k), _p(out), outlen)
    return out[:outlen].tobytes()


def gf16_mul(a: int, b: int) -> int:
    return int(lib().mayo_oracle_gf16_mul(a, b))


def gf16_inv(a: int) -> int:
    return int(lib().mayo_oracle_gf16_inv(a))


def table_digests() -> tuple[str, str]:
    a = np.zeros(32, np.uint8)
    b = np.zeros(32, np.uint8)
    lib().mayo_oracle_table_digest(_p(a), _p(b))
    return a.tobytes().hex(), b.tobytes().hex()


def keypair(set_id: int, rand_index: int, index: int) -> tuple[bytes, bytes]:
    P = params(set_id)
    sk = np.zeros(P.sk_bytes, np.uint8)
    pk = np.zeros(P.pk_bytes, np.uint8)
    lib().mayo_oracle_keypair(set_id, rand_index, index, _p(sk), _p(pk))
    return sk.tobytes(), pk.tobytes()


def keypair_from_seed(set_id: int, seed: bytes) -> bytes:
    P = params(set_id)
    s = _buf(seed)
    pk = np.zeros(P.pk_bytes, np.uint8)
    lib().mayo_oracle_keypair_from_seed(set_id, _p(s), _p(pk))
    return pk.tobytes()


def expandsk(set_id: int, csk: bytes) -> bytes:
    P = params(set_id)
    s = _buf(csk)
    esk = np.zeros(P.esk_bytes, np.uint8)
    lib().mayo_oracle_expandsk(set_id, _p(s), _p(esk))
    return esk.tobytes()


def expandpk(set_id: int, cpk: bytes) -> bytes:
    P = params(set_id)
    s = _buf(cpk)
    epk = np.zeros(P.epk_bytes, np.uint8)
    lib().mayo_oracle_expandpk(set_id, _p(s), _p(epk))
    return epk.tobytes()


def sign(set_id: int, esk: bytes, msg: bytes, force_reject: int = 0) -> tuple[bytes, int]:
    """Returns (signature, attempts used; 0 = every attempt rejected)."""
    P = params(set_id)
    e = _buf(esk)
    m = _buf(msg) if len(msg) else np.zeros(1, np.uint8)
    sig = np.zeros(P.sig_bytes, np.uint8)
    att = lib().mayo_oracle_sign(set_id, _p(e), _p(m), len(msg), _p(sig), force_reject)
    return sig.tobytes(), int(att)


def verify(set_id: int, epk: bytes, msg: bytes, sig: bytes) -> int:
    """0 = accept, 1 = reject."""
    e = _buf(epk)
    m = _buf(msg) if len(msg) else np.zeros(1, np.uint8)
    s = _buf(sig)
    return int(lib().mayo_oracle_verify(set_id, _p(e), _p(m), len(msg), _p(s)))


def max_threads() -> int:
    return int(lib().mayo_oracle_max_threads())


def set_threads(n: int) -> None:
    lib().mayo_oracle_set_threads(int(n))


def keypair_batch(set_id: int, rand_index: int, batch: int) -> tuple[np.ndarray, np.ndarray]:
    P = params(set_id)
    sk = np.zeros((batch, P.sk_bytes), np.uint8)
    pk = np.zeros((batch, P.pk_bytes), np.uint8)
    lib().mayo_oracle_keypair_batch(set_id, rand_index, batch, _p(sk), _p(pk))
    return sk, pk


def keypair_from_seed_batch(set_id: int, seeds: np.ndarray) -> np.ndarray:
    P = params(set_id)
    seeds = np.ascontiguousarray(seeds, dtype=np.uint8)
    pk = np.zeros((seeds.shape[0], P.pk_bytes), np.uint8)
    lib().mayo_oracle_keypair_from_seed_batch(set_id, seeds.shape[0], _p(seeds), _p(pk))
    return pk


def expandsk_batch(set_id: int, csk: np.ndarray) -> np.ndarray:
    P = params(set_id)
    csk = np.ascontiguousarray(csk, dtype=np.uint8)
    esk = np.zeros((csk.shape[0], P.esk_bytes), np.uint8)
    lib().mayo_oracle_expandsk_batch(set_id, csk.shape[0], _p(csk), _p(esk))
    return esk


def expandpk_batch(set_id: int, cpk: np.ndarray) -> np.ndarray:
    P = params(set_id)
    cpk = np.ascontiguousarray(cpk, dtype=np.uint8)
    epk = np.zeros((cpk.shape[0], P.epk_bytes), np.uint8)
    lib().mayo_oracle_expandpk_batch(set_id, cpk.shape[0], _p(cpk), _p(epk))
    return epk


def _msgs(msgs: list[bytes]):
    lens = np.array([len(m) for m in msgs], dtype=np.uint32)
    offs = np.zeros(len(msgs), dtype=np.uint64)
    if len(msgs) > 1:
        offs[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
    flat = np.frombuffer(b"".join(msgs) + b"\0", dtype=np.uint8).copy()
    return flat, offs, lens


def sign_batch(set_id: int, esk: np.ndarray, msgs: list[bytes], shared_key: bool = False):
    P = params(set_id)
    esk = np.ascontiguousarray(esk, dtype=np.uint8)
    flat, offs, lens = _msgs(msgs)
    sig = np.zeros((len(msgs), P.sig_bytes), np.uint8)
    att = np.zeros(len(msgs), np.int32)
    lib().mayo_oracle_sign_batch(set_id, len(msgs), _p(esk), 0 if shared_key else P.esk_bytes, _p(flat),
                                 offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                 lens.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), _p(sig),
                                 att.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return sig, att


def verify_batch(set_id: int, epk: np.ndarray, msgs: list[bytes], sig: np.ndarray,
                 shared_key: bool = False) -> np.ndarray:
    P = params(set_id)
    epk = np.ascontiguousarray(epk, dtype=np.uint8)
    sig = np.ascontiguousarray(sig, dtype=np.uint8)
    flat, offs, lens = _msgs(msgs)
    res = np.zeros(len(msgs), np.uint8)
    lib().mayo_oracle_verify_batch(set_id, len(msgs), _p(epk), 0 if shared_key else P.epk_bytes, _p(flat),
                                   offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                   lens.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), _p(sig), _p(res))
    return res
