"""Drivers for the reference-compatible entry points of libmayo_b200.so, used by the GPU
tests, smoke() and bench.py.  Everything goes through the C-ABI (cumayo_b200.Mayo), with
device pools in torch tensors and host buffers in numpy arrays, like a reference caller."""
from __future__ import annotations

import hashlib

import numpy as np

from cumayo_b200 import A128, Mayo  # noqa: F401  (A128 re-exported for tests)


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def golden_message(s: int, i: int, mlen: int) -> bytes:
    return hashlib.shake_256(f"golden/{s}/{i}/{mlen}".encode()).digest(mlen)


def _sync():
    import torch
    torch.cuda.synchronize()


def pool(m: Mayo, kind: str, batch: int, mlen: int = 0, extra: int = 0):
    """Zeroed pool; `extra` bytes are added to the pitch (to exercise unaligned pitches)."""
    import torch
    row = m.pool_bytes(kind, mlen)
    pitch = (row + 511) // 512 * 512 if extra == 0 else row + extra
    return torch.zeros(batch * pitch + 64, dtype=torch.uint8, device="cuda"), pitch


def keypair(m: Mayo, batch: int, rand_index: int = 0, stream=None):
    t, pitch = pool(m, "keypair", batch)
    z = m.sizes
    pk = np.zeros((batch, z.pk_bytes), np.uint8)
    sk = np.zeros((batch, z.sk_bytes), np.uint8)
    m.crypto_sign_keypair(t, pitch, batch, stream, rand_index)
    m.crypto_sign_keypair_DtH(pk, sk, t, pitch, batch, stream)
    _sync()
    return sk, pk


def keypair_from_seed(m: Mayo, seeds: np.ndarray, extra: int = 0):
    import torch
    batch = seeds.shape[0]
    t, pitch = pool(m, "keypair", batch, extra=extra)
    z = m.sizes
    host = torch.zeros((batch, pitch), dtype=torch.uint8)
    host[:, : z.sk_bytes] = torch.from_numpy(np.ascontiguousarray(seeds))
    t[: batch * pitch].copy_(host.reshape(-1))
    m.crypto_sign_keypair_from_seed(t, pitch, batch)
    pk = np.zeros((batch, z.pk_bytes), np.uint8)
    sk = np.zeros((batch, z.sk_bytes), np.uint8)
    m.crypto_sign_keypair_DtH(pk, sk, t, pitch, batch)
    _sync()
    return sk, pk


def expandsk(m: Mayo, csk: np.ndarray, extra: int = 0):
    batch = csk.shape[0]
    t, pitch = pool(m, "expandsk", batch, extra=extra)
    esk = np.zeros((batch, m.sizes.esk_bytes), np.uint8)
    m.crypto_sign_expandsk_HtD(np.ascontiguousarray(csk), t, pitch, batch)
    m.crypto_sign_expandsk(t, pitch, batch)
    m.crypto_sign_expandsk_DtH(esk, t, pitch, batch)
    _sync()
    return esk


def expandpk(m: Mayo, cpk: np.ndarray, extra: int = 0):
    batch = cpk.shape[0]
    t, pitch = pool(m, "expandpk", batch, extra=extra)
    epk = np.zeros((batch, m.sizes.epk_bytes), np.uint8)
    m.crypto_sign_expandpk_HtD(np.ascontiguousarray(cpk), t, pitch, batch)
    m.crypto_sign_expandpk(t, pitch, batch)
    m.crypto_sign_expandpk_DtH(epk, t, pitch, batch)
    _sync()
    return epk


def _msgs(msgs) -> np.ndarray:
    if isinstance(msgs, np.ndarray):
        return np.ascontiguousarray(msgs)
    mlen = len(msgs[0])
    assert all(len(x) == mlen for x in msgs)
    return np.frombuffer(b"".join(msgs), np.uint8).reshape(len(msgs), mlen).copy() if mlen else \
        np.zeros((len(msgs), 0), np.uint8)


def sign_with_esk(m: Mayo, csk: np.ndarray, msgs, extra: int = 0):
    M = _msgs(msgs)
    batch, mlen = M.shape
    t, pitch = pool(m, "signWithesk", batch, mlen, extra=extra)
    sig = np.zeros((batch, m.sizes.sig_bytes), np.uint8)
    m.crypto_sign_signWithesk_HtD(np.ascontiguousarray(csk), M, mlen, t, pitch, batch)
    m.crypto_sign_signWithesk(t, mlen, pitch, batch)
    m.crypto_sign_signWithesk_DtH(sig, t, mlen, pitch, batch)
    _sync()
    return sig


def sign(m: Mayo, esk: np.ndarray, msgs, extra: int = 0):
    M = _msgs(msgs)
    batch, mlen = M.shape
    t, pitch = pool(m, "sign", batch, mlen, extra=extra)
    sig = np.zeros((batch, m.sizes.sig_bytes), np.uint8)
    m.crypto_sign_sign_HtD(np.ascontiguousarray(esk), M, mlen, t, pitch, batch)
    m.crypto_sign_sign(t, mlen, pitch, batch)
    m.crypto_sign_sign_DtH(sig, t, mlen, pitch, batch)
    _sync()
    return sig


def verify_with_epk(m: Mayo, cpk: np.ndarray, msgs, sig: np.ndarray, extra: int = 0):
    M = _msgs(msgs)
    batch, mlen = M.shape
    t, pitch = pool(m, "verifyWithepk", batch, mlen, extra=extra)
    res = np.full(batch, 0xEE, np.uint8)
    m.crypto_sign_verifyWithepk_HtD(np.ascontiguousarray(cpk), M, np.ascontiguousarray(sig), mlen, t, pitch, batch)
    m.crypto_sign_verifyWithepk(t, mlen, pitch, batch)
    m.crypto_sign_verifyWithepk_DtH(res, mlen, t, pitch, batch)
    _sync()
    return res


def verify(m: Mayo, epk: np.ndarray, msgs, sig: np.ndarray, extra: int = 0):
    """crypto_sign_verify_HtD reads epk and sig with 128-byte-aligned host strides."""
    M = _msgs(msgs)
    batch, mlen = M.shape
    z = m.sizes
    t, pitch = pool(m, "verify", batch, mlen, extra=extra)
    epk_p = np.zeros((batch, A128(z.epk_bytes)), np.uint8)
    epk_p[:, : z.epk_bytes] = epk
    sig_p = np.zeros((batch, A128(z.sig_bytes)), np.uint8)
    sig_p[:, : z.sig_bytes] = sig
    res = np.full(batch, 0xEE, np.uint8)
    m.crypto_sign_verify_HtD(epk_p, M, sig_p, mlen, t, pitch, batch)
    m.crypto_sign_verify(t, mlen, pitch, batch)
    m.crypto_sign_verify_DtH(res, mlen, t, pitch, batch)
    _sync()
    return res


def corrupt(sig: np.ndarray, seed: int) -> np.ndarray:
    """Flip one random nibble per signature (nonzero XOR), deterministic in `seed`."""
    rng = np.random.default_rng(seed)
    bad = sig.copy()
    for i in range(bad.shape[0]):
        pos = int(rng.integers(0, 2 * bad.shape[1]))
        bad[i, pos // 2] ^= np.uint8(int(rng.integers(1, 16)) << (4 * (pos % 2)))
    return bad
