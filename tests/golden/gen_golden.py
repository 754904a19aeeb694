"""Generate golden vectors by running the reference's own CUDA build on a GPU.

Needs a CUDA GPU and the reference libraries built by ``make -C oracle ref``
(oracle/_ref/libref_mayo{1,2,3,5}.so, compiled from the unmodified reference
sources).  Writes tests/golden/ref_mayo{1,2,3,5}.json.  Each file holds, for
one parameter set, what the reference's public entry points (include/api.cuh)
produced:

* keypairs (crypto_sign_keypair) for two rand_index values -- full sk/pk bytes
  for a few instances, SHA-256 of the whole batch;
* SHA-256 of expanded keys (crypto_sign_expandsk / crypto_sign_expandpk);
* signatures (crypto_sign_signWithesk, and crypto_sign_sign on the expanded
  key) of deterministic messages of several lengths, plus the messages from
  rejection_msgs.json whose first attempt is rejected;
* verify bytes (crypto_sign_verifyWithepk and crypto_sign_verify) for good and
  corrupted signatures.

The oracle is then checked against these files by tests/test_oracle_golden.py.
Usage (on a GPU box):  python tests/golden/gen_golden.py [--out DIR] [sets...]
"""
from __future__ import annotations

import ctypes
import hashlib
import json
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def A128(x: int) -> int:
    return (x + 127) // 128 * 128


def sha(b) -> str:
    return hashlib.sha256(bytes(b)).hexdigest()


def message(set_id: int, i: int, mlen: int) -> bytes:
    return hashlib.shake_256(f"golden/{set_id}/{i}/{mlen}".encode()).digest(mlen)


class Ref:
    def __init__(self, set_id: int):
        self.lib = ctypes.CDLL(os.path.join(REF_DIR, f"libref_mayo{set_id}.so"))
        p = (ctypes.c_long * 12)()
        self.lib.ref_params(p)
        (self.n, self.m, self.o, self.k, self.sk, self.pk, self.p, self.ob, self.p1, self.p2,
         self.dig, self.pairs) = list(p)
        self.sig = self.k * self.n // 2 + self.sk
        self.esk = self.sk + self.ob + self.p
        self.epk = self.p + self.pk - 16
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        L = self.lib
        L.ref_keypair.argtypes = [vp, sz, sz, vp, sz]
        L.ref_keypair_DtH.argtypes = [vp, vp, vp, sz, sz, vp]
        for f in ("ref_expandsk_HtD", "ref_expandsk_DtH", "ref_expandpk_HtD", "ref_expandpk_DtH"):
            getattr(L, f).argtypes = [vp, vp, sz, sz, vp]
        for f in ("ref_expandsk", "ref_expandpk"):
            getattr(L, f).argtypes = [vp, sz, sz, vp]
        for f in ("ref_sign_HtD", "ref_signWithesk_HtD"):
            getattr(L, f).argtypes = [vp, vp, sz, vp, sz, sz, vp]
        for f in ("ref_sign", "ref_signWithesk", "ref_verify", "ref_verifyWithepk"):
            getattr(L, f).argtypes = [vp, sz, sz, sz, vp]
        for f in ("ref_sign_DtH", "ref_signWithesk_DtH"):
            getattr(L, f).argtypes = [vp, vp, sz, sz, sz, vp]
        for f in ("ref_verify_HtD", "ref_verifyWithepk_HtD"):
            getattr(L, f).argtypes = [vp, vp, vp, sz, vp, sz, sz, vp]
        for f in ("ref_verify_DtH", "ref_verifyWithepk_DtH"):
            getattr(L, f).argtypes = [vp, sz, vp, sz, sz, vp]
        L.ref_init()

    def sync(self):
        rc = self.lib.ref_sync()
        if rc != 0:
            raise RuntimeError(f"CUDA error {rc}")

    @staticmethod
    def pool(batch: int, row: int):
        pitch = (row + 511) // 512 * 512
        t = torch.zeros(batch * pitch, dtype=torch.uint8, device="cuda")
        return t, pitch

    @staticmethod
    def ptr(a: np.ndarray):
        return a.ctypes.data

    def keypair(self, batch: int, rand_index: int):
        row = A128(self.pk) + A128(self.sk) + A128(self.p1 + self.p2)
        t, pitch = self.pool(batch, row)
        pk = np.zeros((batch, self.pk), np.uint8)
        sk = np.zeros((batch, self.sk), np.uint8)
        self.lib.ref_keypair(t.data_ptr(), pitch, batch, None, rand_index)
        self.lib.ref_keypair_DtH(self.ptr(pk), self.ptr(sk), t.data_ptr(), pitch, batch, None)
        self.sync()
        return sk, pk

    def expandsk(self, csk: np.ndarray):
        batch = csk.shape[0]
        t, pitch = self.pool(batch, self.esk)
        esk = np.zeros((batch, self.esk), np.uint8)
        csk = np.ascontiguousarray(csk)
        self.lib.ref_expandsk_HtD(self.ptr(csk), t.data_ptr(), pitch, batch, None)
        self.lib.ref_expandsk(t.data_ptr(), pitch, batch, None)
        self.lib.ref_expandsk_DtH(self.ptr(esk), t.data_ptr(), pitch, batch, None)
        self.sync()
        return esk

    def expandpk(self, cpk: np.ndarray):
        batch = cpk.shape[0]
        t, pitch = self.pool(batch, self.epk)
        epk = np.zeros((batch, self.epk), np.uint8)
        cpk = np.ascontiguousarray(cpk)
        self.lib.ref_expandpk_HtD(self.ptr(cpk), t.data_ptr(), pitch, batch, None)
        self.lib.ref_expandpk(t.data_ptr(), pitch, batch, None)
        self.lib.ref_expandpk_DtH(self.ptr(epk), t.data_ptr(), pitch, batch, None)
        self.sync()
        return epk

    def sign_with_esk(self, csk: np.ndarray, msgs: np.ndarray):
        batch, mlen = msgs.shape
        scratch = self.k * self.m * ((self.o + 1) // 2)
        row = A128(self.esk) + A128(mlen) + A128(self.sig) + A128(scratch)
        t, pitch = self.pool(batch, row)
        sig = np.zeros((batch, self.sig), np.uint8)
        csk, msgs = np.ascontiguousarray(csk), np.ascontiguousarray(msgs)
        self.lib.ref_signWithesk_HtD(self.ptr(csk), self.ptr(msgs), mlen, t.data_ptr(), pitch, batch, None)
        self.lib.ref_signWithesk(t.data_ptr(), mlen, pitch, batch, None)
        self.lib.ref_signWithesk_DtH(self.ptr(sig), t.data_ptr(), mlen, pitch, batch, None)
        self.sync()
        return sig

    def sign(self, esk: np.ndarray, msgs: np.ndarray):
        batch, mlen = msgs.shape
        scratch = self.k * self.m * ((self.o + 1) // 2)
        row = self.esk + mlen + self.sig + scratch
        t, pitch = self.pool(batch, row)
        sig = np.zeros((batch, self.sig), np.uint8)
        esk, msgs = np.ascontiguousarray(esk), np.ascontiguousarray(msgs)
        self.lib.ref_sign_HtD(self.ptr(esk), self.ptr(msgs), mlen, t.data_ptr(), pitch, batch, None)
        self.lib.ref_sign(t.data_ptr(), mlen, pitch, batch, None)
        self.lib.ref_sign_DtH(self.ptr(sig), t.data_ptr(), mlen, pitch, batch, None)
        self.sync()
        return sig

    def verify_with_epk(self, cpk: np.ndarray, msgs: np.ndarray, sig: np.ndarray):
        batch, mlen = msgs.shape
        row = A128(self.epk) + A128(mlen) + A128(self.sig) + 1
        t, pitch = self.pool(batch, row)
        res = np.full(batch, 0xEE, np.uint8)
        cpk, msgs, sig = (np.ascontiguousarray(x) for x in (cpk, msgs, sig))
        self.lib.ref_verifyWithepk_HtD(self.ptr(cpk), self.ptr(msgs), self.ptr(sig), mlen, t.data_ptr(),
                                       pitch, batch, None)
        self.lib.ref_verifyWithepk(t.data_ptr(), mlen, pitch, batch, None)
        self.lib.ref_verifyWithepk_DtH(self.ptr(res), mlen, t.data_ptr(), pitch, batch, None)
        self.sync()
        return res

    def verify(self, epk: np.ndarray, msgs: np.ndarray, sig: np.ndarray):
        """crypto_sign_verify_HtD takes 128-byte-aligned host strides for epk and sig."""
        batch, mlen = msgs.shape
        row = A128(self.epk) + A128(mlen) + A128(self.sig) + 1
        t, pitch = self.pool(batch, row)
        res = np.full(batch, 0xEE, np.uint8)
        epk_p = np.zeros((batch, A128(self.epk)), np.uint8)
        epk_p[:, :self.epk] = epk
        sig_p = np.zeros((batch, A128(self.sig)), np.uint8)
        sig_p[:, :self.sig] = sig
        msgs = np.ascontiguousarray(msgs)
        self.lib.ref_verify_HtD(self.ptr(epk_p), self.ptr(msgs), self.ptr(sig_p), mlen, t.data_ptr(), pitch,
                                batch, None)
        self.lib.ref_verify(t.data_ptr(), mlen, pitch, batch, None)
        self.lib.ref_verify_DtH(self.ptr(res), mlen, t.data_ptr(), pitch, batch, None)
        self.sync()
        return res


def corrupt(sig: np.ndarray, set_id: int, salt: int) -> np.ndarray:
    """Flip one nibble per row at a deterministic position."""
    bad = sig.copy()
    for i in range(bad.shape[0]):
        h = hashlib.sha256(f"corrupt/{set_id}/{salt}/{i}".encode()).digest()
        pos = int.from_bytes(h[:4], "little") % (2 * bad.shape[1])
        val = (h[4] % 15) + 1
        bad[i, pos // 2] ^= val << (4 * (pos % 2))
    return bad


def gen(set_id: int, rej: dict) -> dict:
    R = Ref(set_id)
    out = {"set": set_id, "generator": "reference CUDA build (oracle/_ref), sm_100a",
           "sizes": {"sk": R.sk, "pk": R.pk, "sig": R.sig, "esk": R.esk, "epk": R.epk}}
    kp = {}
    for ri in (0, 12345):
        sk, pk = R.keypair(64, ri)
        kp[str(ri)] = {"batch": 64, "sk_sha256": sha(sk), "pk_sha256": sha(pk),
                       "sk": [bytes(x).hex() for x in sk[:4]], "pk": [bytes(x).hex() for x in pk[:4]]}
    out["keypair"] = kp

    sk, pk = R.keypair(8, 0)
    esk = R.expandsk(sk)
    epk = R.expandpk(pk)
    out["expandsk_sha256"] = [sha(x) for x in esk]
    out["expandpk_sha256"] = [sha(x) for x in epk]

    sigs = []
    for mlen in (1, 32, 100, 135, 136, 137, 300, 1024):
        msgs = np.stack([np.frombuffer(message(set_id, i, mlen), np.uint8) for i in range(8)])
        s1 = R.sign_with_esk(sk, msgs)
        s2 = R.sign(esk, msgs)
        good = R.verify_with_epk(pk, msgs, s1)
        bad_sig = corrupt(s1, set_id, mlen)
        bad = R.verify_with_epk(pk, msgs, bad_sig)
        good2 = R.verify(epk, msgs, s1)
        bad2 = R.verify(epk, msgs, bad_sig)
        sigs.append({"mlen": mlen, "sig_with_esk": [bytes(x).hex() for x in s1],
                     "sig_plain_equal": bool((s1 == s2).all()),
                     "verify_good": good.tolist(), "verify_bad": bad.tolist(),
                     "verify_plain_good": good2.tolist(), "verify_plain_bad": bad2.tolist(),
                     "bad_sig": [bytes(x).hex() for x in bad_sig]})
    out["sign"] = sigs

    rs = rej.get(str(set_id))
    if rs and rs["messages"]:
        sk1, pk1 = R.keypair(1, rs["rand_index"])
        msgs = np.stack([np.frombuffer(hashlib.shake_256(f"reject-search/{set_id}/{e['index']}".encode())
                                       .digest(rs["mlen"]), np.uint8) for e in rs["messages"]])
        n = msgs.shape[0]
        s = R.sign_with_esk(np.repeat(sk1, n, 0), msgs)
        ok = R.verify_with_epk(np.repeat(pk1, n, 0), msgs, s)
        out["rejection"] = {"indices": [e["index"] for e in rs["messages"]],
                            "attempts_oracle": [e["attempts"] for e in rs["messages"]],
                            "sig": [bytes(x).hex() for x in s], "verify": ok.tolist()}
    return out


def main():
    rej_path = os.path.join(HERE, "rejection_msgs.json")
    rej = json.load(open(rej_path)) if os.path.exists(rej_path) else {}
    args = sys.argv[1:]
    out_dir = HERE
    if "--out" in args:
        i = args.index("--out")
        out_dir = args[i + 1]
        del args[i:i + 2]
    os.makedirs(out_dir, exist_ok=True)
    sets = [int(a) for a in args] or [1, 2, 3, 5]
    for s in sets:
        d = gen(s, rej)
        with open(os.path.join(out_dir, f"ref_mayo{s}.json"), "w") as f:
            json.dump(d, f, indent=0)
        print(f"MAYO_{s}: golden written", flush=True)


if __name__ == "__main__":
    main()
