"""One key for a whole batch, the key's products on the tensor cores (mayo_b200_sign_shared /
mayo_b200_verify_shared): byte-identical to the per-instance path (sign_many / verify_many with
a shared key) and to the oracle, on every parameter set, with ragged message lengths, the
reference's golden retry cases (first attempt singular) and corrupted signatures; the status
word must show that the tensor-core product ran (no fallback)."""
import hashlib
import json
import os

import numpy as np
import pytest

from cumayo_b200 import Mayo, MayoError
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).copy()).cuda()


def _messages(s, n, rng):
    lens = [(37 * i) % 301 for i in range(n)]
    msgs = [rng.integers(0, 256, ln, dtype=np.uint8).tobytes() for ln in lens]
    # first attempt singular under the counter key 0 (tests/golden/rejection_msgs.json)
    g = json.load(open(os.path.join(GOLDEN, f"ref_mayo{s}.json")))["rejection"]
    for q, idx in enumerate(g["indices"][:2]):
        msgs[5 + 40 * q] = hashlib.shake_256(f"reject-search/{s}/{idx}".encode()).digest(32)
    return msgs


@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_shared_key_sign_verify_match(cuda, s):
    import torch
    m = Mayo(s)
    z = m.sizes
    rng = np.random.default_rng(100 + s)
    n = 600 if s == 2 else 150  # 600: the hashing-order sort runs over several CTAs
    sk, pk = O.keypair(s, 0, 0)
    esk = _dev(np.frombuffer(O.expandsk(s, sk), np.uint8))
    epk = _dev(np.frombuffer(O.expandpk(s, pk), np.uint8))
    msgs = _messages(s, n, rng)
    lens = np.array([len(x) for x in msgs], np.uint32)
    offs = np.concatenate([[0], np.cumsum(lens[:-1])]).astype(np.int64)
    blob = np.frombuffer(b"".join(msgs) + b"\0", np.uint8)
    d_msg, d_off, d_len = _dev(blob), _dev(offs), _dev(lens.view(np.int32))

    # per-instance path
    sig_ref = torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda")
    ws_ref = torch.zeros(n * m.sign_ws_bytes(), dtype=torch.uint8, device="cuda")
    m.sign_many(esk, d_msg, sig_ref, ws_ref, n, msg_off=d_off, msg_len=d_len)
    # tensor-core path, twice on the same workspace
    ws = torch.zeros(m.sign_shared_ws_bytes(n), dtype=torch.uint8, device="cuda")
    for _ in range(2):
        sig = torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda")
        m.sign_shared(esk, d_msg, sig, ws, n, msg_off=d_off, msg_len=d_len)
        torch.cuda.synchronize()
        assert int(ws[:4].cpu().numpy().view(np.uint32)[0]) == 0, "tensor-core product fell back"
        assert torch.equal(sig, sig_ref)
    got = sig.cpu().numpy().reshape(n, z.sig_bytes)
    esk_h = O.expandsk(s, sk)
    for i in (0, 1, 5, 45, 77, n - 1):
        assert got[i].tobytes() == O.sign(s, esk_h, msgs[i])[0], i

    # verify: every 10th signature corrupted
    vsig = got.copy()
    bad = np.zeros(n, bool)
    bad[::10] = True
    for i in np.flatnonzero(bad):
        vsig[i, (13 * i) % z.sig_bytes] ^= 0x08
    d_sig = _dev(vsig.reshape(-1))
    res_ref = torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda")
    m.verify_many(epk, d_msg, d_sig, res_ref, n, msg_off=d_off, msg_len=d_len)
    vws = torch.zeros(m.verify_shared_ws_bytes(n), dtype=torch.uint8, device="cuda")
    for _ in range(2):
        res = torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda")
        m.verify_shared(epk, d_msg, d_sig, res, vws, n, msg_off=d_off, msg_len=d_len)
        torch.cuda.synchronize()
        assert int(vws[:4].cpu().numpy().view(np.uint32)[0]) == 0, "tensor-core product fell back"
        assert res.cpu().numpy().tolist() == bad.astype(np.uint8).tolist()
        assert torch.equal(res, res_ref)


@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_shared_key_large_batch(cuda, s):
    """Thousands of instances: every SM runs product CTAs at once, so the key stream from L2 lags
    the tensor cores and the loader / issuer / epilogue handshakes are exercised under load."""
    import torch
    m = Mayo(s)
    z = m.sizes
    n = 8192 if s == 2 else 4096
    mlen = 32
    sk, pk = O.keypair(s, 1, 0)
    esk = _dev(np.frombuffer(O.expandsk(s, sk), np.uint8))
    epk = _dev(np.frombuffer(O.expandpk(s, pk), np.uint8))
    rng = np.random.default_rng(7 + s)
    d_msg = _dev(rng.integers(0, 256, n * mlen, dtype=np.uint8))
    sig_ref = torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda")
    ws_ref = torch.zeros(n * m.sign_ws_bytes(), dtype=torch.uint8, device="cuda")
    m.sign_many(esk, d_msg, sig_ref, ws_ref, n, msg_stride=mlen, mlen=mlen)
    ws = torch.zeros(max(m.sign_shared_ws_bytes(n), m.verify_shared_ws_bytes(n)), dtype=torch.uint8, device="cuda")
    sig = torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda")
    m.sign_shared(esk, d_msg, sig, ws, n, msg_stride=mlen, mlen=mlen)
    torch.cuda.synchronize()
    assert int(ws[:4].cpu().numpy().view(np.uint32)[0]) == 0, "tensor-core product fell back"
    assert torch.equal(sig, sig_ref)
    vsig = sig.clone().view(n, z.sig_bytes)
    vsig[::7, 3] ^= 0x10
    res_ref = torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda")
    m.verify_many(epk, d_msg, vsig.view(-1), res_ref, n, msg_stride=mlen, mlen=mlen)
    res = torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda")
    m.verify_shared(epk, d_msg, vsig.view(-1), res, ws, n, msg_stride=mlen, mlen=mlen)
    torch.cuda.synchronize()
    assert int(ws[:4].cpu().numpy().view(np.uint32)[0]) == 0, "tensor-core product fell back"
    assert torch.equal(res, res_ref)
    expect = np.zeros(n, np.uint8)
    expect[::7] = 1
    assert res.cpu().numpy().tolist() == expect.tolist()


@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_shared_key_block_shapes(cuda, s):
    """Every block shape the autotuner may choose (hash CTA threads, sign-tail instances per CTA,
    CTAs per key-product tile) gives the bytes of the per-instance path, also for an odd batch
    (a last CTA half empty; with CTA pairs, an odd number of product CTAs)."""
    import torch
    m = Mayo(s)
    z = m.sizes
    rng = np.random.default_rng(300 + s)
    n = 301
    sk, pk = O.keypair(s, 0, 0)
    esk = _dev(np.frombuffer(O.expandsk(s, sk), np.uint8))
    epk = _dev(np.frombuffer(O.expandpk(s, pk), np.uint8))
    msgs = _messages(s, n, rng)
    lens = np.array([len(x) for x in msgs], np.uint32)
    offs = np.concatenate([[0], np.cumsum(lens[:-1])]).astype(np.int64)
    d_msg, d_off, d_len = _dev(np.frombuffer(b"".join(msgs) + b"\0", np.uint8)), _dev(offs), _dev(lens.view(np.int32))
    sig_ref = torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda")
    ws_ref = torch.zeros(n * m.sign_ws_bytes(), dtype=torch.uint8, device="cuda")
    m.sign_many(esk, d_msg, sig_ref, ws_ref, n, msg_off=d_off, msg_len=d_len)
    res_ref = torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda")
    m.verify_many(epk, d_msg, sig_ref, res_ref, n, msg_off=d_off, msg_len=d_len)
    ws = torch.zeros(max(m.sign_shared_ws_bytes(n), m.verify_shared_ws_bytes(n)), dtype=torch.uint8, device="cuda")
    try:
        for h, g, p in ((32, 2, 1), (128, 4, 1), (256, 1, 1), (64, 1, 2), (64, 4, 2)):
            try:
                m.set_shared_shape(h, g, p)
            except MayoError:  # four MAYO_5 tails do not fit in one CTA's shared memory
                assert s == 5 and g == 4
                continue
            assert m.shared_shape() == {"hash_threads": h, "tail_instances": g, "product_ctas": p}
            sig = torch.zeros_like(sig_ref)
            m.sign_shared(esk, d_msg, sig, ws, n, msg_off=d_off, msg_len=d_len)
            res = torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda")
            m.verify_shared(epk, d_msg, sig, res, ws, n, msg_off=d_off, msg_len=d_len)
            torch.cuda.synchronize()
            assert int(ws[:4].cpu().numpy().view(np.uint32)[0]) == 0, ("product gave up", h, g, p)
            assert torch.equal(sig, sig_ref), (h, g, p)
            assert torch.equal(res, res_ref) and int(res.sum()) == 0, (h, g, p)
    finally:
        m.set_shared_shape(0, 0, 0)
