"""Parity of the CUDA engine with the reference, through the C-ABI on a GPU.

Pins: golden vectors from the reference's own sm_100a build (tests/golden/ref_mayo*.json),
and the CPU oracle (itself pinned to those vectors) on seeded inputs and edge cases.
Everything is byte/bit exact: keys, expanded keys, signatures, verify bytes."""
import hashlib
import json
import os

import numpy as np
import pytest

import gpu_util as G
from cumayo_b200 import Mayo
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SETS = [1, 2, 3, 5]
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden(s):
    with open(os.path.join(GOLDEN, f"ref_mayo{s}.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module", params=SETS)
def mset(request, cuda):
    return request.param, Mayo(request.param)


def test_keypair_golden(mset):
    s, m = mset
    for ri, kp in golden(s)["keypair"].items():
        sk, pk = G.keypair(m, kp["batch"], int(ri))
        assert [x.tobytes().hex() for x in sk[:4]] == kp["sk"]
        assert [x.tobytes().hex() for x in pk[:4]] == kp["pk"]
        assert G.sha(sk) == kp["sk_sha256"] and G.sha(pk) == kp["pk_sha256"]


def test_expand_golden(mset):
    s, m = mset
    g = golden(s)
    sk, pk = O.keypair_batch(s, 0, 8)
    assert [G.sha(x) for x in G.expandsk(m, sk)] == g["expandsk_sha256"]
    assert [G.sha(x) for x in G.expandpk(m, pk)] == g["expandpk_sha256"]


def test_sign_verify_golden(mset):
    s, m = mset
    g = golden(s)
    sk, pk = O.keypair_batch(s, 0, 8)
    esk = O.expandsk_batch(s, sk)
    epk = O.expandpk_batch(s, pk)
    for ent in g["sign"]:
        msgs = [G.golden_message(s, i, ent["mlen"]) for i in range(8)]
        sig = G.sign_with_esk(m, sk, msgs)
        assert [x.tobytes().hex() for x in sig] == ent["sig_with_esk"], ent["mlen"]
        assert (G.sign(m, esk, msgs) == sig).all(), ent["mlen"]
        bad = np.stack([np.frombuffer(bytes.fromhex(h), np.uint8) for h in ent["bad_sig"]])
        assert list(G.verify_with_epk(m, pk, msgs, sig)) == ent["verify_good"]
        assert list(G.verify_with_epk(m, pk, msgs, bad)) == ent["verify_bad"]
        assert list(G.verify(m, epk, msgs, sig)) == ent["verify_plain_good"]
        assert list(G.verify(m, epk, msgs, bad)) == ent["verify_plain_bad"]


@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_rejection_retry_golden(s, cuda):
    """Messages whose first attempt is singular (attempts == 2): the retry path."""
    m = Mayo(s)
    rej = golden(s)["rejection"]
    sk, pk = O.keypair(s, 0, 0)
    msgs = [hashlib.shake_256(f"reject-search/{s}/{i}".encode()).digest(32) for i in rej["indices"]]
    n = len(msgs)
    csk = np.repeat(np.frombuffer(sk, np.uint8)[None, :], n, 0)
    sig = G.sign_with_esk(m, csk, msgs)
    assert [x.tobytes().hex() for x in sig] == rej["sig"]


def test_seeded_keys_sign_verify_vs_oracle(mset):
    """Caller-seeded keypairs (extension), random messages, mixed in one batch."""
    s, m = mset
    rng = np.random.default_rng(1000 + s)
    batch = 24
    seeds = rng.integers(0, 256, (batch, m.sizes.sk_bytes), dtype=np.uint8)
    sk, pk = G.keypair_from_seed(m, seeds)
    assert (sk == seeds).all()
    assert (pk == O.keypair_from_seed_batch(s, seeds)).all()
    msgs = rng.integers(0, 256, (batch, 77), dtype=np.uint8)
    sig = G.sign_with_esk(m, sk, msgs)
    esk = O.expandsk_batch(s, sk)
    osig, att = O.sign_batch(s, esk, [bytes(x) for x in msgs])
    assert (sig == osig).all()
    bad = G.corrupt(sig, s)
    res = G.verify_with_epk(m, pk, msgs, np.concatenate([sig[:12], bad[12:]]))
    assert list(res) == [0] * 12 + [1] * 12


@pytest.mark.parametrize("mlen", [0, 1, 136, 1024])
def test_message_length_edges(mlen, cuda):
    s = 2
    m = Mayo(s)
    sk, pk = O.keypair_batch(s, 7, 4)
    msgs = [bytes([i + 1]) * mlen for i in range(4)]
    sig = G.sign_with_esk(m, sk, msgs)
    esk = O.expandsk_batch(s, sk)
    osig, _ = O.sign_batch(s, esk, msgs)
    assert (sig == osig).all()
    assert list(G.verify_with_epk(m, pk, msgs, sig)) == [0] * 4


@pytest.mark.parametrize("s", SETS)
def test_unaligned_pitch(s, cuda):
    """Pitches that are not multiples of 16 exercise the unaligned load/store paths."""
    m = Mayo(s)
    sk, pk = O.keypair_batch(s, 3, 3)
    assert (G.expandsk(m, sk, extra=3) == O.expandsk_batch(s, sk)).all()
    assert (G.expandpk(m, pk, extra=5) == O.expandpk_batch(s, pk)).all()
    msgs = [b"abc", b"def", b"ghi"]
    sig = G.sign_with_esk(m, sk, msgs, extra=7)
    osig, _ = O.sign_batch(s, O.expandsk_batch(s, sk), msgs)
    assert (sig == osig).all()
    assert list(G.verify_with_epk(m, pk, msgs, sig, extra=9)) == [0, 0, 0]


def test_multi_stream_sub_batches(cuda):
    """The reference benchmark's pattern: sub-batches of one pool on 10 concurrent streams,
    every sub-batch starting at rand_index 0 (tests/bench_stream.cu:33-44)."""
    import torch
    s = 1
    m = Mayo(s)
    batch, nst = 40, 10
    t, pitch = G.pool(m, "keypair", batch)
    streams = [torch.cuda.Stream() for _ in range(nst)]
    z = m.sizes
    pk = np.zeros((batch, z.pk_bytes), np.uint8)
    sk = np.zeros((batch, z.sk_bytes), np.uint8)
    sub = batch // nst
    for i, st in enumerate(streams):
        base = i * sub
        m.crypto_sign_keypair(t.data_ptr() + base * pitch, pitch, sub, st, 0)
        m.crypto_sign_keypair_DtH(pk[base:].ctypes.data, sk[base:].ctypes.data, t.data_ptr() + base * pitch, pitch,
                                  sub, st)
    torch.cuda.synchronize()
    osk, opk = O.keypair_batch(s, 0, sub)
    for i in range(nst):
        assert (sk[i * sub:(i + 1) * sub] == osk).all() and (pk[i * sub:(i + 1) * sub] == opk).all()


@pytest.mark.parametrize("s", SETS)
def test_many_api_shared_key_variable_lengths(s, cuda):
    """Extension API: one resident expanded key, per-instance message lengths, vs the oracle;
    also equal to the pool API.  Corrupted signatures must be rejected."""
    import torch
    m = Mayo(s)
    z = m.sizes
    rng = np.random.default_rng(77 + s)
    seed = rng.integers(0, 256, (1, z.sk_bytes), dtype=np.uint8)
    sk, pk = G.keypair_from_seed(m, seed)
    esk = O.expandsk_batch(s, sk)[0]
    epk = O.expandpk_batch(s, pk)[0]
    batch = 40
    lens = rng.integers(0, 300, batch).astype(np.uint32)
    msgs = [rng.integers(0, 256, int(n), dtype=np.uint8).tobytes() for n in lens]
    offs = np.zeros(batch, np.uint64)
    offs[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
    d_msgs = torch.from_numpy(np.frombuffer(b"".join(msgs) + b"\0", np.uint8).copy()).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    d_lens = torch.from_numpy(lens.view(np.int32)).cuda()
    d_esk = torch.from_numpy(esk.copy()).cuda()
    d_epk = torch.from_numpy(epk.copy()).cuda()
    sig = torch.zeros(batch * z.sig_bytes, dtype=torch.uint8, device="cuda")
    ws = torch.zeros(batch * m.sign_ws_bytes(), dtype=torch.uint8, device="cuda")
    m.sign_many(d_esk, d_msgs, sig, ws, batch, msg_off=d_offs, msg_len=d_lens)
    res = torch.full((batch,), 0xEE, dtype=torch.uint8, device="cuda")
    m.verify_many(d_epk, d_msgs, sig, res, batch, msg_off=d_offs, msg_len=d_lens)
    torch.cuda.synchronize()
    osig, _ = O.sign_batch(s, esk[None, :], msgs, shared_key=True)
    got = sig.cpu().numpy().reshape(batch, z.sig_bytes)
    assert (got == osig).all()
    assert res.cpu().numpy().tolist() == [0] * batch
    bad = torch.from_numpy(G.corrupt(got, 5 + s).reshape(-1)).cuda()
    m.verify_many(d_epk, d_msgs, bad, res, batch, msg_off=d_offs, msg_len=d_lens)
    torch.cuda.synchronize()
    assert res.cpu().numpy().tolist() == [1] * batch
