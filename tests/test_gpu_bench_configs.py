"""Parity at the benchmark's own configurations, through the C-ABI, against the oracle.

  C1  MAYO_1 keypair -> sign -> verify, batch 1,024, distinct ChaCha20-seeded keys, 32-byte
      messages: every public key, signature and verify byte (with a tenth of the signatures
      corrupted) equals the oracle's.
  C2  MAYO_2 shared-key sign + verify, batch 65,536, messages of uniform length 32..1024 bytes
      (all eight hashing-order bins): every signature from the tensor-core path equals the
      oracle's, and every verify byte (a tenth corrupted) equals the oracle's verify.
  C3  MAYO_3 / MAYO_5 distinct-key verify, batch 16,384, a tenth corrupted: every verify byte
      is right (corrupted -> 1, others 0), and on a sample spread over the batch the public key,
      the signature and the verify byte equal the oracle's.
The inputs are the ones bench.py times (its ChaCha20 generators, rank 0's seed)."""
import numpy as np
import pytest

import bench
from cumayo_b200 import Mayo
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).copy()).cuda()


def test_c1_mayo1_batch_1024(cuda):
    import torch
    s, batch, mlen = 1, 1024, 32
    m = Mayo(s)
    z = m.sizes
    seeds = bench.seeds_for(1, batch, z.sk_bytes)
    msgs = bench.chacha(b"mayo-b200-msgs-1".ljust(32, b"\0"), batch * mlen).reshape(batch, mlen)
    kpool, kp = m.alloc_pool("keypair", batch)
    K2 = kpool.view(batch, kp)
    K2[:, : z.sk_bytes].copy_(torch.from_numpy(seeds))
    m.crypto_sign_keypair_from_seed(kpool, kp, batch)
    pk = np.zeros((batch, z.pk_bytes), np.uint8)
    sk = np.zeros((batch, z.sk_bytes), np.uint8)
    m.crypto_sign_keypair_DtH(pk, sk, kpool, kp, batch)
    spool, sp = m.alloc_pool("signWithesk", batch, mlen)
    sig = np.zeros((batch, z.sig_bytes), np.uint8)
    m.crypto_sign_signWithesk_HtD(sk, msgs, mlen, spool, sp, batch)
    m.crypto_sign_signWithesk(spool, mlen, sp, batch)
    m.crypto_sign_signWithesk_DtH(sig, spool, mlen, sp, batch)
    torch.cuda.synchronize()
    assert (sk == seeds).all()
    opk = O.keypair_from_seed_batch(s, seeds)
    assert (pk == opk).all()
    mlist = [bytes(x) for x in msgs]
    osig, att = O.sign_batch(s, O.expandsk_batch(s, seeds), mlist)
    assert (att >= 1).all()
    assert (sig == osig).all()
    vsig, bad = bench.corrupt_tenth(sig, 1)
    vpool, vp = m.alloc_pool("verifyWithepk", batch, mlen)
    res = np.full(batch, 0xEE, np.uint8)
    m.crypto_sign_verifyWithepk_HtD(pk, msgs, vsig, mlen, vpool, vp, batch)
    m.crypto_sign_verifyWithepk(vpool, mlen, vp, batch)
    m.crypto_sign_verifyWithepk_DtH(res, mlen, vpool, vp, batch)
    torch.cuda.synchronize()
    ores = O.verify_batch(s, O.expandpk_batch(s, opk), mlist, vsig)
    assert (res == ores).all()
    assert res[bad].all() and int(res.sum()) == len(bad)


def test_c2_mayo2_shared_key_batch_65536(cuda):
    import torch
    s, batch = 2, 65536
    m = Mayo(s)
    z = m.sizes
    seed = bench.seeds_for(1, 1, z.sk_bytes)[0]
    st = torch.cuda.current_stream()
    esk, epk = bench.expand_shared_key(m, seed, torch.device("cuda"), st)
    esk_h = np.frombuffer(O.expandsk(s, seed.tobytes()), np.uint8)
    epk_h = np.frombuffer(O.expandpk(s, O.keypair_from_seed(s, seed.tobytes())), np.uint8)
    assert (esk.cpu().numpy() == esk_h).all() and (epk.cpu().numpy() == epk_h).all()
    body, offs, lens = bench.make_messages(1, batch, 32, 1024)
    assert set(np.minimum(lens // 136, 7).tolist()) == set(range(8)), "every hashing-order bin is used"
    d_msg, d_off, d_len = _dev(body), _dev(offs.view(np.int64)), _dev(lens.view(np.int32))
    sig = torch.zeros(batch * z.sig_bytes, dtype=torch.uint8, device="cuda")
    ws = torch.zeros(max(m.sign_shared_ws_bytes(batch), m.verify_shared_ws_bytes(batch)), dtype=torch.uint8,
                     device="cuda")
    m.sign_shared(esk, d_msg, sig, ws, batch, msg_off=d_off, msg_len=d_len)
    torch.cuda.synchronize()
    assert int(ws[:4].cpu().numpy().view(np.uint32)[0]) == 0, "tensor-core product fell back"
    got = sig.cpu().numpy().reshape(batch, z.sig_bytes)
    mlist = [body[int(o):int(o) + int(n)].tobytes() for o, n in zip(offs, lens)]
    osig, att = O.sign_batch(s, esk_h[None, :], mlist, shared_key=True)
    assert (att >= 1).all()
    diff = np.flatnonzero((got != osig).any(axis=1))
    assert diff.size == 0, f"{diff.size} signatures differ from the oracle, first {diff[:8].tolist()}"
    vsig, bad = bench.corrupt_tenth(got, 2)
    res = torch.full((batch,), 0xEE, dtype=torch.uint8, device="cuda")
    m.verify_shared(epk, d_msg, _dev(vsig.reshape(-1)), res, ws, batch, msg_off=d_off, msg_len=d_len)
    torch.cuda.synchronize()
    assert int(ws[:4].cpu().numpy().view(np.uint32)[0]) == 0, "tensor-core product fell back"
    ores = O.verify_batch(s, epk_h[None, :], mlist, vsig, shared_key=True)
    r = res.cpu().numpy()
    assert (r == ores).all()
    assert r[bad].all() and int(r.sum()) == len(bad)


@pytest.mark.parametrize("s", [3, 5])
def test_c3_distinct_key_verify_batch_16384(cuda, s):
    import torch
    batch, mlen = 16384, 32
    m = Mayo(s)
    z = m.sizes
    st = torch.cuda.current_stream()
    dv = bench.build_distinct_verify(m, batch, 1, mlen, st)
    m.crypto_sign_verify(dv["vpool"], mlen, dv["pitch"], batch, st)
    torch.cuda.synchronize()
    res = dv["rows"][:, dv["res_off"]].cpu().numpy()
    expect = np.zeros(batch, np.uint8)
    expect[dv["bad"]] = 1
    assert (res == expect).all()
    # the oracle on a sample spread over the batch (the oracle's MAYO_5 key set-up is slow on a CPU)
    idx = np.arange(0, batch, 32 if s == 5 else 16)
    seeds = dv["seeds"][idx]
    opk = O.keypair_from_seed_batch(s, seeds)
    assert (dv["pks"][idx] == opk).all()
    mlist = [bytes(x) for x in dv["msgs"][idx]]
    osig, _ = O.sign_batch(s, O.expandsk_batch(s, seeds), mlist)
    assert (dv["good_sigs"][idx] == osig).all()
    ores = O.verify_batch(s, O.expandpk_batch(s, opk), mlist, dv["sigs"][idx])
    assert (res[idx] == ores).all()
    assert ores.any(), "the sample holds corrupted signatures"
    # the expanded keys in the verify pool equal the oracle's
    oepk = O.expandpk_batch(s, opk[:4])
    for q in range(4):
        assert (dv["rows"][idx[q], : z.epk_bytes].cpu().numpy() == oepk[q]).all()
