"""Failure detection on the GPU without a fault: bounded device waits are made to run out on
purpose (mayo_b200_test_inject, a flag or a slot that nothing sets), and each test checks that the
error is reported in the status or control words, that every other result is still right
(against the oracle), and that the next call on the same context runs normally.

  * queue: a bucket slot that nothing publishes -> MAYO_B200_QUEUE_ERR_TIMEOUT after spin_limit
  * queue: more re-enqueued signs than slots -> MAYO_B200_QUEUE_ERR_FULL, the item dropped
  * tensor-core product: the key loader stops, the issuers' waits give up -> status word 1 and
    the per-instance engine computes every signature / verify result
The reference has no counterpart: its kernels neither wait nor report errors
(src/sign.cu:244-474 emits the last attempt silently)."""
import hashlib
import json
import os

import numpy as np
import pytest

from cumayo_b200 import Mayo
from cumayo_b200 import api as A
from cumayo_b200 import queue as Q
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).copy()).cuda()


def _reject_msg(s: int, q: int = 0) -> bytes:
    """A 32-byte message whose first sign attempt under the counter key (rand_index 0, instance 0)
    is singular (tests/golden/rejection_msgs.json, pinned by the reference's own build)."""
    g = json.load(open(os.path.join(GOLDEN, f"ref_mayo{s}.json")))["rejection"]
    return hashlib.shake_256(f"reject-search/{s}/{g['indices'][q]}".encode()).digest(32)


@pytest.fixture
def injection():
    yield A.test_inject
    A.test_inject(A.INJECT_NONE)


def test_queue_lost_push_times_out(cuda, injection):
    import torch
    rng = np.random.default_rng(91)
    s = 1
    z = Mayo(s).sizes
    sk, pk = O.keypair(s, 0, 0)
    esk = np.frombuffer(O.expandsk(s, sk), np.uint8)
    epk = np.frombuffer(O.expandpk(s, pk), np.uint8)
    n = 12
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    msgs[3] = np.frombuffer(_reject_msg(s), np.uint8)  # also one re-enqueued sign
    want = np.stack([np.frombuffer(O.sign(s, esk.tobytes(), m.tobytes())[0], np.uint8) for m in msgs])
    vsig = want.copy()
    vsig[5, 7] ^= 0x40
    seeds = rng.integers(0, 256, (4, z.sk_bytes), dtype=np.uint8)

    def operands():
        return Q.SetOperands(kp_seed=_dev(seeds.reshape(-1)),
                             kp_pk=torch.zeros(4 * z.pk_bytes, dtype=torch.uint8, device="cuda"),
                             sg_esk=_dev(esk), sg_nkeys=1, sg_msg=_dev(msgs.reshape(-1)), sg_mlen=32,
                             sg_sig=torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda"),
                             vf_epk=_dev(epk), vf_nkeys=1, vf_msg=_dev(msgs.reshape(-1)), vf_mlen=32,
                             vf_sig=_dev(vsig.reshape(-1)),
                             vf_res=torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda"))

    items = Q.items_array([(Q.OP_KEYPAIR, s, i) for i in range(4)] + [(Q.OP_SIGN, s, i) for i in range(n)] +
                          [(Q.OP_VERIFY, s, i) for i in range(n)])
    expect_res = [1 if i == 5 else 0 for i in range(n)]
    for inject, spin in ((True, 10_000), (False, 0)):  # then the same run without injection
        ops = operands()
        q = Q.Queue(capacity=128, shape=Q.Shape(sms=4))
        q.set_operands(s, ops)
        q.load(items)
        injection(A.INJECT_QUEUE_LOST_PUSH if inject else A.INJECT_NONE)
        q.run(spin_limit=spin)
        torch.cuda.synchronize()
        st = q.stats()
        for op, cnt in ((Q.OP_KEYPAIR, 4), (Q.OP_SIGN, n + 1), (Q.OP_VERIFY, n)):
            p = st["per_bucket"][(s, op)]
            # every real item finished; with injection the bucket's tail holds one more slot
            assert p["finished"] == cnt, (op, p)
            assert p["published"] == cnt + (1 if inject else 0), (op, p)
            assert p["error"] == (Q.QUEUE_ERR_TIMEOUT if inject else Q.QUEUE_OK), (op, p)
        assert (ops.kp_pk.cpu().numpy().reshape(4, z.pk_bytes) == O.keypair_from_seed_batch(s, seeds)).all()
        assert (ops.sg_sig.cpu().numpy().reshape(n, z.sig_bytes) == want).all()
        assert ops.vf_res.cpu().numpy().tolist() == expect_res


def test_queue_full_drops_requeued_sign(cuda):
    """64 sign items in a queue of 64 slots; one needs a second attempt, whose push finds no slot."""
    import torch
    rng = np.random.default_rng(92)
    s = 1
    z = Mayo(s).sizes
    sk, _ = O.keypair(s, 0, 0)
    esk = np.frombuffer(O.expandsk(s, sk), np.uint8)
    n = 64
    msgs = rng.integers(0, 256, (n, 32), dtype=np.uint8)
    r = 17
    msgs[r] = np.frombuffer(_reject_msg(s, 1), np.uint8)
    ops = Q.SetOperands(sg_esk=_dev(esk), sg_nkeys=1, sg_msg=_dev(msgs.reshape(-1)), sg_mlen=32,
                        sg_sig=torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda"))
    q = Q.Queue(capacity=n, shape=Q.Shape(sms=2))  # 64 slots: a multiple of the slot padding
    q.set_operands(s, ops)
    q.load(Q.items_array([(Q.OP_SIGN, s, i) for i in range(n)]))
    q.run(spin_limit=100_000)
    torch.cuda.synchronize()
    p = q.stats()["per_bucket"][(s, Q.OP_SIGN)]
    assert p["error"] == Q.QUEUE_ERR_FULL
    # the push that found no slot raised the tail and counts as finished, so the bucket drains
    # (finished == tail): n items + the dropped second attempt
    assert p["requeued_signs"] == 0 and p["finished"] == p["published"] == n + 1
    got = ops.sg_sig.cpu().numpy().reshape(n, z.sig_bytes)
    want, att = O.sign_batch(s, np.stack([esk] * n), [m.tobytes() for m in msgs])
    assert att[r] == 2 and (att[np.arange(n) != r] == 1).all()
    keep = np.arange(n) != r
    assert (got[keep] == want[keep]).all()
    assert not got[r].any()  # never written


@pytest.mark.parametrize("s", [1, 2, 5])
def test_product_stall_falls_back_to_engine(cuda, injection, s):
    import torch
    m = Mayo(s)
    z = m.sizes
    rng = np.random.default_rng(93 + s)
    n = 300
    sk, pk = O.keypair(s, 0, 0)
    esk_h = O.expandsk(s, sk)
    esk = _dev(np.frombuffer(esk_h, np.uint8))
    epk = _dev(np.frombuffer(O.expandpk(s, pk), np.uint8))
    lens = rng.integers(0, 400, n).astype(np.uint32)
    msgs = [rng.integers(0, 256, int(k), dtype=np.uint8).tobytes() for k in lens]
    msgs[7] = _reject_msg(s)
    lens[7] = 32
    offs = np.concatenate([[0], np.cumsum(lens[:-1])]).astype(np.int64)
    d_msg = _dev(np.frombuffer(b"".join(msgs) + b"\0", np.uint8))
    d_off, d_len = _dev(offs), _dev(lens.view(np.int32))
    want, _ = O.sign_batch(s, np.frombuffer(esk_h, np.uint8)[None, :], msgs, shared_key=True)
    ws = torch.zeros(max(m.sign_shared_ws_bytes(n), m.verify_shared_ws_bytes(n)), dtype=torch.uint8, device="cuda")
    vsig = want.copy()
    vsig[::9, 11] ^= 0x02
    expect = np.zeros(n, np.uint8)
    expect[::9] = 1
    for inject in (True, False):
        injection(A.INJECT_PRODUCT_STALL if inject else A.INJECT_NONE, 1, 4096)
        sig = torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda")
        m.sign_shared(esk, d_msg, sig, ws, n, msg_off=d_off, msg_len=d_len)
        torch.cuda.synchronize()
        assert int(ws[:4].cpu().numpy().view(np.uint32)[0]) == (1 if inject else 0)
        assert (sig.cpu().numpy().reshape(n, z.sig_bytes) == want).all()
        res = torch.full((n,), 0xEE, dtype=torch.uint8, device="cuda")
        m.verify_shared(epk, d_msg, _dev(vsig.reshape(-1)), res, ws, n, msg_off=d_off, msg_len=d_len)
        torch.cuda.synchronize()
        assert int(ws[:4].cpu().numpy().view(np.uint32)[0]) == (1 if inject else 0)
        assert res.cpu().numpy().tolist() == expect.tolist()
