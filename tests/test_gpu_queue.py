"""Persistent work queue on the GPU: keypair / sign / verify items of all four parameter sets in
one run, shuffled together, checked byte for byte against the oracle and the reference's golden
retry cases (a singular first attempt is re-enqueued on the device); the same run captured in a
CUDA graph and replayed; per-instance keys and messages; operand errors; a graph replayed with a
count read on the device."""
import hashlib
import json
import os

import numpy as np
import pytest

from cumayo_b200 import Mayo
from cumayo_b200 import queue as Q
from oracle import oracle as O

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SETS = [1, 2, 3, 5]
MLEN = 32


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def build_case(rng):
    import torch
    operands, expect, entries, n_retry = {}, {}, [], 0
    for s in SETS:
        z = Mayo(s).sizes
        # keypairs from caller seeds
        seeds = rng.integers(0, 256, (3, z.sk_bytes), dtype=np.uint8)
        kp_pk = torch.zeros(3 * z.pk_bytes, dtype=torch.uint8, device="cuda")
        # two signing keys: the counter key (golden retry cases use it) and a random one
        sk0, pk0 = O.keypair(s, 0, 0)
        seed1 = rng.integers(0, 256, z.sk_bytes, dtype=np.uint8).tobytes()
        pk1 = O.keypair_from_seed(s, seed1)
        esk = np.stack([np.frombuffer(O.expandsk(s, k), np.uint8) for k in (sk0, seed1)])
        epk = np.stack([np.frombuffer(O.expandpk(s, k), np.uint8) for k in (pk0, pk1)])
        msgs = rng.integers(0, 256, (4, MLEN), dtype=np.uint8)
        # first attempt singular under key 0 (tests/golden/rejection_msgs.json)
        g = json.load(open(os.path.join(GOLDEN, f"ref_mayo{s}.json")))["rejection"]
        msgs[0] = np.frombuffer(hashlib.shake_256(f"reject-search/{s}/{g['indices'][0]}".encode())
                                .digest(MLEN), np.uint8)
        n_retry += 1
        sig_want = np.stack([np.frombuffer(O.sign(s, esk[i % 2].tobytes(), msgs[i].tobytes())[0], np.uint8)
                             for i in range(4)])
        vsig = sig_want.copy()
        vsig[1, 3] ^= 0x20
        vsig[3, z.sig_bytes - 1] ^= 0x01
        ops = Q.SetOperands(kp_seed=_dev(seeds.reshape(-1)), kp_pk=kp_pk,
                            sg_esk=_dev(esk.reshape(-1)), sg_nkeys=2, sg_msg=_dev(msgs.reshape(-1)), sg_mlen=MLEN,
                            sg_sig=torch.zeros(4 * z.sig_bytes, dtype=torch.uint8, device="cuda"),
                            vf_epk=_dev(epk.reshape(-1)), vf_nkeys=2, vf_msg=_dev(msgs.reshape(-1)), vf_mlen=MLEN,
                            vf_sig=_dev(vsig.reshape(-1)),
                            vf_res=torch.full((4,), 0xEE, dtype=torch.uint8, device="cuda"))
        operands[s] = ops
        expect[s] = dict(pk=O.keypair_from_seed_batch(s, seeds), sig=sig_want, res=[0, 1, 0, 1])
        entries += [(Q.OP_KEYPAIR, s, i) for i in range(3)] + [(Q.OP_SIGN, s, i) for i in range(4)] + \
                   [(Q.OP_VERIFY, s, i) for i in range(4)]
    order = rng.permutation(len(entries))
    return operands, expect, [entries[i] for i in order], n_retry


def check(operands, expect):
    for s in SETS:
        z = Mayo(s).sizes
        ops = operands[s]
        assert (ops.kp_pk.cpu().numpy().reshape(3, z.pk_bytes) == expect[s]["pk"]).all(), s
        assert (ops.sg_sig.cpu().numpy().reshape(4, z.sig_bytes) == expect[s]["sig"]).all(), s
        assert ops.vf_res.cpu().numpy().tolist() == expect[s]["res"], s


def test_queue_mixed_sets_and_ops(cuda):
    import torch
    rng = np.random.default_rng(2024)
    operands, expect, entries, n_retry = build_case(rng)
    q = Q.Queue(capacity=len(entries) + 64, shape=Q.Shape(sms=2))
    for s, ops in operands.items():
        q.set_operands(s, ops)
    q.load(Q.items_array(entries))
    q.run()
    torch.cuda.synchronize()
    st = q.stats()
    assert st["error"] == Q.QUEUE_OK
    assert st["requeued_signs"] == n_retry
    assert st["finished"] == st["published"] == len(entries) + n_retry
    for (s, op), p in st["per_bucket"].items():
        assert p["published"] == 3 + (op != Q.OP_KEYPAIR) + (op == Q.OP_SIGN), (s, op)
    check(operands, expect)


def test_queue_graph_replay(cuda):
    import torch
    rng = np.random.default_rng(7)
    operands, expect, entries, n_retry = build_case(rng)
    q = Q.Queue(capacity=len(entries) + 64)  # default: every SM, the most CTAs per SM
    for s, ops in operands.items():
        q.set_operands(s, ops)
    q.load(Q.items_array(entries))
    q.capture()
    for _ in range(2):
        for ops in operands.values():
            ops.kp_pk.zero_()
            ops.sg_sig.zero_()
            ops.vf_res.fill_(0xEE)
        q.replay()
        torch.cuda.synchronize()
        assert q.stats()["error"] == Q.QUEUE_OK
        check(operands, expect)


def test_queue_per_instance_keys_and_messages(cuda):
    """sg_key / vf_key pick a key per instance; sg_msg_off / sg_msg_len give ragged messages."""
    import torch
    rng = np.random.default_rng(11)
    s = 3
    z = Mayo(s).sizes
    seeds = [rng.integers(0, 256, z.sk_bytes, dtype=np.uint8).tobytes() for _ in range(3)]
    esk = np.stack([np.frombuffer(O.expandsk(s, k), np.uint8) for k in seeds])
    epk = np.stack([np.frombuffer(O.expandpk(s, O.keypair_from_seed(s, k)), np.uint8) for k in seeds])
    lens = [0, 1, 135, 136, 137, 500, 7]
    msgs = [rng.integers(0, 256, n, dtype=np.uint8).tobytes() for n in lens]
    off = np.cumsum([0] + lens[:-1]).astype(np.int64)
    blob = np.frombuffer(b"".join(msgs) + b"\0", np.uint8)
    keys = rng.integers(0, 3, len(lens)).astype(np.uint32)
    want = [O.sign(s, esk[keys[i]].tobytes(), msgs[i])[0] for i in range(len(lens))]
    vsig = np.stack([np.frombuffer(w, np.uint8) for w in want])
    vkeys = keys.copy()
    vkeys[2] = (vkeys[2] + 1) % 3  # wrong key: rejected
    d_msg, d_off = _dev(blob), _dev(off)
    d_len = _dev(np.array(lens, np.uint32))
    ops = Q.SetOperands(sg_esk=_dev(esk.reshape(-1)), sg_nkeys=3, sg_key=_dev(keys), sg_msg=d_msg, sg_msg_off=d_off,
                        sg_msg_len=d_len, sg_sig=torch.zeros(len(lens) * z.sig_bytes, dtype=torch.uint8, device="cuda"),
                        vf_epk=_dev(epk.reshape(-1)), vf_nkeys=3, vf_key=_dev(vkeys), vf_msg=d_msg, vf_msg_off=d_off,
                        vf_msg_len=d_len, vf_sig=_dev(vsig.reshape(-1)),
                        vf_res=torch.full((len(lens),), 0xEE, dtype=torch.uint8, device="cuda"))
    q = Q.Queue(capacity=64, shape=Q.Shape(sms=4))
    q.set_operands(s, ops)
    q.load(Q.items_array([(Q.OP_SIGN, s, i) for i in range(len(lens))] +
                         [(Q.OP_VERIFY, s, i) for i in range(len(lens))]))
    q.run()
    torch.cuda.synchronize()
    assert q.stats()["error"] == Q.QUEUE_OK
    got = ops.sg_sig.cpu().numpy().reshape(len(lens), z.sig_bytes)
    for i in range(len(lens)):
        assert got[i].tobytes() == want[i], i
    assert ops.vf_res.cpu().numpy().tolist() == [1 if i == 2 else 0 for i in range(len(lens))]


def test_queue_operand_errors_skip_items(cuda):
    """An instance beyond its op's count, a key index beyond the key table and an item of a set
    without operands are skipped with QUEUE_ERR_OPERAND; the other items still finish."""
    import torch
    rng = np.random.default_rng(5)
    s = 1
    z = Mayo(s).sizes
    seeds = rng.integers(0, 256, (2, z.sk_bytes), dtype=np.uint8)
    key = rng.integers(0, 256, z.sk_bytes, dtype=np.uint8).tobytes()
    esk = np.frombuffer(O.expandsk(s, key), np.uint8)
    msgs = rng.integers(0, 256, (2, 16), dtype=np.uint8)
    kidx = np.array([0, 4], np.uint32)  # instance 1 names key 4 of a 1-key table
    ops = Q.SetOperands(kp_seed=_dev(seeds.reshape(-1)),
                        kp_pk=torch.zeros(2 * z.pk_bytes, dtype=torch.uint8, device="cuda"),
                        sg_esk=_dev(esk), sg_nkeys=1, sg_key=_dev(kidx), sg_msg=_dev(msgs.reshape(-1)), sg_mlen=16,
                        sg_sig=torch.zeros(2 * z.sig_bytes, dtype=torch.uint8, device="cuda"))
    q = Q.Queue(capacity=32, shape=Q.Shape(sms=2))
    q.set_operands(s, ops)
    q.load(Q.items_array([(Q.OP_KEYPAIR, s, 0), (Q.OP_KEYPAIR, s, 1), (Q.OP_KEYPAIR, s, 2),
                          (Q.OP_SIGN, s, 0), (Q.OP_SIGN, s, 1), (Q.OP_VERIFY, s, 0), (Q.OP_SIGN, 5, 0)]))
    q.run()
    torch.cuda.synchronize()
    st = q.stats()
    pb = st["per_bucket"]
    assert pb[(1, Q.OP_KEYPAIR)]["error"] == Q.QUEUE_ERR_OPERAND  # instance 2 of 2 seeds
    assert pb[(1, Q.OP_KEYPAIR)]["finished"] == pb[(1, Q.OP_KEYPAIR)]["published"] == 3
    assert pb[(1, Q.OP_SIGN)]["error"] == Q.QUEUE_ERR_OPERAND  # key 4 of a 1-key table
    assert pb[(1, Q.OP_SIGN)]["finished"] == 2
    # no verify operands for MAYO_1 and none at all for MAYO_5: no kernel, the items are dropped
    assert pb[(1, Q.OP_VERIFY)]["error"] == Q.QUEUE_ERR_OPERAND and pb[(1, Q.OP_VERIFY)]["taken"] == 1
    assert pb[(5, Q.OP_SIGN)]["error"] == Q.QUEUE_ERR_OPERAND and pb[(5, Q.OP_SIGN)]["taken"] == 1
    pk = ops.kp_pk.cpu().numpy().reshape(2, z.pk_bytes)
    assert (pk == O.keypair_from_seed_batch(s, seeds)).all()
    sig = ops.sg_sig.cpu().numpy().reshape(2, z.sig_bytes)
    assert sig[0].tobytes() == O.sign(s, esk.tobytes(), msgs[0].tobytes())[0]
    assert not sig[1].any()  # skipped


def test_queue_graph_device_count(cuda):
    """One captured graph replayed with different item counts written on the device."""
    import torch
    rng = np.random.default_rng(3)
    s = 2
    z = Mayo(s).sizes
    key = rng.integers(0, 256, z.sk_bytes, dtype=np.uint8).tobytes()
    esk = np.frombuffer(O.expandsk(s, key), np.uint8)
    n = 40
    msgs = rng.integers(0, 256, (n, 24), dtype=np.uint8)
    want = np.stack([np.frombuffer(O.sign(s, esk.tobytes(), m.tobytes())[0], np.uint8) for m in msgs])
    ops = Q.SetOperands(sg_esk=_dev(esk), sg_nkeys=1, sg_msg=_dev(msgs.reshape(-1)), sg_mlen=24,
                        sg_sig=torch.zeros(n * z.sig_bytes, dtype=torch.uint8, device="cuda"))
    q = Q.Queue(capacity=64)
    q.set_operands(s, ops)
    q.load(Q.items_array([(Q.OP_SIGN, s, i) for i in range(n)]))
    q.capture(device_count=True)
    for lo, hi in ((0, 5), (5, 6), (6, 40)):
        q.load(Q.items_array([(Q.OP_SIGN, s, i) for i in range(lo, hi)]))
        q.replay()
        torch.cuda.synchronize()
        st = q.stats()
        assert st["error"] == Q.QUEUE_OK and st["finished"] == hi - lo
    assert (ops.sg_sig.cpu().numpy().reshape(n, z.sig_bytes) == want).all()
