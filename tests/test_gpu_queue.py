"""Persistent work queue on the GPU: keypair / sign / verify items of all four parameter sets in
one launch, shuffled together, checked byte for byte against the oracle and the reference's
golden retry cases (a singular first attempt is re-enqueued on the device); then the same run
captured in a CUDA graph and replayed."""
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
        if s != 2:  # first attempt singular under key 0 (tests/golden/rejection_msgs.json)
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
    q = Q.Queue(capacity=len(entries) + 64, ctas=8)
    for s, ops in operands.items():
        q.set_operands(s, ops)
    q.load(Q.items_array(entries))
    q.run()
    torch.cuda.synchronize()
    st = q.stats()
    assert st["error"] == Q.QUEUE_OK
    assert st["requeued_signs"] == n_retry
    assert st["finished"] == st["published"] == len(entries) + n_retry
    check(operands, expect)


def test_queue_graph_replay(cuda):
    import torch
    rng = np.random.default_rng(7)
    operands, expect, entries, n_retry = build_case(rng)
    q = Q.Queue(capacity=len(entries) + 64)  # default: every resident CTA slot of the device
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
