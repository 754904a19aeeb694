"""Serving loop on the GPU: a Poisson stream of sign / verify requests over all four parameter
sets, keys loaded into a key table too small to hold them all (so keys are evicted and loaded
again while batches are in flight), every result checked against the oracle; then a sample of
the same requests served one per batch, which must give the same bytes as in the mix."""
import numpy as np
import pytest

from cumayo_b200 import queue as Q
from cumayo_b200 import serving as SV
from cumayo_b200.api import sizes
from oracle import oracle as O

pytestmark = pytest.mark.gpu
SETS = [1, 2, 3, 5]
MAX_MSG = 200


class _Case:
    def __init__(self, op, set_id, key, mlen, msg, sig):
        self.op, self.set_id, self.key, self.mlen, self.msg, self.sig = op, set_id, key, mlen, msg, sig

    def __len__(self):
        return int(self.op.shape[0])


def _case(seed=9, n=240, keys_per_set=5):
    rng = np.random.default_rng(seed)
    seeds = {s: rng.integers(0, 256, (keys_per_set, sizes(s).sk_bytes), dtype=np.uint8) for s in SETS}
    esk = {s: [O.expandsk(s, k.tobytes()) for k in seeds[s]] for s in SETS}
    epk = {s: [O.expandpk(s, O.keypair_from_seed(s, k.tobytes())) for k in seeds[s]] for s in SETS}
    op = np.where(rng.random(n) < 0.6, Q.OP_VERIFY, Q.OP_SIGN).astype(np.uint32)
    set_id = rng.choice(SETS, n).astype(np.int64)
    key = rng.integers(0, keys_per_set, n)
    mlen = rng.integers(0, MAX_MSG + 1, n).astype(np.uint32)
    msg = rng.integers(0, 256, (n, MAX_MSG), dtype=np.uint8)
    sig = np.zeros((n, SV.MAX_SIG), np.uint8)
    want_sig, want_res = {}, np.full(n, 0xFF, np.uint8)
    for i in range(n):
        s, k, m = int(set_id[i]), int(key[i]), msg[i, : mlen[i]].tobytes()
        good = O.sign(s, esk[s][k], m)[0]
        if op[i] == Q.OP_SIGN:
            want_sig[i] = good
        else:
            bad = i % 5 == 0
            sg = bytearray(good)
            if bad:
                sg[i % len(sg)] ^= 0x10
            sig[i, : len(sg)] = np.frombuffer(bytes(sg), np.uint8)
            want_res[i] = O.verify(s, epk[s][k], m, bytes(sg))
            assert want_res[i] == (1 if bad else 0)
    return seeds, _Case(op.astype(np.uint8), set_id.astype(np.uint8), key, mlen, msg, sig), want_sig, want_res


def _rows(req, lo, hi, out):
    """Request records for rows lo..hi-1 of the case, results into `out` (rows 0..hi-lo-1)."""
    sl = slice(lo, hi)
    msg = np.ascontiguousarray(req.msg[sl])
    sig = np.ascontiguousarray(req.sig[sl])
    return SV.requests_from_rows(req.op[sl], req.set_id[sl], req.key[sl], req.mlen[sl], msg, sig, out), (msg, sig)


def _check(req, lo, hi, out, want_sig, want_res):
    for j, i in enumerate(range(lo, hi)):
        if req.op[i] == Q.OP_SIGN:
            sb = sizes(int(req.set_id[i])).sig_bytes
            assert out[j, :sb].tobytes() == want_sig[i], i
        else:
            assert out[j, 0] == want_res[i], i


def test_serving_mix_and_alone_match_oracle(cuda):
    """The native server's open-loop run: admission, batching, key eviction and reload while
    batches are in flight; then single requests through submit / drain."""
    seeds, req, want_sig, want_res = _case()
    n = len(req)
    server = SV.Server(seeds, key_slots={s: 3 for s in SETS}, max_batch=32, inflight=2, max_msg=MAX_MSG)
    arrivals = SV.poisson_arrivals(4e3, n, b"serving-test".ljust(32, b"\0"))
    out = np.zeros((n, SV.MAX_SIG), np.uint8)
    reqs, keep = _rows(req, 0, n, out)
    lat, wall = server.run_open_loop(reqs, arrivals)
    assert np.isfinite(lat).all() and (lat >= 0).all() and wall > 0
    server.check_queue()
    _check(req, 0, n, out, want_sig, want_res)
    st = server.stats()
    assert st["requests_done"] == n and st["batches"] > 1 and st["max_batch_seen"] <= 32
    assert st["key_evictions"] > 0  # the tables really were too small
    # the same requests one per batch
    for i in range(0, n, 7):
        o1 = np.zeros((1, SV.MAX_SIG), np.uint8)
        r1, k1 = _rows(req, i, i + 1, o1)
        server.submit(r1, first_tag=i, keep=k1)
        assert server.drain().tolist() == [i]
        _check(req, i, i + 1, o1, want_sig, want_res)
    # several batches through submit / progress, tags reported once each
    out2 = np.zeros((n, SV.MAX_SIG), np.uint8)
    r2, k2 = _rows(req, 0, n, out2)
    server.submit(r2, first_tag=1000)
    tags = []
    while len(tags) < n:
        tags += server.progress().tolist()
    assert sorted(tags) == list(range(1000, 1000 + n))
    _check(req, 0, n, out2, want_sig, want_res)
    server.check_queue()
    server.close()


def test_serving_rejects_bad_requests(cuda):
    seeds, req, _, _ = _case(n=8)
    server = SV.Server(seeds, max_batch=8, inflight=1, max_msg=MAX_MSG)
    out = np.zeros((8, SV.MAX_SIG), np.uint8)
    reqs, keep = _rows(req, 0, 8, out)
    bad = reqs.copy()
    bad["key_id"][3] = 99  # 5 keys per set
    with pytest.raises(SV.MayoError):
        server.submit(bad)
    assert server.stats()["waiting"] == 0  # nothing taken
    server.close()
