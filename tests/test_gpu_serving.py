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


class _Batch:
    """Request records for rows lo..hi-1 of the case, with their output rows."""

    def __init__(self, req, lo, hi):
        sl = slice(lo, hi)
        self.out = np.zeros((hi - lo, SV.MAX_SIG), np.uint8)
        self.msg = np.ascontiguousarray(req.msg[sl])
        self.sig = np.ascontiguousarray(req.sig[sl])
        self.reqs = SV.requests_from_rows(req.op[sl], req.set_id[sl], req.key[sl], req.mlen[sl], self.msg, self.sig,
                                          self.out)


def _check(req, lo, hi, out, want_sig, want_res):
    for j, i in enumerate(range(lo, hi)):
        if req.op[i] == Q.OP_SIGN:
            sb = sizes(int(req.set_id[i])).sig_bytes
            assert out[j, :sb].tobytes() == want_sig[i], i
        else:
            assert out[j, 0] == want_res[i], i


def test_serving_mix_and_alone_match_oracle(cuda):
    seeds, req, want_sig, want_res = _case()
    cache = SV.KeyCache(seeds, {s: 3 for s in SETS})  # 3 slots for 5 keys per set
    server = SV.Server(cache, max_batch=32, inflight=2, max_msg=MAX_MSG)
    arrivals = SV.poisson_arrivals(4e3, len(req), b"serving-test".ljust(32, b"\0"))
    done = []

    def fetch(lo, hi):
        b = _Batch(req, lo, hi)
        return b.reqs, b

    def on_done(lo, hi, b):  # the batch may be a prefix of what fetch returned
        done.append((lo, hi, b))

    lat, wall, sizes_ = SV.run_open_loop(server, arrivals, fetch, on_done)
    assert np.isfinite(lat).all() and (lat >= 0).all()
    server.check_queue()
    assert sum(hi - lo for lo, hi, _ in done) == len(req)
    for lo, hi, b in done:
        _check(req, lo, hi, b.out, want_sig, want_res)
    assert sum(t.evictions for t in cache.tables.values()) > 0  # the table really was too small
    # the same requests one per batch
    for i in range(0, len(req), 7):
        b = _Batch(req, i, i + 1)
        server.launch(b.reqs, tag=(i, i + 1), keep=b)
        server.drain()
        _check(req, i, i + 1, b.out, want_sig, want_res)
    server.check_queue()
