"""Serving loop host logic on the CPU: the key table's LRU eviction and pinning, batch packing
into the staging layout the queue reads, Poisson arrivals, latency statistics."""
import numpy as np
import pytest

from cumayo_b200 import queue as Q
from cumayo_b200 import serving as SV
from cumayo_b200.api import MayoError, sizes


def test_slot_table_hits_misses_and_lru_eviction():
    t = SV.SlotTable(capacity=3, n_keys=10)
    slots, miss, new, su = t.acquire(np.array([4, 4, 7]))
    assert sorted(miss.tolist()) == [4, 7] and slots[0] == slots[1] != slots[2]
    t.release(su)
    slots, miss, _, su = t.acquire(np.array([7, 1]))
    assert miss.tolist() == [1]
    t.release(su)
    # table full (4, 7, 1); key 4 is least recently used -> evicted for key 9
    slots, miss, new, su = t.acquire(np.array([9]))
    assert miss.tolist() == [9] and t.slot_of[4] == -1 and t.slot_of[9] == new[0]
    assert t.evictions == 1
    t.release(su)


def test_slot_table_pins_protect_in_flight_keys():
    t = SV.SlotTable(capacity=2, n_keys=5)
    _, _, _, su_a = t.acquire(np.array([0, 1]))  # batch A in flight holds both slots
    with pytest.raises(SV.CacheFull):
        t.acquire(np.array([2]))
    assert t.slot_of[0] >= 0 and t.slot_of[1] >= 0
    t.release(su_a)
    slots, miss, _, su = t.acquire(np.array([2, 1]))  # 1 stays (used by this batch), 0 goes
    assert miss.tolist() == [2] and t.slot_of[0] == -1 and t.slot_of[1] >= 0
    with pytest.raises(MayoError):
        t.acquire(np.array([5]))  # unknown key id


def test_slot_table_can_load_matches_acquire():
    rng = np.random.default_rng(4)
    t = SV.SlotTable(capacity=4, n_keys=12)
    held = []
    for _ in range(200):
        keys = rng.integers(0, 12, rng.integers(1, 7))
        ok = t.can_load(keys)
        try:
            _, _, _, su = t.acquire(keys)
            assert ok
            held.append(su)
        except SV.CacheFull:
            assert not ok
        if held and (len(held) > 2 or rng.random() < 0.5):
            t.release(held.pop(0))
    assert (t.pins >= 0).all()


def test_capacity_for_budget():
    n = {1: 10, 5: 4}
    assert SV.capacity_for_budget(1 << 40, n) == n
    cap = SV.capacity_for_budget(4 * (sizes(1).esk_bytes + sizes(1).epk_bytes), n)
    assert 1 <= cap[1] < 10 and 1 <= cap[5] < 4


def _requests(rng, n, max_msg):
    op = np.where(rng.random(n) < 0.7, Q.OP_VERIFY, Q.OP_SIGN).astype(np.uint8)
    set_id = rng.choice([1, 2, 3, 5], n).astype(np.uint8)
    key = rng.integers(0, 4, n)
    mlen = rng.integers(0, max_msg + 1, n).astype(np.uint32)
    msg = rng.integers(0, 256, (n, max_msg), dtype=np.uint8)
    sig = rng.integers(0, 256, (n, SV.MAX_SIG), dtype=np.uint8)
    out = np.zeros((n, SV.MAX_SIG), np.uint8)
    reqs = SV.requests_from_rows(op, set_id, key, mlen, msg, sig, out)
    reqs["key_slot"] = key * 10 + set_id
    return reqs, msg, sig, out


def test_pack_layout_round_trip():
    """mayo_b200_serve_pack / _unpack (host code) against a restatement of the layout."""
    rng = np.random.default_rng(1)
    max_msg, n = 64, 300
    reqs, msg, sig, out = _requests(rng, n, max_msg)
    buf = np.zeros(SV.in_bytes(n, max_msg), np.uint8)
    lay = SV.pack(reqs, max_msg, buf, SV.out_bytes(n))
    assert lay.n == n and lay.in_bytes <= buf.size
    items = buf[: 4 * n].view(np.uint32)
    groups = [g for g in lay.group if g.count]
    assert len(groups) == 8
    seen = set()
    for gi, g in enumerate(lay.group):
        if not g.count:
            continue
        assert (g.set, g.op) == ([1, 2, 3, 5][gi // 2], Q.OP_VERIFY if gi & 1 else Q.OP_SIGN)
        rows = np.flatnonzero((reqs["set"] == g.set) & (reqs["op"] == g.op))
        c = rows.size
        assert c == g.count
        assert all(off % 16 == 0 for off in (g.key_off, g.len_off, g.msg_off, g.sig_off, g.out_off))
        for rank, r in enumerate(rows):
            it = int(items[r])
            assert (it >> 30, (it >> 28) & 3, it & 0xFFFFF) == (g.op, Q.SET_INDEX[g.set], rank)
            seen.add(int(r))
            ln = int(reqs["mlen"][r])
            assert (buf[g.msg_off + rank * max_msg: g.msg_off + rank * max_msg + ln] == msg[r, :ln]).all()
        assert (buf[g.key_off: g.key_off + 4 * c].view(np.uint32) == reqs["key_slot"][rows]).all()
        assert (buf[g.len_off: g.len_off + 4 * c].view(np.uint32) == reqs["mlen"][rows]).all()
        if g.op == Q.OP_VERIFY:
            sb = sizes(g.set).sig_bytes
            assert (buf[g.sig_off: g.sig_off + c * sb].reshape(c, sb) == sig[rows, :sb]).all()
    assert seen == set(range(n))
    # outputs: fill each group's region with its row ids, unpack, compare
    stage_out = np.zeros(SV.out_bytes(n), np.uint8)
    for g in groups:
        rows = np.flatnonzero((reqs["set"] == g.set) & (reqs["op"] == g.op))
        c = rows.size
        if g.op == Q.OP_SIGN:
            sb = sizes(g.set).sig_bytes
            stage_out[g.out_off: g.out_off + c * sb] = np.repeat((rows % 251).astype(np.uint8), sb)
        else:
            stage_out[g.out_off: g.out_off + c] = (rows % 2).astype(np.uint8)
    SV.unpack(reqs, lay, stage_out)
    for r in range(n):
        if reqs["op"][r] == Q.OP_SIGN:
            sb = sizes(int(reqs["set"][r])).sig_bytes
            assert (out[r, :sb] == r % 251).all() and not out[r, sb:].any()
        else:
            assert out[r, 0] == r % 2 and not out[r, 1:].any()


def test_pack_rejects_malformed_requests():
    rng = np.random.default_rng(2)
    for field, value in (("mlen", 33), ("op", 0), ("set", 4), ("out", 0)):
        reqs, *_ = _requests(rng, 4, 32)
        reqs[field][1] = value
        with pytest.raises(MayoError):
            SV.pack(reqs, 32, np.zeros(SV.in_bytes(4, 32), np.uint8), SV.out_bytes(4))
    reqs, *_ = _requests(rng, 64, 32)
    with pytest.raises(MayoError):  # staging too small
        SV.pack(reqs, 32, np.zeros(1024, np.uint8), SV.out_bytes(64))


def test_poisson_arrivals():
    a = SV.poisson_arrivals(1e5, 200000, b"k" * 32)
    assert (np.diff(a) > 0).all()
    assert abs(a[-1] / a.size - 1e-5) < 1e-7  # mean gap within 1 % of 1/rate
    assert (SV.poisson_arrivals(1e5, 10, b"k" * 32) == a[:10]).all()
    gaps = np.diff(a) * 1e5
    assert abs(np.mean(gaps > 1.0) - np.exp(-1.0)) < 0.01  # exponential tail


def test_latency_stats():
    st = SV.latency_stats(np.array([0.001, 0.002, np.nan, 0.003]))
    assert st["n"] == 3 and abs(st["p50_ms"] - 2.0) < 1e-9 and st["max_ms"] == 3.0
