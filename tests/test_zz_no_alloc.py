"""mayo_b200_sign_many_noalloc: signing for callers that cannot allocate device memory.

Such a caller (a service with a device-memory budget fixed at start-up, or a host program
that does not let a plug-in library call cudaMalloc) cannot hand mayo_b200_sign_many its
per-instance workspace; the no-alloc entry point keeps that workspace in a fixed array inside
the library.  This test calls it through the C-ABI twice in a row and checks each result
against mayo_b200_sign_many on the same inputs (byte-exact, the tolerance of every signature
test here), and checks that a batch above the fixed limit is refused.  The file name makes
pytest collect it last.
"""
import numpy as np
import pytest

from cumayo_b200 import Mayo, MayoError

pytestmark = pytest.mark.gpu


def _inputs(m, rng, batch):
    import torch
    z = m.sizes
    lens = rng.integers(0, 200, batch).astype(np.uint32)
    offs = np.zeros(batch, np.uint64)
    offs[1:] = np.cumsum(lens[:-1], dtype=np.uint64)
    body = rng.integers(0, 256, int(lens.sum()) + 1, dtype=np.uint8)
    d = lambda a: torch.from_numpy(a).cuda()  # noqa: E731
    return d(body), d(offs.view(np.int64)), d(lens.view(np.int32))


@pytest.mark.parametrize("s", [2, 5])
def test_noalloc_matches_sign_many_twice(s, cuda):
    import torch
    from oracle import oracle as O
    m = Mayo(s)
    z = m.sizes
    rng = np.random.default_rng(4242 + s)
    seed = rng.integers(0, 256, z.sk_bytes, dtype=np.uint8).tobytes()
    esk = torch.from_numpy(np.frombuffer(O.expandsk(s, seed), np.uint8).copy()).cuda()
    batch = min(64, m.sign_noalloc_max_batch())
    ws = torch.zeros(batch * m.sign_ws_bytes(), dtype=torch.uint8, device="cuda")
    for _ in range(2):  # two calls in a row: the shared array keeps the previous call's bytes
        msgs, offs, lens = _inputs(m, rng, batch)
        want = torch.zeros(batch * z.sig_bytes, dtype=torch.uint8, device="cuda")
        m.sign_many(esk, msgs, want, ws, batch, msg_off=offs, msg_len=lens)
        got = torch.full((batch * z.sig_bytes,), 0xAB, dtype=torch.uint8, device="cuda")
        m.sign_many_noalloc(esk, msgs, got, batch, msg_off=offs, msg_len=lens)
        torch.cuda.synchronize()
        assert torch.equal(got, want)


def test_noalloc_full_array_matches_sign_many_and_oracle(cuda):
    """MAYO_5 at exactly mayo_b200_sign_noalloc_max_batch instances: the last instance's
    workspace ends at the end of the fixed array."""
    import torch
    from oracle import oracle as O
    s = 5
    m = Mayo(s)
    z = m.sizes
    batch = m.sign_noalloc_max_batch()
    assert batch * m.sign_ws_bytes() <= 4 << 20 < (batch + 1) * m.sign_ws_bytes()
    rng = np.random.default_rng(5151)
    seed = rng.integers(0, 256, z.sk_bytes, dtype=np.uint8).tobytes()
    esk_h = np.frombuffer(O.expandsk(s, seed), np.uint8)
    esk = torch.from_numpy(esk_h.copy()).cuda()
    msgs, offs, lens = _inputs(m, rng, batch)
    got = torch.full((batch * z.sig_bytes,), 0xAB, dtype=torch.uint8, device="cuda")
    m.sign_many_noalloc(esk, msgs, got, batch, msg_off=offs, msg_len=lens)
    ws = torch.zeros(batch * m.sign_ws_bytes(), dtype=torch.uint8, device="cuda")
    want = torch.zeros_like(got)
    m.sign_many(esk, msgs, want, ws, batch, msg_off=offs, msg_len=lens)
    torch.cuda.synchronize()
    assert torch.equal(got, want)
    body, o_h, l_h = msgs.cpu().numpy(), offs.cpu().numpy().view(np.uint64), lens.cpu().numpy().view(np.uint32)
    ml = [body[int(a):int(a) + int(n)].tobytes() for a, n in zip(o_h, l_h)]
    osig, _ = O.sign_batch(s, esk_h[None, :], ml, shared_key=True)
    assert np.array_equal(got.cpu().numpy().reshape(batch, z.sig_bytes), osig)


def test_noalloc_rejects_batch_above_limit(cuda):
    import torch
    m = Mayo(3)
    limit = m.sign_noalloc_max_batch()
    assert limit > 0
    dummy = torch.zeros(16, dtype=torch.uint8, device="cuda")
    with pytest.raises(MayoError, match="exceeds the fixed workspace"):
        m.sign_many_noalloc(dummy, dummy, dummy, limit + 1, mlen=0)
