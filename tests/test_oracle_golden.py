"""The CPU oracle against the reference's own outputs (golden vectors made by
tests/golden/gen_golden.py from the reference's sm_100a build) and against
independent implementations of its primitives (hashlib SHAKE, `cryptography`
AES-128-CTR)."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SETS = [1, 2, 3, 5]


def golden(s):
    with open(os.path.join(GOLDEN, f"ref_mayo{s}.json")) as f:
        return json.load(f)


def message(s, i, mlen):
    return hashlib.shake_256(f"golden/{s}/{i}/{mlen}".encode()).digest(mlen)


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("n", [0, 1, 7, 8, 135, 136, 137, 167, 168, 169, 500, 1024])
def test_shake_matches_hashlib(n):
    data = hashlib.sha256(str(n).encode()).digest() * (n // 32 + 1)
    data = data[:n]
    assert O.shake256(data, 700) == hashlib.shake_256(data).digest(700)
    assert O.shake128(data, 700) == hashlib.shake_128(data).digest(700)


@pytest.mark.parametrize("n", [1, 15, 16, 17, 1000, 144495 % 4096])
def test_aes_ctr_matches_cryptography(n):
    cg = pytest.importorskip("cryptography.hazmat.primitives.ciphers")
    key = hashlib.sha256(b"k%d" % n).digest()[:16]
    enc = cg.Cipher(cg.algorithms.AES(key), cg.modes.CTR(b"\0" * 16)).encryptor()
    assert O.aes128_ctr(key, n) == enc.update(b"\0" * n)


def test_gf16_field():
    # x^4 + x + 1: 2 * 8 = x * x^3 = x + 1 = 3 (the reference's table row b=2, a=8)
    assert O.gf16_mul(2, 8) == 3
    for a in range(1, 16):
        assert O.gf16_mul(a, O.gf16_inv(a)) == 1
        for b in range(16):
            assert O.gf16_mul(a, b) == O.gf16_mul(b, a)


@pytest.mark.parametrize("s", SETS)
def test_params_match_reference_sizes(s):
    g = golden(s)["sizes"]
    P = O.params(s)
    assert (P.sk_bytes, P.pk_bytes, P.sig_bytes, P.esk_bytes, P.epk_bytes) == (
        g["sk"], g["pk"], g["sig"], g["esk"], g["epk"])
    assert P.v == P.m  # the reference relies on v == m in every set


@pytest.mark.parametrize("s", SETS)
def test_keypair_golden(s):
    for ri, kp in golden(s)["keypair"].items():
        sk, pk = O.keypair_batch(s, int(ri), kp["batch"])
        assert sha(sk) == kp["sk_sha256"]
        assert sha(pk) == kp["pk_sha256"]
        for i in range(len(kp["sk"])):
            assert sk[i].tobytes().hex() == kp["sk"][i]
            assert pk[i].tobytes().hex() == kp["pk"][i]


@pytest.mark.parametrize("s", SETS)
def test_expand_golden(s):
    g = golden(s)
    sk, pk = O.keypair_batch(s, 0, 8)
    assert [sha(x) for x in O.expandsk_batch(s, sk)] == g["expandsk_sha256"]
    assert [sha(x) for x in O.expandpk_batch(s, pk)] == g["expandpk_sha256"]


@pytest.mark.parametrize("s", SETS)
def test_sign_verify_golden(s):
    g = golden(s)
    sk, pk = O.keypair_batch(s, 0, 8)
    esk = O.expandsk_batch(s, sk)
    epk = O.expandpk_batch(s, pk)
    for ent in g["sign"]:
        msgs = [message(s, i, ent["mlen"]) for i in range(8)]
        sig, att = O.sign_batch(s, esk, msgs)
        assert [x.tobytes().hex() for x in sig] == ent["sig_with_esk"], ent["mlen"]
        assert list(O.verify_batch(s, epk, msgs, sig)) == ent["verify_good"] == [0] * 8
        bad = np.stack([np.frombuffer(bytes.fromhex(h), np.uint8) for h in ent["bad_sig"]])
        assert list(O.verify_batch(s, epk, msgs, bad)) == ent["verify_bad"]


@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_rejection_path_golden(s):
    rej = golden(s)["rejection"]
    sk, _ = O.keypair(s, 0, 0)
    esk = O.expandsk(s, sk)
    for idx, h, a in zip(rej["indices"], rej["sig"], rej["attempts_oracle"]):
        m = hashlib.shake_256(f"reject-search/{s}/{idx}".encode()).digest(32)
        sig, att = O.sign(s, esk, m)
        assert att == a >= 2
        assert sig.hex() == h
    assert rej["verify"] == [0] * len(rej["indices"])


def test_force_reject_hook_emits_last_attempt():
    """All 255 attempts rejected: the reference still writes the last attempt's
    (V, x = r) signature; the oracle's test hook reproduces that branch."""
    s = 2
    sk, pk = O.keypair(s, 0, 0)
    esk, epk = O.expandsk(s, sk), O.expandpk(s, pk)
    sig, att = O.sign(s, esk, b"m", force_reject=255)
    assert att == 0
    assert O.verify(s, epk, b"m", sig) == 1
    sig2, att2 = O.sign(s, esk, b"m", force_reject=1)
    assert att2 == 2 and O.verify(s, epk, b"m", sig2) == 0
