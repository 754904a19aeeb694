"""The drop-in header include/api.cuh (the reference's include/api.cuh:9-47 entry points over
libmayo_b200.so).

CPU: a C++ caller written against the reference's API (tests/dropin_driver.cu) compiles and links
against api.cuh + libmayo_b200.so, and so does the reference's own, unmodified benchmark driver
(tests/bench_stream.cu of the reference, where its sources are present: MAYO_REFERENCE, default
/root/reference).
GPU: that caller runs keypair -> signWithesk -> verifyWithepk through api.cuh, and its keys,
signatures and verify bytes equal the oracle's."""
import os
import subprocess

import numpy as np
import pytest

from cumayo_b200 import Mayo
from cumayo_b200.api import LIB_PATH
from cumayo_b200.build import ARCH, nvcc
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFERENCE = os.environ.get("MAYO_REFERENCE", "/root/reference")
DRIVER = os.path.join(ROOT, "tests", "dropin_driver.cu")


def _build(src, out, s, extra_inc=()):
    if not os.path.exists(LIB_PATH):
        pytest.skip("libmayo_b200.so not built")
    try:
        cc = nvcc()
    except RuntimeError:
        pytest.skip("nvcc not available")
    cmd = [cc] + ARCH + ["-O2", "-std=c++17", f"-DMAYO_VERSION={s}", "-I" + os.path.join(ROOT, "include")]
    cmd += ["-I" + d for d in extra_inc]
    cmd += ["-o", str(out), src, "-L" + os.path.dirname(LIB_PATH), "-lmayo_b200",
            "-Xlinker", "-rpath=" + os.path.dirname(LIB_PATH)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return out


def test_dropin_driver_builds(tmp_path):
    for s in (1, 5):
        _build(DRIVER, tmp_path / f"dropin_{s}", s)


@pytest.mark.skipif(not os.path.exists(os.path.join(REFERENCE, "tests", "bench_stream.cu")),
                    reason="the reference's sources are not present")
def test_reference_bench_stream_builds_against_dropin(tmp_path):
    """The reference's own benchmark driver, unmodified, against api.cuh (its other includes --
    params.h, code.h, time.cuh, aes128_ctr.cuh -- come from the reference's include directory)."""
    for s in (2, 3):
        _build(os.path.join(REFERENCE, "tests", "bench_stream.cu"), tmp_path / f"bench_stream_{s}", s,
               extra_inc=(os.path.join(REFERENCE, "include"),))


@pytest.mark.gpu
@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_dropin_driver_matches_oracle(cuda, tmp_path, s):
    batch, mlen = 8, 32
    exe = _build(DRIVER, tmp_path / f"dropin_{s}", s)
    out = tmp_path / "out.bin"
    r = subprocess.run([str(exe), str(out), str(batch), str(mlen)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    z = Mayo(s).sizes
    raw = np.fromfile(out, np.uint8)
    o = 0
    parts = {}
    for name, n in (("sk", z.sk_bytes), ("pk", z.pk_bytes), ("sig", z.sig_bytes), ("res", 2)):
        parts[name] = raw[o:o + batch * n].reshape(batch, n) if name != "res" else raw[o:o + 2 * batch]
        o += batch * n
    assert o == raw.size
    osk, opk = O.keypair_batch(s, 0, batch)
    assert (parts["sk"] == osk).all() and (parts["pk"] == opk).all()
    msgs = [bytes(((i * mlen + j) * 131 + 7) & 0xFF for j in range(mlen)) for i in range(batch)]
    osig, _ = O.sign_batch(s, O.expandsk_batch(s, osk), msgs)
    assert (parts["sig"] == osig).all()
    res = parts["res"]
    assert res[:batch].tolist() == [0] * batch
    assert res[batch:].tolist() == [i % 2 for i in range(batch)]
