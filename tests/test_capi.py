"""The C-ABI library on the CPU: it loads, exports every symbol include/mayo_b200.h
declares, reports sizes equal to the oracle's, and rejects bad arguments before touching
the GPU (no compute calls here)."""
import ctypes
import os
import re
import subprocess

import pytest

import cumayo_b200 as M
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mayo_b200.h")


def declared():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"MAYO_B200_API\s+[\w\s\*]+?\b(mayo_b200_\w+)\s*\(", src)))


def test_header_declares_reference_surface():
    names = declared()
    ref = ["keypair", "keypair_DtH", "expandsk_HtD", "expandsk", "expandsk_DtH", "expandpk_HtD", "expandpk",
           "expandpk_DtH", "sign_HtD", "sign", "sign_DtH", "signWithesk_HtD", "signWithesk", "signWithesk_DtH",
           "verify_HtD", "verify", "verify_DtH", "verifyWithepk_HtD", "verifyWithepk", "verifyWithepk_DtH"]
    for r in ref:  # the 20 entry points of the reference's include/api.cuh
        assert "mayo_b200_" + r in names


def test_library_exports_every_declared_symbol():
    lib = M.lib()
    for name in declared():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", M.api.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert exported == set(declared())


@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_sizes_match_oracle(s):
    z = M.sizes(s, 32)
    P = O.params(s)
    assert (z.n, z.m, z.o, z.k) == (P.n, P.m, P.o, P.k)
    assert (z.sk_bytes, z.pk_bytes, z.sig_bytes, z.esk_bytes, z.epk_bytes, z.p_bytes) == (
        P.sk_bytes, P.pk_bytes, P.sig_bytes, P.esk_bytes, P.epk_bytes, P.p_bytes)
    A = M.A128
    assert z.pitch_keypair == A(P.sk_bytes) + A(P.pk_bytes) + A(P.p_bytes)
    assert z.pitch_verify == A(P.epk_bytes) + A(32) + A(P.sig_bytes) + 1


def test_argument_errors_without_gpu():
    lib = M.lib()
    assert lib.mayo_b200_keypair(4, None, 0, 1, None, 0) == 1          # unknown set
    assert lib.mayo_b200_sign(1, None, 32, 1 << 20, 2, None) == 2       # null pool
    assert lib.mayo_b200_verify(5, 4096, 32, 100, 2, None) == 2         # pitch too small
    assert lib.mayo_b200_verifyWithepk(3, None, 32, 0, 0, None) == 0   # empty batch is a no-op
    assert lib.mayo_b200_get_sizes(9, 0, None) == 1
    assert M.lib().mayo_b200_abi_version() == 1
    with pytest.raises(M.MayoError):
        M.Mayo(4)


@pytest.mark.parametrize("s", [1, 2, 3, 5])
def test_shared_shape_defaults_and_range(s):
    """The shared-key launch shape is host state: defaults (CTA-pair product everywhere, four
    signatures per sign-tail CTA for MAYO_2, two for MAYO_1), a set shape read back, 0 = default,
    bad shapes rejected."""
    m = M.Mayo(s)
    default = {"hash_threads": 64, "tail_instances": {1: 2, 2: 4}.get(s, 1), "product_ctas": 2}
    try:
        m.set_shared_shape(0, 0, 0)
        assert m.shared_shape() == default
        m.set_shared_shape(128, 2, 1)
        assert m.shared_shape() == {"hash_threads": 128, "tail_instances": 2, "product_ctas": 1}
        for bad in ((48, 1, 1), (2048, 1, 1), (64, 3, 1), (64, 1, 3)):
            with pytest.raises(M.MayoError):
                m.set_shared_shape(*bad)
        assert m.shared_shape()["hash_threads"] == 128  # a rejected shape changes nothing
    finally:
        m.set_shared_shape(0, 0, 0)
    assert m.shared_shape() == default


def test_python_mirror_has_reference_names():
    ref = ["crypto_sign_keypair", "crypto_sign_keypair_DtH", "crypto_sign_expandsk_HtD", "crypto_sign_expandsk",
           "crypto_sign_expandsk_DtH", "crypto_sign_expandpk_HtD", "crypto_sign_expandpk",
           "crypto_sign_expandpk_DtH", "crypto_sign_sign_HtD", "crypto_sign_sign", "crypto_sign_sign_DtH",
           "crypto_sign_signWithesk_HtD", "crypto_sign_signWithesk", "crypto_sign_signWithesk_DtH",
           "crypto_sign_verify_HtD", "crypto_sign_verify", "crypto_sign_verify_DtH",
           "crypto_sign_verifyWithepk_HtD", "crypto_sign_verifyWithepk", "crypto_sign_verifyWithepk_DtH"]
    m = M.Mayo(1)
    for r in ref:
        assert callable(getattr(m, r))


def test_queue_structs_match_header(tmp_path):
    """The ctypes mirrors of mayo_b200_queue_ops / _shape have the C layout (offsets, size)."""
    from cumayo_b200 import queue as Q
    structs = {"mayo_b200_queue_ops": Q._QueueOps, "mayo_b200_queue_shape": Q._QueueShape}
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src, exe = tmp_path / "layout.c", tmp_path / "layout"
    src.write_text("\n".join(lines))
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(src)], check=True)
    got = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    for line in filter(None, got):
        cname, f, v = line.split()
        py = structs[cname]
        want = ctypes.sizeof(py) if f == "size" else getattr(py, f).offset
        assert int(v) == want, (cname, f)


def test_queue_item_encoding():
    from cumayo_b200 import queue as Q
    assert Q.item(Q.OP_VERIFY, 5, 0xABCDE) == (2 << 30) | (3 << 28) | 0xABCDE
    assert Q.item(Q.OP_KEYPAIR, 1, 1 << 20) == 0  # instance wraps at 20 bits, as the C helper
    arr = Q.items_array([(Q.OP_SIGN, 3, 7)])
    assert arr.dtype.name == "uint32" and int(arr[0]) == (1 << 30) | (2 << 28) | 7
