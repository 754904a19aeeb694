"""Find MAYO_2 messages whose first sign attempt is singular, on a GPU.

MAYO_2's per-attempt rejection rate is about 16^-5 (k*o - m = 4), too low for the CPU search of
search_rejections.py.  This script signs the same seeded candidates (shake_256 of
"reject-search/2/<index>", 32 bytes, under the counter keypair rand_index 0, instance 0) in large
batches with mayo_b200_sign_shared, whose workspace control word 1 counts the instances whose first
attempt was singular; a batch with a nonzero count is bisected down to single messages.  Each hit
is confirmed with the oracle (its attempt count) and added to rejection_msgs.json, after which
gen_golden.py has the reference itself sign it, which pins MAYO_2's retry path.

Run on a GPU box with the library and the oracle built:
    python tests/golden/search_rejections_gpu.py [want=2] [limit=33554432]
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cumayo_b200 import Mayo  # noqa: E402
from oracle import oracle as O  # noqa: E402

SET, MLEN = 2, 32


def messages(start: int, n: int) -> np.ndarray:
    return np.frombuffer(b"".join(hashlib.shake_256(f"reject-search/{SET}/{i}".encode()).digest(MLEN)
                                  for i in range(start, start + n)), np.uint8)


def main(want: int = 2, limit: int = 1 << 25, chunk: int = 1 << 18):
    import torch
    m = Mayo(SET)
    z = m.sizes
    sk, _ = O.keypair(SET, 0, 0)
    esk_h = O.expandsk(SET, sk)
    esk = torch.from_numpy(np.frombuffer(esk_h, np.uint8).copy()).cuda()
    ws = torch.zeros(m.sign_shared_ws_bytes(chunk), dtype=torch.uint8, device="cuda")
    sig = torch.zeros(chunk * z.sig_bytes, dtype=torch.uint8, device="cuda")

    def singular_count(d_msg, lo, n):
        m.sign_shared(esk, d_msg[lo * MLEN:], sig, ws, n, msg_stride=MLEN, mlen=MLEN)
        c = ws[:8].cpu().numpy().view(np.uint32)
        assert c[0] == 0, "tensor-core product gave up"
        return int(c[1])

    def bisect(d_msg, lo, n, out):
        if singular_count(d_msg, lo, n) == 0:
            return
        if n == 1:
            out.append(lo)
            return
        h = n // 2
        bisect(d_msg, lo, h, out)
        bisect(d_msg, lo + h, n - h, out)

    found = []
    start = 0
    while len(found) < want and start < limit:
        d_msg = torch.from_numpy(messages(start, chunk).copy()).cuda()
        hits = []
        bisect(d_msg, 0, chunk, hits)
        for h in hits:
            idx = start + h
            msg = hashlib.shake_256(f"reject-search/{SET}/{idx}".encode()).digest(MLEN)
            _, att = O.sign(SET, esk_h, msg)
            assert att >= 2, (idx, att)
            found.append({"index": idx, "attempts": int(att)})
        start += chunk
        print(f"MAYO_{SET}: searched {start}, found {len(found)}", flush=True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rejection_msgs.json")
    data = json.load(open(path))
    data[str(SET)] = {"rand_index": 0, "instance": 0, "mlen": MLEN, "messages": found[:want],
                      "searched": start, "search": "GPU, tests/golden/search_rejections_gpu.py"}
    with open(path, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", path, found[:want])


if __name__ == "__main__":
    main(*[int(a) for a in sys.argv[1:]])
