"""Find messages whose signature needs more than one attempt (CPU, oracle).

The reference retries up to 255 times when the linear system is singular
(src/sign.cu:244-470).  The per-attempt rejection rate is about 2.4e-4 for
MAYO_1/3/5, so the retry path is rare; this script searches seeded messages
under the counter keypair (rand_index=0, instance 0) for cases with attempts
>= 2 and records them in rejection_msgs.json.  gen_golden.py then has the
reference itself sign them, which pins the retry path.

Run once in a container with the oracle built:  python tests/golden/search_rejections.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def msg_for(set_id: int, i: int, mlen: int = 32) -> bytes:
    return hashlib.shake_256(f"reject-search/{set_id}/{i}".encode()).digest(mlen)


def main(sets=(1, 3, 5), want=2, chunk=2048, limit=200_000):
    out = {}
    for s in sets:
        sk, _pk = O.keypair(s, 0, 0)
        esk = O.expandsk(s, sk)
        found = []
        start = 0
        while len(found) < want and start < limit:
            msgs = [msg_for(s, i) for i in range(start, start + chunk)]
            sig, att = O.sign_batch(s, esk[None, :] if hasattr(esk, "shape") else
                                    __import__("numpy").frombuffer(esk, dtype="uint8")[None, :],
                                    msgs, shared_key=True)
            for j, a in enumerate(att):
                if a != 1:
                    found.append({"index": start + j, "attempts": int(a)})
            start += chunk
            print(f"MAYO_{s}: searched {start}, found {len(found)}", flush=True)
        out[str(s)] = {"rand_index": 0, "instance": 0, "mlen": 32, "messages": found[:want]}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "rejection_msgs.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
