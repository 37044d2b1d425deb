"""Golden digests of the XMSS^MT / wide-hash mix workload (bench.MIX_SETS:
XMSSMT-SHA2_20/2_256, XMSSMT-SHA2_40/4_256, XMSS-SHA2_10_512 and
XMSS-SHAKE_10_256; 2,048 signatures each at consecutive indices over
messages log-uniform in 32 B..64 KB, from the seeded inputs of
bench.mix_all_draws).

    python tests/golden/make_mix_golden.py

Every key and signature is computed by the CPU oracle (oracle/xmss_oracle.c,
pinned to the reference's C path by tests/test_oracle.py): public keys from
the top-layer tree, signatures by xmss_core.c:183-273 with each layer's
subtree built once on all host cores (the same bytes as a treehash per
signature).  Output: mix_config4.json with each set's public keys and the
SHA-256 of all its signed messages concatenated in order, which bench.py
compares with the GPU's signatures.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def main() -> None:
    import bench
    from oracle import Oracle

    o = Oracle()
    cores = os.cpu_count() or 1
    draws = bench.mix_all_draws(lambda oid, mt: (o.params(oid, mt).n, o.params(oid, mt).full_height))
    out = []
    for (name, oid, mt), (seeds, start, cap, msgs) in zip(bench.MIX_SETS, draws):
        t0 = time.time()
        p = o.params(oid, mt)
        n, th, ib = p.n, p.tree_height, p.index_bytes
        seeds = [s.tobytes() for s in seeds]
        top = [o.tree_nodes(p, s[:n], s[2 * n:], p.d - 1, 0, cores) for s in seeds]
        pks = [t[-n:] + s[2 * n:] for t, s in zip(top, seeds)]
        trees = {}

        def tree_keys(i):
            idx = start + i % cap
            k = i // cap
            return idx, k, [(k, layer, idx >> (th * (layer + 1)) if th * (layer + 1) < 64 else 0)
                            for layer in range(p.d)]

        for i in range(len(msgs)):
            for key in tree_keys(i)[2]:
                if key not in trees:
                    k, layer, tree = key
                    s = seeds[k]
                    trees[key] = o.tree_nodes(p, s[:n], s[2 * n:], layer, tree, cores)

        def sign(i):
            idx, k, keys = tree_keys(i)
            s = seeds[k]
            sk = idx.to_bytes(ib, "big") + s[:2 * n] + pks[k][:n] + s[2 * n:]
            r, _, sm = o.sign(p, sk, msgs[i], trees=b"".join(trees[t] for t in keys))
            assert r == 0
            return sm

        with ThreadPoolExecutor(cores) as ex:  # ctypes calls release the GIL
            sms = list(ex.map(sign, range(len(msgs))))
        for i in range(0, len(sms), 97):
            assert o.sign_open(p, sms[i], pks[i // cap])[0] == 0
        out.append({"set": name, "oid": oid, "mt": mt, "first_index": start, "signatures": len(sms),
                    "subtrees": len(trees), "pks": [pk.hex() for pk in pks],
                    "sms_sha256": hashlib.sha256(b"".join(sms)).hexdigest()})
        print(f"{name}: {len(sms)} signatures, {len(trees)} subtrees in {time.time() - t0:.0f} s", flush=True)
    with open(os.path.join(HERE, "mix_config4.json"), "w") as f:
        json.dump({"workload": "bench.mix_all_draws()", "pk": "root || PUB_SEED (no OID prefix)",
                   "generator": "oracle (xo_tree_nodes + xo_sign_with_trees)", "sets": out}, f, indent=1)


if __name__ == "__main__":
    main()
