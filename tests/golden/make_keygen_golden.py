"""Golden public keys of the batched-keygen workload (8 x XMSS-SHA2_16_256 +
1 x XMSS-SHA2_20_256 from the seeded seeds of bench.keygen_seeds).

    make -C oracle ref && python tests/golden/make_keygen_golden.py

The h = 16 keys are computed by the reference's own C path compiled into
oracle/_ref (xmssmt_core_seed_keypair, cuxmss/xmss_core.c:134-161), one
process per key.  The h = 20 key (4.8 G SHA-256 compressions, about half an
hour for the single-threaded reference) is computed by the oracle's threaded
tree builder (oracle/xmss_oracle.c xo_tree_nodes), which tests/test_oracle.py
pins to the reference; its zero-seed counterpart is also pinned by the
reference's own h = 20 key headers (kat_h20.json).

Output: keygen_config3.json (committed), read by tests/test_gpu_configs.py
and by bench.py's keygen check.
"""
from __future__ import annotations

import json
import multiprocessing as mp
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)


def _ref_keypair(args):
    oid, seed = args
    from oracle import RefLib

    ref = RefLib()
    p = ref.params(oid, False)
    pk, _ = ref.seed_keypair(p, seed)
    return pk.hex()


def main() -> None:
    import bench
    from oracle import Oracle

    o = Oracle()
    keys = []
    for oid, seeds in bench.keygen_seeds():
        p = o.params(oid, False)
        t0 = time.time()
        if p.full_height <= 16:
            with mp.get_context("spawn").Pool(min(len(seeds), os.cpu_count() or 1)) as pool:
                pks = pool.map(_ref_keypair, [(oid, s.tobytes()) for s in seeds])
            gen = "reference C path (oracle/_ref xmssmt_core_seed_keypair)"
        else:
            pks = []
            for s in seeds:
                s = s.tobytes()
                nodes = o.tree_nodes(p, s[:p.n], s[2 * p.n:], 0, 0, os.cpu_count() or 1)
                pks.append((nodes[-p.n:] + s[2 * p.n:]).hex())
            gen = "oracle threaded tree (xo_tree_nodes)"
        for s, pk in zip(seeds, pks):
            keys.append({"oid": oid, "mt": False, "h": p.full_height, "seed": s.tobytes().hex(), "pk": pk,
                         "generator": gen})
        print(f"oid {oid:#x}: {len(seeds)} keys in {time.time() - t0:.0f} s", flush=True)
    doc = {"workload": "bench.keygen_seeds(): 8 x XMSS-SHA2_16_256 + 1 x XMSS-SHA2_20_256",
           "pk": "root || PUB_SEED (no OID prefix)", "keys": keys}
    with open(os.path.join(HERE, "keygen_config3.json"), "w") as f:
        json.dump(doc, f, indent=1)


if __name__ == "__main__":
    main()
